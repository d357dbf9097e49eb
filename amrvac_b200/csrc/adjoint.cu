// Discrete adjoint of the fused finite-volume stage: 2-D hydrodynamics, HLL or
// HLLC Riemann solver (src/mod_finite_volume.t:381-504), minmod or vanleer
// reconstruction (src/limiter/mod_limiter.t:173-209, reconstruct_LR
// 1110-1228), Einfeldt signal speeds (src/hd/mod_hd_phys.t:911-932), for a
// frozen time step.  There is no adjoint in the reference; this is the exact
// transpose of the forward stage kernel's arithmetic.
//
// Per face the forward values are replayed from the staged primitives with
// the forward's own device functions (so the limiter and upwind branches are
// the forward's), then the derivatives run backwards: HLL or HLLC (the
// forward's region, patchf) -> Einfeldt bounds
// -> physical fluxes -> primitive-to-conserved of the face states ->
// reconstruction -> the four stencil cells.  Ties of max/min follow the
// branch the forward value takes (vanleer's max(a*b, 0) takes the product
// branch when a*b >= 0; minmod's slope has a zero derivative unless the
// selected magnitude is > 0).
//
// CTA organisation: one 16x16 block per CTA, 320 threads.  Shared memory
// holds the primitives of the block with a 3-cell halo (the stencils of the
// faces -1..17 that touch the block's cells), lambda with a 2-cell halo (zero
// in physical ghost cells: ghosts are not state), and the per-face stencil
// gradients of one direction.  Faces whose stencil reaches into a neighbour
// block are computed by both blocks, so every cell gathers its four
// contributions per direction from shared memory in a fixed order: the
// result is deterministic (no atomics).  At a cont boundary the gradient of
// the ghost positions folds back onto the edge cell they copy.
#include "adjoint.cuh"

#include "kernels.cuh"

namespace amrvac {

namespace {

constexpr int ADJ_THREADS = 320;
#ifndef AMRVAC_ADJ_MINB
#define AMRVAC_ADJ_MINB 2
#endif
constexpr int WP = 22;            // primitive tile edge: 16 + 2*3
constexpr int LMW = 20;           // lambda tile edge: 16 + 2*2
constexpr int NF = 19;            // faces -1..17 per row and direction
constexpr int NFACE = NF * BN16;    // 304
constexpr int SM_WP = 4 * WP * WP;
constexpr int SM_LM = 4 * LMW * LMW;
constexpr int SM_G = 16 * NFACE;  // [slot][var][face]
constexpr size_t ADJ_SMEM = sizeof(double) * (SM_WP + SM_LM + SM_G);

// Partial derivatives of the limited slope (a: forward difference, b:
// backward difference), on the branch of the forward value.
template <int LIM>
__device__ __forceinline__ void slope_partials(double a, double b, double &da, double &db) {
  if constexpr (LIM == LIM_MINMOD) {
    const double t = copysign(1.0, a);
    const double tb = t * b, aa = fabs(a);
    da = 0.0;
    db = 0.0;
    if (tb < aa) {
      if (tb > 0.0) db = 1.0;  // slope = t*(t*b) = b
    } else if (aa > 0.0) {
      da = 1.0;  // slope = t*|a| = a
    }
  } else {  // vanleer: 2*max(b*a, 0) / (a + b + qsmall)
    if (b * a >= 0.0) {
      const double den = a + b + 1.0e-12, iden = rcp_(den);
      const double s = div_(2.0 * fmax(b * a, 0.0), den);
      da = (2.0 * b - s) * iden;
      db = (2.0 * a - s) * iden;
    } else {
      da = 0.0;
      db = 0.0;
    }
  }
}

// Reverse of the HLL flux (src/mod_finite_volume.t:381-437) for one face.
__device__ __forceinline__ void hll_reverse(const double *cL, const double *cR, const double *fL, const double *fR,
                                            double cmin, double cmax, const double *mu, double *fLb, double *fRb,
                                            double *cLb, double *cRb, double &cmaxb, double &cminb) {
  if (cmin >= 0.0) {
#pragma unroll
    for (int v = 0; v < 4; ++v) fLb[v] = mu[v];
    return;
  }
  if (cmax <= 0.0) {
#pragma unroll
    for (int v = 0; v < 4; ++v) fRb[v] = mu[v];
    return;
  }
  const double iD = rcp_(cmax - cmin);
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const double dW = cR[v] - cL[v];
    const double N = cmax * fL[v] - cmin * fR[v] + cmin * cmax * dW;
    const double F = N * iD;  // the forward's flux to rounding: it enters derivatives only
    fLb[v] = mu[v] * cmax * iD;
    fRb[v] = -mu[v] * cmin * iD;
    cRb[v] = mu[v] * cmin * cmax * iD;
    cLb[v] = -cRb[v];
    cmaxb += mu[v] * (fL[v] + cmin * dW - F) * iD;
    cminb += mu[v] * (-fR[v] + cmax * dW + F) * iD;
  }
}

// Reverse of the HD HLLC flux (get_Riemann_flux_hllc, src/mod_finite_volume.t:
// 439-504, with hd_get_lCD / hd_get_wCD, src/hd/mod_hd_hllc.t:56-257): the
// region (patchf) of the forward, then the star state of the upwind side.
// Rotated variables: 0 rho, 1 normal momentum, 2 tangential momentum, 3 e.
__device__ __forceinline__ void hllc_reverse(const double *cL, const double *cR, const double *fL, const double *fR,
                                             double cmin, double cmax, const double *mu, double *fLb, double *fRb,
                                             double *cLb, double *cRb, double &cmaxb, double &cminb) {
  if (cmin >= 0.0 || cmax <= 0.0) {
    hll_reverse(cL, cR, fL, fR, cmin, cmax, mu, fLb, fRb, cLb, cRb, cmaxb, cminb);
    return;
  }
  const double Dn = cmax - cmin, iDn = rcp_(Dn);
  double whll[2];
#pragma unroll
  for (int v = 0; v < 2; ++v) whll[v] = (cmax * cR[v] - cmin * cL[v] + fL[v] - fR[v]) * iDn;
  const double iwh0 = rcp_(whll[0]);
  double lam = whll[1] * iwh0;
  int patchf = 1;
  bool cond = true;
  if (cmin < 0.0 && lam > 0.0 && lam < cmax) patchf = -1;
  else if (cmax > 0.0 && lam < 0.0 && lam > cmin) patchf = 1;
  else if (lam >= cmax || lam <= cmin) { lam = 0.0; patchf = 3; cond = false; }
  if (cond && lam == 0.0) patchf = (-cmin >= cmax) ? 1 : -1;
  if (patchf == 3) {  // the HLL flux Fhll
    hll_reverse(cL, cR, fL, fR, cmin, cmax, mu, fLb, fRb, cLb, cRb, cmaxb, cminb);
    return;
  }
  const bool right = patchf == 1;
  const double *wS = right ? cR : cL, *fS = right ? fR : fL;
  double *wSb = right ? cRb : cLb, *fSb = right ? fRb : fLb;
  const double cs = right ? cmax : cmin;
  const double iw0 = rcp_(wS[0]);
  const double vS = wS[1] * iw0;
  const double csmls = rcp_(cs - lam);
  double wCD[4];
  wCD[0] = wS[0] * (cs - vS) * csmls;
  wCD[2] = (cs * wS[2] - fS[2]) * csmls;
  wCD[1] = wCD[0] * lam;
  const double pCD = wS[0] * (cs - vS) * (lam - vS) + fS[1] - wS[1] * vS;
  const double numE = cs * wS[3] - fS[3] + lam * pCD;
  wCD[3] = numE * csmls;
  // F = fS + cs (wCD - wS)
  double csb = 0.0, lamb = 0.0, csmlsb = 0.0, vSb = 0.0, wCDb[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    fSb[v] += mu[v];
    wCDb[v] = cs * mu[v];
    wSb[v] -= cs * mu[v];
    csb += mu[v] * (wCD[v] - wS[v]);
  }
  // wCD_e = (cs e - f_e + lam pCD) csmls
  {
    const double nb = wCDb[3] * csmls;
    csmlsb += wCDb[3] * numE;
    csb += nb * wS[3];
    wSb[3] += nb * cs;
    fSb[3] -= nb;
    lamb += nb * pCD;
    const double pb = nb * lam;
    // pCD = rho (cs - v)(lam - v) + f_mn - mn v
    wSb[0] += pb * (cs - vS) * (lam - vS);
    csb += pb * wS[0] * (lam - vS);
    lamb += pb * wS[0] * (cs - vS);
    vSb += pb * (-wS[0] * (lam - vS) - wS[0] * (cs - vS) - wS[1]);
    fSb[1] += pb;
    wSb[1] -= pb * vS;
  }
  // wCD_mn = wCD_rho lam
  wCDb[0] += wCDb[1] * lam;
  lamb += wCDb[1] * wCD[0];
  // wCD_mt = (cs mt - f_mt) csmls
  {
    const double nb = wCDb[2] * csmls;
    csmlsb += wCDb[2] * (cs * wS[2] - fS[2]);
    csb += nb * wS[2];
    wSb[2] += nb * cs;
    fSb[2] -= nb;
  }
  // wCD_rho = rho (cs - v) csmls
  wSb[0] += wCDb[0] * (cs - vS) * csmls;
  csb += wCDb[0] * wS[0] * csmls;
  vSb -= wCDb[0] * wS[0] * csmls;
  csmlsb += wCDb[0] * wS[0] * (cs - vS);
  // csmls = 1 / (cs - lam)
  {
    const double d = -csmlsb * csmls * csmls;
    csb += d;
    lamb -= d;
  }
  // vS = mn / rho
  wSb[1] += vSb * iw0;
  wSb[0] -= vSb * vS * iw0;
  // lam = whll_mn / whll_rho; whll_v = (cmax wR - cmin wL + fL - fR) / Dn
  double whllb[2];
  whllb[1] = lamb * iwh0;
  whllb[0] = -lamb * lam * iwh0;
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    const double b = whllb[v] * iDn;
    cRb[v] += b * cmax;
    cLb[v] -= b * cmin;
    fLb[v] += b;
    fRb[v] -= b;
    cmaxb += b * (cR[v] - whll[v]);
    cminb += b * (whll[v] - cL[v]);
  }
  if (right) cmaxb += csb;
  else cminb += csb;
}

// Vector-Jacobian product of one face flux.  wp: staged primitives; D: face
// direction; fi: face index along D (-1..17, face fi lies between cells fi-1
// and fi); row: the other coordinate; mu: dL/dF in rotated variable order
// (1 = normal, 2 = tangential velocity).  Adds dL/d(primitive) of the four
// stencil cells fi-2..fi+1 to gq (rotated order); returns dL/dgamma.
template <int LIM, int SOLVER>
__device__ __forceinline__ double face_vjp(const double *wp, int D, int fi, int row, const double *mu,
                                           const PhysParams &P, double (&gq)[4][4]) {
  auto at = [&](int o, int ov) -> double {
    const int pos = fi - 2 + o;
    const int x = D == 0 ? pos : row, y = D == 0 ? row : pos;
    return wp[ov * (WP * WP) + (y + 3) * WP + (x + 3)];
  };
  // ---- forward replay: reconstruction (reconstruct_LR), as in the stage kernel
  double L[4], R[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const int ov = orig_index_rt<false, 2>(v, D);
    const double q0 = at(0, ov), q1 = at(1, ov), q2 = at(2, ov), q3 = at(3, ov);
    const double d0 = q1 - q0, d1 = q2 - q1, d2 = q3 - q2;
    L[v] = q1 + 0.5 * limited_slope<double, true, LIM>(LIM, d1, d0, 0.0);
    R[v] = q2 - 0.5 * limited_slope<double, false, LIM>(LIM, d2, d1, 0.0);
  }
  const double g = P.gamma, ig = P.inv_gamma_1;
  // hd_to_conserved of the face states
  const double vL2 = L[1] * L[1] + L[2] * L[2], vR2 = R[1] * R[1] + R[2] * R[2];
  const double cL[4] = {L[0], L[0] * L[1], L[0] * L[2], L[3] * ig + 0.5 * vL2 * L[0]};
  const double cR[4] = {R[0], R[0] * R[1], R[0] * R[2], R[3] * ig + 0.5 * vR2 * R[0]};
  // hd_get_flux
  const double fL[4] = {L[1] * L[0], L[1] * cL[1] + L[3], L[1] * cL[2], L[1] * (cL[3] + L[3])};
  const double fR[4] = {R[1] * R[0], R[1] * cR[1] + R[3], R[1] * cR[2], R[1] * (cR[3] + R[3])};
  // Einfeldt bounds
  const double t1 = sqrt(L[0]), t2 = sqrt(R[0]), t3 = rcp_(t1 + t2);
  const double um = (L[1] * t1 + R[1] * t2) * t3, dv = R[1] - L[1];
  const double iL0 = rcp_(L[0]), iR0 = rcp_(R[0]);
  const double csL = g * L[3] * iL0, csR = g * R[3] * iR0;
  const double dm = sqrt((t1 * csL + t2 * csR) * t3 + 0.5 * t1 * t2 * (t3 * t3) * (dv * dv));
  const double cmin = um - dm, cmax = um + dm;
  // ---- reverse: Riemann solver
  double fLb[4] = {0.0, 0.0, 0.0, 0.0}, fRb[4] = {0.0, 0.0, 0.0, 0.0};
  double cLb[4] = {0.0, 0.0, 0.0, 0.0}, cRb[4] = {0.0, 0.0, 0.0, 0.0};
  double cmaxb = 0.0, cminb = 0.0;
  if constexpr (SOLVER == SOLVER_HLLC) hllc_reverse(cL, cR, fL, fR, cmin, cmax, mu, fLb, fRb, cLb, cRb, cmaxb, cminb);
  else hll_reverse(cL, cR, fL, fR, cmin, cmax, mu, fLb, fRb, cLb, cRb, cmaxb, cminb);
  double Lb[4] = {0.0, 0.0, 0.0, 0.0}, Rb[4] = {0.0, 0.0, 0.0, 0.0}, gb = 0.0;
  // Einfeldt reverse
  {
    const double umb = cmaxb + cminb, dmb = cmaxb - cminb;
    const double Xb = 0.5 * dmb * rcp_(dm);
    const double dv2 = dv * dv, t33 = t3 * t3;
    double t1b = Xb * (csL * t3 + 0.5 * t2 * t33 * dv2) + umb * L[1] * t3;
    double t2b = Xb * (csR * t3 + 0.5 * t1 * t33 * dv2) + umb * R[1] * t3;
    const double t3b = Xb * ((t1 * csL + t2 * csR) + t1 * t2 * t3 * dv2) + umb * (L[1] * t1 + R[1] * t2);
    const double csLb = Xb * t1 * t3, csRb = Xb * t2 * t3;
    const double dvb = Xb * t1 * t2 * t33 * dv;
    Lb[1] += umb * t1 * t3 - dvb;
    Rb[1] += umb * t2 * t3 + dvb;
    t1b -= t3b * t33;
    t2b -= t3b * t33;
    Lb[0] += 0.5 * t1b * rcp_(t1);
    Rb[0] += 0.5 * t2b * rcp_(t2);
    Lb[3] += csLb * g * iL0;
    Lb[0] -= csLb * csL * iL0;
    gb += csLb * L[3] * iL0;
    Rb[3] += csRb * g * iR0;
    Rb[0] -= csRb * csR * iR0;
    gb += csRb * R[3] * iR0;
  }
  // physical flux and to_conserved reverse, per side
  auto side = [&](const double *W, const double *c, const double *fb, const double *cb, double *Wb) {
    Wb[1] += fb[0] * W[0] + fb[1] * c[1] + fb[2] * c[2] + fb[3] * (c[3] + W[3]);
    Wb[0] += fb[0] * W[1] + cb[0];
    const double mnb = cb[1] + fb[1] * W[1];
    const double mtb = cb[2] + fb[2] * W[1];
    const double Eb = cb[3] + fb[3] * W[1];
    Wb[3] += fb[1] + fb[3] * W[1];
    Wb[0] += mnb * W[1] + mtb * W[2] + Eb * 0.5 * (W[1] * W[1] + W[2] * W[2]);
    Wb[1] += mnb * W[0] + Eb * W[0] * W[1];
    Wb[2] += mtb * W[0] + Eb * W[0] * W[2];
    Wb[3] += Eb * ig;
    gb -= Eb * W[3] * ig * ig;
  };
  side(L, cL, fLb, cLb, Lb);
  side(R, cR, fRb, cRb, Rb);
  // reconstruction reverse
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const int ov = orig_index_rt<false, 2>(v, D);
    const double q0 = at(0, ov), q1 = at(1, ov), q2 = at(2, ov), q3 = at(3, ov);
    const double d0 = q1 - q0, d1 = q2 - q1, d2 = q3 - q2;
    double dLa, dLb, dRa, dRb;
    slope_partials<LIM>(d1, d0, dLa, dLb);
    slope_partials<LIM>(d2, d1, dRa, dRb);
    const double sLb = 0.5 * Lb[v], sRb = -0.5 * Rb[v];
    const double d0b = sLb * dLb, d1b = sLb * dLa + sRb * dRb, d2b = sRb * dRa;
    gq[0][v] -= d0b;
    gq[1][v] += Lb[v] + d0b - d1b;
    gq[2][v] += Rb[v] + d1b - d2b;
    gq[3][v] += d2b;
  }
  return gb;
}

template <int LIM, int SOLVER>
__global__ void __launch_bounds__(ADJ_THREADS, AMRVAC_ADJ_MINB) adj_stage_kernel(const AdjArgs A) {
  extern __shared__ __align__(16) double adj_sm[];
  double *wp = adj_sm;
  double *lm = wp + SM_WP;
  double *G = lm + SM_LM;
  __shared__ double gred[ADJ_THREADS / 32];
  const int b = blockIdx.x;
  const int t = threadIdx.x;
  const StageArgs &S = A.sa;
  const PhysParams &P = S.P;
  const bool phys_lo[2] = {S.nbr[b * 27 + dir_index(-1, 0, 0)] < 0, S.nbr[b * 27 + dir_index(0, -1, 0)] < 0};
  const bool phys_hi[2] = {S.nbr[b * 27 + dir_index(1, 0, 0)] < 0, S.nbr[b * 27 + dir_index(0, 1, 0)] < 0};
  // ---- primitives with a 3-cell halo (no corners)
  for (int p = t; p < 22 * 16 + 6 * 16; p += ADJ_THREADS) {
    int x, y;
    if (p < 22 * 16) {
      y = p / 22;
      x = p - y * 22 - 3;
    } else {
      const int q = p - 22 * 16, r = q >> 4;
      y = r < 3 ? r - 3 : r + 13;
      x = q & (BN16 - 1);
    }
    double w[4];
    load_prim<false, 2, false, 2>(S, b, x, y, 0, w);
#pragma unroll
    for (int v = 0; v < 4; ++v) wp[v * (WP * WP) + (y + 3) * WP + (x + 3)] = w[v];
  }
  // ---- lambda with a 2-cell halo; zero at physical ghosts
  for (int p = t; p < 20 * 16 + 4 * 16; p += ADJ_THREADS) {
    int x, y;
    if (p < 20 * 16) {
      y = p / 20;
      x = p - y * 20 - 2;
    } else {
      const int q = p - 20 * 16, r = q >> 4;
      y = r < 2 ? r - 2 : r + 14;
      x = q & (BN16 - 1);
    }
    const bool phys = (x < 0 && phys_lo[0]) || (x >= BN16 && phys_hi[0]) || (y < 0 && phys_lo[1]) ||
                      (y >= BN16 && phys_hi[1]);
    double l[4] = {0.0, 0.0, 0.0, 0.0};
    if (!phys) {
      int i = x, j = y, k = 0;
      uint32_t flip;
      const int blk = resolve_cell<2>(S, b, i, j, k, flip);
#pragma unroll
      for (int v = 0; v < 4; ++v) l[v] = A.lam[cell_offset<2>(blk, 4, v, i, j, 0)];
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) lm[v * (LMW * LMW) + (y + 2) * LMW + (x + 2)] = l[v];
  }
  __syncthreads();
  double gp[4] = {0.0, 0.0, 0.0, 0.0};  // dL/d(primitive) of this thread's cell
  double gg = 0.0;                       // dL/dgamma, this thread's share
#pragma unroll 1
  for (int D = 0; D < 2; ++D) {
    if (t < NFACE) {
      const int row = t / NF, fi = t - row * NF - 1;
      const bool valid = !((fi == -1 && phys_lo[D]) || (fi == BN16 + 1 && phys_hi[D]));
      double gq[4][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
      if (valid) {
        double mu[4];
        const int xr = D == 0 ? fi : row, yr = D == 0 ? row : fi;
        const int xl = D == 0 ? fi - 1 : row, yl = D == 0 ? row : fi - 1;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const int ov = orig_index_rt<false, 2>(v, D);
          mu[v] = A.s[D] * (lm[ov * (LMW * LMW) + (yr + 2) * LMW + (xr + 2)] -
                            lm[ov * (LMW * LMW) + (yl + 2) * LMW + (xl + 2)]);
        }
        const double gface = face_vjp<LIM, SOLVER>(wp, D, fi, row, mu, P, gq);
        // faces next to a block edge are computed by two or three blocks: the
        // gamma term counts once, in the block of the cell right of the face
        // (and face 16 at a physical high side)
        if ((fi >= 0 && fi < BN16) || (fi == BN16 && phys_hi[D])) gg += gface;
      }
#pragma unroll
      for (int o = 0; o < 4; ++o)
#pragma unroll
        for (int v = 0; v < 4; ++v) G[(o * 4 + orig_index_rt<false, 2>(v, D)) * NFACE + t] = gq[o][v];
    }
    __syncthreads();
    if (t < BN16 * BN16) {
      const int ci = t & (BN16 - 1), cj = t >> 4;
      const int c = D == 0 ? ci : cj, row = D == 0 ? cj : ci;
      const int base = row * NF;  // face f is entry base + f + 1
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const double *g0 = G + (0 * 4 + v) * NFACE, *g1 = G + (1 * 4 + v) * NFACE;
        const double *g2 = G + (2 * 4 + v) * NFACE, *g3 = G + (3 * 4 + v) * NFACE;
        // faces c+2, c+1, c, c-1 hold this cell in stencil slots 0, 1, 2, 3
        double sum = g0[base + c + 3] + g1[base + c + 2] + g2[base + c + 1] + g3[base + c];
        if (c == 0 && phys_lo[D])       // ghosts -2, -1 copy cell 0
          sum += g0[base + 1] + g1[base + 1] + g0[base + 2];
        if (c == BN16 - 1 && phys_hi[D])  // ghosts 16, 17 copy cell 15
          sum += g2[base + BN16 + 1] + g3[base + BN16 + 1] + g3[base + BN16];
        gp[v] += sum;
      }
    }
    __syncthreads();
  }
  if (t < BN16 * BN16) {
    const int ci = t & (BN16 - 1), cj = t >> 4;
    double w[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) w[v] = S.uin[cell_offset<2>(b, 4, v, ci, cj, 0)];
    // hd_to_primitive reverse: v = m / rho, p = (gamma-1)(e - rho v^2 / 2)
    const double rho = w[0], ir = rcp_(rho), v1 = w[1] * ir, v2 = w[2] * ir;
    const double vv = v1 * v1 + v2 * v2, g1 = P.gamma_1, pb = gp[3];
    const double v1b = gp[1] - pb * g1 * rho * v1, v2b = gp[2] - pb * g1 * rho * v2;
    double lc[4];
    lc[0] = gp[0] - pb * g1 * 0.5 * vv - (v1b * v1 + v2b * v2) * ir;
    lc[1] = v1b * ir;
    lc[2] = v2b * ir;
    lc[3] = pb * g1;
    gg += pb * (w[3] - 0.5 * rho * vv);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const size_t o = cell_offset<2>(b, 4, v, ci, cj, 0);
      const double ln = lm[v * (LMW * LMW) + (cj + 2) * LMW + (ci + 2)];
      const double acc = A.acc_in ? A.acc_in[o] : 0.0;
      A.lam_out[o] = acc + A.b * ln + lc[v];
      if (A.base) A.base[o] = (A.base_init ? 0.0 : A.base[o]) + A.a * ln;
    }
  }
  // dL/dgamma of this block: fixed-order reduction
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) gg += __shfl_xor_sync(0xffffffffu, gg, o);
  if ((t & 31) == 0) gred[t >> 5] = gg;
  __syncthreads();
  if (t == 0) {
    double sum = 0.0;
    for (int q = 0; q < ADJ_THREADS / 32; ++q) sum += gred[q];
    A.gamma_part[b] += sum;
  }
}

}  // namespace

template <int LIM, int SOLVER>
static cudaError_t prep_one() {
  return cudaFuncSetAttribute(adj_stage_kernel<LIM, SOLVER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)ADJ_SMEM);
}

cudaError_t adjoint_prepare() {
  cudaError_t e = prep_one<LIM_MINMOD, SOLVER_HLL>();
  if (e == cudaSuccess) e = prep_one<LIM_VANLEER, SOLVER_HLL>();
  if (e == cudaSuccess) e = prep_one<LIM_MINMOD, SOLVER_HLLC>();
  if (e == cudaSuccess) e = prep_one<LIM_VANLEER, SOLVER_HLLC>();
  return e;
}

cudaError_t launch_adjoint_stage(const AdjArgs &A, int limiter, int solver, cudaStream_t s) {
  const int nb = A.sa.nblocks;
  if (solver == SOLVER_HLL) {
    if (limiter == LIM_MINMOD) adj_stage_kernel<LIM_MINMOD, SOLVER_HLL><<<nb, ADJ_THREADS, ADJ_SMEM, s>>>(A);
    else if (limiter == LIM_VANLEER) adj_stage_kernel<LIM_VANLEER, SOLVER_HLL><<<nb, ADJ_THREADS, ADJ_SMEM, s>>>(A);
    else return cudaErrorInvalidValue;
  } else if (solver == SOLVER_HLLC) {
    if (limiter == LIM_MINMOD) adj_stage_kernel<LIM_MINMOD, SOLVER_HLLC><<<nb, ADJ_THREADS, ADJ_SMEM, s>>>(A);
    else if (limiter == LIM_VANLEER) adj_stage_kernel<LIM_VANLEER, SOLVER_HLLC><<<nb, ADJ_THREADS, ADJ_SMEM, s>>>(A);
    else return cudaErrorInvalidValue;
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

__global__ void set_scalar_kernel(double *p, double v) { *p = v; }

cudaError_t launch_set_scalar(double *p, double v, cudaStream_t s) {
  set_scalar_kernel<<<1, 1, 0, s>>>(p, v);
  return cudaGetLastError();
}

}  // namespace amrvac
