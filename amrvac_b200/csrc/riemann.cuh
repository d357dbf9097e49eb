// Approximate Riemann solvers for one face (FP64).
//
// Restates get_Riemann_flux_{tvdlf,hll,hllc,hlld} (src/mod_finite_volume.t:348-729)
// and the HD HLLC helpers hd_get_lCD / hd_get_wCD (src/hd/mod_hd_hllc.t:56-257)
// for a single interface, with the reference's flux_type rules
// (src/mhd/mod_mhd_phys.t:566-589): with GLM the normal B and psi fluxes are
// "special" (taken from the left flux); without GLM the normal B uses the
// diffusive tvdlf form.
#pragma once

#include "physics.cuh"

namespace amrvac {

template <bool MHD, int NDIM, bool GLM>
struct FluxTypes {
  static constexpr bool bn_special = MHD && NDIM > 1 && GLM;
  static constexpr bool bn_tvdlf = MHD && NDIM > 1 && !GLM;
};

// get_Riemann_flux_tvdlf (mod_finite_volume.t:348-379)
template <class T, int NW>
__device__ __forceinline__ void riemann_tvdlf(const T *wLC, const T *wRC, const T *fL,
                                              const T *fR, T cmax, T tvdlfeps,
                                              T *F) {
  const T fac = -(T(0.5) * tvdlfeps * cmax);
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    T f = T(0.5) * (fL[v] + fR[v]);
    F[v] = f + fac * (wRC[v] - wLC[v]);
  }
}

// get_Riemann_flux_hll (mod_finite_volume.t:381-437)
template <class T, bool MHD, int NDIR, bool GLM, int NDIM, int D, bool FAST = false>
__device__ __forceinline__ void riemann_hll(const T *wLC, const T *wRC, const T *fL,
                                            const T *fR, T cmax, T cmin,
                                            T tvdlfeps, T *F) {
  using V = Vars<MHD, NDIR, GLM>;
  using FT = FluxTypes<MHD, NDIM, GLM>;
  const T rden = rcp_f<FAST>(cmax - cmin);  // one reciprocal for every variable
#pragma unroll
  for (int v = 0; v < V::NW; ++v) {
    if (FT::bn_tvdlf && v == V::B0 + D) {
      F[v] = -(tvdlfeps * T(0.5) * fmax(cmax, fabs(cmin))) * (wRC[v] - wLC[v]);
    } else if (cmin >= T(0.0)) {
      F[v] = fL[v];
    } else if (cmax <= T(0.0)) {
      F[v] = fR[v];
    } else {
      F[v] = (cmax * fL[v] - cmin * fR[v] + cmin * cmax * (wRC[v] - wLC[v])) * rden;
    }
  }
}

// get_Riemann_flux_hllc (mod_finite_volume.t:439-504) + hd_get_lCD / hd_get_wCD
// (mod_hd_hllc.t:56-257); HD only, no hllcd diffusion, flathllc=.false.
template <class T, int NDIR, int D, bool FAST = false>
__device__ __forceinline__ void riemann_hllc_hd(const T *wLC, const T *wRC, const T *fL,
                                                const T *fR, T cmax, T cmin,
                                                T *F) {
  using V = Vars<false, NDIR, false>;
  constexpr int NW = V::NW, MN = V::M0 + D;
  int patchf = 1;
  if (cmin >= T(0.0)) patchf = -2;
  else if (cmax <= T(0.0)) patchf = 2;
  if (patchf == -2) {
#pragma unroll
    for (int v = 0; v < NW; ++v) F[v] = fL[v];
    return;
  }
  if (patchf == 2) {
#pragma unroll
    for (int v = 0; v < NW; ++v) F[v] = fR[v];
    return;
  }
  T whll[NW], Fhll[NW];
  const T rden = rcp_f<FAST>(cmax - cmin);  // one reciprocal for every variable
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    Fhll[v] = (cmax * fL[v] - cmin * fR[v] + cmin * cmax * (wRC[v] - wLC[v])) * rden;
    whll[v] = (cmax * wRC[v] - cmin * wLC[v] + fL[v] - fR[v]) * rden;
  }
  T lambdaCD = div_f<FAST>(whll[MN], whll[V::RHO]);
  bool cond = true;
  if (cmin < T(0.0) && lambdaCD > T(0.0) && lambdaCD < cmax) {
    patchf = -1;
  } else if (cmax > T(0.0) && lambdaCD < T(0.0) && lambdaCD > cmin) {
    patchf = 1;
  } else if (lambdaCD >= cmax || lambdaCD <= cmin) {
    lambdaCD = T(0.0);
    patchf = 3;
    cond = false;
  }
  if (cond && lambdaCD == T(0.0)) patchf = (-cmin >= cmax) ? 1 : -1;
  if (patchf == 3) {
#pragma unroll
    for (int v = 0; v < NW; ++v) F[v] = Fhll[v];
    return;
  }
  const bool right = (patchf == 1);
  const T *wSub = right ? wRC : wLC;
  const T *fSub = right ? fR : fL;
  const T cspeed = right ? cmax : cmin;
  const T vSub = div_f<FAST>(wSub[MN], wSub[V::RHO]);
  const T csmls = rcp_f<FAST>(cspeed - lambdaCD);
  T wCD[NW];
  wCD[V::RHO] = wSub[V::RHO] * (cspeed - vSub) * csmls;
#pragma unroll
  for (int c = 0; c < NDIR; ++c) {
    if (c != D) wCD[V::M0 + c] = (cspeed * wSub[V::M0 + c] - fSub[V::M0 + c]) * csmls;
    else wCD[V::M0 + c] = wCD[V::RHO] * lambdaCD;
  }
  const T pCD = wSub[V::RHO] * (cspeed - vSub) * (lambdaCD - vSub) + fSub[MN] - wSub[MN] * vSub;
  wCD[V::E] = (cspeed * wSub[V::E] - fSub[V::E] + lambdaCD * pCD) * csmls;
#pragma unroll
  for (int v = 0; v < NW; ++v) F[v] = fSub[v] + cspeed * (wCD[v] - wSub[v]);
}

// get_Riemann_flux_hllc (mod_finite_volume.t:439-504) + mhd_get_lCD /
// mhd_get_wCD (src/mhd/mod_mhd_hllc.t:56-241), no hllcd diffusion,
// flathllc=.false.  The star state keeps the HLL magnetic field; its flux
// has zero normal-B (and psi) entries, which the flux_type rules then
// replace by the diffusive tvdlf form without GLM, and keep with GLM (the
// reference's HLLC takes no flux_special branch).
template <class T, int NDIR, bool GLM, int NDIM, int D, bool FAST = false>
__device__ __forceinline__ void riemann_hllc_mhd(const T *wLC, const T *wRC, const T *fL, const T *fR, T cmax,
                                                 T cmin, T tvdlfeps, T *F) {
  using V = Vars<true, NDIR, GLM>;
  using FT = FluxTypes<true, NDIM, GLM>;
  constexpr int NW = V::NW, MN = V::M0 + D, BNI = V::B0 + D;
  int patchf = 1;
  if (cmin >= T(0.0)) patchf = -2;
  else if (cmax <= T(0.0)) patchf = 2;
  T whll[NW], Fhll[NW], fCD[NW];
  T lambdaCD = T(0.0);
  if (patchf == 1) {
    const T rden = rcp_f<FAST>(cmax - cmin);  // one reciprocal for every variable
#pragma unroll
    for (int v = 0; v < NW; ++v) {
      Fhll[v] = (cmax * fL[v] - cmin * fR[v] + cmin * cmax * (wRC[v] - wLC[v])) * rden;
      whll[v] = (cmax * wRC[v] - cmin * wLC[v] + fL[v] - fR[v]) * rden;
    }
    lambdaCD = div_f<FAST>(whll[MN], whll[V::RHO]);
    bool cond = true;
    if (cmin < T(0.0) && lambdaCD > T(0.0) && lambdaCD < cmax) {
      patchf = -1;
    } else if (cmax > T(0.0) && lambdaCD < T(0.0) && lambdaCD > cmin) {
      patchf = 1;
    } else if (lambdaCD >= cmax || lambdaCD <= cmin) {
      lambdaCD = T(0.0);
      patchf = 3;
      cond = false;
    }
    if (cond && lambdaCD == T(0.0)) patchf = (-cmin >= cmax) ? 1 : -1;
  }
  if (patchf == 1 || patchf == -1) {
    const bool right = (patchf == 1);
    const T *wSub = right ? wRC : wLC;
    const T *fSub = right ? fR : fL;
    const T cspeed = right ? cmax : cmin;
    const T vSub = div_f<FAST>(wSub[MN], wSub[V::RHO]);
    const T rden = rcp_f<FAST>(cspeed - lambdaCD);  // one reciprocal for the star state
    T wCD[NW];
    wCD[V::RHO] = wSub[V::RHO] * (cspeed - vSub) * rden;
#pragma unroll
    for (int c = 0; c < NDIR; ++c) wCD[V::B0 + c] = whll[V::B0 + c];
#pragma unroll
    for (int c = 0; c < NDIR; ++c) {
      if (c != D) wCD[V::M0 + c] = (cspeed * wSub[V::M0 + c] - fSub[V::M0 + c] - wCD[BNI] * wCD[V::B0 + c]) * rden;
      else wCD[V::M0 + c] = wCD[V::RHO] * lambdaCD;
    }
    // V.B of the HLL state (summed in the order the components arrive)
    T vdb = whll[V::M0] * whll[V::B0];
#pragma unroll
    for (int c = 1; c < NDIR; ++c) vdb = vdb + whll[V::M0 + c] * whll[V::B0 + c];
    vdb = div_f<FAST>(vdb, whll[V::RHO]);
    const T pCD = wSub[V::RHO] * (cspeed - vSub) * (lambdaCD - vSub) + fSub[MN] - wSub[MN] * vSub +
                  wCD[BNI] * wCD[BNI];
    wCD[V::E] = (cspeed * wSub[V::E] - fSub[V::E] + lambdaCD * pCD - vdb * wCD[BNI]) * rden;
#pragma unroll
    for (int v = 0; v < NW; ++v) {
      if (v == BNI || (GLM && v == V::PSI)) fCD[v] = T(0.0);
      else fCD[v] = fSub[v] + cspeed * (wCD[v] - wSub[v]);
    }
  }
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    if (FT::bn_tvdlf && v == BNI) {
      F[v] = -(tvdlfeps * T(0.5) * fmax(cmax, fabs(cmin))) * (wRC[v] - wLC[v]);
    } else if (patchf == -2) {
      F[v] = fL[v];
    } else if (patchf == 2) {
      F[v] = fR[v];
    } else if (patchf == 3) {
      F[v] = Fhll[v];
    } else {
      F[v] = fCD[v];
    }
  }
}

// TVD-MUSCL (fs_tvdmu) for hydrodynamics: the central flux of
// get_Riemann_flux_tvdmu (src/mod_finite_volume.t:342-346) with the
// characteristic limiter tvdlimit2 (src/mod_tvd.t:38-112) folded into the
// face flux — the Roe average hd_average, the wave speeds and jumps of
// geteigenjump2 and the right eigenvectors of rtimes2
// (src/hd/mod_hd_roe.t:58-296), entropy fix 'nul', getphi's tvdmu branch
// phi = |a qdt/dx| jump.  tvdlimit2 adds 0.5 R phi to the scaled flux
// -qdt/dx F; here F - 0.5 sum R |a| jump is returned for the same scaling.
// Rotated states: the face normal is component 0, the shear waves follow in
// the tangential components' order.
template <class T, int NDIR>
__device__ __forceinline__ void riemann_tvdmu_hd(const T *wLC, const T *wRC, const T *fL, const T *fR,
                                                 const PhysParams &P, T *F) {
  using V = Vars<false, NDIR, false>;
  constexpr int NW = V::NW;
#pragma unroll
  for (int v = 0; v < NW; ++v) F[v] = T(0.5) * (fL[v] + fR[v]);
  // hd_average
  const T qL = sqrt(wLC[V::RHO]), qR = sqrt(wRC[V::RHO]);
  const T rho = qL * qR;
  const T r = qL / qR;
  T vel[NDIR];
#pragma unroll
  for (int c = 0; c < NDIR; ++c)
    vel[c] = (wLC[V::M0 + c] / wLC[V::RHO] * r + wRC[V::M0 + c] / wRC[V::RHO]) / (T(1.0) + r);
  auto pth = [&](const T *w) {  // hd_get_pthermal
    T m2 = w[V::M0] * w[V::M0];
#pragma unroll
    for (int c = 1; c < NDIR; ++c) m2 = m2 + w[V::M0 + c] * w[V::M0 + c];
    T p = T(P.gamma - 1.0) * (w[V::E] - T(0.5) * m2 / w[V::RHO]);
    if (P.fix_small_values && p < T(P.small_pressure)) p = T(P.small_pressure);
    return p;
  };
  const T pL = pth(wLC), pR = pth(wRC);
  const T hL = (pL + wLC[V::E]) / wLC[V::RHO];
  const T hR = (pR + wRC[V::E]) / wRC[V::RHO];
  const T H = (hL * r + hR) / (T(1.0) + r);
  // geteigenjump2, il = 1 part
  T v2 = vel[0] * vel[0];
#pragma unroll
  for (int c = 1; c < NDIR; ++c) v2 = v2 + vel[c] * vel[c];
  const T kin = T(0.5) * v2;
  T c2 = T(P.gamma - 1.0) * (H - kin);
  c2 = fmax(T(P.gamma) * T(1.0e-12) / rho, c2);  // smalldouble
  const T dpperc2 = (pR - pL) / c2;
  const T cs = sqrt(c2);
  const T dvperc = (wRC[V::M0] / wRC[V::RHO] - wLC[V::M0] / wLC[V::RHO]) / cs;
  const T u = vel[0];
  // sound waves (right, left) and the entropy wave: R columns
  const T aR = fabs(u + cs) * (T(0.5) * (dpperc2 + rho * dvperc));
  const T aL = fabs(u - cs) * (T(0.5) * (dpperc2 - rho * dvperc));
  const T aE = fabs(u) * ((-dpperc2 + wRC[V::RHO]) - wLC[V::RHO]);
  F[V::RHO] = F[V::RHO] - (T(0.5) * aR + T(0.5) * aL + T(0.5) * aE);
  F[V::E] = F[V::E] - (T(0.5) * (aR * (H + u * cs)) + T(0.5) * (aL * (H - u * cs)) + T(0.5) * (aE * kin));
  F[V::M0] = F[V::M0] - (T(0.5) * (aR * (u + cs)) + T(0.5) * (aL * (u - cs)) + T(0.5) * (aE * u));
#pragma unroll
  for (int c = 1; c < NDIR; ++c) {
    // shear wave of component c: a = u, jump = rho (vR_c - vL_c)
    const T aS = fabs(u) * (rho * (wRC[V::M0 + c] / wRC[V::RHO] - wLC[V::M0 + c] / wLC[V::RHO]));
    F[V::E] = F[V::E] - T(0.5) * (aS * vel[c]);
    F[V::M0 + c] = F[V::M0 + c] - (T(0.5) * (aR * vel[c]) + T(0.5) * (aL * vel[c]) + T(0.5) * (aE * vel[c]) +
                                   T(0.5) * aS);
  }
}

// TVD-MUSCL for MHD (no GLM): the central flux with tvdlimit2's
// characteristic limiter folded in, the Roe system of src/mhd/mod_mhd_roe.t
// (average2 61-146 with arithmetic averages, geteigenjump2 160-342,
// rtimes2 355-506; divbwave on, typeentropy 'nul').  The waves are taken in
// the reference's order il = 1..nwflux: Alfven R/L, fast R/L, slow R/L, then
// (ndir 3 only: nwflux = 8) the divB and entropy waves — with ndir 2
// (nwflux = 6) the limiter loop never reaches those two.  Rotated states:
// idim = component 0, idir = 1, jdir = 2 (ndir 3) or 0 (ndir 2, where the
// reference's jdir = idir + 1 - ndir (idir / ndir) wraps to idim).
template <class T, int NDIR>
__device__ __forceinline__ void riemann_tvdmu_mhd(const T *wLC, const T *wRC, const T *fL, const T *fR,
                                                  const PhysParams &P, T *F) {
  using V = Vars<true, NDIR, false>;
  constexpr int NW = V::NW, RHO = V::RHO, E = V::E, M = V::M0, B = V::B0;
  constexpr int ID = 1, JD = NDIR == 3 ? 2 : 0;
  constexpr T smalld = T(1.0e-12);
#pragma unroll
  for (int v = 0; v < NW; ++v) F[v] = T(0.5) * (fL[v] + fR[v]);
  const T g = T(P.gamma);
  auto pth = [&](const T *w) {  // mhd_get_pthermal_origin
    T m2 = w[M] * w[M], b2 = w[B] * w[B];
#pragma unroll
    for (int c = 1; c < NDIR; ++c) { m2 = m2 + w[M + c] * w[M + c]; b2 = b2 + w[B + c] * w[B + c]; }
    T p = T(P.gamma - 1.0) * (w[E] - T(0.5) * (m2 / w[RHO] + b2));
    if (P.fix_small_values && p < T(P.small_pressure)) p = T(P.small_pressure);
    return p;
  };
  // average2
  T rho = T(0.5) * (wLC[RHO] + wRC[RHO]);
  T v[NDIR], b[NDIR], dv[NDIR], db[NDIR];
#pragma unroll
  for (int c = 0; c < NDIR; ++c) {
    v[c] = T(0.5) * (wLC[M + c] / wLC[RHO] + wRC[M + c] / wRC[RHO]);
    b[c] = T(0.5) * (wLC[B + c] + wRC[B + c]);
    dv[c] = wRC[M + c] / wRC[RHO] - wLC[M + c] / wLC[RHO];
    db[c] = wRC[B + c] - wLC[B + c];
  }
  const T pL = pth(wLC), pR = pth(wRC);
  const T pav = T(0.5) * (pL + pR);
  const T dp = pR - pL;
  const T rhodv = wRC[M] - wLC[M] - v[0] * (wRC[RHO] - wLC[RHO]);
  const T cs2 = g * pav / rho;
  T bb = b[0] * b[0];
#pragma unroll
  for (int c = 1; c < NDIR; ++c) bb = bb + b[c] * b[c];
  T cf = bb / rho + cs2;
  T cl = T(0.5) * (cf - sqrt(cf * cf - T(4.0) * cs2 * (b[0] * b[0]) / rho));
  cf = cf - cl;
  T af = (cs2 - cl) / (cf - cl);
  af = fmin(T(1.0), fmax(af, T(0.0)));
  const T as = sqrt(T(1.0) - af);
  af = sqrt(af);
  cf = sqrt(cf);
  cl = sqrt(cl);
  rho = sqrt(rho);
  if (fabs(b[0]) < smalld) b[0] = smalld;
  if constexpr (NDIR == 2) {
    b[ID] = b[ID] >= T(0.0) ? T(1.0) : T(-1.0);
  } else {
    const T tmp = sqrt(b[1] * b[1] + b[2] * b[2]);
    if (tmp > smalld) { b[1] = b[1] / tmp; b[2] = b[2] / tmp; }
    else { b[1] = sqrt(T(0.5)); b[2] = sqrt(T(0.5)); }
  }
  const T u = v[0];
  const T sgn = copysign(T(1.0), b[0]);
  const T sqcs2 = sqrt(cs2);
  T v2 = v[0] * v[0];
#pragma unroll
  for (int c = 1; c < NDIR; ++c) v2 = v2 + v[c] * v[c];
  const T v2a2 = T(0.5) * v2 + (T(2.0) - g) / (g - T(1.0)) * cs2;
  // Alfven waves
  const T bdvA = ((b[JD] * dv[ID] - b[ID] * dv[JD]) * T(0.5)) * (rho * rho);
  const T bdbA = ((b[JD] * db[ID] - b[ID] * db[JD]) * T(0.5)) * copysign(rho, b[0]);
  const T bvA = b[JD] * v[ID] - b[ID] * v[JD];
  // fast and slow waves
  T bdvF = b[ID] * dv[ID], bdbF = b[ID] * db[ID], bvF = b[ID] * v[ID];
  if constexpr (NDIR == 3) {
    bdvF = bdvF + b[JD] * dv[JD];
    bdbF = bdbF + b[JD] * db[JD];
    bvF = bvF + b[JD] * v[JD];
  }
  bdvF = bdvF * copysign(rho * rho, b[0]);
  bdbF = (bdbF * sqcs2) * rho;
  bvF = bvF * sgn;
  const T h = T(0.5) / cs2;
  T D[NW];
#pragma unroll
  for (int w = 0; w < NW; ++w) D[w] = T(0.0);
  // il = alfvR, alfvL, fastR, fastL, slowR, slowL (then divB, entropy for ndir 3)
#pragma unroll
  for (int il = 0; il < (NDIR == 3 ? 8 : 6); ++il) {
    T a, jump;
    switch (il) {
      case 0: a = u + fabs(b[0]) / rho; jump = bdvA - bdbA; break;
      case 1: a = u - fabs(b[0]) / rho; jump = -bdvA - bdbA; break;
      case 2: a = u + cf; jump = h * (af * (cf * rhodv + dp) + as * (-cl * bdvF + bdbF)); break;
      case 3: a = u - cf; jump = h * (af * (-cf * rhodv + dp) + as * (cl * bdvF + bdbF)); break;
      case 4: a = u + cl; jump = h * (as * (cl * rhodv + dp) + af * (cf * bdvF - bdbF)); break;
      case 5: a = u - cl; jump = h * (as * (-cl * rhodv + dp) + af * (-cf * bdvF - bdbF)); break;
      case 6: a = u; jump = db[0]; break;
      default: a = u; jump = (wRC[RHO] - wLC[RHO]) - dp / cs2; break;
    }
    const T q = fabs(a) * jump;
    const bool fast = il == 2 || il == 3, slow = il == 4 || il == 5, alf = il < 2;
    const T pm = (il == 2 || il == 4) ? T(1.0) : T(-1.0);  // R / L of fast and slow
    // rtimes2 rows
    T r_rho, r_e, r_mn, r_bn;
    if (fast) {
      r_rho = q * af;
      r_e = q * (-pm * as * cl * bvF + af * (v2a2 + cf * (cf + pm * u)));
      r_mn = (q * af) * (u + pm * cf);
    } else if (slow) {
      r_rho = q * as;
      r_e = q * (pm * af * cf * bvF + as * (v2a2 + cl * (cl + pm * u)));
      r_mn = (q * as) * (u + pm * cl);
    } else if (alf) {
      r_rho = T(0.0);
      r_e = il == 0 ? q * bvA : -q * bvA;
      r_mn = T(0.0);
    } else if (il == 6) {
      r_rho = T(0.0);
      r_e = q * b[0];
      r_mn = T(0.0);
    } else {
      r_rho = q;
      r_e = q * T(0.5) * v2;
      r_mn = q * u;
    }
    r_bn = il == 6 ? q : T(0.0);
    D[RHO] = D[RHO] + T(0.5) * r_rho;
    D[E] = D[E] + T(0.5) * r_e;
    D[M] = D[M] + T(0.5) * r_mn;
    D[B] = D[B] + T(0.5) * r_bn;
#pragma unroll
    for (int t = 1; t < NDIR; ++t) {
      T r_m, r_b;
      if (fast) {
        r_m = q * (af * v[t] - pm * as * cl * b[t] * sgn);
        r_b = ((q * as) * sqcs2) * b[t] / rho;
      } else if (slow) {
        r_m = q * (as * v[t] + pm * af * cf * b[t] * sgn);
        r_b = -((q * af) * sqcs2) * b[t] / rho;
      } else if (alf) {
        const T s = il == 0 ? T(1.0) : T(-1.0);
        r_m = t == ID ? s * q * b[JD] : -s * q * b[ID];
        r_b = t == ID ? -q * b[JD] / copysign(rho, b[0]) : q * b[ID] / copysign(rho, b[0]);
      } else if (il == 6) {
        r_m = T(0.0);
        r_b = T(0.0);
      } else {
        r_m = q * v[t];
        r_b = T(0.0);
      }
      D[M + t] = D[M + t] + T(0.5) * r_m;
      D[B + t] = D[B + t] + T(0.5) * r_b;
    }
  }
#pragma unroll
  for (int w = 0; w < NW; ++w) F[w] = F[w] - D[w];
}

// get_Riemann_flux_hlld (mod_finite_volume.t:507-729), no B0 / equilibrium split.
template <class T, int NDIR, bool GLM, int NDIM, int D, bool FAST = false>
__device__ __forceinline__ void riemann_hlld(const T *wLC, const T *wRC, const T *wLp,
                                             const T *wRp, const T *fL, const T *fR,
                                             T sR, T sL, T *F) {
  using V = Vars<true, NDIR, GLM>;
  using FT = FluxTypes<true, NDIM, GLM>;
  constexpr int NW = V::NW, RHO = V::RHO, E = V::E, M0 = V::M0, B0 = V::B0;
  constexpr int ip1 = D, ip2 = (D + 1) % NDIR, ip3 = (D + 2) % NDIR;
  constexpr int m1 = M0 + ip1, m2 = M0 + ip2, m3 = M0 + ip3;
  constexpr int b1 = B0 + ip1, b2 = B0 + ip2, b3 = B0 + ip3;
  const T Bx = div_f<FAST>(sR * wRC[b1] - sL * wLC[b1], sR - sL);
  T bR2 = wRC[B0] * wRC[B0], bL2 = wLC[B0] * wLC[B0];
#pragma unroll
  for (int c = 1; c < NDIR; ++c) {
    bR2 = bR2 + wRC[B0 + c] * wRC[B0 + c];
    bL2 = bL2 + wLC[B0 + c] * wLC[B0 + c];
  }
  const T ptR = wRp[E] + T(0.5) * bR2;
  const T ptL = wLp[E] + T(0.5) * bL2;
  const T vR = wRp[m1], vL = wLp[m1];
  const T suR = (sR - vR) * wRC[RHO];
  const T suL = (sL - vL) * wLC[RHO];
  const T sm = div_f<FAST>(suR * vR - suL * vL - ptR + ptL, suR - suL);
  // star states w1 (velocities in the momentum slots until the final conversion)
  T w1R[NW], w1L[NW], w2R[NW], w2L[NW];
  w1R[m1] = sm; w1L[m1] = sm; w2R[m1] = sm; w2L[m1] = sm;
  w1R[b1] = Bx; w1L[b1] = Bx;
  // one reciprocal of s - s_M per side serves the star density and energy
  const T isR = rcp_f<FAST>(sR - sm), isL = rcp_f<FAST>(sL - sm);
  w1R[RHO] = suR * isR;
  w1L[RHO] = suL * isL;
  T r1R = suR * (sR - sm) - Bx * Bx;
  if (r1R != T(0.0)) r1R = rcp_f<FAST>(r1R);
  T r1L = suL * (sL - sm) - Bx * Bx;
  if (r1L != T(0.0)) r1L = rcp_f<FAST>(r1L);
  w1R[m2] = wRp[m2] - Bx * wRC[b2] * (sm - vR) * r1R;
  w1L[m2] = wLp[m2] - Bx * wLC[b2] * (sm - vL) * r1L;
  T pb2R = (suR * (sR - vR) - Bx * Bx) * r1R;
  T pb2L = (suL * (sL - vL) - Bx * Bx) * r1L;
  if constexpr (NDIR == 3) {
    w1R[m3] = wRp[m3] - Bx * wRC[b3] * (sm - vR) * r1R;
    w1L[m3] = wLp[m3] - Bx * wLC[b3] * (sm - vL) * r1L;
    w1R[b3] = wRC[b3] * pb2R;
    w1L[b3] = wLC[b3] * pb2L;
  }
  w1R[b2] = wRC[b2] * pb2R;
  w1L[b2] = wLC[b2] * pb2L;
  const T pts = suR * (sm - vR) + ptR;  // w1R(p_) = w1L(p_)
  {
    T vbR = wRp[M0] * wRC[B0], vbL = wLp[M0] * wLC[B0];
    T v1bR = w1R[M0] * w1R[B0], v1bL = w1L[M0] * w1L[B0];
#pragma unroll
    for (int c = 1; c < NDIR; ++c) {
      vbR = vbR + wRp[M0 + c] * wRC[B0 + c];
      vbL = vbL + wLp[M0 + c] * wLC[B0 + c];
      v1bR = v1bR + w1R[M0 + c] * w1R[B0 + c];
      v1bL = v1bL + w1L[M0 + c] * w1L[B0 + c];
    }
    w1R[E] = ((sR - vR) * wRC[E] - ptR * vR + pts * sm + Bx * (vbR - v1bR)) * isR;
    w1L[E] = ((sL - vL) * wLC[E] - ptL * vL + pts * sm + Bx * (vbL - v1bL)) * isL;
  }
  w2R[RHO] = w1R[RHO]; w2L[RHO] = w1L[RHO];
  w2R[b1] = Bx; w2L[b1] = Bx;
  const T sqR = sqrt_f<FAST>(w1R[RHO]);
  const T sqL = sqrt_f<FAST>(w1L[RHO]);
  const T tmp = rcp_f<FAST>(sqR + sqL);
  const T signBx = copysign(T(1.0), Bx);
  const T s1R = sm + div_f<FAST>(fabs(Bx), sqR);
  const T s1L = sm - div_f<FAST>(fabs(Bx), sqL);
  w2R[m2] = (sqL * w1L[m2] + sqR * w1R[m2] + (w1R[b2] - w1L[b2]) * signBx) * tmp;
  w2L[m2] = w2R[m2];
  w2R[b2] = (sqL * w1R[b2] + sqR * w1L[b2] + sqL * sqR * (w1R[m2] - w1L[m2]) * signBx) * tmp;
  w2L[b2] = w2R[b2];
  if constexpr (NDIR == 3) {
    w2R[m3] = (sqL * w1L[m3] + sqR * w1R[m3] + (w1R[b3] - w1L[b3]) * signBx) * tmp;
    w2L[m3] = w2R[m3];
    w2R[b3] = (sqL * w1R[b3] + sqR * w1L[b3] + sqL * sqR * (w1R[m3] - w1L[m3]) * signBx) * tmp;
    w2L[b3] = w2R[b3];
  }
  {
    T a1R = w1R[M0] * w1R[B0], a2R = w2R[M0] * w2R[B0];
    T a1L = w1L[M0] * w1L[B0], a2L = w2L[M0] * w2L[B0];
#pragma unroll
    for (int c = 1; c < NDIR; ++c) {
      a1R = a1R + w1R[M0 + c] * w1R[B0 + c];
      a2R = a2R + w2R[M0 + c] * w2R[B0 + c];
      a1L = a1L + w1L[M0 + c] * w1L[B0 + c];
      a2L = a2L + w2L[M0 + c] * w2L[B0 + c];
    }
    w2R[E] = w1R[E] + sqR * (a1R - a2R) * signBx;
    w2L[E] = w1L[E] - sqL * (a1L - a2L) * signBx;
  }
#pragma unroll
  for (int c = 0; c < NDIR; ++c) {
    w1R[M0 + c] = w1R[M0 + c] * w1R[RHO];
    w1L[M0 + c] = w1L[M0 + c] * w1L[RHO];
    w2R[M0 + c] = w2R[M0 + c] * w2R[RHO];
    w2L[M0 + c] = w2L[M0 + c] * w2L[RHO];
  }
  if constexpr (GLM) {
    // psi star values are never used (flux_special); keep them defined.
    w1R[V::PSI] = w1L[V::PSI] = w2R[V::PSI] = w2L[V::PSI] = T(0.0);
  }
  // region selection (Miyoshi eq. 66), branch-free: the candidate fluxes of
  // the chosen side are formed for every variable and the region picks one
  int region;
  if (sL > T(0.0)) region = 0;
  else if (s1L >= T(0.0)) region = 1;
  else if (sm >= T(0.0)) region = 2;
  else if (s1R >= T(0.0)) region = 3;
  else if (sR >= T(0.0)) region = 4;
  else region = 5;  // sR < 0 (a NaN speed also lands here)
  const bool left = region <= 2;
  const bool one_star = region == 1 || region == 4;
  const bool two_star = region == 2 || region == 3;
  const T c1 = left ? sL : sR;
  const T c2 = left ? s1L : s1R;
#pragma unroll
  for (int v = 0; v < NW; ++v) {
    if (FT::bn_special && (v == b1 || v == V::PSI)) {
      F[v] = fL[v];
      continue;
    }
    const T fs = left ? fL[v] : fR[v];
    const T ws = left ? wLC[v] : wRC[v];
    const T w1 = left ? w1L[v] : w1R[v];
    const T w2 = left ? w2L[v] : w2R[v];
    const T t1 = fs + c1 * (w1 - ws);
    const T t2 = t1 + c2 * (w2 - w1);
    F[v] = two_star ? t2 : (one_star ? t1 : fs);
  }
}

}  // namespace amrvac
