// Device physics for the finite-volume face update (HD and ideal MHD).
//
// Each routine restates one reference routine for a single face or cell; the
// expression order follows the reference so that the FP64 path agrees with it
// to rounding (the only reordering is FMA contraction by the compiler).
// Reference files (relative to the MPI-AMRVAC repository root):
//   hd:   src/hd/mod_hd_phys.t, src/hd/mod_hd_hllc.t
//   mhd:  src/mhd/mod_mhd_phys.t
//   fv:   src/mod_finite_volume.t, src/limiter/mod_limiter.t
#pragma once

#include <cstdint>

namespace amrvac {

// Limiter ids as in src/limiter/mod_limiter.t:14-24.
enum : int { LIM_MINMOD = 1, LIM_WOODWARD = 2, LIM_MCBETA = 3, LIM_SUPERBEE = 4,
             LIM_VANLEER = 5, LIM_ALBADA = 6, LIM_KOREN = 7, LIM_CADA = 8, LIM_CADA3 = 9,
             LIM_SCHMID = 10, LIM_VENK = 11, LIM_MP5 = 13, LIM_WENO3 = 14, LIM_WENOYC3 = 15, LIM_WENO5 = 16,
             LIM_WENOZ5 = 18, LIM_WENOZP5 = 20 };
enum : int { BS_EINFELDT = 1, BS_CMAXMEAN = 2, BS_CMAXLEFTRIGHT = 3 };
enum : int { SOLVER_TVDLF = 1, SOLVER_HLL = 2, SOLVER_HLLC = 3, SOLVER_HLLD = 4, SOLVER_TVDMU = 5,
             SOLVER_HANCOCK = 8 };
enum : int { DIVB_NONE = 0, DIVB_GLM = 1, DIVB_LINDE = 4 };
// Runtime status bits (atomicOr into the context's status word).
enum : uint32_t { ST_SMALL_VALUE = 1u, ST_NAN = 2u, ST_DT_TOO_SMALL = 4u, ST_BOUNDS = 8u };

// Physics constants shared by all kernels of one context.
struct PhysParams {
  double gamma, gamma_1, inv_gamma_1;
  double small_density, small_pressure, small_e;
  double tvdlfeps, cada3_radius, glm_alpha, divbdiff, courantpar;
  double schmid_rad[3];
  int limiter, boundspeed, divb, glm_extended, schmid_global;
  int fix_small_values, check_small_values, small_values_method;
};

// Variable layout in the reference order: rho, m(1:ndir), e, [b(1:ndir), psi].
template <bool MHD, int NDIR, bool GLM>
struct Vars {
  static constexpr int RHO = 0;
  static constexpr int M0 = 1;
  static constexpr int E = NDIR + 1;
  static constexpr int B0 = NDIR + 2;
  static constexpr int PSI = 2 * NDIR + 2;
  static constexpr int NW = MHD ? (2 * NDIR + 2 + (GLM ? 1 : 0)) : (NDIR + 2);
};

__device__ __forceinline__ double fsign(double a, double b) { return copysign(a, b); }
__device__ __forceinline__ float fsign(float a, float b) { return copysignf(a, b); }
// single-precision division / reciprocal of the mixed form: IEEE (correctly rounded)
__device__ __forceinline__ float rcp_(float y) { return 1.0f / y; }
__device__ __forceinline__ float div_(float x, float y) { return x / y; }

#ifndef AMRVAC_IEEE_DIV
#define AMRVAC_NR_DIV 1
#endif
#ifdef AMRVAC_NR_DIV
// Reciprocal and quotient by Newton-Raphson iteration from a single-precision
// seed (Markstein, "IA-64 and Elementary Functions", 2000, ch. 8): each step
// r <- r + r(1 - y r) squares the relative error (2^-23 -> 2^-46 -> 2^-92); the
// quotient gets one residual correction q <- q + r(x - y q).  Branch-free;
// valid for |y| within the single-precision normal range (the path's
// denominators are densities, wave speeds and limiter slopes >= 2^-26).
__device__ __forceinline__ double rcp_(double y) {
  double r = (double)__frcp_rn(__double2float_rn(y));
  double e = fma(-y, r, 1.0);
  r = fma(r, e, r);
  e = fma(-y, r, 1.0);
  return fma(r, e, r);
}
__device__ __forceinline__ double div_(double x, double y) {
  const double r = rcp_(y);
  const double q = x * r;
  return fma(fma(-y, q, x), r, q);
}
#else
__device__ __forceinline__ double rcp_(double y) { return 1.0 / y; }
__device__ __forceinline__ double div_(double x, double y) { return x / y; }
#endif

// ------------------------------------------------------------------ conversions
// hd_to_primitive (mod_hd_phys.t:703-734) / mhd_to_primitive_origin (mod_mhd_phys.t:1741-1765)
template <bool MHD, int NDIR, bool GLM>
__device__ __forceinline__ void to_primitive(double *w, const PhysParams &P) {
  using V = Vars<MHD, NDIR, GLM>;
  const double inv_rho = rcp_(w[V::RHO]);
#pragma unroll
  for (int c = 0; c < NDIR; ++c) w[V::M0 + c] = w[V::M0 + c] * inv_rho;
  double v2 = w[V::M0] * w[V::M0];
#pragma unroll
  for (int c = 1; c < NDIR; ++c) v2 = v2 + w[V::M0 + c] * w[V::M0 + c];
  if constexpr (MHD) {
    double b2 = w[V::B0] * w[V::B0];
#pragma unroll
    for (int c = 1; c < NDIR; ++c) b2 = b2 + w[V::B0 + c] * w[V::B0 + c];
    w[V::E] = P.gamma_1 * (w[V::E] - 0.5 * (w[V::RHO] * v2 + b2));
  } else {
    w[V::E] = P.gamma_1 * (w[V::E] - 0.5 * w[V::RHO] * v2);
  }
}

// hd_to_conserved (mod_hd_phys.t:677-700) / mhd_to_conserved_origin (mod_mhd_phys.t:1562-1579)
template <class T, bool MHD, int NDIR, bool GLM>
__device__ __forceinline__ void to_conserved(T *w, const PhysParams &P) {
  using V = Vars<MHD, NDIR, GLM>;
  T v2 = w[V::M0] * w[V::M0];
#pragma unroll
  for (int c = 1; c < NDIR; ++c) v2 = v2 + w[V::M0 + c] * w[V::M0 + c];
  if constexpr (MHD) {
    T b2 = w[V::B0] * w[V::B0];
#pragma unroll
    for (int c = 1; c < NDIR; ++c) b2 = b2 + w[V::B0 + c] * w[V::B0 + c];
    w[V::E] = w[V::E] * T(P.inv_gamma_1) + T(0.5) * (v2 * w[V::RHO] + b2);
  } else {
    w[V::E] = w[V::E] * T(P.inv_gamma_1) + T(0.5) * v2 * w[V::RHO];
  }
#pragma unroll
  for (int c = 0; c < NDIR; ++c) w[V::M0 + c] = w[V::RHO] * w[V::M0 + c];
}

// Small-value check and "replace" fix on one state (hd_check_w mod_hd_phys.t:648-674,
// mhd_check_w_origin mod_mhd_phys.t:1452-1473, replace branches mod_hd_phys.t:1436-1466
// and mod_mhd_phys.t:2208-2222).  Returns true if the state was flagged.
template <class T, bool MHD, int NDIR, bool GLM>
__device__ __forceinline__ bool small_values(T *w, bool primitive, const PhysParams &P) {
  using V = Vars<MHD, NDIR, GLM>;
  const bool frho = w[V::RHO] < T(P.small_density);
  T m2 = w[V::M0] * w[V::M0];
#pragma unroll
  for (int c = 1; c < NDIR; ++c) m2 = m2 + w[V::M0 + c] * w[V::M0 + c];
  T b2 = T(0.0);
  if constexpr (MHD) {
    b2 = w[V::B0] * w[V::B0];
#pragma unroll
    for (int c = 1; c < NDIR; ++c) b2 = b2 + w[V::B0 + c] * w[V::B0 + c];
  }
  bool fe;
  if (primitive) fe = w[V::E] < T(P.small_pressure);
  else if (MHD) fe = w[V::E] - T(0.5) * (m2 / w[V::RHO] + b2) < T(P.small_e);
  else fe = T(P.gamma_1) * (w[V::E] - T(0.5) * m2 / w[V::RHO]) < T(P.small_pressure);
  if (!(frho || fe)) return false;
  if (P.small_values_method == 1) {
    if (frho) {
      w[V::RHO] = T(P.small_density);
#pragma unroll
      for (int c = 0; c < NDIR; ++c) w[V::M0 + c] = T(0.0);
    }
    if ((!MHD && frho) || fe) {
      if (primitive) {
        w[V::E] = T(P.small_pressure);
      } else {
        T mm = w[V::M0] * w[V::M0];
#pragma unroll
        for (int c = 1; c < NDIR; ++c) mm = mm + w[V::M0 + c] * w[V::M0 + c];
        w[V::E] = MHD ? T(P.small_e) + T(0.5) * (mm / w[V::RHO] + b2) : T(P.small_e) + T(0.5) * mm / w[V::RHO];
      }
    }
  }
  return true;
}

// ------------------------------------------------------------------ fluxes
// hd_get_flux (mod_hd_phys.t:1097-1146) / mhd_get_flux (mod_mhd_phys.t:3810-3889).
// wc: conserved, w: primitive state at the face; D: face normal (0-based).
template <class T, bool MHD, int NDIR, bool GLM, int D>
__device__ __forceinline__ void phys_flux(const T *wc, const T *w, T cg,
                                          T *f) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int MN = V::M0 + D;
  if constexpr (!MHD) {
    f[V::RHO] = w[MN] * w[V::RHO];
#pragma unroll
    for (int c = 0; c < NDIR; ++c) f[V::M0 + c] = w[MN] * wc[V::M0 + c];
    f[MN] = f[MN] + w[V::E];
    f[V::E] = w[MN] * (wc[V::E] + w[V::E]);
  } else {
    constexpr int BN = V::B0 + D;
    f[V::RHO] = w[MN] * w[V::RHO];
#pragma unroll
    for (int c = 0; c < NDIR; ++c) f[V::M0 + c] = wc[MN] * w[V::M0 + c] - w[BN] * w[V::B0 + c];
    T b2 = w[V::B0] * w[V::B0];
#pragma unroll
    for (int c = 1; c < NDIR; ++c) b2 = b2 + w[V::B0 + c] * w[V::B0 + c];
    const T ptotal = w[V::E] + T(0.5) * b2;
    f[MN] = f[MN] + ptotal;
    T bv = w[V::B0] * w[V::M0];
#pragma unroll
    for (int c = 1; c < NDIR; ++c) bv = bv + w[V::B0 + c] * w[V::M0 + c];
    f[V::E] = w[MN] * (wc[V::E] + ptotal) - w[BN] * bv;
#pragma unroll
    for (int c = 0; c < NDIR; ++c) f[V::B0 + c] = w[MN] * w[V::B0 + c] - w[BN] * w[V::M0 + c];
    if constexpr (GLM) {
      f[BN] = w[V::PSI];
      f[V::PSI] = (cg * cg) * w[BN];
    }
  }
}

// mhd_get_csound_prim (mod_mhd_phys.t:3329-3379): fast magnetosonic speed.
template <class T, int NDIR, int BN>
__device__ __forceinline__ T fast_speed(const T *w, const PhysParams &P) {
  constexpr int RHO = 0, E = NDIR + 1, B0 = NDIR + 2;
  const T inv_rho = rcp_(w[RHO]);
  const T cs = T(P.gamma) * w[E] * inv_rho;
  T b2 = w[B0] * w[B0];
#pragma unroll
  for (int c = 1; c < NDIR; ++c) b2 = b2 + w[B0 + c] * w[B0 + c];
  const T cfast2 = b2 * inv_rho + cs;
  T av = cfast2 * cfast2 - T(4.0) * cs * (w[BN] * w[BN]) * inv_rho;
  if (av < T(0.0)) av = T(0.0);
  return sqrt(T(0.5) * (cfast2 + sqrt(av)));
}

// hd_get_cbounds (mod_hd_phys.t:891-1001) / mhd_get_cbounds (mod_mhd_phys.t:3037-3127).
// WITH_MIN=false gives the tvdlf form (cmax only).  Returns a status bit.
template <class T, bool MHD, int NDIR, bool GLM, int D, bool WITH_MIN, int BS = 0>
__device__ __forceinline__ uint32_t cbounds(const T *wLC, const T *wRC, const T *wLp,
                                            const T *wRp, const PhysParams &P, T &cmax,
                                            T &cmin) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int MN = V::M0 + D;
  uint32_t st = 0;
  const int bsel = BS ? BS : P.boundspeed;
  if (bsel == BS_EINFELDT) {
    const T tmp1 = sqrt(wLp[V::RHO]);
    const T tmp2 = sqrt(wRp[V::RHO]);
    const T tmp3 = rcp_(tmp1 + tmp2);
    const T umean = (wLp[MN] * tmp1 + wRp[MN] * tmp2) * tmp3;
    const T dv = wRp[MN] - wLp[MN];
    T dmean;
    if constexpr (MHD) {
      const T csL = fast_speed<T, NDIR, V::B0 + D>(wLp, P);
      const T csR = fast_speed<T, NDIR, V::B0 + D>(wRp, P);
      dmean = sqrt((tmp1 * (csL * csL) + tmp2 * (csR * csR)) * tmp3 +
                   T(0.5) * tmp1 * tmp2 * (tmp3 * tmp3) * (dv * dv));
    } else {
      const T csL = T(P.gamma) * wLp[V::E] / wLp[V::RHO];
      const T csR = T(P.gamma) * wRp[V::E] / wRp[V::RHO];
      dmean = sqrt((tmp1 * csL + tmp2 * csR) * tmp3 + T(0.5) * tmp1 * tmp2 * (tmp3 * tmp3) * (dv * dv));
    }
    if (WITH_MIN) {
      cmin = umean - dmean;
      cmax = umean + dmean;
    } else {
      cmax = fabs(umean) + dmean;
    }
  } else if (bsel == BS_CMAXMEAN) {
    if constexpr (MHD) {
      T wm[V::NW];
#pragma unroll
      for (int v = 0; v < V::NW; ++v) wm[v] = T(0.5) * (wLp[v] + wRp[v]);
      const T cs = fast_speed<T, NDIR, V::B0 + D>(wm, P);
      if (WITH_MIN) {
        cmax = fmax(wm[MN] + cs, T(0.0));
        cmin = fmin(wm[MN] - cs, T(0.0));
      } else {
        cmax = fabs(wm[MN]) + cs;
      }
    } else {
      T wm[V::NW];
#pragma unroll
      for (int v = 0; v < V::NW; ++v) wm[v] = T(0.5) * (wLC[v] + wRC[v]);
      const T tmp1 = wm[MN] / wm[V::RHO];
      T m2 = wm[V::M0] * wm[V::M0];
#pragma unroll
      for (int c = 1; c < NDIR; ++c) m2 = m2 + wm[V::M0 + c] * wm[V::M0 + c];
      T pth = T(P.gamma_1) * (wm[V::E] - T(0.5) * m2 / wm[V::RHO]);
      if (P.fix_small_values) {
        if (pth < T(P.small_pressure)) pth = T(P.small_pressure);
      } else if (P.check_small_values) {
        if (pth < T(P.small_pressure)) st |= ST_SMALL_VALUE;
      }
      const T cs = sqrt(P.gamma * pth / wm[V::RHO]);
      if (WITH_MIN) {
        cmax = fmax(tmp1 + cs, T(0.0));
        cmin = fmin(tmp1 - cs, T(0.0));
      } else {
        cmax = fabs(tmp1) + cs;
      }
    }
  } else {  // cmaxleftright
    T cs;
    if constexpr (MHD) {
      cs = fmax(fast_speed<T, NDIR, V::B0 + D>(wLp, P), fast_speed<T, NDIR, V::B0 + D>(wRp, P));
    } else {
      const T csL = T(P.gamma) * wLp[V::E] / wLp[V::RHO];
      const T csR = T(P.gamma) * wRp[V::E] / wRp[V::RHO];
      cs = fmax(sqrt(csL), sqrt(csR));
    }
    if (WITH_MIN) cmin = fmin(wLp[MN], wRp[MN]) - cs;
    cmax = fmax(wLp[MN], wRp[MN]) + cs;
  }
  return st;
}

// ------------------------------------------------------------------ limiters
// dwlimiter2 (mod_limiter.t:128-334) for one cell: a = dwC(ix) (forward
// difference), b = dwC(ix-1) (backward difference).  LEFT selects ldw, else rdw.
template <class T, bool LEFT>
__device__ __forceinline__ T slope_impl(int lim, T a, T b, T rdelinv) {
  constexpr T qsmall = T(1.0e-12), qsmall2 = T(2.0e-12);
  constexpr T eps = T(1.4901161193847656e-08);  // sqrt(epsilon(1d0)) = 2**-26
  constexpr T c_mcbeta = T(1.4), cadalfa = T(0.5), cadbeta = T(2.0), cadgamma = T(1.6);
  constexpr T cadepsilon = T(1.0e-14), invcadepsilon = T(1.0e14);
  constexpr T third = T(1.0) / T(3.0);
  switch (lim) {
    case LIM_MINMOD: {
      const T t = fsign(T(1.0), a);
      return t * fmax(T(0.0), fmin(fabs(a), t * b));
    }
    case LIM_VANLEER:
      return div_(T(2.0) * fmax(b * a, T(0.0)), a + b + qsmall);
    case LIM_CADA3: {
      // branch-free: both the asymptotic and the limited form are evaluated
      // and the reference's three-way choice is made with selects
      const T tmpeta = (a * a + b * b) * rdelinv;
      const T t = LEFT ? div_(b, a + fsign(eps, a)) : div_(a, b + fsign(eps, b));
      const T A = (T(2.0) + t) * third;
      const T lim2 = fmax(T(0.0), fmin(A, fmax(-(cadalfa * t), fmin(fmin(cadbeta * t, A), cadgamma))));
      const T t2 = (tmpeta - T(1.0)) * invcadepsilon;
      const T blend = T(0.5) * ((T(1.0) - t2) * A + (T(1.0) + t2) * lim2);
      const T phi = tmpeta <= T(1.0) - cadepsilon ? A : (tmpeta >= T(1.0) + cadepsilon ? lim2 : blend);
      return phi * (LEFT ? a : b);
    }
    case LIM_SCHMID: {
      // dwlimiter2 limiter_schmid (src/limiter/mod_limiter.t:291-333), the
      // schmid2 form: rdelinv carries (a2max + cadepsilon) dx^2 here
      const T tmpeta = sqrt(T(0.4) * (a * a + b * b)) / rdelinv;
      const T t = LEFT ? div_(b, a + fsign(eps, a)) : div_(a, b + fsign(eps, b));
      const T A = (T(2.0) + t) * third;
      const T lim2 = fmax(T(0.0), fmin(A, fmax(-t, fmin(fmin(cadbeta * t, A), T(1.5)))));
      const T t2 = (tmpeta - T(1.0)) * invcadepsilon;
      const T blend = T(0.5) * ((T(1.0) - t2) * A + (T(1.0) + t2) * lim2);
      const T phi = tmpeta <= T(1.0) - cadepsilon ? A : (tmpeta >= T(1.0) + cadepsilon ? lim2 : blend);
      return phi * (LEFT ? a : b);
    }
    case LIM_WOODWARD: {
      const T t = fsign(T(1.0), a);
      return T(2.0) * t * fmax(T(0.0), fmin(fmin(fabs(a), t * b), t * T(0.25) * (b + a)));
    }
    case LIM_MCBETA: {
      const T t = fsign(T(1.0), a);
      return t * fmax(T(0.0), fmin(fmin(c_mcbeta * fabs(a), c_mcbeta * t * b), t * T(0.5) * (b + a)));
    }
    case LIM_SUPERBEE: {
      const T t = fsign(T(1.0), a);
      return t * fmax(fmax(T(0.0), fmin(T(2.0) * fabs(a), t * b)), fmin(fabs(a), T(2.0) * t * b));
    }
    case LIM_ALBADA:
      return (b * (a * a + qsmall) + a * (b * b + qsmall)) / (a * a + b * b + qsmall2);
    case LIM_KOREN: {
      const T t = fsign(T(1.0), a);
      const T t2 = fmin(T(2.0) * fabs(a), T(2.0) * t * b);
      if (LEFT) return t * fmax(T(0.0), fmin(t2, (b * t + T(2.0) * fabs(a)) * third));
      return t * fmax(T(0.0), fmin(t2, (T(2.0) * b * t + fabs(a)) * third));
    }
    default: {  // cada
      const T t = LEFT ? b / (a + fsign(eps, a)) : a / (b + fsign(eps, b));
      const T t2 = (T(2.0) + t) * third;
      return fmax(T(0.0), fmin(t2, fmax(-(cadalfa * t), fmin(fmin(cadbeta * t, t2), cadgamma)))) *
             (LEFT ? a : b);
    }
  }
}

// LIM != 0 fixes the limiter at compile time (the switch folds away);
// LIM == 0 selects it at run time from lim_rt.
template <class T, bool LEFT, int LIM>
__device__ __forceinline__ T limited_slope(int lim_rt, T a, T b, T rdelinv) {
  return slope_impl<T, LEFT>(LIM ? LIM : lim_rt, a, b, rdelinv);
}

// Index in the reference variable order of entry v of a state whose vector
// components are cyclically rotated so that direction D comes first
// (rotated component c holds original component (c + D) mod ndir).
template <bool MHD, int NDIR, int D>
__host__ __device__ constexpr int orig_index(int v) {
  return (v >= 1 && v <= NDIR) ? 1 + (v - 1 + D) % NDIR
         : (MHD && v >= NDIR + 2 && v <= 2 * NDIR + 1) ? NDIR + 2 + (v - NDIR - 2 + D) % NDIR
                                                         : v;
}

}  // namespace amrvac
