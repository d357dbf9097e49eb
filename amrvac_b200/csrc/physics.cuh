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
enum : uint32_t { ST_SMALL_VALUE = 1u, ST_NAN = 2u, ST_DT_TOO_SMALL = 4u, ST_BOUNDS = 8u, ST_TIMEOUT = 16u };
// Per-block only (block_status): small_values_method 'average' needs the
// block's whole-block recomputation (smallavg.cu).
enum : uint32_t { ST_SV_AVG = 32u };

// Physics constants shared by all kernels of one context.
struct PhysParams {
  double gamma, gamma_1, inv_gamma_1;
  double small_density, small_pressure, small_e;
  double tvdlfeps, cada3_radius, glm_alpha, divbdiff, courantpar;
  double schmid_rad[3];
  int limiter, boundspeed, divb, glm_extended, schmid_global;
  int fix_small_values, check_small_values, small_values_method;
  int small_values_daverage;  // 'average': largest cube half-width
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
// Correctly rounded IEEE division, out of line: the cold path of rcp_/div_.
static __device__ __noinline__ double div_ieee(double x, double y) { return x / y; }
// The hardware's approximate double-precision reciprocal (PTX
// rcp.approx.ftz.f64): the seed of the Newton-Raphson reciprocal below.
__device__ __forceinline__ double rcp_seed(double y) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(y));
  return r;
}
#ifdef AMRVAC_NR_DIV
// Reciprocal and quotient by Newton-Raphson iteration (Markstein, "IA-64 and
// Elementary Functions", 2000, ch. 8) from the hardware's approximate
// double-precision reciprocal (PTX rcp.approx.ftz.f64, about 20 correct bits
// over the whole double exponent range).  Each step r <- r + r(1 - y r)
// squares the relative error (2^-20 -> 2^-40 -> 2^-80); the quotient takes
// one step and then the residual correction q <- q + r(x - y q), which
// leaves an error of order 2^-80 before the final rounding.
// Guard (integer operations on the high word): y zero, subnormal, infinite,
// NaN or with |y| >= 2^1021 (1/y at or near the subnormal range), and a
// quotient that came out non-finite, take the correctly rounded division
// instead, so that every input gives IEEE's special values.
__device__ __forceinline__ bool nr_range(double y) {
  const unsigned e = ((unsigned)__double2hiint(y) >> 20) & 0x7ffu;  // biased exponent
  return e - 1u < 2043u;  // 2^-1022 <= |y| < 2^1021
}
__device__ __forceinline__ bool finite_hi(double q) {
  return ((unsigned)__double2hiint(q) & 0x7ff00000u) != 0x7ff00000u;
}
__device__ __forceinline__ double rcp_(double y) {
  double r = rcp_seed(y);
  r = fma(r, fma(-y, r, 1.0), r);
  r = fma(r, fma(-y, r, 1.0), r);
  if (!nr_range(y)) r = div_ieee(1.0, y);
  return r;
}
__device__ __forceinline__ double div_(double x, double y) {
  double r = rcp_seed(y);
  r = fma(r, fma(-y, r, 1.0), r);
  const double q0 = x * r;
  double q = fma(fma(-y, q0, x), r, q0);
  if (!(nr_range(y) && finite_hi(q))) q = div_ieee(x, y);
  return q;
}
#else
__device__ __forceinline__ double rcp_(double y) { return 1.0 / y; }
__device__ __forceinline__ double div_(double x, double y) { return x / y; }
#endif

// Unguarded forms for the hot face loop of the FP64 stage kernel, which
// checks every face's flux and recomputes a face whose flux is not finite
// with the guarded forms (rcp_, div_, IEEE sqrt).  On finite normal
// operands in range they give the guarded forms' results; a zero,
// subnormal, infinite or NaN denominator gives NaN (IEEE: +-inf or NaN),
// which reaches the flux and sends the face to the recomputation.
#ifdef AMRVAC_NR_DIV
__device__ __forceinline__ double rcp_nr(double y) {
  double r = rcp_seed(y);
  r = fma(r, fma(-y, r, 1.0), r);
  return fma(r, fma(-y, r, 1.0), r);
}
__device__ __forceinline__ double div_nr(double x, double y) {
  double r = rcp_seed(y);
  r = fma(r, fma(-y, r, 1.0), r);
  const double q0 = x * r;
  return fma(fma(-y, q0, x), r, q0);
}
#else
__device__ __forceinline__ double rcp_nr(double y) { return 1.0 / y; }
__device__ __forceinline__ double div_nr(double x, double y) { return x / y; }
#endif
// Square root by the coupled Newton iteration for sqrt(x) and 1/(2 sqrt(x))
// (Markstein, ch. 8; Goldschmidt's form) from the hardware's approximate
// reciprocal square root (PTX rsqrt.approx.ftz.f64): one coupled step takes
// the seed's ~2^-20 to ~2^-40, the residual correction s + (x - s^2) h to the
// order of 2^-80 before the final rounding.  The seed is capped at 2^511 so
// that x = 0 gives 0 (the seed of 0 is infinite); a negative x gives NaN.
__device__ __forceinline__ double sqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  y = fmin(y, 0x1.0p511);
  double s = x * y, h = 0.5 * y;
  const double r = fma(-s, h, 0.5);
  s = fma(s, r, s);
  h = fma(h, r, h);
  return fma(fma(-s, s, x), h, s);
}
template <bool FAST> __device__ __forceinline__ double rcp_f(double y) {
  if constexpr (FAST) return rcp_nr(y); else return rcp_(y);
}
template <bool FAST> __device__ __forceinline__ double div_f(double x, double y) {
  if constexpr (FAST) return div_nr(x, y); else return div_(x, y);
}
template <bool FAST> __device__ __forceinline__ double sqrt_f(double x) {
  if constexpr (FAST) return sqrt_nr(x); else return sqrt(x);
}
// Single precision (the mixed form's faces): IEEE, or with FAST the hardware
// approximations of PTX (rcp.approx.ftz.f32, sqrt.approx.ftz.f32, about one
// unit in the last place of FP32; the quotient x * (1/y) adds a rounding).
// The mixed form's faces are accurate to FP32 rounding either way; a face
// whose flux is not finite is recomputed in FP64.
__device__ __forceinline__ float rcp_approx(float y) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(y));
  return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
template <bool FAST> __device__ __forceinline__ float rcp_f(float y) {
  if constexpr (FAST) return rcp_approx(y); else return rcp_(y);
}
template <bool FAST> __device__ __forceinline__ float div_f(float x, float y) {
  if constexpr (FAST) return x * rcp_approx(y); else return div_(x, y);
}
template <bool FAST> __device__ __forceinline__ float sqrt_f(float x) {
  if constexpr (FAST) return sqrt_approx(x); else return sqrtf(x);
}

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
template <class T, int NDIR, int BN, bool FAST = false>
__device__ __forceinline__ T fast_speed(const T *w, const PhysParams &P) {
  constexpr int RHO = 0, E = NDIR + 1, B0 = NDIR + 2;
  const T inv_rho = rcp_f<FAST>(w[RHO]);
  const T cs = T(P.gamma) * w[E] * inv_rho;
  T b2 = w[B0] * w[B0];
#pragma unroll
  for (int c = 1; c < NDIR; ++c) b2 = b2 + w[B0 + c] * w[B0 + c];
  const T cfast2 = b2 * inv_rho + cs;
  T av = cfast2 * cfast2 - T(4.0) * cs * (w[BN] * w[BN]) * inv_rho;
  if (av < T(0.0)) av = T(0.0);
  return sqrt_f<FAST>(T(0.5) * (cfast2 + sqrt_f<FAST>(av)));
}

// hd_get_cbounds (mod_hd_phys.t:891-1001) / mhd_get_cbounds (mod_mhd_phys.t:3037-3127).
// WITH_MIN=false gives the tvdlf form (cmax only).  Returns a status bit.
template <class T, bool MHD, int NDIR, bool GLM, int D, bool WITH_MIN, int BS = 0, bool FAST = false>
__device__ __forceinline__ uint32_t cbounds(const T *wLC, const T *wRC, const T *wLp,
                                            const T *wRp, const PhysParams &P, T &cmax,
                                            T &cmin) {
  using V = Vars<MHD, NDIR, GLM>;
  constexpr int MN = V::M0 + D;
  uint32_t st = 0;
  const int bsel = BS ? BS : P.boundspeed;
  if (bsel == BS_EINFELDT) {
    const T tmp1 = sqrt_f<FAST>(wLp[V::RHO]);
    const T tmp2 = sqrt_f<FAST>(wRp[V::RHO]);
    const T tmp3 = rcp_f<FAST>(tmp1 + tmp2);
    const T umean = (wLp[MN] * tmp1 + wRp[MN] * tmp2) * tmp3;
    const T dv = wRp[MN] - wLp[MN];
    T dmean;
    if constexpr (MHD) {
      const T csL = fast_speed<T, NDIR, V::B0 + D, FAST>(wLp, P);
      const T csR = fast_speed<T, NDIR, V::B0 + D, FAST>(wRp, P);
      dmean = sqrt_f<FAST>((tmp1 * (csL * csL) + tmp2 * (csR * csR)) * tmp3 +
                   T(0.5) * tmp1 * tmp2 * (tmp3 * tmp3) * (dv * dv));
    } else {
      const T csL = div_f<FAST>(T(P.gamma) * wLp[V::E], wLp[V::RHO]);
      const T csR = div_f<FAST>(T(P.gamma) * wRp[V::E], wRp[V::RHO]);
      dmean = sqrt_f<FAST>((tmp1 * csL + tmp2 * csR) * tmp3 + T(0.5) * tmp1 * tmp2 * (tmp3 * tmp3) * (dv * dv));
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
      const T cs = fast_speed<T, NDIR, V::B0 + D, FAST>(wm, P);
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
      const T tmp1 = div_f<FAST>(wm[MN], wm[V::RHO]);
      T m2 = wm[V::M0] * wm[V::M0];
#pragma unroll
      for (int c = 1; c < NDIR; ++c) m2 = m2 + wm[V::M0 + c] * wm[V::M0 + c];
      T pth = T(P.gamma_1) * (wm[V::E] - div_f<FAST>(T(0.5) * m2, wm[V::RHO]));
      if (P.fix_small_values) {
        if (pth < T(P.small_pressure)) pth = T(P.small_pressure);
      } else if (P.check_small_values) {
        if (pth < T(P.small_pressure)) st |= ST_SMALL_VALUE;
      }
      const T cs = sqrt_f<FAST>(div_f<FAST>(T(P.gamma) * pth, wm[V::RHO]));
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
      cs = fmax(fast_speed<T, NDIR, V::B0 + D, FAST>(wLp, P), fast_speed<T, NDIR, V::B0 + D, FAST>(wRp, P));
    } else {
      const T csL = div_f<FAST>(T(P.gamma) * wLp[V::E], wLp[V::RHO]);
      const T csR = div_f<FAST>(T(P.gamma) * wRp[V::E], wRp[V::RHO]);
      cs = fmax(sqrt_f<FAST>(csL), sqrt_f<FAST>(csR));
    }
    if (WITH_MIN) cmin = fmin(wLp[MN], wRp[MN]) - cs;
    cmax = fmax(wLp[MN], wRp[MN]) + cs;
  }
  return st;
}

// ------------------------------------------------------------------ limiters
// dwlimiter2 (mod_limiter.t:128-334) for one cell: a = dwC(ix) (forward
// difference), b = dwC(ix-1) (backward difference).  LEFT selects ldw, else rdw.
template <class T, bool LEFT, bool FAST = false>
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
      return div_f<FAST>(T(2.0) * fmax(b * a, T(0.0)), a + b + qsmall);
    case LIM_CADA3: {
      // branch-free: both the asymptotic and the limited form are evaluated
      // and the reference's three-way choice is made with selects
      const T tmpeta = (a * a + b * b) * rdelinv;
      const T t = LEFT ? div_f<FAST>(b, a + fsign(eps, a)) : div_f<FAST>(a, b + fsign(eps, b));
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
      const T t = LEFT ? div_f<FAST>(b, a + fsign(eps, a)) : div_f<FAST>(a, b + fsign(eps, b));
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

// phi of the cada3 / schmid limiters (dwlimiter2, src/limiter/mod_limiter.t:
// 253-290, 291-333) from the slope ratio t and tmpeta: the asymptotic third-
// order form below 1 - cadepsilon, the limited form above 1 + cadepsilon,
// their blend in between.  alfa / gam: 0.5 / 1.6 (cada3), 1 / 1.5 (schmid).
// The blend is formed only inside its 2e-14 wide band.
template <class T>
__device__ __forceinline__ T cada_blend_phi(T t, T tmpeta, T alfa, T gam) {
  constexpr T cadbeta = T(2.0), cadepsilon = T(1.0e-14), invcadepsilon = T(1.0e14);
  constexpr T third = T(1.0) / T(3.0);
  const T A = (T(2.0) + t) * third;
  const T lim2 = fmax(T(0.0), fmin(A, fmax(-(alfa * t), fmin(fmin(cadbeta * t, A), gam))));
  const bool low = tmpeta <= T(1.0) - cadepsilon;
  T phi = low ? A : lim2;
  if (!low && !(tmpeta >= T(1.0) + cadepsilon)) {
    const T t2 = (tmpeta - T(1.0)) * invcadepsilon;
    phi = T(0.5) * ((T(1.0) - t2) * A + (T(1.0) + t2) * lim2);
  }
  return phi;
}

// Both limited slopes of one face i+1/2 and one variable from the centred
// differences d0 = w(i)-w(i-1), d1 = w(i+1)-w(i), d2 = w(i+2)-w(i+1):
// ldw of cell i (dwlimiter2 with a = d1, b = d0) and rdw of cell i+1
// (a = d2, b = d1).  The cada family divides both ratios by the same
// d1 + sign(eps, d1), so one reciprocal serves the face; the other limiters
// take slope_impl as it is.
template <class T, int LIM, bool FAST = false>
__device__ __forceinline__ void face_slopes(int lim_rt, T d0, T d1, T d2, T rdelinv, T &ldw, T &rdw) {
  constexpr T eps = T(1.4901161193847656e-08);  // sqrt(epsilon(1d0)) = 2**-26
  const int lim = LIM ? LIM : lim_rt;
  if (lim == LIM_CADA3 || lim == LIM_CADA || lim == LIM_SCHMID) {
    const T rinv = rcp_f<FAST>(d1 + fsign(eps, d1));
    const T tl = d0 * rinv, tr = d2 * rinv;
    T pl, pr;
    if (lim == LIM_CADA3) {
      pl = cada_blend_phi<T>(tl, (d1 * d1 + d0 * d0) * rdelinv, T(0.5), T(1.6));
      pr = cada_blend_phi<T>(tr, (d2 * d2 + d1 * d1) * rdelinv, T(0.5), T(1.6));
    } else if (lim == LIM_SCHMID) {  // rdelinv carries (a2max + cadepsilon) dx^2
      pl = cada_blend_phi<T>(tl, sqrt_f<FAST>(T(0.4) * (d1 * d1 + d0 * d0)) / rdelinv, T(1.0), T(1.5));
      pr = cada_blend_phi<T>(tr, sqrt_f<FAST>(T(0.4) * (d2 * d2 + d1 * d1)) / rdelinv, T(1.0), T(1.5));
    } else {  // cada
      constexpr T third = T(1.0) / T(3.0);
      const T al = (T(2.0) + tl) * third, ar = (T(2.0) + tr) * third;
      pl = fmax(T(0.0), fmin(al, fmax(-(T(0.5) * tl), fmin(fmin(T(2.0) * tl, al), T(1.6)))));
      pr = fmax(T(0.0), fmin(ar, fmax(-(T(0.5) * tr), fmin(fmin(T(2.0) * tr, ar), T(1.6)))));
    }
    ldw = pl * d1;  // phi * a (left), phi * b (right): both d1
    rdw = pr * d1;
  } else {
    ldw = slope_impl<T, true, FAST>(lim, d1, d0, rdelinv);
    rdw = slope_impl<T, false, FAST>(lim, d2, d1, rdelinv);
  }
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
