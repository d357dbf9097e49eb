// CPU oracle: FP64 restatement of MPI-AMRVAC's per-block finite-volume update.
//
// TEST INFRASTRUCTURE ONLY (see amrvac_oracle.h).  Every routine follows the
// reference Fortran operation by operation (same expression order, no FMA
// contraction: compiled with -ffp-contract=off), so that per-cell results
// agree with the reference to rounding.  Each function cites the reference
// file:line it restates (paths relative to the reference repository root).
//
// All routines are templates on the scalar type R: R=double is the oracle,
// R=Counted counts +,-,*,/,sqrt,exp (FMA never occurs here) to give the
// algorithmic flop count per zone update, and R=Dual carries one directional
// derivative (forward mode) for the reference gradient of the adjoint.

#include "amrvac_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <array>
#include <map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ---------------------------------------------------------------- scalars
static thread_local long long g_ops = 0;

struct Counted {
  double v;
  Counted() : v(0) {}
  Counted(double x) : v(x) {}
  explicit operator double() const { return v; }
};
inline Counted operator+(Counted a, Counted b) { ++g_ops; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { ++g_ops; return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { ++g_ops; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { ++g_ops; return Counted(a.v / b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline Counted &operator+=(Counted &a, Counted b) { a = a + b; return a; }
inline Counted &operator-=(Counted &a, Counted b) { a = a - b; return a; }
inline Counted &operator*=(Counted &a, Counted b) { a = a * b; return a; }
inline bool operator<(Counted a, Counted b) { return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { return a.v != b.v; }

inline double val(double x) { return x; }
inline double val(Counted x) { return x.v; }
inline double rsqrt_(double x) { return std::sqrt(x); }
inline Counted rsqrt_(Counted x) { ++g_ops; return Counted(std::sqrt(x.v)); }
inline double rexp_(double x) { return std::exp(x); }
inline Counted rexp_(Counted x) { ++g_ops; return Counted(std::exp(x.v)); }
// Forward-mode dual number: value and one directional derivative.  Branches
// (limiters, upwind choices, max/min) follow the value, so the derivative is
// that of the discrete scheme along the branch the value takes.
struct Dual {
  double v, d;
  Dual() : v(0), d(0) {}
  Dual(double x) : v(x), d(0) {}
  Dual(double x, double dx) : v(x), d(dx) {}
};
inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
inline Dual &operator+=(Dual &a, Dual b) { a = a + b; return a; }
inline Dual &operator-=(Dual &a, Dual b) { a = a - b; return a; }
inline Dual &operator*=(Dual &a, Dual b) { a = a * b; return a; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline bool operator==(Dual a, Dual b) { return a.v == b.v; }
inline bool operator!=(Dual a, Dual b) { return a.v != b.v; }
inline double val(Dual x) { return x.v; }
inline Dual rsqrt_(Dual x) {
  const double r = std::sqrt(x.v);
  return Dual(r, x.d / (2.0 * r));
}
inline Dual rexp_(Dual x) {
  const double e = std::exp(x.v);
  return Dual(e, e * x.d);
}
inline Dual rabs(Dual x) { return x.v < 0.0 ? -x : x; }

template <class R> inline R rabs(R x) { return R(std::fabs(val(x))); }
template <class R> inline R rmax(R a, R b) { return (b > a) ? b : a; }
template <class R> inline R rmin(R a, R b) { return (b < a) ? b : a; }
// Fortran sign(a,b): |a| with the sign of b (signed zero honoured).
template <class R> inline R rsign(double a, R b) { return R(std::copysign(a, val(b))); }

// Fortran parameters (src/mod_constants.t).
constexpr double zero = 0.0, one = 1.0, two = 2.0, half = 0.5, quarter = 0.25;
constexpr double third = 1.0 / 3.0;
constexpr double smalldouble = 1.0e-12, bigdouble = 1.0e99;

// ---------------------------------------------------------------- layout
struct Box {
  int lo[3], hi[3];
};
inline Box shift(Box b, int d, int s) { b.lo[d] += s; b.hi[d] += s; return b; }

template <class F> inline void forbox(const Box &b, F &&f) {
  for (int k = b.lo[2]; k <= b.hi[2]; ++k)
    for (int j = b.lo[1]; j <= b.hi[1]; ++j)
      for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k);
}

struct Geo {
  int ndim, ng, n[3], nx[3];
  size_t cells;
  int idx(int i, int j, int k) const { return i + n[0] * (j + n[1] * k); }
  Box ixG() const { Box b; for (int d = 0; d < 3; ++d) { b.lo[d] = 0; b.hi[d] = n[d] - 1; } return b; }
  Box ixM() const {
    Box b;
    for (int d = 0; d < 3; ++d) {
      if (d < ndim) { b.lo[d] = ng; b.hi[d] = ng + nx[d] - 1; }
      else { b.lo[d] = 0; b.hi[d] = 0; }
    }
    return b;
  }
  int off(int d) const { return d == 0 ? 1 : (d == 1 ? n[0] : n[0] * n[1]); }
};

inline Geo make_geo(const orc_cfg &c) {
  Geo g;
  g.ndim = c.ndim;
  g.ng = c.nghost;
  for (int d = 0; d < 3; ++d) {
    g.nx[d] = d < c.ndim ? c.block_nx[d] : 1;
    g.n[d] = d < c.ndim ? c.block_nx[d] + 2 * c.nghost : 1;
  }
  g.cells = (size_t)g.n[0] * g.n[1] * g.n[2];
  return g;
}

// Variable indices, 0-based, in the reference order
// (src/hd/mod_hd_phys.t:210-226, src/mhd/mod_mhd_phys.t:478-503).
struct Ix {
  int rho, mom[3], e, mag[3], psi, nw, ndir;
  bool mhd, glm;
};
inline Ix make_ix(const orc_cfg &c) {
  Ix x;
  x.ndir = c.ndir;
  x.mhd = c.physics == 1;
  x.glm = x.mhd && c.divb == ORC_DIVB_GLM && c.ndim > 1;
  x.rho = 0;
  for (int d = 0; d < 3; ++d) x.mom[d] = d < c.ndir ? 1 + d : -1;
  x.e = c.ndir + 1;
  for (int d = 0; d < 3; ++d) x.mag[d] = (x.mhd && d < c.ndir) ? c.ndir + 2 + d : -1;
  x.psi = x.glm ? 2 * c.ndir + 2 : -1;
  x.nw = x.mhd ? (2 * c.ndir + 2 + (x.glm ? 1 : 0)) : c.ndir + 2;
  return x;
}

// Flux types (src/mhd/mod_mhd_phys.t:566-589): 0 default, 1 tvdlf, 2 special, 3 hll.
enum { FT_DEFAULT = 0, FT_TVDLF = 1, FT_SPECIAL = 2 };
inline int flux_type(const orc_cfg &c, const Ix &x, int idims /*0-based*/, int iw) {
  if (!x.mhd || c.ndim <= 1) return FT_DEFAULT;
  if (x.glm) {
    if (iw == x.psi) return FT_SPECIAL;
    if (iw == x.mag[idims]) return FT_SPECIAL;
    return FT_DEFAULT;
  }
  if (iw == x.mag[idims]) return FT_TVDLF;
  return FT_DEFAULT;
}

// Block array w(ixG^S,1:nv), column-major.
template <class R> struct Arr {
  const Geo *g = nullptr;
  int nv = 0;
  std::vector<R> d;
  Arr() {}
  Arr(const Geo &geo, int nvars) : g(&geo), nv(nvars), d(geo.cells * nvars) {}
  R &operator()(int i, int j, int k, int v) { return d[g->idx(i, j, k) + g->cells * (size_t)v]; }
  const R &operator()(int i, int j, int k, int v) const { return d[g->idx(i, j, k) + g->cells * (size_t)v]; }
};

struct State {
  orc_cfg c;
  Geo g;
  Ix x;
  double gamma_1, inv_gamma_1, small_e;
  // the directions advect1 advances (idim^LIM; a dimensionally split sweep
  // sets one), 0-based
  int idlo = 0, idhi = 0;
};

inline State make_state(const orc_cfg &c) {
  State s;
  s.c = c;
  s.g = make_geo(c);
  s.x = make_ix(c);
  s.gamma_1 = c.gamma - 1.0;
  s.inv_gamma_1 = 1.0 / s.gamma_1;
  s.idlo = 0;
  s.idhi = c.ndim - 1;
  // hd_check_params (src/hd/mod_hd_phys.t:541) / mhd_check_params (1213-1214)
  s.small_e = c.physics == 1 ? c.small_pressure * s.inv_gamma_1 : c.small_pressure / (c.gamma - 1.0);
  return s;
}

// gamma, gamma-1 and 1/(gamma-1) as scalars of type R.  double and Counted
// use the values precomputed in State (no counted operation, bit-identical
// to using them directly); Dual carries d(gamma) = g_dual_dgamma so that the
// forward-mode run differentiates with respect to gamma as well.
static double g_dual_dgamma = 0.0;
template <class R> inline R gam_(const State &s) { return R(s.c.gamma); }
template <class R> inline R gam1_(const State &s) { return R(s.gamma_1); }
template <class R> inline R igam1_(const State &s) { return R(s.inv_gamma_1); }
template <> inline Dual gam_<Dual>(const State &s) { return Dual(s.c.gamma, g_dual_dgamma); }
template <> inline Dual gam1_<Dual>(const State &s) { return Dual(s.gamma_1, g_dual_dgamma); }
template <> inline Dual igam1_<Dual>(const State &s) {
  return Dual(s.inv_gamma_1, -s.inv_gamma_1 * s.inv_gamma_1 * g_dual_dgamma);
}

// Accessor for one cell's variables inside an Arr.
#define W(a, v) a(i, j, k, v)

// ---------------------------------------------------------------- physics
// hd_to_conserved (src/hd/mod_hd_phys.t:677-700)
// mhd_to_conserved_origin (src/mhd/mod_mhd_phys.t:1562-1579)
template <class R> void to_conserved(const State &s, const Box &b, Arr<R> &w) {
  const Ix &x = s.x;
  forbox(b, [&](int i, int j, int k) {
    R v2 = W(w, x.mom[0]) * W(w, x.mom[0]);
    for (int c = 1; c < x.ndir; ++c) v2 = v2 + W(w, x.mom[c]) * W(w, x.mom[c]);
    if (x.mhd) {
      R b2 = W(w, x.mag[0]) * W(w, x.mag[0]);
      for (int c = 1; c < x.ndir; ++c) b2 = b2 + W(w, x.mag[c]) * W(w, x.mag[c]);
      W(w, x.e) = W(w, x.e) * igam1_<R>(s) + half * (v2 * W(w, x.rho) + b2);
    } else {
      W(w, x.e) = W(w, x.e) * igam1_<R>(s) + half * v2 * W(w, x.rho);
    }
    for (int c = 0; c < x.ndir; ++c) W(w, x.mom[c]) = W(w, x.rho) * W(w, x.mom[c]);
  });
}

template <class R> int handle_small_values(const State &s, bool primitive, Arr<R> &w, const Box &b);

// hd_to_primitive (src/hd/mod_hd_phys.t:703-734)
// mhd_to_primitive_origin (src/mhd/mod_mhd_phys.t:1741-1765)
template <class R> int to_primitive(const State &s, const Box &b, Arr<R> &w) {
  int st = 0;
  if (s.c.fix_small_values) st |= handle_small_values(s, false, w, b);
  const Ix &x = s.x;
  forbox(b, [&](int i, int j, int k) {
    R inv_rho = R(1.0) / W(w, x.rho);
    for (int c = 0; c < x.ndir; ++c) W(w, x.mom[c]) = W(w, x.mom[c]) * inv_rho;
    R v2 = W(w, x.mom[0]) * W(w, x.mom[0]);
    for (int c = 1; c < x.ndir; ++c) v2 = v2 + W(w, x.mom[c]) * W(w, x.mom[c]);
    if (x.mhd) {
      R b2 = W(w, x.mag[0]) * W(w, x.mag[0]);
      for (int c = 1; c < x.ndir; ++c) b2 = b2 + W(w, x.mag[c]) * W(w, x.mag[c]);
      W(w, x.e) = gam1_<R>(s) * (W(w, x.e) - half * (W(w, x.rho) * v2 + b2));
    } else {
      W(w, x.e) = gam1_<R>(s) * (W(w, x.e) - half * W(w, x.rho) * v2);
    }
  });
  return st;
}

// small_values_average (src/mod_small_values.t:89-144) of component iw over
// ixO: a flagged value becomes the mean of the unflagged values of the
// smallest cube of half-width 1 .. small_values_daverage around it (clipped
// to the whole block array, ixI) that holds one, summed x fastest as
// Fortran's sum(mask) does; with none, rho -> small_density and e ->
// small_pressure.  flag: per cell of the array, false outside ixO.
template <class R>
void small_values_average(const State &s, Arr<R> &w, const Box &ixO, const std::vector<char> &flag, int iw) {
  const Geo &g = s.g;
  const Box ixI = g.ixG();
  const int nd = s.c.ndim, dav = std::max(s.c.small_values_daverage, 1);
  const size_t vo = g.cells * (size_t)iw;
  forbox(ixO, [&](int i, int j, int k) {
    if (!flag[g.idx(i, j, k)]) return;
    const int ix[3] = {i, j, k};
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool ok = false;
    for (int r = 1; r <= dav && !ok; ++r) {
      for (int d = 0; d < 3; ++d) {
        lo[d] = d < nd ? std::max(ix[d] - r, ixI.lo[d]) : ix[d];
        hi[d] = d < nd ? std::min(ix[d] + r, ixI.hi[d]) : ix[d];
      }
      for (int kk = lo[2]; kk <= hi[2] && !ok; ++kk)
        for (int jj = lo[1]; jj <= hi[1] && !ok; ++jj)
          for (int ii = lo[0]; ii <= hi[0] && !ok; ++ii) ok = !flag[g.idx(ii, jj, kk)];
    }
    if (ok) {
      R sum(0.0);
      int cnt = 0;
      for (int kk = lo[2]; kk <= hi[2]; ++kk)
        for (int jj = lo[1]; jj <= hi[1]; ++jj)
          for (int ii = lo[0]; ii <= hi[0]; ++ii) {
            const size_t p = g.idx(ii, jj, kk);
            if (!flag[p]) { sum = sum + w.d[vo + p]; ++cnt; }
          }
      w.d[vo + g.idx(i, j, k)] = sum / R(double(cnt));
    } else if (iw == s.x.e) {
      w.d[vo + g.idx(i, j, k)] = R(s.c.small_pressure);
    } else if (iw == s.x.rho) {
      w.d[vo + g.idx(i, j, k)] = R(s.c.small_density);
    }
  });
}

// hd_check_w (src/hd/mod_hd_phys.t:648-674), mhd_check_w_origin (1452-1473),
// handle_small_values replace/error/average (src/hd/mod_hd_phys.t:1420-1516,
// src/mhd/mod_mhd_phys.t:2191-2253, src/mod_small_values.t:25-144).  The
// array w spans the whole block (ixI); b is ixO.
template <class R> int handle_small_values(const State &s, bool primitive, Arr<R> &w, const Box &b) {
  const Ix &x = s.x;
  const orc_cfg &c = s.c;
  int st = 0;
  if (c.small_values_method == 2) {  // average: flags first, then the averages
    const Geo &g = s.g;
    std::vector<char> frho(g.cells, 0), fe(g.cells, 0);
    bool any = false;
    forbox(b, [&](int i, int j, int k) {
      R m2 = W(w, x.mom[0]) * W(w, x.mom[0]);
      for (int q = 1; q < x.ndir; ++q) m2 = m2 + W(w, x.mom[q]) * W(w, x.mom[q]);
      bool fl_e;
      if (primitive) {
        fl_e = W(w, x.e) < R(c.small_pressure);
      } else if (x.mhd) {
        R b2 = W(w, x.mag[0]) * W(w, x.mag[0]);
        for (int q = 1; q < x.ndir; ++q) b2 = b2 + W(w, x.mag[q]) * W(w, x.mag[q]);
        fl_e = W(w, x.e) - half * (m2 / W(w, x.rho) + b2) < R(s.small_e);
      } else {
        fl_e = gam1_<R>(s) * (W(w, x.e) - half * m2 / W(w, x.rho)) < R(c.small_pressure);
      }
      const bool fl_r = W(w, x.rho) < R(c.small_density);
      frho[g.idx(i, j, k)] = fl_r;
      fe[g.idx(i, j, k)] = fl_e;
      any = any || fl_r || fl_e;
    });
    if (!any) return 0;
    const Box ixI = g.ixG();
    auto m2_of = [&](int i, int j, int k) {
      R m2 = W(w, x.mom[0]) * W(w, x.mom[0]);
      for (int q = 1; q < x.ndir; ++q) m2 = m2 + W(w, x.mom[q]) * W(w, x.mom[q]);
      return m2;
    };
    auto b2_of = [&](int i, int j, int k) {
      R b2 = W(w, x.mag[0]) * W(w, x.mag[0]);
      for (int q = 1; q < x.ndir; ++q) b2 = b2 + W(w, x.mag[q]) * W(w, x.mag[q]);
      return b2;
    };
    small_values_average(s, w, b, frho, x.rho);
    if (primitive) {
      small_values_average(s, w, b, fe, x.e);
    } else if (x.mhd) {  // internal energy, averaged, back (mod_mhd_phys.t:2227-2240)
      forbox(ixI, [&](int i, int j, int k) {
        W(w, x.e) = W(w, x.e) - half * (m2_of(i, j, k) / W(w, x.rho) + b2_of(i, j, k));
      });
      small_values_average(s, w, b, fe, x.e);
      forbox(ixI, [&](int i, int j, int k) {
        W(w, x.e) = W(w, x.e) + half * (m2_of(i, j, k) / W(w, x.rho) + b2_of(i, j, k));
      });
    } else {  // pressure, averaged, back (mod_hd_phys.t:1482-1489)
      forbox(ixI, [&](int i, int j, int k) {
        W(w, x.e) = gam1_<R>(s) * (W(w, x.e) - R(0.5) * m2_of(i, j, k) / W(w, x.rho));
      });
      small_values_average(s, w, b, fe, x.e);
      forbox(ixI, [&](int i, int j, int k) {
        W(w, x.e) = W(w, x.e) / gam1_<R>(s) + R(0.5) * m2_of(i, j, k) / W(w, x.rho);
      });
    }
    return 0;
  }
  forbox(b, [&](int i, int j, int k) {
    bool frho = W(w, x.rho) < R(c.small_density);
    bool fe;
    R m2 = W(w, x.mom[0]) * W(w, x.mom[0]);
    for (int q = 1; q < x.ndir; ++q) m2 = m2 + W(w, x.mom[q]) * W(w, x.mom[q]);
    if (primitive) {
      fe = W(w, x.e) < R(c.small_pressure);
    } else if (x.mhd) {
      R b2 = W(w, x.mag[0]) * W(w, x.mag[0]);
      for (int q = 1; q < x.ndir; ++q) b2 = b2 + W(w, x.mag[q]) * W(w, x.mag[q]);
      fe = W(w, x.e) - half * (m2 / W(w, x.rho) + b2) < R(s.small_e);
    } else {
      R tmp = gam1_<R>(s) * (W(w, x.e) - half * m2 / W(w, x.rho));
      fe = tmp < R(c.small_pressure);
    }
    if (!frho && !fe) return;
    if (c.small_values_method == 1) {  // replace
      if (frho) {
        W(w, x.rho) = R(c.small_density);
        for (int q = 0; q < x.ndir; ++q) W(w, x.mom[q]) = R(0.0);
      }
      auto kin_mag = [&]() {
        R mm = W(w, x.mom[0]) * W(w, x.mom[0]);
        for (int q = 1; q < x.ndir; ++q) mm = mm + W(w, x.mom[q]) * W(w, x.mom[q]);
        if (x.mhd) {
          R bb = W(w, x.mag[0]) * W(w, x.mag[0]);
          for (int q = 1; q < x.ndir; ++q) bb = bb + W(w, x.mag[q]) * W(w, x.mag[q]);
          return half * (mm / W(w, x.rho) + bb);
        }
        return half * mm / W(w, x.rho);
      };
      if (!x.mhd && frho) {
        if (primitive) W(w, x.e) = R(c.small_pressure);
        else W(w, x.e) = R(s.small_e) + kin_mag();
      }
      if (fe) {
        if (primitive) W(w, x.e) = R(c.small_pressure);
        else W(w, x.e) = R(s.small_e) + kin_mag();
      }
    } else {
      st |= ORC_ST_SMALL_VALUE;
    }
  });
  return st;
}

// hd_get_flux (src/hd/mod_hd_phys.t:1097-1146),
// mhd_get_flux (src/mhd/mod_mhd_phys.t:3810-3889)
template <class R>
void get_flux(const State &s, const Arr<R> &wC, const Arr<R> &w, const Box &b, int idim,
              double cmax_global, Arr<R> &f) {
  const Ix &x = s.x;
  const int mn = x.mom[idim];
  forbox(b, [&](int i, int j, int k) {
    if (!x.mhd) {
      W(f, x.rho) = W(w, mn) * W(w, x.rho);
      for (int c = 0; c < x.ndir; ++c) W(f, x.mom[c]) = W(w, mn) * W(wC, x.mom[c]);
      W(f, mn) = W(f, mn) + W(w, x.e);
      W(f, x.e) = W(w, mn) * (W(wC, x.e) + W(w, x.e));
      return;
    }
    const int bn = x.mag[idim];
    W(f, x.rho) = W(w, mn) * W(w, x.rho);
    for (int c = 0; c < x.ndir; ++c)
      W(f, x.mom[c]) = W(wC, mn) * W(w, x.mom[c]) - W(w, bn) * W(w, x.mag[c]);
    R b2 = W(w, x.mag[0]) * W(w, x.mag[0]);
    for (int c = 1; c < x.ndir; ++c) b2 = b2 + W(w, x.mag[c]) * W(w, x.mag[c]);
    R ptotal = W(w, x.e) + half * b2;
    W(f, mn) = W(f, mn) + ptotal;
    R bv = W(w, x.mag[0]) * W(w, x.mom[0]);
    for (int c = 1; c < x.ndir; ++c) bv = bv + W(w, x.mag[c]) * W(w, x.mom[c]);
    W(f, x.e) = W(w, mn) * (W(wC, x.e) + ptotal) - W(w, bn) * bv;
    for (int c = 0; c < x.ndir; ++c)
      W(f, x.mag[c]) = W(w, mn) * W(w, x.mag[c]) - W(w, bn) * W(w, x.mom[c]);
    if (x.glm) {
      W(f, bn) = W(w, x.psi);
      W(f, x.psi) = R(cmax_global * cmax_global) * W(w, bn);
    }
  });
}

// mhd_get_csound_prim (src/mhd/mod_mhd_phys.t:3329-3379), one cell.
template <class R>
R csound_prim(const State &s, const Arr<R> &w, int i, int j, int k, int idim) {
  const Ix &x = s.x;
  R inv_rho = R(1.0) / W(w, x.rho);
  R cs = gam_<R>(s) * W(w, x.e) * inv_rho;
  R b2 = W(w, x.mag[0]) * W(w, x.mag[0]);
  for (int c = 1; c < x.ndir; ++c) b2 = b2 + W(w, x.mag[c]) * W(w, x.mag[c]);
  R cfast2 = b2 * inv_rho + cs;
  R bn = W(w, x.mag[idim]);
  R av = cfast2 * cfast2 - R(4.0) * cs * (bn * bn) * inv_rho;
  if (av < R(zero)) av = R(zero);
  return rsqrt_(half * (cfast2 + rsqrt_(av)));
}

// hd_get_pthermal + hd_get_csound2 on a conserved state (src/hd/mod_hd_phys.t:1003-1065)
template <class R>
R hd_csound2_cons(const State &s, const Arr<R> &w, int i, int j, int k, int &st) {
  const Ix &x = s.x;
  R m2 = W(w, x.mom[0]) * W(w, x.mom[0]);
  for (int c = 1; c < x.ndir; ++c) m2 = m2 + W(w, x.mom[c]) * W(w, x.mom[c]);
  R ke = R(0.5) * m2 / W(w, x.rho);
  R pth = gam1_<R>(s) * (W(w, x.e) - ke);
  if (s.c.fix_small_values) {
    if (pth < R(s.c.small_pressure)) pth = R(s.c.small_pressure);
  } else if (s.c.check_small_values) {
    if (pth < R(s.c.small_pressure)) st |= ORC_ST_SMALL_VALUE;
  }
  return gam_<R>(s) * pth / W(w, x.rho);
}

// hd_get_cbounds (src/hd/mod_hd_phys.t:891-1001),
// mhd_get_cbounds (src/mhd/mod_mhd_phys.t:3037-3127).  cmin==nullptr: tvdlf form.
template <class R>
int get_cbounds(const State &s, const Arr<R> &wLC, const Arr<R> &wRC, const Arr<R> &wLp,
                const Arr<R> &wRp, const Box &b, int idim, Arr<R> &cmax, Arr<R> *cmin) {
  const Ix &x = s.x;
  const int mn = x.mom[idim];
  int st = 0;
  Arr<R> wmean;
  if (s.c.boundspeed == ORC_BS_CMAXMEAN) wmean = Arr<R>(s.g, x.nw);
  forbox(b, [&](int i, int j, int k) {
    switch (s.c.boundspeed) {
      case ORC_BS_EINFELDT: {
        R csL, csR;
        if (x.mhd) {
          csL = csound_prim(s, wLp, i, j, k, idim);
          csR = csound_prim(s, wRp, i, j, k, idim);
        }
        R tmp1 = rsqrt_(W(wLp, x.rho));
        R tmp2 = rsqrt_(W(wRp, x.rho));
        R tmp3 = R(1.0) / (tmp1 + tmp2);
        R umean = (W(wLp, mn) * tmp1 + W(wRp, mn) * tmp2) * tmp3;
        R dv = W(wRp, mn) - W(wLp, mn);
        R dmean;
        if (x.mhd) {
          dmean = rsqrt_((tmp1 * (csL * csL) + tmp2 * (csR * csR)) * tmp3 +
                         half * tmp1 * tmp2 * (tmp3 * tmp3) * (dv * dv));
        } else {
          csL = gam_<R>(s) * W(wLp, x.e) / W(wLp, x.rho);
          csR = gam_<R>(s) * W(wRp, x.e) / W(wRp, x.rho);
          dmean = (tmp1 * csL + tmp2 * csR) * tmp3 + R(0.5) * tmp1 * tmp2 * (tmp3 * tmp3) * (dv * dv);
          dmean = rsqrt_(dmean);
        }
        if (cmin) {
          (*cmin)(i, j, k, 0) = umean - dmean;
          cmax(i, j, k, 0) = umean + dmean;
        } else {
          cmax(i, j, k, 0) = rabs(umean) + dmean;
        }
        break;
      }
      case ORC_BS_CMAXMEAN: {
        if (x.mhd) {
          for (int iw = 0; iw < x.nw; ++iw) W(wmean, iw) = R(0.5) * (W(wLp, iw) + W(wRp, iw));
          R csR = csound_prim(s, wmean, i, j, k, idim);
          if (cmin) {
            cmax(i, j, k, 0) = rmax(W(wmean, mn) + csR, R(zero));
            (*cmin)(i, j, k, 0) = rmin(W(wmean, mn) - csR, R(zero));
          } else {
            cmax(i, j, k, 0) = rabs(W(wmean, mn)) + csR;
          }
        } else {
          for (int iw = 0; iw < x.nw; ++iw) W(wmean, iw) = R(0.5) * (W(wLC, iw) + W(wRC, iw));
          R tmp1 = W(wmean, mn) / W(wmean, x.rho);
          R csR = rsqrt_(hd_csound2_cons(s, wmean, i, j, k, st));
          if (cmin) {
            cmax(i, j, k, 0) = rmax(tmp1 + csR, R(zero));
            (*cmin)(i, j, k, 0) = rmin(tmp1 - csR, R(zero));
          } else {
            cmax(i, j, k, 0) = rabs(tmp1) + csR;
          }
        }
        break;
      }
      default: {  // cmaxleftright
        R csL, csR;
        if (x.mhd) {
          csL = csound_prim(s, wLp, i, j, k, idim);
          csR = csound_prim(s, wRp, i, j, k, idim);
          csL = rmax(csL, csR);
        } else {
          csL = gam_<R>(s) * W(wLp, x.e) / W(wLp, x.rho);
          csR = gam_<R>(s) * W(wRp, x.e) / W(wRp, x.rho);
          csL = rmax(rsqrt_(csL), rsqrt_(csR));
        }
        if (cmin) {
          (*cmin)(i, j, k, 0) = rmin(W(wLp, mn), W(wRp, mn)) - csL;
          cmax(i, j, k, 0) = rmax(W(wLp, mn), W(wRp, mn)) + csL;
        } else {
          cmax(i, j, k, 0) = rmax(W(wLp, mn), W(wRp, mn)) + csL;
        }
        break;
      }
    }
  });
  return st;
}

// dwlimiter2 (src/limiter/mod_limiter.t:128-334) on the box ixC; results on
// ixC contracted by one at its lower end in direction idims.
template <class R>
void dwlimiter2(const State &s, const Arr<R> &dwC, const Box &ixC, int idims, double dxlevel,
                Arr<R> &ldw, Arr<R> &rdw) {
  const double qsmall = 1.0e-12, qsmall2 = 2.0e-12;
  const double eps = std::sqrt(2.220446049250313e-16);
  const double c_mcbeta = 1.4, cadalfa = 0.5, cadbeta = 2.0, cadgamma = 1.6;
  const double cadepsilon = 1.0e-14, invcadepsilon = 1.0e14;
  Box ixO = ixC;
  ixO.lo[idims] += 1;
  const int o = s.g.off(idims);
  const int lim = s.c.limiter;
  R rdelinv(0.0);
  if (lim == ORC_LIM_CADA3) {
    R r = R(s.c.cada3_radius) * R(dxlevel);
    rdelinv = R(one) / (r * r);
  }
  forbox(ixO, [&](int i, int j, int k) {
    const int p = s.g.idx(i, j, k);
    R a = dwC.d[p];      // dwC(ixO)
    R bb = dwC.d[p - o]; // dwC(hxO)
    R l, r;
    switch (lim) {
      case ORC_LIM_MINMOD: {
        R t = rsign(one, a);
        t = t * rmax(R(zero), rmin(rabs(a), t * bb));
        l = r = t;
        break;
      }
      case ORC_LIM_WOODWARD: {
        R t = rsign(one, a);
        t = R(2.0) * t * rmax(R(zero), rmin(rmin(rabs(a), t * bb), t * R(quarter) * (bb + a)));
        l = r = t;
        break;
      }
      case ORC_LIM_MCBETA: {
        R t = rsign(one, a);
        t = t * rmax(R(zero), rmin(rmin(R(c_mcbeta) * rabs(a), R(c_mcbeta) * t * bb), t * R(half) * (bb + a)));
        l = r = t;
        break;
      }
      case ORC_LIM_SUPERBEE: {
        R t = rsign(one, a);
        t = t * rmax(rmax(R(zero), rmin(R(2.0) * rabs(a), t * bb)), rmin(rabs(a), R(2.0) * t * bb));
        l = r = t;
        break;
      }
      case ORC_LIM_VANLEER: {
        R t = R(2.0) * rmax(bb * a, R(zero)) / (a + bb + R(qsmall));
        l = r = t;
        break;
      }
      case ORC_LIM_ALBADA: {
        R t = (bb * (a * a + R(qsmall)) + a * (bb * bb + R(qsmall))) / (a * a + bb * bb + R(qsmall2));
        l = r = t;
        break;
      }
      case ORC_LIM_KOREN: {
        R t = rsign(one, a);
        R t2 = rmin(R(2.0) * rabs(a), R(2.0) * t * bb);
        l = t * rmax(R(zero), rmin(t2, (bb * t + R(2.0) * rabs(a)) * R(third)));
        r = t * rmax(R(zero), rmin(t2, (R(2.0) * bb * t + rabs(a)) * R(third)));
        break;
      }
      case ORC_LIM_CADA: {
        R t = bb / (a + rsign(eps, a));
        R t2 = (R(2.0) + t) * R(third);
        l = rmax(R(zero), rmin(t2, rmax(-(R(cadalfa) * t), rmin(rmin(R(cadbeta) * t, t2), R(cadgamma))))) * a;
        t = a / (bb + rsign(eps, bb));
        t2 = (R(2.0) + t) * R(third);
        r = rmax(R(zero), rmin(t2, rmax(-(R(cadalfa) * t), rmin(rmin(R(cadbeta) * t, t2), R(cadgamma))))) * bb;
        break;
      }
      case ORC_LIM_SCHMID: {  // schmid2: a2max = schmid_rad(idims) (src/limiter/mod_limiter.t:291-333)
        R tmpeta = rsqrt_(R(0.4) * (a * a + bb * bb)) /
                   ((R(s.c.schmid_rad[idims]) + R(cadepsilon)) * (R(dxlevel) * R(dxlevel)));
        auto phi = [&](R t) {
          R A = (R(two) + t) * R(third);
          R B = rmax(R(zero), rmin(A, rmax(-t, rmin(rmin(R(cadbeta) * t, A), R(1.5)))));
          if (tmpeta <= R(one - cadepsilon)) return A;
          if (tmpeta >= R(one + cadepsilon)) return B;
          R t2 = (tmpeta - R(one)) * R(invcadepsilon);
          return R(half) * ((R(one) - t2) * A + (R(one) + t2) * B);
        };
        l = phi(bb / (a + rsign(eps, a))) * a;
        r = phi(a / (bb + rsign(eps, bb))) * bb;
        break;
      }
      default: {  // cada3
        R tmpeta = (a * a + bb * bb) * rdelinv;
        auto phi = [&](R t) {
          R A = (R(two) + t) * R(third);
          R res;
          if (tmpeta <= R(one - cadepsilon)) {
            res = A;
          } else if (tmpeta >= R(one + cadepsilon)) {
            res = rmax(R(zero), rmin(A, rmax(-(R(cadalfa) * t), rmin(rmin(R(cadbeta) * t, A), R(cadgamma)))));
          } else {
            R t2 = (tmpeta - R(one)) * R(invcadepsilon);
            res = R(half) * ((R(one) - t2) * A +
                             (R(one) + t2) * rmax(R(zero), rmin(A, rmax(-(R(cadalfa) * t), rmin(rmin(R(cadbeta) * t, A), R(cadgamma))))));
          }
          return res;
        };
        l = phi(bb / (a + rsign(eps, a))) * a;
        r = phi(a / (bb + rsign(eps, bb))) * bb;
        break;
      }
    }
    ldw.d[p] = l;
    rdw.d[p] = r;
  });
}

// MP5limiter (src/limiter/mod_mp5.t:16-201) with its minmod and median
// (404-432), one variable of one face: the left state at face i+1/2 from
// w(i-2) .. w(i+2); the right state is the same expression on the data
// mirrored about the face (w(i+3) .. w(i-1)), term for term the reference's
// right-side formulas.
template <class R> R mp5_minmod(R a, R b) {
  return (rsign(one, a) + rsign(one, b)) / R(2.0) * rmin(rabs(a), rabs(b));
}
template <class R> R mp5_median(R a, R b, R c) {
  R t1 = b - a, t2 = c - a;
  return a + (rsign(one, t1) + rsign(one, t2)) / R(2.0) * rmin(rabs(t1), rabs(t2));
}
template <class R> R mp5_side(R wmm, R wm, R w0, R wp, R wpp) {
  R f = R(1.0 / 60.0) * ((((R(2.0) * wmm - R(13.0) * wm) + R(47.0) * w0) + R(27.0) * wp) - R(3.0) * wpp);
  R b = R(4.0) * (w0 - wm);
  R fmp = w0 + mp5_minmod(wp - w0, b);
  R ful = w0 + b;
  R dm = (w0 - R(2.0) * wm) + wmm, d0 = (wp - R(2.0) * w0) + wm, dp = (wpp - R(2.0) * wp) + w0;
  R dm4_0 = mp5_minmod(mp5_minmod(R(4.0) * d0 - dp, R(4.0) * dp - d0), mp5_minmod(d0, dp));
  R dm4_m = mp5_minmod(mp5_minmod(R(4.0) * dm - d0, R(4.0) * d0 - dm), mp5_minmod(dm, d0));
  R fmd = (w0 + wp) / R(2.0) - dm4_0 / R(2.0);
  R flc = R(half) * (R(3.0) * w0 - wm) + R(4.0 / 3.0) * dm4_m;
  R fmn = rmax(rmin(rmin(w0, wp), fmd), rmin(rmin(w0, ful), flc));
  R fmx = rmin(rmax(rmax(w0, wp), fmd), rmax(rmax(w0, ful), flc));
  if ((f - w0) * (f - fmp) <= R(0.0)) return f;
  return mp5_median(fmn, f, fmx);
}

// WENO5limiter (src/limiter/mod_weno.t:254-377), one variable of one face;
// var 1 WENO-JS, 2 WENO-Z, 3 WENO-Z+ (lambda = dx^(2/3)).  Left state from
// w(i-2) .. w(i+2); the right state is the same expression on the mirrored
// data, term for term the reference's right-side formulas.
template <class R> R weno5_side(R wmm, R wm, R w0, R wp, R wpp, int var, R lambda) {
  const double eps = 1.0e-18;  // weno_eps_machine
  const double b1 = 1.0833333333333333, b2 = 0.25;
  const double d[3] = {1.0 / 10.0, 3.0 / 5.0, 3.0 / 10.0};
  R f[3], be[3], a[3];
  f[0] = R(1.0 / 3.0) * wmm + R(-7.0 / 6.0) * wm + R(11.0 / 6.0) * w0;
  f[1] = R(-1.0 / 6.0) * wm + R(5.0 / 6.0) * w0 + R(1.0 / 3.0) * wp;
  f[2] = R(1.0 / 3.0) * w0 + R(5.0 / 6.0) * wp + R(-1.0 / 6.0) * wpp;
  R s1 = wmm + w0 - R(2.0) * wm, t1 = wmm - R(4.0) * wm + R(3.0) * w0;
  R s2 = wm + wp - R(2.0) * w0, t2 = wm - wp;
  R s3 = w0 + wpp - R(2.0) * wp, t3 = R(3.0) * w0 - R(4.0) * wp + wpp;
  be[0] = R(b1) * (s1 * s1) + R(b2) * (t1 * t1);
  be[1] = R(b1) * (s2 * s2) + R(b2) * (t2 * t2);
  be[2] = R(b1) * (s3 * s3) + R(b2) * (t3 * t3);
  const R tau = rabs(be[0] - be[2]);
  for (int i = 0; i < 3; ++i) {
    if (var == 1) {
      a[i] = R(d[i]) / ((be[i] + R(eps)) * (be[i] + R(eps)));
    } else if (var == 2) {
      R r = tau / (be[i] + R(eps));
      a[i] = R(d[i]) * (R(1.0) + r * r);
    } else {
      R r = (tau + R(eps)) / (be[i] + R(eps));
      a[i] = R(d[i]) * (R(1.0) + r * r + lambda / r);
    }
  }
  R asum = ((R(0.0) + a[0]) + a[1]) + a[2];
  R out(0.0);
  for (int i = 0; i < 3; ++i) out = out + f[i] * a[i] / asum;
  return out;
}

// WENO3limiter (src/limiter/mod_weno.t:165-252), one variable of one face;
// var 1 WENO3, 2 WENO-YC3.  Left state from w(i-1), w(i), w(i+1); the right
// state on the mirrored data w(i+2), w(i+1), w(i).
template <class R> R weno3_side(R wm, R w0, R wp, int var, double dx2) {
  const double eps = 1.0e-18;
  R f1 = R(-1.0 / 2.0) * wm + R(3.0 / 2.0) * w0;
  R f2 = R(1.0 / 2.0) * w0 + R(1.0 / 2.0) * wp;
  R be1 = (w0 - wm) * (w0 - wm), be2 = (wp - w0) * (wp - w0);
  R a1, a2;
  if (var == 1) {
    a1 = R(1.0 / 3.0) / ((be1 + R(eps)) * (be1 + R(eps)));
    a2 = R(2.0 / 3.0) / ((be2 + R(eps)) * (be2 + R(eps)));
  } else {
    R tau = rabs(be2 - be1);
    a1 = R(1.0 / 3.0) * (R(1.0) + tau / (be1 + R(dx2)));
    a2 = R(2.0 / 3.0) * (R(1.0) + tau / (be2 + R(dx2)));
  }
  R asum = (R(0.0) + a1) + a2;
  return (R(0.0) + f1 * a1 / asum) + f2 * a2 / asum;
}

// venklimiter (src/limiter/mod_venk.t:6-106): phi of one cell.
template <class R> R venk_phi(R wm, R w0, R wp, R eps2) {
  const double omega = 1.0e-12;
  R wmax = rmax(rmax(wm, w0), wp), wmin = rmin(rmin(wm, w0), wp);
  R westp = w0 + (wp - wm) * R(0.25), westm = w0 - (wp - wm) * R(0.25);
  auto ratio = [&](R dp, R dmr) {
    R dm = rsign(val(rabs(dmr)) + omega, dmr);
    R p1 = (dp * dp + eps2) + R(2.0) * dp * dm;
    R p2 = dp * dp + R(2.0) * (dm * dm) + dp * dm + eps2;
    return p1 / p2;
  };
  R phip(1.0), phim(1.0);
  if (westp > w0) phip = ratio(wmax - w0, westp - w0);
  else if (westp < w0) phip = ratio(wmin - w0, westp - w0);
  if (westm < w0) phim = ratio(-(wmax - w0), westm - w0);
  else if (westm > w0) phim = ratio(-(wmin - w0), westm - w0);
  return rmin(phim, phip);
}

// reconstruct_LR default (limiter) branch (src/mod_finite_volume.t:1110-1228)
// and its MP5 branch (1131-1132: MP5limiter with fix_limiter1,
// src/limiter/mod_weno.t:135-163; no small-value fix of the states)
template <class R>
int reconstruct_LR(const State &s, const Box &ixL, const Box &ixR, int idims, const Arr<R> &w,
                   Arr<R> &wLC, Arr<R> &wRC, Arr<R> &wLp, Arr<R> &wRp, double dxdim) {
  const Ix &x = s.x;
  const Geo &g = s.g;
  const int o = g.off(idims);
  if (s.c.limiter == ORC_LIM_VENK) {
    // venklimiter, then the small-value fix of both states (1157-1162)
    const R kd = R(0.3) * R(dxdim);
    const R eps2 = kd * kd * kd;
    for (int iw = 0; iw < x.nw; ++iw)
      forbox(ixL, [&](int i, int j, int k) {
        const size_t p = g.idx(i, j, k) + g.cells * (size_t)iw;
        const R *q = &w.d[p];
        wLp.d[p] = q[0] + R(0.25) * (q[o] - q[-o]) * venk_phi(q[-o], q[0], q[o], eps2);
        wRp.d[p] = q[o] - R(0.25) * (q[2 * o] - q[0]) * venk_phi(q[0], q[o], q[2 * o], eps2);
      });
    int st = 0;
    if (s.c.fix_small_values) {
      st |= handle_small_values(s, true, wLp, ixL);
      st |= handle_small_values(s, true, wRp, ixR);
    }
    for (int iw = 0; iw < x.nw; ++iw) {
      forbox(ixL, [&](int i, int j, int k) { wLC(i, j, k, iw) = wLp(i, j, k, iw); });
      forbox(ixR, [&](int i, int j, int k) { wRC(i, j, k, iw) = wRp(i, j, k, iw); });
    }
    to_conserved(s, ixL, wLC);
    to_conserved(s, ixR, wRC);
    return st;
  }
  if (s.c.limiter == ORC_LIM_WENO3 || s.c.limiter == ORC_LIM_WENOYC3) {
    // WENO3limiter then fix_limiter (any flagged density or pressure: every
    // variable of the face flat)
    const int var = s.c.limiter == ORC_LIM_WENO3 ? 1 : 2;
    const double dx2 = dxdim * dxdim;
    forbox(ixL, [&](int i, int j, int k) {
      const size_t p = g.idx(i, j, k);
      R wl[16], wr[16];
      for (int iw = 0; iw < x.nw; ++iw) {
        const R *q = &w.d[p + g.cells * (size_t)iw];
        wl[iw] = weno3_side(q[-o], q[0], q[o], var, dx2);
        wr[iw] = weno3_side(q[2 * o], q[o], q[0], var, dx2);
      }
      const bool flag = wl[x.rho] < R(s.c.small_density) || wr[x.rho] < R(s.c.small_density) ||
                        wl[x.e] < R(s.c.small_pressure) || wr[x.e] < R(s.c.small_pressure);
      if (flag) return;
      for (int iw = 0; iw < x.nw; ++iw) {
        wLp.d[p + g.cells * (size_t)iw] = wl[iw];
        wRp.d[p + g.cells * (size_t)iw] = wr[iw];
      }
    });
    for (int iw = 0; iw < x.nw; ++iw) {
      forbox(ixL, [&](int i, int j, int k) { wLC(i, j, k, iw) = wLp(i, j, k, iw); });
      forbox(ixR, [&](int i, int j, int k) { wRC(i, j, k, iw) = wRp(i, j, k, iw); });
    }
    to_conserved(s, ixL, wLC);
    to_conserved(s, ixR, wRC);
    return 0;
  }
  if (s.c.limiter == ORC_LIM_WENO5 || s.c.limiter == ORC_LIM_WENOZ5 || s.c.limiter == ORC_LIM_WENOZP5) {
    // WENO5limiter then fix_limiter (src/limiter/mod_weno.t:100-133): any
    // flagged density or pressure keeps every variable of the face flat
    const int var = s.c.limiter == ORC_LIM_WENO5 ? 1 : (s.c.limiter == ORC_LIM_WENOZ5 ? 2 : 3);
    const R lambda = R(std::pow(dxdim, 2.0 / 3.0));
    forbox(ixL, [&](int i, int j, int k) {
      const size_t p = g.idx(i, j, k);
      R wl[16], wr[16];
      for (int iw = 0; iw < x.nw; ++iw) {
        const R *q = &w.d[p + g.cells * (size_t)iw];
        wl[iw] = weno5_side(q[-2 * o], q[-o], q[0], q[o], q[2 * o], var, lambda);
        wr[iw] = weno5_side(q[3 * o], q[2 * o], q[o], q[0], q[-o], var, lambda);
      }
      const bool flag = wl[x.rho] < R(s.c.small_density) || wr[x.rho] < R(s.c.small_density) ||
                        wl[x.e] < R(s.c.small_pressure) || wr[x.e] < R(s.c.small_pressure);
      if (flag) return;
      for (int iw = 0; iw < x.nw; ++iw) {
        wLp.d[p + g.cells * (size_t)iw] = wl[iw];
        wRp.d[p + g.cells * (size_t)iw] = wr[iw];
      }
    });
    for (int iw = 0; iw < x.nw; ++iw) {
      forbox(ixL, [&](int i, int j, int k) { wLC(i, j, k, iw) = wLp(i, j, k, iw); });
      forbox(ixR, [&](int i, int j, int k) { wRC(i, j, k, iw) = wRp(i, j, k, iw); });
    }
    to_conserved(s, ixL, wLC);
    to_conserved(s, ixR, wRC);
    return 0;
  }
  if (s.c.limiter == ORC_LIM_MP5) {
    // faces iL = ixL (ixR == ixL here: finite_volume's ixCR)
    forbox(ixL, [&](int i, int j, int k) {
      const size_t p = g.idx(i, j, k);
      R wl[16], wr[16];
      for (int iw = 0; iw < x.nw; ++iw) {
        const R *q = &w.d[p + g.cells * (size_t)iw];
        wl[iw] = mp5_side(q[-2 * o], q[-o], q[0], q[o], q[2 * o]);
        wr[iw] = mp5_side(q[3 * o], q[2 * o], q[o], q[0], q[-o]);
      }
      // fix_limiter1: phys_check_w flags (primitive) on both states
      const bool frho = wl[x.rho] < R(s.c.small_density) || wr[x.rho] < R(s.c.small_density);
      const bool fe = wl[x.e] < R(s.c.small_pressure) || wr[x.e] < R(s.c.small_pressure);
      for (int iw = 0; iw < x.nw; ++iw) {
        if ((iw == x.rho && frho) || (iw == x.e && fe)) continue;
        wLp.d[p + g.cells * (size_t)iw] = wl[iw];
        wRp.d[p + g.cells * (size_t)iw] = wr[iw];
      }
    });
    for (int iw = 0; iw < x.nw; ++iw) {
      forbox(ixL, [&](int i, int j, int k) { wLC(i, j, k, iw) = wLp(i, j, k, iw); });
      forbox(ixR, [&](int i, int j, int k) { wRC(i, j, k, iw) = wRp(i, j, k, iw); });
    }
    to_conserved(s, ixL, wLC);
    to_conserved(s, ixR, wRC);
    (void)dxdim;
    return 0;
  }
  Box jxR = shift(ixR, idims, 1);
  Box ixC;
  for (int d = 0; d < 3; ++d) { ixC.hi[d] = jxR.hi[d]; ixC.lo[d] = ixL.lo[d]; }
  ixC.lo[idims] -= 1;
  Arr<R> dwC(g, 1), ldw(g, 1), rdw(g, 1);
  for (int iw = 0; iw < x.nw; ++iw) {
    forbox(ixC, [&](int i, int j, int k) {
      const int p = g.idx(i, j, k);
      dwC.d[p] = w.d[p + o + g.cells * (size_t)iw] - w.d[p + g.cells * (size_t)iw];
    });
    dwlimiter2(s, dwC, ixC, idims, dxdim, ldw, rdw);
    forbox(ixL, [&](int i, int j, int k) {
      wLp(i, j, k, iw) = wLp(i, j, k, iw) + R(half) * ldw.d[g.idx(i, j, k)];
    });
    forbox(ixR, [&](int i, int j, int k) {
      wRp(i, j, k, iw) = wRp(i, j, k, iw) - R(half) * rdw.d[g.idx(i, j, k) + o];
    });
  }
  int st = 0;
  if (s.c.fix_small_values) {
    st |= handle_small_values(s, true, wLp, ixL);
    st |= handle_small_values(s, true, wRp, ixR);
  }
  for (int iw = 0; iw < x.nw; ++iw) {
    forbox(ixL, [&](int i, int j, int k) { wLC(i, j, k, iw) = wLp(i, j, k, iw); });
    forbox(ixR, [&](int i, int j, int k) { wRC(i, j, k, iw) = wRp(i, j, k, iw); });
  }
  to_conserved(s, ixL, wLC);
  to_conserved(s, ixR, wRC);
  return st;
}

// mhd_modify_wLR GLM branch (src/mhd/mod_mhd_phys.t:6326-6377)
template <class R>
void modify_wLR(const State &s, const Box &b, Arr<R> &wLC, Arr<R> &wRC, Arr<R> &wLp, Arr<R> &wRp,
                int idir, double cmax_global) {
  const Ix &x = s.x;
  const int bn = x.mag[idir], ps = x.psi, e = x.e;
  const R cg(cmax_global);
  forbox(b, [&](int i, int j, int k) {
    R dB = W(wRp, bn) - W(wLp, bn);
    R dPsi = W(wRp, ps) - W(wLp, ps);
    W(wLp, bn) = R(half) * (W(wRp, bn) + W(wLp, bn) - dPsi / cg);
    W(wLp, ps) = R(half) * (W(wRp, ps) + W(wLp, ps) - dB * cg);
    W(wRp, bn) = W(wLp, bn);
    W(wRp, ps) = W(wLp, ps);
    W(wRC, e) = W(wRC, e) - R(half) * (W(wRC, bn) * W(wRC, bn));
    W(wLC, e) = W(wLC, e) - R(half) * (W(wLC, bn) * W(wLC, bn));
    W(wRC, bn) = W(wLp, bn);
    W(wRC, ps) = W(wLp, ps);
    W(wLC, bn) = W(wLp, bn);
    W(wLC, ps) = W(wLp, ps);
    W(wRC, e) = W(wRC, e) + R(half) * (W(wRC, bn) * W(wRC, bn));
    W(wLC, e) = W(wLC, e) + R(half) * (W(wLC, bn) * W(wLC, bn));
  });
}

struct FaceBufs;

// get_Riemann_flux_hll (src/mod_finite_volume.t:381-437)
template <class R>
void riemann_hll(const State &s, const Box &b, int idims, const Arr<R> &wLC, const Arr<R> &wRC,
                 const Arr<R> &fLC, const Arr<R> &fRC, const Arr<R> &cmaxC, const Arr<R> &cminC,
                 Arr<R> &fC) {
  const Ix &x = s.x;
  for (int iw = 0; iw < x.nw; ++iw) {
    if (flux_type(s.c, x, idims, iw) == FT_TVDLF) {
      forbox(b, [&](int i, int j, int k) {
        W(fC, iw) = -(R(s.c.tvdlfeps) * R(half) * rmax(cmaxC(i, j, k, 0), rabs(cminC(i, j, k, 0)))) *
                    (W(wRC, iw) - W(wLC, iw));
      });
      continue;
    }
    forbox(b, [&](int i, int j, int k) {
      R cmin = cminC(i, j, k, 0), cmax = cmaxC(i, j, k, 0);
      if (cmin >= R(zero)) W(fC, iw) = W(fLC, iw);
      else if (cmax <= R(zero)) W(fC, iw) = W(fRC, iw);
      else
        W(fC, iw) = (cmax * W(fLC, iw) - cmin * W(fRC, iw) + cmin * cmax * (W(wRC, iw) - W(wLC, iw))) /
                    (cmax - cmin);
    });
  }
}

// get_Riemann_flux_tvdlf (src/mod_finite_volume.t:348-379)
template <class R>
void riemann_tvdlf(const State &s, const Box &b, int idims, const Arr<R> &wLC, const Arr<R> &wRC,
                   const Arr<R> &fLC, const Arr<R> &fRC, const Arr<R> &cmaxC, Arr<R> &fC) {
  const Ix &x = s.x;
  for (int iw = 0; iw < x.nw; ++iw) {
    forbox(b, [&](int i, int j, int k) {
      R fac = -(R(0.5) * R(s.c.tvdlfeps) * cmaxC(i, j, k, 0));
      W(fC, iw) = R(0.5) * (W(fLC, iw) + W(fRC, iw));
      W(fC, iw) = W(fC, iw) + fac * (W(wRC, iw) - W(wLC, iw));
    });
  }
}

// get_Riemann_flux_hllc (src/mod_finite_volume.t:439-504) with hd_get_lCD and
// hd_get_wCD (src/hd/mod_hd_hllc.t:56-257), or mhd_get_lCD and mhd_get_wCD
// (src/mhd/mod_mhd_hllc.t:56-241) for MHD.
template <class R>
void riemann_hllc(const State &s, const Box &b, int idims, const Arr<R> &wLC, const Arr<R> &wRC,
                  Arr<R> &fLC, const Arr<R> &fRC, const Arr<R> &cmaxC, const Arr<R> &cminC,
                  Arr<R> &fC) {
  const Ix &x = s.x;
  const int nw = x.nw, mn = x.mom[idims];
  forbox(b, [&](int i, int j, int k) {
    R cmin = cminC(i, j, k, 0), cmax = cmaxC(i, j, k, 0);
    int patchf = 1;
    if (cmin >= R(zero)) patchf = -2;
    else if (cmax <= R(zero)) patchf = 2;
    R whll[16], Fhll[16], fCD[16];
    R lambdaCD(0.0);
    if (patchf == 1) {
      for (int iw = 0; iw < nw; ++iw) {
        Fhll[iw] = (cmax * W(fLC, iw) - cmin * W(fRC, iw) + cmin * cmax * (W(wRC, iw) - W(wLC, iw))) /
                   (cmax - cmin);
        whll[iw] = (cmax * W(wRC, iw) - cmin * W(wLC, iw) + W(fLC, iw) - W(fRC, iw)) / (cmax - cmin);
      }
      lambdaCD = whll[mn] / whll[x.rho];
      bool cond = true;
      if (cmin < R(zero) && lambdaCD > R(zero) && lambdaCD < cmax) patchf = -1;
      else if (cmax > R(zero) && lambdaCD < R(zero) && lambdaCD > cmin) patchf = 1;
      else if (lambdaCD >= cmax || lambdaCD <= cmin) { lambdaCD = R(zero); patchf = 3; }
      if (patchf == 3) cond = false;
      if (cond && lambdaCD == R(zero)) patchf = (-cmin >= cmax) ? 1 : -1;
    }
    if (patchf == 1 || patchf == -1) {
      R cspeed, vSub;
      const Arr<R> *wSub, *fSub;
      if (patchf == 1) { cspeed = cmax; vSub = W(wRC, mn) / W(wRC, x.rho); wSub = &wRC; fSub = &fRC; }
      else { cspeed = cmin; vSub = W(wLC, mn) / W(wLC, x.rho); wSub = &wLC; fSub = &fLC; }
      if (x.mhd) {
        // mhd_get_wCD: the star state keeps the HLL magnetic field (Li 2005)
        const R den = cspeed - lambdaCD;
        const int bn = x.mag[idims];
        R wCD[16];
        wCD[x.rho] = (*wSub)(i, j, k, x.rho) * (cspeed - vSub) / den;
        for (int c = 0; c < x.ndir; ++c) wCD[x.mag[c]] = whll[x.mag[c]];
        for (int c = 0; c < x.ndir; ++c) {
          if (c != idims)
            wCD[x.mom[c]] = (cspeed * (*wSub)(i, j, k, x.mom[c]) - (*fSub)(i, j, k, x.mom[c]) -
                             wCD[bn] * wCD[x.mag[c]]) / den;
          else
            wCD[x.mom[c]] = wCD[x.rho] * lambdaCD;
        }
        R vdb = whll[x.mom[0]] * whll[x.mag[0]];
        for (int c = 1; c < x.ndir; ++c) vdb = vdb + whll[x.mom[c]] * whll[x.mag[c]];
        vdb = vdb / whll[x.rho];
        R pCD = (*wSub)(i, j, k, x.rho) * (cspeed - vSub) * (lambdaCD - vSub) + (*fSub)(i, j, k, mn) -
                (*wSub)(i, j, k, mn) * vSub + wCD[bn] * wCD[bn];
        wCD[x.e] = (cspeed * (*wSub)(i, j, k, x.e) - (*fSub)(i, j, k, x.e) + lambdaCD * pCD - vdb * wCD[bn]) / den;
        for (int iw = 0; iw < nw; ++iw) {
          if (iw == bn || (x.glm && iw == x.psi)) fCD[iw] = R(zero);
          else fCD[iw] = (*fSub)(i, j, k, iw) + cspeed * (wCD[iw] - (*wSub)(i, j, k, iw));
        }
      } else {
      R csmls = R(one) / (cspeed - lambdaCD);
      R wCD[8];
      wCD[x.rho] = (*wSub)(i, j, k, x.rho) * (cspeed - vSub) * csmls;
      for (int c = 0; c < x.ndir; ++c) {
        if (c != idims)
          wCD[x.mom[c]] = (cspeed * (*wSub)(i, j, k, x.mom[c]) - (*fSub)(i, j, k, x.mom[c])) * csmls;
        else
          wCD[x.mom[c]] = wCD[x.rho] * lambdaCD;
      }
      R pCD = (*wSub)(i, j, k, x.rho) * (cspeed - vSub) * (lambdaCD - vSub) + (*fSub)(i, j, k, mn) -
              (*wSub)(i, j, k, mn) * vSub;
      wCD[x.e] = (cspeed * (*wSub)(i, j, k, x.e) - (*fSub)(i, j, k, x.e) + lambdaCD * pCD) * csmls;
      for (int iw = 0; iw < nw; ++iw)
        fCD[iw] = (*fSub)(i, j, k, iw) + cspeed * (wCD[iw] - (*wSub)(i, j, k, iw));
      }
    }
    for (int iw = 0; iw < nw; ++iw) {
      R out = W(fLC, iw);
      if (flux_type(s.c, x, idims, iw) == FT_TVDLF)
        out = -(R(s.c.tvdlfeps) * R(half) * rmax(cmax, rabs(cmin))) * (W(wRC, iw) - W(wLC, iw));
      else if (patchf == -2) out = W(fLC, iw);
      else if (patchf == 1 || patchf == -1) out = fCD[iw];
      else if (patchf == 2) out = W(fRC, iw);
      else if (patchf == 3) out = Fhll[iw];
      W(fC, iw) = out;
    }
  });
}

// get_Riemann_flux_hlld (src/mod_finite_volume.t:507-729), no B0/equi split.
template <class R>
void riemann_hlld(const State &s, const Box &b, int idims, const Arr<R> &wLC, const Arr<R> &wRC,
                  const Arr<R> &wLp, const Arr<R> &wRp, const Arr<R> &fLC, const Arr<R> &fRC,
                  const Arr<R> &cmaxC, const Arr<R> &cminC, Arr<R> &fC) {
  const Ix &x = s.x;
  const int nw = x.nw, ndir = x.ndir;
  const int ip1 = idims;                 // 0-based
  int ip2 = (idims + 1) % ndir;          // mod(ip1+1,ndir) (1-based) -> 0-based
  int ip3 = (idims + 2) % ndir;
  const int rho = x.rho, e = x.e;
  forbox(b, [&](int i, int j, int k) {
    R sR = cmaxC(i, j, k, 0), sL = cminC(i, j, k, 0);
    R BR[3], BL[3];
    for (int c = 0; c < ndir; ++c) { BR[c] = W(wRC, x.mag[c]); BL[c] = W(wLC, x.mag[c]); }
    R Bx = (sR * BR[ip1] - sL * BL[ip1]) / (sR - sL);
    R w1R[10], w1L[10], w2R[10], w2L[10];
    for (int q = 0; q < 10; ++q) { w1R[q] = w1L[q] = w2R[q] = w2L[q] = R(0.0); }
    R bR2 = BR[0] * BR[0], bL2 = BL[0] * BL[0];
    for (int c = 1; c < ndir; ++c) { bR2 = bR2 + BR[c] * BR[c]; bL2 = bL2 + BL[c] * BL[c]; }
    R ptR = W(wRp, x.e) + R(0.5) * bR2;
    R ptL = W(wLp, x.e) + R(0.5) * bL2;
    const int m1 = x.mom[ip1];
    R suR = (sR - W(wRp, m1)) * W(wRC, rho);
    R suL = (sL - W(wLp, m1)) * W(wLC, rho);
    R sm = (suR * W(wRp, m1) - suL * W(wLp, m1) - ptR + ptL) / (suR - suL);
    w1R[m1] = sm; w1L[m1] = sm; w2R[m1] = sm; w2L[m1] = sm;
    w1R[x.mag[ip1]] = Bx; w1L[x.mag[ip1]] = Bx;
    w1R[rho] = suR / (sR - sm);
    w1L[rho] = suL / (sL - sm);
    R r1R = suR * (sR - sm) - Bx * Bx;
    if (r1R != R(0.0)) r1R = R(1.0) / r1R;
    R r1L = suL * (sL - sm) - Bx * Bx;
    if (r1L != R(0.0)) r1L = R(1.0) / r1L;
    const int m2 = x.mom[ip2], b2 = x.mag[ip2];
    w1R[m2] = W(wRp, m2) - Bx * BR[ip2] * (sm - W(wRp, m1)) * r1R;
    w1L[m2] = W(wLp, m2) - Bx * BL[ip2] * (sm - W(wLp, m1)) * r1L;
    w1R[b2] = (suR * (sR - W(wRp, m1)) - Bx * Bx) * r1R;
    w1L[b2] = (suL * (sL - W(wLp, m1)) - Bx * Bx) * r1L;
    if (ndir == 3) {
      const int m3 = x.mom[ip3], b3 = x.mag[ip3];
      w1R[m3] = W(wRp, m3) - Bx * BR[ip3] * (sm - W(wRp, m1)) * r1R;
      w1L[m3] = W(wLp, m3) - Bx * BL[ip3] * (sm - W(wLp, m1)) * r1L;
      w1R[b3] = BR[ip3] * w1R[b2];
      w1L[b3] = BL[ip3] * w1L[b2];
    }
    w1R[b2] = BR[ip2] * w1R[b2];
    w1L[b2] = BL[ip2] * w1L[b2];
    // energy (p_ == e_)
    w1R[e] = suR * (sm - W(wRp, m1)) + ptR;
    w1L[e] = w1R[e];
    {
      R vbR = W(wRp, x.mom[0]) * W(wRC, x.mag[0]);
      R vbL = W(wLp, x.mom[0]) * W(wLC, x.mag[0]);
      R v1bR = w1R[x.mom[0]] * w1R[x.mag[0]];
      R v1bL = w1L[x.mom[0]] * w1L[x.mag[0]];
      for (int c = 1; c < ndir; ++c) {
        vbR = vbR + W(wRp, x.mom[c]) * W(wRC, x.mag[c]);
        vbL = vbL + W(wLp, x.mom[c]) * W(wLC, x.mag[c]);
        v1bR = v1bR + w1R[x.mom[c]] * w1R[x.mag[c]];
        v1bL = v1bL + w1L[x.mom[c]] * w1L[x.mag[c]];
      }
      R pR = w1R[e], pL = w1L[e];
      w1R[e] = ((sR - W(wRp, m1)) * W(wRC, e) - ptR * W(wRp, m1) + pR * sm + Bx * (vbR - v1bR)) / (sR - sm);
      w1L[e] = ((sL - W(wLp, m1)) * W(wLC, e) - ptL * W(wLp, m1) + pL * sm + Bx * (vbL - v1bL)) / (sL - sm);
    }
    w2R[rho] = w1R[rho]; w2L[rho] = w1L[rho];
    w2R[x.mag[ip1]] = w1R[x.mag[ip1]]; w2L[x.mag[ip1]] = w1L[x.mag[ip1]];
    r1R = rsqrt_(w1R[rho]);
    r1L = rsqrt_(w1L[rho]);
    R tmp = R(1.0) / (r1R + r1L);
    R signBx = rsign(1.0, Bx);
    R s1R = sm + rabs(Bx) / r1R;
    R s1L = sm - rabs(Bx) / r1L;
    w2R[m2] = (r1L * w1L[m2] + r1R * w1R[m2] + (w1R[b2] - w1L[b2]) * signBx) * tmp;
    w2L[m2] = w2R[m2];
    w2R[b2] = (r1L * w1R[b2] + r1R * w1L[b2] + r1L * r1R * (w1R[m2] - w1L[m2]) * signBx) * tmp;
    w2L[b2] = w2R[b2];
    if (ndir == 3) {
      const int m3 = x.mom[ip3], b3 = x.mag[ip3];
      w2R[m3] = (r1L * w1L[m3] + r1R * w1R[m3] + (w1R[b3] - w1L[b3]) * signBx) * tmp;
      w2L[m3] = w2R[m3];
      w2R[b3] = (r1L * w1R[b3] + r1R * w1L[b3] + r1L * r1R * (w1R[m3] - w1L[m3]) * signBx) * tmp;
      w2L[b3] = w2R[b3];
    }
    {
      R a1R = w1R[x.mom[0]] * w1R[x.mag[0]], a2R = w2R[x.mom[0]] * w2R[x.mag[0]];
      R a1L = w1L[x.mom[0]] * w1L[x.mag[0]], a2L = w2L[x.mom[0]] * w2L[x.mag[0]];
      for (int c = 1; c < ndir; ++c) {
        a1R = a1R + w1R[x.mom[c]] * w1R[x.mag[c]];
        a2R = a2R + w2R[x.mom[c]] * w2R[x.mag[c]];
        a1L = a1L + w1L[x.mom[c]] * w1L[x.mag[c]];
        a2L = a2L + w2L[x.mom[c]] * w2L[x.mag[c]];
      }
      w2R[e] = w1R[e] + r1R * (a1R - a2R) * signBx;
      w2L[e] = w1L[e] - r1L * (a1L - a2L) * signBx;
    }
    for (int c = 0; c < ndir; ++c) {
      const int m = x.mom[c];
      w1R[m] = w1R[m] * w1R[rho];
      w1L[m] = w1L[m] * w1L[rho];
      w2R[m] = w2R[m] * w2R[rho];
      w2L[m] = w2L[m] * w2L[rho];
    }
    for (int iw = 0; iw < nw; ++iw) {
      int ft = flux_type(s.c, x, idims, iw);
      if (ft == FT_SPECIAL) {
        W(fC, iw) = W(fLC, iw);
      } else {
        R out = W(fC, iw);
        if (sL > R(0.0)) out = W(fLC, iw);
        else if (s1L >= R(0.0)) out = W(fLC, iw) + sL * (w1L[iw] - W(wLC, iw));
        else if (sm >= R(0.0)) out = W(fLC, iw) + sL * (w1L[iw] - W(wLC, iw)) + s1L * (w2L[iw] - w1L[iw]);
        else if (s1R >= R(0.0)) out = W(fRC, iw) + sR * (w1R[iw] - W(wRC, iw)) + s1R * (w2R[iw] - w1R[iw]);
        else if (sR >= R(0.0)) out = W(fRC, iw) + sR * (w1R[iw] - W(wRC, iw));
        else if (sR < R(0.0)) out = W(fRC, iw);
        W(fC, iw) = out;
      }
    }
  });
}

// gradient, Cartesian nth=1 (src/mod_geometry.t:329-394)
template <class R>
void gradient(const State &s, const Arr<R> &q, int iq, const Box &ixO, int idir, double dxlevel,
              std::vector<R> &gradq) {
  const int o = s.g.off(idir);
  forbox(ixO, [&](int i, int j, int k) {
    const int p = s.g.idx(i, j, k);
    const size_t vo = s.g.cells * (size_t)iq;
    R gq = (q.d[vo + p + o] - q.d[vo + p - o]) * R(half);
    gradq[p] = gq / R(dxlevel);
  });
}

// divvector on the magnetic field, slab_uniform, nth = 1 or 2
// (src/mod_geometry.t:582-651), as called by get_divb
// (src/physics/mod_functions_bfield.t:14-46).
template <class R>
void divb_central(const State &s, const Arr<R> &w, const Box &ixO, const double *dxlevel, int nth,
                  std::vector<R> &divq) {
  const Ix &x = s.x;
  R invdx[3];
  for (int d = 0; d < s.c.ndim; ++d) invdx[d] = R(1.0) / R(dxlevel[d]);
  forbox(ixO, [&](int i, int j, int k) { divq[s.g.idx(i, j, k)] = R(0.0); });
  for (int d = 0; d < s.c.ndim; ++d) {
    const int o = s.g.off(d);
    const size_t vo = s.g.cells * (size_t)x.mag[d];
    forbox(ixO, [&](int i, int j, int k) {
      const int p = s.g.idx(i, j, k);
      if (nth == 1) {
        divq[p] = divq[p] + R(half) * (w.d[vo + p + o] - w.d[vo + p - o]) * invdx[d];
      } else {
        divq[p] = divq[p] + (-w.d[vo + p + 2 * o] + R(8.0) * w.d[vo + p + o] - R(8.0) * w.d[vo + p - o] +
                             w.d[vo + p - 2 * o]) /
                                (R(12.0) * R(dxlevel[d]));
      }
    });
  }
}

// add_source_glm (src/mhd/mod_mhd_phys.t:5472-5531)
// Both divB sources end with the small-value fix of the updated state
// (src/mhd/mod_mhd_phys.t:5529, 5662); the status of that fix is returned.
template <class R>
int add_source_glm(const State &s, double qdt, const Box &ixI, const Box &ixO, const Arr<R> &wCT,
                   Arr<R> &w, const double *dxlevel, double cmax_global) {
  const Ix &x = s.x;
  const orc_cfg &c = s.c;
  double mindx = dxlevel[0];
  for (int d = 1; d < c.ndim; ++d) mindx = std::min(mindx, dxlevel[d]);
  if (c.glm_alpha < 0) {
    forbox(ixO, [&](int i, int j, int k) { W(w, x.psi) = R(std::fabs(c.glm_alpha)) * W(wCT, x.psi); });
  } else {
    R fac = rexp_(-(R(qdt) * R(cmax_global) * R(c.glm_alpha)) / R(mindx));
    forbox(ixO, [&](int i, int j, int k) { W(w, x.psi) = fac * W(w, x.psi); });
  }
  if (c.glm_extended) {
    std::vector<R> grad(s.g.cells), divb(s.g.cells);
    for (int d = 0; d < c.ndim; ++d) {
      gradient(s, wCT, x.psi, ixO, d, dxlevel[d], grad);
      forbox(ixO, [&](int i, int j, int k) {
        W(w, x.e) = W(w, x.e) - R(qdt) * W(wCT, x.mag[d]) * grad[s.g.idx(i, j, k)];
      });
    }
    divb_central(s, wCT, ixO, dxlevel, 1, divb);
    for (int d = 0; d < x.ndir; ++d) {
      forbox(ixO, [&](int i, int j, int k) {
        W(w, x.mom[d]) = W(w, x.mom[d]) - R(qdt) * W(wCT, x.mag[d]) * divb[s.g.idx(i, j, k)];
      });
    }
  }
  (void)ixI;
  return c.fix_small_values ? handle_small_values(s, false, w, ixO) : 0;
}

// add_source_linde (src/mhd/mod_mhd_phys.t:5599-5665).  jump_faces bit
// 2d+side marks a face with a coarser or finer neighbour: the source skips the
// cell layer next to it ("for AMR stability", 5616-5642).
template <class R>
int add_source_linde(const State &s, double qdt, const Box &ixO, const Arr<R> &wCT, Arr<R> &w,
                     const double *dxlevel, int jump_faces = 0) {
  const Ix &x = s.x;
  const orc_cfg &c = s.c;
  Box ixp = ixO;
  for (int d = 0; d < c.ndim; ++d) { ixp.lo[d] -= 1; ixp.hi[d] += 1; }
  std::vector<R> divb(s.g.cells), grad(s.g.cells);
  divb_central(s, wCT, ixp, dxlevel, 1, divb);
  R inv2(0.0);
  {
    R acc = R(1.0) / (R(dxlevel[0]) * R(dxlevel[0]));
    for (int d = 1; d < c.ndim; ++d) acc = acc + R(1.0) / (R(dxlevel[d]) * R(dxlevel[d]));
    inv2 = acc;
  }
  Box ixq = ixO;
  for (int d = 0; d < c.ndim; ++d) {
    if ((jump_faces >> (2 * d)) & 1) ixq.lo[d] += 1;
    if ((jump_faces >> (2 * d + 1)) & 1) ixq.hi[d] -= 1;
  }
  for (int d = 0; d < c.ndim; ++d) {
    const int o = s.g.off(d);
    forbox(ixq, [&](int i, int j, int k) {
      const int p = s.g.idx(i, j, k);
      R gq = (divb[p + o] - divb[p - o]) * R(half);
      gq = gq / R(dxlevel[d]);
      gq = gq * R(c.divbdiff) / inv2;
      W(w, x.mag[d]) = W(w, x.mag[d]) + gq;
      W(w, x.e) = W(w, x.e) + W(wCT, x.mag[d]) * gq;
    });
  }
  (void)qdt;
  return c.fix_small_values ? handle_small_values(s, false, w, ixO) : 0;
}

// tvdlimit2 (src/mod_tvd.t:38-112) for fs_tvdmu with hydrodynamics: the Roe
// average hd_average, the waves of geteigenjump2 and the right eigenvectors
// of rtimes2 (src/hd/mod_hd_roe.t:58-296), typeentropy 'nul', getphi's
// tvdmu branch phi = |a qdt/dx| jump; each characteristic adds
// rphi = R phi / 2 to the scaled face flux and rphi(i) - rphi(i-1) to wnew.
template <class R>
void tvdlimit2_hd(const State &s, double qdt, const Box &ixO, int idims, const Arr<R> &wL, const Arr<R> &wR,
                  Arr<R> &wnew, Arr<R> &fC, const double *dxs) {
  const Ix &x = s.x;
  const Geo &g = s.g;
  const int nw = x.nw, ndir = x.ndir, o = g.off(idims);
  const double gam = s.c.gamma;
  Box ixC = ixO;
  ixC.lo[idims] -= 1;
  Arr<R> wroe(g, nw), csound(g, 1), dpperc2(g, 1), dvperc(g, 1), a(g, 1), jump(g, 1), phi(g, 1), rphi(g, 1);
  auto pth = [&](const Arr<R> &w, int i, int j, int k) {  // hd_get_pthermal
    R m2 = W(w, x.mom[0]) * W(w, x.mom[0]);
    for (int c = 1; c < ndir; ++c) m2 = m2 + W(w, x.mom[c]) * W(w, x.mom[c]);
    R p = R(gam - 1.0) * (W(w, x.e) - R(0.5) * m2 / W(w, x.rho));
    if (s.c.fix_small_values && p < R(s.c.small_pressure)) p = R(s.c.small_pressure);
    return p;
  };
  // hd_average
  forbox(ixC, [&](int i, int j, int k) {
    R w1 = rsqrt_(W(wL, x.rho)), w2 = rsqrt_(W(wR, x.rho));
    W(wroe, x.rho) = w1 * w2;
    w1 = w1 / w2;
    for (int c = 0; c < ndir; ++c)
      W(wroe, x.mom[c]) = (W(wL, x.mom[c]) / W(wL, x.rho) * w1 + W(wR, x.mom[c]) / W(wR, x.rho)) / (R(one) + w1);
    W(wroe, x.e) = (pth(wL, i, j, k) + W(wL, x.e)) / W(wL, x.rho);
    R t2 = (pth(wR, i, j, k) + W(wR, x.e)) / W(wR, x.rho);
    W(wroe, x.e) = (W(wroe, x.e) * w1 + t2) / (R(one) + w1);
  });
  const double dxinv = qdt / dxs[idims];
  const int soundR = 0, soundL = 1, entrop = 2;  // il - 1; shear waves from 3
  for (int il = 0; il < nw; ++il) {
    // geteigenjump2
    forbox(ixC, [&](int i, int j, int k) {
      const int p = g.idx(i, j, k);
      if (il == 0) {
        R v2 = W(wroe, x.mom[0]) * W(wroe, x.mom[0]);
        for (int c = 1; c < ndir; ++c) v2 = v2 + W(wroe, x.mom[c]) * W(wroe, x.mom[c]);
        R kin = R(0.5) * v2;
        R c2 = R(gam - 1.0) * (W(wroe, x.e) - kin);
        c2 = rmax(R(gam * 1.0e-12) / W(wroe, x.rho), c2);  // smalldouble
        dpperc2.d[p] = (pth(wR, i, j, k) - pth(wL, i, j, k)) / c2;
        csound.d[p] = rsqrt_(c2);
        dvperc.d[p] = (W(wR, x.mom[idims]) / W(wR, x.rho) - W(wL, x.mom[idims]) / W(wL, x.rho)) / csound.d[p];
      }
      const R u = W(wroe, x.mom[idims]);
      if (il == soundR) {
        a.d[p] = u + csound.d[p];
        jump.d[p] = R(half) * (dpperc2.d[p] + W(wroe, x.rho) * dvperc.d[p]);
      } else if (il == soundL) {
        a.d[p] = u - csound.d[p];
        jump.d[p] = R(half) * (dpperc2.d[p] - W(wroe, x.rho) * dvperc.d[p]);
      } else if (il == entrop) {
        a.d[p] = u;
        jump.d[p] = -dpperc2.d[p] + W(wR, x.rho) - W(wL, x.rho);
      } else {
        int idir = il - 3;
        if (idir >= idims) idir += 1;
        a.d[p] = u;
        jump.d[p] = W(wroe, x.rho) * (W(wR, x.mom[idir]) / W(wR, x.rho) - W(wL, x.mom[idir]) / W(wL, x.rho));
      }
      phi.d[p] = rabs(a.d[p] * R(dxinv)) * jump.d[p];  // getphi, tvdmu, typeentropy 'nul'
    });
    const bool shear = il > entrop;
    int sdir = idims;
    if (shear) { sdir = il - 3; if (sdir >= idims) sdir += 1; }
    for (int iw = 0; iw < nw; ++iw) {
      // rtimes2
      forbox(ixC, [&](int i, int j, int k) {
        const int p = g.idx(i, j, k);
        const R q = phi.d[p];
        R rq;
        if (iw == x.rho) {
          rq = shear ? R(zero) : q;
        } else if (iw == x.e) {
          if (il == soundR) rq = q * (W(wroe, x.e) + W(wroe, x.mom[idims]) * csound.d[p]);
          else if (il == soundL) rq = q * (W(wroe, x.e) - W(wroe, x.mom[idims]) * csound.d[p]);
          else if (il == entrop) {
            R v2 = W(wroe, x.mom[0]) * W(wroe, x.mom[0]);
            for (int c = 1; c < ndir; ++c) v2 = v2 + W(wroe, x.mom[c]) * W(wroe, x.mom[c]);
            rq = q * R(0.5) * v2;
          } else rq = q * W(wroe, x.mom[sdir]);
        } else if (iw == x.mom[idims]) {
          if (il == soundR) rq = q * (W(wroe, x.mom[idims]) + csound.d[p]);
          else if (il == soundL) rq = q * (W(wroe, x.mom[idims]) - csound.d[p]);
          else if (il == entrop) rq = q * W(wroe, x.mom[idims]);
          else rq = R(zero);
        } else {
          if (shear) rq = (iw == x.mom[sdir]) ? q : R(zero);
          else rq = q * W(wroe, iw);
        }
        rphi.d[p] = rq * R(half);
        W(fC, iw) = W(fC, iw) + rphi.d[p];
      });
      forbox(ixO, [&](int i, int j, int k) {
        const int p = g.idx(i, j, k);
        W(wnew, iw) = W(wnew, iw) + rphi.d[p] - rphi.d[p - o];
      });
    }
  }
}

// tvdlimit2 for MHD without GLM (src/mod_tvd.t:38-112) with the Roe system
// of src/mhd/mod_mhd_roe.t: average2 (61-146), geteigenjump2 (160-342),
// rtimes2 (355-506); divbwave on, typeentropy 'nul'; characteristic fields
// il = 1..nwflux with alfvRW 1, alfvLW 2, fastRW 3, fastLW 4, slowRW 5,
// slowLW 6, diverW 7, entroW 8 (ndir 2: nwflux 6, the last two never
// enter).  idir = idim+1-ndir*(idim/ndir), jdir likewise from idir (1-based).
template <class R>
void tvdlimit2_mhd(const State &s, double qdt, const Box &ixO, int idims, const Arr<R> &wL, const Arr<R> &wR,
                   Arr<R> &wnew, Arr<R> &fC, const double *dxs) {
  const Ix &x = s.x;
  const Geo &g = s.g;
  const int nw = x.nw, ndir = x.ndir, o = g.off(idims);
  const double gam = s.c.gamma;
  const double smalld = 1.0e-12;
  // 1-based direction rule of the reference, back to 0-based
  const int idim1 = idims + 1;
  const int idir1 = idim1 + 1 - ndir * (idim1 / ndir), jdir1 = idir1 + 1 - ndir * (idir1 / ndir);
  const int idir = idir1 - 1, jdir = jdir1 - 1;
  Box ixC = ixO;
  ixC.lo[idims] -= 1;
  struct Roe { R rho, v[3], b[3], cs2, cf, cl, af, as, dp, rhodv, bdv, bdb, bv, v2a2; };
  std::vector<Roe> roe(g.cells);
  auto pth = [&](const Arr<R> &w, int i, int j, int k) {
    R m2 = W(w, x.mom[0]) * W(w, x.mom[0]), b2 = W(w, x.mag[0]) * W(w, x.mag[0]);
    for (int c = 1; c < ndir; ++c) {
      m2 = m2 + W(w, x.mom[c]) * W(w, x.mom[c]);
      b2 = b2 + W(w, x.mag[c]) * W(w, x.mag[c]);
    }
    R p = R(gam - 1.0) * (W(w, x.e) - R(half) * (m2 / W(w, x.rho) + b2));
    if (s.c.fix_small_values && p < R(s.c.small_pressure)) p = R(s.c.small_pressure);
    return p;
  };
  forbox(ixC, [&](int i, int j, int k) {  // average2
    Roe &r = roe[g.idx(i, j, k)];
    r.rho = R(half) * (W(wL, x.rho) + W(wR, x.rho));
    for (int c = 0; c < ndir; ++c) {
      r.v[c] = R(half) * (W(wL, x.mom[c]) / W(wL, x.rho) + W(wR, x.mom[c]) / W(wR, x.rho));
      r.b[c] = R(half) * (W(wL, x.mag[c]) + W(wR, x.mag[c]));
    }
    const R pL = pth(wL, i, j, k), pR = pth(wR, i, j, k);
    const R pav = R(half) * (pL + pR);
    r.dp = pR - pL;
    r.rhodv = W(wR, x.mom[idims]) - W(wL, x.mom[idims]) - r.v[idims] * (W(wR, x.rho) - W(wL, x.rho));
    r.cs2 = R(gam) * pav / r.rho;
    R bb = r.b[0] * r.b[0];
    for (int c = 1; c < ndir; ++c) bb = bb + r.b[c] * r.b[c];
    r.cf = bb / r.rho + r.cs2;
    r.cl = R(half) * (r.cf - rsqrt_(r.cf * r.cf - R(4.0) * r.cs2 * (r.b[idims] * r.b[idims]) / r.rho));
    r.cf = r.cf - r.cl;
    r.af = (r.cs2 - r.cl) / (r.cf - r.cl);
    r.af = rmin(R(one), rmax(r.af, R(zero)));
    r.as = rsqrt_(R(one) - r.af);
    r.af = rsqrt_(r.af);
    r.cf = rsqrt_(r.cf);
    r.cl = rsqrt_(r.cl);
    r.rho = rsqrt_(r.rho);
    if (rabs(r.b[idims]) < R(smalld)) r.b[idims] = R(smalld);
    if (ndir == 2) {
      r.b[idir] = r.b[idir] >= R(zero) ? R(one) : R(-1.0);
    } else {
      R t = rsqrt_(r.b[idir] * r.b[idir] + r.b[jdir] * r.b[jdir]);
      if (t > R(smalld)) { r.b[idir] = r.b[idir] / t; r.b[jdir] = r.b[jdir] / t; }
      else { r.b[idir] = rsqrt_(R(half)); r.b[jdir] = rsqrt_(R(half)); }
    }
  });
  const double dxinv = qdt / dxs[idims];
  Arr<R> phi(g, 1), rphi(g, 1);
  auto dvel = [&](int i, int j, int k, int c) {
    return W(wR, x.mom[c]) / W(wR, x.rho) - W(wL, x.mom[c]) / W(wL, x.rho);
  };
  auto dmag = [&](int i, int j, int k, int c) { return W(wR, x.mag[c]) - W(wL, x.mag[c]); };
  for (int il = 1; il <= nw; ++il) {
    if (il > 8) break;
    // geteigenjump2
    forbox(ixC, [&](int i, int j, int k) {
      Roe &r = roe[g.idx(i, j, k)];
      if (il == 3) {  // fastRW_
        r.bdv = r.b[idir] * dvel(i, j, k, idir);
        if (ndir == 3) r.bdv = r.bdv + r.b[jdir] * dvel(i, j, k, jdir);
        r.bdv = r.bdv * rsign(val(r.rho * r.rho), r.b[idims]);
        r.bdb = r.b[idir] * dmag(i, j, k, idir);
        if (ndir == 3) r.bdb = r.bdb + r.b[jdir] * dmag(i, j, k, jdir);
        r.bdb = r.bdb * rsqrt_(r.cs2) * r.rho;
      }
      if (il == 1) {  // alfvRW_
        r.bdv = r.b[jdir] * dvel(i, j, k, idir) - r.b[idir] * dvel(i, j, k, jdir);
        r.bdb = r.b[jdir] * dmag(i, j, k, idir) - r.b[idir] * dmag(i, j, k, jdir);
        r.bdv = r.bdv * R(half) * (r.rho * r.rho);
        r.bdb = r.bdb * R(half) * rsign(val(r.rho), r.b[idims]);
      }
      const R u = r.v[idims], h = R(half) / r.cs2;
      R a, jump;
      switch (il) {
        case 3: a = u + r.cf; jump = h * (r.af * (r.cf * r.rhodv + r.dp) + r.as * (-r.cl * r.bdv + r.bdb)); break;
        case 4: a = u - r.cf; jump = h * (r.af * (-r.cf * r.rhodv + r.dp) + r.as * (r.cl * r.bdv + r.bdb)); break;
        case 5: a = u + r.cl; jump = h * (r.as * (r.cl * r.rhodv + r.dp) + r.af * (r.cf * r.bdv - r.bdb)); break;
        case 6: a = u - r.cl; jump = h * (r.as * (-r.cl * r.rhodv + r.dp) + r.af * (-r.cf * r.bdv - r.bdb)); break;
        case 8: a = u; jump = W(wR, x.rho) - W(wL, x.rho) - r.dp / r.cs2; break;
        case 7: a = u; jump = dmag(i, j, k, idims); break;
        case 1: a = u + rabs(r.b[idims]) / r.rho; jump = r.bdv - r.bdb; break;
        default: a = u - rabs(r.b[idims]) / r.rho; jump = -r.bdv - r.bdb; break;
      }
      phi.d[g.idx(i, j, k)] = rabs(a * R(dxinv)) * jump;
    });
    for (int iw = 0; iw < nw; ++iw) {
      forbox(ixC, [&](int i, int j, int k) {  // rtimes2
        Roe &r = roe[g.idx(i, j, k)];
        const R q = phi.d[g.idx(i, j, k)];
        const R u = r.v[idims];
        R rq(0.0);
        if (iw == x.rho) {
          if (il == 3 || il == 4) rq = q * r.af;
          else if (il == 5 || il == 6) rq = q * r.as;
          else if (il == 8) rq = q;
        } else if (iw == x.e) {
          if (il == 3) {
            R v2 = r.v[0] * r.v[0];
            for (int c = 1; c < ndir; ++c) v2 = v2 + r.v[c] * r.v[c];
            r.v2a2 = R(half) * v2 + R((2.0 - gam) / (gam - 1.0)) * r.cs2;
            r.bv = r.b[idir] * r.v[idir];
            if (ndir == 3) r.bv = r.bv + r.b[jdir] * r.v[jdir];
            r.bv = r.bv * rsign(one, r.b[idims]);
          } else if (il == 1) {
            r.bv = r.b[jdir] * r.v[idir] - r.b[idir] * r.v[jdir];
          }
          switch (il) {
            case 3: rq = q * (-r.as * r.cl * r.bv + r.af * (r.v2a2 + r.cf * (r.cf + u))); break;
            case 4: rq = q * (r.as * r.cl * r.bv + r.af * (r.v2a2 + r.cf * (r.cf - u))); break;
            case 5: rq = q * (r.af * r.cf * r.bv + r.as * (r.v2a2 + r.cl * (r.cl + u))); break;
            case 6: rq = q * (-r.af * r.cf * r.bv + r.as * (r.v2a2 + r.cl * (r.cl - u))); break;
            case 8: {
              R v2 = r.v[0] * r.v[0];
              for (int c = 1; c < ndir; ++c) v2 = v2 + r.v[c] * r.v[c];
              rq = q * R(half) * v2;
              break;
            }
            case 7: rq = q * r.b[idims]; break;
            case 1: rq = q * r.bv; break;
            default: rq = -q * r.bv; break;
          }
        } else if (iw >= x.mom[0] && iw < x.mom[0] + ndir) {
          const int c = iw - x.mom[0];
          if (c == idims) {
            switch (il) {
              case 3: rq = q * r.af * (r.v[c] + r.cf); break;
              case 4: rq = q * r.af * (r.v[c] - r.cf); break;
              case 5: rq = q * r.as * (r.v[c] + r.cl); break;
              case 6: rq = q * r.as * (r.v[c] - r.cl); break;
              case 8: rq = q * r.v[c]; break;
              default: break;
            }
          } else {
            const R sg = rsign(one, r.b[idims]);
            switch (il) {
              case 3: rq = q * (r.af * r.v[c] - r.as * r.cl * r.b[c] * sg); break;
              case 4: rq = q * (r.af * r.v[c] + r.as * r.cl * r.b[c] * sg); break;
              case 5: rq = q * (r.as * r.v[c] + r.af * r.cf * r.b[c] * sg); break;
              case 6: rq = q * (r.as * r.v[c] - r.af * r.cf * r.b[c] * sg); break;
              case 8: rq = q * r.v[c]; break;
              case 7: break;
              case 1: rq = c == idir ? q * r.b[jdir] : -q * r.b[idir]; break;
              default: rq = c == idir ? -q * r.b[jdir] : q * r.b[idir]; break;
            }
          }
        } else {  // magnetic field
          const int c = iw - x.mag[0];
          if (c == idims) {
            if (il == 7) rq = q;
          } else {
            switch (il) {
              case 3: case 4: rq = q * r.as * rsqrt_(r.cs2) * r.b[c] / r.rho; break;
              case 5: case 6: rq = -q * r.af * rsqrt_(r.cs2) * r.b[c] / r.rho; break;
              case 1: case 2:
                rq = c == idir ? -q * r.b[jdir] / rsign(val(r.rho), r.b[idims])
                               : q * r.b[idir] / rsign(val(r.rho), r.b[idims]);
                break;
              default: break;
            }
          }
        }
        rphi.d[g.idx(i, j, k)] = rq * R(half);
        W(fC, iw) = W(fC, iw) + rphi.d[g.idx(i, j, k)];
      });
      forbox(ixO, [&](int i, int j, int k) {
        const int p = g.idx(i, j, k);
        W(wnew, iw) = W(wnew, iw) + rphi.d[p] - rphi.d[p - o];
      });
    }
  }
}

// finite_volume (src/mod_finite_volume.t:116-339), slab_uniform, no local dt.
template <class R>
int finite_volume(const State &s, const Arr<R> &wCT, Arr<R> &wnew, double qdt, double dtfactor,
                  const double *dxs, double cmax_global, std::vector<Arr<R>> *keep_fc = nullptr,
                  int jump_faces = 0) {
  const Ix &x = s.x;
  const orc_cfg &c = s.c;
  const Geo &g = s.g;
  const int nw = x.nw, ndim = c.ndim;
  Box ixI = g.ixG(), ixO = g.ixM();
  int st = 0;
  Arr<R> wprim = wCT;
  st |= to_primitive(s, ixI, wprim);
  Arr<R> wLp(g, nw), wRp(g, nw), wLC(g, nw), wRC(g, nw), fLC(g, nw), fRC(g, nw);
  Arr<R> cmaxC(g, 1), cminC(g, 1);
  std::vector<Arr<R>> fC;
  for (int d = 0; d < ndim; ++d) fC.emplace_back(g, nw);
  for (int idims = s.idlo; idims <= s.idhi; ++idims) {
    const int o = g.off(idims);
    Box kxC = ixI;
    kxC.hi[idims] -= 1;
    wLp.d = wprim.d;
    wRp.d = wprim.d;
    for (int iw = 0; iw < nw; ++iw)
      forbox(kxC, [&](int i, int j, int k) {
        const size_t p = g.idx(i, j, k) + g.cells * (size_t)iw;
        wRp.d[p] = wprim.d[p + o];
      });
    Box ixC = ixO;
    ixC.lo[idims] -= 1;
    Box ixCR = ixC;
    st |= reconstruct_LR(s, ixCR, ixCR, idims, wprim, wLC, wRC, wLp, wRp, dxs[idims]);
    if (x.glm) modify_wLR(s, ixCR, wLC, wRC, wLp, wRp, idims, cmax_global);
    get_flux(s, wLC, wLp, ixC, idims, cmax_global, fLC);
    get_flux(s, wRC, wRp, ixC, idims, cmax_global, fRC);
    if (c.flux_scheme == ORC_FS_TVDMU) {
      // get_Riemann_flux_tvdmu (src/mod_finite_volume.t:342-346)
      for (int iw = 0; iw < nw; ++iw)
        forbox(ixC, [&](int i, int j, int k) { W(fC[idims], iw) = R(half) * (W(fLC, iw) + W(fRC, iw)); });
    } else if (c.flux_scheme == ORC_FS_TVDLF) {
      st |= get_cbounds(s, wLC, wRC, wLp, wRp, ixC, idims, cmaxC, (Arr<R> *)nullptr);
      riemann_tvdlf(s, ixC, idims, wLC, wRC, fLC, fRC, cmaxC, fC[idims]);
    } else {
      st |= get_cbounds(s, wLC, wRC, wLp, wRp, ixC, idims, cmaxC, &cminC);
      switch (c.flux_scheme) {
        case ORC_FS_HLL: riemann_hll(s, ixC, idims, wLC, wRC, fLC, fRC, cmaxC, cminC, fC[idims]); break;
        case ORC_FS_HLLC: riemann_hllc(s, ixC, idims, wLC, wRC, fLC, fRC, cmaxC, cminC, fC[idims]); break;
        default: riemann_hlld(s, ixC, idims, wLC, wRC, wLp, wRp, fLC, fRC, cmaxC, cminC, fC[idims]); break;
      }
    }
  }
  // conservative update (src/mod_finite_volume.t:269-284)
  for (int idims = s.idlo; idims <= s.idhi; ++idims) {
    const int o = g.off(idims);
    R dxinv = -R(qdt) / R(dxs[idims]);
    Box hb = ixO;
    hb.lo[idims] -= 1;
    for (int iw = 0; iw < nw; ++iw) {
      forbox(hb, [&](int i, int j, int k) { fC[idims](i, j, k, iw) = dxinv * fC[idims](i, j, k, iw); });
      forbox(ixO, [&](int i, int j, int k) {
        const size_t p = g.idx(i, j, k) + g.cells * (size_t)iw;
        wnew.d[p] = wnew.d[p] + fC[idims].d[p] - fC[idims].d[p - o];
      });
    }
    // the MUSCL scheme's characteristic limiter, with the states of the
    // last direction reconstructed (one direction per dimensionally split sweep)
    if (c.flux_scheme == ORC_FS_TVDMU) {
      if (x.mhd) tvdlimit2_mhd(s, qdt, ixO, idims, wLC, wRC, wnew, fC[idims], dxs);
      else tvdlimit2_hd(s, qdt, ixO, idims, wLC, wRC, wnew, fC[idims], dxs);
    }
  }
  if (c.fix_small_values) {
    int s2 = handle_small_values(s, false, wnew, ixO);
    st |= s2;
    if (s2 & ORC_ST_SMALL_VALUE) wnew.d = wCT.d;
  }
  // addsource2 -> mhd_add_source divB part (src/mod_source.t:130-160)
  if (x.mhd && ndim > 1) {
    double qsrc = qdt * double(s.idhi - s.idlo + 1) / double(ndim);
    if (c.divb == ORC_DIVB_GLM) st |= add_source_glm(s, qsrc, ixI, ixO, wCT, wnew, dxs, cmax_global);
    else if (c.divb == ORC_DIVB_LINDE) st |= add_source_linde(s, qsrc, ixO, wCT, wnew, dxs, jump_faces);
  }
  (void)dtfactor;
  if (keep_fc) *keep_fc = std::move(fC);  // scaled face fluxes -qdt/dx F, for store_flux
  return st;
}

// hancock (src/mod_finite_volume.t:19-113), slab_uniform, no local dt: the
// MUSCL-Hancock predictor of twostep Predictor_Corrector for tvdlf.  Per
// direction the cell's edge states (wLp on ixO: right edge; wRp on hxO = ixO -
// e_d: the left edge of the cell above), their physical fluxes and
// wnew(ixO) += -qdt/dx (fLC(ixO) - fRC(hxO)); then the divB sources and the
// small-value check on wnew (no restore to wCT).
template <class R>
int hancock(const State &s, const Arr<R> &wCT, Arr<R> &wnew, double qdt, const double *dxs,
            double cmax_global, int jump_faces = 0) {
  const Ix &x = s.x;
  const orc_cfg &c = s.c;
  const Geo &g = s.g;
  const int nw = x.nw, ndim = c.ndim;
  Box ixI = g.ixG(), ixO = g.ixM();
  int st = 0;
  Arr<R> wprim = wCT;
  st |= to_primitive(s, ixI, wprim);
  Arr<R> wLp(g, nw), wRp(g, nw), wLC(g, nw), wRC(g, nw), fLC(g, nw), fRC(g, nw);
  for (int idims = s.idlo; idims <= s.idhi; ++idims) {
    const int o = g.off(idims);
    const Box hxO = shift(ixO, idims, -1);
    for (int iw = 0; iw < nw; ++iw)
      forbox(ixO, [&](int i, int j, int k) {
        const size_t p = g.idx(i, j, k) + g.cells * (size_t)iw;
        wRp.d[p - o] = wprim.d[p];
        wLp.d[p] = wprim.d[p];
      });
    st |= reconstruct_LR(s, ixO, hxO, idims, wprim, wLC, wRC, wLp, wRp, dxs[idims]);
    get_flux(s, wRC, wRp, hxO, idims, cmax_global, fRC);
    get_flux(s, wLC, wLp, ixO, idims, cmax_global, fLC);
    const R dxinv = -R(qdt) / R(dxs[idims]);
    for (int iw = 0; iw < nw; ++iw)
      forbox(ixO, [&](int i, int j, int k) {
        const size_t p = g.idx(i, j, k) + g.cells * (size_t)iw;
        wnew.d[p] = wnew.d[p] + dxinv * (fLC.d[p] - fRC.d[p - o]);
      });
  }
  if (x.mhd && ndim > 1) {
    double qsrc = qdt * double(s.idhi - s.idlo + 1) / double(ndim);
    if (c.divb == ORC_DIVB_GLM) st |= add_source_glm(s, qsrc, ixI, ixO, wCT, wnew, dxs, cmax_global);
    else if (c.divb == ORC_DIVB_LINDE) st |= add_source_linde(s, qsrc, ixO, wCT, wnew, dxs, jump_faces);
  }
  if (c.fix_small_values) st |= handle_small_values(s, false, wnew, ixO);
  return st;
}

// getdt_courant (src/mod_dt.t:160-287) with hd_get_cmax (src/hd/mod_hd_phys.t:787-811)
// and mhd_get_cmax_origin (src/mhd/mod_mhd_phys.t:2482-2550).
template <class R>
int getdt_block(const State &s, const Arr<R> &w, const double *dx, double *dtnew, double *cmax_mype) {
  const Ix &x = s.x;
  const orc_cfg &c = s.c;
  const Geo &g = s.g;
  Box ixI = g.ixG(), ixO = g.ixM();
  Arr<R> wprim = w;
  int st = to_primitive(s, ixI, wprim);
  std::vector<R> cmax(g.cells), cmaxtot(g.cells);
  R courantmax(0.0), courantmaxtot(0.0);
  double dtn = bigdouble;
  R dxinv[3];
  for (int d = 0; d < c.ndim; ++d) dxinv[d] = R(one) / R(dx[d]);
  for (int idims = 0; idims < c.ndim; ++idims) {
    forbox(ixO, [&](int i, int j, int k) {
      const int mn = x.mom[idims];
      R cm;
      if (x.mhd) {
        R inv_rho = R(1.0) / W(wprim, x.rho);
        R cs = gam_<R>(s) * W(wprim, x.e) * inv_rho;
        R b2 = W(wprim, x.mag[0]) * W(wprim, x.mag[0]);
        for (int q = 1; q < x.ndir; ++q) b2 = b2 + W(wprim, x.mag[q]) * W(wprim, x.mag[q]);
        R cfast2 = b2 * inv_rho + cs;
        R bn = W(wprim, x.mag[idims]);
        R av = cfast2 * cfast2 - R(4.0) * cs * (bn * bn) * inv_rho;
        if (av < R(zero)) av = R(zero);
        cm = rsqrt_(R(half) * (cfast2 + rsqrt_(av)));
        cm = rabs(W(wprim, mn)) + cm;
      } else {
        cm = rabs(W(wprim, mn)) + rsqrt_(gam_<R>(s) * W(wprim, x.e) / W(wprim, x.rho));
      }
      cmax[g.idx(i, j, k)] = cm;
    });
    R cmx(0.0);
    bool first = true;
    forbox(ixO, [&](int i, int j, int k) {
      R v = cmax[g.idx(i, j, k)];
      if (first || v > cmx) { cmx = v; first = false; }
    });
    if (val(cmx) > *cmax_mype) *cmax_mype = val(cmx);
    if (c.type_courant == ORC_COURANT_MAXSUM) {
      forbox(ixO, [&](int i, int j, int k) {
        const int p = g.idx(i, j, k);
        if (idims == 0) cmaxtot[p] = cmax[p] * dxinv[idims];
        else cmaxtot[p] = cmaxtot[p] + cmax[p] * dxinv[idims];
      });
    } else {
      R m(0.0);
      bool f2 = true;
      forbox(ixO, [&](int i, int j, int k) {
        R v = cmax[g.idx(i, j, k)] * dxinv[idims];
        if (f2 || v > m) { m = v; f2 = false; }
      });
      courantmax = rmax(courantmax, m);
      if (c.type_courant == ORC_COURANT_SUMMAX) courantmaxtot = courantmaxtot + courantmax;
    }
  }
  if (c.type_courant == ORC_COURANT_MAXSUM) {
    R m(0.0);
    bool f = true;
    forbox(ixO, [&](int i, int j, int k) {
      R v = cmaxtot[g.idx(i, j, k)];
      if (f || v > m) { m = v; f = false; }
    });
    if (val(m) > smalldouble) dtn = std::min(dtn, val(R(c.courantpar) / m));
  } else if (c.type_courant == ORC_COURANT_SUMMAX) {
    if (val(courantmaxtot) > smalldouble) dtn = std::min(dtn, val(R(c.courantpar) / courantmaxtot));
  } else {
    if (val(courantmax) > smalldouble) dtn = std::min(dtn, val(R(c.courantpar) / courantmax));
  }
  *dtnew = dtn;
  return st;
}

// ---------------------------------------------------------------- grid
struct Grid {
  State s;
  int nb[3];
  int nblocks;
  double dx[3], xmin[3], xmax[3];
  int bc[6];
  std::vector<int> nbr;  // [ib][27] neighbour block or -1 (physical boundary)
  std::vector<double> reg[4];
  size_t bsize;
  long it = 0;  // steps advanced (the parity of a split step's sweep order)
};

inline int dir_index(int di, int dj, int dk) { return (di + 1) + 3 * ((dj + 1) + 3 * (dk + 1)); }

}  // namespace orc

using namespace orc;

struct orc_grid : public Grid {};

extern "C" {

int orc_cfg_finalize(orc_cfg *cfg) {
  Ix x = make_ix(*cfg);
  cfg->nw = x.nw;
  if (cfg->ssprk_order == 0) cfg->ssprk_order = 3;
  if (cfg->time_stepper == 0) cfg->time_stepper = 3;
  return x.nw;
}

static Arr<double> wrap_in(const Geo &g, int nw, const double *src) {
  Arr<double> a(g, nw);
  std::memcpy(a.d.data(), src, sizeof(double) * a.d.size());
  return a;
}

int orc_finite_volume(const orc_cfg *cfg, const double *wct, double *wnew, double qdt, double dtfactor,
                      const double *dx, double cmax_global) {
  State s = make_state(*cfg);
  Arr<double> a = wrap_in(s.g, s.x.nw, wct), b = wrap_in(s.g, s.x.nw, wnew);
  int st = finite_volume(s, a, b, qdt, dtfactor, dx, cmax_global);
  std::memcpy(wnew, b.d.data(), sizeof(double) * b.d.size());
  return st;
}

int orc_getdt_block(const orc_cfg *cfg, const double *w, const double *dx, double *dtnew,
                    double *cmax_max) {
  State s = make_state(*cfg);
  Arr<double> a = wrap_in(s.g, s.x.nw, w);
  return getdt_block(s, a, dx, dtnew, cmax_max);
}

void orc_to_primitive(const orc_cfg *cfg, double *w) {
  State s = make_state(*cfg);
  Arr<double> a = wrap_in(s.g, s.x.nw, w);
  to_primitive(s, s.g.ixG(), a);
  std::memcpy(w, a.d.data(), sizeof(double) * a.d.size());
}

void orc_to_conserved(const orc_cfg *cfg, double *w) {
  State s = make_state(*cfg);
  Arr<double> a = wrap_in(s.g, s.x.nw, w);
  to_conserved(s, s.g.ixG(), a);
  std::memcpy(w, a.d.data(), sizeof(double) * a.d.size());
}

// Points API: a 1-D "block" of n cells, state-major input.
static State point_state(const orc_cfg *cfg, int n) {
  orc_cfg c = *cfg;
  c.block_nx[0] = n; c.block_nx[1] = 1; c.block_nx[2] = 1;
  c.nghost = 0;
  State s = make_state(c);
  s.g.ndim = 1;
  s.g.ng = 0;
  s.g.n[0] = n; s.g.n[1] = 1; s.g.n[2] = 1;
  s.g.nx[0] = n; s.g.nx[1] = 1; s.g.nx[2] = 1;
  s.g.cells = n;
  return s;
}
static void load_points(const State &s, int n, const double *src, Arr<double> &a) {
  for (int p = 0; p < n; ++p)
    for (int iw = 0; iw < s.x.nw; ++iw) a(p, 0, 0, iw) = src[(size_t)p * s.x.nw + iw];
}
static Box line_box(int n) { Box b; b.lo[0] = 0; b.hi[0] = n - 1; b.lo[1] = b.hi[1] = b.lo[2] = b.hi[2] = 0; return b; }

void orc_get_flux_points(const orc_cfg *cfg, int n, const double *wc, const double *wp, int idim,
                         double cmax_global, double *f) {
  State s = point_state(cfg, n);
  Arr<double> C(s.g, s.x.nw), P(s.g, s.x.nw), F(s.g, s.x.nw);
  load_points(s, n, wc, C);
  load_points(s, n, wp, P);
  get_flux(s, C, P, line_box(n), idim - 1, cmax_global, F);
  for (int p = 0; p < n; ++p)
    for (int iw = 0; iw < s.x.nw; ++iw) f[(size_t)p * s.x.nw + iw] = F(p, 0, 0, iw);
}

void orc_get_cbounds_points(const orc_cfg *cfg, int n, const double *wlc, const double *wrc,
                            const double *wlp, const double *wrp, int idim, double *cmax, double *cmin) {
  State s = point_state(cfg, n);
  Arr<double> LC(s.g, s.x.nw), RC(s.g, s.x.nw), LP(s.g, s.x.nw), RP(s.g, s.x.nw), CX(s.g, 1), CN(s.g, 1);
  load_points(s, n, wlc, LC); load_points(s, n, wrc, RC);
  load_points(s, n, wlp, LP); load_points(s, n, wrp, RP);
  get_cbounds(s, LC, RC, LP, RP, line_box(n), idim - 1, CX, cmin ? &CN : (Arr<double> *)nullptr);
  for (int p = 0; p < n; ++p) {
    cmax[p] = CX(p, 0, 0, 0);
    if (cmin) cmin[p] = CN(p, 0, 0, 0);
  }
}

void orc_riemann_points(const orc_cfg *cfg, int n, const double *wlp_in, const double *wrp_in, int idim,
                        double cmax_global, double *f) {
  State s = point_state(cfg, n);
  const int d = idim - 1;
  Arr<double> LP(s.g, s.x.nw), RP(s.g, s.x.nw), LC(s.g, s.x.nw), RC(s.g, s.x.nw), FL(s.g, s.x.nw),
      FR(s.g, s.x.nw), FC(s.g, s.x.nw), CX(s.g, 1), CN(s.g, 1);
  load_points(s, n, wlp_in, LP);
  load_points(s, n, wrp_in, RP);
  Box b = line_box(n);
  LC.d = LP.d; RC.d = RP.d;
  to_conserved(s, b, LC);
  to_conserved(s, b, RC);
  if (s.x.mhd && cfg->divb == ORC_DIVB_GLM && cfg->ndim > 1) modify_wLR(s, b, LC, RC, LP, RP, d, cmax_global);
  get_flux(s, LC, LP, b, d, cmax_global, FL);
  get_flux(s, RC, RP, b, d, cmax_global, FR);
  if (cfg->flux_scheme == ORC_FS_TVDLF) {
    get_cbounds(s, LC, RC, LP, RP, b, d, CX, (Arr<double> *)nullptr);
    riemann_tvdlf(s, b, d, LC, RC, FL, FR, CX, FC);
  } else {
    get_cbounds(s, LC, RC, LP, RP, b, d, CX, &CN);
    if (cfg->flux_scheme == ORC_FS_HLL) riemann_hll(s, b, d, LC, RC, FL, FR, CX, CN, FC);
    else if (cfg->flux_scheme == ORC_FS_HLLC) riemann_hllc(s, b, d, LC, RC, FL, FR, CX, CN, FC);
    else riemann_hlld(s, b, d, LC, RC, LP, RP, FL, FR, CX, CN, FC);
  }
  for (int p = 0; p < n; ++p)
    for (int iw = 0; iw < s.x.nw; ++iw) f[(size_t)p * s.x.nw + iw] = FC(p, 0, 0, iw);
}

void orc_limiter_line(const orc_cfg *cfg, int n, const double *dwc, double dxlevel, double *ldw,
                      double *rdw) {
  orc_cfg c = *cfg;
  c.ndim = 1;
  State s = point_state(&c, n);
  Arr<double> D(s.g, 1), L(s.g, 1), R(s.g, 1);
  for (int p = 0; p < n; ++p) { D.d[p] = dwc[p]; L.d[p] = ldw[p]; R.d[p] = rdw[p]; }
  dwlimiter2(s, D, line_box(n), 0, dxlevel, L, R);
  for (int p = 0; p < n; ++p) { ldw[p] = L.d[p]; rdw[p] = R.d[p]; }
}

// ---------------------------------------------------------------- grid API
orc_grid *orc_grid_create(const orc_cfg *cfg, const int *domain_nx, const double *xprobmin,
                          const double *xprobmax, const int *bc) {
  orc_grid *g = new orc_grid();
  g->s = make_state(*cfg);
  g->nblocks = 1;
  for (int d = 0; d < 3; ++d) {
    if (d < cfg->ndim) {
      g->nb[d] = domain_nx[d] / cfg->block_nx[d];
      g->dx[d] = (xprobmax[d] - xprobmin[d]) / double(domain_nx[d]);
      g->xmin[d] = xprobmin[d];
      g->xmax[d] = xprobmax[d];
    } else {
      g->nb[d] = 1; g->dx[d] = 1.0; g->xmin[d] = 0; g->xmax[d] = 1;
    }
    g->nblocks *= g->nb[d];
  }
  for (int q = 0; q < 6; ++q) g->bc[q] = q < 2 * cfg->ndim ? bc[q] : ORC_BC_PERIODIC;
  g->bsize = g->s.g.cells * (size_t)g->s.x.nw;
  for (int r = 0; r < 4; ++r) g->reg[r].assign(g->bsize * g->nblocks, 0.0);
  g->nbr.assign((size_t)g->nblocks * 27, -1);
  for (int ib = 0; ib < g->nblocks; ++ib) {
    int ig[3] = {ib % g->nb[0], (ib / g->nb[0]) % g->nb[1], ib / (g->nb[0] * g->nb[1])};
    for (int dk = -1; dk <= 1; ++dk)
      for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) {
          int dd[3] = {di, dj, dk};
          int jg[3];
          bool ok = true;
          for (int d = 0; d < 3; ++d) {
            if (d >= cfg->ndim) { if (dd[d] != 0) ok = false; jg[d] = 0; continue; }
            jg[d] = ig[d] + dd[d];
            if (jg[d] < 0 || jg[d] >= g->nb[d]) {
              int side = jg[d] < 0 ? 0 : 1;
              if (g->bc[2 * d + side] == ORC_BC_PERIODIC) jg[d] = (jg[d] + g->nb[d]) % g->nb[d];
              else ok = false;
            }
          }
          if (ok) g->nbr[(size_t)ib * 27 + dir_index(di, dj, dk)] = jg[0] + g->nb[0] * (jg[1] + g->nb[1] * jg[2]);
        }
  }
  return g;
}

void orc_grid_destroy(orc_grid *g) { delete g; }
int orc_grid_nblocks(const orc_grid *g) { return g->nblocks; }
void orc_grid_block_index(const orc_grid *g, int ib, int *ig) {
  ig[0] = ib % g->nb[0];
  ig[1] = (ib / g->nb[0]) % g->nb[1];
  ig[2] = ib / (g->nb[0] * g->nb[1]);
}
void orc_grid_dx(const orc_grid *g, double *dx) { for (int d = 0; d < g->s.c.ndim; ++d) dx[d] = g->dx[d]; }

// Block geometry (src/amr/mod_amr_solution_node.t:158-164)
double orc_grid_x(const orc_grid *g, int ib, int idim, int i) {
  int ig[3];
  orc_grid_block_index(g, ib, ig);
  const int d = idim;
  double dg = g->s.c.block_nx[d] * g->dx[d];
  double rxmin = g->xmin[d] + double(ig[d]) * dg;
  return rxmin + (double(i + 1 - g->s.c.nghost) - half) * g->dx[d];
}

void orc_grid_set_block(orc_grid *g, int ib, const double *w) {
  std::memcpy(&g->reg[0][g->bsize * ib], w, sizeof(double) * g->bsize);
}
void orc_grid_get_block(const orc_grid *g, int ib, double *w) {
  std::memcpy(w, &g->reg[0][g->bsize * ib], sizeof(double) * g->bsize);
}

// ixS_srl_/ixR_srl_ (src/mod_ghostcells_update.t:150-162), 0-based inclusive,
// indexed by i+1 for i in {-1,0,1}.
void orc_srl_maps(int nghost, int block_nx, int *s_min, int *s_max, int *r_min, int *r_max) {
  // Fortran 1-based: ixMmin = nghost+1, ixMmax = nghost+block_nx, ixGmax = block_nx+2*nghost
  int ixMmin = nghost + 1, ixMmax = nghost + block_nx, ixGmax = block_nx + 2 * nghost;
  int smin[3] = {ixMmin, ixMmin, ixMmax + 1 - nghost};
  int smax[3] = {ixMmin - 1 + nghost, ixMmax, ixMmax};
  int rmin[3] = {1, ixMmin, ixMmax + 1};
  int rmax[3] = {nghost, ixMmax, ixGmax};
  for (int q = 0; q < 3; ++q) {
    s_min[q] = smin[q] - 1; s_max[q] = smax[q] - 1;
    r_min[q] = rmin[q] - 1; r_max[q] = rmax[q] - 1;
  }
}

extern "C++" {
template <class R, class NBT>
static void bc_phys_block(const State &s, const int *bcs, R *w, NBT nbt);

template <class R>
static void getbc_reg(const Grid &G, std::vector<R> &reg) {
  const State &s = G.s;
  const Geo &g = s.g;
  const int ndim = s.c.ndim, nw = s.x.nw;
  int smin[3], smax[3], rmin[3], rmax[3];
  int sminA[3][3], smaxA[3][3], rminA[3][3], rmaxA[3][3];
  for (int d = 0; d < 3; ++d) {
    if (d < ndim) {
      orc_srl_maps(s.c.nghost, s.c.block_nx[d], smin, smax, rmin, rmax);
      for (int q = 0; q < 3; ++q) { sminA[d][q] = smin[q]; smaxA[d][q] = smax[q]; rminA[d][q] = rmin[q]; rmaxA[d][q] = rmax[q]; }
    } else {
      for (int q = 0; q < 3; ++q) { sminA[d][q] = smaxA[d][q] = rminA[d][q] = rmaxA[d][q] = 0; }
    }
  }
  // same-resolution fill: bc_fill_srl (src/mod_ghostcells_update.t:812-852)
  for (int ib = 0; ib < G.nblocks; ++ib) {
    for (int dk = (ndim > 2 ? -1 : 0); dk <= (ndim > 2 ? 1 : 0); ++dk)
      for (int dj = (ndim > 1 ? -1 : 0); dj <= (ndim > 1 ? 1 : 0); ++dj)
        for (int di = -1; di <= 1; ++di) {
          if (di == 0 && dj == 0 && dk == 0) continue;
          int nb = G.nbr[(size_t)ib * 27 + dir_index(di, dj, dk)];
          if (nb < 0) continue;
          int dd[3] = {di, dj, dk};
          Box S, Rb;
          for (int d = 0; d < 3; ++d) {
            S.lo[d] = sminA[d][dd[d] + 1]; S.hi[d] = smaxA[d][dd[d] + 1];
            Rb.lo[d] = rminA[d][-dd[d] + 1]; Rb.hi[d] = rmaxA[d][-dd[d] + 1];
          }
          R *src = &reg[G.bsize * ib], *dst = &reg[G.bsize * nb];
          for (int iw = 0; iw < nw; ++iw)
            for (int k = 0; k <= S.hi[2] - S.lo[2]; ++k)
              for (int j = 0; j <= S.hi[1] - S.lo[1]; ++j)
                for (int i = 0; i <= S.hi[0] - S.lo[0]; ++i)
                  dst[g.idx(Rb.lo[0] + i, Rb.lo[1] + j, Rb.lo[2] + k) + g.cells * (size_t)iw] =
                      src[g.idx(S.lo[0] + i, S.lo[1] + j, S.lo[2] + k) + g.cells * (size_t)iw];
        }
  }
  for (int ib = 0; ib < G.nblocks; ++ib)
    bc_phys_block(s, G.bc, &reg[G.bsize * ib],
                  [&](int di, int dj, int dk) { return G.nbr[(size_t)ib * 27 + dir_index(di, dj, dk)] < 0; });
}

// physical boundaries of one ghosted block: fill_boundary_after_gc
// (src/mod_ghostcells_update.t:580-615) with bc_phys cont/symm/asymm
// (src/mod_boundary_conditions.t:12-265); nbt(dir) is true for a direction
// that leaves the domain.
template <class R, class NBT>
static void bc_phys_block(const State &s, const int *bcs, R *w, NBT nbt) {
  const Geo &g = s.g;
  const int ndim = s.c.ndim, nw = s.x.nw;
  const int ng = s.c.nghost;
  {
    for (int idims = 0; idims < ndim; ++idims) {
      int kmin[3] = {0, 0, 0}, kmax[3] = {0, 0, 0};
      if (ndim >= 2) { kmin[1] = (idims < 1 && nbt(0, -1, 0)) ? 1 : 0; kmax[1] = (idims < 1 && nbt(0, 1, 0)) ? 1 : 0; }
      if (ndim >= 3) { kmin[2] = (idims < 2 && nbt(0, 0, -1)) ? 1 : 0; kmax[2] = (idims < 2 && nbt(0, 0, 1)) ? 1 : 0; }
      Box B;
      for (int d = 0; d < 3; ++d) { B.lo[d] = kmin[d] * ng; B.hi[d] = g.n[d] - 1 - kmax[d] * ng; }
      if (ndim < 3) { B.lo[2] = B.hi[2] = 0; }
      if (ndim < 2) { B.lo[1] = B.hi[1] = 0; }
      for (int iside = 0; iside < 2; ++iside) {
        int dd[3] = {0, 0, 0};
        dd[idims] = iside == 0 ? -1 : 1;
        if (!nbt(dd[0], dd[1], dd[2])) continue;
        int type = bcs[2 * idims + iside];
        Box O = B;
        if (iside == 1) O.lo[idims] = B.hi[idims] + 1 - ng;
        else O.hi[idims] = B.lo[idims] - 1 + ng;
        const int o = g.off(idims);
        for (int iw = 0; iw < nw; ++iw) {
          double sgn = 1.0;
          if (type == ORC_BC_ASYMM) sgn = -1.0;
          forbox(O, [&](int i, int j, int k) {
            int p = g.idx(i, j, k);
            int c[3] = {i, j, k};
            int q;
            if (type == ORC_BC_CONT) {
              int src = iside == 1 ? O.lo[idims] - 1 : O.hi[idims] + 1;
              q = p + (src - c[idims]) * o;
              w[p + g.cells * (size_t)iw] = w[q + g.cells * (size_t)iw];
            } else {
              // mirror: ghost ixOmin+m <- ixOmin-1-m (max side), ixOmax-m <- ixOmax+1+m (min side)
              int src = iside == 1 ? 2 * O.lo[idims] - 1 - c[idims] : 2 * O.hi[idims] + 1 - c[idims];
              q = p + (src - c[idims]) * o;
              w[p + g.cells * (size_t)iw] = R(sgn) * w[q + g.cells * (size_t)iw];
            }
          });
        }
      }
    }
  }
}
}  // extern "C++"

void orc_grid_getbc(orc_grid *g) { getbc_reg(*g, g->reg[0]); }

// phys_get_a2max (src/hd/mod_hd_phys.t:813-833, src/mhd/mod_mhd_phys.t:
// 2678-2698) of one ghosted block, maxed into a2m (getdt_courant,
// src/mod_dt.t:193-197): |-w(i+2) + 16 w(i+1) - 30 w(i) + 16 w(i-1) - w(i-2)|
// over the interior and every conserved variable, / 12 / dx^2.
static void a2max_block(const State &s, const Arr<double> &w, const double *dx, double *a2m) {
  const Box O = s.g.ixM();
  for (int d = 0; d < s.c.ndim; ++d) {
    const int o = s.g.off(d);
    double m = 0.0;
    for (int iw = 0; iw < s.x.nw; ++iw)
      forbox(O, [&](int i, int j, int k) {
        const double *q = &w.d[s.g.idx(i, j, k) + s.g.cells * (size_t)iw];
        m = std::max(m, std::fabs((((-q[2 * o] + 16.0 * q[o]) - 30.0 * q[0]) + 16.0 * q[-o]) - q[-2 * o]));
      });
    a2m[d] = std::max(a2m[d], m / 12.0 / (dx[d] * dx[d]));
  }
}

int orc_grid_getdt(orc_grid *g, double *dt, double *cmax_global) {
  const size_t bs = g->bsize;
  double dtmin = bigdouble, cmx = 0.0;
  double a2m[3] = {0.0, 0.0, 0.0};
  int st = 0;
  for (int ib = 0; ib < g->nblocks; ++ib) {
    Arr<double> a = wrap_in(g->s.g, g->s.x.nw, &g->reg[0][bs * ib]);
    double dtn;
    st |= getdt_block(g->s, a, g->dx, &dtn, &cmx);
    dtmin = std::min(dtmin, dtn);
    if (g->s.c.schmid_global) a2max_block(g->s, a, g->dx, a2m);
  }
  // schmid1: the limiter's a2max is a2max_global of this setdt
  if (g->s.c.schmid_global)
    for (int d = 0; d < 3; ++d) g->s.c.schmid_rad[d] = a2m[d];
  *dt = dtmin;
  *cmax_global = cmx;
  return st;
}

// predictor: the twostep Predictor_Corrector predictor, advect1 with
// typepred1 (hancock for tvdlf and tvdmu, src/io/mod_input_output.t:787-797).
static int grid_advect1(orc_grid *g, int ra, int rb, double qdt, double dtfactor, double cmax_global, int nthreads,
                        bool predictor) {
  const size_t bs = g->bsize;
  const bool hk = predictor && (g->s.c.flux_scheme == ORC_FS_TVDLF || g->s.c.flux_scheme == ORC_FS_TVDMU);
  int st = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic) reduction(| : st)
#endif
  for (int ib = 0; ib < g->nblocks; ++ib) {
    Arr<double> a = wrap_in(g->s.g, g->s.x.nw, &g->reg[ra][bs * ib]);
    Arr<double> b = wrap_in(g->s.g, g->s.x.nw, &g->reg[rb][bs * ib]);
    if (hk) st |= hancock(g->s, a, b, qdt, g->dx, cmax_global);
    else st |= finite_volume(g->s, a, b, qdt, dtfactor, g->dx, cmax_global);
    std::memcpy(&g->reg[rb][bs * ib], b.d.data(), sizeof(double) * bs);
  }
  getbc_reg(*g, g->reg[rb]);
  return st;
}

int orc_grid_advect1(orc_grid *g, int ra, int rb, double qdt, double dtfactor, double cmax_global,
                     int nthreads) {
  return grid_advect1(g, ra, rb, qdt, dtfactor, cmax_global, nthreads, false);
}

void orc_grid_copy_reg(orc_grid *g, int dst, int src) { g->reg[dst] = g->reg[src]; }

void orc_grid_combine_reg(orc_grid *g, int dst, double a, int ra, double b, int rb) {
  std::vector<double> &D = g->reg[dst];
  const std::vector<double> &A = g->reg[ra], &B = g->reg[rb];
  for (size_t p = 0; p < D.size(); ++p) D[p] = a * A[p] + b * B[p];
}

extern "C++" {
// fourstep (src/mod_advance.t:454-512), coefficients
// src/io/mod_input_output.t:1036-1067, on registers 0..3 through the grid's
// advect1 (stage plus getbc), copy and two-term combination.
template <class Adv, class Copy, class Comb, class Comb4>
int fourstep(const orc_cfg &c, double dt, Adv advect1, Copy copy, Comb combine, Comb4 rk4_combine) {
  int st = 0;
  copy(1, 0);  // advect: ps1 = ps before the stepper
  if (c.time_integrator == 1) {  // rk4
    copy(2, 0);
    copy(3, 0);
    st |= advect1(0, 1, 0.5 * dt, 0.5);
    st |= advect1(1, 2, 0.5 * dt, 0.5);
    st |= advect1(2, 3, 1.0 * dt, 1.0);
    rk4_combine();
    st |= advect1(3, 0, (1.0 / 6.0) * dt, 1.0 / 6.0);
    return st;
  }
  double b11, b22, b33, b44, a21, a31, a41;
  if (c.ssprk_order == 2) {
    b11 = 1.0 / 3.0; b22 = 1.0 / 3.0; b33 = 1.0 / 3.0; b44 = 1.0 / 4.0; a21 = 0.0; a31 = 0.0; a41 = 1.0 / 4.0;
  } else {
    b11 = 1.0 / 2.0; b22 = 1.0 / 2.0; b33 = 1.0 / 6.0; b44 = 1.0 / 2.0; a21 = 0.0; a31 = 2.0 / 3.0; a41 = 0.0;
  }
  st |= advect1(0, 1, b11 * dt, b11);
  combine(2, a21, 0, 1.0 - a21, 1);
  st |= advect1(1, 2, b22 * dt, b22);
  combine(1, a31, 0, 1.0 - a31, 2);
  st |= advect1(2, 1, b33 * dt, b33);
  combine(0, a41, 0, 1.0 - a41, 1);
  st |= advect1(1, 0, b44 * dt, b44);
  return st;
}

// fivestep ssprk5 (src/mod_advance.t:513-557), coefficients
// src/io/mod_input_output.t:1079-1140 (ssprk_order 3: Gottlieb 2005, the
// default; 2: Spiteri-Ruuth), over whole (ghosted) registers 0..3.
template <class Adv, class Copy, class Comb>
int fivestep(const orc_cfg &c, double dt, Adv advect1, Copy copy, Comb combine, std::vector<double> *reg) {
  double b11, b22, b33, b44, b54, b55, a21, a31, a41, a53, a54, a22, a33, a44, a55;
  if (c.ssprk_order == 2) {
    b11 = 0.39175222700392; b22 = 0.36841059262959; b33 = 0.25189177424738; b44 = 0.54497475021237;
    a21 = 0.44437049406734; a31 = 0.62010185138540; a41 = 0.17807995410773; a53 = 0.51723167208978;
    a22 = 1.0 - a21; a33 = 1.0 - a31; a44 = 1.0 - a41;
    const double rka51 = 0.00683325884039, rka54 = 0.12759831133288, rkb54 = 0.08460416338212;
    b54 = rkb54 - b44 * rka51 / a41;
    a54 = rka54 - a44 * rka51 / a41;
    a55 = 1.0 - a53 - a54;
    const double c2 = b11, c3 = a22 * c2 + b22, c4 = a33 * c3 + b33, c5 = a44 * c4 + b44;
    b55 = 1.0 - b54 - a53 * c3 - a54 * c4 - a55 * c5;
  } else {
    b11 = 0.391752226571890; b22 = 0.368410593050371; b33 = 0.251891774271694; b44 = 0.544974750228521;
    b54 = 0.063692468666290; b55 = 0.226007483236906; a21 = 0.444370493651235; a31 = 0.620101851488403;
    a41 = 0.178079954393132; a53 = 0.517231671970585; a54 = 0.096059710526147;
    a22 = 1.0 - a21; a33 = 1.0 - a31; a44 = 1.0 - a41; a55 = 1.0 - a53 - a54;
  }
  int st = 0;
  copy(1, 0);  // advect: ps1 = ps before the stepper
  copy(2, 0);  // (sizes registers 2 and 3)
  copy(3, 0);
  st |= advect1(0, 1, b11 * dt, b11);
  combine(2, a21, 0, a22, 1);
  st |= advect1(1, 2, b22 * dt, b22);
  combine(1, a31, 0, a33, 2);
  st |= advect1(2, 1, b33 * dt, b33);
  combine(3, a53, 2, a54, 1);
  combine(2, a41, 0, a44, 1);
  st |= advect1(1, 2, b44 * dt, b44);
  const double r = b54 / b44;
  for (size_t p = 0; p < reg[0].size(); ++p)
    reg[0][p] = (reg[3][p] + a55 * reg[2][p]) + r * (reg[2][p] - (a41 * reg[0][p] + a44 * reg[1][p]));
  st |= advect1(2, 0, b55 * dt, b55);
  return st;
}

// twostep (src/mod_advance.t:102-133): Predictor_Corrector — predictor
// ps1 = ps + dt/2 L(ps) with typepred1 (the same scheme for hll, hllc, hlld;
// hancock for tvdlf) and no flux fix, corrector ps = ps + dt L(ps1) — or
// ssprk2.  advect1's last argument is false for the predictor only.
template <class Adv, class Copy, class Comb>
int twostep(const orc_cfg &c, double dt, Adv advect1, Copy copy, Comb combine) {
  int st = 0;
  copy(1, 0);
  if (c.time_integrator == 2) {
    st |= advect1(0, 1, dt, 1.0, true);
    combine(0, 0.5, 0, 0.5, 1);
    st |= advect1(1, 0, 0.5 * dt, 0.5, true);
    return st;
  }
  st |= advect1(0, 1, 0.5 * dt, 0.5, false);
  st |= advect1(1, 0, dt, 1.0, true);
  return st;
}

// ps = (1/3)(-ps + ps1 + 2 ps2 + ps3) over whole (ghosted) registers
inline void rk4_combine_regs(std::vector<double> *reg) {
  for (size_t p = 0; p < reg[0].size(); ++p)
    reg[0][p] = (1.0 / 3.0) * (((-reg[0][p] + reg[1][p]) + 2.0 * reg[2][p]) + reg[3][p]);
}
}  // extern "C++"

// advect threestep/ssprk3 (src/mod_advance.t:56-73, 249-267), coefficients
// src/io/mod_input_output.t:941-964; fourstep as above.
static int grid_advance_stepper(orc_grid *g, double dt, double cmax_global, int nthreads) {
  if (g->s.c.time_stepper == 2)
    return twostep(
        g->s.c, dt,
        [&](int ra, int rb, double qdt, double f, bool corr) {
          return grid_advect1(g, ra, rb, qdt, f, cmax_global, nthreads, !corr);
        },
        [&](int d, int s2) { orc_grid_copy_reg(g, d, s2); },
        [&](int d, double a, int ra, double b, int rb) { orc_grid_combine_reg(g, d, a, ra, b, rb); });
  if (g->s.c.time_stepper == 5)
    return fivestep(
        g->s.c, dt,
        [&](int ra, int rb, double qdt, double f) { return orc_grid_advect1(g, ra, rb, qdt, f, cmax_global, nthreads); },
        [&](int d, int s2) { orc_grid_copy_reg(g, d, s2); },
        [&](int d, double a, int ra, double b, int rb) { orc_grid_combine_reg(g, d, a, ra, b, rb); }, g->reg);
  if (g->s.c.time_stepper == 4)
    return fourstep(
        g->s.c, dt,
        [&](int ra, int rb, double qdt, double f) { return orc_grid_advect1(g, ra, rb, qdt, f, cmax_global, nthreads); },
        [&](int d, int s2) { orc_grid_copy_reg(g, d, s2); },
        [&](int d, double a, int ra, double b, int rb) { orc_grid_combine_reg(g, d, a, ra, b, rb); },
        [&]() { rk4_combine_regs(g->reg); });
  double b11, b22, b33, a21, a31;
  if (g->s.c.ssprk_order == 2) { b11 = 0.5; b22 = 0.5; b33 = 1.0 / 3.0; a21 = 0.0; a31 = 1.0 / 3.0; }
  else { b11 = 1.0; b22 = 1.0 / 4.0; b33 = 2.0 / 3.0; a21 = 3.0 / 4.0; a31 = 1.0 / 3.0; }
  double a22 = 1.0 - a21, a33 = 1.0 - a31;
  int st = 0;
  orc_grid_copy_reg(g, 1, 0);
  st |= orc_grid_advect1(g, 0, 1, b11 * dt, b11, cmax_global, nthreads);
  orc_grid_combine_reg(g, 2, a21, 0, a22, 1);
  st |= orc_grid_advect1(g, 1, 2, b22 * dt, b22, cmax_global, nthreads);
  orc_grid_combine_reg(g, 0, a31, 0, a33, 2);
  st |= orc_grid_advect1(g, 2, 0, b33 * dt, b33, cmax_global, nthreads);
  return st;
}

void orc_grid_volume_average(const orc_grid *g, int power, double *mean) {
  const Geo &geo = g->s.g;
  const int nw = g->s.x.nw;
  double dvol = 1.0;
  for (int d = 0; d < g->s.c.ndim; ++d) dvol *= g->dx[d];
  std::vector<double> wsum(nw + 1, 0.0);
  Box O = geo.ixM();
  for (int ib = 0; ib < g->nblocks; ++ib) {
    const double *w = &g->reg[0][g->bsize * ib];
    double vs = 0;
    forbox(O, [&](int i, int j, int k) { vs += dvol; });
    wsum[nw] += vs;
    for (int iw = 0; iw < nw; ++iw) {
      double acc = 0;
      forbox(O, [&](int i, int j, int k) {
        double v = w[geo.idx(i, j, k) + geo.cells * (size_t)iw];
        acc += dvol * (power == 1 ? v : v * v);
      });
      wsum[iw] += acc;
    }
  }
  for (int iw = 0; iw < nw; ++iw) mean[iw] = wsum[iw] / wsum[nw];
}

// ---------------------------------------------------------------- field loop
// tests/mhd/field_loop_2.5D/mod_usr.t: A0=1e-3, R0=0.3, v0=(2,1), vector-potential init.
static double fmodulo(double a, double p) { return a - std::floor(a / p) * p; }

static void fl_bfield(const orc_grid *g, int ib, double t, std::vector<double> &bx, std::vector<double> &by) {
  const Geo &geo = g->s.g;
  const double A0 = 1.0e-3, R0 = 0.3, v[2] = {2.0, 1.0};
  std::vector<double> Az(geo.cells, 0.0);
  for (int j = 0; j < geo.n[1]; ++j)
    for (int i = 0; i < geo.n[0]; ++i) {
      double x1 = orc_grid_x(g, ib, 0, i) - v[0] * t - g->xmin[0];
      x1 = g->xmin[0] + fmodulo(x1, g->xmax[0] - g->xmin[0]);
      double x2 = orc_grid_x(g, ib, 1, j) - v[1] * t - g->xmin[1];
      x2 = g->xmin[1] + fmodulo(x2, g->xmax[1] - g->xmin[1]);
      double r2 = x1 * x1 + x2 * x2;
      Az[geo.idx(i, j, 0)] = r2 < R0 * R0 ? A0 * (R0 - std::sqrt(r2)) : 0.0;
    }
  bx.assign(geo.cells, 0.0);
  by.assign(geo.cells, 0.0);
  Box O = geo.ixM();
  const int oy = geo.off(1), ox = geo.off(0);
  forbox(O, [&](int i, int j, int k) {
    int p = geo.idx(i, j, k);
    bx[p] = ((Az[p + oy] - Az[p - oy]) * half) / g->dx[1];
    double gy = ((Az[p + ox] - Az[p - ox]) * half) / g->dx[0];
    by[p] = -gy;
  });
}

int orc_run_field_loop(const orc_cfg *cfg_in, double courantpar, double time_max, double dtsave, int nrow_max,
                       double *rows, int nthreads) {
  orc_cfg cfg = *cfg_in;
  cfg.courantpar = courantpar;
  orc_cfg_finalize(&cfg);
  const int dom[3] = {128, 64, 1};
  const double xmn[3] = {-1.0, -0.5, 0}, xmx[3] = {1.0, 0.5, 1};
  const int bc[6] = {0, 0, 0, 0, 0, 0};
  orc_grid *g = orc_grid_create(&cfg, dom, xmn, xmx, bc);
  const Geo &geo = g->s.g;
  const Ix &x = g->s.x;
  const int nw = x.nw;
  Box O = geo.ixM();
  for (int ib = 0; ib < g->nblocks; ++ib) {
    double *w = &g->reg[0][g->bsize * ib];
    std::vector<double> bx, by;
    fl_bfield(g, ib, 0.0, bx, by);
    Arr<double> a(geo, nw);
    forbox(O, [&](int i, int j, int k) {
      a(i, j, k, x.rho) = 1.0;
      a(i, j, k, x.mom[0]) = 2.0;
      a(i, j, k, x.mom[1]) = 1.0;
      a(i, j, k, x.e) = 1.0;
      int p = geo.idx(i, j, k);
      a(i, j, k, x.mag[0]) = bx[p];
      a(i, j, k, x.mag[1]) = by[p];
    });
    to_conserved(g->s, O, a);
    std::memcpy(w, a.d.data(), sizeof(double) * g->bsize);
  }
  orc_grid_getbc(g);
  double t = 0.0, tsavelast = 0.0;
  const double dtmin = 1.0e-10;
  int it = 0, nrow = 0, st = 0;
  const int ncol = 1 + 2 * (nw + 3);
  double dvol = g->dx[0] * g->dx[1];
  for (;;) {
    // setdt (src/mod_dt.t:10-155)
    double dt, cmax_global;
    st |= orc_grid_getdt(g, &dt, &cmax_global);
    if (dt < dtmin) st |= ORC_ST_DT_TOO_SMALL;
    bool final_exit = false;
    if (time_max - t <= dtmin) final_exit = true;
    dt = std::min(dt, time_max - t);
    {
      double dtmax = std::ceil(t / dtsave) * dtsave;
      double other = (t > 0) ? std::ceil(t / bigdouble) * bigdouble : 0.0;
      dtmax = std::min(dtmax, other) - t;
      if (dtmax > smalldouble) dt = std::min(dt, dtmax);
      else dt = std::min(dt, dtsave);
    }
    // timetosave (src/amrvac.t:407-439) + usr_modify_output + printlog_regression_test
    if (t >= tsavelast + dtsave - smalldouble) {
      tsavelast = t;
      if (nrow < nrow_max) {
        double *row = rows + (size_t)nrow * ncol;
        std::vector<double> s1(nw + 3, 0.0), s2(nw + 3, 0.0);
        double vol = 0;
        for (int ib = 0; ib < g->nblocks; ++ib) {
          Arr<double> a = wrap_in(geo, nw, &g->reg[0][g->bsize * ib]);
          std::vector<double> d2(geo.cells), d4(geo.cells), bx, by;
          divb_central(g->s, a, O, g->dx, 1, d2);
          divb_central(g->s, a, O, g->dx, 2, d4);
          fl_bfield(g, ib, t, bx, by);
          forbox(O, [&](int i, int j, int k) {
            int p = geo.idx(i, j, k);
            vol += dvol;
            for (int iw = 0; iw < nw; ++iw) {
              double v = a(i, j, k, iw);
              s1[iw] += dvol * v;
              s2[iw] += dvol * v * v;
            }
            double e1 = a(i, j, k, x.mag[0]) - bx[p], e2 = a(i, j, k, x.mag[1]) - by[p];
            double ex[3] = {d2[p], d4[p], std::sqrt(e1 * e1 + e2 * e2)};
            for (int q = 0; q < 3; ++q) {
              s1[nw + q] += dvol * ex[q];
              s2[nw + q] += dvol * ex[q] * ex[q];
            }
          });
        }
        row[0] = t;
        for (int q = 0; q < nw + 3; ++q) {
          row[1 + q] = s1[q] / vol;
          row[1 + nw + 3 + q] = s2[q] / vol;
        }
      }
      ++nrow;
    }
    if (t >= time_max || final_exit) break;
    st |= orc_grid_advance(g, dt, cmax_global, nthreads);
    if (st & ORC_ST_SMALL_VALUE) break;
    ++it;
    t = t + dt;
  }
  orc_grid_destroy(g);
  if (st & ORC_ST_SMALL_VALUE) return -st;
  return nrow;
}

// ---------------------------------------------------------------- op counts
double orc_count_flops_stage(const orc_cfg *cfg, const double *wct, const double *wnew, double qdt,
                             const double *dx, double cmax_global) {
  State s = make_state(*cfg);
  Arr<Counted> a(s.g, s.x.nw), b(s.g, s.x.nw);
  for (size_t p = 0; p < a.d.size(); ++p) { a.d[p] = Counted(wct[p]); b.d[p] = Counted(wnew[p]); }
  g_ops = 0;
  finite_volume(s, a, b, qdt, 1.0, dx, cmax_global);
  double cells = 1;
  for (int d = 0; d < cfg->ndim; ++d) cells *= cfg->block_nx[d];
  return double(g_ops) / cells;
}

double orc_count_flops_getdt(const orc_cfg *cfg, const double *w, const double *dx) {
  State s = make_state(*cfg);
  Arr<Counted> a(s.g, s.x.nw);
  for (size_t p = 0; p < a.d.size(); ++p) a.d[p] = Counted(w[p]);
  g_ops = 0;
  double dtn, cm = 0;
  getdt_block(s, a, dx, &dtn, &cm);
  double cells = 1;
  for (int d = 0; d < cfg->ndim; ++d) cells *= cfg->block_nx[d];
  return double(g_ops) / cells;
}


// ---------------------------------------------------------------- forward mode
// Reference gradient for the discrete adjoint: the run w0 -> nsteps SSP-RK3
// steps (src/mod_advance.t:249-267, getbc after every stage) with a frozen
// dt sequence, in dual numbers seeded with the direction (dw0, dgamma), and
// the loss sum over interior cells of mask * rho^2.  Returns the loss and its
// directional derivative; w_final (optional) receives the final values.
// Not reentrant (the gamma seed is a process-wide static).
int orc_dual_run(const orc_cfg *cfg, const int *domain_nx, const double *xprobmin, const double *xprobmax,
                 const int *bc, const double *w0, const double *dw0, double dgamma, int nsteps,
                 const double *dts, const double *mask, int nthreads, double *loss, double *dloss,
                 double *w_final) {
  orc_grid *g = orc_grid_create(cfg, domain_nx, xprobmin, xprobmax, bc);
  const size_t n = g->bsize * g->nblocks;
  std::vector<Dual> reg[3];
  for (int r = 0; r < 3; ++r) reg[r].assign(n, Dual(0.0));
  for (size_t p = 0; p < n; ++p) reg[0][p] = Dual(w0[p], dw0 ? dw0[p] : 0.0);
  g_dual_dgamma = dgamma;
  const State &s = g->s;
  const size_t bs = g->bsize;
  double b11, b22, b33, a21, a31;
  if (s.c.ssprk_order == 2) { b11 = 0.5; b22 = 0.5; b33 = 1.0 / 3.0; a21 = 0.0; a31 = 1.0 / 3.0; }
  else { b11 = 1.0; b22 = 1.0 / 4.0; b33 = 2.0 / 3.0; a21 = 3.0 / 4.0; a31 = 1.0 / 3.0; }
  const double a22 = 1.0 - a21, a33 = 1.0 - a31;
  auto advect = [&](int ra, int rb, double qdt, double dtfactor) {
    int st = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic) reduction(| : st)
#endif
    for (int ib = 0; ib < g->nblocks; ++ib) {
      Arr<Dual> a(s.g, s.x.nw), b(s.g, s.x.nw);
      std::copy(reg[ra].begin() + bs * ib, reg[ra].begin() + bs * (ib + 1), a.d.begin());
      std::copy(reg[rb].begin() + bs * ib, reg[rb].begin() + bs * (ib + 1), b.d.begin());
      st |= finite_volume(s, a, b, qdt, dtfactor, g->dx, 0.0);
      std::copy(b.d.begin(), b.d.end(), reg[rb].begin() + bs * ib);
    }
    getbc_reg(*g, reg[rb]);
    return st;
  };
  auto combine = [&](int dst, double a, int ra, double b, int rb) {
    for (size_t p = 0; p < n; ++p) reg[dst][p] = Dual(a) * reg[ra][p] + Dual(b) * reg[rb][p];
  };
  int st = 0;
  getbc_reg(*g, reg[0]);
  for (int it = 0; it < nsteps; ++it) {
    const double dt = dts[it];
    reg[1] = reg[0];
    st |= advect(0, 1, b11 * dt, b11);
    combine(2, a21, 0, a22, 1);
    st |= advect(1, 2, b22 * dt, b22);
    combine(0, a31, 0, a33, 2);
    st |= advect(2, 0, b33 * dt, b33);
  }
  Dual L(0.0);
  const Geo &geo = s.g;
  const Ix &x = s.x;
  for (int ib = 0; ib < g->nblocks; ++ib) {
    Arr<Dual> a(geo, x.nw);
    std::copy(reg[0].begin() + bs * ib, reg[0].begin() + bs * (ib + 1), a.d.begin());
    Box ixM;
    for (int d = 0; d < 3; ++d) {
      ixM.lo[d] = d < s.c.ndim ? s.c.nghost : 0;
      ixM.hi[d] = d < s.c.ndim ? s.c.nghost + s.c.block_nx[d] - 1 : 0;
    }
    const double *mb = mask + bs / x.nw * ib;
    forbox(ixM, [&](int i, int j, int k) {
      const double m = mb[geo.idx(i, j, k)];
      if (m != 0.0) L = L + Dual(m) * (W(a, x.rho) * W(a, x.rho));
    });
  }
  if (w_final)
    for (size_t p = 0; p < n; ++p) w_final[p] = reg[0][p].v;
  *loss = L.v;
  *dloss = L.d;
  g_dual_dgamma = 0.0;
  orc_grid_destroy(g);
  return st;
}


// ---------------------------------------------------------------- Löhner estimator
// lohner_grid (src/amr/mod_errest.t:63-200), refine_criterion 3, without B0
// and user variables: on one ghosted block (>= 2 ghost layers filled).
// error[interior cells] (optional), *refine / *coarsen as the reference sets
// refine(igrid) / coarsen(igrid).
void orc_lohner_block(const orc_cfg *cfg, const double *wblk, const double *weight, const int *logflag,
                      double wavefilter, double threshold, double derefine, int level, int refine_max_level,
                      double *error_out, int *refine, int *coarsen) {
  State s = make_state(*cfg);
  const Geo &g = s.g;
  const int nw = s.x.nw, ndim = s.c.ndim;
  Arr<double> w = wrap_in(g, nw, wblk);
  const double epsilon = 1.0e-6;
  Box ixM, ix;
  for (int d = 0; d < 3; ++d) {
    ixM.lo[d] = d < ndim ? s.c.nghost : 0;
    ixM.hi[d] = d < ndim ? s.c.nghost + s.c.block_nx[d] - 1 : 0;
    ix.lo[d] = d < ndim ? ixM.lo[d] - 1 : 0;
    ix.hi[d] = d < ndim ? ixM.hi[d] + 1 : 0;
  }
  Arr<double> error(g, 1), numer(g, 1), denom(g, 1), tmp(g, 1), tmp2(g, 1);
  forbox(ixM, [&](int i, int j, int k) { error(i, j, k, 0) = 0.0; });
  auto val = [&](int iw, int i, int j, int k) {
    const double v = w(i, j, k, iw);
    return logflag[iw] ? std::log10(v) : v;
  };
  for (int iw = 0; iw < nw; ++iw) {
    if (weight[iw] == 0.0) continue;
    forbox(ixM, [&](int i, int j, int k) { numer(i, j, k, 0) = 0.0; denom(i, j, k, 0) = 0.0; });
    for (int d = 0; d < ndim; ++d) {
      int e[3] = {0, 0, 0};
      e[d] = 1;
      forbox(ix, [&](int i, int j, int k) {
        tmp(i, j, k, 0) = val(iw, i + e[0], j + e[1], k + e[2]) - val(iw, i - e[0], j - e[1], k - e[2]);
      });
      for (int d2 = 0; d2 < ndim; ++d2) {
        int f[3] = {0, 0, 0};
        f[d2] = 1;
        forbox(ixM, [&](int i, int j, int k) {
          const double q = tmp(i + f[0], j + f[1], k + f[2], 0) - tmp(i - f[0], j - f[1], k - f[2], 0);
          numer(i, j, k, 0) = numer(i, j, k, 0) + q * q;
        });
      }
    }
    for (int d = 0; d < ndim; ++d) {
      int e[3] = {0, 0, 0};
      e[d] = 1;
      // tmp = |w| over the block; tmp2 on the extended box; then tmp on ixM
      Box all;
      for (int q = 0; q < 3; ++q) { all.lo[q] = 0; all.hi[q] = g.n[q] - 1; }
      forbox(all, [&](int i, int j, int k) { tmp(i, j, k, 0) = std::fabs(val(iw, i, j, k)); });
      forbox(ix, [&](int i, int j, int k) {
        tmp2(i, j, k, 0) = tmp(i + e[0], j + e[1], k + e[2], 0) + tmp(i - e[0], j - e[1], k - e[2], 0);
      });
      forbox(ixM, [&](int i, int j, int k) {
        const double c = val(iw, i, j, k);
        tmp(i, j, k, 0) = std::fabs(val(iw, i + 2 * e[0], j + 2 * e[1], k + 2 * e[2]) - c) +
                          std::fabs(c - val(iw, i - 2 * e[0], j - 2 * e[1], k - 2 * e[2]));
      });
      for (int d2 = 0; d2 < ndim; ++d2) {
        int f[3] = {0, 0, 0};
        f[d2] = 1;
        forbox(ixM, [&](int i, int j, int k) {
          const double q = tmp(i, j, k, 0) + wavefilter * (tmp2(i + f[0], j + f[1], k + f[2], 0) +
                                                           tmp2(i - f[0], j - f[1], k - f[2], 0));
          denom(i, j, k, 0) = denom(i, j, k, 0) + q * q;
        });
      }
    }
    forbox(ixM, [&](int i, int j, int k) {
      error(i, j, k, 0) = error(i, j, k, 0) +
                          weight[iw] * std::sqrt(numer(i, j, k, 0) / std::max(denom(i, j, k, 0), epsilon));
    });
  }
  bool any_ref = false, all_coa = true;
  size_t q = 0;
  forbox(ixM, [&](int i, int j, int k) {
    const double e = error(i, j, k, 0);
    if (error_out) error_out[q++] = e;
    if (e >= threshold) any_ref = true;
    else if (!(e <= derefine * threshold)) all_coa = false;
    if (e >= threshold) all_coa = false;
  });
  *refine = any_ref && level < refine_max_level;
  *coarsen = all_coa && level > 1;
}


// ---------------------------------------------------------------- AMR grid
// A static hierarchy of leaf blocks (2:1 balanced), restating the reference's
// multi-level getbc (src/mod_ghostcells_update.t:350-578: coarsen_grid into
// psc, bc_fill_srl, bc_fill_restrict, bc_fill_prolong, gc_prolong /
// bc_prolong / interpolation_linear, with the index maps of init_bc 116-305,
// nghostcells 2, interpolation order 2, conserved-variable restriction and
// prolongation) and the flux correction (store_flux / fix_conserve,
// src/mod_fix_conserve.t:465-648) applied after every stage, as advect1 does
// (src/mod_advance.t:611-666).  Physical boundaries: periodic only.
}  // extern "C"

namespace orc {

enum { NT_BOUNDARY = 0, NT_COARSE = 1, NT_SIBLING = 2, NT_FINE = 3 };

struct AmrGrid {
  long it = 0;  // steps advanced (the parity of a split step's sweep order)
  State s;      // block state (block_nx bn)
  State sc;     // coarse representation (block_nx bn/2)
  int ndim, nb;
  int bn = 16;  // block edge (block_nx, the same in every direction)
  int nbase[3];
  double xmin[3], xmax[3];
  int bc[6];                                  // ORC_BC_* per side
  std::vector<int> level, ig;                 // ig[3*b]
  std::vector<int> ntype, nid;                // [b*27]
  std::vector<int> child;                     // [(b*27+q)*8 + cbits]
  std::vector<double> reg[4];                 // ghosted blocks
  std::vector<double> psc;                    // [b] coarse representation
  std::vector<std::vector<double>> pflux;     // [b*6 + 2*d + side]
  size_t bsize, csize;
  double dx(int b, int d) const { return (xmax[d] - xmin[d]) / (nbase[d] * double(bn) * double(1 << (level[b] - 1))); }
  double bxmin(int b, int d) const { return xmin[d] + ig[3 * b + d] * double(bn) * dx(b, d); }
};

inline int q27(const int *dd) { return (dd[0] + 1) + 3 * ((dd[1] + 1) + 3 * (dd[2] + 1)); }

// Index maps of init_bc (1-based, nghostcells 2, block bn, coarse bn/2).
struct AmrMaps {
  int srlS[3][2], srlR[3][2];   // by i+1: ixS_srl / ixR_srl
  int rS[3][2], rR[4][2];       // ixS_r by i+1, ixR_r by n_inc 0..3
  int pS[4][2], pR[4][2];       // ixS_p, ixR_p by inc / n_inc 0..3
};

inline AmrMaps amr_maps(int bn) {
  const int ng = 2, nx = bn, nxCo = bn / 2, ixMmin = ng + 1, ixMmax = ng + nx, ixGmax = nx + 2 * ng;
  const int ixCoMmin = ng + 1, ixCoMmax = ng + nxCo;
  const int ngCo = (ng + 1) / 2, io = 2;
  AmrMaps m;
  const int srlS[3][2] = {{ixMmin, ixMmin - 1 + ng}, {ixMmin, ixMmax}, {ixMmax + 1 - ng, ixMmax}};
  const int srlR[3][2] = {{1, ng}, {ixMmin, ixMmax}, {ixMmax + 1, ixGmax}};
  const int rS[3][2] = {{ixCoMmin, ixCoMmin - 1 + ng}, {ixCoMmin, ixCoMmax}, {ixCoMmax + 1 - ng, ixCoMmax}};
  const int rR[4][2] = {{1, ng}, {ixMmin, ixMmin - 1 + nxCo}, {ixMmin + nxCo, ixMmax}, {ixMmax + 1, ixGmax}};
  const int pS[4][2] = {{ixMmin - (io - 1), ixMmin - 1 + ngCo + (io - 1)},
                        {ixMmin - (io - 1), ixMmin - 1 + nxCo + ngCo + (io - 1)},
                        {ixMmin + nxCo - ngCo - (io - 1), ixMmax + (io - 1)},
                        {ixMmax + 1 - ngCo - (io - 1), ixMmax + (io - 1)}};
  const int pR[4][2] = {{ixCoMmin - ngCo - (io - 1), ng + (io - 1)},
                        {ixCoMmin - (io - 1), ixCoMmax + ngCo + (io - 1)},
                        {ixCoMmin - ngCo - (io - 1), ixCoMmax + (io - 1)},
                        {ixCoMmax + 1 - (io - 1), ixCoMmax + ngCo + (io - 1)}};
  std::memcpy(m.srlS, srlS, sizeof(srlS)); std::memcpy(m.srlR, srlR, sizeof(srlR));
  std::memcpy(m.rS, rS, sizeof(rS)); std::memcpy(m.rR, rR, sizeof(rR));
  std::memcpy(m.pS, pS, sizeof(pS)); std::memcpy(m.pR, pR, sizeof(pR));
  return m;
}

// copy a 1-based box of block-geometry ga array a into geometry gb array b
inline void copy_box(const Geo &ga, const double *a, const int lo_a[3], const Geo &gb, double *b, const int lo_b[3],
                     const int ext[3], int nw) {
  for (int iw = 0; iw < nw; ++iw)
    for (int k = 0; k < ext[2]; ++k)
      for (int j = 0; j < ext[1]; ++j)
        for (int i = 0; i < ext[0]; ++i)
          b[gb.idx(lo_b[0] - 1 + i, lo_b[1] - 1 + j, lo_b[2] - 1 + k) + gb.cells * (size_t)iw] =
              a[ga.idx(lo_a[0] - 1 + i, lo_a[1] - 1 + j, lo_a[2] - 1 + k) + ga.cells * (size_t)iw];
}

void amr_getbc(AmrGrid &G, std::vector<double> &reg) {
  const int nd = G.ndim, nw = G.s.x.nw;
  const Geo &g = G.s.g, &gc = G.sc.g;
  const AmrMaps M = amr_maps(G.bn);
  auto has = [&](int b, int t) {
    for (int q = 0; q < 27; ++q) if (q != 13 && G.ntype[b * 27 + q] == t) return true;
    return false;
  };
  auto dir_of = [&](int q, int *dd) { dd[0] = q % 3 - 1; dd[1] = (q / 3) % 3 - 1; dd[2] = q / 9 - 1; };
  auto valid_q = [&](int q) {
    int dd[3];
    dir_of(q, dd);
    if (q == 13) return false;
    for (int d = nd; d < 3; ++d) if (dd[d]) return false;
    return true;
  };
  // coarsen_grid of blocks with a coarser neighbour: psc interior
  for (int b = 0; b < G.nb; ++b) {
    if (!has(b, NT_COARSE)) continue;
    const double *w = &reg[G.bsize * b];
    double *wc = &G.psc[G.csize * b];
    const double cofi = 1.0 / double(1 << nd);
    const int half = G.bn / 2;
    for (int iw = 0; iw < nw; ++iw)
      for (int kc = 0; kc < (nd > 2 ? half : 1); ++kc)
        for (int jc = 0; jc < (nd > 1 ? half : 1); ++jc)
          for (int icc = 0; icc < half; ++icc) {
            const int i0 = 2 + 2 * icc, j0 = nd > 1 ? 2 + 2 * jc : 0, k0 = nd > 2 ? 2 + 2 * kc : 0;
            double sum = 0.0;
            bool first = true;
            for (int kk = 0; kk < (nd > 2 ? 2 : 1); ++kk)
              for (int jj = 0; jj < (nd > 1 ? 2 : 1); ++jj)
                for (int ii = 0; ii < 2; ++ii) {
                  const double v = w[g.idx(i0 + ii, j0 + jj, k0 + kk) + g.cells * (size_t)iw];
                  sum = first ? v : sum + v;
                  first = false;
                }
            wc[gc.idx(2 + icc, nd > 1 ? 2 + jc : 0, nd > 2 ? 2 + kc : 0) + gc.cells * (size_t)iw] = sum * cofi;
          }
  }
  // same-level copies (bc_fill_srl) and restriction into coarser neighbours (bc_fill_restrict)
  for (int b = 0; b < G.nb; ++b)
    for (int q = 0; q < 27; ++q) {
      if (!valid_q(q)) continue;
      int dd[3];
      dir_of(q, dd);
      const int t = G.ntype[b * 27 + q];
      if (t == NT_SIBLING) {
        const int nbk = G.nid[b * 27 + q];
        int lo_s[3], lo_r[3], ext[3];
        for (int d = 0; d < 3; ++d) {
          if (d < nd) {
            lo_s[d] = M.srlS[dd[d] + 1][0];
            lo_r[d] = M.srlR[-dd[d] + 1][0];
            ext[d] = M.srlS[dd[d] + 1][1] - M.srlS[dd[d] + 1][0] + 1;
          } else { lo_s[d] = lo_r[d] = 1; ext[d] = 1; }
        }
        copy_box(g, &reg[G.bsize * b], lo_s, g, &reg[G.bsize * nbk], lo_r, ext, nw);
      } else if (t == NT_COARSE) {
        int ic[3] = {1, 1, 1};
        bool ok = true;
        for (int d = 0; d < nd; ++d) {
          ic[d] = 1 + (G.ig[3 * b + d] % 2);
          if (!(dd[d] == 0 || dd[d] == 2 * ic[d] - 3)) ok = false;
        }
        if (!ok) continue;
        const int nbk = G.nid[b * 27 + q];
        int lo_s[3], lo_r[3], ext[3];
        for (int d = 0; d < 3; ++d) {
          if (d < nd) {
            const int ninc = -2 * dd[d] + ic[d];
            lo_s[d] = M.rS[dd[d] + 1][0];
            lo_r[d] = M.rR[ninc][0];
            ext[d] = M.rS[dd[d] + 1][1] - M.rS[dd[d] + 1][0] + 1;
          } else { lo_s[d] = lo_r[d] = 1; ext[d] = 1; }
        }
        copy_box(gc, &G.psc[G.csize * b], lo_s, g, &reg[G.bsize * nbk], lo_r, ext, nw);
      }
    }
  // physical boundaries of every block before the coarse values are sent:
  // the coarse neighbours' ghost cells across the domain boundary are then
  // those of the current data (the reference leaves whatever the register
  // held from its previous fill there)
  auto phys_all = [&]() {
    for (int b = 0; b < G.nb; ++b)
      bc_phys_block(G.s, G.bc, &reg[G.bsize * b],
                    [&](int di, int dj, int dk) { return G.ntype[b * 27 + dir_index(di, dj, dk)] == NT_BOUNDARY; });
  };
  phys_all();
  // coarse values into the finer neighbours' psc (bc_fill_prolong)
  for (int b = 0; b < G.nb; ++b)
    for (int q = 0; q < 27; ++q) {
      if (!valid_q(q) || G.ntype[b * 27 + q] != NT_FINE) continue;
      int dd[3];
      dir_of(q, dd);
      int icr[3][2];
      for (int d = 0; d < 3; ++d) {
        if (d < nd) { icr[d][0] = 1 + (1 - dd[d]) / 2; icr[d][1] = 2 - (1 + dd[d]) / 2; }
        else { icr[d][0] = icr[d][1] = 1; }
      }
      for (int c2 = icr[2][0]; c2 <= icr[2][1]; ++c2)
        for (int c1 = icr[1][0]; c1 <= icr[1][1]; ++c1)
          for (int c0 = icr[0][0]; c0 <= icr[0][1]; ++c0) {
            const int ic[3] = {c0, c1, c2};
            const int cbits = (c0 - 1) + 2 * (nd > 1 ? c1 - 1 : 0) + 4 * (nd > 2 ? c2 - 1 : 0);
            const int chd = G.child[(b * 27 + q) * 8 + cbits];
            int lo_s[3], lo_r[3], ext[3];
            for (int d = 0; d < 3; ++d) {
              if (d < nd) {
                const int inc = 2 * dd[d] + ic[d], ninc = ic[d] - dd[d];
                lo_s[d] = M.pS[inc][0];
                lo_r[d] = M.pR[ninc][0];
                ext[d] = M.pS[inc][1] - M.pS[inc][0] + 1;
              } else { lo_s[d] = lo_r[d] = 1; ext[d] = 1; }
            }
            copy_box(g, &reg[G.bsize * b], lo_s, gc, &G.psc[G.csize * chd], lo_r, ext, nw);
          }
    }
  // prolongation of ghost cells from coarser neighbours (gc_prolong -> bc_prolong -> interpolation_linear)
  for (int b = 0; b < G.nb; ++b)
    for (int q = 0; q < 27; ++q) {
      if (!valid_q(q) || G.ntype[b * 27 + q] != NT_COARSE) continue;
      int dd[3];
      dir_of(q, dd);
      int lo[3] = {1, 1, 1}, hi[3] = {1, 1, 1};
      double dxF[3] = {1, 1, 1}, dxC[3] = {1, 1, 1}, invC[3] = {1, 1, 1}, xFmin[3] = {0, 0, 0}, xCmin[3] = {0, 0, 0};
      for (int d = 0; d < nd; ++d) {
        lo[d] = M.srlR[dd[d] + 1][0];
        hi[d] = M.srlR[dd[d] + 1][1];
        dxF[d] = G.dx(b, d);
        dxC[d] = 2.0 * dxF[d];
        invC[d] = 1.0 / dxC[d];
        xFmin[d] = G.bxmin(b, d) - 2.0 * dxF[d];
        xCmin[d] = G.bxmin(b, d) - 2.0 * dxC[d];
      }
      const double *wc = &G.psc[G.csize * b];
      double *w = &reg[G.bsize * b];
      for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
          for (int i = lo[0]; i <= hi[0]; ++i) {
            const int ixF[3] = {i, j, k};
            int ixC[3] = {1, 1, 1};
            double eta[3] = {0, 0, 0};
            for (int d = 0; d < nd; ++d) {
              const double xF = xFmin[d] + (double(ixF[d]) - 0.5) * dxF[d];
              ixC[d] = int((xF - xCmin[d]) * invC[d]) + 1;
              const double xC = xCmin[d] + (double(ixC[d]) - 0.5) * dxC[d];
              eta[d] = (xF - xC) * invC[d];
            }
            for (int iw = 0; iw < nw; ++iw) {
              auto C = [&](int a, int bb, int cc) {
                return wc[gc.idx(a - 1, nd > 1 ? bb - 1 : 0, nd > 2 ? cc - 1 : 0) + gc.cells * (size_t)iw];
              };
              const double c0 = C(ixC[0], ixC[1], ixC[2]);
              double slope[3] = {0, 0, 0};
              for (int d = 0; d < nd; ++d) {
                int h[3] = {ixC[0], ixC[1], ixC[2]}, jx[3] = {ixC[0], ixC[1], ixC[2]};
                h[d] -= 1;
                jx[d] += 1;
                const double slopeL = c0 - C(h[0], h[1], h[2]);
                const double slopeR = C(jx[0], jx[1], jx[2]) - c0;
                const double slopeC = 0.5 * (slopeR + slopeL);
                const double signC = std::copysign(1.0, slopeC);
                slope[d] = signC * std::max(0.0, std::min(std::min(std::fabs(slopeC), signC * slopeL), signC * slopeR));
              }
              // psc(ixCo) + (slope_1 eta_1) + (slope_2 eta_2) + ..., left to right
              double v = c0;
              for (int d = 0; d < nd; ++d) v = v + slope[d] * eta[d];
              w[g.idx(ixF[0] - 1, nd > 1 ? ixF[1] - 1 : 0, nd > 2 ? ixF[2] - 1 : 0) + g.cells * (size_t)iw] = v;
            }
          }
    }
  phys_all();  // fill_boundary_after_gc
}

// store_flux (src/mod_fix_conserve.t:597-648) for one block from its scaled face fluxes.
void amr_store_flux(AmrGrid &G, int b, const std::vector<Arr<double>> &fC) {
  const int nd = G.ndim, nw = G.s.x.nw;
  for (int d = 0; d < nd; ++d)
    for (int side = 0; side < 2; ++side) {
      int dd[3] = {0, 0, 0};
      dd[d] = side ? 1 : -1;
      const int t = G.ntype[b * 27 + q27(dd)];
      std::vector<double> &pf = G.pflux[b * 6 + 2 * d + side];
      const int t1 = (d + 1) % 3 < nd ? (d + 1) % 3 : -1, t2 = (d + 2) % 3 < nd ? (d + 2) % 3 : -1;
      // tangential dimensions in increasing order
      int ta = -1, tb = -1;
      for (int e = 0; e < nd; ++e) if (e != d) { if (ta < 0) ta = e; else tb = e; }
      (void)t1; (void)t2;
      const int iface = side ? G.bn + 1 : 1;  // 0-based face index: right face of cell iface
      if (t == NT_FINE) {
        const int n1 = ta >= 0 ? G.bn : 1, n2 = tb >= 0 ? G.bn : 1;
        pf.assign((size_t)nw * n1 * n2, 0.0);
        for (int iw = 0; iw < nw; ++iw)
          for (int b2 = 0; b2 < n2; ++b2)
            for (int a1 = 0; a1 < n1; ++a1) {
              int c[3] = {0, 0, 0};
              c[d] = iface;
              if (ta >= 0) c[ta] = 2 + a1;
              if (tb >= 0) c[tb] = 2 + b2;
              const double f = fC[d](c[0], c[1], c[2], iw);
              pf[((size_t)iw * n2 + b2) * n1 + a1] = side ? f : -f;
            }
      } else if (t == NT_COARSE) {
        const int n1 = ta >= 0 ? G.bn / 2 : 1, n2 = tb >= 0 ? G.bn / 2 : 1;
        pf.assign((size_t)nw * n1 * n2, 0.0);
        for (int iw = 0; iw < nw; ++iw)
          for (int b2 = 0; b2 < n2; ++b2)
            for (int a1 = 0; a1 < n1; ++a1) {
              double sum = 0.0;
              bool first = true;
              for (int y = 0; y < (tb >= 0 ? 2 : 1); ++y)
                for (int x = 0; x < (ta >= 0 ? 2 : 1); ++x) {
                  int c[3] = {0, 0, 0};
                  c[d] = iface;
                  if (ta >= 0) c[ta] = 2 + 2 * a1 + x;
                  if (tb >= 0) c[tb] = 2 + 2 * b2 + y;
                  const double f = fC[d](c[0], c[1], c[2], iw);
                  sum = first ? f : sum + f;
                  first = false;
                }
              pf[((size_t)iw * n2 + b2) * n1 + a1] = side ? -sum : sum;
            }
      } else {
        pf.clear();
      }
    }
}

// fix_conserve (src/mod_fix_conserve.t:465-595) on one register.
void amr_fix_conserve(AmrGrid &G, std::vector<double> &reg) {
  const int nd = G.ndim, nw = G.s.x.nw;
  const Geo &g = G.s.g;
  const double cofi = 1.0 / double(1 << nd);
  for (int b = 0; b < G.nb; ++b)
    for (int d = G.s.idlo; d <= G.s.idhi; ++d)  // idim^LIM
      for (int side = 0; side < 2; ++side) {
        int dd[3] = {0, 0, 0};
        dd[d] = side ? 1 : -1;
        const int q = q27(dd);
        if (G.ntype[b * 27 + q] != NT_FINE) continue;
        int ta = -1, tb = -1;
        for (int e = 0; e < nd; ++e) if (e != d) { if (ta < 0) ta = e; else tb = e; }
        const int ix = side ? G.bn + 1 : 2;  // 0-based boundary cell
        double *w = &reg[G.bsize * b];
        const std::vector<double> &pc = G.pflux[b * 6 + 2 * d + side];
        const int n1 = ta >= 0 ? G.bn : 1, n2 = tb >= 0 ? G.bn : 1;
        for (int iw = 0; iw < nw; ++iw)
          for (int b2 = 0; b2 < n2; ++b2)
            for (int a1 = 0; a1 < n1; ++a1) {
              int c[3] = {0, 0, 0};
              c[d] = ix;
              if (ta >= 0) c[ta] = 2 + a1;
              if (tb >= 0) c[tb] = 2 + b2;
              double &v = w[g.idx(c[0], c[1], c[2]) + g.cells * (size_t)iw];
              v = v - pc[((size_t)iw * n2 + b2) * n1 + a1];
            }
        // children adjacent across the face
        for (int c2 = 1; c2 <= (tb >= 0 ? 2 : 1); ++c2)
          for (int c1 = 1; c1 <= (ta >= 0 ? 2 : 1); ++c1) {
            int ic[3] = {1, 1, 1};
            ic[d] = side ? 1 : 2;
            if (ta >= 0) ic[ta] = c1;
            if (tb >= 0) ic[tb] = c2;
            const int cbits = (ic[0] - 1) + 2 * (nd > 1 ? ic[1] - 1 : 0) + 4 * (nd > 2 ? ic[2] - 1 : 0);
            const int chd = G.child[(b * 27 + q) * 8 + cbits];
            const std::vector<double> &pf = G.pflux[chd * 6 + 2 * d + (1 - side)];
            const int half = G.bn / 2;
            const int m1 = ta >= 0 ? half : 1, m2 = tb >= 0 ? half : 1;
            for (int iw = 0; iw < nw; ++iw)
              for (int b2 = 0; b2 < m2; ++b2)
                for (int a1 = 0; a1 < m1; ++a1) {
                  int c[3] = {0, 0, 0};
                  c[d] = ix;
                  if (ta >= 0) c[ta] = 2 + (c1 - 1) * half + a1;
                  if (tb >= 0) c[tb] = 2 + (c2 - 1) * half + b2;
                  double &v = w[g.idx(c[0], c[1], c[2]) + g.cells * (size_t)iw];
                  v = v + pf[((size_t)iw * m2 + b2) * m1 + a1] * cofi;
                }
          }
      }
}

// fix == false: the Predictor_Corrector predictor (no flux fix; hancock for
// tvdlf, which stores no fluxes).
int amr_advect1(AmrGrid &G, int ra, int rb, double qdt, double dtfactor, double cmax_global, int nthreads,
                bool fix = true) {
  const bool hk = !fix && (G.s.c.flux_scheme == ORC_FS_TVDLF || G.s.c.flux_scheme == ORC_FS_TVDMU);
  int st = 0;
  const size_t bs = G.bsize;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic) reduction(| : st)
#endif
  for (int b = 0; b < G.nb; ++b) {
    Arr<double> a = wrap_in(G.s.g, G.s.x.nw, &G.reg[ra][bs * b]);
    Arr<double> w = wrap_in(G.s.g, G.s.x.nw, &G.reg[rb][bs * b]);
    double dxb[3];
    for (int d = 0; d < 3; ++d) dxb[d] = d < G.ndim ? G.dx(b, d) : 1.0;
    std::vector<Arr<double>> fc;
    int jumps = 0;  // faces with a coarser or finer neighbour
    for (int d = 0; d < G.ndim; ++d)
      for (int side = 0; side < 2; ++side) {
        int dd[3] = {0, 0, 0};
        dd[d] = side ? 1 : -1;
        const int t = G.ntype[b * 27 + q27(dd)];
        if (t == NT_COARSE || t == NT_FINE) jumps |= 1 << (2 * d + side);
      }
    if (hk) {
      st |= hancock(G.s, a, w, qdt, dxb, cmax_global, jumps);
      std::memcpy(&G.reg[rb][bs * b], w.d.data(), sizeof(double) * bs);
      continue;
    }
    st |= finite_volume(G.s, a, w, qdt, dtfactor, dxb, cmax_global, &fc, jumps);
    std::memcpy(&G.reg[rb][bs * b], w.d.data(), sizeof(double) * bs);
    amr_store_flux(G, b, fc);
  }
  if (fix) amr_fix_conserve(G, G.reg[rb]);
  amr_getbc(G, G.reg[rb]);
  return st;
}

}  // namespace orc

extern "C" {

orc_amr *orc_amr_create(const orc_cfg *cfg, const int *nbase, const double *xprobmin, const double *xprobmax,
                        int nleaf, const int *leaf /* [nleaf][4]: level, ig0, ig1, ig2 */, const int *bc) {
  AmrGrid *G = new AmrGrid();
  for (int q = 0; q < 6; ++q) G->bc[q] = (bc && q < 2 * cfg->ndim) ? bc[q] : ORC_BC_PERIODIC;
  G->s = make_state(*cfg);
  G->bn = cfg->block_nx[0];
  orc_cfg c8 = *cfg;
  for (int d = 0; d < 3; ++d) c8.block_nx[d] = d < cfg->ndim ? G->bn / 2 : 1;
  G->sc = make_state(c8);
  G->ndim = cfg->ndim;
  G->nb = nleaf;
  for (int d = 0; d < 3; ++d) {
    G->nbase[d] = d < cfg->ndim ? nbase[d] : 1;
    G->xmin[d] = d < cfg->ndim ? xprobmin[d] : 0.0;
    G->xmax[d] = d < cfg->ndim ? xprobmax[d] : 1.0;
  }
  G->level.resize(nleaf);
  G->ig.resize(3 * (size_t)nleaf);
  std::map<std::array<int, 4>, int> key;
  for (int b = 0; b < nleaf; ++b) {
    G->level[b] = leaf[4 * b];
    for (int d = 0; d < 3; ++d) G->ig[3 * b + d] = d < cfg->ndim ? leaf[4 * b + 1 + d] : 0;
    key[{G->level[b], G->ig[3 * b], G->ig[3 * b + 1], G->ig[3 * b + 2]}] = b;
  }
  auto find = [&](int l, const int *jg) -> int {
    auto it = key.find({l, jg[0], jg[1], jg[2]});
    return it == key.end() ? -1 : it->second;
  };
  G->ntype.assign(27 * (size_t)nleaf, NT_BOUNDARY);
  G->nid.assign(27 * (size_t)nleaf, -1);
  G->child.assign(27 * 8 * (size_t)nleaf, -1);
  const int nd = cfg->ndim;
  for (int b = 0; b < nleaf; ++b) {
    const int l = G->level[b];
    for (int q = 0; q < 27; ++q) {
      int dd[3] = {q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1};
      bool ok = true;
      int jg[3] = {0, 0, 0};
      bool outside = false;
      for (int d = 0; d < 3; ++d) {
        if (d >= nd) { if (dd[d]) ok = false; continue; }
        const int nl = G->nbase[d] << (l - 1);
        const int j = G->ig[3 * b + d] + dd[d];
        if ((j < 0 || j >= nl) && G->bc[2 * d + (j < 0 ? 0 : 1)] != ORC_BC_PERIODIC) outside = true;
        jg[d] = (j % nl + nl) % nl;
      }
      if (!ok || outside) continue;  // outside: a physical boundary
      if (q == 13) { G->ntype[b * 27 + q] = NT_SIBLING; G->nid[b * 27 + q] = b; continue; }
      int s2 = find(l, jg);
      if (s2 >= 0) { G->ntype[b * 27 + q] = NT_SIBLING; G->nid[b * 27 + q] = s2; continue; }
      int pg[3] = {jg[0] / 2, nd > 1 ? jg[1] / 2 : 0, nd > 2 ? jg[2] / 2 : 0};
      int cb = l > 1 ? find(l - 1, pg) : -1;
      if (cb >= 0) { G->ntype[b * 27 + q] = NT_COARSE; G->nid[b * 27 + q] = cb; continue; }
      G->ntype[b * 27 + q] = NT_FINE;
      for (int cbits = 0; cbits < 8; ++cbits) {
        int cg[3] = {2 * jg[0] + (cbits & 1), nd > 1 ? 2 * jg[1] + ((cbits >> 1) & 1) : 0,
                     nd > 2 ? 2 * jg[2] + ((cbits >> 2) & 1) : 0};
        if ((nd < 2 && (cbits & 2)) || (nd < 3 && (cbits & 4))) continue;
        G->child[(b * 27 + q) * 8 + cbits] = find(l + 1, cg);
      }
    }
  }
  G->bsize = G->s.g.cells * (size_t)G->s.x.nw;
  G->csize = G->sc.g.cells * (size_t)G->s.x.nw;
  for (int r = 0; r < 4; ++r) G->reg[r].assign(G->bsize * nleaf, 0.0);
  G->psc.assign(G->csize * nleaf, 0.0);
  G->pflux.assign(6 * (size_t)nleaf, {});
  return reinterpret_cast<orc_amr *>(G);
}

void orc_amr_destroy(orc_amr *a) { delete reinterpret_cast<AmrGrid *>(a); }

int orc_amr_neighbors(const orc_amr *a, int *ntype, int *nid, int *child) {
  const AmrGrid *G = reinterpret_cast<const AmrGrid *>(a);
  std::memcpy(ntype, G->ntype.data(), sizeof(int) * G->ntype.size());
  std::memcpy(nid, G->nid.data(), sizeof(int) * G->nid.size());
  if (child) std::memcpy(child, G->child.data(), sizeof(int) * G->child.size());
  return G->nb;
}

void orc_amr_set_block(orc_amr *a, int b, const double *w) {
  AmrGrid *G = reinterpret_cast<AmrGrid *>(a);
  std::memcpy(&G->reg[0][G->bsize * b], w, sizeof(double) * G->bsize);
}

void orc_amr_get_block(const orc_amr *a, int reg, int b, double *w) {
  const AmrGrid *G = reinterpret_cast<const AmrGrid *>(a);
  std::memcpy(w, &G->reg[reg][G->bsize * b], sizeof(double) * G->bsize);
}

void orc_amr_getbc(orc_amr *a) {
  AmrGrid *G = reinterpret_cast<AmrGrid *>(a);
  amr_getbc(*G, G->reg[0]);
}

int orc_amr_getdt(orc_amr *a, double *dt, double *cmax_global) {
  AmrGrid *G = reinterpret_cast<AmrGrid *>(a);
  double dtmin = bigdouble, cmx = 0.0;
  double a2m[3] = {0.0, 0.0, 0.0};
  int st = 0;
  for (int b = 0; b < G->nb; ++b) {
    Arr<double> w = wrap_in(G->s.g, G->s.x.nw, &G->reg[0][G->bsize * b]);
    double dxb[3];
    for (int d = 0; d < 3; ++d) dxb[d] = d < G->ndim ? G->dx(b, d) : 1.0;
    double dtn;
    st |= getdt_block(G->s, w, dxb, &dtn, &cmx);
    dtmin = std::min(dtmin, dtn);
    if (G->s.c.schmid_global) a2max_block(G->s, w, dxb, a2m);
  }
  if (G->s.c.schmid_global)
    for (int d = 0; d < 3; ++d) G->s.c.schmid_rad[d] = a2m[d];
  *dt = dtmin;
  *cmax_global = cmx;
  return st;
}

// One stage reg_a -> reg_b (reg_b holds the RK base combination on entry),
// flux correction and multi-level getbc on reg_b.
int orc_amr_advect1(orc_amr *a, int ra, int rb, double qdt, double dtfactor, double cmax_global, int nthreads) {
  return amr_advect1(*reinterpret_cast<AmrGrid *>(a), ra, rb, qdt, dtfactor, cmax_global, nthreads);
}

void orc_amr_combine_reg(orc_amr *a, int dst, double ca, int ra, double cb, int rb) {
  AmrGrid *G = reinterpret_cast<AmrGrid *>(a);
  for (size_t p = 0; p < G->reg[dst].size(); ++p) G->reg[dst][p] = ca * G->reg[ra][p] + cb * G->reg[rb][p];
}

static int amr_advance_stepper(orc_amr *a, double dt, double cmax_global, int nthreads) {
  AmrGrid *G = reinterpret_cast<AmrGrid *>(a);
  if (G->s.c.time_stepper == 2)
    return twostep(
        G->s.c, dt,
        [&](int ra, int rb, double qdt, double f, bool fix) {
          return amr_advect1(*G, ra, rb, qdt, f, cmax_global, nthreads, fix);
        },
        [&](int d, int s2) { G->reg[d] = G->reg[s2]; },
        [&](int d, double x, int ra, double y, int rb) { orc_amr_combine_reg(a, d, x, ra, y, rb); });
  if (G->s.c.time_stepper == 5)
    return fivestep(
        G->s.c, dt,
        [&](int ra, int rb, double qdt, double f) { return amr_advect1(*G, ra, rb, qdt, f, cmax_global, nthreads); },
        [&](int d, int s2) { G->reg[d] = G->reg[s2]; },
        [&](int d, double x, int ra, double y, int rb) { orc_amr_combine_reg(a, d, x, ra, y, rb); }, G->reg);
  if (G->s.c.time_stepper == 4)
    return fourstep(
        G->s.c, dt,
        [&](int ra, int rb, double qdt, double f) { return amr_advect1(*G, ra, rb, qdt, f, cmax_global, nthreads); },
        [&](int d, int s2) { G->reg[d] = G->reg[s2]; },
        [&](int d, double x, int ra, double y, int rb) { orc_amr_combine_reg(a, d, x, ra, y, rb); },
        [&]() { rk4_combine_regs(G->reg); });
  double b11, b22, b33, a21, a31;
  if (G->s.c.ssprk_order == 2) { b11 = 0.5; b22 = 0.5; b33 = 1.0 / 3.0; a21 = 0.0; a31 = 1.0 / 3.0; }
  else { b11 = 1.0; b22 = 1.0 / 4.0; b33 = 2.0 / 3.0; a21 = 3.0 / 4.0; a31 = 1.0 / 3.0; }
  int st = 0;
  G->reg[1] = G->reg[0];
  st |= amr_advect1(*G, 0, 1, b11 * dt, b11, cmax_global, nthreads);
  orc_amr_combine_reg(a, 2, a21, 0, 1.0 - a21, 1);
  st |= amr_advect1(*G, 1, 2, b22 * dt, b22, cmax_global, nthreads);
  orc_amr_combine_reg(a, 0, a31, 0, 1.0 - a31, 2);
  st |= amr_advect1(*G, 2, 0, b33 * dt, b33, cmax_global, nthreads);
  return st;
}

// advect with dimsplit (src/mod_advance.t:23-45): one full stepper per
// direction, increasing order on even steps (always with typedimsplit 'xy'),
// decreasing on odd steps ('xyyx').
extern "C++" {
template <class G, class Stepper>
static int split_advance(G &grid, State &s, Stepper stepper) {
  int st = 0;
  if (!s.c.dimsplit) {
    st = stepper();
  } else {
    const int nd = s.c.ndim;
    const bool fwd = s.c.dimsplit == 2 || (grid.it % 2) == 0;
    for (int q = 0; q < nd; ++q) {
      const int d = fwd ? q : nd - 1 - q;
      s.idlo = s.idhi = d;
      st |= stepper();
    }
    s.idlo = 0;
    s.idhi = nd - 1;
  }
  ++grid.it;
  return st;
}
}  // extern "C++"

int orc_grid_advance(orc_grid *g, double dt, double cmax_global, int nthreads) {
  return split_advance(*g, g->s, [&]() { return grid_advance_stepper(g, dt, cmax_global, nthreads); });
}

int orc_amr_advance(orc_amr *a, double dt, double cmax_global, int nthreads) {
  AmrGrid *G = reinterpret_cast<AmrGrid *>(a);
  return split_advance(*G, G->s, [&]() { return amr_advance_stepper(a, dt, cmax_global, nthreads); });
}

// prolong_2nd (src/amr/mod_refine.t:81-167) for a child of a refined block
// and coarsen_grid (src/amr/mod_coarsen.t:12-79) for a coarsened parent, on
// the old grid's ghosted register 0.
orc_amr *orc_amr_remap(const orc_amr *old, int nleaf, const int *leaf, const int *op) {
  const AmrGrid *O = reinterpret_cast<const AmrGrid *>(old);
  orc_amr *res = orc_amr_create(&O->s.c, O->nbase, O->xmin, O->xmax, nleaf, leaf, O->bc);
  AmrGrid *N = reinterpret_cast<AmrGrid *>(res);
  const Geo &g = O->s.g;
  const int nd = O->ndim, nw = O->s.x.nw;
  const double cofi = 1.0 / double(1 << nd);
  for (int b = 0; b < nleaf; ++b) {
    const int *o = op + 9 * (size_t)b;
    double *wn = &N->reg[0][N->bsize * b];
    if (o[0] == 0) {
      std::memcpy(wn, &O->reg[0][O->bsize * o[1]], sizeof(double) * O->bsize);
      continue;
    }
    const int bn = O->bn, half = bn / 2;
    for (int iw = 0; iw < nw; ++iw)
      for (int k = 0; k < (nd > 2 ? bn : 1); ++k)
        for (int j = 0; j < (nd > 1 ? bn : 1); ++j)
          for (int i = 0; i < bn; ++i) {
            const int F[3] = {i, j, k};
            double val;
            if (o[0] == 1) {
              const double *wc = &O->reg[0][O->bsize * o[1]];
              int co[3] = {0, 0, 0};  // 0-based ghosted index of the coarse cell
              for (int d = 0; d < nd; ++d) co[d] = 2 + half * ((o[2] >> d) & 1) + (F[d] >> 1);
              auto wco = [&](int a, int bb, int cc) { return wc[g.idx(a, bb, cc) + g.cells * (size_t)iw]; };
              const double c0 = wco(co[0], co[1], co[2]);
              double slope[3] = {0, 0, 0};
              for (int d = 0; d < nd; ++d) {
                int h[3] = {co[0], co[1], co[2]}, jx[3] = {co[0], co[1], co[2]};
                h[d] -= 1;
                jx[d] += 1;
                const double slopeL = c0 - wco(h[0], h[1], h[2]);
                const double slopeR = wco(jx[0], jx[1], jx[2]) - c0;
                const double slopeC = 0.5 * (slopeR + slopeL);
                const double signC = std::copysign(1.0, slopeC);
                slope[d] = signC * std::max(0.0, std::min(std::min(std::fabs(slopeC), signC * slopeL), signC * slopeR));
              }
              val = c0;
              for (int d = 0; d < nd; ++d) val = val + slope[d] * (0.5 * (double(F[d] & 1) - 0.5));
            } else {
              int cb = 0;
              for (int d = 0; d < nd; ++d) cb |= (F[d] >= half ? 1 : 0) << d;
              const double *wf = &O->reg[0][O->bsize * o[1 + cb]];
              double sum = 0.0;
              bool first = true;
              for (int kk = 0; kk < (nd > 2 ? 2 : 1); ++kk)
                for (int jj = 0; jj < (nd > 1 ? 2 : 1); ++jj)
                  for (int ii = 0; ii < 2; ++ii) {
                    const int fi = 2 + 2 * (F[0] % half) + ii, fj = nd > 1 ? 2 + 2 * (F[1] % half) + jj : 0,
                              fk = nd > 2 ? 2 + 2 * (F[2] % half) + kk : 0;
                    const double x = wf[g.idx(fi, fj, fk) + g.cells * (size_t)iw];
                    sum = first ? x : sum + x;
                    first = false;
                  }
              val = sum * cofi;
            }
            wn[g.idx(2 + i, nd > 1 ? 2 + j : 0, nd > 2 ? 2 + k : 0) + g.cells * (size_t)iw] = val;
          }
  }
  return res;
}

}  // extern "C"
