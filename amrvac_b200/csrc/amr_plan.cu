// Host-side tree decision of a regrid (no device work): amr_coarsen_refine
// with proper_nesting (src/amr/mod_coarsen_refine.t:20-319) on a tree of
// leaves (level, ig).
//
//   1. refinement flags of leaves below the finest level, coarsening flags of
//      leaves above level 1;
//   2. proper nesting, levels from fine to coarse: a leaf of level L flagged
//      for refinement flags the leaves of level L-1 next to its parent on the
//      parent's sides it touches (directions ic-2..ic-1 per dimension; none
//      across a physical boundary);
//   3. refinement wins over coarsening;
//   4. sibling groups, finer levels first: a group coarsens only when all
//      2^d siblings are flagged leaves and no neighbour across the siblings'
//      outer sides is a leaf that refines, or a refined block whose first
//      child is not a leaf flagged for coarsening; a group that fails is
//      unflagged before coarser levels look at it;
//   5. the new leaves, sorted by (level, ig0, ig1, ig2), each with its origin
//      op (copy / child of a refined leaf / parent of coarsened leaves).
//
// The same decision is restated in Python (amrvac_b200/amr.py Tree.regrid);
// a test compares the two on random flags.
#include <algorithm>
#include <array>
#include <cstdint>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/amrvac_gpu.h"

namespace {

using Leaf = std::array<int, 4>;  // level, ig0, ig1, ig2

inline uint64_t key(int L, int i, int j, int k) {
  return (uint64_t(L) << 57) | (uint64_t(uint32_t(i) & 0x7ffffu) << 38) | (uint64_t(uint32_t(j) & 0x7ffffu) << 19) |
         uint64_t(uint32_t(k) & 0x7ffffu);
}
inline uint64_t key(const Leaf &t) { return key(t[0], t[1], t[2], t[3]); }
inline int d_or0(int nd, int d, const int *t) { return d < nd ? t[1 + d] : 0; }

struct Plan {
  int nd, max_level;
  int nbase[3];
  bool periodic[3];
  std::unordered_map<uint64_t, int> pos;     // leaf -> old index
  std::unordered_set<uint64_t> refined;      // non-leaf ancestors
  std::vector<Leaf> leaves;

  // index i of level L in dimension d inside the domain, or -1 across a
  // physical (non-periodic) boundary
  int wrap(int L, int d, int i) const {
    const int n = nbase[d] << (L - 1);
    if ((i < 0 || i >= n) && !periodic[d]) return -1;
    return ((i % n) + n) % n;
  }
  bool is_leaf(const Leaf &t) const { return pos.count(key(t)) != 0; }
};

}  // namespace

extern "C" int amrvac_amr_plan(int ndim, const int *nbase, const int *periodic, int max_level, int nleaf,
                               const int *leaf, const unsigned char *refine, const unsigned char *coarsen, int cap,
                               int *nnew, int *leaf_new, int *op) {
  if (ndim < 1 || ndim > 3 || !nbase || max_level < 1 || max_level > 20 || nleaf <= 0 || !leaf || !nnew)
    return AMRVAC_E_ARG;
  Plan P;
  P.nd = ndim;
  P.max_level = max_level;
  for (int d = 0; d < 3; ++d) {
    P.nbase[d] = d < ndim ? nbase[d] : 1;
    P.periodic[d] = d >= ndim || !periodic || periodic[d];
  }
  P.leaves.resize(nleaf);
  for (int b = 0; b < nleaf; ++b) {
    Leaf t = {leaf[4 * b], d_or0(ndim, 0, leaf + 4 * b), d_or0(ndim, 1, leaf + 4 * b), d_or0(ndim, 2, leaf + 4 * b)};
    if (t[0] < 1 || t[0] > max_level) return AMRVAC_E_ARG;
    P.leaves[b] = t;
    P.pos[key(t)] = b;
    for (int L2 = t[0] - 1; L2 >= 1; --L2) {
      const int s = t[0] - L2;
      P.refined.insert(key(L2, t[1] >> s, t[2] >> s, t[3] >> s));
    }
  }
  const int nd = ndim, nch = 1 << nd;
  std::unordered_set<uint64_t> ref, coa;
  int levmax = 1;
  for (int b = 0; b < nleaf; ++b) {
    const Leaf &t = P.leaves[b];
    levmax = std::max(levmax, t[0]);
    if (refine && refine[b] && t[0] < max_level) ref.insert(key(t));
    if (coarsen && coarsen[b] && t[0] > 1) coa.insert(key(t));
  }
  // proper nesting, refinement part
  auto lo_hi = [&](int d, int ic, int &lo, int &hi) {
    if (d >= nd) { lo = hi = 0; return; }
    lo = ic == 0 ? -1 : 0;
    hi = ic == 0 ? 0 : 1;
  };
  for (int L = std::min(levmax, max_level - 1); L >= 2; --L) {
    std::vector<Leaf> lev;
    for (const Leaf &t : P.leaves)
      if (t[0] == L && ref.count(key(t))) lev.push_back(t);
    for (const Leaf &t : lev) {
      int lo[3], hi[3];
      for (int d = 0; d < 3; ++d) lo_hi(d, t[1 + d] & 1, lo[d], hi[d]);
      for (int a = lo[2]; a <= hi[2]; ++a)
        for (int bb = lo[1]; bb <= hi[1]; ++bb)
          for (int c = lo[0]; c <= hi[0]; ++c) {
            if (!a && !bb && !c) continue;
            const int inp[3] = {c, bb, a};
            Leaf p = {L - 1, 0, 0, 0};
            bool inside = true;
            for (int d = 0; d < nd; ++d) {
              p[1 + d] = P.wrap(L - 1, d, (t[1 + d] >> 1) + inp[d]);
              inside = inside && p[1 + d] >= 0;
            }
            if (inside && P.is_leaf(p)) ref.insert(key(p));
          }
    }
  }
  for (uint64_t k : ref) coa.erase(k);
  // coarsening part: sibling groups, finer levels first
  std::unordered_map<uint64_t, std::vector<int>> groups;  // parent key -> kid indices
  std::vector<Leaf> parents;
  for (int b = 0; b < nleaf; ++b) {
    const Leaf &t = P.leaves[b];
    if (!coa.count(key(t))) continue;
    const Leaf par = {t[0] - 1, t[1] >> 1, t[2] >> 1, t[3] >> 1};
    auto it = groups.find(key(par));
    if (it == groups.end()) {
      groups[key(par)] = {b};
      parents.push_back(par);
    } else {
      it->second.push_back(b);
    }
  }
  std::sort(parents.begin(), parents.end(), [](const Leaf &x, const Leaf &y) {
    if (x[0] != y[0]) return x[0] > y[0];
    return std::lexicographical_compare(x.begin() + 1, x.end(), y.begin() + 1, y.end());
  });
  std::vector<std::pair<Leaf, std::vector<int>>> coarsened;
  for (const Leaf &par : parents) {
    std::vector<int> kids = groups[key(par)];
    auto cbits = [&](int b) {
      int c = 0;
      for (int d = 0; d < 3; ++d) c |= (P.leaves[b][1 + d] & 1) << d;
      return c;
    };
    std::sort(kids.begin(), kids.end(), [&](int x, int y) { return cbits(x) < cbits(y); });
    bool ok = (int)kids.size() == nch;
    for (size_t q = 0; ok && q < kids.size(); ++q) {
      const Leaf &t = P.leaves[kids[q]];
      int lo[3], hi[3];
      for (int d = 0; d < 3; ++d) lo_hi(d, t[1 + d] & 1, lo[d], hi[d]);
      for (int a = lo[2]; ok && a <= hi[2]; ++a)
        for (int bb = lo[1]; ok && bb <= hi[1]; ++bb)
          for (int c = lo[0]; ok && c <= hi[0]; ++c) {
            if (!a && !bb && !c) continue;
            const int inc[3] = {c, bb, a};
            Leaf nb = {t[0], 0, 0, 0};
            bool inside = true;
            for (int d = 0; d < nd; ++d) {
              nb[1 + d] = P.wrap(t[0], d, t[1 + d] + inc[d]);
              inside = inside && nb[1 + d] >= 0;
            }
            if (!inside) continue;  // a physical boundary: no neighbour
            if (P.is_leaf(nb)) {
              if (ref.count(key(nb))) ok = false;
            } else if (P.refined.count(key(nb))) {
              Leaf ch = {t[0] + 1, 0, 0, 0};
              for (int d = 0; d < nd; ++d) ch[1 + d] = 2 * nb[1 + d];
              if (!(P.is_leaf(ch) && coa.count(key(ch)))) ok = false;
            }
          }
    }
    if (ok) coarsened.push_back({par, kids});
    else
      for (int b : kids) coa.erase(key(P.leaves[b]));
  }
  // the new leaves with their origins
  std::vector<std::pair<Leaf, std::array<int, 9>>> out;
  std::vector<char> gone(nleaf, 0);
  for (auto &pc : coarsened) {
    std::array<int, 9> o{};
    o[0] = 2;
    for (size_t q = 0; q < pc.second.size(); ++q) {
      o[1 + q] = pc.second[q];
      gone[pc.second[q]] = 1;
    }
    out.push_back({pc.first, o});
  }
  for (int b = 0; b < nleaf; ++b) {
    if (gone[b]) continue;
    const Leaf &t = P.leaves[b];
    if (ref.count(key(t))) {
      for (int cb = 0; cb < nch; ++cb) {
        Leaf ch = {t[0] + 1, 0, 0, 0};
        for (int d = 0; d < nd; ++d) ch[1 + d] = 2 * t[1 + d] + ((cb >> d) & 1);
        std::array<int, 9> o{};
        o[0] = 1;
        o[1] = b;
        o[2] = cb;
        out.push_back({ch, o});
      }
    } else {
      std::array<int, 9> o{};
      o[1] = b;
      out.push_back({t, o});
    }
  }
  std::sort(out.begin(), out.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
  *nnew = (int)out.size();
  if ((int)out.size() > cap || !leaf_new || !op) return AMRVAC_E_ARG;
  for (size_t b = 0; b < out.size(); ++b) {
    for (int q = 0; q < 4; ++q) leaf_new[4 * b + q] = out[b].first[q];
    for (int q = 0; q < 9; ++q) op[9 * b + q] = out[b].second[q];
  }
  return 0;
}
