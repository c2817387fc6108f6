// Hierarchical-matrix partition of the boundary double-layer matrix (host side).
//
// tetmag compresses its BEM matrix with H2Lib (main/h2interface.c:315-399: geometric
// cluster tree with leaf size clf = 32, admissibility parameter eta = 2, block-wise
// low-rank approximation then H2 recompression).  H2Lib is not vendored (branch
// "collocation", external/CMakeLists.txt:47-55), so this is an independent H-matrix with
// the same cluster parameters:
//   cluster tree   recursive median bisection of the boundary nodes along the longest
//                  bounding-box axis, down to <= leaf nodes; nodes are renumbered so every
//                  cluster is a contiguous index range
//   admissibility  min(diam tau, diam sigma) <= eta * dist(tau, sigma) on bounding boxes
//   blocks         admissible pairs of at most max_block rows and columns become low-rank
//                  blocks (adaptive cross approximation on the device, k_hmatrix.cu; larger
//                  admissible pairs are subdivided to bound the work of one CTA);
//                  inadmissible leaf pairs stay dense.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <stdexcept>
#include <vector>

#include "tmb_host.h"

namespace tmb {

namespace {

struct Box {
  double lo[3], hi[3];
};

Box bounds(const double* xyz, const int* idx, int b, int e) {
  Box B;
  for (int d = 0; d < 3; ++d) {
    B.lo[d] = 1e300;
    B.hi[d] = -1e300;
  }
  for (int i = b; i < e; ++i)
    for (int d = 0; d < 3; ++d) {
      const double v = xyz[3 * idx[i] + d];
      B.lo[d] = std::min(B.lo[d], v);
      B.hi[d] = std::max(B.hi[d], v);
    }
  return B;
}

double diam(const HCluster& c) {
  double s = 0.0;
  for (int d = 0; d < 3; ++d) s += (c.hi[d] - c.lo[d]) * (c.hi[d] - c.lo[d]);
  return std::sqrt(s);
}

double dist(const HCluster& a, const HCluster& b) {
  double s = 0.0;
  for (int d = 0; d < 3; ++d) {
    const double g = std::max(0.0, std::max(a.lo[d] - b.hi[d], b.lo[d] - a.hi[d]));
    s += g * g;
  }
  return std::sqrt(s);
}

// Bisection: while a cluster holds nodes of several orientation classes (`cls`, may be null)
// it is split between classes; then along the longest extent of the split coordinates `sc`
// (nsc per node).  The stored boxes are spatial (admissibility).
int build_clusters(const double* xyz, const double* sc, int nsc, const int* cls, std::vector<int>& perm, int b,
                   int e, int leaf, std::vector<HCluster>& out) {
  const int id = int(out.size());
  out.push_back(HCluster{});
  const Box B = bounds(xyz, perm.data(), b, e);
  HCluster c;
  c.begin = b;
  c.end = e;
  for (int d = 0; d < 3; ++d) {
    c.lo[d] = B.lo[d];
    c.hi[d] = B.hi[d];
  }
  c.child[0] = c.child[1] = -1;
  if (e - b > leaf && cls) {
    // several orientation classes: split at the class boundary nearest to the median
    int cmin = cls[perm[b]], cmax = cmin;
    for (int i = b; i < e; ++i) {
      cmin = std::min(cmin, cls[perm[i]]);
      cmax = std::max(cmax, cls[perm[i]]);
    }
    if (cmin != cmax) {
      std::stable_sort(perm.begin() + b, perm.begin() + e, [&](int x, int y) { return cls[x] < cls[y]; });
      int cut = -1, best_gap = e - b;
      for (int i = b + 1; i < e; ++i)
        if (cls[perm[i]] != cls[perm[i - 1]] && std::abs(i - (b + e) / 2) < best_gap) {
          best_gap = std::abs(i - (b + e) / 2);
          cut = i;
        }
      c.child[0] = build_clusters(xyz, sc, nsc, cls, perm, b, cut, leaf, out);
      c.child[1] = build_clusters(xyz, sc, nsc, cls, perm, cut, e, leaf, out);
      out[id] = c;
      return id;
    }
  }
  if (e - b > leaf) {
    int ax = 0;
    double best = -1.0;
    for (int d = 0; d < nsc; ++d) {
      double lo = 1e300, hi = -1e300;
      for (int i = b; i < e; ++i) {
        const double v = sc[size_t(nsc) * perm[i] + d];
        lo = std::min(lo, v);
        hi = std::max(hi, v);
      }
      if (hi - lo > best) {
        best = hi - lo;
        ax = d;
      }
    }
    const int mid = b + (e - b) / 2;
    std::nth_element(perm.begin() + b, perm.begin() + mid, perm.begin() + e,
                     [&](int x, int y) { return sc[size_t(nsc) * x + ax] < sc[size_t(nsc) * y + ax]; });
    c.child[0] = build_clusters(xyz, sc, nsc, cls, perm, b, mid, leaf, out);
    c.child[1] = build_clusters(xyz, sc, nsc, cls, perm, mid, e, leaf, out);
  }
  out[id] = c;
  return id;
}

void build_blocks(const std::vector<HCluster>& C, int t, int s, double eta, int max_block, HPartition& P) {
  const HCluster& a = C[t];
  const HCluster& b = C[s];
  const bool la = a.child[0] < 0, lb = b.child[0] < 0;
  const bool small = std::max(a.end - a.begin, b.end - b.begin) <= max_block || (la && lb);
  if (small && std::min(diam(a), diam(b)) <= eta * dist(a, b)) {
    P.far.push_back({t, s});
    return;
  }
  if (la && lb) {
    P.near.push_back({t, s});
  } else if (la) {
    build_blocks(C, t, b.child[0], eta, max_block, P);
    build_blocks(C, t, b.child[1], eta, max_block, P);
  } else if (lb) {
    build_blocks(C, a.child[0], s, eta, max_block, P);
    build_blocks(C, a.child[1], s, eta, max_block, P);
  } else {
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) build_blocks(C, a.child[i], b.child[j], eta, max_block, P);
  }
}

}  // namespace

void h_partition(const double* bxyz, const double* bnrm, int nb, int leaf, double eta, int max_block,
                 HPartition& P) {
  if (nb <= 0) throw std::runtime_error("h_partition: no boundary nodes");
  P = HPartition{};
  P.perm.resize(nb);
  std::iota(P.perm.begin(), P.perm.end(), 0);
  P.clusters.reserve(size_t(4) * nb / std::max(leaf, 1) + 8);
  // orientation class of a node: its normal's dominant axis and sign (6 classes)
  std::vector<int> cls;
  if (bnrm) {
    cls.resize(nb);
    for (int i = 0; i < nb; ++i) {
      int ax = 0;
      for (int d = 1; d < 3; ++d)
        if (std::fabs(bnrm[3 * i + d]) > std::fabs(bnrm[3 * i + ax])) ax = d;
      cls[i] = 2 * ax + (bnrm[3 * i + ax] < 0.0 ? 1 : 0);
    }
  }
  build_clusters(bxyz, bxyz, 3, bnrm ? cls.data() : nullptr, P.perm, 0, nb, leaf, P.clusters);
  build_blocks(P.clusters, 0, 0, eta, max_block, P);
  // near blocks sorted by row cluster so one CTA per leaf row cluster can own its rows
  std::sort(P.near.begin(), P.near.end(), [&](const std::pair<int, int>& x, const std::pair<int, int>& y) {
    return P.clusters[x.first].begin < P.clusters[y.first].begin ||
           (P.clusters[x.first].begin == P.clusters[y.first].begin &&
            P.clusters[x.second].begin < P.clusters[y.second].begin);
  });
  std::sort(P.far.begin(), P.far.end(), [&](const std::pair<int, int>& x, const std::pair<int, int>& y) {
    return x.first < y.first || (x.first == y.first && x.second < y.second);
  });
}

}  // namespace tmb
