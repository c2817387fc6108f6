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
//   blocks         admissible pairs become low-rank blocks (adaptive cross approximation
//                  on the device, k_hmatrix.cu); inadmissible leaf pairs stay dense.
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

int build_clusters(const double* xyz, std::vector<int>& perm, int b, int e, int leaf, std::vector<HCluster>& out) {
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
  if (e - b > leaf) {
    int ax = 0;
    for (int d = 1; d < 3; ++d)
      if (B.hi[d] - B.lo[d] > B.hi[ax] - B.lo[ax]) ax = d;
    const int mid = b + (e - b) / 2;
    std::nth_element(perm.begin() + b, perm.begin() + mid, perm.begin() + e,
                     [&](int x, int y) { return xyz[3 * x + ax] < xyz[3 * y + ax]; });
    c.child[0] = build_clusters(xyz, perm, b, mid, leaf, out);
    c.child[1] = build_clusters(xyz, perm, mid, e, leaf, out);
  }
  out[id] = c;
  return id;
}

void build_blocks(const std::vector<HCluster>& C, int t, int s, double eta, HPartition& P) {
  const HCluster& a = C[t];
  const HCluster& b = C[s];
  if (std::min(diam(a), diam(b)) <= eta * dist(a, b)) {
    P.far.push_back({t, s});
    return;
  }
  const bool la = a.child[0] < 0, lb = b.child[0] < 0;
  if (la && lb) {
    P.near.push_back({t, s});
  } else if (la) {
    build_blocks(C, t, b.child[0], eta, P);
    build_blocks(C, t, b.child[1], eta, P);
  } else if (lb) {
    build_blocks(C, a.child[0], s, eta, P);
    build_blocks(C, a.child[1], s, eta, P);
  } else {
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) build_blocks(C, a.child[i], b.child[j], eta, P);
  }
}

}  // namespace

void h_partition(const double* bxyz, int nb, int leaf, double eta, HPartition& P) {
  if (nb <= 0) throw std::runtime_error("h_partition: no boundary nodes");
  P = HPartition{};
  P.perm.resize(nb);
  std::iota(P.perm.begin(), P.perm.end(), 0);
  P.clusters.reserve(size_t(4) * nb / std::max(leaf, 1) + 8);
  build_clusters(bxyz, P.perm, 0, nb, leaf, P.clusters);
  build_blocks(P.clusters, 0, 0, eta, P);
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
