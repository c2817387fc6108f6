// Recompression of the hierarchical boundary matrix into an H2 matrix (nested cluster bases).
//
// tetmag compresses its double-layer matrix with H2Lib in two steps: a hierarchical matrix by
// cross approximation, then compress_hmatrix_h2matrix with a relative Euclidean truncation at
// 1e-5 (main/h2interface.c:315-369); the matvec is H2_mvp_sub (:77-95).  H2Lib is not vendored;
// this file restates the published algebraic recompression (S. Borm, "Efficient Numerical
// Methods for Non-local Operators", EMS 2010, ch. 6: orthogonal cluster bases from the total
// cluster basis matrices, nested through transfer matrices, then coupling matrices by projection)
// on the low-rank blocks U_b V_b^T that the device's cross approximation produced:
//
//   row basis     for every row cluster t, the left singular vectors of the matrix of every
//                 admissible block whose row cluster is t or an ancestor of t, restricted to the
//                 rows of t; kept down to eps times the largest singular value.  A leaf basis is explicit (|t| x k_t); a parent's is
//                 [V_t1 E_t1; V_t2 E_t2], the transfers E from the singular vectors of the same
//                 matrix projected onto the children's bases, so the Gram matrices of the
//                 parents are (k_t1 + k_t2) square and the bases stay nested.
//   column basis  the same with V_b for U_b.
//   coupling      S_b = (V_t^T U_b) (W_s^T V_b)^T, k_t x k_s.
//
// Everything works on Gram matrices: the total matrix of t is [U_b|t L_b] with L_b L_b^T =
// V_b^T V_b, so its Gram is sum_b w_b^2 U_b|t (V_b^T V_b) U_b|t^T, and only k x k Gram matrices
// of the factors and k_t x k_b projections V_t^T U_b|t travel up the tree.  Symmetric eigen-
// decompositions by cyclic Jacobi rotations (the matrices are at most 2 kmax square).
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <vector>

#include "tmb_host.h"

namespace tmb {

namespace {

// Eigen-decomposition of a symmetric n x n matrix (row-major a, destroyed) by cyclic Jacobi
// rotations: eigenvalues in w (descending), eigenvectors as the columns of v (column-major).
void sym_eig(int n, std::vector<double>& a, std::vector<double>& w, std::vector<double>& v) {
  v.assign(size_t(n) * n, 0.0);
  for (int i = 0; i < n; ++i) v[size_t(i) * n + i] = 1.0;
  auto A = [&](int i, int j) -> double& { return a[size_t(i) * n + j]; };
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        tot += A(i, j) * A(i, j);
        if (i != j) off += A(i, j) * A(i, j);
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A(p, q);
        if (std::fabs(apq) <= 1e-300) continue;
        const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {   // A <- J^T A J
          const double akp = A(k, p), akq = A(k, q);
          A(k, p) = c * akp - s * akq;
          A(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = A(p, k), aqk = A(q, k);
          A(p, k) = c * apk - s * aqk;
          A(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = v[size_t(p) * n + k], vkq = v[size_t(q) * n + k];
          v[size_t(p) * n + k] = c * vkp - s * vkq;
          v[size_t(q) * n + k] = s * vkp + c * vkq;
        }
      }
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int x, int y) { return A(x, x) > A(y, y); });
  std::vector<double> vs(size_t(n) * n);
  w.resize(n);
  for (int k = 0; k < n; ++k) {
    w[k] = A(order[k], order[k]);
    std::copy(v.begin() + size_t(order[k]) * n, v.begin() + size_t(order[k] + 1) * n, vs.begin() + size_t(k) * n);
  }
  v.swap(vs);
}

// number of eigenvalues kept: above eps^2 times the largest (relative Euclidean truncation of the
// singular values), positive, at most kmax
int truncate(const std::vector<double>& w, double eps, int kmax) {
  if (w.empty() || !(w[0] > 0.0)) return 0;
  int k = 0;
  while (k < int(w.size()) && k < kmax && w[k] > eps * eps * w[0]) ++k;
  return k;
}

struct Dense {  // column-major r x c
  int r = 0, c = 0;
  std::vector<double> a;
  Dense() = default;
  Dense(int rr, int cc) : r(rr), c(cc), a(size_t(rr) * cc, 0.0) {}
  double& operator()(int i, int j) { return a[i + size_t(j) * r]; }
  double operator()(int i, int j) const { return a[i + size_t(j) * r]; }
};

// One side (rows or columns) of the recompression.
class SideBuilder {
 public:
  // fac(q): the block's factor on this side (U for rows, V for columns), column-major with leading
  // dimension ld(q); gram(q): the Gram matrix of the other factor (k x k); blocks(c): the blocks
  // whose cluster on this side is c; origin(q): that cluster's first position
  SideBuilder(const HPartition& P, const std::vector<std::vector<int>>& blocks, const std::vector<const double*>& fac,
              const std::vector<int>& ld, const std::vector<int>& rank, const std::vector<int>& origin,
              const std::vector<Dense>& gram, const std::vector<double>& w2, double eps, int kmax, H2Side& out,
              std::vector<Dense>& own)
      : P_(P), blocks_(blocks), fac_(fac), ld_(ld), rank_(rank), origin_(origin), gram_(gram), w2_(w2), eps_(eps),
        kmax_(kmax), out_(out), own_(own) {
    const size_t nc = P.clusters.size();
    out_.k.assign(nc, 0);
    out_.leaf_basis.assign(nc, {});
    out_.transfer.assign(nc, {});
    parent_.assign(nc, -1);
    for (size_t c = 0; c < nc; ++c)
      for (int ch : P.clusters[c].child)
        if (ch >= 0) parent_[ch] = int(c);
  }
  void run() {
    std::vector<int> none;
    rec(0, none, 0);
  }

 private:
  const HPartition& P_;
  const std::vector<std::vector<int>>& blocks_;
  const std::vector<const double*>& fac_;
  const std::vector<int>& ld_;
  const std::vector<int>& rank_;
  const std::vector<int>& origin_;
  const std::vector<Dense>& gram_;
  const std::vector<double>& w2_;
  double eps_;
  int kmax_;
  H2Side& out_;
  std::vector<Dense>& own_;
  std::vector<int> parent_;

  // returns, for every block of Qall = Qup + blocks(c), the projection of its factor restricted
  // to c onto c's basis (k_c x k_q)
  std::vector<Dense> rec(int c, const std::vector<int>& Qup, int depth) {
    const HCluster& C = P_.clusters[c];
    std::vector<int> Qall = Qup;
    Qall.insert(Qall.end(), blocks_[c].begin(), blocks_[c].end());
    std::vector<Dense> proj(Qall.size());
    if (C.child[0] < 0) {
      const int m = C.end - C.begin;
      // Gram of the weighted total matrix restricted to c
      std::vector<double> G(size_t(m) * m, 0.0);
      std::vector<double> t;
      for (int q : Qall) {
        const int k = rank_[q];
        if (k == 0) continue;
        const double* F = fac_[q] + (C.begin - origin_[q]);
        const int l = ld_[q];
        const Dense& g = gram_[q];
        t.assign(size_t(m) * k, 0.0);   // t = F|c * g  (m x k)
        for (int j = 0; j < k; ++j)
          for (int p = 0; p < k; ++p) {
            const double gv = g(p, j);
            for (int i = 0; i < m; ++i) t[i + size_t(j) * m] += F[i + size_t(p) * l] * gv;
          }
        const double wq = w2_[q];
        for (int i = 0; i < m; ++i)
          for (int i2 = 0; i2 < m; ++i2) {
            double s = 0.0;
            for (int j = 0; j < k; ++j) s += t[i + size_t(j) * m] * F[i2 + size_t(j) * l];
            G[size_t(i) * m + i2] += wq * s;
          }
      }
      std::vector<double> ev, vec;
      sym_eig(m, G, ev, vec);
      const int kc = truncate(ev, eps_, std::min(kmax_, m));
      out_.k[c] = kc;
      out_.leaf_basis[c].assign(vec.begin(), vec.begin() + size_t(kc) * m);   // m x kc, column-major
      for (size_t a = 0; a < Qall.size(); ++a) {
        const int q = Qall[a], k = rank_[q];
        Dense P(kc, k);
        const double* F = fac_[q] + (C.begin - origin_[q]);
        const int l = ld_[q];
        for (int j = 0; j < k; ++j)
          for (int b = 0; b < kc; ++b) {
            double s = 0.0;
            for (int i = 0; i < m; ++i) s += vec[i + size_t(b) * m] * F[i + size_t(j) * l];
            P(b, j) = s;
          }
        proj[a] = std::move(P);
      }
    } else {
      std::vector<Dense> p1, p2;
      if (depth < 6) {
#pragma omp task shared(p1, Qall)
        p1 = rec(C.child[0], Qall, depth + 1);
#pragma omp task shared(p2, Qall)
        p2 = rec(C.child[1], Qall, depth + 1);
#pragma omp taskwait
      } else {
        p1 = rec(C.child[0], Qall, depth + 1);
        p2 = rec(C.child[1], Qall, depth + 1);
      }
      const int k1 = out_.k[C.child[0]], k2 = out_.k[C.child[1]], n = k1 + k2;
      std::vector<double> G(size_t(n) * n, 0.0);
      for (size_t a = 0; a < Qall.size(); ++a) {
        const int q = Qall[a], k = rank_[q];
        if (k == 0 || n == 0) continue;
        Dense X(n, k);
        for (int j = 0; j < k; ++j) {
          for (int i = 0; i < k1; ++i) X(i, j) = p1[a](i, j);
          for (int i = 0; i < k2; ++i) X(k1 + i, j) = p2[a](i, j);
        }
        const Dense& g = gram_[q];
        Dense T(n, k);   // X g
        for (int j = 0; j < k; ++j)
          for (int p = 0; p < k; ++p) {
            const double gv = g(p, j);
            for (int i = 0; i < n; ++i) T(i, j) += X(i, p) * gv;
          }
        const double wq = w2_[q];
        for (int i = 0; i < n; ++i)
          for (int i2 = 0; i2 < n; ++i2) {
            double s = 0.0;
            for (int j = 0; j < k; ++j) s += T(i, j) * X(i2, j);
            G[size_t(i) * n + i2] += wq * s;
          }
      }
      std::vector<double> ev, vec;
      int kc = 0;
      if (n > 0) {
        sym_eig(n, G, ev, vec);
        kc = truncate(ev, eps_, kmax_);
      }
      out_.k[c] = kc;
      // transfers: child basis coefficients of the parent's basis vectors
      for (int s = 0; s < 2; ++s) {
        const int ch = C.child[s], kk = s == 0 ? k1 : k2, o = s == 0 ? 0 : k1;
        std::vector<double>& E = out_.transfer[ch];
        E.assign(size_t(kk) * kc, 0.0);   // kk x kc, column-major
        for (int j = 0; j < kc; ++j)
          for (int i = 0; i < kk; ++i) E[i + size_t(j) * kk] = vec[o + i + size_t(j) * n];
      }
      for (size_t a = 0; a < Qall.size(); ++a) {
        const int q = Qall[a], k = rank_[q];
        Dense Pq(kc, k);
        for (int j = 0; j < k; ++j)
          for (int b = 0; b < kc; ++b) {
            double s = 0.0;
            for (int i = 0; i < k1; ++i) s += vec[i + size_t(b) * n] * p1[a](i, j);
            for (int i = 0; i < k2; ++i) s += vec[k1 + i + size_t(b) * n] * p2[a](i, j);
            Pq(b, j) = s;
          }
        proj[a] = std::move(Pq);
      }
    }
    // the projections of this cluster's own blocks (the last ones of Qall) are kept for the
    // coupling matrices
    for (size_t a = Qup.size(); a < Qall.size(); ++a) own_[Qall[a]] = proj[a];
    proj.resize(Qup.size());
    return proj;
  }
};

}  // namespace

void h2_build_host(const HPartition& P, const H2Factors& F, double eps, int kmax, H2Host& out) {
  const int nf = int(P.far.size());
  if (int(F.U.size()) != nf || int(F.V.size()) != nf) throw std::runtime_error("h2_build_host: factor count");
  const size_t nc = P.clusters.size();
  std::vector<std::vector<int>> rows(nc), cols(nc);
  std::vector<int> rorigin(nf), corigin(nf);
  for (int q = 0; q < nf; ++q) {
    rows[P.far[q].first].push_back(q);
    cols[P.far[q].second].push_back(q);
    rorigin[q] = P.clusters[P.far[q].first].begin;
    corigin[q] = P.clusters[P.far[q].second].begin;
  }
  // Gram matrices of both factors and the block weights 1 / ||U V^T||_F^2
  std::vector<Dense> gU(nf), gV(nf);
  std::vector<double> w2(nf, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int q = 0; q < nf; ++q) {
    const int k = F.rank[q];
    const int m = P.clusters[P.far[q].first].end - rorigin[q];
    const int n = P.clusters[P.far[q].second].end - corigin[q];
    Dense a(k, k), b(k, k);
    for (int i = 0; i < k; ++i)
      for (int j = 0; j <= i; ++j) {
        double su = 0.0, sv = 0.0;
        for (int r = 0; r < m; ++r) su += F.U[q][r + size_t(i) * F.ldu[q]] * F.U[q][r + size_t(j) * F.ldu[q]];
        for (int r = 0; r < n; ++r) sv += F.V[q][r + size_t(i) * F.ldv[q]] * F.V[q][r + size_t(j) * F.ldv[q]];
        a(i, j) = a(j, i) = su;
        b(i, j) = b(j, i) = sv;
      }
    double fro = 0.0;
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j) fro += a(i, j) * b(j, i);
    // unweighted total matrices (H2Lib's relative Euclidean truncation of the cluster's total
    // matrix): weak far blocks may lose relatively more, their absolute error stays below eps
    // times the cluster's largest singular value
    w2[q] = fro > 0.0 ? 1.0 : 0.0;
    gU[q] = std::move(a);
    gV[q] = std::move(b);
  }
  std::vector<Dense> ownU(nf), ownV(nf);
  out = H2Host{};
  {
    SideBuilder rb(P, rows, F.U, F.ldu, F.rank, rorigin, gV, w2, eps, kmax, out.row, ownU);
    SideBuilder cb(P, cols, F.V, F.ldv, F.rank, corigin, gU, w2, eps, kmax, out.col, ownV);
#pragma omp parallel
#pragma omp single
    {
      rb.run();
      cb.run();
    }
  }
  // couplings S_q = (V_t^T U_q)(W_s^T V_q)^T
  out.coupling.assign(nf, {});
#pragma omp parallel for schedule(dynamic, 64)
  for (int q = 0; q < nf; ++q) {
    const Dense& a = ownU[q];
    const Dense& b = ownV[q];
    const int kt = a.r, ks = b.r, k = F.rank[q];
    std::vector<double> S(size_t(kt) * ks, 0.0);   // kt x ks, column-major
    for (int j = 0; j < ks; ++j)
      for (int i = 0; i < kt; ++i) {
        double s = 0.0;
        for (int p = 0; p < k; ++p) s += a(i, p) * b(j, p);
        S[i + size_t(j) * kt] = s;
      }
    out.coupling[q] = std::move(S);
  }
}

}  // namespace tmb
