// Smoothed-aggregation AMG hierarchy, built on the host, applied on the device.
//
// tetmag preconditions its FEM solves with AMGCL's smoothed aggregation
// (main/AMGCLSolver.h:89-101; parameters main/AMGCLSolver.cpp:39-45:
// relax = 0.75, coarse_enough = 100, direct_coarse = false) and an ILU0
// relaxation.  AMGCL is not vendored (external/CMakeLists.txt:71-81, branch
// master, unpinned), so this is an independent implementation of the
// published method (Vanek, Mandel, Brezina, Computing 56 (1996) 179-196):
//   strength     |a_ij|^2 > eps^2 |a_ii a_jj|
//   aggregation  root + strong neighbours, then attach leftovers
//   tentative P  piecewise constant (null space = constants)
//   smoothed P   (I - w D_F^-1 A_F) P_tent, w = relax * 4/3 / rho(D_F^-1 A_F)
//   coarse A     P^T A P (Galerkin)
// Differences from AMGCL, chosen for a device V-cycle inside CG: the smoother
// is damped Jacobi (symmetric and parallel) instead of ILU0, the prolongation
// smoother takes relax = 1 (fewer PCG iterations under the Jacobi cycle than
// 0.75), and the coarsest level (<= coarse_enough unknowns) is solved exactly
// in FP64 with a dense inverse.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <stdexcept>
#include <vector>

#include "tmb_host.h"

namespace tmb {

void csr_transpose(const Csr& A, Csr& T) {
  T.nrows = A.ncols;
  T.ncols = A.nrows;
  T.ptr.assign(T.nrows + 1, 0);
  for (int64_t k = 0; k < A.nnz(); ++k) T.ptr[A.col[k] + 1]++;
  for (int i = 0; i < T.nrows; ++i) T.ptr[i + 1] += T.ptr[i];
  T.col.resize(A.nnz());
  T.val.resize(A.nnz());
  std::vector<int> pos(T.ptr.begin(), T.ptr.end() - 1);
  for (int i = 0; i < A.nrows; ++i)
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
      const int p = pos[A.col[k]]++;
      T.col[p] = i;
      T.val[p] = A.val[k];
    }
}

// Gustavson row-by-row product, two passes (symbolic, numeric), OpenMP over rows.
void csr_multiply(const Csr& A, const Csr& B, Csr& C) {
  if (A.ncols != B.nrows) throw std::runtime_error("csr_multiply: shape mismatch");
  C.nrows = A.nrows;
  C.ncols = B.ncols;
  C.ptr.assign(C.nrows + 1, 0);
  std::vector<int> rowcount(C.nrows, 0);
#pragma omp parallel
  {
    std::vector<int> marker(B.ncols, -1);
#pragma omp for schedule(dynamic, 256)
    for (int i = 0; i < A.nrows; ++i) {
      int cnt = 0;
      for (int ka = A.ptr[i]; ka < A.ptr[i + 1]; ++ka) {
        const int j = A.col[ka];
        for (int kb = B.ptr[j]; kb < B.ptr[j + 1]; ++kb) {
          const int c = B.col[kb];
          if (marker[c] != i) { marker[c] = i; ++cnt; }
        }
      }
      rowcount[i] = cnt;
    }
  }
  for (int i = 0; i < C.nrows; ++i) C.ptr[i + 1] = C.ptr[i] + rowcount[i];
  C.col.resize(C.ptr[C.nrows]);
  C.val.resize(C.ptr[C.nrows]);
#pragma omp parallel
  {
    std::vector<int> pos(B.ncols, -1);
#pragma omp for schedule(dynamic, 256)
    for (int i = 0; i < A.nrows; ++i) {
      int base = C.ptr[i], len = 0;
      for (int ka = A.ptr[i]; ka < A.ptr[i + 1]; ++ka) {
        const int j = A.col[ka];
        const double a = A.val[ka];
        for (int kb = B.ptr[j]; kb < B.ptr[j + 1]; ++kb) {
          const int c = B.col[kb];
          if (pos[c] < base) {
            pos[c] = base + len;
            C.col[base + len] = c;
            C.val[base + len] = a * B.val[kb];
            ++len;
          } else {
            C.val[pos[c]] += a * B.val[kb];
          }
        }
      }
      // sort the row by column (keeps device gathers monotone)
      std::vector<std::pair<int, double>> tmp(len);
      for (int q = 0; q < len; ++q) tmp[q] = {C.col[base + q], C.val[base + q]};
      std::sort(tmp.begin(), tmp.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
      for (int q = 0; q < len; ++q) { C.col[base + q] = tmp[q].first; C.val[base + q] = tmp[q].second; }
      for (int q = 0; q < len; ++q) pos[C.col[base + q]] = -1;
    }
  }
}

namespace {

std::vector<double> diagonal(const Csr& A) {
  std::vector<double> d(A.nrows, 0.0);
  for (int i = 0; i < A.nrows; ++i)
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
      if (A.col[k] == i) d[i] += A.val[k];
  return d;
}

// Largest eigenvalue of D^-1 A by power iteration (deterministic start vector).
double spectral_radius(const Csr& A, const std::vector<double>& dinv, int iters = 12) {
  const int n = A.nrows;
  if (n == 0) return 1.0;
  std::vector<double> x(n), y(n);
  uint64_t s = 0x9E3779B97F4A7C15ull;
  for (int i = 0; i < n; ++i) {
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    x[i] = double(s >> 11) * (1.0 / 9007199254740992.0) + 0.5;
  }
  double rho = 1.0;
  for (int it = 0; it < iters; ++it) {
    double nx = 0.0, ny = 0.0;
#pragma omp parallel for reduction(+ : nx, ny)
    for (int i = 0; i < n; ++i) {
      double acc = 0.0;
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) acc += A.val[k] * x[A.col[k]];
      y[i] = dinv[i] * acc;
      nx += x[i] * x[i];
      ny += y[i] * y[i];
    }
    rho = std::sqrt(ny / std::max(nx, 1e-300));
    const double inv = 1.0 / std::sqrt(std::max(ny, 1e-300));
    for (int i = 0; i < n; ++i) x[i] = y[i] * inv;
  }
  return rho;
}

void dense_inverse(std::vector<double>& a, int n) {
  // Gauss-Jordan with partial pivoting, FP64, row-major in place.
  std::vector<double> inv(size_t(n) * n, 0.0);
  for (int i = 0; i < n; ++i) inv[size_t(i) * n + i] = 1.0;
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(a[size_t(r) * n + c]) > std::fabs(a[size_t(piv) * n + c])) piv = r;
    if (a[size_t(piv) * n + c] == 0.0) throw std::runtime_error("AMG coarsest matrix is singular");
    if (piv != c)
      for (int k = 0; k < n; ++k) {
        std::swap(a[size_t(c) * n + k], a[size_t(piv) * n + k]);
        std::swap(inv[size_t(c) * n + k], inv[size_t(piv) * n + k]);
      }
    const double d = 1.0 / a[size_t(c) * n + c];
    for (int k = 0; k < n; ++k) { a[size_t(c) * n + k] *= d; inv[size_t(c) * n + k] *= d; }
#pragma omp parallel for schedule(static) if (n >= 256)
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = a[size_t(r) * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; ++k) {
        a[size_t(r) * n + k] -= f * a[size_t(c) * n + k];
        inv[size_t(r) * n + k] -= f * inv[size_t(c) * n + k];
      }
    }
  }
  a.swap(inv);
}

}  // namespace

void amg_build(const Csr& A0, const AmgParams& prm, AmgHierarchy& H) {
  const auto t0 = std::chrono::steady_clock::now();
  H.levels.clear();
  Csr A = A0;
  for (int lev = 0;; ++lev) {
    AmgLevel L;
    const int n = A.nrows;
    std::vector<double> d = diagonal(A);
    for (int i = 0; i < n; ++i)
      if (!(d[i] > 0.0)) throw std::runtime_error("AMG: non-positive diagonal");

    bool coarsest = (n <= prm.coarse_enough) || (lev + 1 >= prm.max_levels);
    std::vector<int> agg;
    int naggr = 0;
    std::vector<char> strong;
    if (!coarsest) {
      // --- strength of connection
      strong.assign(A.nnz(), 0);
      std::vector<int> nstrong(n, 0);
      const double e2 = prm.eps_strong * prm.eps_strong;
      for (int i = 0; i < n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
          const int j = A.col[k];
          if (j == i) continue;
          const double v = A.val[k];
          if (v * v > e2 * std::fabs(d[i] * d[j])) { strong[k] = 1; ++nstrong[i]; }
        }
      // --- aggregation: -2 undecided, -1 isolated (never aggregated)
      agg.assign(n, -2);
      for (int i = 0; i < n; ++i)
        if (nstrong[i] == 0) agg[i] = -1;
      for (int i = 0; i < n; ++i) {  // pass 1: roots whose strong neighbourhood is free
        if (agg[i] != -2) continue;
        bool free_nbhd = true;
        for (int k = A.ptr[i]; k < A.ptr[i + 1] && free_nbhd; ++k)
          if (strong[k] && agg[A.col[k]] >= 0) free_nbhd = false;
        if (!free_nbhd) continue;
        agg[i] = naggr;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
          if (strong[k] && agg[A.col[k]] == -2) agg[A.col[k]] = naggr;
        ++naggr;
      }
      std::vector<int> agg1 = agg;
      for (int i = 0; i < n; ++i) {  // pass 2: join the most strongly coupled aggregate
        if (agg1[i] != -2) continue;
        double best = 0.0;
        int target = -1;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
          if (strong[k] && agg1[A.col[k]] >= 0 && std::fabs(A.val[k]) > best) {
            best = std::fabs(A.val[k]);
            target = agg1[A.col[k]];
          }
        if (target >= 0) agg[i] = target;
      }
      for (int i = 0; i < n; ++i) {  // pass 3: leftovers form their own aggregates
        if (agg[i] != -2) continue;
        agg[i] = naggr;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
          if (strong[k] && agg[A.col[k]] == -2) agg[A.col[k]] = naggr;
        ++naggr;
      }
      if (naggr == 0 || naggr > int(0.8 * n)) coarsest = true;  // coarsening stalled
    }

    // --- Jacobi smoother weights: w / a_ii with w = jacobi_omega * (4/3) / rho(D^-1 A);
    //     rows without off-diagonal entries (eliminated constraints) are solved exactly.  rho from
    //     30 power steps: 12 left it 6-9 % low on FEM Laplacians (the oscillating top mode converges
    //     slowly), and the weight must stay below 2 / rho for the V-cycle to remain SPD
    L.dinv.resize(n);
    {
      std::vector<double> di(n);
      for (int i = 0; i < n; ++i) di[i] = 1.0 / d[i];
      const double rho = spectral_radius(A, di, 30);
      const double w = prm.jacobi_omega * (4.0 / 3.0) / std::max(rho, 1e-12);
      for (int i = 0; i < n; ++i) {
        const bool alone = (A.ptr[i + 1] - A.ptr[i]) == 1;
        L.dinv[i] = alone ? di[i] : w * di[i];
      }
    }

    if (coarsest) {
      constexpr int kMaxDense = 4096;
      // rows without off-diagonal entries (the eliminated constraints of a Dirichlet matrix whose
      // nodes are nearly all on the boundary, for instance) decouple: solve them by their
      // diagonal and invert the coupled rows only
      std::vector<int> core;
      H.coarse_idx.clear();
      H.coarse_diag_inv.clear();
      if (n > kMaxDense) {
        for (int i = 0; i < n; ++i)
          if (A.ptr[i + 1] - A.ptr[i] > 1) core.push_back(i);
        if (int(core.size()) > kMaxDense) throw std::runtime_error("AMG: coarsest level too large for a dense solve");
        H.coarse_idx = core;
        H.coarse_diag_inv.resize(n);
        for (int i = 0; i < n; ++i) H.coarse_diag_inv[i] = 1.0 / d[i];
      }
      const bool subset = n > kMaxDense;
      const int nd = subset ? int(core.size()) : n;
      std::vector<int> where(n, -1);
      for (int q = 0; q < nd; ++q) where[subset ? core[q] : q] = q;
      H.ncoarse = nd;
      std::vector<double> dense(size_t(nd) * nd, 0.0);
      for (int q = 0; q < nd; ++q) {
        const int i = subset ? core[q] : q;
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
          if (where[A.col[k]] >= 0) dense[size_t(q) * nd + where[A.col[k]]] += A.val[k];
      }
      if (prm.singular) {
        // constants span the null space on every level (P 1 = 1 since A 1 = 0): invert
        // A_c + a 1 1^T, which acts as the pseudo-inverse on the range of A_c
        double tr = 0.0;
        for (int i = 0; i < nd; ++i) tr += dense[size_t(i) * nd + i];
        if (nd == 0) tr = 0.0;
        const double a = tr / (double(nd) * nd);
        for (auto& v : dense) v += a;
      }
      dense_inverse(dense, nd);
      H.coarse_inv.swap(dense);
      L.A = std::move(A);
      H.levels.push_back(std::move(L));
      break;
    }

    // --- filtered diagonal and prolongator smoothing
    std::vector<double> dF(n);
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
        if (A.col[k] == i || !strong[k]) s += A.val[k];
      dF[i] = s;
    }
    // rho(D_F^-1 A_F) estimate with the filtered operator
    Csr AF;
    AF.nrows = AF.ncols = n;
    AF.ptr.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
      int c = 0;
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
        if (A.col[k] == i || strong[k]) ++c;
      AF.ptr[i + 1] = AF.ptr[i] + c;
    }
    AF.col.resize(AF.ptr[n]);
    AF.val.resize(AF.ptr[n]);
    for (int i = 0; i < n; ++i) {
      int p = AF.ptr[i];
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
        if (A.col[k] == i) { AF.col[p] = i; AF.val[p++] = dF[i]; }
        else if (strong[k]) { AF.col[p] = A.col[k]; AF.val[p++] = A.val[k]; }
      }
    }
    std::vector<double> dFi(n);
    for (int i = 0; i < n; ++i) dFi[i] = (dF[i] != 0.0) ? 1.0 / dF[i] : 0.0;
    const double rhoF = spectral_radius(AF, dFi);
    const double omega = prm.relax * (4.0 / 3.0) / std::max(rhoF, 1e-12);

    Csr P;
    P.nrows = n;
    P.ncols = naggr;
    P.ptr.assign(n + 1, 0);
    {
      std::vector<std::vector<std::pair<int, double>>> rows(n);
#pragma omp parallel for schedule(dynamic, 512)
      for (int i = 0; i < n; ++i) {
        std::vector<std::pair<int, double>>& r = rows[i];
        for (int k = AF.ptr[i]; k < AF.ptr[i + 1]; ++k) {
          const int j = AF.col[k];
          const int a = agg[j];
          if (a < 0) continue;
          double v = -omega * dFi[i] * AF.val[k];
          if (j == i) v += 1.0;
          bool found = false;
          for (auto& e : r)
            if (e.first == a) { e.second += v; found = true; break; }
          if (!found) r.emplace_back(a, v);
        }
        std::sort(r.begin(), r.end());
      }
      for (int i = 0; i < n; ++i) P.ptr[i + 1] = P.ptr[i] + int(rows[i].size());
      P.col.resize(P.ptr[n]);
      P.val.resize(P.ptr[n]);
      for (int i = 0; i < n; ++i)
        for (size_t q = 0; q < rows[i].size(); ++q) {
          P.col[P.ptr[i] + q] = rows[i][q].first;
          P.val[P.ptr[i] + q] = rows[i][q].second;
        }
    }
    Csr R, AP, Ac;
    csr_transpose(P, R);
    csr_multiply(A, P, AP);
    csr_multiply(R, AP, Ac);
    L.A = std::move(A);
    L.P = std::move(P);
    L.R = std::move(R);
    H.levels.push_back(std::move(L));
    A = std::move(Ac);
  }
  H.setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace tmb
