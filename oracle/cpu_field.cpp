// CPU restatement (FP64, OpenMP) of one full field evaluation of tetmag with its CPU solver
// configuration: the reference arm and cpu_baseline leg of bench.py.
//
// TEST / BENCH INFRASTRUCTURE ONLY.  Nothing in the library (tetmag_b200/) links or loads this
// file's build; only tests/, __graft_entry__.smoke() and bench.py's CPU legs do.
//
// One evaluation (the reference's DemagField::calcField + TheLLG right-hand side):
//   rhs   = sum_d tGrad_d (Js m_d) / mu0                       main/DemagField.cpp:124-136
//   u1    = K_N^-1 rhs   (row N/2 pinned)                      main/DemagField.cpp:204-240
//   u2_b  = B u1_b       (dense matrix or hierarchical matrix) main/DemagField.cpp:139-147,184-201
//   u2    = K_D^-1 (0, u2_b)   (boundary rows replaced)        main/DemagField.cpp:223-230
//   Hdem  = -grad (u1 + u2)                                    main/DemagField.cpp:102-113
//   H     = (-2 A/V K m + 2 Ku (k.m) k) / Js + Hext + Hdem     main/EffFieldCalc.cpp:59-84, main/TheLLG.cpp:238-254
//   ydot  = -m x H - alpha m x (m x H)                         main/TheLLG.cpp:150-178
//
// The solves restate the reference's AMGCL configuration (main/AMGCLSolver.cpp:39-53,
// main/AMGCLSolver.h:89-101): GMRES(30) with right preconditioning by an algebraic multigrid
// V-cycle of smoothed aggregation (relax 0.75, coarse_enough 100, no direct coarse solve) with
// ILU(0) relaxation (one pre- and one post-sweep), relative tolerance tol, at most maxiter
// iterations, warm-started from the previous solution (AMGCLSolver::solve, :97-103).  AMGCL is
// not vendored; the steps below follow its published algorithm (Demidov, "AMGCL: an efficient,
// flexible, and extensible algebraic multigrid implementation", Lobachevskii J. Math. 40, 2019;
// smoothed aggregation of Vanek, Mandel, Brezina 1996): strength threshold eps_strong = 0.08,
// plain aggregates on the strong graph, piecewise-constant tentative prolongation smoothed by one
// damped-Jacobi step on the filtered matrix with omega = relax * 4/3 / rho(D^-1 A_f) (rho bounded
// by the largest absolute row sum of D^-1 A_f), Galerkin coarse operators R A P with R = P^T.
// ILU(0) triangular solves are level-scheduled across threads.
//
// The hierarchical boundary matrix (for boundaries too large for the dense one) is an H-matrix:
// cluster tree of the boundary nodes (split by node-normal orientation first, then median
// bisection of the longest bounding-box axis, leaves <= leaf), strict admissibility
// min(diam) <= eta dist, dense near-field tiles with tetmag's Lindholm arithmetic
// (preproc/Lindholm.cpp:41-128, D. A. Lindholm, IEEE Trans. Magn. 20, 2025 (1984)) and low-rank
// far-field blocks by adaptive cross approximation with partial pivoting of the same weights in a
// far-field-accurate arithmetic (solid angle by atan2, Van Oosterom & Strackee 1983; log1p edge
// terms) to relative accuracy eps.  tetmag's own H2 matrix (H2Lib, main/h2interface.c:315-399)
// is not vendored.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

constexpr double kMu0 = 1.256637061435917295376e-6;
constexpr double kPi = 3.14159265358979323846;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ------------------------------------------------------------------------------------------
// CSR and kernels
// ------------------------------------------------------------------------------------------
struct Csr {
  int n = 0, m = 0;  // rows, cols
  std::vector<int> ptr, col;
  std::vector<double> val;
  long long nnz() const { return (long long)col.size(); }
};

void spmv(const Csr& A, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A.n; ++i) {
    double s = 0.0;
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) s += A.val[k] * x[A.col[k]];
    y[i] = s;
  }
}

void residual(const Csr& A, const double* b, const double* x, double* r) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A.n; ++i) {
    double s = b[i];
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) s -= A.val[k] * x[A.col[k]];
    r[i] = s;
  }
}

double dot(const double* a, const double* b, int n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

Csr transpose(const Csr& A) {
  Csr T;
  T.n = A.m;
  T.m = A.n;
  T.ptr.assign(T.n + 1, 0);
  for (int c : A.col) T.ptr[c + 1]++;
  for (int i = 0; i < T.n; ++i) T.ptr[i + 1] += T.ptr[i];
  T.col.resize(A.col.size());
  T.val.resize(A.col.size());
  std::vector<int> fill(T.ptr.begin(), T.ptr.end() - 1);
  for (int i = 0; i < A.n; ++i)
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
      const int q = fill[A.col[k]]++;
      T.col[q] = i;
      T.val[q] = A.val[k];
    }
  return T;
}

// C = A * B (row-by-row with a dense accumulator per thread)
Csr spgemm(const Csr& A, const Csr& B) {
  Csr C;
  C.n = A.n;
  C.m = B.m;
  std::vector<std::vector<int>> rc(A.n);
  std::vector<std::vector<double>> rv(A.n);
#pragma omp parallel
  {
    std::vector<double> acc(B.m, 0.0);
    std::vector<int> mark(B.m, -1), used;
#pragma omp for schedule(dynamic, 256)
    for (int i = 0; i < A.n; ++i) {
      used.clear();
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
        const int a = A.col[k];
        const double av = A.val[k];
        for (int q = B.ptr[a]; q < B.ptr[a + 1]; ++q) {
          const int j = B.col[q];
          if (mark[j] != i) {
            mark[j] = i;
            acc[j] = 0.0;
            used.push_back(j);
          }
          acc[j] += av * B.val[q];
        }
      }
      std::sort(used.begin(), used.end());
      rc[i] = used;
      rv[i].resize(used.size());
      for (size_t t = 0; t < used.size(); ++t) rv[i][t] = acc[used[t]];
    }
  }
  C.ptr.assign(C.n + 1, 0);
  for (int i = 0; i < C.n; ++i) C.ptr[i + 1] = C.ptr[i] + int(rc[i].size());
  C.col.resize(C.ptr[C.n]);
  C.val.resize(C.ptr[C.n]);
  for (int i = 0; i < C.n; ++i) {
    std::copy(rc[i].begin(), rc[i].end(), C.col.begin() + C.ptr[i]);
    std::copy(rv[i].begin(), rv[i].end(), C.val.begin() + C.ptr[i]);
  }
  return C;
}

// ------------------------------------------------------------------------------------------
// ILU(0) relaxation with level-scheduled triangular solves
// ------------------------------------------------------------------------------------------
struct Ilu0 {
  int n = 0;
  std::vector<int> ptr, col, diag;   // factors in the pattern of A (L unit lower, U upper)
  std::vector<double> val;
  std::vector<int> lvl_ptr_l, lvl_rows_l, lvl_ptr_u, lvl_rows_u;
  std::vector<double> tmp;

  void build(const Csr& A) {
    n = A.n;
    ptr = A.ptr;
    col = A.col;
    val = A.val;
    diag.assign(n, -1);
    for (int i = 0; i < n; ++i)
      for (int k = ptr[i]; k < ptr[i + 1]; ++k)
        if (col[k] == i) diag[i] = k;
    std::vector<int> pos(n, -1);
    for (int i = 0; i < n; ++i) {
      if (diag[i] < 0) throw std::runtime_error("ilu0: missing diagonal");
      for (int k = ptr[i]; k < ptr[i + 1]; ++k) pos[col[k]] = k;
      for (int k = ptr[i]; k < ptr[i + 1] && col[k] < i; ++k) {
        const int c = col[k];
        val[k] /= val[diag[c]];
        const double f = val[k];
        for (int q = diag[c] + 1; q < ptr[c + 1]; ++q) {
          const int p = pos[col[q]];
          if (p >= 0) val[p] -= f * val[q];
        }
      }
      for (int k = ptr[i]; k < ptr[i + 1]; ++k) pos[col[k]] = -1;
      if (val[diag[i]] == 0.0) throw std::runtime_error("ilu0: zero pivot");
    }
    // levels: L solve rows in dependency order, U solve in reverse
    std::vector<int> lev(n, 0);
    int maxl = 0;
    for (int i = 0; i < n; ++i) {
      int l = 0;
      for (int k = ptr[i]; k < diag[i]; ++k) l = std::max(l, lev[col[k]] + 1);
      lev[i] = l;
      maxl = std::max(maxl, l);
    }
    bucket(lev, maxl, lvl_ptr_l, lvl_rows_l);
    std::fill(lev.begin(), lev.end(), 0);
    maxl = 0;
    for (int i = n - 1; i >= 0; --i) {
      int l = 0;
      for (int k = diag[i] + 1; k < ptr[i + 1]; ++k) l = std::max(l, lev[col[k]] + 1);
      lev[i] = l;
      maxl = std::max(maxl, l);
    }
    bucket(lev, maxl, lvl_ptr_u, lvl_rows_u);
    tmp.assign(n, 0.0);
  }
  static void bucket(const std::vector<int>& lev, int maxl, std::vector<int>& lp, std::vector<int>& rows) {
    lp.assign(maxl + 2, 0);
    for (int l : lev) lp[l + 1]++;
    for (int l = 0; l <= maxl; ++l) lp[l + 1] += lp[l];
    rows.resize(lev.size());
    std::vector<int> fill(lp.begin(), lp.end() - 1);
    for (int i = 0; i < int(lev.size()); ++i) rows[fill[lev[i]]++] = i;
  }
  // z = (LU)^-1 r
  void solve(const double* r, double* z) {
    double* y = tmp.data();
    const int nl = int(lvl_ptr_l.size()) - 1;
#pragma omp parallel
    {
      for (int l = 0; l < nl; ++l) {
#pragma omp for schedule(static)
        for (int q = lvl_ptr_l[l]; q < lvl_ptr_l[l + 1]; ++q) {
          const int i = lvl_rows_l[q];
          double s = r[i];
          for (int k = ptr[i]; k < diag[i]; ++k) s -= val[k] * y[col[k]];
          y[i] = s;
        }
      }
      const int nu = int(lvl_ptr_u.size()) - 1;
      for (int l = 0; l < nu; ++l) {
#pragma omp for schedule(static)
        for (int q = lvl_ptr_u[l]; q < lvl_ptr_u[l + 1]; ++q) {
          const int i = lvl_rows_u[q];
          double s = y[i];
          for (int k = diag[i] + 1; k < ptr[i + 1]; ++k) s -= val[k] * z[col[k]];
          z[i] = s / val[diag[i]];
        }
      }
    }
  }
};

// ------------------------------------------------------------------------------------------
// Smoothed-aggregation AMG (AMGCL's algorithm as configured by tetmag) and GMRES(30)
// ------------------------------------------------------------------------------------------
struct Level {
  Csr A, P, R;
  Ilu0 ilu;
  std::vector<double> x, b, r, z;
};

struct Amg {
  std::vector<Level> lev;
  double eps_strong = 0.08, relax = 0.75;
  int coarse_enough = 100;

  void build(const Csr& A0) {
    lev.clear();
    lev.emplace_back();
    lev[0].A = A0;
    while (lev.back().A.n > coarse_enough) {
      Csr P;
      if (!coarsen(lev.back().A, P) || P.m == 0 || P.m >= lev.back().A.n) break;
      Level& f = lev.back();
      f.P = P;
      f.R = transpose(P);
      Csr Ac = spgemm(f.R, spgemm(f.A, f.P));
      lev.emplace_back();
      lev.back().A = std::move(Ac);
    }
    for (Level& l : lev) {
      l.ilu.build(l.A);
      l.x.assign(l.A.n, 0.0);
      l.b.assign(l.A.n, 0.0);
      l.r.assign(l.A.n, 0.0);
      l.z.assign(l.A.n, 0.0);
    }
  }

  // plain aggregation on the strong graph + smoothed tentative prolongation
  bool coarsen(const Csr& A, Csr& P) {
    const int n = A.n;
    std::vector<double> d(n, 0.0);
    for (int i = 0; i < n; ++i)
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
        if (A.col[k] == i) d[i] = A.val[k];
    std::vector<char> strong(A.nnz(), 0);
    const double e2 = eps_strong * eps_strong;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i)
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
        const int j = A.col[k];
        strong[k] = (j != i) && (A.val[k] * A.val[k] > e2 * std::fabs(d[i] * d[j]));
      }
    // aggregates: -2 unassigned, -1 isolated (no strong connection: left out of the coarse level)
    std::vector<int> agg(n, -2);
    int na = 0;
    for (int i = 0; i < n; ++i) {
      bool any = false;
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) any |= strong[k] != 0;
      if (!any) agg[i] = -1;
    }
    for (int i = 0; i < n; ++i) {
      if (agg[i] != -2) continue;
      bool free_nb = true;
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
        if (strong[k] && agg[A.col[k]] >= 0) {
          free_nb = false;
          break;
        }
      if (!free_nb) continue;
      agg[i] = na;
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
        if (strong[k] && agg[A.col[k]] == -2) agg[A.col[k]] = na;
      ++na;
    }
    for (int i = 0; i < n; ++i) {
      if (agg[i] != -2) continue;
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
        if (strong[k] && agg[A.col[k]] >= 0) {
          agg[i] = agg[A.col[k]];
          break;
        }
      if (agg[i] == -2) agg[i] = na++;  // a strong neighbour of an isolated node only
    }
    if (na == 0) return false;
    // filtered matrix: strong couplings and the diagonal plus the lumped weak couplings
    std::vector<double> df(n, 0.0);
    for (int i = 0; i < n; ++i) {
      double s = d[i];
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
        if (A.col[k] != i && !strong[k]) s += A.val[k];
      df[i] = s;
    }
    // omega = relax * 4/3 / rho(D_f^-1 A_f), rho bounded by the largest absolute row sum
    double rho = 0.0;
    for (int i = 0; i < n; ++i) {
      if (df[i] == 0.0) continue;
      double s = std::fabs(df[i]);
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
        if (strong[k]) s += std::fabs(A.val[k]);
      rho = std::max(rho, s / std::fabs(df[i]));
    }
    const double omega = rho > 0.0 ? relax * (4.0 / 3.0) / rho : 0.0;
    // P = (I - omega D_f^-1 A_f) P_tent, P_tent(i, agg(i)) = 1
    P.n = n;
    P.m = na;
    P.ptr.assign(n + 1, 0);
    std::vector<std::vector<std::pair<int, double>>> rows(n);
#pragma omp parallel for schedule(dynamic, 512)
    for (int i = 0; i < n; ++i) {
      std::vector<std::pair<int, double>> e;
      if (agg[i] >= 0) e.emplace_back(agg[i], 1.0);
      if (df[i] != 0.0) {
        const double s = omega / df[i];
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
          const int j = A.col[k];
          double a;
          if (j == i) a = df[i];
          else if (strong[k]) a = A.val[k];
          else continue;
          if (agg[j] >= 0) e.emplace_back(agg[j], -s * a);
        }
      }
      std::sort(e.begin(), e.end());
      std::vector<std::pair<int, double>> m;
      for (auto& p : e) {
        if (!m.empty() && m.back().first == p.first) m.back().second += p.second;
        else m.push_back(p);
      }
      rows[i] = std::move(m);
    }
    for (int i = 0; i < n; ++i) P.ptr[i + 1] = P.ptr[i] + int(rows[i].size());
    P.col.resize(P.ptr[n]);
    P.val.resize(P.ptr[n]);
    for (int i = 0; i < n; ++i)
      for (size_t t = 0; t < rows[i].size(); ++t) {
        P.col[P.ptr[i] + t] = rows[i][t].first;
        P.val[P.ptr[i] + t] = rows[i][t].second;
      }
    return true;
  }

  // one ILU(0) sweep: x += (LU)^-1 (b - A x)
  static void relax_sweep(Level& L, const double* b, double* x) {
    residual(L.A, b, x, L.r.data());
    L.ilu.solve(L.r.data(), L.z.data());
    const int n = L.A.n;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) x[i] += L.z[i];
  }

  void cycle(size_t l, const double* b, double* x) {
    Level& L = lev[l];
    const int n = L.A.n;
    std::fill(x, x + n, 0.0);
    if (l + 1 == lev.size()) {   // no direct coarse solve: the relaxation as the coarse solver
      L.ilu.solve(b, x);
      return;
    }
    relax_sweep(L, b, x);
    residual(L.A, b, x, L.r.data());
    Level& C = lev[l + 1];
    spmv(L.R, L.r.data(), C.b.data());
    cycle(l + 1, C.b.data(), C.x.data());
    // x += P xc
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int k = L.P.ptr[i]; k < L.P.ptr[i + 1]; ++k) s += L.P.val[k] * C.x[L.P.col[k]];
      x[i] += s;
    }
    relax_sweep(L, b, x);
  }
  void apply(const double* r, double* z) { cycle(0, r, z); }
};

struct Gmres {
  int M = 30;
  std::vector<std::vector<double>> V;
  std::vector<double> H, cs, sn, s, y, w, z, r;

  // right-preconditioned restarted GMRES; returns iterations, relres out
  int solve(const Csr& A, Amg& pre, const double* b, double* x, double tol, int maxiter, double& relres) {
    const int n = A.n;
    V.assign(M + 1, std::vector<double>(n, 0.0));
    H.assign(size_t(M + 1) * M, 0.0);
    cs.assign(M, 0.0);
    sn.assign(M, 0.0);
    s.assign(M + 1, 0.0);
    y.assign(M, 0.0);
    w.assign(n, 0.0);
    z.assign(n, 0.0);
    r.assign(n, 0.0);
    const double nb = std::sqrt(dot(b, b, n));
    if (nb == 0.0) {
      std::fill(x, x + n, 0.0);
      relres = 0.0;
      return 0;
    }
    int it = 0;
    residual(A, b, x, r.data());
    double beta = std::sqrt(dot(r.data(), r.data(), n));
    relres = beta / nb;
    while (relres > tol && it < maxiter) {
      for (int i = 0; i < n; ++i) V[0][i] = r[i] / beta;
      std::fill(s.begin(), s.end(), 0.0);
      s[0] = beta;
      int j = 0;
      for (; j < M && it < maxiter; ++j) {
        ++it;
        pre.apply(V[j].data(), z.data());
        spmv(A, z.data(), w.data());
        for (int q = 0; q <= j; ++q) {   // modified Gram-Schmidt
          const double h = dot(w.data(), V[q].data(), n);
          H[size_t(q) * M + j] = h;
          const double* vq = V[q].data();
#pragma omp parallel for schedule(static)
          for (int i = 0; i < n; ++i) w[i] -= h * vq[i];
        }
        const double hn = std::sqrt(dot(w.data(), w.data(), n));
        H[size_t(j + 1) * M + j] = hn;
        if (hn > 0.0)
          for (int i = 0; i < n; ++i) V[j + 1][i] = w[i] / hn;
        for (int q = 0; q < j; ++q) {   // previous rotations
          const double a = H[size_t(q) * M + j], c = H[size_t(q + 1) * M + j];
          H[size_t(q) * M + j] = cs[q] * a + sn[q] * c;
          H[size_t(q + 1) * M + j] = -sn[q] * a + cs[q] * c;
        }
        const double a = H[size_t(j) * M + j], c = H[size_t(j + 1) * M + j];
        const double den = std::hypot(a, c);
        cs[j] = den > 0.0 ? a / den : 1.0;
        sn[j] = den > 0.0 ? c / den : 0.0;
        H[size_t(j) * M + j] = den;
        H[size_t(j + 1) * M + j] = 0.0;
        s[j + 1] = -sn[j] * s[j];
        s[j] = cs[j] * s[j];
        relres = std::fabs(s[j + 1]) / nb;
        if (relres <= tol || hn == 0.0) {
          ++j;
          break;
        }
      }
      // y = H^-1 s, x += M^-1 (V y)
      for (int q = j - 1; q >= 0; --q) {
        double t = s[q];
        for (int p = q + 1; p < j; ++p) t -= H[size_t(q) * M + p] * y[p];
        y[q] = t / H[size_t(q) * M + q];
      }
      std::fill(w.begin(), w.end(), 0.0);
      for (int q = 0; q < j; ++q) {
        const double yq = y[q];
        const double* vq = V[q].data();
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) w[i] += yq * vq[i];
      }
      pre.apply(w.data(), z.data());
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; ++i) x[i] += z[i];
      residual(A, b, x, r.data());
      beta = std::sqrt(dot(r.data(), r.data(), n));
      relres = beta / nb;
    }
    return it;
  }
};

struct LinSolver {
  Csr A;
  Amg amg;
  Gmres gmres;
  std::vector<double> x;
  double tol = 1e-7;
  int maxiter = 100, last_iters = 0;
  double last_relres = 0.0, setup_s = 0.0;
  void setup(Csr Ain) {
    const double t = now_s();
    A = std::move(Ain);
    amg.build(A);
    x.assign(A.n, 0.0);
    setup_s = now_s() - t;
  }
  const double* solve(const double* b) {
    last_iters = gmres.solve(A, amg, b, x.data(), tol, maxiter, last_relres);
    return x.data();
  }
};

// ------------------------------------------------------------------------------------------
// Lindholm weights: tetmag's arithmetic (near field) and the far-field-accurate form
// ------------------------------------------------------------------------------------------
struct V3 {
  double x, y, z;
};
inline V3 sub(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double dt3(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 crs(const V3& a, const V3& b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double nrm(const V3& a) { return std::sqrt(dt3(a, a)); }
inline V3 scl(const V3& a, double s) { return {a.x * s, a.y * s, a.z * s}; }

bool are_equal(double x, double y) {
  const double eps = 2.220446049250313e-16, ulp = 100.0;
  return std::fabs(x - y) < eps * std::fabs(x + y) * ulp || (std::fabs(x) < eps * ulp && std::fabs(y) < eps * ulp);
}

// tetmag's solid angle (Lindholm.cpp:41-61)
double solid_angle_acos(const V3& x, const V3& t1, const V3& t2, const V3& t3) {
  const V3 r1 = sub(t1, x), r2 = sub(t2, x), r3 = sub(t3, x);
  const double r1n = nrm(r1), r2n = nrm(r2), r3n = nrm(r3);
  const double r23 = dt3(r2, r3), r12 = dt3(r1, r2), r31 = dt3(r3, r1);
  const double numer = r1n * r2n * r3n + r1n * r23 + r2n * r31 + r3n * r12;
  const double denom = std::sqrt(2.0 * (r2n * r3n + r23) * (r3n * r1n + r31) * (r1n * r2n + r12));
  double arg = numer / denom;
  if (are_equal(arg, 1.0)) arg = 1.0;
  return 2.0 * std::acos(arg);
}

// weights of triangle p[0..2] (area, outward normal nv) for observation point x0 -> w[3]
void lindholm(const V3& x0, const V3* p, double area, const V3& nv, bool accurate, double* w) {
  V3 rv[3], xi[3];
  double s[3], rho[3];
  for (int i = 0; i < 3; ++i) rv[i] = sub(p[i], x0);
  const V3 c = crs(sub(p[1], p[0]), sub(p[2], p[0]));
  const double cn = nrm(c);
  V3 chi;
  if (accurate) {
    chi = scl(c, 1.0 / cn);
  } else {   // auxiliaries.cpp:71-76: cross(p0 - p1, p0 - p2) normalised
    const V3 c2 = crs(sub(p[0], p[1]), sub(p[0], p[2]));
    chi = scl(c2, 1.0 / nrm(c2));
  }
  for (int i = 0; i < 3; ++i) {
    const V3 e = accurate ? sub(p[(i + 1) % 3], p[i]) : sub(rv[(i + 1) % 3], rv[i]);
    s[i] = nrm(e);
    xi[i] = scl(e, 1.0 / s[i]);
    rho[i] = nrm(rv[i]);
  }
  const double chi0 = dt3(chi, rv[0]);
  double omega, P[3];
  if (accurate) {
    const double d01 = dt3(rv[0], rv[1]), d02 = dt3(rv[0], rv[2]), d12 = dt3(rv[1], rv[2]);
    const double D = rho[0] * rho[1] * rho[2] + d01 * rho[2] + d02 * rho[1] + d12 * rho[0];
    omega = 2.0 * std::atan2(cn * chi0, D);
    for (int i = 0; i < 3; ++i) P[i] = std::log1p(2.0 * s[i] / (rho[i] + rho[(i + 1) % 3] - s[i]));
  } else {
    omega = solid_angle_acos(x0, p[0], p[1], p[2]);
    if (chi0 < 0.0) omega = -omega;
    for (int i = 0; i < 3; ++i) {
      const double rs = rho[i] + rho[(i + 1) % 3];
      P[i] = std::log((rs + s[i]) / (rs - s[i]));
    }
  }
  double eta0[3];
  for (int i = 0; i < 3; ++i) eta0[i] = dt3(crs(chi, xi[i]), rv[i]);
  const double flip = dt3(nv, chi) < 0.0 ? -1.0 : 1.0;
  for (int i = 0; i < 3; ++i) {
    double gP = 0.0;
    for (int j = 0; j < 3; ++j) gP += dt3(xi[(i + 1) % 3], xi[j]) * P[j];
    w[i] = flip * s[(i + 1) % 3] / (8.0 * kPi * area) * (eta0[(i + 1) % 3] * omega - chi0 * gP);
  }
}

// ------------------------------------------------------------------------------------------
// Boundary matrix: dense or hierarchical
// ------------------------------------------------------------------------------------------
struct Boundary {
  int nb = 0, ntri = 0;
  std::vector<V3> x;             // boundary node coordinates (boundary order)
  std::vector<int> tri;          // 3 * ntri boundary indices
  std::vector<double> area;
  std::vector<V3> tnormal, nnormal;
  std::vector<double> diag;      // Omega / 4 pi - 1
  std::vector<int> adj_ptr, adj;  // node -> triangles
};

// B_ij, i != j, with the self-triangle rule of BEMprocessing::assembleLaplaceBEMmatrix
double bem_entry(const Boundary& G, int i, int j, bool accurate) {
  if (i == j) return G.diag[i];
  double s = 0.0;
  for (int q = G.adj_ptr[j]; q < G.adj_ptr[j + 1]; ++q) {
    const int t = G.adj[q];
    const int* v = &G.tri[3 * t];
    if (v[0] == i || v[1] == i || v[2] == i) continue;
    const V3 p[3] = {G.x[v[0]], G.x[v[1]], G.x[v[2]]};
    double w[3];
    lindholm(G.x[i], p, G.area[t], G.tnormal[t], accurate, w);
    s += w[v[0] == j ? 0 : (v[1] == j ? 1 : 2)];
  }
  return s;
}

struct Cluster {
  int lo, hi;     // range in the permuted order
  V3 bmin, bmax;
  int child[2] = {-1, -1};
  double diam() const { return nrm(sub(bmax, bmin)); }
};

struct HBlock {
  int r, c;            // clusters
  bool dense;
  int rank = 0;
  size_t off = 0;      // into dense storage (rows x cols, row-major) or U (rows x k) / V (cols x k)
};

struct HMatrix {
  std::vector<int> perm;          // permuted position -> boundary index
  std::vector<Cluster> cl;
  std::vector<HBlock> blocks;
  std::vector<int> row_ptr, row_blocks;   // blocks grouped by row cluster
  std::vector<double> D, U, V;
  std::vector<size_t> voff;               // per block: offset of its V factor
  long long bytes() const { return (long long)(D.size() + U.size() + V.size()) * 8; }
};

class HBuilder {
 public:
  HBuilder(const Boundary& g, int leaf, double eta, double eps, int kmax)
      : G(g), leaf_(leaf), eta_(eta), eps_(eps), kmax_(kmax) {}
  HMatrix build() {
    HMatrix H;
    support_ = 0.0;
    for (int t = 0; t < G.ntri; ++t)
      for (int k = 0; k < 3; ++k)
        support_ = std::max(support_, nrm(sub(G.x[G.tri[3 * t + k]], G.x[G.tri[3 * t + (k + 1) % 3]])));
    H.perm.resize(G.nb);
    std::iota(H.perm.begin(), H.perm.end(), 0);
    // orientation classes of the node normals (dominant axis and sign) as the first split
    std::vector<int> cls(G.nb);
    for (int i = 0; i < G.nb; ++i) {
      const V3& n = G.nnormal[i];
      const double a[3] = {std::fabs(n.x), std::fabs(n.y), std::fabs(n.z)};
      const int d = (a[0] >= a[1] && a[0] >= a[2]) ? 0 : (a[1] >= a[2] ? 1 : 2);
      const double v = d == 0 ? n.x : (d == 1 ? n.y : n.z);
      cls[i] = 2 * d + (v < 0.0 ? 1 : 0);
    }
    std::stable_sort(H.perm.begin(), H.perm.end(), [&](int a, int b) { return cls[a] < cls[b]; });
    std::vector<int> starts;
    for (int k = 0; k < G.nb; ++k)
      if (k == 0 || cls[H.perm[k]] != cls[H.perm[k - 1]]) starts.push_back(k);
    starts.push_back(G.nb);
    // the class clusters, bisected, then joined pairwise into one root
    std::vector<int> roots;
    for (size_t c = 0; c + 1 < starts.size(); ++c) roots.push_back(make_cluster(H, starts[c], starts[c + 1]));
    while (roots.size() > 1) {
      std::vector<int> next;
      for (size_t k = 0; k + 1 < roots.size(); k += 2) next.push_back(join(H, roots[k], roots[k + 1]));
      if (roots.size() % 2) next.push_back(roots.back());
      roots = next;
    }
    partition(H, roots[0], roots[0]);
    std::sort(H.blocks.begin(), H.blocks.end(), [](const HBlock& a, const HBlock& b) { return a.r < b.r; });
    fill(H);
    return H;
  }

 private:
  const Boundary& G;
  int leaf_;
  double eta_, eps_;
  int kmax_;
  double support_ = 0.0;   // longest boundary edge

  void bbox(HMatrix& H, Cluster& c) {
    c.bmin = {1e300, 1e300, 1e300};
    c.bmax = {-1e300, -1e300, -1e300};
    for (int k = c.lo; k < c.hi; ++k) {
      const V3& p = G.x[H.perm[k]];
      c.bmin = {std::min(c.bmin.x, p.x), std::min(c.bmin.y, p.y), std::min(c.bmin.z, p.z)};
      c.bmax = {std::max(c.bmax.x, p.x), std::max(c.bmax.y, p.y), std::max(c.bmax.z, p.z)};
    }
  }
  int join(HMatrix& H, int a, int b) {
    Cluster c;
    c.lo = H.cl[a].lo;
    c.hi = H.cl[b].hi;
    bbox(H, c);
    c.child[0] = a;
    c.child[1] = b;
    H.cl.push_back(c);
    return int(H.cl.size()) - 1;
  }
  int make_cluster(HMatrix& H, int lo, int hi) {
    Cluster c;
    c.lo = lo;
    c.hi = hi;
    bbox(H, c);
    const int id = int(H.cl.size());
    H.cl.push_back(c);
    if (hi - lo > leaf_) {
      const V3 e = sub(c.bmax, c.bmin);
      const int d = (e.x >= e.y && e.x >= e.z) ? 0 : (e.y >= e.z ? 1 : 2);
      auto key = [&](int i) { return d == 0 ? G.x[i].x : (d == 1 ? G.x[i].y : G.x[i].z); };
      const int mid = (lo + hi) / 2;
      std::nth_element(H.perm.begin() + lo, H.perm.begin() + mid, H.perm.begin() + hi,
                       [&](int a, int b) { return key(a) < key(b); });
      const int a = make_cluster(H, lo, mid);
      const int b = make_cluster(H, mid, hi);
      H.cl[id].child[0] = a;
      H.cl[id].child[1] = b;
    }
    return id;
  }
  static double dist(const Cluster& a, const Cluster& b) {
    const double dx = std::max(0.0, std::max(a.bmin.x - b.bmax.x, b.bmin.x - a.bmax.x));
    const double dy = std::max(0.0, std::max(a.bmin.y - b.bmax.y, b.bmin.y - a.bmax.y));
    const double dz = std::max(0.0, std::max(a.bmin.z - b.bmax.z, b.bmin.z - a.bmax.z));
    return std::sqrt(dx * dx + dy * dy + dz * dz);
  }
  void partition(HMatrix& H, int r, int c) {
    const Cluster &R = H.cl[r], &C = H.cl[c];
    // the column functions reach one triangle beyond their nodes: the distance of the supports
    const double d = dist(R, C) - support_;
    if (d > 0.0 && std::min(R.diam(), C.diam()) <= eta_ * d) {
      H.blocks.push_back(HBlock{r, c, false});
      return;
    }
    const bool rl = R.child[0] < 0, cleaf = C.child[0] < 0;
    if (rl && cleaf) {
      H.blocks.push_back(HBlock{r, c, true});
      return;
    }
    if (rl) {
      for (int q : C.child) partition(H, r, q);
    } else if (cleaf) {
      for (int q : R.child) partition(H, q, c);
    } else {
      for (int p : R.child)
        for (int q : C.child) partition(H, p, q);
    }
  }
  // per-thread scratch of the row evaluation: column position of each boundary node (-1: not
  // in the block), a visit stamp per triangle and the triangles touching the block's columns
  struct Scratch {
    std::vector<int> pos, stamp, tris;
    int epoch = 0;
    Scratch(int nb, int ntri) : pos(nb, -1), stamp(ntri, -1) {}
  };
  // out[r * n + c] = B(rows[r], column c of cluster C): each triangle touching the columns is
  // evaluated once per row and its three weights go to the columns it holds
  void rows_of(const HMatrix& H, const Cluster& C, const int* rows, int nr, bool accurate, double* out,
               Scratch& s) const {
    const int n = C.hi - C.lo;
    ++s.epoch;
    s.tris.clear();
    for (int c = 0; c < n; ++c) {
      const int gj = H.perm[C.lo + c];
      s.pos[gj] = c;
      for (int q = G.adj_ptr[gj]; q < G.adj_ptr[gj + 1]; ++q) {
        const int t = G.adj[q];
        if (s.stamp[t] != s.epoch) {
          s.stamp[t] = s.epoch;
          s.tris.push_back(t);
        }
      }
    }
    for (int r = 0; r < nr; ++r) {
      const int gi = rows[r];
      double* o = out + size_t(r) * n;
      std::fill(o, o + n, 0.0);
      for (int t : s.tris) {
        const int* v = &G.tri[3 * t];
        if (v[0] == gi || v[1] == gi || v[2] == gi) continue;
        const V3 p[3] = {G.x[v[0]], G.x[v[1]], G.x[v[2]]};
        double w[3];
        lindholm(G.x[gi], p, G.area[t], G.tnormal[t], accurate, w);
        for (int k = 0; k < 3; ++k)
          if (s.pos[v[k]] >= 0) o[s.pos[v[k]]] += w[k];
      }
      if (s.pos[gi] >= 0) o[s.pos[gi]] = G.diag[gi];
    }
    for (int c = 0; c < n; ++c) s.pos[H.perm[C.lo + c]] = -1;
  }
  // adaptive cross approximation with partial pivoting: block ~ U V^T
  void aca(const HMatrix& H, const HBlock& b, std::vector<double>& U, std::vector<double>& V, int& k,
           Scratch& sc) {
    const Cluster &R = H.cl[b.r], &C = H.cl[b.c];
    const int m = R.hi - R.lo, n = C.hi - C.lo;
    std::vector<char> used_r(m, 0), used_c(n, 0);
    U.clear();
    V.clear();
    k = 0;
    double norm2 = 0.0;
    int i = 0;
    std::vector<double> row(n), colv(m);
    for (int it = 0; it < std::min(kmax_, std::min(m, n)); ++it) {
      used_r[i] = 1;
      const int gi = H.perm[R.lo + i];
      rows_of(H, C, &gi, 1, true, row.data(), sc);
      for (int q = 0; q < k; ++q) {
        const double u = U[size_t(q) * m + i];
        for (int j = 0; j < n; ++j) row[j] -= u * V[size_t(q) * n + j];
      }
      int jp = -1;
      for (int j = 0; j < n; ++j)
        if (!used_c[j] && (jp < 0 || std::fabs(row[j]) > std::fabs(row[jp]))) jp = j;
      if (jp < 0) break;
      // a pivot at round-off level of the approximation so far: this row is exhausted
      if (std::fabs(row[jp]) <= 1e-14 * std::sqrt(std::max(norm2, 0.0))) row[jp] = 0.0;
      if (row[jp] == 0.0) {
        int nxt = -1;
        for (int q = 0; q < m; ++q)
          if (!used_r[q]) {
            nxt = q;
            break;
          }
        if (nxt < 0) break;
        i = nxt;
        continue;
      }
      const double piv = row[jp];
      used_c[jp] = 1;
      const int gj = H.perm[C.lo + jp];
      for (int q = 0; q < m; ++q) colv[q] = bem_entry(G, H.perm[R.lo + q], gj, true);
      for (int q = 0; q < k; ++q) {
        const double v = V[size_t(q) * n + jp];
        for (int p = 0; p < m; ++p) colv[p] -= U[size_t(q) * m + p] * v;
      }
      U.insert(U.end(), colv.begin(), colv.end());
      for (int j = 0; j < n; ++j) row[j] /= piv;
      V.insert(V.end(), row.begin(), row.end());
      // ||S_k||_F^2 update
      double uu = 0.0, vv = 0.0, cross = 0.0;
      for (int p = 0; p < m; ++p) uu += colv[p] * colv[p];
      for (int j = 0; j < n; ++j) vv += row[j] * row[j];
      for (int q = 0; q < k; ++q) {
        double a = 0.0, c2 = 0.0;
        for (int p = 0; p < m; ++p) a += U[size_t(q) * m + p] * colv[p];
        for (int j = 0; j < n; ++j) c2 += V[size_t(q) * n + j] * row[j];
        cross += a * c2;
      }
      norm2 += uu * vv + 2.0 * cross;
      ++k;
      int best = -1;
      if (std::sqrt(uu * vv) <= eps_ * std::sqrt(std::max(norm2, 0.0))) {
        // converged by the estimate: check a sample of unvisited rows before accepting (partial
        // pivoting can miss a part of the block that the visited rows do not see)
        best = check_rows(H, b, U, V, k, used_r, std::sqrt(std::max(norm2, 0.0)), sc);
        if (best < 0) break;
      } else {
        // next row: largest entry of the new column among unused rows
        for (int p = 0; p < m; ++p)
          if (!used_r[p] && (best < 0 || std::fabs(colv[p]) > std::fabs(colv[best]))) best = p;
        if (best < 0) break;
      }
      i = best;
    }
  }
  // residual of up to 8 unvisited rows against the current approximation; returns the worst
  // row if its residual exceeds eps * ||S_k||_F * sqrt(1 / m) (its share of the block), else -1
  int check_rows(const HMatrix& H, const HBlock& b, const std::vector<double>& U, const std::vector<double>& V,
                 int k, const std::vector<char>& used_r, double snorm, Scratch& sc) const {
    const Cluster &R = H.cl[b.r], &C = H.cl[b.c];
    const int m = R.hi - R.lo, n = C.hi - C.lo;
    std::vector<int> cand;
    for (int p = 0; p < m; ++p)
      if (!used_r[p]) cand.push_back(p);
    if (cand.empty()) return -1;
    const int step = std::max<int>(1, int(cand.size()) / 8);
    int worst = -1;
    double wres = eps_ * snorm / std::sqrt(double(m));
    std::vector<double> row(n);
    for (size_t t = 0; t < cand.size(); t += step) {
      const int p = cand[t];
      const int gi = H.perm[R.lo + p];
      rows_of(H, C, &gi, 1, true, row.data(), sc);
      double r2 = 0.0;
      for (int j = 0; j < n; ++j) {
        double v = row[j];
        for (int q = 0; q < k; ++q) v -= U[size_t(q) * m + p] * V[size_t(q) * n + j];
        r2 += v * v;
      }
      if (std::sqrt(r2) > wres) {
        wres = std::sqrt(r2);
        worst = p;
      }
    }
    return worst;
  }
  void fill(HMatrix& H) {
    const int nbk = int(H.blocks.size());
    std::vector<std::vector<double>> Us(nbk), Vs(nbk);
    std::vector<int> ranks(nbk, 0);
#pragma omp parallel
    {
      Scratch sc(G.nb, G.ntri);
#pragma omp for schedule(dynamic, 16)
      for (int q = 0; q < nbk; ++q) {
        const HBlock& b = H.blocks[q];
        if (b.dense) {
          const Cluster &R = H.cl[b.r], &C = H.cl[b.c];
          const int m = R.hi - R.lo, n = C.hi - C.lo;
          Us[q].resize(size_t(m) * n);
          rows_of(H, C, H.perm.data() + R.lo, m, false, Us[q].data(), sc);
        } else {
          aca(H, b, Us[q], Vs[q], ranks[q], sc);
        }
      }
    }
    size_t od = 0, ou = 0, ov = 0;
    H.voff.assign(nbk, 0);
    for (int q = 0; q < nbk; ++q) {
      HBlock& b = H.blocks[q];
      if (b.dense) {
        b.off = od;
        od += Us[q].size();
      } else {
        b.rank = ranks[q];
        b.off = ou;
        H.voff[q] = ov;
        ou += Us[q].size();
        ov += Vs[q].size();
      }
    }
    H.D.resize(od);
    H.U.resize(ou);
    H.V.resize(ov);
    for (int q = 0; q < nbk; ++q) {
      const HBlock& b = H.blocks[q];
      if (b.dense) {
        std::copy(Us[q].begin(), Us[q].end(), H.D.begin() + b.off);
      } else {
        std::copy(Us[q].begin(), Us[q].end(), H.U.begin() + b.off);
        std::copy(Vs[q].begin(), Vs[q].end(), H.V.begin() + H.voff[q]);
      }
    }
    H.row_ptr.assign(H.cl.size() + 1, 0);
    for (const HBlock& b : H.blocks) H.row_ptr[b.r + 1]++;
    for (size_t c = 0; c < H.cl.size(); ++c) H.row_ptr[c + 1] += H.row_ptr[c];
    H.row_blocks.resize(nbk);
    std::vector<int> fillp(H.row_ptr.begin(), H.row_ptr.end() - 1);
    for (int q = 0; q < nbk; ++q) H.row_blocks[fillp[H.blocks[q].r]++] = q;
  }
};

struct HMat {
  HMatrix H;
  std::vector<double> xp, yp, ypart;
  // y = H x (boundary order in and out)
  void matvec(const double* x, double* y) {
    const int nb = int(H.perm.size());
    xp.resize(nb);
    yp.assign(nb, 0.0);
    for (int k = 0; k < nb; ++k) xp[k] = x[H.perm[k]];
    const int ncl = int(H.cl.size());
    // row clusters of different tree levels overlap: every thread sums into its own vector
    const int nt = omp_get_max_threads();
    ypart.assign(size_t(nt) * nb, 0.0);
#pragma omp parallel
    {
      std::vector<double> t;
      double* ymine = ypart.data() + size_t(omp_get_thread_num()) * nb;
#pragma omp for schedule(dynamic, 8)
      for (int c = 0; c < ncl; ++c) {
        if (H.row_ptr[c] == H.row_ptr[c + 1]) continue;
        const Cluster& R = H.cl[c];
        const int m = R.hi - R.lo;
        double* yr = ymine + R.lo;
        for (int q = H.row_ptr[c]; q < H.row_ptr[c + 1]; ++q) {
          const HBlock& b = H.blocks[H.row_blocks[q]];
          const Cluster& C = H.cl[b.c];
          const int n = C.hi - C.lo;
          const double* xc = xp.data() + C.lo;
          if (b.dense) {
            const double* D = H.D.data() + b.off;
            for (int i = 0; i < m; ++i) {
              double s = 0.0;
              for (int j = 0; j < n; ++j) s += D[size_t(i) * n + j] * xc[j];
              yr[i] += s;
            }
          } else {
            const double* U = H.U.data() + b.off;
            const double* V = H.V.data() + H.voff[H.row_blocks[q]];
            t.assign(b.rank, 0.0);
            for (int k = 0; k < b.rank; ++k) {
              double s = 0.0;
              for (int j = 0; j < n; ++j) s += V[size_t(k) * n + j] * xc[j];
              t[k] = s;
            }
            for (int k = 0; k < b.rank; ++k) {
              const double tk = t[k];
              for (int i = 0; i < m; ++i) yr[i] += U[size_t(k) * m + i] * tk;
            }
          }
        }
      }
    }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nb; ++k) {
      double v = 0.0;
      for (int q = 0; q < nt; ++q) v += ypart[size_t(q) * nb + k];
      y[H.perm[k]] = v;
    }
  }
};

// ------------------------------------------------------------------------------------------
// The field evaluation
// ------------------------------------------------------------------------------------------
struct Field {
  int n = 0, nb = 0;
  Csr K, g[3], tg[3];
  std::vector<double> vol, js, xc, ku2, axis, hext;
  double alpha = 1.0;
  std::vector<int> bnodes, bindex;
  LinSolver neu, dir;
  std::vector<double> Bdense;   // nb x nb row-major
  std::unique_ptr<HMat> Hm;
  std::vector<double> rhs, u1b, u2b, bdir, u, hdem;
  double t[6] = {};
  long long evals = 0;

  void setup(int nx, const int* ptr, const int* col, const double* K_, const double* const* g_,
             const double* const* tg_, const double* vol_, int nb_, const int* bn, const double* Js,
             const double* A, const double* Ku, const double* ax, const double* hx, double alpha_, double tol,
             int maxiter) {
    n = nx;
    nb = nb_;
    auto mk = [&](const double* v) {
      Csr M;
      M.n = M.m = nx;
      M.ptr.assign(ptr, ptr + nx + 1);
      M.col.assign(col, col + ptr[nx]);
      M.val.assign(v, v + ptr[nx]);
      return M;
    };
    K = mk(K_);
    for (int d = 0; d < 3; ++d) {
      g[d] = mk(g_[d]);
      tg[d] = mk(tg_[d]);
    }
    vol.assign(vol_, vol_ + nx);
    js.assign(Js, Js + nx);
    xc.resize(nx);
    ku2.assign(nx, 0.0);
    for (int i = 0; i < nx; ++i) {
      const double ij = Js[i] != 0.0 ? 1.0 / Js[i] : 0.0;
      xc[i] = -2.0 * A[i] / vol_[i] * ij;
      if (Ku) ku2[i] = 2.0 * Ku[i] * ij;
    }
    axis.assign(size_t(3) * nx, 0.0);
    if (ax) axis.assign(ax, ax + size_t(3) * nx);
    hext.assign(hx, hx + size_t(3) * nx);
    alpha = alpha_;
    bnodes.assign(bn, bn + nb_);
    bindex.assign(nx, -1);
    for (int k = 0; k < nb_; ++k) bindex[bn[k]] = k;
    // Neumann: row N/2 -> unit row (prepareNeumannMatrix); Dirichlet: boundary rows -> unit rows
    auto replaced = [&](auto pinned) {
      Csr M;
      M.n = M.m = nx;
      M.ptr.assign(nx + 1, 0);
      for (int i = 0; i < nx; ++i) {
        if (pinned(i)) {
          M.col.push_back(i);
          M.val.push_back(1.0);
        } else {
          for (int k = ptr[i]; k < ptr[i + 1]; ++k)
            if (K_[k] != 0.0 || col[k] == i) {   // zeros pruned, as the reference's prune()
              M.col.push_back(col[k]);
              M.val.push_back(K_[k]);
            }
        }
        M.ptr[i + 1] = int(M.col.size());
      }
      return M;
    };
    const int pin = nx / 2;
    neu.tol = dir.tol = tol;
    neu.maxiter = dir.maxiter = maxiter;
    neu.setup(replaced([&](int i) { return i == pin; }));
    dir.setup(replaced([&](int i) { return bindex[i] >= 0; }));
    rhs.assign(nx, 0.0);
    bdir.assign(nx, 0.0);
    u.assign(nx, 0.0);
    u1b.assign(nb, 0.0);
    u2b.assign(nb, 0.0);
    hdem.assign(size_t(3) * nx, 0.0);
  }

  void boundary_product() {
    if (Hm) {
      Hm->matvec(u1b.data(), u2b.data());
      return;
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nb; ++i) {
      const double* row = Bdense.data() + size_t(i) * nb;
      double s = 0.0;
      for (int j = 0; j < nb; ++j) s += row[j] * u1b[j];
      u2b[i] = s;
    }
  }

  void eval(const double* m, double* ydot, double* hdem_out) {
    double t0 = now_s();
    // divergence
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int k = K.ptr[i]; k < K.ptr[i + 1]; ++k) {
        const int j = K.col[k];
        s += js[j] * (tg[0].val[k] * m[j] + tg[1].val[k] * m[n + j] + tg[2].val[k] * m[2 * n + j]);
      }
      rhs[i] = s / kMu0;
    }
    double t1 = now_s();
    t[0] += t1 - t0;
    const double* u1 = neu.solve(rhs.data());
    double t2 = now_s();
    t[1] += t2 - t1;
    for (int k = 0; k < nb; ++k) u1b[k] = u1[bnodes[k]];
    boundary_product();
    std::fill(bdir.begin(), bdir.end(), 0.0);
    for (int k = 0; k < nb; ++k) bdir[bnodes[k]] = u2b[k];
    double t3 = now_s();
    t[2] += t3 - t2;
    const double* u2 = dir.solve(bdir.data());
    double t4 = now_s();
    t[3] += t4 - t3;
    // gradient, local field, LLG
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      double h[3] = {0.0, 0.0, 0.0}, e[3] = {0.0, 0.0, 0.0};
      for (int k = K.ptr[i]; k < K.ptr[i + 1]; ++k) {
        const int j = K.col[k];
        const double uj = u1[j] + u2[j];
        for (int d = 0; d < 3; ++d) h[d] -= g[d].val[k] * uj;
        const double kv = K.val[k];
        e[0] += kv * m[j];
        e[1] += kv * m[n + j];
        e[2] += kv * m[2 * n + j];
      }
      const double mi[3] = {m[i], m[n + i], m[2 * n + i]};
      const double ka[3] = {axis[i], axis[n + i], axis[2 * n + i]};
      const double km = ka[0] * mi[0] + ka[1] * mi[1] + ka[2] * mi[2];
      double H[3];
      for (int d = 0; d < 3; ++d) {
        hdem[size_t(d) * n + i] = h[d];
        H[d] = xc[i] * e[d] + ku2[i] * km * ka[d] + hext[size_t(d) * n + i] + h[d];
      }
      const double mxh[3] = {mi[1] * H[2] - mi[2] * H[1], mi[2] * H[0] - mi[0] * H[2], mi[0] * H[1] - mi[1] * H[0]};
      const double mmh[3] = {mi[1] * mxh[2] - mi[2] * mxh[1], mi[2] * mxh[0] - mi[0] * mxh[2],
                             mi[0] * mxh[1] - mi[1] * mxh[0]};
      for (int d = 0; d < 3; ++d) ydot[size_t(d) * n + i] = -mxh[d] - alpha * mmh[d];
    }
    if (hdem_out) std::memcpy(hdem_out, hdem.data(), sizeof(double) * 3 * n);
    t[4] += now_s() - t4;
    ++evals;
  }
};

thread_local std::string g_err;

}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

int orc_threads() { return omp_get_max_threads(); }
void orc_set_threads(int t) {
  if (t > 0) omp_set_num_threads(t);
}

void* orc_create(int nx, const int* ptr, const int* col, const double* K, const double* gx, const double* gy,
                 const double* gz, const double* tgx, const double* tgy, const double* tgz, const double* vol, int nb,
                 const int* bnodes, const double* Js, const double* A, const double* Ku, const double* axis,
                 const double* hext, double alpha, double tol, int maxiter) {
  try {
    auto* f = new Field();
    const double* g[3] = {gx, gy, gz};
    const double* tg[3] = {tgx, tgy, tgz};
    f->setup(nx, ptr, col, K, g, tg, vol, nb, bnodes, Js, A, Ku, axis, hext, alpha, tol, maxiter);
    return f;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void orc_destroy(void* h) { delete static_cast<Field*>(h); }

int orc_set_bem_dense(void* h, const double* B_rowmajor) {
  auto* f = static_cast<Field*>(h);
  f->Bdense.assign(B_rowmajor, B_rowmajor + size_t(f->nb) * f->nb);
  f->Hm.reset();
  return 0;
}

// xyz: boundary node coordinates (nb x 3, boundary order); tri: 3*ntri boundary indices;
// tri_area, tri_normal (ntri x 3, outward), node_normal (nb x 3), solid_angle (nb).
// out[0..3]: dense tiles, low-rank blocks, bytes, seconds.
int orc_build_hmatrix(void* h, const double* xyz, int ntri, const int* tri, const double* tri_area,
                      const double* tri_normal, const double* node_normal, const double* solid_angle, int leaf,
                      double eta, double eps, int kmax, double* out) {
  try {
    auto* f = static_cast<Field*>(h);
    const double t0 = now_s();
    Boundary G;
    G.nb = f->nb;
    G.ntri = ntri;
    G.x.resize(G.nb);
    G.nnormal.resize(G.nb);
    G.diag.resize(G.nb);
    for (int i = 0; i < G.nb; ++i) {
      G.x[i] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
      G.nnormal[i] = {node_normal[3 * i], node_normal[3 * i + 1], node_normal[3 * i + 2]};
      G.diag[i] = solid_angle[i] / (4.0 * kPi) - 1.0;
    }
    G.tri.assign(tri, tri + 3 * ntri);
    G.area.assign(tri_area, tri_area + ntri);
    G.tnormal.resize(ntri);
    for (int t = 0; t < ntri; ++t) G.tnormal[t] = {tri_normal[3 * t], tri_normal[3 * t + 1], tri_normal[3 * t + 2]};
    G.adj_ptr.assign(G.nb + 1, 0);
    for (int v : G.tri) G.adj_ptr[v + 1]++;
    for (int i = 0; i < G.nb; ++i) G.adj_ptr[i + 1] += G.adj_ptr[i];
    G.adj.resize(G.tri.size());
    std::vector<int> fillp(G.adj_ptr.begin(), G.adj_ptr.end() - 1);
    for (int t = 0; t < ntri; ++t)
      for (int k = 0; k < 3; ++k) G.adj[fillp[G.tri[3 * t + k]]++] = t;
    HBuilder b(G, leaf, eta, eps, kmax);
    auto hm = std::make_unique<HMat>();
    hm->H = b.build();
    int nd = 0, nl = 0;
    for (const HBlock& q : hm->H.blocks) (q.dense ? nd : nl)++;
    out[0] = nd;
    out[1] = nl;
    out[2] = double(hm->H.bytes());
    out[3] = now_s() - t0;
    f->Hm = std::move(hm);
    f->Bdense.clear();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

// y = B x with the current boundary matrix (dense or hierarchical), boundary order
int orc_bem_matvec(void* h, const double* x, double* y) {
  auto* f = static_cast<Field*>(h);
  std::copy(x, x + f->nb, f->u1b.begin());
  f->boundary_product();
  std::copy(f->u2b.begin(), f->u2b.end(), y);
  return 0;
}

int orc_field_eval(void* h, const double* m, double* ydot, double* hdem) {
  try {
    static_cast<Field*>(h)->eval(m, ydot, hdem);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

// out[0..11]: evals, seconds in divergence, Neumann solve, boundary product, Dirichlet solve,
// gradient + local field; last Neumann / Dirichlet iterations and relative residuals; AMG levels
// (Neumann, Dirichlet); AMG setup seconds (both)
int orc_info(void* h, double* out) {
  auto* f = static_cast<Field*>(h);
  out[0] = double(f->evals);
  for (int k = 0; k < 5; ++k) out[1 + k] = f->t[k];
  out[6] = f->neu.last_iters;
  out[7] = f->dir.last_iters;
  out[8] = f->neu.last_relres;
  out[9] = f->dir.last_relres;
  out[10] = double(f->neu.amg.lev.size()) + 1000.0 * double(f->dir.amg.lev.size());
  out[11] = f->neu.setup_s + f->dir.setup_s;
  return 0;
}

void orc_reset_timers(void* h) {
  auto* f = static_cast<Field*>(h);
  for (double& x : f->t) x = 0.0;
  f->evals = 0;
}

}  // extern "C"
