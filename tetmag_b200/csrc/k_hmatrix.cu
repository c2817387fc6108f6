// Hierarchical-matrix compression and matvec of the boundary double-layer matrix.
//
// Replaces the H2Lib path of tetmag's demag chain (DemagField::h2MVP ->
// H2_mvp_sub, main/DemagField.cpp:139-142, main/h2interface.c:77-95).  The
// partition comes from hmatrix.cpp; here:
//   * inadmissible leaf blocks become column-major dense tiles (FP64 and FP32 copies),
//     copied out of the dense FP64 matrix or assembled from the boundary mesh;
//   * every admissible block is compressed by adaptive cross approximation with
//     partial pivoting (Bebendorf, Numer. Math. 86 (2000) 565-589), one CTA per
//     block, reading entries of the dense matrix or evaluating them from the mesh
//     (accurate far-field Lindholm weights, below).  Two ranks are recorded: the
//     first k meeting the loose tolerance (stored in FP32 for the mixed path) and
//     the first k meeting the tight tolerance (stored in FP64 for the plain path).
//     After convergence a few unvisited rows are checked and, if any still has a
//     significant residual, the approximation continues from that row;
//   * the matvec y = H x works in the cluster-tree order: dense tiles by leaf row
//     cluster (plain stores); then t_b = V_b^T x_sigma for every term of every low-rank
//     block (k_h_vt, eight lanes per term), and y_tau += U_b t_b per run of blocks of one
//     row cluster (k_h_ut), with one atomic add per row and run.
#include <cmath>

#include "lindholm_accurate.cuh"
#include "tmb_dev.cuh"

namespace tmb {

namespace {

__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum (all threads receive the result).
__device__ double cta_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum_d(v);
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < nw; ++w) t += sh[w];
  return t;
}

// Block-wide argmax of |v| (all threads receive index and value); ties -> smallest index.
__device__ void cta_argmax(double v, int idx, double* shv, int* shi, double& best, int& bidx) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double a = fabs(v);
  for (int o = 16; o > 0; o >>= 1) {
    const double b = __shfl_xor_sync(0xffffffffu, a, o);
    const int j = __shfl_xor_sync(0xffffffffu, idx, o);
    if (b > a || (b == a && j < idx)) {
      a = b;
      idx = j;
    }
  }
  __syncthreads();
  if (lane == 0) {
    shv[warp] = a;
    shi[warp] = idx;
  }
  __syncthreads();
  best = -1.0;
  bidx = 0x7fffffff;
  for (int w = 0; w < nw; ++w)
    if (shv[w] > best || (shv[w] == best && shi[w] < bidx)) {
      best = shv[w];
      bidx = shi[w];
    }
}

// Entry (i, j) of the dense matrix in cluster order.
struct DenseEntry {
  const double* B;
  size_t ld;
  const int* perm;
  __device__ __forceinline__ double operator()(int i, int j) const { return B[size_t(perm[i]) * ld + perm[j]]; }
};

// Entry (i, j), i != j, evaluated from the boundary mesh: the weights of position j over the
// triangles that touch j and do not contain i (preproc/BEMprocessing.cpp:375-411), in the
// far-field-accurate arithmetic of lindholm_accurate.cuh.
struct MeshEntry {
  const double* xp;
  const int* tri;
  const double* tarea;
  const double* tnrm;
  const int* adj_ptr;
  const int2* adj;
  __device__ double operator()(int i, int j) const {
    const double x0[3] = {xp[3 * i], xp[3 * i + 1], xp[3 * i + 2]};
    double s = 0.0;
    for (int k = adj_ptr[j]; k < adj_ptr[j + 1]; ++k) {
      const int2 a = adj[k];
      const int* v = tri + 3 * a.x;
      if (v[0] == i || v[1] == i || v[2] == i) continue;
      double p[3][3];
      for (int q = 0; q < 3; ++q)
        for (int d = 0; d < 3; ++d) p[q][d] = xp[3 * v[q] + d];
      double L[3];
      lindholm_accurate(x0, p, tarea[a.x], tnrm + 3 * a.x, L);
      s += (a.y == 0) ? L[0] : (a.y == 1) ? L[1] : L[2];
    }
    return s;
  }
};

__global__ void k_h_near_gather(const HBlockDev* __restrict__ blk, DenseEntry E, double* __restrict__ d64,
                                float* __restrict__ d32) {
  const HBlockDev b = blk[blockIdx.x];
  const int mn = b.m * b.n;
  for (int t = threadIdx.x; t < mn; t += blockDim.x) {
    const int i = t % b.m, j = t / b.m;  // column-major tile
    const double v = E(b.rb + i, b.cb + j);
    d64[b.off + t] = v;
    d32[b.off + t] = static_cast<float>(v);
  }
}

// Largest residual |A_ij - sum_l U_il V_lj| over unvisited rows (a strided sample of about
// 128 rows on larger blocks); CTA-wide, every thread receives value and row.
template <typename E>
__device__ void aca_verify(const HBlockDev& b, const E& entry, const double* U, const double* V,
                           const unsigned char* usd, int k, int pass, double* shv, int* shi, double& val, int& row) {
  const int m = b.m, n = b.n;
  const int stride = (m > 128) ? (m + 127) / 128 : 1;
  const int offset = pass % stride;
  const int nrows = (m - offset + stride - 1) / stride;
  double best = 0.0;
  int bi = 0x7fffffff;
  for (long long t = threadIdx.x; t < (long long)nrows * n; t += blockDim.x) {
    const int i = offset + int(t / n) * stride;
    const int j = int(t % n);
    if (usd[i]) continue;
    double r = entry(b.rb + i, b.cb + j);
    for (int l = 0; l < k; ++l) r -= U[size_t(l) * m + i] * V[size_t(l) * n + j];
    if (fabs(r) > best || (fabs(r) == best && i < bi)) {
      best = fabs(r);
      bi = i;
    }
  }
  cta_argmax(best, bi, shv, shi, val, row);
}

// Adaptive cross approximation of one admissible block per CTA.  Partial pivoting can miss
// parts of a block whose rows couple to disjoint column sets (on a film, top-face rows see
// only bottom-face columns and vice versa), so each time the loose tolerance is reached the
// residual is checked on the unvisited rows, and the approximation restarts from the worst
// one if it is significant; the same check guards the final (tight) stop.
// gscale > 0 is an entry scale of the whole matrix: a block may then also stop once its last
// term is below eps * gscale * sqrt(m n) (and its unvisited rows below eps * gscale per entry),
// i.e. at its share of a matrix-relative error budget instead of its own norm's.
template <typename E>
__global__ void __launch_bounds__(256) k_h_aca(const HBlockDev* __restrict__ blk, E entry, double* __restrict__ Us,
                                               double* __restrict__ Vs, unsigned char* __restrict__ used, int kmax,
                                               double eps_tight, double eps_loose, double gscale,
                                               int* __restrict__ out_rank) {
  constexpr int kMaxPasses = 8;
  __shared__ double shv[32];
  __shared__ int shi[32];
  __shared__ double shd[32];
  const HBlockDev b = blk[blockIdx.x];
  const int m = b.m, n = b.n;
  double* U = Us + b.uoff;  // kmax columns of length m
  double* V = Vs + b.voff;  // kmax columns of length n
  unsigned char* usd = used + b.used_off;
  for (int i = threadIdx.x; i < m; i += blockDim.x) usd[i] = 0;
  __syncthreads();
  int k = 0, k_loose = -1, k_tight = -1, status = 0, istar = 0, passes = 0;
  bool verified = false;
  double norm2 = 0.0;
  // first unvisited row after `from` (cyclic), -1 if every row was visited
  auto next_unvisited = [&](int from) {
    for (int q = 1; q <= m; ++q)
      if (!usd[(from + q) % m]) return (from + q) % m;
    return -1;
  };
  while (true) {
    if (k >= kmax) {
      status = 1;
      break;
    }
    // residual of row istar -> V[:, k]
    double* v = V + size_t(k) * n;
    double lb = 0.0;
    int lj = 0x7fffffff;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      double r = entry(b.rb + istar, b.cb + j);
      for (int l = 0; l < k; ++l) r -= U[size_t(l) * m + istar] * V[size_t(l) * n + j];
      v[j] = r;
      if (fabs(r) > lb || (fabs(r) == lb && j < lj)) {
        lb = fabs(r);
        lj = j;
      }
    }
    double piv_abs;
    int jstar;
    cta_argmax(lb, lj, shv, shi, piv_abs, jstar);
    if (threadIdx.x == 0) usd[istar] = 1;
    __syncthreads();
    const double rms = (k > 0) ? sqrt(fabs(norm2) / (double(m) * n)) : 0.0;
    int nxt = -1;
    bool converged = k_tight >= 0;
    if (piv_abs == 0.0 || piv_abs <= 1e-14 * rms) {
      if (!converged) nxt = next_unvisited(istar);  // nothing left in this row
    } else {
      const double piv = v[jstar];
      __syncthreads();
      for (int j = threadIdx.x; j < n; j += blockDim.x) v[j] /= piv;
      __syncthreads();
      // residual of column jstar -> U[:, k]
      double* u = U + size_t(k) * m;
      double li_best = 0.0, uu_part = 0.0, vv_part = 0.0;
      int li = 0x7fffffff;
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        double c = entry(b.rb + i, b.cb + jstar);
        for (int l = 0; l < k; ++l) c -= V[size_t(l) * n + jstar] * U[size_t(l) * m + i];
        u[i] = c;
        uu_part += c * c;
        if (!usd[i] && (fabs(c) > li_best || (fabs(c) == li_best && i < li))) {
          li_best = fabs(c);
          li = i;
        }
      }
      for (int j = threadIdx.x; j < n; j += blockDim.x) vv_part += v[j] * v[j];
      const double uu = cta_sum(uu_part, shd);
      const double vv = cta_sum(vv_part, shd);
      double cross = 0.0;
      for (int l = 0; l < k; ++l) {
        double pu = 0.0, pv = 0.0;
        for (int i = threadIdx.x; i < m; i += blockDim.x) pu += u[i] * U[size_t(l) * m + i];
        for (int j = threadIdx.x; j < n; j += blockDim.x) pv += v[j] * V[size_t(l) * n + j];
        cross += cta_sum(pu, shd) * cta_sum(pv, shd);
      }
      norm2 += uu * vv + 2.0 * cross;
      ++k;
      const double term = sqrt(uu * vv), fro = fmax(sqrt(fabs(norm2)), gscale * sqrt(double(m) * n));
      if (term <= eps_tight * fro) {
        if (k_tight < 0) k_tight = k;
      } else {
        k_tight = -1;
      }
      if (term <= eps_loose * fro) {
        if (k_loose < 0) k_loose = k;
      } else {
        k_loose = -1;
        verified = false;
      }
      converged = k_tight >= 0;
      double best;
      int inext;
      cta_argmax(li_best, li, shv, shi, best, inext);
      if (k_loose >= 0 && !verified && passes < kMaxPasses) {
        double val;
        int row;
        aca_verify(b, entry, U, V, usd, k, passes++, shv, shi, val, row);
        if (row != 0x7fffffff && val > eps_loose * fmax(sqrt(fabs(norm2) / (double(m) * n)), gscale)) {
          k_loose = k_tight = -1;  // a part of the block is still missing: restart there
          istar = row;
          continue;
        }
        verified = true;
      }
      if (!converged) nxt = (inext != 0x7fffffff && best > 0.0) ? inext : next_unvisited(istar);
    }
    if (converged && nxt < 0) {
      if (passes >= kMaxPasses) break;
      double val;
      int row;
      aca_verify(b, entry, U, V, usd, k, passes++, shv, shi, val, row);
      if (row == 0x7fffffff || val <= eps_tight * fmax(sqrt(fabs(norm2) / (double(m) * n)), gscale)) break;
      nxt = row;
    }
    if (nxt < 0) break;
    istar = nxt;
  }
  if (threadIdx.x == 0) {
    if (k_tight < 0) k_tight = k;
    if (k_loose < 0 || k_loose > k_tight) k_loose = k_tight;
    out_rank[3 * blockIdx.x] = k_tight;
    out_rank[3 * blockIdx.x + 1] = k_loose;
    out_rank[3 * blockIdx.x + 2] = status;
  }
}

// Copies the first `rank` columns of U / V out of the ACA scratch into compact storage.
template <typename T>
__global__ void k_h_compact(const HBlockDev* __restrict__ blk, const double* __restrict__ Us,
                            const double* __restrict__ Vs, const long long* __restrict__ dst_u,
                            const long long* __restrict__ dst_v, const int* __restrict__ rank, T* __restrict__ U,
                            T* __restrict__ V) {
  const HBlockDev b = blk[blockIdx.x];
  const int k = rank[blockIdx.x];
  const int mp = pad4(b.m), np = pad4(b.n);
  const long long nu = (long long)k * mp, nv = (long long)k * np;
  for (long long t = threadIdx.x; t < nu; t += blockDim.x) {
    const int l = int(t / mp), i = int(t - (long long)l * mp);
    U[dst_u[blockIdx.x] + t] = i < b.m ? static_cast<T>(Us[b.uoff + (long long)l * b.m + i]) : T(0);
  }
  for (long long t = threadIdx.x; t < nv; t += blockDim.x) {
    const int l = int(t / np), j = int(t - (long long)l * np);
    V[dst_v[blockIdx.x] + t] = j < b.n ? static_cast<T>(Vs[b.voff + (long long)l * b.n + j]) : T(0);
  }
}

// x in cluster order: xp[i] = u[gidx[i]] (gidx = boundary node of permuted position i).
template <typename T>
__global__ void k_h_gather(int nb, const double* __restrict__ u, const int* __restrict__ gidx, T* __restrict__ xp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nb) xp[i] = static_cast<T>(u[gidx[i]]);
}

// Dense leaf tiles: one CTA per leaf row cluster (<= 32 rows), warps stride over its tiles.
template <typename T>
__device__ __forceinline__ void h_near_row(int bx, const HNearRow* __restrict__ rows, const HBlockDev* __restrict__ blk,
                                           const T* __restrict__ D, const T* __restrict__ xp, double* __restrict__ y) {
  __shared__ double acc[8][33];
  const HNearRow R = rows[bx];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double a = 0.0;
  for (int q = R.first + warp; q < R.last; q += 8) {
    const HBlockDev b = blk[q];
    if (lane < b.m) {
      const T* tile = D + b.off;
      for (int j = 0; j < b.n; ++j) a = fma(double(tile[size_t(j) * b.m + lane]), double(xp[b.cb + j]), a);
    }
  }
  acc[warp][lane] = a;
  __syncthreads();
  if (warp == 0 && lane < R.m) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += acc[w][lane];
    y[R.rb + lane] = s;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_h_near(const HNearRow* __restrict__ rows, const HBlockDev* __restrict__ blk,
                                                const T* __restrict__ D, const T* __restrict__ xp,
                                                double* __restrict__ y) {
  h_near_row<T>(blockIdx.x, rows, blk, D, xp, y);
}

// Transposed near field: one CTA per leaf column cluster sigma, y_sigma = sum_b D_b^T x_tau over
// its dense tiles (column-major m x n, so lane j reads tile column j, contiguous in i).
template <typename T>
__global__ void __launch_bounds__(256) k_h_near_t(const HNearRow* __restrict__ cols, const HBlockDev* __restrict__ blk,
                                                  const T* __restrict__ D, const T* __restrict__ xp,
                                                  double* __restrict__ y) {
  __shared__ double acc[8][33];
  const HNearRow C = cols[blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double a = 0.0;
  for (int q = C.first + warp; q < C.last; q += 8) {
    const HBlockDev b = blk[q];
    if (lane < b.n) {
      const T* col = D + b.off + size_t(lane) * b.m;
      for (int i = 0; i < b.m; ++i) a = fma(double(col[i]), double(xp[b.rb + i]), a);
    }
  }
  acc[warp][lane] = a;
  __syncthreads();
  if (warp == 0 && lane < C.m) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += acc[w][lane];
    y[C.rb + lane] = s;
  }
}

// Deterministic probe value in [-1, 1) for position j (cluster order): splitmix64 of j.
__device__ __forceinline__ double probe_value(long long j) {
  unsigned long long z = static_cast<unsigned long long>(j) + 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return double(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// Accuracy of every low-rank block against the entries it was built from, one CTA per block:
// y = A_b x_sigma for the probe vector x, then out = {|y|^2, |y - U64 V64^T x|^2, |y - U32 V32^T x|^2}.
template <typename E>
__global__ void __launch_bounds__(256) k_h_verify(const HBlockDev* __restrict__ blk, E entry, const int* __restrict__ rk64,
                                                  const long long* __restrict__ uo64, const long long* __restrict__ vo64,
                                                  const double* __restrict__ U64, const double* __restrict__ V64,
                                                  const int* __restrict__ rk32, const long long* __restrict__ uo32,
                                                  const long long* __restrict__ vo32, const float* __restrict__ U32,
                                                  const float* __restrict__ V32, double* __restrict__ out) {
  __shared__ double t64[128], t32[128], shd[32];
  const HBlockDev b = blk[blockIdx.x];
  const int k64 = rk64[blockIdx.x], k32 = rk32[blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int l = warp; l < k64 + k32; l += 8) {
    const bool f = l < k64;
    const int q = f ? l : l - k64;
    double a = 0.0;
    for (int j = lane; j < b.n; j += 32) {
      const long long o = (long long)q * pad4(b.n) + j;
      const double v = f ? V64[vo64[blockIdx.x] + o] : double(V32[vo32[blockIdx.x] + o]);
      a = fma(v, probe_value(b.cb + j), a);
    }
    a = warp_sum_d(a);
    if (lane == 0) (f ? t64 : t32)[q] = a;
  }
  __syncthreads();
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int i = threadIdx.x; i < b.m; i += blockDim.x) {
    double y = 0.0;
    for (int j = 0; j < b.n; ++j) y = fma(entry(b.rb + i, b.cb + j), probe_value(b.cb + j), y);
    double y64 = 0.0, y32 = 0.0;
    const int mp = pad4(b.m);
    for (int l = 0; l < k64; ++l) y64 = fma(U64[uo64[blockIdx.x] + (long long)l * mp + i], t64[l], y64);
    for (int l = 0; l < k32; ++l) y32 = fma(double(U32[uo32[blockIdx.x] + (long long)l * mp + i]), t32[l], y32);
    s0 += y * y;
    s1 += (y - y64) * (y - y64);
    s2 += (y - y32) * (y - y32);
  }
  s0 = cta_sum(s0, shd);
  s1 = cta_sum(s1, shd);
  s2 = cta_sum(s2, shd);
  if (threadIdx.x == 0) {
    out[3 * blockIdx.x] = s0;
    out[3 * blockIdx.x + 1] = s1;
    out[3 * blockIdx.x + 2] = s2;
  }
}

// 16-byte vectors of the factor type: 4 floats or 2 doubles.
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int n = 4;
  __device__ static void add(double* a, const float4& u, double t) {
    a[0] = fma(double(u.x), t, a[0]);
    a[1] = fma(double(u.y), t, a[1]);
    a[2] = fma(double(u.z), t, a[2]);
    a[3] = fma(double(u.w), t, a[3]);
  }
  __device__ static double dot(const float4& v, const float* x) {
    return double(v.x) * double(x[0]) + double(v.y) * double(x[1]) + double(v.z) * double(x[2]) +
           double(v.w) * double(x[3]);
  }
};
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int n = 2;
  __device__ static void add(double* a, const double2& u, double t) {
    a[0] = fma(u.x, t, a[0]);
    a[1] = fma(u.y, t, a[1]);
  }
  __device__ static double dot(const double2& v, const double* x) { return fma(v.x, x[0], v.y * x[1]); }
};

// Far field, first pass: t_p = V_p^T x_sigma for every term p of every admissible block.  Eight
// lanes take one term (a warp four terms): each lane issues four 16-byte streaming loads of its
// term's row of V before it uses them (each entry read once; x from cache), and the eight partial
// dots are reduced with three shuffles.  The padded tail of V is zero and x has four zero entries
// past its end.
constexpr int kLanesPerTerm = 8;
template <typename T>
__device__ __forceinline__ void h_vt_block(long long bx, long long nterms, const HTerm* __restrict__ terms,
                                           const T* __restrict__ V, const T* __restrict__ xp, double* __restrict__ t) {
  using W = Vec16<T>;
  using VT = typename W::type;
  constexpr int L = kLanesPerTerm;
  const long long p = (bx * blockDim.x + threadIdx.x) / L;
  const int sub = threadIdx.x & (L - 1);
  const bool ok = p < nterms;
  const HTerm h = terms[ok ? p : 0];
  const VT* v = reinterpret_cast<const VT*>(V + h.v);
  const T* x = xp + h.cb;
  const int nv = ok ? h.n4 / W::n : 0;
  double acc = 0.0;
  int j = sub;
  for (; j + 3 * L < nv; j += 4 * L) {
    VT a[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) a[c] = __ldcs(v + j + c * L);
#pragma unroll
    for (int c = 0; c < 4; ++c) acc += W::dot(a[c], x + W::n * (j + c * L));
  }
  for (; j < nv; j += L) acc += W::dot(__ldcs(v + j), x + W::n * j);
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (sub == 0 && ok) t[p] = acc;
}

template <typename T>
__global__ void __launch_bounds__(256) k_h_vt(long long nterms, const HTerm* __restrict__ terms,
                                              const T* __restrict__ V, const T* __restrict__ xp,
                                              double* __restrict__ t) {
  h_vt_block<T>(blockIdx.x, nterms, terms, V, xp, t);
}

// The dense near field and the far field's first pass are independent: one launch whose first
// nrows CTAs take the leaf row clusters' tiles and whose others take the terms, so the
// latency-bound tile rows run beside the streaming V^T x instead of before it.
template <typename T>
__global__ void __launch_bounds__(256) k_h_near_vt(int nrows, const HNearRow* __restrict__ rows,
                                                   const HBlockDev* __restrict__ blk, const T* __restrict__ D,
                                                   double* __restrict__ y, long long nterms,
                                                   const HTerm* __restrict__ terms, const T* __restrict__ V,
                                                   const T* __restrict__ xp, double* __restrict__ t) {
  if (int(blockIdx.x) < nrows) h_near_row<T>(blockIdx.x, rows, blk, D, xp, y);
  else h_vt_block<T>((long long)blockIdx.x - nrows, nterms, terms, V, xp, t);
}

// Far field, second pass: y_tau += sum_b U_b t_b over the admissible blocks of one work item (a
// run of blocks of one row cluster tau, hence a contiguous range of terms), one CTA per item.
// The item's term offsets and values are staged in shared memory (up to kStage at a time), then
// thread -> (16-byte row vector, term slice) streams its U entries with independent 16-byte loads
// (each entry read once); one atomic add per row at the end.
constexpr int kStage = 512;
constexpr int kUtLoads = 4;  // U loads in flight per thread (8 measured slower: 443 against 437 us on c2)
template <typename T>
__global__ void __launch_bounds__(256) k_h_ut(const HFarGroup* __restrict__ grp, const long long* __restrict__ toff,
                                              const HTerm* __restrict__ terms, const T* __restrict__ U,
                                              const double* __restrict__ t, double* __restrict__ y) {
  using W = Vec16<T>;
  using VT = typename W::type;
  constexpr int E = W::n;
  __shared__ double red[256 * E];
  __shared__ long long su[kStage];
  __shared__ double st[kStage];
  const HFarGroup g = grp[blockIdx.x];
  const int mp = pad4(g.m), nvec = mp / E;
  // nvec <= 256 (floats, m <= 1024): thread -> (vec, slice); doubles with nvec > 256: two vecs
  const int per = (nvec + 255) / 256;
  const int slices = nvec >= 256 ? 1 : 256 / nvec;
  const int vec = nvec >= 256 ? threadIdx.x : threadIdx.x % nvec;
  const int slice = nvec >= 256 ? 0 : threadIdx.x / nvec;
  const long long pbeg = toff[g.first], pend = toff[g.last];  // toff has an entry past the last block
  double acc[2][E];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int e = 0; e < E; ++e) acc[r][e] = 0.0;
  for (long long c0 = pbeg; c0 < pend; c0 += kStage) {
    const int nc = int(min((long long)kStage, pend - c0));
    __syncthreads();  // the previous stage is consumed
    for (int i = threadIdx.x; i < nc; i += 256) {
      su[i] = terms[c0 + i].u;
      st[i] = t[c0 + i];
    }
    __syncthreads();
    if (slice < slices) {
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int vv = vec + 256 * r;
        if (r < per && vv < nvec) {
          int i = slice;
          for (; i + (kUtLoads - 1) * slices < nc; i += kUtLoads * slices) {
            VT uv[kUtLoads];
#pragma unroll
            for (int c = 0; c < kUtLoads; ++c)
              uv[c] = __ldcs(reinterpret_cast<const VT*>(U + su[i + c * slices]) + vv);
#pragma unroll
            for (int c = 0; c < kUtLoads; ++c) W::add(acc[r], uv[c], st[i + c * slices]);
          }
          for (; i < nc; i += slices) W::add(acc[r], __ldcs(reinterpret_cast<const VT*>(U + su[i]) + vv), st[i]);
        }
      }
    }
  }
  if (nvec >= 256) {
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int i = E * (vec + 256 * r) + e;
        if (r < per && i < g.m) atomicAdd(&y[g.rb + i], acc[r][e]);
      }
  } else {
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E; ++e) red[threadIdx.x * E + e] = acc[0][e];
    __syncthreads();
    for (int i = threadIdx.x; i < g.m; i += 256) {
      const int v = i / E, e = i - v * E;
      double s = 0.0;
      for (int sl = 0; sl < slices; ++sl) s += red[(sl * nvec + v) * E + e];
      atomicAdd(&y[g.rb + i], s);
    }
  }
}

// Dirichlet load from the H-matrix result: b[node] = y[pos[node]] on the boundary, 0 inside.
__global__ void k_h_dirichlet(int n, const int* __restrict__ pos, const double* __restrict__ y, double* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = pos[i];
  b[i] = (p >= 0) ? y[p] : 0.0;
}

DenseEntry dense_entry(const HSource& s) { return DenseEntry{s.B, s.ld, s.perm}; }
MeshEntry mesh_entry(const HSource& s) { return MeshEntry{s.xp, s.tri, s.tarea, s.tnrm, s.adj_ptr, s.adj}; }

}  // namespace

void launch_h_near_gather(int nblk, const HBlockDev* blk, const HSource& src, double* d64, float* d32,
                          cudaStream_t st) {
  if (nblk == 0) return;
  if (!src.B) throw std::runtime_error("dense tile gather without a dense matrix");
  note_launch();
  k_h_near_gather<<<nblk, 256, 0, st>>>(blk, dense_entry(src), d64, d32);
  TMB_CUDA(cudaGetLastError());
}

void launch_h_aca(int nblk, const HBlockDev* blk, const HSource& src, double* Us, double* Vs, unsigned char* used,
                  int kmax, double eps_tight, double eps_loose, double gscale, int* out_rank, cudaStream_t st) {
  if (nblk == 0) return;
  note_launch();
  if (src.B)
    k_h_aca<<<nblk, 256, 0, st>>>(blk, dense_entry(src), Us, Vs, used, kmax, eps_tight, eps_loose, gscale, out_rank);
  else
    k_h_aca<<<nblk, 256, 0, st>>>(blk, mesh_entry(src), Us, Vs, used, kmax, eps_tight, eps_loose, gscale, out_rank);
  TMB_CUDA(cudaGetLastError());
}

void launch_h_verify(int nblk, const HBlockDev* blk, const HSource& src, const int* rk64, const long long* uo64,
                     const long long* vo64, const double* U64, const double* V64, const int* rk32,
                     const long long* uo32, const long long* vo32, const float* U32, const float* V32, double* out,
                     cudaStream_t st) {
  if (nblk == 0) return;
  note_launch();
  if (src.B)
    k_h_verify<<<nblk, 256, 0, st>>>(blk, dense_entry(src), rk64, uo64, vo64, U64, V64, rk32, uo32, vo32, U32, V32,
                                     out);
  else
    k_h_verify<<<nblk, 256, 0, st>>>(blk, mesh_entry(src), rk64, uo64, vo64, U64, V64, rk32, uo32, vo32, U32, V32,
                                     out);
  TMB_CUDA(cudaGetLastError());
}

template <typename T>
void launch_h_compact(int nblk, const HBlockDev* blk, const double* Us, const double* Vs, const long long* du,
                      const long long* dv, const int* rank, T* U, T* V, cudaStream_t st) {
  if (nblk == 0) return;
  note_launch();
  k_h_compact<T><<<nblk, 256, 0, st>>>(blk, Us, Vs, du, dv, rank, U, V);
  TMB_CUDA(cudaGetLastError());
}

template <typename T>
void launch_h_matvec(const HMatView<T>& H, const double* u, double* y, T* xp, const int* pos, int n, double* bdir,
                     cudaStream_t st) {
  note_launch();
  k_h_gather<T><<<grid_for(H.nb), kBlock, 0, st>>>(H.nb, u, H.gidx, xp);
  note_launch();
  const long long vt_blocks = (H.nterms * kLanesPerTerm + 255) / 256;
  k_h_near_vt<T><<<unsigned(H.nrows + vt_blocks), 256, 0, st>>>(H.nrows, H.near_rows, H.near, H.D, y, H.nterms,
                                                                H.terms, H.V, xp, H.t);
  if (H.nterms > 0) {
    note_launch();
    k_h_ut<T><<<H.ngroups, 256, 0, st>>>(H.groups, H.toff, H.terms, H.U, H.t, y);
  }
  note_launch();
  k_h_dirichlet<<<grid_for(n), kBlock, 0, st>>>(n, pos, y, bdir);
  TMB_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------------------------------
// H2 matvec (nested cluster bases built by h2.cpp).  Coefficient vectors are FP64; basis,
// transfer and coupling values are T.  Every kernel gives one warp to one cluster (ranks <= 64:
// two coefficients per lane).
// ------------------------------------------------------------------------------------------
namespace {

// column leaves: xh_l = W_l^T x_l (W_l row-major m x kc: lane j reads W[i * kc + j], coalesced)
template <typename T>
__global__ void k_h2_leaf_up(int nleaf, const int* __restrict__ leaves, const H2Node* __restrict__ node,
                             const T* __restrict__ colb, const T* __restrict__ xp, double* __restrict__ xh) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nleaf) return;
  const H2Node c = node[leaves[w]];
  if (c.kc == 0) return;
  const T* W = colb + c.cl;
  double a0 = 0.0, a1 = 0.0;
  const bool two = lane + 32 < c.kc;
  for (int i = 0; i < c.m; ++i) {
    const double xi = double(xp[c.begin + i]);
    if (lane < c.kc) a0 = fma(double(W[size_t(i) * c.kc + lane]), xi, a0);
    if (two) a1 = fma(double(W[size_t(i) * c.kc + lane + 32]), xi, a1);
  }
  if (lane < c.kc) xh[c.xo + lane] = a0;
  if (two) xh[c.xo + lane + 32] = a1;
}

// Asynchronous element copies global -> shared (cp.async): a thread issues all of its copies
// before waiting for any, so a CTA has its whole panel in flight at once.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  if constexpr (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// One depth of the upward or downward pass: out[o] (+)= sum_i P[i * ld + o] v[i], o < nout,
// i < nin (nin, nout <= 64), for one cluster per CTA of 256 threads.  The panel P (nout x nin,
// column-major: entry (o, i) at i * nout + o) is staged in shared memory by cp.async, so its loads overlap instead
// of forming one chain per warp; thread t then sums the terms i = t / 64 (mod 4) of output
// t % 64 and the four partial sums are added in a fixed order.  The tree's upper depths have only
// a few clusters each: with one warp per cluster they were bound by that chain (one memory
// latency per term, over 60 long-scoreboard stalls per issued instruction).
template <typename T>
__device__ __forceinline__ double cta_panel_dot(const T* __restrict__ P, int nout, const double* __restrict__ v,
                                                int nin, T* sp, double* sv, double* red) {
  const int t = threadIdx.x;
  const int total = nin * nout;
  for (int k = t; k < total; k += 256) cp_async_elem(sp + k, P + k);
  if (t < nin) sv[t] = v[t];
  cp_async_wait_all();
  __syncthreads();
  const int o = t & 63, g = t >> 6;
  double a = 0.0;
  if (o < nout)
    for (int i = g; i < nin; i += 4) a = fma(double(sp[i * nout + o]), sv[i], a);
  red[t] = a;
  __syncthreads();
  double r = 0.0;
  if (t < 64) r = ((red[t] + red[t + 64]) + red[t + 128]) + red[t + 192];
  __syncthreads();  // sp, sv and red are reused by the caller's next panel
  return r;
}

// upward pass, one depth: xh_c = sum over children F_ch^T xh_ch (the transposed transfer of a
// child is stored kc x kc_child column-major: F[j + i * kc]); one CTA per cluster
template <typename T>
__global__ void __launch_bounds__(256) k_h2_up(int count, const int* __restrict__ ids,
                                               const H2Node* __restrict__ node, const T* __restrict__ colb,
                                               double* __restrict__ xh) {
  __shared__ T sp[64 * 64];
  __shared__ double sv[64], red[256];
  if (int(blockIdx.x) >= count) return;
  const H2Node c = node[ids[blockIdx.x]];
  if (c.child0 < 0 || c.kc == 0) return;
  double acc = 0.0;
  for (int s = 0; s < 2; ++s) {
    const H2Node ch = node[s == 0 ? c.child0 : c.child1];
    if (ch.kc == 0) continue;
    acc += cta_panel_dot(colb + ch.ct, c.kc, xh + ch.xo, ch.kc, sp, sv, red);
  }
  if (threadIdx.x < c.kc) xh[c.xo + threadIdx.x] = acc;
}

// couplings: yh_t += S_b xh_s for every admissible block b = (t, s) (S_b kr x kc column-major);
// one warp per block (row clusters own very different numbers of blocks: a warp per row cluster
// left the largest clusters' warps running long after the rest), FP64 atomic adds into yh_t
template <typename T>
__global__ void __launch_bounds__(256) k_h2_couple(int nblk, const int* __restrict__ brow,
                                                   const H2Blk* __restrict__ blk, const H2Node* __restrict__ node,
                                                   const T* __restrict__ S, const double* __restrict__ xh,
                                                   double* __restrict__ yh) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nblk) return;
  const H2Blk b = blk[w];
  const H2Node t = node[brow[w]];
  const H2Node s = node[b.s];
  if (t.kr == 0 || s.kc == 0) return;
  const T* Sq = S + b.so;
  double a0 = 0.0, a1 = 0.0, c0 = 0.0, c1 = 0.0;
  const bool one = lane < t.kr, two = lane + 32 < t.kr;
  int j = 0;
  for (; j + 1 < s.kc; j += 2) {   // two independent accumulation chains
    const double x0 = xh[s.xo + j], x1 = xh[s.xo + j + 1];
    if (one) {
      a0 = fma(double(Sq[size_t(j) * t.kr + lane]), x0, a0);
      c0 = fma(double(Sq[size_t(j + 1) * t.kr + lane]), x1, c0);
    }
    if (two) {
      a1 = fma(double(Sq[size_t(j) * t.kr + lane + 32]), x0, a1);
      c1 = fma(double(Sq[size_t(j + 1) * t.kr + lane + 32]), x1, c1);
    }
  }
  if (j < s.kc) {
    const double x0 = xh[s.xo + j];
    if (one) a0 = fma(double(Sq[size_t(j) * t.kr + lane]), x0, a0);
    if (two) a1 = fma(double(Sq[size_t(j) * t.kr + lane + 32]), x0, a1);
  }
  if (one) atomicAdd(yh + t.yo + lane, a0 + c0);
  if (two) atomicAdd(yh + t.yo + lane + 32, a1 + c1);
}

// downward pass, one depth: yh_c += E_c yh_parent (E_c kr x kr_parent column-major); one CTA per
// cluster (cta_panel_dot)
template <typename T>
__global__ void __launch_bounds__(256) k_h2_down(int count, const int* __restrict__ ids,
                                                 const H2Node* __restrict__ node, const T* __restrict__ rowb,
                                                 double* __restrict__ yh) {
  __shared__ T sp[64 * 64];
  __shared__ double sv[64], red[256];
  if (int(blockIdx.x) >= count) return;
  const H2Node c = node[ids[blockIdx.x]];
  if (c.parent < 0 || c.kr == 0 || c.child0 < 0) return;
  const H2Node p = node[c.parent];
  if (p.kr == 0) return;
  const double a = cta_panel_dot(rowb + c.rt, c.kr, yh + p.yo, p.kr, sp, sv, red);
  if (threadIdx.x < c.kr) yh[c.yo + threadIdx.x] += a;
}

// row leaves: y_l += V_l (yh_l + E_l yh_parent) (V_l m x kr column-major: lane i reads V[i + j m]);
// the leaf's own share of its parent's coefficients is applied here instead of in k_h2_down
template <typename T>
__global__ void k_h2_leaf_down(int nleaf, const int* __restrict__ leaves, const H2Node* __restrict__ node,
                               const T* __restrict__ rowb, const double* __restrict__ yh, double* __restrict__ y) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nleaf) return;
  const H2Node c = node[leaves[w]];
  if (c.kr == 0) return;
  // coefficients of the leaf: its own couplings plus the transfer of the parent's
  __shared__ double coef[8][64];
  double* cf = coef[(threadIdx.x >> 5) & 7];
  for (int i = lane; i < c.kr; i += 32) {
    double a = yh[c.yo + i];
    if (c.parent >= 0) {
      const H2Node p = node[c.parent];
      const T* E = rowb + c.rt;
      for (int j = 0; j < p.kr; ++j) a = fma(double(E[size_t(j) * c.kr + i]), yh[p.yo + j], a);
    }
    cf[i] = a;
  }
  __syncwarp();
  if (lane < c.m) {
    const T* V = rowb + c.rl;
    double a = 0.0;
    for (int j = 0; j < c.kr; ++j) a = fma(double(V[size_t(j) * c.m + lane]), cf[j], a);
    y[c.begin + lane] += a;
  }
}

}  // namespace

template <typename T>
void launch_h2_matvec(const H2View<T>& H, const double* u, double* y, T* xp, const int* pos, int n, double* bdir,
                      const std::vector<std::pair<int, int>>& up, const std::vector<std::pair<int, int>>& down,
                      cudaStream_t st) {
  const int wpb = 8;   // warps per 256-thread block
  auto blocks = [&](int warps) { return unsigned((warps + wpb - 1) / wpb); };
  note_launch();
  k_h_gather<T><<<grid_for(H.nb), kBlock, 0, st>>>(H.nb, u, H.gidx, xp);
  note_launch();
  k_h_near<T><<<H.nrows, 256, 0, st>>>(H.near_rows, H.near, H.D, xp, y);
  TMB_CUDA(cudaMemsetAsync(H.yh, 0, sizeof(double) * size_t(H.nyh), st));
  if (H.nleaf > 0) {
    note_launch();
    k_h2_leaf_up<T><<<blocks(H.nleaf), 256, 0, st>>>(H.nleaf, H.leaves, H.node, H.colb, xp, H.xh);
  }
  for (const auto& d : up) {
    note_launch();
    k_h2_up<T><<<unsigned(d.second), 256, 0, st>>>(d.second, H.lvl_nodes + d.first, H.node, H.colb, H.xh);
  }
  if (H.nblk > 0) {
    note_launch();
    k_h2_couple<T><<<blocks(H.nblk), 256, 0, st>>>(H.nblk, H.brow, H.blk, H.node, H.S, H.xh, H.yh);
  }
  for (const auto& d : down) {
    note_launch();
    k_h2_down<T><<<unsigned(d.second), 256, 0, st>>>(d.second, H.lvl_nodes + d.first, H.node, H.rowb, H.yh);
  }
  if (H.nleaf > 0) {
    note_launch();
    k_h2_leaf_down<T><<<blocks(H.nleaf), 256, 0, st>>>(H.nleaf, H.leaves, H.node, H.rowb, H.yh, y);
  }
  note_launch();
  k_h_dirichlet<<<grid_for(n), kBlock, 0, st>>>(n, pos, y, bdir);
  TMB_CUDA(cudaGetLastError());
}

template void launch_h2_matvec<double>(const H2View<double>&, const double*, double*, double*, const int*, int,
                                       double*, const std::vector<std::pair<int, int>>&,
                                       const std::vector<std::pair<int, int>>&, cudaStream_t);
template void launch_h2_matvec<float>(const H2View<float>&, const double*, double*, float*, const int*, int,
                                      double*, const std::vector<std::pair<int, int>>&,
                                      const std::vector<std::pair<int, int>>&, cudaStream_t);

template void launch_h_compact<double>(int, const HBlockDev*, const double*, const double*, const long long*,
                                       const long long*, const int*, double*, double*, cudaStream_t);
template void launch_h_compact<float>(int, const HBlockDev*, const double*, const double*, const long long*,
                                      const long long*, const int*, float*, float*, cudaStream_t);
template <typename T>
void launch_h_matvec_t(const HMatView<T>& H, const double* u, double* y, T* xp, cudaStream_t st) {
  note_launch();
  k_h_gather<T><<<grid_for(H.nb), kBlock, 0, st>>>(H.nb, u, H.gidx, xp);
  note_launch();
  k_h_near_t<T><<<H.nrows, 256, 0, st>>>(H.near_rows, H.near, H.D, xp, y);
  if (H.nterms > 0) {
    note_launch();
    const long long threads = H.nterms * kLanesPerTerm;
    k_h_vt<T><<<unsigned((threads + 255) / 256), 256, 0, st>>>(H.nterms, H.terms, H.V, xp, H.t);
    note_launch();
    k_h_ut<T><<<H.ngroups, 256, 0, st>>>(H.groups, H.toff, H.terms, H.U, H.t, y);
  }
  TMB_CUDA(cudaGetLastError());
}

template void launch_h_matvec_t<double>(const HMatView<double>&, const double*, double*, double*, cudaStream_t);
template void launch_h_matvec_t<float>(const HMatView<float>&, const double*, double*, float*, cudaStream_t);
template void launch_h_matvec<double>(const HMatView<double>&, const double*, double*, double*, const int*, int,
                                      double*, cudaStream_t);
template void launch_h_matvec<float>(const HMatView<float>&, const double*, double*, float*, const int*, int,
                                     double*, cudaStream_t);

}  // namespace tmb
