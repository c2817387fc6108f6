// Hierarchical-matrix compression and matvec of the boundary double-layer matrix.
//
// Replaces the H2Lib path of tetmag's demag chain (DemagField::h2MVP ->
// H2_mvp_sub, main/DemagField.cpp:139-142, main/h2interface.c:77-95).  The
// partition comes from hmatrix.cpp; here:
//   * inadmissible leaf blocks are copied out of the device-assembled dense FP64
//     matrix into column-major dense tiles (FP64 and FP32 copies);
//   * every admissible block is compressed by adaptive cross approximation with
//     partial pivoting (Bebendorf, Numer. Math. 86 (2000) 565-589), one CTA per
//     block, reading entries of the dense matrix.  Two ranks are recorded: the
//     first k meeting the loose tolerance (stored in FP32 for the mixed path) and
//     the first k meeting the tight tolerance (stored in FP64 for the plain path).
//     After convergence a few unvisited rows are checked and, if any still has a
//     significant residual, the approximation continues from that row;
//   * the matvec y = H x works in the cluster-tree order: dense tiles by leaf row
//     cluster (plain stores), then t_b = V_b^T x_sigma per low-rank block, then
//     y_tau += U_b t_b with one atomic add per row and row cluster.
#include <cmath>

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

__device__ __forceinline__ double entry(const double* B, size_t ld, const int* perm, int gi, int gj) {
  return B[size_t(perm[gi]) * ld + perm[gj]];
}

__global__ void k_h_near_gather(const HBlockDev* __restrict__ blk, const double* __restrict__ B, size_t ld,
                                const int* __restrict__ perm, double* __restrict__ d64, float* __restrict__ d32) {
  const HBlockDev b = blk[blockIdx.x];
  const int mn = b.m * b.n;
  for (int t = threadIdx.x; t < mn; t += blockDim.x) {
    const int i = t % b.m, j = t / b.m;  // column-major tile
    const double v = entry(B, ld, perm, b.rb + i, b.cb + j);
    d64[b.off + t] = v;
    d32[b.off + t] = static_cast<float>(v);
  }
}

// Largest residual |A_ij - sum_l U_il V_lj| over unvisited rows (a strided sample of about
// 128 rows on larger blocks); CTA-wide, every thread receives value and row.
__device__ void aca_verify(const HBlockDev& b, const double* __restrict__ B, size_t ld, const int* __restrict__ perm,
                           const double* U, const double* V, const unsigned char* usd, int k, int pass, double* shv,
                           int* shi, double& val, int& row) {
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
    double r = entry(B, ld, perm, b.rb + i, b.cb + j);
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
__global__ void __launch_bounds__(256) k_h_aca(const HBlockDev* __restrict__ blk, const double* __restrict__ B,
                                               size_t ld, const int* __restrict__ perm, double* __restrict__ Us,
                                               double* __restrict__ Vs, unsigned char* __restrict__ used, int kmax,
                                               double eps_tight, double eps_loose, int* __restrict__ out_rank) {
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
      double r = entry(B, ld, perm, b.rb + istar, b.cb + j);
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
        double c = entry(B, ld, perm, b.rb + i, b.cb + jstar);
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
      const double term = sqrt(uu * vv), fro = sqrt(fabs(norm2));
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
        aca_verify(b, B, ld, perm, U, V, usd, k, passes++, shv, shi, val, row);
        if (row != 0x7fffffff && val > eps_loose * sqrt(fabs(norm2) / (double(m) * n))) {
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
      aca_verify(b, B, ld, perm, U, V, usd, k, passes++, shv, shi, val, row);
      if (row == 0x7fffffff || val <= eps_tight * sqrt(fabs(norm2) / (double(m) * n))) break;
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
  const long long nu = (long long)k * b.m, nv = (long long)k * b.n;
  for (long long t = threadIdx.x; t < nu; t += blockDim.x) U[dst_u[blockIdx.x] + t] = static_cast<T>(Us[b.uoff + t]);
  for (long long t = threadIdx.x; t < nv; t += blockDim.x) V[dst_v[blockIdx.x] + t] = static_cast<T>(Vs[b.voff + t]);
}

// x in cluster order: xp[i] = u[gidx[i]] (gidx = boundary node of permuted position i).
template <typename T>
__global__ void k_h_gather(int nb, const double* __restrict__ u, const int* __restrict__ gidx, T* __restrict__ xp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nb) xp[i] = static_cast<T>(u[gidx[i]]);
}

// Dense leaf tiles: one CTA per leaf row cluster (<= 32 rows), warps stride over its tiles.
template <typename T>
__global__ void __launch_bounds__(256) k_h_near(const HNearRow* __restrict__ rows, const HBlockDev* __restrict__ blk,
                                                const T* __restrict__ D, const T* __restrict__ xp,
                                                double* __restrict__ y) {
  __shared__ double acc[8][33];
  const HNearRow R = rows[blockIdx.x];
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

// t_b = V_b^T x_sigma for every low-rank block: one warp per term (block, column l).
template <typename T>
__global__ void __launch_bounds__(256) k_h_far_vt(const int2* __restrict__ terms, long long nterms,
                                                  const HBlockDev* __restrict__ blk, const long long* __restrict__ voff,
                                                  const long long* __restrict__ toff, const T* __restrict__ V,
                                                  const T* __restrict__ xp, double* __restrict__ t) {
  const long long w = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= nterms) return;
  const int2 bl = terms[w];
  const HBlockDev b = blk[bl.x];
  const T* v = V + voff[bl.x] + (long long)bl.y * b.n;
  double a = 0.0;
  for (int j = lane; j < b.n; j += 32) a = fma(double(v[j]), double(xp[b.cb + j]), a);
  a = warp_sum_d(a);
  if (lane == 0) t[toff[bl.x] + bl.y] = a;
}

// y_tau += sum_b U_b t_b over the low-rank blocks of each row cluster; one thread per row.
template <typename T>
__global__ void __launch_bounds__(256) k_h_far_u(const HFarGroup* __restrict__ grp, const HBlockDev* __restrict__ blk,
                                                 const int* __restrict__ rank, const long long* __restrict__ uoff,
                                                 const long long* __restrict__ toff, const T* __restrict__ U,
                                                 const double* __restrict__ t, double* __restrict__ y) {
  const HFarGroup g = grp[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.m) return;
  double a = 0.0;
  for (int q = g.first; q < g.last; ++q) {
    const int k = rank[q];
    const T* u = U + uoff[q] + i;
    const double* tb = t + toff[q];
    const int m = blk[q].m;
    for (int l = 0; l < k; ++l) a = fma(double(u[(long long)l * m]), tb[l], a);
  }
  if (a != 0.0) atomicAdd(&y[g.rb + i], a);
}

// Dirichlet load from the H-matrix result: b[node] = y[pos[node]] on the boundary, 0 inside.
__global__ void k_h_dirichlet(int n, const int* __restrict__ pos, const double* __restrict__ y, double* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = pos[i];
  b[i] = (p >= 0) ? y[p] : 0.0;
}

}  // namespace

void launch_h_near_gather(int nblk, const HBlockDev* blk, const double* B, size_t ld, const int* perm, double* d64,
                          float* d32, cudaStream_t st) {
  if (nblk == 0) return;
  note_launch();
  k_h_near_gather<<<nblk, 256, 0, st>>>(blk, B, ld, perm, d64, d32);
  TMB_CUDA(cudaGetLastError());
}

void launch_h_aca(int nblk, const HBlockDev* blk, const double* B, size_t ld, const int* perm, double* Us,
                  double* Vs, unsigned char* used, int kmax, double eps_tight, double eps_loose, int* out_rank,
                  cudaStream_t st) {
  if (nblk == 0) return;
  note_launch();
  k_h_aca<<<nblk, 256, 0, st>>>(blk, B, ld, perm, Us, Vs, used, kmax, eps_tight, eps_loose, out_rank);
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
void launch_h_matvec(const HMatView<T>& H, const double* u, double* y, double* t, T* xp, const int* pos, int n,
                     double* bdir, cudaStream_t st) {
  note_launch();
  k_h_gather<T><<<grid_for(H.nb), kBlock, 0, st>>>(H.nb, u, H.gidx, xp);
  note_launch();
  k_h_near<T><<<H.nrows, 256, 0, st>>>(H.near_rows, H.near, H.D, xp, y);
  if (H.nterms > 0) {
    note_launch();
    k_h_far_vt<T><<<int((H.nterms * 32 + 255) / 256), 256, 0, st>>>(H.terms, H.nterms, H.far, H.voff, H.toff, H.V,
                                                                      xp, t);
    dim3 grid(unsigned((H.max_group_m + 255) / 256), unsigned(H.ngroups));
    note_launch();
    k_h_far_u<T><<<grid, 256, 0, st>>>(H.groups, H.far, H.rank, H.uoff, H.toff, H.U, t, y);
  }
  note_launch();
  k_h_dirichlet<<<grid_for(n), kBlock, 0, st>>>(n, pos, y, bdir);
  TMB_CUDA(cudaGetLastError());
}

template void launch_h_compact<double>(int, const HBlockDev*, const double*, const double*, const long long*,
                                       const long long*, const int*, double*, double*, cudaStream_t);
template void launch_h_compact<float>(int, const HBlockDev*, const double*, const double*, const long long*,
                                      const long long*, const int*, float*, float*, cudaStream_t);
template void launch_h_matvec<double>(const HMatView<double>&, const double*, double*, double*, double*, const int*,
                                      int, double*, cudaStream_t);
template void launch_h_matvec<float>(const HMatView<float>&, const double*, double*, double*, float*, const int*, int,
                                     double*, cudaStream_t);

}  // namespace tmb
