// Device kernels of the preconditioned CG solver and its AMG V-cycle.
//
// These replace the linear-solver plugin of tetmag's demag chain
// (SolverFactory, main/SolverFactory.h:42-65; the AMGCL-CUDA GPUSolver,
// gpu/GPUSolver.cu:43-97), which copies b to the device and x back on every
// solve.  Here the right-hand side is produced on the device, the scalars of
// CG (rho, alpha, beta, ||r||) live in device memory and are updated by the
// last block of each reduction kernel, and the host only polls a converged
// flag.  Dot products are accumulated in FP64 with warp shuffles, a fixed
// per-block order and a fixed final order (deterministic for a given grid).
#include "tmb_dev.cuh"

namespace tmb {

namespace {

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block; the result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  if (warp == 0) {
    v = (lane < nw) ? sh[lane] : 0.0;
    v = warp_sum(v);
  }
  return v;
}

// Publishes this block's partial sums; returns true in every thread of the last
// block to finish, which then holds the grid totals in tot[0..K-1] (thread 0).
template <int K>
__device__ __forceinline__ bool grid_reduce(const double (&v)[K], double* partials, unsigned int* ticket,
                                            double (&tot)[K]) {
  __shared__ bool last;
  double bs[K];
#pragma unroll
  for (int q = 0; q < K; ++q) bs[q] = block_sum(v[q]);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < K; ++q) partials[size_t(q) * gridDim.x + blockIdx.x] = bs[q];
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < K; ++q) {
    double s = 0.0;
    for (int i = threadIdx.x; i < int(gridDim.x); i += blockDim.x) s += __ldcg(partials + size_t(q) * gridDim.x + i);
    tot[q] = block_sum(s);
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// Entries of a SELL-32 row are visited in chunks of kChunk: the chunk's column indices and
// values are loaded first (coalesced across the warp, values kept in the operator's type), then
// its kChunk gathers are issued together (FEM rows hold 10-15 entries; 16-entry chunks measured
// slower: more registers, fewer resident threads).
constexpr int kChunk = 8;

// Dot of operator row g / rep with replica g % rep of x (state row g).
template <typename V>
__device__ __forceinline__ double sell_row_dot(const SellView& s, const V* __restrict__ val,
                                               const double* __restrict__ x, int g) {
  const int R = s.rep;
  const int row = g / R, r = g - row * R;
  const int sl = row >> 5;
  const int beg = __ldg(s.soff + sl) + (row & 31);
  const int end = __ldg(s.soff + sl + 1);
  double acc = 0.0;
  for (int k0 = beg; k0 < end; k0 += kChunk * kSlice) {
    int j[kChunk];
    V v[kChunk];
#pragma unroll
    for (int u = 0; u < kChunk; ++u) {
      const int k = k0 + u * kSlice;
      const bool ok = k < end;
      j[u] = ok ? __ldg(s.col + k) * R + r : g;
      v[u] = ok ? __ldg(val + k) : V(0);
    }
#pragma unroll
    for (int u = 0; u < kChunk; ++u) acc = fma(opval(v[u], s.tab), __ldg(x + j[u]), acc);
  }
  return acc;
}

// Interleaved replicas in pairs (an even replica count of 8 or more): state rows g and g + 1 (g
// even) are two replicas of one operator row, so one thread gathers both replicas' entries with one
// 16-byte load (the pair's offset j R + r is even, so the load is aligned).
__device__ __forceinline__ double2 ld2(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ void st2(double* p, double2 v) { *reinterpret_cast<double2*>(p) = v; }

template <typename V>
__device__ __forceinline__ double2 sell_row_dot2(const SellView& s, const V* __restrict__ val,
                                                 const double* __restrict__ x, int g) {
  const int R = s.rep;
  const int row = g / R, r = g - row * R;
  const int sl = row >> 5;
  const int beg = __ldg(s.soff + sl) + (row & 31);
  const int end = __ldg(s.soff + sl + 1);
  double2 acc = make_double2(0.0, 0.0);
  for (int k0 = beg; k0 < end; k0 += kChunk * kSlice) {
    int j[kChunk];
    V v[kChunk];
#pragma unroll
    for (int u = 0; u < kChunk; ++u) {
      const int k = k0 + u * kSlice;
      const bool ok = k < end;
      j[u] = ok ? __ldg(s.col + k) * R + r : g;
      v[u] = ok ? __ldg(val + k) : V(0);
    }
#pragma unroll
    for (int u = 0; u < kChunk; ++u) {
      const double2 xv = __ldg(reinterpret_cast<const double2*>(x + j[u]));
      const double vu = opval(v[u], s.tab);
      acc.x = fma(vu, xv.x, acc.x);
      acc.y = fma(vu, xv.y, acc.y);
    }
  }
  return acc;
}

template <typename V>
__global__ void __launch_bounds__(kBlock) k_jacobi(SellView s, const V* __restrict__ val,
                                                   const double* __restrict__ dinv, const double* __restrict__ b,
                                                   const double* __restrict__ xin, double* __restrict__ xout,
                                                   const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < s.n * s.rep) xout[g] = xin[g] + dinv[g / s.rep] * (b[g] - sell_row_dot(s, val, xin, g));
}

// First smoothing sweep from zero fused with the residual: x = D_w^-1 b, r = b - A x,
// gathering D_w^-1 b on the fly instead of reading back x.
template <typename V>
__global__ void __launch_bounds__(kBlock) k_jacobi0_residual(SellView s, const V* __restrict__ val,
                                                             const double* __restrict__ dinv,
                                                             const double* __restrict__ b, double* __restrict__ x,
                                                             double* __restrict__ r, const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int R = s.rep;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= s.n * R) return;
  const int row = g / R, rr = g - row * R;
  const int sl = row >> 5;
  const int beg = __ldg(s.soff + sl) + (row & 31);
  const int end = __ldg(s.soff + sl + 1);
  double acc = 0.0;
  for (int k0 = beg; k0 < end; k0 += kChunk * kSlice) {
    int j[kChunk];
    V v[kChunk];
#pragma unroll
    for (int u = 0; u < kChunk; ++u) {
      const int k = k0 + u * kSlice;
      const bool ok = k < end;
      j[u] = ok ? __ldg(s.col + k) : row;
      v[u] = ok ? __ldg(val + k) : V(0);
    }
#pragma unroll
    for (int u = 0; u < kChunk; ++u)
      acc = fma(opval(v[u], s.tab), __ldg(dinv + j[u]) * __ldg(b + j[u] * R + rr), acc);
  }
  const double bi = b[g];
  x[g] = dinv[row] * bi;
  r[g] = bi - acc;
}

// Sum over the T consecutive lanes that share a row (T a power of two dividing 32).
template <int T>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = T / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Partial dot of a CSR row over the entries k = beg + sub, beg + sub + T, ... (x premultiplied by
// w when w is not null).
constexpr int kCsrChunk = 8;
template <typename V, int T>
__device__ __forceinline__ double csr_row_part(const CsrView& c, const V* __restrict__ val, const double* __restrict__ x,
                                               const double* __restrict__ w, int g, int sub) {
  double acc = 0.0;
  const int R = c.rep;
  if (g < c.n * R) {
    const int row = g / R, r = g - row * R;
    const int beg = __ldg(c.ptr + row), end = __ldg(c.ptr + row + 1);
    // chunks of kCsrChunk entries per thread: indices and values first, then the gathers
    for (int k0 = beg + sub; k0 < end; k0 += kCsrChunk * T) {
      int j[kCsrChunk];
      V v[kCsrChunk];
#pragma unroll
      for (int u = 0; u < kCsrChunk; ++u) {
        const int k = k0 + u * T;
        const bool ok = k < end;
        j[u] = ok ? __ldg(c.col + k) : 0;
        v[u] = ok ? __ldg(val + k) : V(0);
      }
#pragma unroll
      for (int u = 0; u < kCsrChunk; ++u) {
        const double xj = w ? __ldg(w + j[u]) * __ldg(x + j[u] * R + r) : __ldg(x + j[u] * R + r);
        acc = fma(static_cast<double>(v[u]), xj, acc);
      }
    }
  }
  return acc;
}

// CSR product (transfer operators, coarse levels); T threads cooperate on a row.
template <typename V, int T>
__global__ void __launch_bounds__(kBlock) k_csr_spmv(CsrView c, const V* __restrict__ val,
                                                     const double* __restrict__ x, double* __restrict__ y,
                                                     int accumulate, const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = t / T, sub = t & (T - 1);
  const double acc = group_sum<T>(csr_row_part<V, T>(c, val, x, nullptr, row, sub));
  if (row < c.n * c.rep && sub == 0) y[row] = accumulate ? y[row] + acc : acc;
}

// Coarse levels (rows of 20-60 entries): the first Jacobi sweep from zero fused with the
// residual, x = D_w^-1 b, r = b - A x, T threads per row.
template <typename V, int T>
__global__ void __launch_bounds__(kBlock) k_csr_jacobi0_residual(CsrView c, const V* __restrict__ val,
                                                                 const double* __restrict__ dinv,
                                                                 const double* __restrict__ b, double* __restrict__ x,
                                                                 double* __restrict__ r, const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = t / T, sub = t & (T - 1);
  const double acc = group_sum<T>(csr_row_part<V, T>(c, val, b, dinv, row, sub));
  if (row < c.n * c.rep && sub == 0) {
    const double bi = b[row];
    x[row] = dinv[row / c.rep] * bi;
    r[row] = bi - acc;
  }
}

// Coarse levels: xout = xin + D_w^-1 (b - A xin), T threads per row.
template <typename V, int T>
__global__ void __launch_bounds__(kBlock) k_csr_jacobi(CsrView c, const V* __restrict__ val,
                                                       const double* __restrict__ dinv, const double* __restrict__ b,
                                                       const double* __restrict__ xin, double* __restrict__ xout,
                                                       const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = t / T, sub = t & (T - 1);
  const double acc = group_sum<T>(csr_row_part<V, T>(c, val, xin, nullptr, row, sub));
  if (row < c.n * c.rep && sub == 0) xout[row] = xin[row] + dinv[row / c.rep] * (b[row] - acc);
}

// Coarse levels, one replica: the first sweep from zero with its residual (x = D_w^-1 b,
// r = b - A x) and the restriction of that residual in one launch.  The restricted residual needs
// no sweep result: R r = R (I - A D_w^-1) b = M b with M = R - (R A) D_w^-1, so the first nm
// blocks run the rows of M (tm threads a row: few, long rows, placed first so that they start at
// once) and the others the sweep's rows (ta threads a row).
__device__ __forceinline__ double group_sum_rt(double v, int T) {
  for (int o = T >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <typename V>
__device__ __forceinline__ double csr_row_part_rt(const CsrView& c, const V* __restrict__ val,
                                                  const double* __restrict__ x, const double* __restrict__ w, int row,
                                                  int sub, int T) {
  double acc = 0.0;
  if (row < c.n) {
    const int beg = __ldg(c.ptr + row), end = __ldg(c.ptr + row + 1);
    for (int k0 = beg + sub; k0 < end; k0 += kCsrChunk * T) {
      int j[kCsrChunk];
      V v[kCsrChunk];
#pragma unroll
      for (int u = 0; u < kCsrChunk; ++u) {
        const int k = k0 + u * T;
        const bool ok = k < end;
        j[u] = ok ? __ldg(c.col + k) : 0;
        v[u] = ok ? __ldg(val + k) : V(0);
      }
#pragma unroll
      for (int u = 0; u < kCsrChunk; ++u) {
        const double xj = w ? __ldg(w + j[u]) * __ldg(x + j[u]) : __ldg(x + j[u]);
        acc = fma(static_cast<double>(v[u]), xj, acc);
      }
    }
  }
  return acc;
}
template <typename V>
__global__ void __launch_bounds__(kBlock) k_csr_pre_restrict(CsrView a, const V* __restrict__ aval,
                                                             const double* __restrict__ dinv,
                                                             const double* __restrict__ b, double* __restrict__ x,
                                                             double* __restrict__ r, int ta, int nm, CsrView m,
                                                             const V* __restrict__ mval, double* __restrict__ bc,
                                                             int tm, const int* done) {
  pdl_enter();
  if (done && *done) return;
  if (int(blockIdx.x) < nm) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = t / tm, sub = t & (tm - 1);
    const double acc = group_sum_rt(csr_row_part_rt(m, mval, b, nullptr, row, sub, tm), tm);
    if (row < m.n && sub == 0) bc[row] = acc;
  } else {
    const int t = (blockIdx.x - nm) * blockDim.x + threadIdx.x;
    const int row = t / ta, sub = t & (ta - 1);
    const double acc = group_sum_rt(csr_row_part_rt(a, aval, b, dinv, row, sub, ta), ta);
    if (row < a.n && sub == 0) {
      const double bi = b[row];
      x[row] = dinv[row] * bi;
      r[row] = bi - acc;
    }
  }
}

// Coarse levels: the prolongation x += P c and the post-smoothing sweep in one pass.  With X0, R0
// the pre-smoothed iterate and its residual (R0 = b - A X0), the sweep from X0 + P c is
//   out = X0 + P c + D_w^-1 (R0 - (A P) c),
// so one product over the rows of A P (whose pattern holds P's, a row of each per entry: pv, apv)
// replaces the transfer kernel and the sweep's product with A; c is the coarser level's result.
template <typename V, int T>
__global__ void __launch_bounds__(kBlock) k_csr_prolong_smooth(CsrView m, const V* __restrict__ apv,
                                                               const V* __restrict__ pv,
                                                               const double* __restrict__ dinv,
                                                               const double* __restrict__ x0,
                                                               const double* __restrict__ r0,
                                                               const double* __restrict__ c, double* __restrict__ out,
                                                               const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int g = t / T, sub = t & (T - 1);
  const int R = m.rep;
  double ap = 0.0, pp = 0.0;
  if (g < m.n * R) {
    const int row = g / R, r = g - row * R;
    const int beg = __ldg(m.ptr + row), end = __ldg(m.ptr + row + 1);
    for (int k0 = beg + sub; k0 < end; k0 += kCsrChunk * T) {
      int j[kCsrChunk];
      V a[kCsrChunk], p[kCsrChunk];
#pragma unroll
      for (int u = 0; u < kCsrChunk; ++u) {
        const int k = k0 + u * T;
        const bool ok = k < end;
        j[u] = ok ? __ldg(m.col + k) : 0;
        a[u] = ok ? __ldg(apv + k) : V(0);
        p[u] = ok ? __ldg(pv + k) : V(0);
      }
#pragma unroll
      for (int u = 0; u < kCsrChunk; ++u) {
        const double cj = __ldg(c + j[u] * R + r);
        ap = fma(static_cast<double>(a[u]), cj, ap);
        pp = fma(static_cast<double>(p[u]), cj, pp);
      }
    }
  }
  ap = group_sum<T>(ap);
  pp = group_sum<T>(pp);
  if (g < m.n * R && sub == 0) out[g] = x0[g] + pp + dinv[g / R] * (r0[g] - ap);
}

// x = A_c^-1 b on the coarsest level (dense FP64 inverse, row-major, even leading dimension ld):
// one warp per row and replica.
__global__ void k_coarse_solve(int n, int ld, int R, const double* __restrict__ inv, const double* __restrict__ b,
                               double* __restrict__ x, const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (g >= n * R) return;
  const int i = g / R, r = g - i * R;
  const double* row = inv + size_t(i) * ld;
  double acc = 0.0;
  for (int j = lane; j < n; j += 32) acc = fma(row[j], b[j * R + r], acc);
  acc = warp_sum(acc);
  if (lane == 0) x[g] = acc;
}

// Coarsest level with decoupled rows (AmgHierarchy::coarse_idx): x = D^-1 b on every row, then the
// coupled rows are gathered into a compact vector, solved densely, and scattered back.
__global__ void k_coarse_diag(int n, int R, const double* __restrict__ dinv, const double* __restrict__ b,
                              double* __restrict__ x, const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n * R) return;
  x[g] = dinv[g / R] * b[g];
}

// dst[k * R + r] = src[idx[k] * R + r] (gather), or dst[idx[k] * R + r] = src[k * R + r] (scatter)
__global__ void k_rows_move(int m, int R, const int* __restrict__ idx, const double* __restrict__ src,
                            double* __restrict__ dst, int scatter, const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= m * R) return;
  const int k = g / R, r = g - k * R;
  if (scatter) dst[idx[k] * R + r] = src[g];
  else dst[g] = src[idx[k] * R + r];
}

// The same product for one replica and a larger coarsest level: one 128-thread CTA per row, all
// of a thread's 16-byte loads of the row issued together.
__global__ void __launch_bounds__(128) k_coarse_solve_rows(int n, int ld, const double* __restrict__ inv,
                                                           const double* __restrict__ b, double* __restrict__ x,
                                                           const int* done) {
  pdl_enter();
  if (done && *done) return;
  __shared__ double red[4];
  const double2* row = reinterpret_cast<const double2*>(inv + size_t(blockIdx.x) * ld);
  const int np = ld / 2;
  double a0 = 0.0, a1 = 0.0;
  for (int j = threadIdx.x; j < np; j += 128) {
    const double2 v = __ldg(row + j);
    const int c = 2 * j;
    a0 = fma(v.x, __ldg(b + c), a0);
    if (c + 1 < n) a1 = fma(v.y, __ldg(b + c + 1), a1);
  }
  double a = warp_sum(a0 + a1);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) x[blockIdx.x] = (red[0] + red[1]) + (red[2] + red[3]);
}

// The mixed path's form: an FP32 copy of the inverse (rows padded to a multiple of 4, 16-byte loads
// of four entries), FP64 products and sums.  The coarsest solve only feeds the preconditioner.
__global__ void __launch_bounds__(128) k_coarse_solve_rows_f32(int n, int ld, const float* __restrict__ inv,
                                                               const double* __restrict__ b, double* __restrict__ x,
                                                               const int* done) {
  pdl_enter();
  if (done && *done) return;
  __shared__ double red[4];
  const float4* row = reinterpret_cast<const float4*>(inv + size_t(blockIdx.x) * ld);
  const int nq = ld / 4;
  double a0 = 0.0, a1 = 0.0;
  for (int j = threadIdx.x; j < nq; j += 128) {
    const float4 v = __ldg(row + j);
    const int c = 4 * j;  // padded entries are zero; b is read only below n
    a0 = fma(double(v.x), __ldg(b + c), a0);
    if (c + 1 < n) a1 = fma(double(v.y), __ldg(b + c + 1), a1);
    if (c + 2 < n) a0 = fma(double(v.z), __ldg(b + c + 2), a0);
    if (c + 3 < n) a1 = fma(double(v.w), __ldg(b + c + 3), a1);
  }
  double a = warp_sum(a0 + a1);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) x[blockIdx.x] = (red[0] + red[1]) + (red[2] + red[3]);
}

template <typename V>
__global__ void k_cg_init(int n, CsrView lift, const V* __restrict__ lval, const int* __restrict__ cmask,
                          const double* __restrict__ b, double* __restrict__ bprime, double* __restrict__ x) {
  pdl_enter();
  const int R = lift.rep;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n * R) return;
  const int i = g / R, r = g - i * R;
  if (cmask[i]) {
    bprime[g] = b[g];
    x[g] = b[g];
  } else {
    double acc = b[g];
    for (int k = lift.ptr[i]; k < lift.ptr[i + 1]; ++k) acc -= static_cast<double>(lval[k]) * b[lift.col[k] * R + r];
    bprime[g] = acc;
  }
}

template <typename V>
__global__ void __launch_bounds__(kBlock) k_cg_residual(SellView s, const V* __restrict__ val,
                                                        const double* __restrict__ bp, const double* __restrict__ x,
                                                        double* __restrict__ r, CgScalars* S, double* partials) {
  pdl_enter();
  double v[2] = {0.0, 0.0};
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < s.n * s.rep; g += gridDim.x * blockDim.x) {
    const double ri = bp[g] - sell_row_dot(s, val, x, g);
    r[g] = ri;
    v[0] = fma(ri, ri, v[0]);
    v[1] = fma(bp[g], bp[g], v[1]);
  }
  double tot[2];
  if (grid_reduce<2>(v, partials, &S->ticket[0], tot) && threadIdx.x == 0) {
    S->rr = tot[0];
    S->bb = tot[1];
    S->iter = 0;
    S->status = 0;
    if (tot[1] == 0.0) {
      S->done = 1;
      S->status = 2;  // zero right-hand side: the host sets x = 0
    } else {
      S->done = (tot[0] <= S->tol2 * tot[1]) ? 1 : 0;
    }
  }
}

__global__ void __launch_bounds__(kBlock) k_cg_rz(int n, const double* __restrict__ r, const double* __restrict__ z,
                                                  CgScalars* S, double* partials, int first) {
  pdl_enter();
  if (S->done) return;
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[0] = fma(r[i], z[i], v[0]);
  double tot[1];
  if (grid_reduce<1>(v, partials, &S->ticket[1], tot) && threadIdx.x == 0) {
    if (first) {
      S->beta = 0.0;
    } else {
      S->beta = tot[0] / S->rz;
    }
    S->rz = tot[0];
  }
}

// Last post-smoothing sweep of the finest level fused with rho = r.z:
// z = x + D_w^-1 (r - A x); the last block sets beta = rho_new / rho (0 on the first pass).
template <typename V>
__global__ void __launch_bounds__(kBlock) k_jacobi_rz(SellView s, const V* __restrict__ val,
                                                      const double* __restrict__ dinv, const double* __restrict__ r,
                                                      const double* __restrict__ xin, double* __restrict__ z,
                                                      CgScalars* S, double* partials, int first) {
  pdl_enter();
  if (S->done) return;
  double v[1] = {0.0};
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < s.n * s.rep; g += gridDim.x * blockDim.x) {
    const double ri = r[g];
    const double zi = xin[g] + dinv[g / s.rep] * (ri - sell_row_dot(s, val, xin, g));
    z[g] = zi;
    v[0] = fma(ri, zi, v[0]);
  }
  double tot[1];
  if (grid_reduce<1>(v, partials, &S->ticket[1], tot) && threadIdx.x == 0) {
    S->beta = first ? 0.0 : tot[0] / S->rz;
    S->rz = tot[0];
  }
}

// New direction and its product without gathering p: p = z + beta p and q = A p = A z + beta q
// (the previous q is A p_old), both updated in place for the own row, so the product gathers z
// alone; p.q reduced, the last block sets alpha.  beta = 0 (first pass) reads neither old vector.
template <typename V>
__global__ void __launch_bounds__(kBlock) k_cg_dir_spmv(SellView s, const V* __restrict__ val,
                                                        const double* __restrict__ z, double* __restrict__ p,
                                                        double* __restrict__ q, CgScalars* S, double* partials) {
  pdl_enter();
  if (S->done) return;
  const double beta = S->beta;
  double v[1] = {0.0};
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < s.n * s.rep; g += gridDim.x * blockDim.x) {
    const double az = sell_row_dot(s, val, z, g);
    const double zi = z[g];
    const double pi = (beta == 0.0) ? zi : fma(beta, p[g], zi);
    const double qi = (beta == 0.0) ? az : fma(beta, q[g], az);
    p[g] = pi;
    q[g] = qi;
    v[0] = fma(pi, qi, v[0]);
  }
  double tot[1];
  if (grid_reduce<1>(v, partials, &S->ticket[2], tot) && threadIdx.x == 0) {
    S->pq = tot[0];
    S->alpha = S->rz / tot[0];
  }
}

// The CG update fused with the first smoothing sweep of the V-cycle on the finest level:
// x += alpha p and r_new = r - alpha q for the own row (||r_new||^2 reduced, the last block
// decides convergence as k_cg_update does), then X = D_w^-1 r_new and R = r_new - A X, with the
// neighbours' r_new formed on the fly from r and q.  r and r_new are different buffers.
template <typename V>
__global__ void __launch_bounds__(kBlock) k_cg_update_jacobi0(SellView s, const V* __restrict__ val,
                                                              const double* __restrict__ dinv,
                                                              const double* __restrict__ p,
                                                              const double* __restrict__ q, double* __restrict__ x,
                                                              const double* __restrict__ r, double* __restrict__ r_new,
                                                              double* __restrict__ X, double* __restrict__ Rres,
                                                              CgScalars* S, double* partials) {
  pdl_enter();
  if (S->done) return;
  const double alpha = S->alpha;
  const int R = s.rep;
  double v[1] = {0.0};
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < s.n * R; g += gridDim.x * blockDim.x) {
    const int row = g / R, rr = g - row * R;
    const int sl = row >> 5;
    const int beg = __ldg(s.soff + sl) + (row & 31);
    const int end = __ldg(s.soff + sl + 1);
    double acc = 0.0;
    for (int k0 = beg; k0 < end; k0 += kChunk * kSlice) {
      int j[kChunk];
      V w[kChunk];
#pragma unroll
      for (int u = 0; u < kChunk; ++u) {
        const int k = k0 + u * kSlice;
        const bool ok = k < end;
        j[u] = ok ? __ldg(s.col + k) : row;
        w[u] = ok ? __ldg(val + k) : V(0);
      }
#pragma unroll
      for (int u = 0; u < kChunk; ++u) {
        const int jj = j[u] * R + rr;
        acc = fma(opval(w[u], s.tab), __ldg(dinv + j[u]) * fma(-alpha, __ldg(q + jj), __ldg(r + jj)), acc);
      }
    }
    const double ri = fma(-alpha, q[g], r[g]);
    x[g] = fma(alpha, p[g], x[g]);
    r_new[g] = ri;
    X[g] = dinv[row] * ri;
    Rres[g] = ri - acc;
    v[0] = fma(ri, ri, v[0]);
  }
  double tot[1];
  if (grid_reduce<1>(v, partials, &S->ticket[3], tot) && threadIdx.x == 0) {
    S->rr = tot[0];
    S->iter += 1;
    if (!(tot[0] == tot[0]) || !(S->pq > 0.0)) {
      S->done = 1;
      S->status = 5;  // breakdown / NaN
    } else if (tot[0] <= S->tol2 * S->bb) {
      S->done = 1;
    } else if (S->iter >= S->maxit) {
      S->done = 1;
      S->status = 3;  // not converged within maxit
    }
  }
}

__global__ void __launch_bounds__(kBlock) k_cg_update(int n, const double* __restrict__ p,
                                                      const double* __restrict__ q, double* __restrict__ x,
                                                      double* __restrict__ r, CgScalars* S, double* partials) {
  pdl_enter();
  if (S->done) return;
  const double alpha = S->alpha;
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = fma(alpha, p[i], x[i]);
    const double ri = fma(-alpha, q[i], r[i]);
    r[i] = ri;
    v[0] = fma(ri, ri, v[0]);
  }
  double tot[1];
  if (grid_reduce<1>(v, partials, &S->ticket[3], tot) && threadIdx.x == 0) {
    S->rr = tot[0];
    S->iter += 1;
    if (!(tot[0] == tot[0]) || !(S->pq > 0.0)) {
      S->done = 1;
      S->status = 5;  // breakdown / NaN
    } else if (tot[0] <= S->tol2 * S->bb) {
      S->done = 1;
    } else if (S->iter >= S->maxit) {
      S->done = 1;
      S->status = 3;  // not converged within maxit
    }
  }
}

// Pair forms of the three finest-level kernels for interleaved replicas (see sell_row_dot2).
template <typename V>
__global__ void __launch_bounds__(kBlock) k_jacobi0_residual2(SellView s, const V* __restrict__ val,
                                                              const double* __restrict__ dinv,
                                                              const double* __restrict__ b, double* __restrict__ x,
                                                              double* __restrict__ r, const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int R = s.rep;
  const int g = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (g >= s.n * R) return;
  const int row = g / R, rr = g - row * R;
  const int sl = row >> 5;
  const int beg = __ldg(s.soff + sl) + (row & 31);
  const int end = __ldg(s.soff + sl + 1);
  double2 acc = make_double2(0.0, 0.0);
  for (int k0 = beg; k0 < end; k0 += kChunk * kSlice) {
    int j[kChunk];
    V v[kChunk];
#pragma unroll
    for (int u = 0; u < kChunk; ++u) {
      const int k = k0 + u * kSlice;
      const bool ok = k < end;
      j[u] = ok ? __ldg(s.col + k) : row;
      v[u] = ok ? __ldg(val + k) : V(0);
    }
#pragma unroll
    for (int u = 0; u < kChunk; ++u) {
      const double w = opval(v[u], s.tab) * __ldg(dinv + j[u]);
      const double2 bj = __ldg(reinterpret_cast<const double2*>(b + j[u] * R + rr));
      acc.x = fma(w, bj.x, acc.x);
      acc.y = fma(w, bj.y, acc.y);
    }
  }
  const double2 bi = ld2(b + g);
  const double d = dinv[row];
  st2(x + g, make_double2(d * bi.x, d * bi.y));
  st2(r + g, make_double2(bi.x - acc.x, bi.y - acc.y));
}

template <typename V>
__global__ void __launch_bounds__(kBlock) k_jacobi_rz2(SellView s, const V* __restrict__ val,
                                                       const double* __restrict__ dinv, const double* __restrict__ r,
                                                       const double* __restrict__ xin, double* __restrict__ z,
                                                       CgScalars* S, double* partials, int first) {
  pdl_enter();
  if (S->done) return;
  double v[1] = {0.0};
  const int n2 = s.n * s.rep / 2;
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < n2; h += gridDim.x * blockDim.x) {
    const int g = 2 * h;
    const double2 ax = sell_row_dot2(s, val, xin, g);
    const double2 ri = ld2(r + g), xi = ld2(xin + g);
    const double d = dinv[g / s.rep];
    const double2 zi = make_double2(xi.x + d * (ri.x - ax.x), xi.y + d * (ri.y - ax.y));
    st2(z + g, zi);
    v[0] = fma(ri.x, zi.x, v[0]);
    v[0] = fma(ri.y, zi.y, v[0]);
  }
  double tot[1];
  if (grid_reduce<1>(v, partials, &S->ticket[1], tot) && threadIdx.x == 0) {
    S->beta = first ? 0.0 : tot[0] / S->rz;
    S->rz = tot[0];
  }
}

template <typename V>
__global__ void __launch_bounds__(kBlock) k_cg_dir_spmv2(SellView s, const V* __restrict__ val,
                                                         const double* __restrict__ z, double* __restrict__ p,
                                                         double* __restrict__ q, CgScalars* S, double* partials) {
  pdl_enter();
  if (S->done) return;
  const double beta = S->beta;
  double v[1] = {0.0};
  const int n2 = s.n * s.rep / 2;
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < n2; h += gridDim.x * blockDim.x) {
    const int g = 2 * h;
    const double2 az = sell_row_dot2(s, val, z, g);
    const double2 zi = ld2(z + g);
    double2 pi = zi, qi = az;
    if (beta != 0.0) {
      const double2 po = ld2(p + g), qo = ld2(q + g);
      pi = make_double2(fma(beta, po.x, zi.x), fma(beta, po.y, zi.y));
      qi = make_double2(fma(beta, qo.x, az.x), fma(beta, qo.y, az.y));
    }
    st2(p + g, pi);
    st2(q + g, qi);
    v[0] = fma(pi.x, qi.x, v[0]);
    v[0] = fma(pi.y, qi.y, v[0]);
  }
  double tot[1];
  if (grid_reduce<1>(v, partials, &S->ticket[2], tot) && threadIdx.x == 0) {
    S->pq = tot[0];
    S->alpha = S->rz / tot[0];
  }
}

// Pair forms of the CSR kernels (coarser levels and transfer operators) for interleaved replicas:
// thread -> state rows g, g + 1 (g even) of one operator row, one aligned 16-byte gather per entry.
template <typename V>
__device__ __forceinline__ double2 csr_row_part2(const CsrView& c, const V* __restrict__ val,
                                                 const double* __restrict__ x, const double* __restrict__ w, int g) {
  const int R = c.rep;
  const int row = g / R, r = g - row * R;
  const int beg = __ldg(c.ptr + row), end = __ldg(c.ptr + row + 1);
  double2 acc = make_double2(0.0, 0.0);
  for (int k0 = beg; k0 < end; k0 += kCsrChunk) {
    int j[kCsrChunk];
    V v[kCsrChunk];
#pragma unroll
    for (int u = 0; u < kCsrChunk; ++u) {
      const int k = k0 + u;
      const bool ok = k < end;
      j[u] = ok ? __ldg(c.col + k) : 0;
      v[u] = ok ? __ldg(val + k) : V(0);
    }
#pragma unroll
    for (int u = 0; u < kCsrChunk; ++u) {
      const double wv = w ? static_cast<double>(v[u]) * __ldg(w + j[u]) : static_cast<double>(v[u]);
      const double2 xv = __ldg(reinterpret_cast<const double2*>(x + j[u] * R + r));
      acc.x = fma(wv, xv.x, acc.x);
      acc.y = fma(wv, xv.y, acc.y);
    }
  }
  return acc;
}

template <typename V>
__global__ void __launch_bounds__(kBlock) k_csr_spmv2(CsrView c, const V* __restrict__ val,
                                                      const double* __restrict__ x, double* __restrict__ y,
                                                      int accumulate, const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int g = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (g >= c.n * c.rep) return;
  const double2 acc = csr_row_part2(c, val, x, nullptr, g);
  if (accumulate) {
    const double2 yo = ld2(y + g);
    st2(y + g, make_double2(yo.x + acc.x, yo.y + acc.y));
  } else {
    st2(y + g, acc);
  }
}

template <typename V>
__global__ void __launch_bounds__(kBlock) k_csr_jacobi0_residual2(CsrView c, const V* __restrict__ val,
                                                                  const double* __restrict__ dinv,
                                                                  const double* __restrict__ b, double* __restrict__ x,
                                                                  double* __restrict__ r, const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int g = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (g >= c.n * c.rep) return;
  const double2 acc = csr_row_part2(c, val, b, dinv, g);
  const double2 bi = ld2(b + g);
  const double d = dinv[g / c.rep];
  st2(x + g, make_double2(d * bi.x, d * bi.y));
  st2(r + g, make_double2(bi.x - acc.x, bi.y - acc.y));
}

template <typename V>
__global__ void __launch_bounds__(kBlock) k_csr_jacobi2(CsrView c, const V* __restrict__ val,
                                                        const double* __restrict__ dinv, const double* __restrict__ b,
                                                        const double* __restrict__ xin, double* __restrict__ xout,
                                                        const int* done) {
  pdl_enter();
  if (done && *done) return;
  const int g = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (g >= c.n * c.rep) return;
  const double2 acc = csr_row_part2(c, val, xin, nullptr, g);
  const double2 bi = ld2(b + g), xi = ld2(xin + g);
  const double d = dinv[g / c.rep];
  st2(xout + g, make_double2(xi.x + d * (bi.x - acc.x), xi.y + d * (bi.y - acc.y)));
}

}  // namespace

// Interleaved replicas taken in pairs by the finest-level kernels: an even count of 8 or more.
static bool paired(const SellView& s) { return s.rep >= 8 && s.rep % 2 == 0; }
static bool paired(const CsrView& c, int tpr) { return tpr == 1 && c.rep >= 8 && c.rep % 2 == 0; }

// Grid of the reduction kernels: at most eight 256-thread blocks per SM (a full SM); the rows
// beyond are covered by a grid-stride loop, so that the blocks' publish-and-count tails are few.
int reduce_grid(long long n) {
  static int cap = 0;
  if (cap == 0) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cap = 8 * sms;
  }
  const int g = grid_for(n);
  return g < cap ? g : cap;
}

template <typename V>
void launch_jacobi(const SellView& s, const V* val, const double* dinv, const double* b, const double* xin,
                   double* xout, const int* done, cudaStream_t st) {
  note_launch();
  launch_pdl(k_jacobi<V>, grid_for(1LL * s.n * s.rep), kBlock, 0, st, s, val, dinv, b, xin, xout, done);
}
int csr_threads_per_row(long long nrows, long long nnz) {
  const double avg = nrows > 0 ? double(nnz) / double(nrows) : 0.0;
  int t = 1;
  while (t < 32 && t * 6 < avg) t *= 2;  // about six entries per thread
  return t;
}

#define TMB_CSR_DISPATCH(T, KERNEL, NROWS, ...)                                                            \
  switch (T) {                                                                                            \
    case 1: launch_pdl(KERNEL<V, 1>, grid_for(1LL * (NROWS)), kBlock, 0, st, __VA_ARGS__); break;                 \
    case 2: launch_pdl(KERNEL<V, 2>, grid_for(2LL * (NROWS)), kBlock, 0, st, __VA_ARGS__); break;                 \
    case 4: launch_pdl(KERNEL<V, 4>, grid_for(4LL * (NROWS)), kBlock, 0, st, __VA_ARGS__); break;                 \
    case 8: launch_pdl(KERNEL<V, 8>, grid_for(8LL * (NROWS)), kBlock, 0, st, __VA_ARGS__); break;                 \
    case 16: launch_pdl(KERNEL<V, 16>, grid_for(16LL * (NROWS)), kBlock, 0, st, __VA_ARGS__); break;              \
    default: launch_pdl(KERNEL<V, 32>, grid_for(32LL * (NROWS)), kBlock, 0, st, __VA_ARGS__); break;              \
  }

template <typename V>
void launch_csr_spmv(const CsrView& c, const V* val, const double* x, double* y, bool accumulate,
                     const int* done, cudaStream_t st, int tpr) {
  note_launch();
  if (paired(c, tpr)) {
    launch_pdl(k_csr_spmv2<V>, grid_for(1LL * c.n * c.rep / 2), kBlock, 0, st, c, val, x, y, accumulate ? 1 : 0, done);
    return;
  }
  TMB_CSR_DISPATCH(tpr, k_csr_spmv, 1LL * c.n * c.rep, c, val, x, y, accumulate ? 1 : 0, done)
}
template <typename V>
void launch_csr_jacobi0_residual(const CsrView& c, const V* val, const double* dinv, const double* b, double* x,
                                 double* r, const int* done, cudaStream_t st, int tpr) {
  note_launch();
  if (paired(c, tpr)) {
    launch_pdl(k_csr_jacobi0_residual2<V>, grid_for(1LL * c.n * c.rep / 2), kBlock, 0, st, c, val, dinv, b, x, r, done);
    return;
  }
  TMB_CSR_DISPATCH(tpr, k_csr_jacobi0_residual, 1LL * c.n * c.rep, c, val, dinv, b, x, r, done)
}
template <typename V>
void launch_csr_jacobi(const CsrView& c, const V* val, const double* dinv, const double* b, const double* xin,
                       double* xout, const int* done, cudaStream_t st, int tpr) {
  note_launch();
  if (paired(c, tpr)) {
    launch_pdl(k_csr_jacobi2<V>, grid_for(1LL * c.n * c.rep / 2), kBlock, 0, st, c, val, dinv, b, xin, xout, done);
    return;
  }
  TMB_CSR_DISPATCH(tpr, k_csr_jacobi, 1LL * c.n * c.rep, c, val, dinv, b, xin, xout, done)
}
template <typename V>
void launch_csr_pre_restrict(const CsrView& a, const V* aval, const double* dinv, const double* b, double* x,
                             double* r, int ta, const CsrView& m, const V* mval, double* bc, int tm, const int* done,
                             cudaStream_t st) {
  note_launch();
  const int na = grid_for(1LL * ta * a.n), nm = grid_for(1LL * tm * m.n);
  launch_pdl(k_csr_pre_restrict<V>, na + nm, kBlock, 0, st, a, aval, dinv, b, x, r, ta, nm, m, mval, bc, tm, done);
}
template <typename V>
void launch_csr_prolong_smooth(const CsrView& m, const V* apv, const V* pv, const double* dinv, const double* x0,
                               const double* r0, const double* c, double* out, const int* done, cudaStream_t st,
                               int tpr) {
  note_launch();
  TMB_CSR_DISPATCH(tpr, k_csr_prolong_smooth, 1LL * m.n * m.rep, m, apv, pv, dinv, x0, r0, c, out, done)
}
#undef TMB_CSR_DISPATCH
void launch_coarse_solve(int n, int ld, int rep, const double* inv, const double* b, double* x, const int* done,
                         cudaStream_t st, const float* invf, int ldf) {
  note_launch();
  if (rep == 1 && n >= 256 && invf) launch_pdl(k_coarse_solve_rows_f32, n, 128, 0, st, n, ldf, invf, b, x, done);
  else if (rep == 1 && n >= 256) launch_pdl(k_coarse_solve_rows, n, 128, 0, st, n, ld, inv, b, x, done);
  else launch_pdl(k_coarse_solve, grid_for(32LL * n * rep), kBlock, 0, st, n, ld, rep, inv, b, x, done);
}
void launch_coarse_diag(int n, int rep, const double* dinv, const double* b, double* x, const int* done,
                        cudaStream_t st) {
  note_launch();
  launch_pdl(k_coarse_diag, grid_for(1LL * n * rep), kBlock, 0, st, n, rep, dinv, b, x, done);
}
void launch_rows_move(int m, int rep, const int* idx, const double* src, double* dst, bool scatter,
                      const int* done, cudaStream_t st) {
  if (m <= 0) return;
  note_launch();
  launch_pdl(k_rows_move, grid_for(1LL * m * rep), kBlock, 0, st, m, rep, idx, src, dst, scatter ? 1 : 0, done);
}
template <typename V>
void launch_cg_init(int n, const CsrView& lift, const V* lval, const int* cmask, const double* b,
                    double* bprime, double* x, cudaStream_t st) {
  note_launch();
  launch_pdl(k_cg_init<V>, grid_for(1LL * n * lift.rep), kBlock, 0, st, n, lift, lval, cmask, b, bprime, x);
}
template <typename V>
void launch_cg_residual(const SellView& s, const V* val, const double* bp, const double* x, double* r,
                        CgScalars* S, double* partials, cudaStream_t st) {
  note_launch();
  launch_pdl(k_cg_residual<V>, reduce_grid(1LL * s.n * s.rep), kBlock, 0, st, s, val, bp, x, r, S, partials);
}
void launch_cg_rz(int n, const double* r, const double* z, CgScalars* S, double* partials, bool first,
                  cudaStream_t st) {
  note_launch();
  launch_pdl(k_cg_rz, reduce_grid(n), kBlock, 0, st, n, r, z, S, partials, first ? 1 : 0);
}
template <typename V>
void launch_jacobi0_residual(const SellView& s, const V* val, const double* dinv, const double* b, double* x,
                             double* r, const int* done, cudaStream_t st) {
  note_launch();
  if (paired(s)) launch_pdl(k_jacobi0_residual2<V>, grid_for(1LL * s.n * s.rep / 2), kBlock, 0, st, s, val, dinv, b, x, r, done);
  else launch_pdl(k_jacobi0_residual<V>, grid_for(1LL * s.n * s.rep), kBlock, 0, st, s, val, dinv, b, x, r, done);
}
template <typename V>
void launch_jacobi_rz(const SellView& s, const V* val, const double* dinv, const double* r, const double* xin,
                      double* z, CgScalars* S, double* partials, bool first, cudaStream_t st) {
  note_launch();
  if (paired(s))
    launch_pdl(k_jacobi_rz2<V>, reduce_grid(1LL * s.n * s.rep / 2), kBlock, 0, st, s, val, dinv, r, xin, z, S, partials,
               first ? 1 : 0);
  else
    launch_pdl(k_jacobi_rz<V>, reduce_grid(1LL * s.n * s.rep), kBlock, 0, st, s, val, dinv, r, xin, z, S, partials,
               first ? 1 : 0);
}
template <typename V>
void launch_cg_dir_spmv(const SellView& s, const V* val, const double* z, double* p, double* q, CgScalars* S,
                        double* partials, cudaStream_t st) {
  note_launch();
  if (paired(s)) launch_pdl(k_cg_dir_spmv2<V>, reduce_grid(1LL * s.n * s.rep / 2), kBlock, 0, st, s, val, z, p, q, S, partials);
  else launch_pdl(k_cg_dir_spmv<V>, reduce_grid(1LL * s.n * s.rep), kBlock, 0, st, s, val, z, p, q, S, partials);
}
template <typename V>
void launch_cg_update_jacobi0(const SellView& s, const V* val, const double* dinv, const double* p, const double* q,
                              double* x, const double* r, double* r_new, double* X, double* Rres, CgScalars* S,
                              double* partials, cudaStream_t st) {
  note_launch();
  launch_pdl(k_cg_update_jacobi0<V>, reduce_grid(1LL * s.n * s.rep), kBlock, 0, st, s, val, dinv, p, q, x, r, r_new,
               X, Rres, S, partials);
}

void launch_cg_update(int n, const double* p, const double* q, double* x, double* r, CgScalars* S,
                      double* partials, cudaStream_t st) {
  note_launch();
  launch_pdl(k_cg_update, reduce_grid(n), kBlock, 0, st, n, p, q, x, r, S, partials);
}

#define TMB_INST(V)                                                                                          \
  template void launch_jacobi<V>(const SellView&, const V*, const double*, const double*, const double*,    \
                                 double*, const int*, cudaStream_t);                                        \
  template void launch_csr_spmv<V>(const CsrView&, const V*, const double*, double*, bool, const int*,      \
                                   cudaStream_t, int);                                                      \
  template void launch_csr_jacobi0_residual<V>(const CsrView&, const V*, const double*, const double*,      \
                                               double*, double*, const int*, cudaStream_t, int);            \
  template void launch_csr_pre_restrict<V>(const CsrView&, const V*, const double*, const double*, double*,  \
                                           double*, int, const CsrView&, const V*, double*, int, const int*,  \
                                           cudaStream_t);                                                     \
  template void launch_csr_prolong_smooth<V>(const CsrView&, const V*, const V*, const double*,             \
                                             const double*, const double*, const double*, double*,          \
                                             const int*, cudaStream_t, int);                                \
  template void launch_csr_jacobi<V>(const CsrView&, const V*, const double*, const double*, const double*, \
                                     double*, const int*, cudaStream_t, int);                               \
  template void launch_cg_init<V>(int, const CsrView&, const V*, const int*, const double*, double*,        \
                                  double*, cudaStream_t);                                                   \
  template void launch_cg_residual<V>(const SellView&, const V*, const double*, const double*, double*,     \
                                      CgScalars*, double*, cudaStream_t);                                   \
  template void launch_jacobi0_residual<V>(const SellView&, const V*, const double*, const double*, double*, \
                                           double*, const int*, cudaStream_t);                              \
  template void launch_jacobi_rz<V>(const SellView&, const V*, const double*, const double*, const double*, \
                                    double*, CgScalars*, double*, bool, cudaStream_t);                      \
  template void launch_cg_dir_spmv<V>(const SellView&, const V*, const double*, double*, double*, CgScalars*, \
                                      double*, cudaStream_t);                                                 \
  template void launch_cg_update_jacobi0<V>(const SellView&, const V*, const double*, const double*,         \
                                            const double*, double*, const double*, double*, double*, double*, \
                                            CgScalars*, double*, cudaStream_t);
TMB_INST(double)
TMB_INST(float)
#undef TMB_INST

// Finest-level kernels on dictionary-coded values (one-byte indices into SellView::tab).
#define TMB_INST_SELL(V)                                                                                     \
  template void launch_jacobi<V>(const SellView&, const V*, const double*, const double*, const double*,    \
                                 double*, const int*, cudaStream_t);                                        \
  template void launch_cg_residual<V>(const SellView&, const V*, const double*, const double*, double*,     \
                                      CgScalars*, double*, cudaStream_t);                                   \
  template void launch_jacobi0_residual<V>(const SellView&, const V*, const double*, const double*, double*, \
                                           double*, const int*, cudaStream_t);                              \
  template void launch_jacobi_rz<V>(const SellView&, const V*, const double*, const double*, const double*, \
                                    double*, CgScalars*, double*, bool, cudaStream_t);                      \
  template void launch_cg_dir_spmv<V>(const SellView&, const V*, const double*, double*, double*, CgScalars*, \
                                      double*, cudaStream_t);                                                 \
  template void launch_cg_update_jacobi0<V>(const SellView&, const V*, const double*, const double*,         \
                                            const double*, double*, const double*, double*, double*, double*, \
                                            CgScalars*, double*, cudaStream_t);
TMB_INST_SELL(uint8_t)
#undef TMB_INST_SELL

}  // namespace tmb
