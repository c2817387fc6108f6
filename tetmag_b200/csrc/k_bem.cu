// Boundary-element kernels of the demag chain: the dense boundary matvec and
// its gather / scatter (the assembly is in k_bem_assemble.cu).
//
// The matvec replaces DemagField::boundaryIntegral / denseMVP
// (main/DemagField.cpp:145-147, 184-201), which gathers u1 on the host and
// runs an Eigen GEMV there.
#include <cmath>

#include "tmb_dev.cuh"

namespace tmb {

namespace {

__global__ void k_to_float(const double* __restrict__ s, float* __restrict__ d, size_t n) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) d[i] = static_cast<float>(s[i]);
}

// x_b = u[bnodes] in the value type of the BEM matrix (FP32 on the mixed path).
template <typename V>
__global__ void k_gather(int nb, const double* __restrict__ u, const int* __restrict__ idx, V* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nb) out[i] = static_cast<V>(u[idx[i]]);
}

template <typename V>
struct Vec16;  // 16-byte vector of V
template <>
struct Vec16<float> {
  using T = float4;
  static constexpr int W = 4;
  __device__ static double dot(const float4& a, const float4& b) {
    return double(a.x) * double(b.x) + double(a.y) * double(b.y) + double(a.z) * double(b.z) +
           double(a.w) * double(b.w);
  }
};
template <>
struct Vec16<double> {
  using T = double2;
  static constexpr int W = 2;
  __device__ static double dot(const double2& a, const double2& b) { return fma(a.x, b.x, a.y * b.y); }
};

// y = B x with B row-major (leading dimension ld: rows 16-byte aligned); a warp owns R
// consecutive rows, so each 16-byte load of x feeds R rows, and B streams through with
// evict-first loads.  Accumulation in FP64.
template <typename V, int R>
__global__ void __launch_bounds__(kBlock) k_gemv_rows(int nb, size_t ld, const V* __restrict__ B,
                                                      const V* __restrict__ x, double* __restrict__ y) {
  using VT = typename Vec16<V>::T;
  constexpr int W = Vec16<V>::W;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int r0 = warp * R;
  if (r0 >= nb) return;
  const VT* rows[R];
#pragma unroll
  for (int r = 0; r < R; ++r) rows[r] = reinterpret_cast<const VT*>(B + size_t(min(r0 + r, nb - 1)) * ld);
  const VT* xv = reinterpret_cast<const VT*>(x);
  const int nv = nb / W;
  double acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = 0.0;
#pragma unroll(R == 1 ? 8 : 2)
  for (int j = lane; j < nv; j += 32) {
    const VT xx = __ldg(xv + j);
    VT b[R];
#pragma unroll
    for (int r = 0; r < R; ++r) b[r] = __ldcs(rows[r] + j);
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] += Vec16<V>::dot(b[r], xx);
  }
  for (int j = nv * W + lane; j < nb; j += 32) {
    const double xs = double(x[j]);
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = fma(double(reinterpret_cast<const V*>(rows[r])[j]), xs, acc[r]);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    double a = acc[r];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0 && r0 + r < nb) y[r0 + r] = a;
  }
}

// x_pad[pos[i]] = u[bnodes[i]]: boundary values of every component at 32-element aligned offsets.
template <typename V>
__global__ void k_gather_pad(int nb, const double* __restrict__ u, const int* __restrict__ idx,
                             const int* __restrict__ pos, V* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nb) out[pos[i]] = static_cast<V>(u[idx[i]]);
}

// Batched dense matvecs of components with their own matrices (uneven sizes): one warp per
// tile of up to R consecutive rows of one component, the same inner loop as k_gemv_rows.
template <typename V, int R>
__global__ void __launch_bounds__(kBlock) k_gemv_tiles(int ntiles, const GemvTile* __restrict__ tiles,
                                                       const V* __restrict__ B, const V* __restrict__ x,
                                                       double* __restrict__ y) {
  using VT = typename Vec16<V>::T;
  constexpr int W = Vec16<V>::W;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= ntiles) return;
  const GemvTile T = tiles[warp];
  const VT* rows[R];
#pragma unroll
  for (int r = 0; r < R; ++r) rows[r] = reinterpret_cast<const VT*>(B + T.b + size_t(min(r, T.nrows - 1)) * T.ld);
  const V* xs = x + T.x;
  const VT* xv = reinterpret_cast<const VT*>(xs);
  const int nv = T.ncols / W;
  double acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = 0.0;
#pragma unroll 2
  for (int j = lane; j < nv; j += 32) {
    const VT xx = __ldg(xv + j);
    VT b[R];
#pragma unroll
    for (int r = 0; r < R; ++r) b[r] = __ldcs(rows[r] + j);
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] += Vec16<V>::dot(b[r], xx);
  }
  for (int j = nv * W + lane; j < T.ncols; j += 32) {
    const double xsj = double(xs[j]);
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = fma(double(reinterpret_cast<const V*>(rows[r])[j]), xsj, acc[r]);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    double a = acc[r];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0 && r < T.nrows) y[T.y + r] = a;
  }
}

// Replicas sharing one matrix: Y = B X with B (nbc x nbc, row-major, leading dimension ld) and
// X the replicas' boundary values (column c at c * xs).  CTA tile 64 rows x 64 replicas over a
// K range of kchunk columns (split-K partial sums are added atomically into a zeroed Y); thread
// tile 4 x 4; each 32-wide K step is accumulated in the value type, then added into FP64.
template <typename V>
__global__ void __launch_bounds__(256) k_bem_gemm(int nbc, int ncomp, size_t ld, const V* __restrict__ B,
                                                  const V* __restrict__ X, int xs, double* __restrict__ Y,
                                                  int kchunk) {
  constexpr int TM = 64, TN = 64, TK = 32;
  __shared__ __align__(16) V As[TK][TM + 4];
  __shared__ __align__(16) V Xs[TK][TN + 4];
  const int m0 = blockIdx.x * TM, c0 = blockIdx.y * TN;
  const int k0 = blockIdx.z * kchunk, k1 = min(nbc, k0 + kchunk);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (int kb = k0; kb < k1; kb += TK) {
    for (int e = threadIdx.x; e < TM * TK; e += 256) {
      const int r = e / TK, k = e % TK, gr = m0 + r, gk = kb + k;
      As[k][r] = (gr < nbc && gk < k1) ? B[size_t(gr) * ld + gk] : V(0);
    }
    for (int e = threadIdx.x; e < TN * TK; e += 256) {
      const int c = e / TK, k = e % TK, gc = c0 + c, gk = kb + k;
      Xs[k][c] = (gc < ncomp && gk < k1) ? X[size_t(gc) * xs + gk] : V(0);
    }
    __syncthreads();
    V part[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) part[i][j] = V(0);
#pragma unroll 8
    for (int k = 0; k < TK; ++k) {
      V a[4], xv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = As[k][ty * 4 + i];
        xv[i] = Xs[k][tx * 4 + i];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) part[i][j] = fma(a[i], xv[j], part[i][j]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] += double(part[i][j]);
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = m0 + ty * 4 + i, c = c0 + tx * 4 + j;
      if (r < nbc && c < ncomp) {
        if (gridDim.z > 1) atomicAdd(&Y[size_t(c) * nbc + r], acc[i][j]);
        else Y[size_t(c) * nbc + r] = acc[i][j];
      }
    }
}

// Interleaved replicas: X[r * xs + b] = u[bnodes[b] * R + r] (t over nb * R, coalesced reads).
template <typename V>
__global__ void k_gather_rep(int nb, int R, const double* __restrict__ u, const int* __restrict__ idx, int xs,
                             V* __restrict__ X) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nb * R) return;
  const int b = int(t / R), r = int(t - (long long)b * R);
  X[size_t(r) * xs + b] = static_cast<V>(u[size_t(__ldg(idx + b)) * R + r]);
}

// Interleaved replicas: Dirichlet load of state row g = i * R + r from the GEMM output
// Y[r * nb + bindex[i]] (0 inside).
__global__ void k_dirichlet_rep(int n, int R, const int* __restrict__ bindex, const double* __restrict__ Y, int nb,
                                double* __restrict__ b) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long long)n * R) return;
  const int i = int(g / R), r = int(g - (long long)i * R);
  const int k = bindex[i];
  b[g] = (k >= 0) ? Y[size_t(r) * nb + k] : 0.0;
}

__global__ void k_dirichlet_values(int n, const int* __restrict__ bindex, const double* __restrict__ u2b,
                                   double* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = bindex[i];
  b[i] = (k >= 0) ? u2b[k] : 0.0;
}

}  // namespace

size_t bem_ld(int nb) { return (size_t(nb) + 31) / 32 * 32; }

void launch_to_float(const double* src, float* dst, size_t n, cudaStream_t st) {
  note_launch();
  k_to_float<<<grid_for((long long)n), kBlock, 0, st>>>(src, dst, n);
  TMB_CUDA(cudaGetLastError());
}

template <typename V>
void launch_gather(int nb, const double* u, const int* idx, V* out, cudaStream_t st) {
  note_launch();
  k_gather<V><<<grid_for(nb), kBlock, 0, st>>>(nb, u, idx, out);
  TMB_CUDA(cudaGetLastError());
}

template <typename V>
void launch_bem_gemv(int nb, const V* B, const V* xb, double* u2b, cudaStream_t st) {
  note_launch();
  // several rows per warp only when there are enough rows to fill the GPU
  if (nb >= 16384) k_gemv_rows<V, 4><<<grid_for(32LL * ((nb + 3) / 4)), kBlock, 0, st>>>(nb, bem_ld(nb), B, xb, u2b);
  else k_gemv_rows<V, 1><<<grid_for(32LL * nb), kBlock, 0, st>>>(nb, bem_ld(nb), B, xb, u2b);
  TMB_CUDA(cudaGetLastError());
}

template <typename V>
void launch_gather_pad(int nb, const double* u, const int* idx, const int* pos, V* out, cudaStream_t st) {
  note_launch();
  k_gather_pad<V><<<grid_for(nb), kBlock, 0, st>>>(nb, u, idx, pos, out);
  TMB_CUDA(cudaGetLastError());
}

template <typename V>
void launch_bem_gemv_tiles(int ntiles, const GemvTile* tiles, int rows_per_tile, const V* B, const V* x, double* y,
                           cudaStream_t st) {
  if (ntiles == 0) return;
  note_launch();
  if (rows_per_tile == 4) k_gemv_tiles<V, 4><<<grid_for(32LL * ntiles), kBlock, 0, st>>>(ntiles, tiles, B, x, y);
  else k_gemv_tiles<V, 1><<<grid_for(32LL * ntiles), kBlock, 0, st>>>(ntiles, tiles, B, x, y);
  TMB_CUDA(cudaGetLastError());
}

template <typename V>
void launch_bem_gemm(int nbc, int ncomp, const V* B, const V* X, int xs, double* Y, int num_sms, cudaStream_t st) {
  const int mt = (nbc + 63) / 64, ct = (ncomp + 63) / 64;
  // split K until there are about four CTAs per SM
  int split = 1;
  while (split < 16 && mt * ct * split < 4 * num_sms && nbc / (split * 2) >= 256) split *= 2;
  const int kchunk = ((nbc + split - 1) / split + 31) / 32 * 32;
  split = (nbc + kchunk - 1) / kchunk;
  if (split > 1) TMB_CUDA(cudaMemsetAsync(Y, 0, sizeof(double) * size_t(nbc) * ncomp, st));
  note_launch();
  k_bem_gemm<V><<<dim3(mt, ct, split), 256, 0, st>>>(nbc, ncomp, bem_ld(nbc), B, X, xs, Y, kchunk);
  TMB_CUDA(cudaGetLastError());
}

template <typename V>
void launch_gather_rep(int nb, int R, const double* u, const int* idx, int xs, V* X, cudaStream_t st) {
  note_launch();
  k_gather_rep<V><<<grid_for(1LL * nb * R), kBlock, 0, st>>>(nb, R, u, idx, xs, X);
  TMB_CUDA(cudaGetLastError());
}

void launch_dirichlet_rep(int n, int R, const int* bindex, const double* Y, int nb, double* b, cudaStream_t st) {
  note_launch();
  k_dirichlet_rep<<<grid_for(1LL * n * R), kBlock, 0, st>>>(n, R, bindex, Y, nb, b);
  TMB_CUDA(cudaGetLastError());
}

void launch_dirichlet_values(int n, const int* bindex, const double* u2b, double* b, cudaStream_t st) {
  note_launch();
  k_dirichlet_values<<<grid_for(n), kBlock, 0, st>>>(n, bindex, u2b, b);
  TMB_CUDA(cudaGetLastError());
}

template void launch_bem_gemv<double>(int, const double*, const double*, double*, cudaStream_t);
template void launch_bem_gemv<float>(int, const float*, const float*, double*, cudaStream_t);
template void launch_gather<double>(int, const double*, const int*, double*, cudaStream_t);
template void launch_gather_pad<double>(int, const double*, const int*, const int*, double*, cudaStream_t);
template void launch_gather_pad<float>(int, const double*, const int*, const int*, float*, cudaStream_t);
template void launch_bem_gemv_tiles<double>(int, const GemvTile*, int, const double*, const double*, double*,
                                            cudaStream_t);
template void launch_bem_gemv_tiles<float>(int, const GemvTile*, int, const float*, const float*, double*,
                                           cudaStream_t);
template void launch_bem_gemm<double>(int, int, const double*, const double*, int, double*, int, cudaStream_t);
template void launch_bem_gemm<float>(int, int, const float*, const float*, int, double*, int, cudaStream_t);
template void launch_gather<float>(int, const double*, const int*, float*, cudaStream_t);
template void launch_gather_rep<double>(int, int, const double*, const int*, int, double*, cudaStream_t);
template void launch_gather_rep<float>(int, int, const double*, const int*, int, float*, cudaStream_t);

}  // namespace tmb
