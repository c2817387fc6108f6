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

void launch_dirichlet_values(int n, const int* bindex, const double* u2b, double* b, cudaStream_t st) {
  note_launch();
  k_dirichlet_values<<<grid_for(n), kBlock, 0, st>>>(n, bindex, u2b, b);
  TMB_CUDA(cudaGetLastError());
}

template void launch_bem_gemv<double>(int, const double*, const double*, double*, cudaStream_t);
template void launch_bem_gemv<float>(int, const float*, const float*, double*, cudaStream_t);
template void launch_gather<double>(int, const double*, const int*, double*, cudaStream_t);
template void launch_gather<float>(int, const double*, const int*, float*, cudaStream_t);

}  // namespace tmb
