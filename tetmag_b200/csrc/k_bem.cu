// Boundary-element kernels: dense double-layer matrix assembly and the
// boundary matvec of the demag chain.
//
// Assembly follows BEMprocessing::assembleLaplaceBEMmatrix
// (preproc/BEMprocessing.cpp:375-411) with the Lindholm weights of
// Lindholm::weights (preproc/Lindholm.cpp:64-128; D.A. Lindholm, IEEE Trans.
// Magn. 20, 2025 (1984)) and the solid angle of Lindholm::solidAngle
// (:41-61): row n, column m of B sums, over the boundary triangles with vertex
// m that do not contain node n, the weight of vertex m seen from node n; the
// diagonal is Omega_n / (4 pi) - 1.  tetmag assembles it on the host row by
// row (O(Nb * Ntri) weight evaluations); here one CTA owns one row.
//
// The matvec replaces DemagField::boundaryIntegral / denseMVP
// (main/DemagField.cpp:145-147, 184-201), which gathers u1 on the host and
// runs an Eigen GEMV there.
#include <cmath>

#include "tmb_dev.cuh"

namespace tmb {

namespace {

constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

__device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// Solid angle of the triangle (r1, r2, r3 relative to the observer) with norms rn.
__device__ __forceinline__ double solid_angle_rel(const double* r1, const double* r2, const double* r3,
                                                  double r1n, double r2n, double r3n) {
  const double r23 = dot3(r2, r3), r12 = dot3(r1, r2), r31 = dot3(r3, r1);
  const double numer = r1n * r2n * r3n + r1n * r23 + r2n * r31 + r3n * r12;
  const double denom = sqrt(2.0 * (r2n * r3n + r23) * (r3n * r1n + r31) * (r1n * r2n + r12));
  double arg = numer / denom;
  if (fabs(arg - 1.0) < 2.220446049250313e-16 * fabs(arg + 1.0) * 100.0) arg = 1.0;
  return 2.0 * acos(arg);
}

// Lindholm weights of the three vertices p[0..2] seen from x0.
__device__ void lindholm(const double* x0, const double (*p)[3], double area, const double* nv, double* L) {
  double v12[3], v13[3], chi[3];
  for (int d = 0; d < 3; ++d) { v12[d] = p[0][d] - p[1][d]; v13[d] = p[0][d] - p[2][d]; }
  cross3(v12, v13, chi);
  const double cn = sqrt(dot3(chi, chi));
  for (int d = 0; d < 3; ++d) chi[d] /= cn;
  double rv[3][3], xi[3][3], s[3], eta0[3], rho[3];
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) rv[i][d] = p[i][d] - x0[d];
  for (int i = 0; i < 3; ++i) {
    const int i1 = (i + 1) % 3;
    for (int d = 0; d < 3; ++d) xi[i][d] = rv[i1][d] - rv[i][d];
    s[i] = sqrt(dot3(xi[i], xi[i]));
    for (int d = 0; d < 3; ++d) xi[i][d] /= s[i];
    double eta[3];
    cross3(chi, xi[i], eta);
    eta0[i] = dot3(eta, rv[i]);
    rho[i] = sqrt(dot3(rv[i], rv[i]));
  }
  const double chi0 = dot3(chi, rv[0]);
  double P[3];
  for (int i = 0; i < 3; ++i) {
    const double rs = rho[i] + rho[(i + 1) % 3];
    P[i] = log((rs + s[i]) / (rs - s[i]));
  }
  double omega = solid_angle_rel(rv[0], rv[1], rv[2], rho[0], rho[1], rho[2]);
  if (chi0 < 0.0) omega = -omega;
  const double flip = (dot3(nv, chi) < 0.0) ? -1.0 : 1.0;
  const double inv8pa = 1.0 / (8.0 * kPi * area);
  for (int i = 0; i < 3; ++i) {
    const double* xa = xi[(i + 1) % 3];
    const double gP = dot3(xa, xi[0]) * P[0] + dot3(xa, xi[1]) * P[1] + dot3(xa, xi[2]) * P[2];
    L[i] = flip * s[(i + 1) % 3] * inv8pa * (eta0[(i + 1) % 3] * omega - chi0 * gP);
  }
}

// One CTA per row; row accumulated in shared memory (small Nb) or in global memory.
template <bool SHARED_ROW>
__global__ void __launch_bounds__(kBlock) k_bem_assemble(int nb, int ntri, const double* __restrict__ bxyz,
                                                         const int* __restrict__ tri, const double* __restrict__ area,
                                                         const double* __restrict__ nrm,
                                                         const double* __restrict__ solid, double* __restrict__ B,
                                                         size_t ld) {
  extern __shared__ double srow[];
  const int row = blockIdx.x;
  double* out = B + size_t(row) * ld;
  if (SHARED_ROW) {
    for (int j = threadIdx.x; j < nb; j += blockDim.x) srow[j] = 0.0;
    __syncthreads();
  }
  const double x0[3] = {bxyz[3 * row], bxyz[3 * row + 1], bxyz[3 * row + 2]};
  for (int t = threadIdx.x; t < ntri; t += blockDim.x) {
    const int a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
    if (a == row || b == row || c == row) continue;
    double p[3][3];
    for (int d = 0; d < 3; ++d) {
      p[0][d] = bxyz[3 * a + d];
      p[1][d] = bxyz[3 * b + d];
      p[2][d] = bxyz[3 * c + d];
    }
    double L[3];
    lindholm(x0, p, area[t], nrm + 3 * t, L);
    if (SHARED_ROW) {
      atomicAdd(&srow[a], L[0]);
      atomicAdd(&srow[b], L[1]);
      atomicAdd(&srow[c], L[2]);
    } else {
      atomicAdd(&out[a], L[0]);
      atomicAdd(&out[b], L[1]);
      atomicAdd(&out[c], L[2]);
    }
  }
  __syncthreads();
  if (SHARED_ROW) {
    for (int j = threadIdx.x; j < nb; j += blockDim.x) out[j] = srow[j];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[row] = solid[row] / (4.0 * kPi) - 1.0;
}

__global__ void k_to_float(const double* __restrict__ s, float* __restrict__ d, size_t n) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) d[i] = static_cast<float>(s[i]);
}

__global__ void k_gather(int nb, const double* __restrict__ u, const int* __restrict__ idx, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nb) out[i] = u[idx[i]];
}

// y = B x with B row-major (leading dimension ld, 16-byte aligned rows); one warp per row.
template <typename V>
__global__ void __launch_bounds__(kBlock) k_gemv_rows(int nb, size_t ld, const V* __restrict__ B,
                                                      const double* __restrict__ x, double* __restrict__ y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nb) return;
  const V* row = B + size_t(warp) * ld;
  double acc = 0.0;
  if constexpr (sizeof(V) == 4) {
    const float4* r4 = reinterpret_cast<const float4*>(row);
    const int n4 = nb >> 2;
    for (int j = lane; j < n4; j += 32) {
      const float4 b = __ldcs(r4 + j);
      const double* xx = x + 4 * j;
      acc = fma(double(b.x), __ldg(xx), acc);
      acc = fma(double(b.y), __ldg(xx + 1), acc);
      acc = fma(double(b.z), __ldg(xx + 2), acc);
      acc = fma(double(b.w), __ldg(xx + 3), acc);
    }
    for (int j = 4 * n4 + lane; j < nb; j += 32) acc = fma(double(row[j]), __ldg(x + j), acc);
  } else {
    const double2* r2 = reinterpret_cast<const double2*>(row);
    const int n2 = nb >> 1;
    for (int j = lane; j < n2; j += 32) {
      const double2 b = __ldcs(r2 + j);
      acc = fma(b.x, __ldg(x + 2 * j), acc);
      acc = fma(b.y, __ldg(x + 2 * j + 1), acc);
    }
    for (int j = 2 * n2 + lane; j < nb; j += 32) acc = fma(double(row[j]), __ldg(x + j), acc);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) y[warp] = acc;
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

void launch_bem_assemble(int nb, int ntri, const double* bxyz, const int* tri, const double* area,
                         const double* nrm, const double* solid, double* B, cudaStream_t st) {
  note_launch();
  const size_t ld = bem_ld(nb);
  const size_t smem = size_t(nb) * sizeof(double);
  if (smem <= 200 * 1024) {
    TMB_CUDA(cudaFuncSetAttribute(k_bem_assemble<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k_bem_assemble<true><<<nb, kBlock, smem, st>>>(nb, ntri, bxyz, tri, area, nrm, solid, B, ld);
  } else {
    TMB_CUDA(cudaMemsetAsync(B, 0, sizeof(double) * ld * nb, st));
    k_bem_assemble<false><<<nb, kBlock, 0, st>>>(nb, ntri, bxyz, tri, area, nrm, solid, B, ld);
  }
  TMB_CUDA(cudaGetLastError());
}

void launch_to_float(const double* src, float* dst, size_t n, cudaStream_t st) {
  note_launch();
  k_to_float<<<grid_for((long long)n), kBlock, 0, st>>>(src, dst, n);
  TMB_CUDA(cudaGetLastError());
}

void launch_gather(int nb, const double* u, const int* idx, double* out, cudaStream_t st) {
  note_launch();
  k_gather<<<grid_for(nb), kBlock, 0, st>>>(nb, u, idx, out);
  TMB_CUDA(cudaGetLastError());
}

template <typename V>
void launch_bem_gemv(int nb, const V* B, const double* xb, const int* /*unused*/, double* u2b, cudaStream_t st) {
  note_launch();
  k_gemv_rows<V><<<grid_for(32LL * nb), kBlock, 0, st>>>(nb, bem_ld(nb), B, xb, u2b);
  TMB_CUDA(cudaGetLastError());
}

void launch_dirichlet_values(int n, const int* bindex, const double* u2b, double* b, cudaStream_t st) {
  note_launch();
  k_dirichlet_values<<<grid_for(n), kBlock, 0, st>>>(n, bindex, u2b, b);
  TMB_CUDA(cudaGetLastError());
}

template void launch_bem_gemv<double>(int, const double*, const double*, const int*, double*, cudaStream_t);
template void launch_bem_gemv<float>(int, const float*, const double*, const int*, double*, cudaStream_t);

}  // namespace tmb
