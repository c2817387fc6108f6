// Dense double-layer BEM assembly on the device (FP64).
//
// Follows BEMprocessing::assembleLaplaceBEMmatrix (preproc/BEMprocessing.cpp:375-411)
// with the Lindholm weights of Lindholm::weights (preproc/Lindholm.cpp:64-128;
// D.A. Lindholm, IEEE Trans. Magn. 20, 2025 (1984)) and the solid angle of
// Lindholm::solidAngle (:41-61): row n, column m of B sums, over the boundary
// triangles with vertex m that do not contain node n, the weight of vertex m
// seen from node n; the diagonal is Omega_n / (4 pi) - 1.  One CTA owns one row.
//
// This file is compiled with -fmad=false: the solid angle 2 acos(arg) is
// ill-conditioned for small angles (d Omega ~ d arg / sqrt(1 - arg)), so a
// one-ulp change of arg from fused multiply-adds moves far-field entries by
// ~1e-7 relative.  Without contraction the operation order matches the FP64
// restatement used as the test oracle.
#include <cmath>

#include "lindholm_accurate.cuh"
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
  const double den = 8.0 * kPi * area;
  for (int i = 0; i < 3; ++i) {
    const double* xa = xi[(i + 1) % 3];
    const double gP = dot3(xa, xi[0]) * P[0] + dot3(xa, xi[1]) * P[1] + dot3(xa, xi[2]) * P[2];
    L[i] = flip * (s[(i + 1) % 3] / den * (eta0[(i + 1) % 3] * omega - chi0 * gP));
  }
}

// One CTA per row; row accumulated in shared memory (small Nb) or in global memory.  ACCURATE
// selects the far-field-accurate weights of lindholm_accurate.cuh instead of the reference form.
template <bool SHARED_ROW, bool ACCURATE>
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
    if (ACCURATE) lindholm_accurate(x0, p, area[t], nrm + 3 * t, L);
    else lindholm(x0, p, area[t], nrm + 3 * t, L);
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

// Dense tiles of the hierarchical matrix straight from the boundary mesh, with the same
// arithmetic as the dense assembly: entry (i, j) of a tile sums the weight of position j over
// the triangles touching j that do not contain i; the diagonal is Omega / (4 pi) - 1.
__global__ void __launch_bounds__(kBlock) k_h_near_mesh(const HBlockDev* __restrict__ blk, HSource g,
                                                        double* __restrict__ d64, float* __restrict__ d32) {
  const HBlockDev b = blk[blockIdx.x];
  const int mn = b.m * b.n;
  for (int t = threadIdx.x; t < mn; t += blockDim.x) {
    const int i = b.rb + t % b.m, j = b.cb + t / b.m;  // column-major tile
    double v = 0.0;
    if (i == j) {
      v = g.solid[i] / (4.0 * kPi) - 1.0;
    } else {
      const double x0[3] = {g.xp[3 * i], g.xp[3 * i + 1], g.xp[3 * i + 2]};
      for (int k = g.adj_ptr[j]; k < g.adj_ptr[j + 1]; ++k) {
        const int2 a = g.adj[k];
        const int* vt = g.tri + 3 * a.x;
        if (vt[0] == i || vt[1] == i || vt[2] == i) continue;
        double p[3][3];
        for (int q = 0; q < 3; ++q)
          for (int d = 0; d < 3; ++d) p[q][d] = g.xp[3 * vt[q] + d];
        double L[3];
        lindholm(x0, p, g.tarea[a.x], g.tnrm + 3 * a.x, L);
        v += L[a.y];
      }
    }
    d64[b.off + t] = v;
    d32[b.off + t] = static_cast<float>(v);
  }
}

}  // namespace

void launch_h_near_mesh(int nblk, const HBlockDev* blk, const HSource& src, double* d64, float* d32,
                        cudaStream_t st) {
  if (nblk == 0) return;
  note_launch();
  k_h_near_mesh<<<nblk, kBlock, 0, st>>>(blk, src, d64, d32);
  TMB_CUDA(cudaGetLastError());
}

void launch_bem_assemble(int nb, int ntri, const double* bxyz, const int* tri, const double* area,
                         const double* nrm, const double* solid, double* B, bool accurate, cudaStream_t st) {
  note_launch();
  const size_t ld = bem_ld(nb);
  const size_t smem = size_t(nb) * sizeof(double);
  if (smem <= 200 * 1024) {
    auto k = accurate ? k_bem_assemble<true, true> : k_bem_assemble<true, false>;
    TMB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k<<<nb, kBlock, smem, st>>>(nb, ntri, bxyz, tri, area, nrm, solid, B, ld);
  } else {
    TMB_CUDA(cudaMemsetAsync(B, 0, sizeof(double) * ld * nb, st));
    auto k = accurate ? k_bem_assemble<false, true> : k_bem_assemble<false, false>;
    k<<<nb, kBlock, 0, st>>>(nb, ntri, bxyz, tri, area, nrm, solid, B, ld);
  }
  TMB_CUDA(cudaGetLastError());
}

}  // namespace tmb
