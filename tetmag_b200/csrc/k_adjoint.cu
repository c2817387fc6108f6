// Kernels of the discrete adjoint of the fixed-step LLG integration (no tetmag counterpart:
// tetmag integrates forward only).  What is transposed is tetmag's right-hand side
// (TheLLG::rhs, main/TheLLG.cpp:670-711) with the full effective field (exchange, uniaxial,
// interfacial DMI, applied, demag; main/TheLLG.cpp:238-254).
//
// For f(m) = -m x H - alpha m x (m x H) with H = L m + h(t) (L linear):
//   (df/dm)^T a = a x H - alpha [(m.H) a + (m.a) H - 2 (H.a) m] + L^T mu,
//   mu = (df/dH)^T a = m x a - alpha m x (m x a).
// L^T is applied operator by operator: the exchange row scale moves to the columns
// (K diag(xc) mu), the uniaxial and interfacial-DMI terms are symmetric in the node-volume
// weighted sense (W H(mu / W), W = V Js), and the demag chain runs backwards (see runtime.cu).
#include "tmb_dev.cuh"

namespace tmb {

namespace {

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename V>
__device__ __forceinline__ double ldv(const V* p, int k) {
  return static_cast<double>(__ldg(p + k));
}

}  // namespace

// hext_z = hbase_z + hz (the sampled Bz(t) pulse on top of the static applied field)
__global__ void k_set_hz(int n, const double* __restrict__ hbase, double hz, double* __restrict__ hext) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) hext[2 * n + i] = hbase[2 * n + i] + hz;
}

// out = c0 v0 + c1 v1 + c2 v2 (null vectors are skipped; out may alias an input)
__global__ void k_lincomb(int n3, double* out, double c0, const double* v0, double c1, const double* v1, double c2,
                          const double* v2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  double s = c0 * v0[i];
  if (v1) s = fma(c1, v1[i], s);
  if (v2) s = fma(c2, v2[i], s);
  out[i] = s;
}

// classical RK4 update in place: y <- y + h/6 (k1 + 2 k2 + 2 k3 + k4)
__global__ void k_rk4_final(int n3, double* y, const double* __restrict__ k1, const double* __restrict__ k2,
                            const double* __restrict__ k3, const double* __restrict__ k4, double h) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  const double s = k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i];
  y[i] = fma(h / 6.0, s, y[i]);
}

// y <- y / |y| per node, |y| kept for the adjoint of the normalisation
__global__ void k_normalize_keep(int n, double* __restrict__ y, double* __restrict__ zn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = y[i], b = y[i + n], c = y[i + 2 * n];
  const double r = sqrt(a * a + b * b + c * c);
  const double inv = 1.0 / r;
  y[i] = a * inv;
  y[i + n] = b * inv;
  y[i + 2 * n] = c * inv;
  zn[i] = r;
}

// adjoint of y = z / |z|: lam <- (lam - y (y . lam)) / |z|
__global__ void k_adj_normalize(int n, const double* __restrict__ y, const double* __restrict__ zn,
                                double* __restrict__ lam) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double y0 = y[i], y1 = y[i + n], y2 = y[i + 2 * n];
  const double l0 = lam[i], l1 = lam[i + n], l2 = lam[i + 2 * n];
  const double d = y0 * l0 + y1 * l1 + y2 * l2;
  const double inv = 1.0 / zn[i];
  lam[i] = (l0 - y0 * d) * inv;
  lam[i + n] = (l1 - y1 * d) * inv;
  lam[i + 2 * n] = (l2 - y2 * d) * inv;
}

// Per node: mu = m x a - alpha m x (m x a); g = a x H - alpha [(m.H) a + (m.a) H - 2 (H.a) m]
// (precession = 0 drops the first terms); dku += 2/Js (k.m)(k.mu); one partial sum of mu_z per
// block (the Bz-pulse gradient), reduced on the host in a fixed order.
__global__ void __launch_bounds__(kBlock) k_adj_pre(AdjPreArgs a) {
  __shared__ double wsum[kBlock / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double muz = 0.0;
  if (i < a.n) {
    const int n = a.n;
    const double m0 = a.m[i], m1 = a.m[i + n], m2 = a.m[i + 2 * n];
    const double H0 = a.H[i], H1 = a.H[i + n], H2 = a.H[i + 2 * n];
    const double b0 = a.abar[i], b1 = a.abar[i + n], b2 = a.abar[i + 2 * n];
    const double al = a.alpha;
    const double x0 = m1 * b2 - m2 * b1, x1 = m2 * b0 - m0 * b2, x2 = m0 * b1 - m1 * b0;  // m x a
    const double d0 = m1 * x2 - m2 * x1, d1 = m2 * x0 - m0 * x2, d2 = m0 * x1 - m1 * x0;  // m x (m x a)
    double u0 = -al * d0, u1 = -al * d1, u2 = -al * d2;
    const double mH = m0 * H0 + m1 * H1 + m2 * H2, ma = m0 * b0 + m1 * b1 + m2 * b2;
    const double Ha = H0 * b0 + H1 * b1 + H2 * b2;
    double g0 = -al * (mH * b0 + ma * H0 - 2.0 * Ha * m0);
    double g1 = -al * (mH * b1 + ma * H1 - 2.0 * Ha * m1);
    double g2 = -al * (mH * b2 + ma * H2 - 2.0 * Ha * m2);
    if (a.precession) {
      u0 += x0;
      u1 += x1;
      u2 += x2;
      g0 += b1 * H2 - b2 * H1;
      g1 += b2 * H0 - b0 * H2;
      g2 += b0 * H1 - b1 * H0;
    }
    a.mu[i] = u0;
    a.mu[i + n] = u1;
    a.mu[i + 2 * n] = u2;
    a.g[i] = g0;
    a.g[i + n] = g1;
    a.g[i + 2 * n] = g2;
    muz = u2;
    if (a.dku) {
      const double J = a.js[i];
      const double ij = J != 0.0 ? 1.0 / J : 0.0;
      const double e0 = a.kax[i], e1 = a.kax[i + n], e2 = a.kax[i + 2 * n];
      a.dku[i] += 2.0 * ij * (e0 * m0 + e1 * m1 + e2 * m2) * (e0 * u0 + e1 * u1 + e2 * u2);
    }
  }
  if (a.zpart) {
    muz = warp_sum_d(muz);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = muz;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < kBlock / 32; ++w) s += wsum[w];
      a.zpart[blockIdx.x] = s;
    }
  }
}

// g_i += (K diag(xc) mu)_i + [DMI transpose]_i + ku2_i (k.mu_i) k_i - (Js_i V_i / mu0) q_i
// with q = -grad a1 (the transposed demag chain's last step).  DMI 2 (interfacial): W_i H_idmi(mu / W)_i,
// W = V Js.  DMI 1 (bulk, H = ds (a m x n + 2 C m) with ds = D / (V Js) and the curl
// C m = [ty mz - tz my, tz mx - tx mz, tx my - ty mx] of the tGrad operators t,
// main/EffFieldCalc.cpp:159-170, 280-298): ds_i a_i (n_i x mu_i) + 2 C^T (ds mu), where the
// transposed tGrad rows are read from the gradient operators, t_d^T = diag(V) grad_d (both come
// from the same P1 integrals, tGrad = (V grad)^T).
template <typename V, bool UNI, int DMI>
__global__ void __launch_bounds__(kBlock) k_adj_local(SellView s, const V* __restrict__ K, const V* __restrict__ tg0,
                                                      const V* __restrict__ tg1, const V* __restrict__ gr0,
                                                      const V* __restrict__ gr1, const V* __restrict__ gr2,
                                                      AdjLocalArgs a) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= a.n) return;
  const int n = a.n;
  const double* __restrict__ ux = a.mu;
  const double* __restrict__ uy = a.mu + n;
  const double* __restrict__ uz = a.mu + 2 * n;
  const int sl = row >> 5;
  const int beg = __ldg(s.soff + sl) + (row & 31);
  const int end = __ldg(s.soff + sl + 1);
  double ex = 0.0, ey = 0.0, ez = 0.0;
  double cxz = 0.0, cyz = 0.0, czx = 0.0, cxy = 0.0, cyx = 0.0, czy = 0.0;
#pragma unroll 4
  for (int k = beg; k < end; k += kSlice) {
    const int j = __ldg(s.col + k);
    const double v = ldv(K, k) * __ldg(a.xc + j);
    const double u0 = __ldg(ux + j), u1 = __ldg(uy + j), u2 = __ldg(uz + j);
    ex = fma(v, u0, ex);
    ey = fma(v, u1, ey);
    ez = fma(v, u2, ez);
    if (DMI == 2) {
      const double w = __ldg(a.idm_b + j);  // 1 / (V_j Js_j)
      const double n0 = u0 * w, n1 = u1 * w, n2 = u2 * w;
      const double g0 = ldv(gr0, k), g1 = ldv(gr1, k);
      const double dj = __ldg(a.idm_d + j);
      const double t0 = ldv(tg0, k) * dj, t1 = ldv(tg1, k) * dj;
      cxz = fma(g0, n2, cxz);
      cyz = fma(g1, n2, cyz);
      czx = fma(g0, n0, fma(g1, n1, czx));
      cxy = fma(t0, n2, cxy);
      cyx = fma(t1, n2, cyx);
      czy = fma(t0, n0, fma(t1, n1, czy));
    }
    if (DMI == 1) {
      // c_ab = (grad_a (ds mu_b))_i
      const double d = __ldg(a.dmi_s + j);
      const double v0 = d * u0, v1 = d * u1, v2 = d * u2;
      const double g0 = ldv(gr0, k), g1 = ldv(gr1, k), g2 = ldv(gr2, k);
      cxy = fma(g0, v1, cxy);
      cxz = fma(g0, v2, cxz);
      cyx = fma(g1, v0, cyx);
      cyz = fma(g1, v2, cyz);
      czx = fma(g2, v0, czx);
      czy = fma(g2, v1, czy);
    }
  }
  double o0 = ex, o1 = ey, o2 = ez;
  if (DMI == 2) {
    const double vd = a.vol[row] * a.idm_d[row];
    o0 += vd * cxz - cxy;
    o1 += vd * cyz - cyx;
    o2 += czy - vd * czx;
  }
  if (DMI == 1) {
    const double w = 2.0 * a.vol[row];
    o0 += w * (czy - cyz);
    o1 += w * (cxz - czx);
    o2 += w * (cyx - cxy);
    const double f = a.dmi_s[row] * a.area[row];
    if (f != 0.0) {
      const double n0 = a.nvn[row], n1 = a.nvn[row + n], n2 = a.nvn[row + 2 * n];
      const double u0 = ux[row], u1 = uy[row], u2 = uz[row];
      o0 = fma(f, n1 * u2 - n2 * u1, o0);
      o1 = fma(f, n2 * u0 - n0 * u2, o1);
      o2 = fma(f, n0 * u1 - n1 * u0, o2);
    }
  }
  if (UNI) {
    const double e0 = a.kax[row], e1 = a.kax[row + n], e2 = a.kax[row + 2 * n];
    const double f = a.ku2[row] * (e0 * ux[row] + e1 * uy[row] + e2 * uz[row]);
    o0 = fma(f, e0, o0);
    o1 = fma(f, e1, o1);
    o2 = fma(f, e2, o2);
  }
  if (a.q) {
    const double c = -a.js[row] * a.vol[row] * a.inv_mu0;
    o0 = fma(c, a.q[row], o0);
    o1 = fma(c, a.q[row + n], o1);
    o2 = fma(c, a.q[row + 2 * n], o2);
  }
  a.g[row] += o0;
  a.g[row + n] += o1;
  a.g[row + 2 * n] += o2;
}

// Transposed dense boundary matvec: part[c][j] = sum over rows i of chunk c of B[i][j] x[i]
// (row-major B with leading dimension ld; a warp reads 32 consecutive columns of one row).
template <typename V>
__global__ void __launch_bounds__(kBlock) k_bem_gemv_t(int nb, size_t ld, const V* __restrict__ B,
                                                       const double* __restrict__ x, int rows_per_chunk,
                                                       double* __restrict__ part) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  const int r0 = c * rows_per_chunk;
  const int r1 = min(nb, r0 + rows_per_chunk);
  if (j >= nb) return;
  double acc = 0.0;
#pragma unroll 4
  for (int i = r0; i < r1; ++i) acc = fma(static_cast<double>(__ldcs(B + size_t(i) * ld + j)), __ldg(x + i), acc);
  part[size_t(c) * nb + j] = acc;
}

// out[j] = sum_c part[c][j] in chunk order
__global__ void k_sum_chunks(int nb, int nchunk, const double* __restrict__ part, double* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nb) return;
  double s = 0.0;
  for (int c = 0; c < nchunk; ++c) s += part[size_t(c) * nb + j];
  out[j] = s;
}

// out = c with the constrained entries set to zero
__global__ void k_mask_constrained(int n, const int* __restrict__ cmask, const double* __restrict__ c,
                                   double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = cmask[i] ? 0.0 : c[i];
}

// Transposed constrained solve, last step: out_F = x_F, out_C = c_C - (L^T x)_C
template <typename V>
__global__ void k_lift_t(int n, CsrView lt, const V* __restrict__ lval, const int* __restrict__ cmask,
                         const double* __restrict__ c, const double* __restrict__ x, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!cmask[i]) {
    out[i] = x[i];
    return;
  }
  double acc = c[i];
  for (int k = lt.ptr[i]; k < lt.ptr[i + 1]; ++k) acc -= static_cast<double>(lval[k]) * x[lt.col[k]];
  out[i] = acc;
}

// a[idx[b]] += z[b] (boundary node ids are distinct)
__global__ void k_scatter_add(int nb, const int* __restrict__ idx, const double* __restrict__ z,
                              double* __restrict__ a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nb) a[idx[b]] += z[b];
}

// ---------------------------------------------------------------------------------------------
void launch_set_hz(int n, const double* hbase, double hz, double* hext, cudaStream_t st) {
  note_launch();
  k_set_hz<<<grid_for(n), kBlock, 0, st>>>(n, hbase, hz, hext);
  TMB_CUDA(cudaGetLastError());
}

void launch_lincomb(int n3, double* out, double c0, const double* v0, double c1, const double* v1, double c2,
                    const double* v2, cudaStream_t st) {
  note_launch();
  k_lincomb<<<grid_for(n3), kBlock, 0, st>>>(n3, out, c0, v0, c1, v1, c2, v2);
  TMB_CUDA(cudaGetLastError());
}

void launch_rk4_final(int n3, double* y, const double* k1, const double* k2, const double* k3, const double* k4,
                      double h, cudaStream_t st) {
  note_launch();
  k_rk4_final<<<grid_for(n3), kBlock, 0, st>>>(n3, y, k1, k2, k3, k4, h);
  TMB_CUDA(cudaGetLastError());
}

void launch_normalize_keep(int n, double* y, double* zn, cudaStream_t st) {
  note_launch();
  k_normalize_keep<<<grid_for(n), kBlock, 0, st>>>(n, y, zn);
  TMB_CUDA(cudaGetLastError());
}

void launch_adj_normalize(int n, const double* y, const double* zn, double* lam, cudaStream_t st) {
  note_launch();
  k_adj_normalize<<<grid_for(n), kBlock, 0, st>>>(n, y, zn, lam);
  TMB_CUDA(cudaGetLastError());
}

int adj_pre_blocks(int n) { return grid_for(n); }

void launch_adj_pre(const AdjPreArgs& a, cudaStream_t st) {
  note_launch();
  k_adj_pre<<<grid_for(a.n), kBlock, 0, st>>>(a);
  TMB_CUDA(cudaGetLastError());
}

template <typename V>
void launch_adj_local(const SellView& s, const V* K, const V* tg0, const V* tg1, const V* gr0, const V* gr1, const V* gr2,
                      const AdjLocalArgs& a, cudaStream_t st) {
  note_launch();
  const int g = grid_for(a.n);
  const bool uni = a.ku2 != nullptr;
  const int dmi = a.idm_b ? 2 : (a.dmi_s ? 1 : 0);
#define TMB_ADJ(U, D) k_adj_local<V, U, D><<<g, kBlock, 0, st>>>(s, K, tg0, tg1, gr0, gr1, gr2, a)
  if (uni) {
    if (dmi == 2) TMB_ADJ(true, 2);
    else if (dmi == 1) TMB_ADJ(true, 1);
    else TMB_ADJ(true, 0);
  } else {
    if (dmi == 2) TMB_ADJ(false, 2);
    else if (dmi == 1) TMB_ADJ(false, 1);
    else TMB_ADJ(false, 0);
  }
#undef TMB_ADJ
  TMB_CUDA(cudaGetLastError());
}

int bem_gemv_t_chunks(int nb, int num_sms) {
  const int colblocks = grid_for(nb);
  int c = (4 * num_sms + colblocks - 1) / colblocks;
  c = c < 1 ? 1 : c;
  const int maxc = (nb + 31) / 32;  // at least 32 rows per chunk
  return c > maxc ? (maxc < 1 ? 1 : maxc) : c;
}

template <typename V>
void launch_bem_gemv_t(int nb, const V* B, const double* x, double* part, int nchunk, double* out, cudaStream_t st) {
  if (nb <= 0) return;
  note_launches(2);
  const int rpc = (nb + nchunk - 1) / nchunk;
  dim3 grid(grid_for(nb), nchunk);
  k_bem_gemv_t<V><<<grid, kBlock, 0, st>>>(nb, bem_ld(nb), B, x, rpc, part);
  k_sum_chunks<<<grid_for(nb), kBlock, 0, st>>>(nb, nchunk, part, out);
  TMB_CUDA(cudaGetLastError());
}

void launch_mask_constrained(int n, const int* cmask, const double* c, double* out, cudaStream_t st) {
  note_launch();
  k_mask_constrained<<<grid_for(n), kBlock, 0, st>>>(n, cmask, c, out);
  TMB_CUDA(cudaGetLastError());
}

template <typename V>
void launch_lift_t(int n, const CsrView& lt, const V* lval, const int* cmask, const double* c, const double* x,
                   double* out, cudaStream_t st) {
  note_launch();
  k_lift_t<V><<<grid_for(n), kBlock, 0, st>>>(n, lt, lval, cmask, c, x, out);
  TMB_CUDA(cudaGetLastError());
}

void launch_scatter_add(int nb, const int* idx, const double* z, double* a, cudaStream_t st) {
  if (nb <= 0) return;
  note_launch();
  k_scatter_add<<<grid_for(nb), kBlock, 0, st>>>(nb, idx, z, a);
  TMB_CUDA(cudaGetLastError());
}

#define TMB_INST(V)                                                                                          \
  template void launch_adj_local<V>(const SellView&, const V*, const V*, const V*, const V*, const V*,      \
                                    const V*, const AdjLocalArgs&, cudaStream_t);                           \
  template void launch_bem_gemv_t<V>(int, const V*, const double*, double*, int, double*, cudaStream_t);    \
  template void launch_lift_t<V>(int, const CsrView&, const V*, const int*, const double*, const double*,   \
                                 double*, cudaStream_t);
TMB_INST(double)
TMB_INST(float)
#undef TMB_INST

}  // namespace tmb
