// Field kernels: fused local effective field + LLG right-hand side, the
// demag divergence and gradient, normalisation and Runge-Kutta vector ops.
//
// The fused kernel replaces, per right-hand-side evaluation, the chain of
// tetmag's GPU path: three exchange SpMVs (gpu/EffFieldGPU.cu:71-86), the
// uniaxial Thrust passes (:538-560), six tGrad SpMVs + two passes for bulk
// DMI (:150-162, 596-622), the host-side sum of the field terms
// (main/TheLLG.cpp:238-254) and the LLG functor (gpu/EffFieldGPU.cu:316-339,
// 407-430), plus the max-torque reduction (:484-512).  One thread owns one
// node (row); its SELL-32 row is read once for all three components.
#include <atomic>
#include <cmath>

#include "tmb_dev.cuh"

namespace tmb {

namespace {

__device__ __forceinline__ unsigned long long ordered_bits(double v) {
  // Non-negative doubles order like their bit patterns; NaN maps above +inf.
  if (v != v) return 0x7FF8000000000000ull;
  return static_cast<unsigned long long>(__double_as_longlong(v));
}

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = (w != w || w > v) ? w : v;
  }
  return v;
}

template <typename V>
__device__ __forceinline__ double ld(const V* p, int k) {
  return static_cast<double>(__ldg(p + k));
}

// Stored entry k of an operator that may be dictionary-coded (one-byte codes into the FP64 table of
// SellView::tab; the three operators of one kind share the table in sections of 32).
template <typename V>
__device__ __forceinline__ double ldc(const V* p, int k, const double* /*tab*/) {
  return static_cast<double>(__ldg(p + k));
}
template <>
__device__ __forceinline__ double ldc<uint8_t>(const uint8_t* p, int k, const double* tab) {
  return __ldg(tab + __ldg(p + k));
}

// DMI: 0 none, 1 bulk (tetmag), 2 interfacial (no tetmag counterpart; see the epilogue).
template <typename V, bool UNI, int DMI>
__global__ void __launch_bounds__(kBlock) k_local_field(SellView s, const V* __restrict__ K,
                                                        const V* __restrict__ tg0, const V* __restrict__ tg1,
                                                        const V* __restrict__ tg2, const V* __restrict__ gr0,
                                                        const V* __restrict__ gr1, LocalFieldArgs a) {
  if (a.active && *a.active == 0) return;
  const int R = s.rep;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;  // state row (node row of replica r)
  double torque = 0.0;
  if (g < a.n * R) {
    const int nn = a.n;          // operator rows: stride of the per-node arrays
    const int n = nn * R;        // stride of the state components
    const int row = g / R, r = g - row * R;
    const double* __restrict__ mx = a.m;
    const double* __restrict__ my = a.m + n;
    const double* __restrict__ mz = a.m + 2 * n;
    const int sl = row >> 5;
    const int beg = __ldg(s.soff + sl) + (row & 31);
    const int end = __ldg(s.soff + sl + 1);
    double kx = 0.0, ky = 0.0, kz = 0.0;
    double cxy = 0.0, cxz = 0.0, cyx = 0.0, cyz = 0.0, czx = 0.0, czy = 0.0;
#pragma unroll 4
    for (int k = beg; k < end; k += kSlice) {
      const int j = __ldg(s.col + k);
      const int jj = j * R + r;
      const double v = ld(K, k);
      const double ax = __ldg(mx + jj), ay = __ldg(my + jj), az = __ldg(mz + jj);
      kx = fma(v, ax, kx);
      ky = fma(v, ay, ky);
      kz = fma(v, az, kz);
      if (DMI == 1) {
        const double t0 = ld(tg0, k), t1 = ld(tg1, k), t2 = ld(tg2, k);
        cxy = fma(t0, ay, cxy);
        cxz = fma(t0, az, cxz);
        cyx = fma(t1, ax, cyx);
        cyz = fma(t1, az, cyz);
        czx = fma(t2, ax, czx);
        czy = fma(t2, ay, czy);
      }
      if (DMI == 2) {
        // grad_x, grad_y on m (cxz = gx mz, cyz = gy mz, czx = gx mx + gy my) and the transposes
        // through tGrad = (V grad)^T on D m (cxy = tgx D mz, cyx = tgy D mz, czy = tgx D mx + tgy D my)
        const double g0 = ld(gr0, k), g1 = ld(gr1, k), t0 = ld(tg0, k), t1 = ld(tg1, k);
        const double dj = __ldg(a.idm_d + j);
        cxz = fma(g0, az, cxz);
        cyz = fma(g1, az, cyz);
        czx = fma(g0, ax, fma(g1, ay, czx));
        cxy = fma(t0, dj * az, cxy);
        cyx = fma(t1, dj * az, cyx);
        czy = fma(t0, dj * ax, fma(t1, dj * ay, czy));
      }
    }
    const double m0 = mx[g], m1 = my[g], m2 = mz[g];
    const double xc = a.xc[row];
    double H0 = xc * kx, H1 = xc * ky, H2 = xc * kz;
    if (UNI) {
      const double e0 = a.kax[row], e1 = a.kax[row + nn], e2 = a.kax[row + 2 * nn];
      const double f = a.ku2[row] * (e0 * m0 + e1 * m1 + e2 * m2);
      H0 = fma(f, e0, H0);
      H1 = fma(f, e1, H1);
      H2 = fma(f, e2, H2);
    }
    if (a.cub_k1) {
      // cubic anisotropy (EffFieldCalc::cubicAnisotropyField, main/EffFieldCalc.cpp:249-272):
      // alpha = C^T m, dE/dalpha_j = -2 alpha_j (Kc1 (a_j+1^2 + a_j+2^2) + Kc2 a_j+1^2 a_j+2^2), H = C dE
      double c[3][3], al[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
#pragma unroll
        for (int d = 0; d < 3; ++d) c[j][d] = a.cub_ax[(3 * j + d) * nn + row];
        al[j] = c[j][0] * m0 + c[j][1] * m1 + c[j][2] * m2;
      }
      const double k1 = a.cub_k1[row], k2 = a.cub_k2[row];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const double b1 = al[(j + 1) % 3] * al[(j + 1) % 3], b2 = al[(j + 2) % 3] * al[(j + 2) % 3];
        const double de = -2.0 * al[j] * (k1 * (b1 + b2) + k2 * b1 * b2);
        H0 = fma(de, c[j][0], H0);
        H1 = fma(de, c[j][1], H1);
        H2 = fma(de, c[j][2], H2);
      }
    }
    if (a.srf_k) {
      // surface anisotropy (EffFieldCalc::surfaceAnisotropyField, main/EffFieldCalc.cpp:128-149):
      // -2 Ks nm (nm m - n) / V with nm = m . n
      const double q0 = a.nvn[row], q1 = a.nvn[row + nn], q2 = a.nvn[row + 2 * nn];
      const double nm = m0 * q0 + m1 * q1 + m2 * q2, f = -2.0 * a.srf_k[row] * nm;
      H0 = fma(f, nm * m0 - q0, H0);
      H1 = fma(f, nm * m1 - q1, H1);
      H2 = fma(f, nm * m2 - q2, H2);
    }
    if (DMI == 2) {
      // interfacial DMI, E = sum_i V_i D_i [m_z div m - (m . grad) m_z]_i with the nodal gradient
      // operators; H = -(1/V) dE/dm (exact gradient of the discrete energy), divided by Js
      const double da = a.idm_a[row], db = a.idm_b[row];  // D_i / Js_i, 1 / (V_i Js_i)
      H0 += da * cxz - db * cxy;
      H1 += da * cyz - db * cyx;
      H2 += db * czy - da * czx;
    }
    if (DMI == 1) {
      // curl m with tGrad' = -tGrad (main/EffFieldCalc.cpp:43, 280-298)
      const double c0 = -(cyz - czy), c1 = -(czx - cxz), c2 = -(cxy - cyx);
      const double ar = a.area[row];
      const double n0 = a.nvn[row], n1 = a.nvn[row + nn], n2 = a.nvn[row + 2 * nn];
      const double s0 = ar * (m1 * n2 - m2 * n1), s1 = ar * (m2 * n0 - m0 * n2), s2 = ar * (m0 * n1 - m1 * n0);
      const double ds = a.dmi_s[row];
      H0 += ds * (s0 - 2.0 * c0);
      H1 += ds * (s1 - 2.0 * c1);
      H2 += ds * (s2 - 2.0 * c2);
    }
    if (a.hfix) {
      H0 += a.hfix[g];
      H1 += a.hfix[g + n];
      H2 += a.hfix[g + 2 * n];
    }
    if (a.hout) {
      a.hout[g] = H0;
      a.hout[g + n] = H1;
      a.hout[g + 2 * n] = H2;
    }
    const double x0 = m1 * H2 - m2 * H1, x1 = m2 * H0 - m0 * H2, x2 = m0 * H1 - m1 * H0;  // m x H
    torque = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
    if (a.ydot) {
      const double d0 = m1 * x2 - m2 * x1, d1 = m2 * x0 - m0 * x2, d2 = m0 * x1 - m1 * x0;  // m x (m x H)
      const double al = a.alpha;
      if (a.precession) {
        a.ydot[g] = -x0 - al * d0;
        a.ydot[g + n] = -x1 - al * d1;
        a.ydot[g + 2 * n] = -x2 - al * d2;
      } else {
        a.ydot[g] = -al * d0;
        a.ydot[g + n] = -al * d1;
        a.ydot[g + 2 * n] = -al * d2;
      }
    }
  }
  if (a.torque_bits) {
    const double t = warp_max(torque);
    if ((threadIdx.x & 31) == 0) atomicMax(a.torque_bits, ordered_bits(t));
  }
}

template <typename V>
__global__ void __launch_bounds__(kBlock) k_divergence(SellView s, const V* __restrict__ tg0,
                                                       const V* __restrict__ tg1, const V* __restrict__ tg2,
                                                       const double* __restrict__ m, const double* __restrict__ js,
                                                       double inv_mu0, double* __restrict__ rhs) {
  const int R = s.rep;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= s.n * R) return;
  const int n = s.n * R;
  const int row = g / R, r = g - row * R;
  const int sl = row >> 5;
  const int beg = __ldg(s.soff + sl) + (row & 31);
  const int end = __ldg(s.soff + sl + 1);
  double acc = 0.0;
#pragma unroll 4
  for (int k = beg; k < end; k += kSlice) {
    const int j = __ldg(s.col + k);
    const int jj = j * R + r;
    const double J = __ldg(js + j);
    const double t = ldc(tg0, k, s.tab) * __ldg(m + jj) + ldc(tg1, k, s.tab) * __ldg(m + n + jj) +
                     ldc(tg2, k, s.tab) * __ldg(m + 2 * n + jj);
    acc = fma(t, J, acc);
  }
  rhs[g] = acc * inv_mu0;
}

template <typename V>
__global__ void __launch_bounds__(kBlock) k_gradient(SellView s, const V* __restrict__ g0, const V* __restrict__ g1,
                                                     const V* __restrict__ g2, const double* __restrict__ u1,
                                                     const double* __restrict__ u2, const double* __restrict__ hext,
                                                     double* __restrict__ hdem, double* __restrict__ hfix) {
  const int R = s.rep;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= s.n * R) return;
  const int n = s.n * R;
  const int row = g / R, r = g - row * R;
  const int sl = row >> 5;
  const int beg = __ldg(s.soff + sl) + (row & 31);
  const int end = __ldg(s.soff + sl + 1);
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll 4
  for (int k = beg; k < end; k += kSlice) {
    const int j = __ldg(s.col + k) * R + r;
    const double u = u2 ? __ldg(u1 + j) + __ldg(u2 + j) : __ldg(u1 + j);
    a0 = fma(ldc(g0, k, s.tab), u, a0);
    a1 = fma(ldc(g1, k, s.tab), u, a1);
    a2 = fma(ldc(g2, k, s.tab), u, a2);
  }
  if (hdem) {
    hdem[g] = -a0;
    hdem[g + n] = -a1;
    hdem[g + 2 * n] = -a2;
  }
  if (hfix) {
    const double e0 = hext ? hext[g] : 0.0, e1 = hext ? hext[g + n] : 0.0, e2 = hext ? hext[g + 2 * n] : 0.0;
    hfix[g] = e0 - a0;
    hfix[g + n] = e1 - a1;
    hfix[g + 2 * n] = e2 - a2;
  }
}

__global__ void k_normalize(int n, double* m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = m[i], b = m[i + n], c = m[i + 2 * n];
  const double inv = 1.0 / sqrt(a * a + b * b + c * c);
  m[i] = a * inv;
  m[i + n] = b * inv;
  m[i + 2 * n] = c * inv;
}

struct Ptrs7 {
  const double* p[7];
  double c[7];
};

__global__ void k_rk_combine(int n3, const double* __restrict__ y, Ptrs7 k, int nk, double h, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  double acc = 0.0;
  for (int j = 0; j < nk; ++j)
    if (k.c[j] != 0.0) acc = fma(k.c[j], k.p[j][i], acc);
  out[i] = fma(h, acc, y[i]);
}

__global__ void k_rk_error(int n3, const double* __restrict__ y, const double* __restrict__ k1, Ptrs7 k, int nk,
                           double h, double eps_abs, double eps_rel, unsigned long long* err_bits) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double r = 0.0;
  if (i < n3) {
    double acc = 0.0;
    for (int j = 0; j < nk; ++j)
      if (k.c[j] != 0.0) acc = fma(k.c[j], k.p[j][i], acc);
    const double sc = eps_abs + eps_rel * (fabs(y[i]) + h * fabs(k1[i]));
    r = fabs(h * acc) / sc;
  }
  r = warp_max(r);
  if ((threadIdx.x & 31) == 0) atomicMax(err_bits, ordered_bits(r));
}

// --- device-side step control (one attempt of the Dormand-Prince loop per graph segment) -------
__device__ __forceinline__ double bits_value(unsigned long long b) { return __longlong_as_double((long long)b); }

__global__ void k_step_begin(StepCtl* c) {
  if (c->done) {
    c->active = 0;
    return;
  }
  if (++c->attempts > c->max_attempts) {
    c->status = 6;   // TMB_ERR_STEP
    c->done = 1;
    c->active = 0;
    return;
  }
  double h = c->dt;
  int last = 0;
  if (c->t + h >= c->t1) {
    h = c->t1 - c->t;
    last = 1;
  }
  if (!(h > 0.0) || h < 1e-300) {
    c->status = 6;
    c->done = 1;
    c->active = 0;
    return;
  }
  c->h = h;
  c->last = last;
  c->err_bits = 0ull;
  c->active = 1;
}

__global__ void k_rk_combine_dev(int n3, const double* __restrict__ y, Ptrs7 k, int nk, const StepCtl* __restrict__ c,
                                 double* __restrict__ out) {
  if (!c->active) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  double acc = 0.0;
  for (int j = 0; j < nk; ++j)
    if (k.c[j] != 0.0) acc = fma(k.c[j], k.p[j][i], acc);
  out[i] = fma(c->h, acc, y[i]);
}

__global__ void k_rk_error_dev(int n3, const double* __restrict__ y, const double* __restrict__ k1, Ptrs7 k, int nk,
                               StepCtl* c) {
  if (!c->active) return;
  const double h = c->h;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double r = 0.0;
  if (i < n3) {
    double acc = 0.0;
    for (int j = 0; j < nk; ++j)
      if (k.c[j] != 0.0) acc = fma(k.c[j], k.p[j][i], acc);
    const double sc = c->eps_abs + c->eps_rel * (fabs(y[i]) + h * fabs(k1[i]));
    r = fabs(h * acc) / sc;
  }
  r = warp_max(r);
  if ((threadIdx.x & 31) == 0) atomicMax(&c->err_bits, ordered_bits(r));
}

// accepted attempt (finite error <= 1): y <- y5 and, first-same-as-last, k1 <- k7
__global__ void k_step_accept(int n3, const StepCtl* __restrict__ c, double* __restrict__ y,
                              const double* __restrict__ y5, double* __restrict__ k1, const double* __restrict__ k7) {
  if (!c->active) return;
  const double err = bits_value(c->err_bits);
  if (!(err <= 1.0)) return;   // NaN or > 1: rejected
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  y[i] = y5[i];
  k1[i] = k7[i];
}

// step-size control of odeint's controlled stepper (the host loop's arithmetic): reject with
// dt = h max(0.9 err^-1/3, 0.2); accept, and grow dt = 0.9 h max(err, 5^-5)^-1/5 when err < 0.5
__global__ void k_step_update(StepCtl* c, int rhs_per_attempt) {
  if (!c->active) return;
  c->rhs += rhs_per_attempt;
  const double err = bits_value(c->err_bits), h = c->h;
  if (!(err <= 1.0)) {
    const double e = isfinite(err) ? err : 1e30;
    c->dt = h * fmax(0.9 * pow(e, -1.0 / 3.0), 0.2);
    c->rejected += 1;
    return;
  }
  c->accepted += 1;
  const double dtn = (err < 0.5) ? h * 0.9 * pow(fmax(err, pow(5.0, -5.0)), -1.0 / 5.0) : h;
  if (c->last) {
    c->t = c->t1;
    c->dt = (h < c->dt) ? fmax(c->dt, dtn) : dtn;
    c->done = 1;
  } else {
    c->t += h;
    c->dt = dtn;
  }
}

__global__ void k_fill(double* p, double v, size_t n) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

__global__ void k_add(int n, const double* a, const double* b, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + b[i];
}

std::atomic<long long> g_launches{0};

}  // namespace

// Zhang-Li spin-transfer torque added to the right-hand side (TheLLG::sttDynamics,
// main/TheLLG.cpp:201-220; u term TheLLG::calcUtermSTT, :402-415; GPU form gpu/EffFieldGPU.cu:
// 107-148, 434-475): U = sum_d eta_d (grad_d m) per component, ydot += s [-(beta - alpha) m x U
// - (1 + alpha beta) m x (m x U)], s the current pulse value.  R interleaved replicas.
template <typename V>
__global__ void __launch_bounds__(kBlock) k_stt_add(SellView sv, const V* __restrict__ g0, const V* __restrict__ g1,
                                                    const V* __restrict__ g2, const double* __restrict__ m,
                                                    const double* __restrict__ eta, double alpha, double beta,
                                                    double scale, double* __restrict__ ydot,
                                                    const int* __restrict__ active) {
  if (active && *active == 0) return;
  const int R = sv.rep;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= sv.n * R) return;
  const int nn = sv.n, n = nn * R;
  const int row = g / R, r = g - row * R;
  const int sl = row >> 5;
  const int beg = __ldg(sv.soff + sl) + (row & 31);
  const int end = __ldg(sv.soff + sl + 1);
  double d[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};  // d[c][k] = (grad_k m_c)
#pragma unroll 4
  for (int k = beg; k < end; k += kSlice) {
    const int jj = __ldg(sv.col + k) * R + r;
    const double w0 = ld(g0, k), w1 = ld(g1, k), w2 = ld(g2, k);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double mc = __ldg(m + c * n + jj);
      d[c][0] = fma(w0, mc, d[c][0]);
      d[c][1] = fma(w1, mc, d[c][1]);
      d[c][2] = fma(w2, mc, d[c][2]);
    }
  }
  const double ex = eta[row], ey = eta[row + nn], ez = eta[row + 2 * nn];
  double u[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c] = ex * d[c][0] + ey * d[c][1] + ez * d[c][2];
  const double m0 = m[g], m1 = m[g + n], m2 = m[g + 2 * n];
  const double x0 = m1 * u[2] - m2 * u[1], x1 = m2 * u[0] - m0 * u[2], x2 = m0 * u[1] - m1 * u[0];  // m x U
  const double y0 = m1 * x2 - m2 * x1, y1 = m2 * x0 - m0 * x2, y2 = m0 * x1 - m1 * x0;            // m x (m x U)
  const double a = -(beta - alpha) * scale, b = -(1.0 + alpha * beta) * scale;
  ydot[g] += a * x0 + b * y0;
  ydot[g + n] += a * x1 + b * y1;
  ydot[g + 2 * n] += a * x2 + b * y2;
}

template <typename V>
void launch_stt_add(const SellView& s, const V* g0, const V* g1, const V* g2, const double* m, const double* eta,
                    double alpha, double beta, double scale, double* ydot, cudaStream_t st, const int* active) {
  note_launch();
  k_stt_add<V><<<grid_for(1LL * s.n * s.rep), kBlock, 0, st>>>(s, g0, g1, g2, m, eta, alpha, beta, scale, ydot,
                                                                active);
  TMB_CUDA(cudaGetLastError());
}
// Loads the code of every kernel the local right-hand side can launch (both operator types,
// with and without uniaxial anisotropy, each DMI form, the spin-transfer term).  With lazy module
// loading a kernel's code is otherwise loaded, and its device memory taken, at its first launch;
// cudaFuncGetAttributes loads it now.
void preload_local_kernels() {
  cudaFuncAttributes at;
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<double, false, 0>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<double, false, 1>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<double, false, 2>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<double, true, 0>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<double, true, 1>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<double, true, 2>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<float, false, 0>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<float, false, 1>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<float, false, 2>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<float, true, 0>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<float, true, 1>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_local_field<float, true, 2>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_stt_add<double>));
  TMB_CUDA(cudaFuncGetAttributes(&at, k_stt_add<float>));
}

template void launch_stt_add<double>(const SellView&, const double*, const double*, const double*, const double*,
                                     const double*, double, double, double, double*, cudaStream_t, const int*);
template void launch_stt_add<float>(const SellView&, const float*, const float*, const float*, const double*,
                                    const double*, double, double, double, double*, cudaStream_t, const int*);

// Per-block partial sums of the energy terms (TheSimulation::calculateEnergies,
// main/TheSimulation.cpp:385-396), state row g = i * R + r:
//   [0] sum V Js (H_ex . m)      exchange (E = -1/2 of it)
//   [1] sum V Js (H_dmi . m)     DMI      (E = -1/2 of it)
//   [2] sum V Ku (k . m)^2       uniaxial (E = sum V Ku - it)
//   [3] sum V Js (H_ext . m)     Zeeman   (E = -it)
//   [4] sum V Js (H_dem . m)     demag    (E = -1/2 of it)
//   [5] sum V (Kc1 (a0^2 a1^2 + a1^2 a2^2 + a0^2 a2^2) + Kc2 a0^2 a1^2 a2^2), a = C^T m   cubic
//   [6] sum Ks a (n . m)^2       surface  (E = sum Ks a - it)
// Fields here are the library's per-Js fields (A/m); Ku = ku2 Js / 2.
__global__ void __launch_bounds__(kBlock) k_energy_terms(int n, int R, const double* __restrict__ m,
                                                         const double* __restrict__ hex, const double* __restrict__ hdmi,
                                                         const double* __restrict__ hext, const double* __restrict__ hdem,
                                                         const double* __restrict__ js, const double* __restrict__ vol,
                                                         const double* __restrict__ ku2, const double* __restrict__ kax,
                                                         EnergyExtra x, double* __restrict__ part) {
  __shared__ double sh[kEnergyTerms][kBlock / 32];
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = n * R;
  double e[kEnergyTerms] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (g < N) {
    const int i = g / R;
    const double m0 = m[g], m1 = m[g + N], m2 = m[g + 2 * N];
    const double w = vol[i] * js[i];
    auto dot = [&](const double* h) { return h[g] * m0 + h[g + N] * m1 + h[g + 2 * N] * m2; };
    e[0] = w * dot(hex);
    if (hdmi) e[1] = w * dot(hdmi);
    if (ku2) {
      const double km = kax[i] * m0 + kax[i + n] * m1 + kax[i + 2 * n] * m2;
      e[2] = vol[i] * 0.5 * ku2[i] * js[i] * km * km;
    }
    if (hext) e[3] = w * dot(hext);
    if (hdem) e[4] = w * dot(hdem);
    if (x.kc1) {
      double al[3];
#pragma unroll
      for (int j = 0; j < 3; ++j)
        al[j] = x.cax[(3 * j) * n + i] * m0 + x.cax[(3 * j + 1) * n + i] * m1 + x.cax[(3 * j + 2) * n + i] * m2;
      const double s0 = al[0] * al[0], s1 = al[1] * al[1], s2 = al[2] * al[2];
      e[5] = vol[i] * (x.kc1[i] * (s0 * s1 + s1 * s2 + s0 * s2) + x.kc2[i] * s0 * s1 * s2);
    }
    if (x.ksa) {
      const double nm = x.nvn[i] * m0 + x.nvn[i + n] * m1 + x.nvn[i + 2 * n] * m2;
      e[6] = x.ksa[i] * nm * nm;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < kEnergyTerms; ++q) {
    double v = e[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[q][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < kEnergyTerms) {
    double s = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) s += sh[threadIdx.x][w];
    part[size_t(blockIdx.x) * kEnergyTerms + threadIdx.x] = s;
  }
}

int energy_blocks(int n, int R) { return grid_for(1LL * n * R); }

void launch_energy_terms(int n, int R, const double* m, const double* hex, const double* hdmi, const double* hext,
                         const double* hdem, const double* js, const double* vol, const double* ku2, const double* kax,
                         const EnergyExtra& x, double* part, cudaStream_t st) {
  note_launch();
  k_energy_terms<<<grid_for(1LL * n * R), kBlock, 0, st>>>(n, R, m, hex, hdmi, hext, hdem, js, vol, ku2, kax, x,
                                                          part);
  TMB_CUDA(cudaGetLastError());
}

long long launch_count() { return g_launches.load(); }
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void note_launches(long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

template <typename V>
void launch_local_field(const SellView& s, const V* K, const V* tg0, const V* tg1, const V* tg2, const V* gr0,
                        const V* gr1, const LocalFieldArgs& a, cudaStream_t st) {
  note_launch();
  const int g = grid_for(1LL * a.n * s.rep);
  const bool uni = a.ku2 != nullptr;
  const int dmi = a.idm_a ? 2 : (a.dmi_s ? 1 : 0);
#define TMB_LF(U, D) k_local_field<V, U, D><<<g, kBlock, 0, st>>>(s, K, tg0, tg1, tg2, gr0, gr1, a)
  if (uni) {
    if (dmi == 2) TMB_LF(true, 2);
    else if (dmi == 1) TMB_LF(true, 1);
    else TMB_LF(true, 0);
  } else {
    if (dmi == 2) TMB_LF(false, 2);
    else if (dmi == 1) TMB_LF(false, 1);
    else TMB_LF(false, 0);
  }
#undef TMB_LF
  TMB_CUDA(cudaGetLastError());
}

template <typename V>
void launch_divergence(const SellView& s, const V* tg0, const V* tg1, const V* tg2, const double* m,
                       const double* js, double inv_mu0, double* rhs, cudaStream_t st) {
  note_launch();
  k_divergence<V><<<grid_for(1LL * s.n * s.rep), kBlock, 0, st>>>(s, tg0, tg1, tg2, m, js, inv_mu0, rhs);
  TMB_CUDA(cudaGetLastError());
}

template <typename V>
void launch_gradient(const SellView& s, const V* g0, const V* g1, const V* g2, const double* u1,
                     const double* u2, const double* hext, double* hdem, double* hfix, cudaStream_t st) {
  note_launch();
  k_gradient<V><<<grid_for(1LL * s.n * s.rep), kBlock, 0, st>>>(s, g0, g1, g2, u1, u2, hext, hdem, hfix);
  TMB_CUDA(cudaGetLastError());
}

void launch_normalize(int n, double* m, cudaStream_t st) {
  note_launch();
  k_normalize<<<grid_for(n), kBlock, 0, st>>>(n, m);
  TMB_CUDA(cudaGetLastError());
}

void launch_rk_combine(int n3, const double* y, const double* const* k, const double* a, int nk, double h,
                       double* out, cudaStream_t st) {
  note_launch();
  Ptrs7 P{};
  for (int j = 0; j < nk && j < 7; ++j) { P.p[j] = k[j]; P.c[j] = a[j]; }
  k_rk_combine<<<grid_for(n3), kBlock, 0, st>>>(n3, y, P, nk, h, out);
  TMB_CUDA(cudaGetLastError());
}

void launch_rk_error(int n3, const double* y, const double* k1, const double* const* k, const double* e, int nk,
                     double h, double eps_abs, double eps_rel, unsigned long long* err_bits, cudaStream_t st) {
  note_launch();
  Ptrs7 P{};
  for (int j = 0; j < nk && j < 7; ++j) { P.p[j] = k[j]; P.c[j] = e[j]; }
  k_rk_error<<<grid_for(n3), kBlock, 0, st>>>(n3, y, k1, P, nk, h, eps_abs, eps_rel, err_bits);
  TMB_CUDA(cudaGetLastError());
}

void launch_step_begin(StepCtl* c, cudaStream_t st) {
  note_launch();
  k_step_begin<<<1, 1, 0, st>>>(c);
  TMB_CUDA(cudaGetLastError());
}

void launch_rk_combine_dev(int n3, const double* y, const double* const* k, const double* a, int nk,
                           const StepCtl* c, double* out, cudaStream_t st) {
  note_launch();
  Ptrs7 P{};
  for (int j = 0; j < nk && j < 7; ++j) { P.p[j] = k[j]; P.c[j] = a[j]; }
  k_rk_combine_dev<<<grid_for(n3), kBlock, 0, st>>>(n3, y, P, nk, c, out);
  TMB_CUDA(cudaGetLastError());
}

void launch_rk_error_dev(int n3, const double* y, const double* k1, const double* const* k, const double* e, int nk,
                         StepCtl* c, cudaStream_t st) {
  note_launch();
  Ptrs7 P{};
  for (int j = 0; j < nk && j < 7; ++j) { P.p[j] = k[j]; P.c[j] = e[j]; }
  k_rk_error_dev<<<grid_for(n3), kBlock, 0, st>>>(n3, y, k1, P, nk, c);
  TMB_CUDA(cudaGetLastError());
}

void launch_step_accept(int n3, const StepCtl* c, double* y, const double* y5, double* k1, const double* k7,
                        cudaStream_t st) {
  note_launch();
  k_step_accept<<<grid_for(n3), kBlock, 0, st>>>(n3, c, y, y5, k1, k7);
  TMB_CUDA(cudaGetLastError());
}

void launch_step_update(StepCtl* c, int rhs_per_attempt, cudaStream_t st) {
  note_launch();
  k_step_update<<<1, 1, 0, st>>>(c, rhs_per_attempt);
  TMB_CUDA(cudaGetLastError());
}

void launch_fill(double* p, double v, size_t n, cudaStream_t st) {
  note_launch();
  if (n == 0) return;
  k_fill<<<grid_for((long long)n), kBlock, 0, st>>>(p, v, n);
  TMB_CUDA(cudaGetLastError());
}

void launch_add(int n, const double* a, const double* b, double* out, cudaStream_t st) {
  note_launch();
  k_add<<<grid_for(n), kBlock, 0, st>>>(n, a, b, out);
  TMB_CUDA(cudaGetLastError());
}

#define TMB_INST(V)                                                                                         \
  template void launch_local_field<V>(const SellView&, const V*, const V*, const V*, const V*, const V*,   \
                                      const V*, const LocalFieldArgs&, cudaStream_t);                      \
  template void launch_divergence<V>(const SellView&, const V*, const V*, const V*, const double*,         \
                                     const double*, double, double*, cudaStream_t);                        \
  template void launch_gradient<V>(const SellView&, const V*, const V*, const V*, const double*,           \
                                   const double*, const double*, double*, double*, cudaStream_t);
TMB_INST(double)
TMB_INST(float)
#undef TMB_INST
// divergence and gradient on dictionary-coded operators
template void launch_divergence<uint8_t>(const SellView&, const uint8_t*, const uint8_t*, const uint8_t*,
                                         const double*, const double*, double, double*, cudaStream_t);
template void launch_gradient<uint8_t>(const SellView&, const uint8_t*, const uint8_t*, const uint8_t*,
                                       const double*, const double*, const double*, double*, double*,
                                       cudaStream_t);

}  // namespace tmb
