// Boundary GEMM of shared-mesh replicas on the 5th-generation tensor cores (mixed path).
//
// Y (FP64, [replica][row]) = B (FP32, nbc x ld row-major) . X (FP32, [replica][xs]): the
// replicas' boundary product of tetmag's demag chain (DemagField::boundaryIntegral /
// denseMVP, main/DemagField.cpp:145-147, 184-201) for all replicas at once.
//
// Precision: 3xTF32.  Each FP32 operand is split into hi = tf32(x) (round to nearest) and
// lo = x - hi (exact in FP32); D += Bhi.Xhi + Bhi.Xlo + Blo.Xhi with FP32 accumulation in tensor
// memory over kGroup 32-wide K stages (128 products), which keeps about 21 mantissa bits of each
// product (the dropped lo.lo term is below 2^-21 relative); the groups are summed in FP64, and
// the partial sums of the K splits are added into Y in FP64.
//
// Structure (one CTA per 128-row tile x 64 replicas x K range; 192 threads):
//   warp 0      TMA producer: cp.async.bulk.tensor 2D tiles of B (128 x 32) and of the
//               pre-split X_hi, X_lo (64 x 32 each), 128-byte swizzle, into a 2- to 4-stage ring;
//               one mbarrier "full" per stage
//   warp 1      MMA issuer (one elected lane): tcgen05.mma.cta_group::1.kind::tf32,
//               M = 128, N = 64, K = 8 per instruction, 12 per stage; groups of kGroup stages
//               alternate between two TMEM accumulator buffers; tcgen05.commit releases the
//               stage ("empty") and marks a group's buffer full ("accf")
//   warps 2..5  split each landed B tile into hi / lo in place ("conv" barrier), drain the
//               previous group's buffer (tcgen05.ld 32x32b, one TMEM lane quarter per warp) into
//               FP64 registers ("acce"), and finally add the sums into Y
// Every wait is bounded: on time-out the thread sets the CTA's abort flag and the error word,
// the other roles see the flag and stop, and the allocating warp still frees its TMEM.
#include <cuda.h>

#include <cstdint>

#include "tmb_dev.cuh"

namespace tmb {

namespace {

constexpr int kTcM = 128, kTcN = 64, kTcK = 32;
constexpr int kTileA = kTcM * kTcK * 4;           // 16 KiB
constexpr int kTileX = kTcN * kTcK * 4;           // 8 KiB
constexpr int kStageBytes = 2 * (kTileA + kTileX);  // hi + lo tiles
constexpr int kGroup = 4;                         // K stages accumulated in FP32 before an FP64 drain
constexpr int kTcThreads = 192;
constexpr unsigned kWaitLimit = 1u << 22;
constexpr uint32_t kTmemCols = 128;  // two 64-column accumulator buffers

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on a barrier phase; false on time-out or when the CTA is aborting.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    if (mbar_try(bar, parity)) return true;
    if (*abort_flag) return false;
  }
  *abort_flag = 1;
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr & 0x3FFFF) >> 4);          // start address
  d |= uint64_t(1) << 16;                          // leading byte offset (unused for swizzled K-major)
  d |= uint64_t(1024 >> 4) << 32;                  // stride byte offset
  d |= uint64_t(1) << 46;                          // descriptor version (Blackwell)
  d |= uint64_t(2) << 61;                          // layout: 128-byte swizzle
  return d;
}

// Instruction descriptor: D F32, A/B TF32, both K-major, M = 128, N = 64.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(kTcN >> 3) << 17) |
                            (uint32_t(kTcM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// In place: x -> hi = tf32(x); lo buffer <- x - hi (same byte positions, so the swizzled layout
// written by TMA carries over).  Used for the B tiles; X is split once per GEMM (k_split_tf32).
__device__ __forceinline__ void split_tile(float4* hi, float4* lo, int nvec, int t, int nt) {
  for (int i = t; i < nvec; i += nt) {
    const float4 v = hi[i];
    float4 h, l;
    h.x = tf32_round(v.x);
    h.y = tf32_round(v.y);
    h.z = tf32_round(v.z);
    h.w = tf32_round(v.w);
    l.x = v.x - h.x;
    l.y = v.y - h.y;
    l.z = v.z - h.z;
    l.w = v.w - h.w;
    hi[i] = h;
    lo[i] = l;
  }
}

template <int kTcStages>
struct TcSmem {
  uint64_t full[kTcStages], conv[kTcStages], empty[kTcStages], accf[2], acce[2];
  uint32_t tmem_base;
  int abort_flag;
};

// 64 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, uint32_t (&v)[kTcN]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,"
      "%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63},"
      " [%64];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31]), "=r"(v[32]),
        "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]),
        "=r"(v[41]), "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]), "=r"(v[48]),
        "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]), "=r"(v[55]), "=r"(v[56]),
        "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace

// Each 32-wide K stage is accumulated by the tensor cores in FP32 into one of two TMEM buffers
// (64 columns each) and drained by the epilogue warps into FP64 registers while the next stage
// runs, so the FP32 part of every sum is 32 products long.
// kTcStages: depth of the TMA ring (2, 3 or 4 stages of 48 KiB), picked with the K split by the
// autotuner (Ctx::tune_gemm_tc).
template <int kTcStages>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_bem_gemm_tc(const __grid_constant__ CUtensorMap mapB, const __grid_constant__ CUtensorMap mapXhi,
                  const __grid_constant__ CUtensorMap mapXlo, int nbc,
                  int ncomp, int kslices_per_cta, int nkslices, double* __restrict__ Y, int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  // tiles need 1024-byte alignment (128-byte swizzle atoms)
  uint8_t* tiles = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  TcSmem<kTcStages>* S = reinterpret_cast<TcSmem<kTcStages>*>(tiles + kTcStages * kStageBytes);
  volatile int* abort_flag = &S->abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kTcM, n0 = blockIdx.y * kTcN;
  const int ks0 = blockIdx.z * kslices_per_cta;
  const int ks1 = min(nkslices, ks0 + kslices_per_cta);
  const int nks = ks1 - ks0;

  auto tileA = [&](int s) { return tiles + s * kStageBytes; };
  auto tileX = [&](int s) { return tiles + s * kStageBytes + kTileA; };
  auto tileAlo = [&](int s) { return tiles + s * kStageBytes + kTileA + kTileX; };
  auto tileXlo = [&](int s) { return tiles + s * kStageBytes + 2 * kTileA + kTileX; };

  if (threadIdx.x == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      mbar_init(&S->full[s], 1);
      mbar_init(&S->conv[s], 4);      // one arrival per converter warp
      mbar_init(&S->empty[s], 1);     // tcgen05.commit
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&S->accf[b], 1);      // tcgen05.commit: stage accumulated
      mbar_init(&S->acce[b], 4);      // one arrival per epilogue warp: buffer drained
    }
    S->abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S->tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S->tmem_base;

  if (nks > 0) {
    if (warp == 0) {
      // ---- TMA producer ----
      if (lane == 0) {
        int issued = 0;
        for (int i = 0; i < nks; ++i) {
          const int s = i % kTcStages;
          if (i >= kTcStages && !mbar_wait(&S->empty[s], ((i / kTcStages) - 1) & 1, abort_flag)) break;
          const int kx = (ks0 + i) * kTcK;
          mbar_expect_tx(&S->full[s], kTileA + 2 * kTileX);
          tma_load_2d(tileA(s), &mapB, kx, m0, &S->full[s]);
          tma_load_2d(tileX(s), &mapXhi, kx, n0, &S->full[s]);
          tma_load_2d(tileXlo(s), &mapXlo, kx, n0, &S->full[s]);
          issued = i + 1;
        }
        // no copy may still be landing when the CTA exits: wait (bounded) for the last load of
        // every stage (their phases complete in order)
        for (int i = (issued > kTcStages ? issued - kTcStages : 0); i < issued; ++i)
          for (unsigned it = 0; it < kWaitLimit; ++it)
            if (mbar_try(&S->full[i % kTcStages], (i / kTcStages) & 1)) break;
      }
    } else if (warp == 1) {
      // ---- MMA issuer ----
      if (lane == 0) {
        for (int i = 0; i < nks; ++i) {
          const int s = i % kTcStages, g = i / kGroup, b = g & 1;
          if (i % kGroup == 0 && g >= 2 && !mbar_wait(&S->acce[b], ((g >> 1) - 1) & 1, abort_flag)) break;
          if (!mbar_wait(&S->conv[s], (i / kTcStages) & 1, abort_flag)) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t d = tmem + uint32_t(b * kTcN);
          const uint32_t a_hi = smem_u32(tileA(s)), x_hi = smem_u32(tileX(s));
          const uint32_t a_lo = smem_u32(tileAlo(s)), x_lo = smem_u32(tileXlo(s));
#pragma unroll
          for (int kk = 0; kk < kTcK / 8; ++kk) {
            const uint32_t off = kk * 32;  // 8 TF32 elements along K inside the 128-byte row
            mma_tf32(d, sw128_desc(a_hi + off), sw128_desc(x_hi + off), (i % kGroup != 0 || kk > 0) ? 1u : 0u);
            mma_tf32(d, sw128_desc(a_hi + off), sw128_desc(x_lo + off), 1u);
            mma_tf32(d, sw128_desc(a_lo + off), sw128_desc(x_hi + off), 1u);
          }
          mma_commit(&S->empty[s]);
          if (i % kGroup == kGroup - 1 || i == nks - 1) mma_commit(&S->accf[b]);
        }
      }
    } else {
      // ---- converters and epilogue (warps 2..5) ----
      const int t = threadIdx.x - 64;
      const int q = warp & 3;  // TMEM lane quarter this warp may access
      double acc[kTcN];
#pragma unroll
      for (int c = 0; c < kTcN; ++c) acc[c] = 0.0;
      bool ok = true;
      auto drain = [&](int g) {
        const int b = g & 1;
        if (!mbar_wait(&S->accf[b], (g >> 1) & 1, abort_flag)) return false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t v[kTcN];
        tmem_ld64(tmem + (uint32_t(q * 32) << 16) + uint32_t(b * kTcN), v);
#pragma unroll
        for (int c = 0; c < kTcN; ++c) acc[c] += double(__uint_as_float(v[c]));
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&S->acce[b]);
        return true;
      };
      for (int i = 0; i < nks && ok; ++i) {
        const int s = i % kTcStages;
        if (!mbar_wait(&S->full[s], (i / kTcStages) & 1, abort_flag)) {
          ok = false;
          break;
        }
        split_tile(reinterpret_cast<float4*>(tileA(s)), reinterpret_cast<float4*>(tileAlo(s)), kTileA / 16, t, 128);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&S->conv[s]);
        // the first stage of a group is converted: drain the group before it while it runs
        if (i % kGroup == 0 && i >= kGroup) ok = drain(i / kGroup - 1);
      }
      if (ok) ok = drain((nks - 1) / kGroup);
      if (ok && !*abort_flag) {
        const int row = m0 + q * 32 + lane;
        if (row < nbc) {
#pragma unroll
          for (int c = 0; c < kTcN; ++c) {
            const int col = n0 + c;
            if (col < ncomp) {
              if (gridDim.z > 1) atomicAdd(&Y[size_t(col) * nbc + row], acc[c]);
              else Y[size_t(col) * nbc + row] = acc[c];
            }
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (*abort_flag && threadIdx.x == 0) atomicExch(err, 1);
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

}  // namespace tmb

// ---------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------
namespace tmb {

// hi = tf32(x) (round to nearest), lo = x - hi, elementwise (the replicas' boundary panel).
__global__ void k_split_tf32(size_t n, const float* __restrict__ x, float* __restrict__ hi, float* __restrict__ lo) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float v = x[i], h = tf32_round(v);
  hi[i] = h;
  lo[i] = v - h;
}

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    TMB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p) throw std::runtime_error("CUDA error: cuTensorMapEncodeTiled unavailable");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 2D FP32 tensor map: rows x cols (cols contiguous, row pitch `pitch` elements), box 32 x box_rows,
// 128-byte swizzle; out-of-range elements read as zero.
CUtensorMap make_map(const float* base, int rows, int cols, size_t pitch, int box_rows) {
  CUtensorMap m;
  const cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(pitch * sizeof(float))};
  const cuuint32_t box[2] = {cuuint32_t(kTcK), cuuint32_t(box_rows)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box,
                                 estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw std::runtime_error("CUDA error: cuTensorMapEncodeTiled failed");
  return m;
}

template <int kTcStages>
constexpr size_t tc_smem_bytes() {
  return size_t(kTcStages) * kStageBytes + sizeof(TcSmem<kTcStages>) + 1024;
}

template <int kTcStages>
void launch_tc_kernel(dim3 grid, cudaStream_t st, const CUtensorMap& mb, const CUtensorMap& mxh,
                      const CUtensorMap& mxl, int nbc, int ncomp, int per, int nks, double* Y, int* err) {
  static bool attr_set = false;
  if (!attr_set) {
    TMB_CUDA(cudaFuncSetAttribute(k_bem_gemm_tc<kTcStages>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(tc_smem_bytes<kTcStages>())));
    attr_set = true;
  }
  k_bem_gemm_tc<kTcStages><<<grid, kTcThreads, tc_smem_bytes<kTcStages>(), st>>>(mb, mxh, mxl, nbc, ncomp, per, nks,
                                                                                  Y, err);
}

}  // namespace

bool bem_gemm_tc_supported(int nbc, size_t ld, int xs) {
  // TMA: 16-byte aligned row pitches; the kernel handles any nbc and replica count
  return nbc > 0 && (ld * sizeof(float)) % 16 == 0 && (size_t(xs) * sizeof(float)) % 16 == 0;
}

void launch_bem_gemm_tc(int nbc, int ncomp, size_t ld, const float* B, const float* X, int xs, float* Xhi,
                        float* Xlo, double* Y, int split, int stages, int* err, cudaStream_t st) {
  const size_t nx = size_t(xs) * ncomp;
  note_launch();
  k_split_tf32<<<grid_for((long long)nx), kBlock, 0, st>>>(nx, X, Xhi, Xlo);
  const CUtensorMap mb = make_map(B, nbc, nbc, ld, kTcM);
  const CUtensorMap mxh = make_map(Xhi, ncomp, nbc, size_t(xs), kTcN);
  const CUtensorMap mxl = make_map(Xlo, ncomp, nbc, size_t(xs), kTcN);
  const int nks = (nbc + kTcK - 1) / kTcK;
  split = split < 1 ? 1 : (split > nks ? nks : split);
  const int per = (nks + split - 1) / split;
  split = (nks + per - 1) / per;
  if (split > 1) TMB_CUDA(cudaMemsetAsync(Y, 0, sizeof(double) * size_t(nbc) * ncomp, st));
  note_launch();
  const dim3 grid((nbc + kTcM - 1) / kTcM, (ncomp + kTcN - 1) / kTcN, split);
  if (stages == 2) launch_tc_kernel<2>(grid, st, mb, mxh, mxl, nbc, ncomp, per, nks, Y, err);
  else if (stages == 3) launch_tc_kernel<3>(grid, st, mb, mxh, mxl, nbc, ncomp, per, nks, Y, err);
  else launch_tc_kernel<4>(grid, st, mb, mxh, mxl, nbc, ncomp, per, nks, Y, err);
  TMB_CUDA(cudaGetLastError());
}

}  // namespace tmb
