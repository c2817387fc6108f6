// Host runtime of the tetmag B200 library and its C ABI (include/tmb.h).
//
// Mirrors the reference's host classes on the hot path:
//   Solver    <- SolverFactory / AMGCLSolver / GPUSolver (main/SolverFactory.h:42-65,
//                main/AMGCLSolver.cpp:39-113, gpu/GPUSolver.cu:43-97)
//   Ctx::demag <- DemagField::calcField (main/DemagField.cpp:92-240)
//   Ctx::local <- TheLLG::classicVersion / noPrecession + totalEffectiveField
//                (main/TheLLG.cpp:150-199, 238-254)
//   Ctx::relax <- TheSimulation::start outer loop (main/TheSimulation.cpp:231-311)
//                with the Dormand-Prince stepper of TheLLG::IntegrateODEINT
//                (main/TheLLG.cpp:514-572)
// Everything between the caller's input and output stays on the device; the
// host only launches kernels and polls convergence / step-error scalars.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/tmb.h"
#include "tmb_dev.cuh"
#include "tmb_host.h"

namespace tmb {

constexpr double kMu0 = 1.256637061435917295376e-6;   // utils/PhysicalConstants.h:39
constexpr double kGamma0 = 221276.14886372426114160400;  // utils/PhysicalConstants.h:43

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

template <typename T>
struct DevArray {
  T* p = nullptr;
  size_t n = 0;
  DevArray() = default;
  DevArray(const DevArray&) = delete;
  DevArray& operator=(const DevArray&) = delete;
  DevArray(DevArray&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DevArray& operator=(DevArray&& o) noexcept {
    if (this != &o) {
      reset();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevArray() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count == n && p) return;
    reset();
    if (count) TMB_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void upload(const T* h, size_t count, cudaStream_t st) {
    alloc(count);
    if (count) TMB_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
  }
  void upload(const std::vector<T>& v, cudaStream_t st) { upload(v.data(), v.size(), st); }
  void zero(cudaStream_t st) {
    if (n) TMB_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), st));
  }
  void swap(DevArray& o) noexcept {
    std::swap(p, o.p);
    std::swap(n, o.n);
  }
};

// ------------------------------------------------------------------------------------------
// SELL-32 construction
// ------------------------------------------------------------------------------------------
struct SellHost {
  int n = 0, nslice = 0;
  std::vector<int> soff, col;
  std::vector<int64_t> map;  // CSR position -> SELL position
};

static SellHost build_sell(int n, const int* ptr, const int* col) {
  SellHost S;
  S.n = n;
  S.nslice = (n + kSlice - 1) / kSlice;
  S.soff.assign(S.nslice + 1, 0);
  for (int s = 0; s < S.nslice; ++s) {
    int w = 0;
    for (int r = s * kSlice; r < std::min(n, (s + 1) * kSlice); ++r) w = std::max(w, ptr[r + 1] - ptr[r]);
    const int64_t next = int64_t(S.soff[s]) + int64_t(kSlice) * w;
    if (next > 0x7fffffffLL) throw Error(TMB_ERR_ARG, "operator too large for int32 SELL offsets");
    S.soff[s + 1] = int(next);
  }
  S.col.assign(S.soff[S.nslice], 0);
  S.map.assign(ptr[n], 0);
  for (int s = 0; s < S.nslice; ++s) {
    const int w = (S.soff[s + 1] - S.soff[s]) / kSlice;
    for (int lane = 0; lane < kSlice; ++lane) {
      const int r = s * kSlice + lane;
      const int len = (r < n) ? ptr[r + 1] - ptr[r] : 0;
      const int pad = (r < n) ? r : n - 1;
      for (int k = 0; k < w; ++k) {
        const int pos = S.soff[s] + k * kSlice + lane;
        if (k < len) {
          S.col[pos] = col[ptr[r] + k];
          S.map[ptr[r] + k] = pos;
        } else {
          S.col[pos] = pad;
        }
      }
    }
  }
  return S;
}

template <typename V>
static std::vector<V> sell_values(const SellHost& S, const double* v) {
  std::vector<V> out(S.col.size(), V(0));
  for (size_t k = 0; k < S.map.size(); ++k) out[S.map[k]] = static_cast<V>(v[k]);
  return out;
}

struct DevSell {
  int n = 0, nslice = 0;
  DevArray<int> soff, col;
  SellView view(int rep = 1) const { return SellView{n, nslice, soff.p, col.p, rep}; }
  void upload(const SellHost& S, cudaStream_t st) {
    n = S.n;
    nslice = S.nslice;
    soff.upload(S.soff, st);
    col.upload(S.col, st);
  }
};

struct DevCsr {
  int n = 0;
  DevArray<int> ptr, col;
  DevArray<double> v;
  DevArray<float> vf;
  CsrView view(int rep = 1) const { return CsrView{n, ptr.p, col.p, rep}; }
  void upload(const Csr& A, cudaStream_t st) {
    n = A.nrows;
    ptr.upload(A.ptr, st);
    col.upload(A.col, st);
    v.upload(A.val, st);
    std::vector<float> f(A.val.begin(), A.val.end());
    vf.upload(f, st);
  }
};

struct Ctx;

// ------------------------------------------------------------------------------------------
// Live kernel profiler: CUDA events around the main kernels on the launching stream.
// ids: 0 local field + LLG, 1 divergence, 2 gradient, 3 BEM matvec, 4 Neumann solve,
//      5 Dirichlet solve, 6 CG fine-level SpMV, 7 whole demag chain (4, 5, 7 are containers),
//      8 fused CG update + first fine smoothing sweep, 9 fine post-smoothing sweep + r.z,
//      10 fine pre-smoothing sweep (unfused), 11 restriction (every level), 12 prolongation
//      (every level), 13 coarse-level smoothing sweeps, 14 coarsest dense solve, 15 CG start
//      (lift, initial residual), 16 CG vector update (unfused)
// ------------------------------------------------------------------------------------------
constexpr int kProfIds = 17;
struct Prof {
  bool on = false;
  struct Rec {
    int id;
    cudaEvent_t a, b;
    double bytes;
  };
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  std::vector<Rec> recs;
  double count[kProfIds] = {}, ms[kProfIds] = {}, bytes[kProfIds] = {};
  ~Prof() {
    for (auto e : pool) cudaEventDestroy(e);
  }
  cudaEvent_t get() {
    if (used == pool.size()) {
      cudaEvent_t e;
      TMB_CUDA(cudaEventCreate(&e));
      pool.push_back(e);
    }
    return pool[used++];
  }
  std::vector<size_t> open;  // indices of records whose end is pending (nesting allowed)
  void begin(int id, cudaStream_t st, double b) {
    if (!on) return;
    Rec r{id, get(), get(), b};
    TMB_CUDA(cudaEventRecord(r.a, st));
    open.push_back(recs.size());
    recs.push_back(r);
  }
  void end(cudaStream_t st) {
    if (!on || open.empty()) return;
    TMB_CUDA(cudaEventRecord(recs[open.back()].b, st));
    open.pop_back();
    if (open.empty() && used > 4000) flush();
  }
  void flush() {
    if (!open.empty()) return;
    for (const Rec& r : recs) {
      TMB_CUDA(cudaEventSynchronize(r.b));
      float t = 0.f;
      TMB_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
      count[r.id] += 1;
      ms[r.id] += t;
      bytes[r.id] += r.bytes;
    }
    recs.clear();
    used = 0;
  }
  void reset() {
    open.clear();
    recs.clear();
    used = 0;
    for (int i = 0; i < kProfIds; ++i) count[i] = ms[i] = bytes[i] = 0.0;
  }
};

// ------------------------------------------------------------------------------------------
// Solver: PCG + smoothed-aggregation V-cycle for row-constrained SPD systems
// ------------------------------------------------------------------------------------------
// The mixed path keeps the CG's own operator (the lift of the constrained columns, the start
// residual and the product A p) in FP64 and only the preconditioner (every V-cycle level and
// transfer) in FP32.  A CG on FP32 operator values converges to the solution of the rounded system,
// which differs from the FP64 one by up to the condition number times the FP32 rounding (about 1e-5
// of the field on the small dots of the batched workload); with the FP64 operator the solution
// matches the FP64 path to the CG tolerance and the FP32 preconditioner only changes the iteration
// count.
constexpr bool kCgOperatorF64 = true;

// A finest-level operator with at most this many distinct values (0.0 included) stores them as
// one-byte codes into an FP64 table.
constexpr int kDictMax = 32;

struct DevLevel {
  int n = 0;
  DevSell A;                 // fine level: SELL-32, one thread per row (about 14 entries per row)
  // fine level, dictionary-coded values: the stiffness matrix of a Kuhn-split cuboid has about a
  // dozen distinct entries, so one-byte codes into an FP64 table give exact FP64 values at a
  // quarter of FP32's bytes (both precision paths then read the same exact operator)
  bool dict = false;
  DevArray<uint8_t> Aq;
  DevArray<double> Atab;
  SellView fine_view(int rep) const {
    SellView v = A.view(rep);
    v.tab = dict ? Atab.p : nullptr;
    return v;
  }
  double fine_value_bytes(bool f64) const { return dict ? 1.0 : (f64 ? 8.0 : 4.0); }
  DevCsr Ac;                 // coarser levels: CSR, tA threads per row (Galerkin rows of 20-60 entries)
  int tA = 1, tP = 1, tR = 1;
  DevArray<double> Ad, dinv, X, R, b, out;
  DevArray<float> Af;
  DevCsr P, Rop;
  // coarse levels with one replica: A P (values) with P's values on its pattern, for the fused
  // prolongation + post-smoothing sweep
  bool fused_post = false;
  DevCsr AP;
  DevArray<double> pv;
  DevArray<float> pvf;
  int tAP = 1;
  // coarse levels with one replica: M = R - (R A) D_w^-1, the restriction of the first sweep's
  // residual straight from the level's right-hand side (merged with that sweep's launch)
  bool fused_pre = false;
  DevCsr M;
  int tM = 1;
};

// P's values on the pattern of M = A P (which holds P's pattern when A has its diagonal); false if
// an entry of P has no place in M.
static bool values_on_pattern(const Csr& M, const Csr& P, std::vector<double>& out) {
  out.assign(size_t(M.nnz()), 0.0);
  for (int i = 0; i < P.nrows; ++i) {
    int k = M.ptr[i];
    for (int q = P.ptr[i]; q < P.ptr[i + 1]; ++q) {
      while (k < M.ptr[i + 1] && M.col[k] < P.col[q]) ++k;
      if (k == M.ptr[i + 1] || M.col[k] != P.col[q]) return false;
      out[size_t(k)] = P.val[q];
    }
  }
  return true;
}

struct Solver {
  Ctx* ctx;
  Csr A;                      // as given (rows may be constraints)
  double tol = 1e-7;
  int maxit = 100;
  int check_every = 2;
  bool computed = false;
  int n = 0;
  int rep = 1;                // interleaved replicas: every vector holds n * rep entries
  int want_rep = -1;          // >= 1: fixed by the owner (the solver plugin); else the context's
  AmgParams prm;
  AmgHierarchy H;
  std::vector<DevLevel> lev;
  DevArray<double> cinv;
  DevArray<float> cinvf;
  int ncoarse = 0, cld = 0, cldf = 0;
  // coarsest level with decoupled rows (AmgHierarchy::coarse_idx): its coupled rows, the exact
  // inverse diagonal of every row, and compact vectors for the dense solve of the coupled rows
  bool csubset = false;
  DevArray<int> cidx;
  DevArray<double> cdiag, cb, cx;
  DevCsr lift;
  DevArray<int> cmask;
  // transposed solve (the adjoint): lift^T, masked load, and a warm start kept apart from the
  // forward one
  DevCsr liftT;
  static constexpr int kAdjSlots = 4;   // one warm start per RK stage
  DevArray<double> ct, xfwd, xadj[kAdjSlots];
  bool has_xadj[kAdjSlots] = {false, false, false, false};
  DevArray<double> x, rbuf[2], z, p, q, bp, partials;
  CgScalars* Sd = nullptr;
  CgScalars* Sh = nullptr;
  int last_iters = 0, last_status = 0;
  double last_relres = 0.0;
  bool has_x = false;

  explicit Solver(Ctx* c) : ctx(c) {}
  ~Solver() {
    drop_graphs();
    if (Sd) cudaFree(Sd);
    if (Sh) cudaFreeHost(Sh);
  }
  void set_matrix(int nn, const int* ptr, const int* col, const double* val) {
    A.nrows = A.ncols = nn;
    A.ptr.assign(ptr, ptr + nn + 1);
    A.col.assign(col, col + ptr[nn]);
    A.val.assign(val, val + ptr[nn]);
    computed = false;
  }
  void compute();
  void solve(const double* b_dev, int precision);
  // out = A^-T c for the row-replaced matrix A = [A_FF L; 0 I] (constrained rows C are unit
  // rows): out_F = A_FF^-1 c_F (A_FF is symmetric), out_C = c_C - (L^T out_F)_C
  // slot: which of kAdjSlots warm-start vectors to use (the adjoint keeps one per RK stage, since
  // the same stage's load changes little from one substep to the next)
  void solve_t(const double* c_dev, double* out, int precision, int slot = 0);
  // presmoothed: the finest level's first sweep (X, R) was already done by the fused CG update
  void vcycle(size_t l, const double* b, double* out, int precision, cudaStream_t st, int rz_mode,
              bool presmoothed = false);
  void precondition_rz(int precision, cudaStream_t st, bool first);
  int rc = 0;  // which of rbuf[0], rbuf[1] holds the current residual
  double nnz_fine = 0.0;

  void ctx_prof_begin(int id, cudaStream_t st, double bytes);
  void ctx_prof_end(cudaStream_t st);
  bool ctx_prof_on() const;
  // one PCG iteration: direction update, A p with p.Ap, x/r update with r.r, V-cycle, r.z
  void iteration_body(int precision, cudaStream_t st, bool profile);
  // CUDA graph of kGraphIters iteration bodies per precision, captured on first use.  Each fused
  // iteration swaps the two residual buffers and every graph is captured starting from rbuf[0], so
  // a graph must hold an even count (an odd one makes the next launch read the wrong residual).
  // 2 measured faster than 4.
  static constexpr int kGraphIters = 2;
  static_assert(kGraphIters % 2 == 0, "CG graphs must end on the residual buffer they start from");
  cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
  long long graph_nodes[2] = {0, 0};
  cudaGraphExec_t graph_for(int precision);
  // the start of a solve: lift, first residual, first V-cycle with r.z
  void solve_start(const double* b_dev, int precision, cudaStream_t st);
  void drop_graphs() {
    for (auto& g : graph_exec)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }
};

// ------------------------------------------------------------------------------------------
// Context
// ------------------------------------------------------------------------------------------
struct Ctx {
  int device = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  int precision = TMB_FP64;
  int n = 0, nb = 0;
  // Interleaved replicas of one mesh (tmb_set_replicas): every state vector holds rep copies,
  // node i of replica r at i * rep + r; operators, material and the BEM matrix are stored once.
  int rep = 1;
  int nr() const { return n * rep; }
  void set_replicas(int R);
  // operators
  DevSell pat;
  DevArray<double> K, g[3], tg[3];
  DevArray<float> Kf, gf[3], tgf[3];
  // K alone on its non-zero entries (and the diagonal), for local fields without DMI: on Kuhn-split
  // cuboids half of the shared pattern holds exact zeros of K (the face-diagonal couplings).  Built
  // only when it drops at least a tenth of the entries; otherwise the shared pattern serves.
  // grad and tGrad dictionary-coded (each of the three operators of a kind has at most 32 distinct
  // values on a Kuhn-split cuboid): one-byte codes into a shared FP64 table, section 32 d for
  // operator d; exact FP64 values for the divergence and gradient of both paths
  bool g_coded = false, tg_coded = false;
  DevArray<uint8_t> gq[3], tgq[3];
  DevArray<double> gtab, tgtab;
  void launch_div(const double* m, const double* js_, double scale, double* out, cudaStream_t st);
  void launch_grad(const double* u1, const double* u2, const double* he, double* hd, double* hf, cudaStream_t st);
  bool has_patx = false;
  long long nnz_x = 0;
  DevSell patx;
  DevArray<double> Kx;
  DevArray<float> Kxf;
  void launch_local_kernel(const LocalFieldArgs& a, cudaStream_t st);
  std::vector<int> hptr, hcol, hbnodes;
  std::vector<double> hK, hvol;
  DevArray<double> node_vol, area, nvn;
  DevArray<int> bnodes, bindex;
  // material
  bool has_material = false, has_uni = false, has_dmi = false;
  double alpha = 1.0, gamma = kGamma0;
  int precession = 1;
  DevArray<double> js, xc, ku2, kax, dmi_s, hext, hdem, hfix;
  // DMI form: 0 bulk (tetmag), 1 interfacial (no tetmag counterpart)
  int dmi_kind = 0;
  DevArray<double> idm_d, idm_a, idm_b;
  std::vector<double> hD, hij;          // D and 1/Js per node, kept to switch the DMI form
  void upload_dmi();
  // cubic and surface anisotropy (EffFieldCalc.cpp:128-149, 249-272): raw per-node constants on the
  // host, device copies scaled by 1/Js (fields) and raw (energies)
  std::vector<double> hKc1, hKc2, hcax, hKs, harea;
  DevArray<double> cub_k1, cub_k2, cub_ax, srf_k, kc1_raw, kc2_raw, ksa_raw;
  bool has_cub = false, has_srf = false;
  void upload_extra();
  // Zhang-Li spin-transfer torque (TheLLG::sttDynamics, main/TheLLG.cpp:201-220)
  bool has_stt = false;
  double stt_beta = 0.0, stt_scale = 1.0;
  DevArray<double> stt_eta;
  LocalFieldArgs local_args(const double* m, double* ydot, double* hout, unsigned long long* tq) const;
  void launch_local(const LocalFieldArgs& a, cudaStream_t st);
  // BEM
  DevArray<double> Bd;
  DevArray<float> Bf;
  bool has_bem = false;
  // Disjoint components (batched instances): nodes [coff[c], coff[c+1]), boundary indices
  // [cboff[c], cboff[c+1]).  Each component has its own BEM block in Bd / Bf (row-major,
  // leading dimension bem_ld(nb_c)); with shared_bem the components are replicas of one mesh and
  // share one block, and the boundary matvec is one GEMM over the replicas.
  std::vector<int> coff, cboff;
  bool shared_bem = false;
  int num_sms = 148;
  DevArray<int> xpos;                   // boundary index -> padded position of its component
  DevArray<double> xpad64;
  DevArray<float> xpad32, xhi32, xlo32;
  int xstride = 0;                      // shared: padded length of one replica's boundary
  // tensor-core (3xTF32) boundary GEMM of the mixed path: on by default, split-K picked by
  // tune_gemm_tc on first use; tc_err is the kernel's time-out word
  bool gemm_tc = true;
  int tc_split = 0, tc_stages = 4;
  DevArray<int> tc_err;
  std::vector<double> tc_tune_ms;       // per candidate split 1..8 (0: not tried)
  void tune_gemm_tc();
  void bem_gemm(bool f64, cudaStream_t st);
  DevArray<GemvTile> tiles;
  int ntiles = 0, tile_rows = 1;
  double bem_entries = 0.0;             // matrix entries streamed by one boundary matvec
  int ncomp() const { return int(coff.size()) - 1; }
  void set_components(int nc, const int* off, bool shared);
  void plan_components();
  // hierarchical BEM (tmb_bem_compress)
  struct HMat {
    bool built = false;
    int nnear = 0, nfar = 0, nrows = 0, ngroups[2] = {0, 0}, failed = 0;
    long long terms[2] = {0, 0};          // [0] FP64 (tight), [1] FP32 (loose)
    double bytes[2] = {0, 0}, ms = 0.0;
    int max_rank = 0;
    DevArray<int> gidx, pos, perm;
    std::vector<int> ranks;               // per low-rank block: tight rank, loose rank, status
    DevArray<HBlockDev> nearb, farb;
    DevArray<HNearRow> rows;
    DevArray<HFarGroup> groups[2];        // per precision, largest work first
    DevArray<double> D64, U64, V64, y, xp64;
    DevArray<float> D32, U32, V32, xp32;
    DevArray<int> rank[2];
    DevArray<long long> uoff[2], voff[2], toff[2];
    DevArray<HTerm> termd[2];             // per-term descriptors of the far-field product
    DevArray<double> tval;                // the terms' values, one matvec at a time
    // the transposed product (the adjoint's B^T), built on first use: blocks ordered by column
    std::vector<HBlockDev> hnearb, hfarb;
    bool tbuilt = false;
    int ntcols = 0, ntgroups[2] = {0, 0};
    DevArray<HBlockDev> tnearb;
    DevArray<HNearRow> tcols;
    DevArray<HFarGroup> tgroups[2];
    DevArray<long long> ttoff[2];
    DevArray<HTerm> ttermd[2];
    DevArray<double> ty;
    // the partition and the FP64 factors' offsets and ranks (host), for the H2 recompression
    HPartition part;
    std::vector<long long> huoff, hvoff;
    std::vector<int> hrank;
    long long hsu = 0, hsv = 0;
    // boundary geometry in cluster order when the matrix was built from the mesh
    bool from_mesh = false;
    int ntri = 0;
    DevArray<double> gx, garea, gnrm, gsolid;
    DevArray<int> gtri, gadj_ptr;
    DevArray<int2> gadj;
  } H;
  // H2 matrix: nested cluster bases recompressed from H's admissible blocks (h2.cpp); one per
  // precision ([0] FP64 for the plain path, [1] FP32 for the mixed path); the near field is H's
  struct H2Mat {
    bool built = false;
    int nleaf = 0, nruns = 0, nlevels = 0, max_kr = 0, max_kc = 0;
    long long ncoef_r = 0, ncoef_c = 0;
    double bytes = 0.0, coupling_bytes = 0.0, basis_bytes = 0.0, ms = 0.0, eps = 0.0;
    DevArray<H2Node> node;
    DevArray<int> leaves, lvl_nodes;
    DevArray<H2Run> runs;
    DevArray<H2Blk> blk;
    DevArray<int> brow;
    DevArray<double> xh, yh;
    DevArray<double> rowb64, colb64, S64;
    DevArray<float> rowb32, colb32, S32;
    std::vector<std::pair<int, int>> up, down;
  } H2[2];
  void h2_build(double eps_fp64, double eps_mixed, int kmax);
  template <typename T>
  H2View<T> h2_view(int which) const;
  HSource h_source() const;
  int bem_mode = 0;  // 0 dense, 1 hierarchical, 2 H2
  // matrix-relative accuracy of the next compression (tmb_set_bem_accuracy): 0 block-relative only
  double h_share = 0.0;
  double h_gscale = 0.0;  // the entry scale the last compression used
  void h_compress(const double* bxyz, const double* bnrm, int leaf, double eta, double eps_mixed, double eps_fp64,
                  int kmax, bool keep_dense, const MeshHost* mesh = nullptr);
  void h_verify(double* block_out, double* out);
  // the boundary product alone (DemagField::mvp), boundary vectors in boundary-node order
  void bem_apply(const double* xb, double* yb, bool transpose);
  DevArray<double> bap_u, bap_w, bap_part;
  DevArray<float> bap_f;
  template <typename T>
  HMatView<T> h_view(int which) const;
  void h_transpose_build();
  template <typename T>
  HMatView<T> ht_view(int which) const;
  // demag
  std::unique_ptr<Solver> neu, dir;
  double tol = 1e-7;
  int maxit = 100;
  DevArray<double> rhs, u1, u2, u1b, u2b, bdir;
  DevArray<float> u1bf;
  // integrator / scratch
  DevArray<double> ybuf[2], kst[7], ytmp, in3, out3;
  DevArray<unsigned long long> bits;
  unsigned long long* bits_h = nullptr;
  Prof prof;

  explicit Ctx(int dev) : device(dev) {
    TMB_CUDA(cudaSetDevice(dev));
    TMB_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
    stream = own;
    TMB_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    TMB_CUDA(cudaMallocHost(&bits_h, 4 * sizeof(unsigned long long)));
    std::memset(bits_h, 0, 4 * sizeof(unsigned long long));
    bits.alloc(4);
  }
  ~Ctx() {
    drop_step_graphs();
    if (ctl_d) cudaFree(ctl_d);
    if (ctl_h) cudaFreeHost(ctl_h);
    neu.reset();
    dir.reset();
    if (bits_h) cudaFreeHost(bits_h);
    if (own) cudaStreamDestroy(own);
  }
  void require_mesh() const {
    if (n == 0) throw Error(TMB_ERR_STATE, "no mesh operators set");
  }
  void require_material() const {
    if (!has_material) throw Error(TMB_ERR_STATE, "no material set");
  }

  void set_operators(int nx, const int* ptr, const int* col, const double* K_, const double* const* g_,
                     const double* const* tg_, const double* vol, int nb_, const int* bn, const double* area_,
                     const double* nvn_soa);
  void set_material(const double* Js, const double* A, const double* Ku, const double* axis, const double* D,
                    double alpha_);
  void set_bem_rowmajor(const double* Brow_dev_or_null);
  void ensure_demag();
  void demag(const double* m_dev);
  void local(const double* m, double* ydot, double* hout, unsigned long long* torque_bits);
  double max_torque(const double* m_dev);
  void energies(const double* m_dev, double* out8);
  DevArray<double> ebuf[2], epart;
  int integrate_segment(double*& y, double*& yalt, double t0, double t1, double& dt, double eps_abs,
                        double eps_rel, double* stats);
  // the same loop with the step control on the device: kStepAttempts attempts per CUDA graph
  // launch, the host polls the control block once per launch instead of once per step
  static constexpr int kStepAttempts = 8;
  StepCtl* ctl_d = nullptr;
  StepCtl* ctl_h = nullptr;
  cudaGraphExec_t step_graph[2] = {nullptr, nullptr};
  std::vector<unsigned char> step_sig[2];
  bool device_steps = true;
  long long step_nodes = 0;
  void integrate_segment_dev(double* y, double* yalt, double t0, double t1, double& dt, double eps_abs,
                             double eps_rel, double* stats);
  cudaGraphExec_t step_graph_for(double* y, double* yalt);
  void drop_step_graphs() {
    for (auto& g : step_graph)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }
  int relax(double* m_dev, double duration_ps, double segment_ps, double eps_abs, double eps_rel, double* stats);
  // Fixed-step integration with the full field at every stage, and its discrete adjoint.
  std::vector<double> bz;               // Bz(t) samples [T], uniformly spaced over [bz_t0, bz_t1] ps
  double bz_t0 = 0.0, bz_t1 = 0.0;
  struct AdjBuf {
    DevArray<double> hbase, ck, segY, segH, segZ, segYend, lam, g[4], abar, mu, w, v, vb, z, a1, q, bpart, zpart,
        dku, ninvvol, zn, io[5];
  } ab;
  double cnt[8] = {};                   // stage evals, recomputed evals, VJPs, CG its fwd / transposed, ...
  double pulse_hz(double t_ps) const;
  void begin_timed_field();
  void end_timed_field();
  void stage_eval(const double* Y, double t_ps, double* k, double* H);
  void rk4_substep(double* y, double t_ps, double ds_ps, double* Ys, double* Hs);
  void vjp(const double* Y, const double* H, const double* abar, double* gout, double* zpart, int stage);
  void step_rk4(double* m_dev, int nsteps, double dt_ps, int nsub, double t0_ps, bool normalize);
  void adjoint_rk4(const double* m0, int nsteps, double dt_ps, int nsub, int ckpt, double t0_ps, bool normalize,
                   const double* w, double* m_final, double* grad_m0, double* grad_ku, double* grad_bz);
  double time_scale() const { return gamma / (1.0 + alpha * alpha) * 1e-12; }
  void sync() { TMB_CUDA(cudaStreamSynchronize(stream)); }
};

void Solver::ctx_prof_begin(int id, cudaStream_t st, double bytes) { ctx->prof.begin(id, st, bytes); }
void Solver::ctx_prof_end(cudaStream_t st) { ctx->prof.end(st); }
bool Solver::ctx_prof_on() const { return ctx->prof.on; }

void Solver::iteration_body(int precision, cudaStream_t st, bool profile) {
  const SellView A0 = lev[0].fine_view(rep);
  const bool f64 = precision == TMB_FP64;
  // p = z + beta p and q = A z + beta q: the product gathers z only (FP64 operator values on both
  // paths: the CG's own operator, see kCgOperatorF64; exact through the dictionary when coded)
  const bool op64 = f64 || kCgOperatorF64;
  if (profile) ctx_prof_begin(6, st, nnz_fine * (lev[0].fine_value_bytes(op64) + 4.0) + 5.0 * 8.0 * n * rep);
  if (lev[0].dict) launch_cg_dir_spmv<uint8_t>(A0, lev[0].Aq.p, z.p, p.p, q.p, Sd, partials.p, st);
  else if (op64) launch_cg_dir_spmv<double>(A0, lev[0].Ad.p, z.p, p.p, q.p, Sd, partials.p, st);
  else launch_cg_dir_spmv<float>(A0, lev[0].Af.p, z.p, p.p, q.p, Sd, partials.p, st);
  if (profile) ctx_prof_end(st);
  if (lev.size() > 1 && rep < 8) {
    // x, r update fused with the V-cycle's first sweep; the residual alternates between buffers
    // (with many interleaved replicas the two gathered vectors no longer stay in L2: separate)
    const double* rold = rbuf[rc].p;
    double* rnew = rbuf[rc ^ 1].p;
    rc ^= 1;
    DevLevel& L = lev[0];
    if (profile) ctx_prof_begin(8, st, nnz_fine * (L.fine_value_bytes(f64) + 4.0) + 9.0 * 8.0 * n * rep);
    if (L.dict)
      launch_cg_update_jacobi0<uint8_t>(A0, L.Aq.p, L.dinv.p, p.p, q.p, x.p, rold, rnew, L.X.p, L.R.p, Sd,
                                        partials.p, st);
    else if (f64)
      launch_cg_update_jacobi0<double>(A0, L.Ad.p, L.dinv.p, p.p, q.p, x.p, rold, rnew, L.X.p, L.R.p, Sd,
                                       partials.p, st);
    else
      launch_cg_update_jacobi0<float>(A0, L.Af.p, L.dinv.p, p.p, q.p, x.p, rold, rnew, L.X.p, L.R.p, Sd,
                                      partials.p, st);
    if (profile) ctx_prof_end(st);
    vcycle(0, rnew, z.p, precision, st, 0, true);
  } else {
    if (profile) ctx_prof_begin(16, st, 6.0 * 8.0 * n * rep);
    launch_cg_update(n * rep, p.p, q.p, x.p, rbuf[rc].p, Sd, partials.p, st);
    if (profile) ctx_prof_end(st);
    precondition_rz(precision, st, false);
  }
}

cudaGraphExec_t Solver::graph_for(int precision) {
  if (graph_exec[precision]) return graph_exec[precision];
  cudaStream_t st = ctx->stream;
  cudaGraph_t graph = nullptr;
  const long long before = launch_count();
  TMB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    for (int q = 0; q < kGraphIters; ++q) iteration_body(precision, st, false);
  } catch (...) {
    cudaStreamEndCapture(st, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  TMB_CUDA(cudaStreamEndCapture(st, &graph));
  graph_nodes[precision] = launch_count() - before;
  note_launches(-graph_nodes[precision]);  // captured, not launched
  const cudaError_t e = cudaGraphInstantiate(&graph_exec[precision], graph, 0);
  cudaGraphDestroy(graph);
  TMB_CUDA(e);
  return graph_exec[precision];
}

// ------------------------------------------------------------------------------------------
// Solver implementation
// ------------------------------------------------------------------------------------------
void Solver::compute() {
  cudaStream_t st = ctx->stream;
  n = A.nrows;
  rep = want_rep >= 1 ? want_rep : ctx->rep;
  if (n <= 0) throw Error(TMB_ERR_ARG, "solver: empty matrix");
  // constraints: rows whose only non-zero entry is a unit diagonal
  std::vector<int> cm(n, 0);
  for (int i = 0; i < n; ++i) {
    bool unit = false, other = false;
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
      if (A.col[k] == i && A.val[k] == 1.0) unit = true;
      else if (A.val[k] != 0.0) other = true;
    }
    cm[i] = unit && !other;
  }
  // symmetric elimination: A' keeps free-free couplings, the free-constrained ones go to the lift.
  // Stored entries that are exactly zero are dropped (they add nothing to any product): on meshes of
  // Kuhn-split cuboids the face-diagonal couplings of the stiffness matrix vanish exactly, about
  // half of the pattern, so every product over A' gathers half as many entries there.
  Csr Ap, L;
  Ap.nrows = Ap.ncols = L.nrows = L.ncols = n;
  Ap.ptr.assign(n + 1, 0);
  L.ptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    if (cm[i]) {
      Ap.col.push_back(i);
      Ap.val.push_back(1.0);
    } else {
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
        const int j = A.col[k];
        if (A.val[k] == 0.0 && j != i) continue;
        if (cm[j]) {
          L.col.push_back(j);
          L.val.push_back(A.val[k]);
        } else {
          Ap.col.push_back(j);
          Ap.val.push_back(A.val[k]);
        }
      }
    }
    Ap.ptr[i + 1] = int(Ap.col.size());
    L.ptr[i + 1] = int(L.col.size());
  }
  Csr LT;
  LT.nrows = LT.ncols = n;
  LT.ptr.assign(n + 1, 0);
  for (int j : L.col) LT.ptr[j + 1]++;
  for (int i = 0; i < n; ++i) LT.ptr[i + 1] += LT.ptr[i];
  LT.col.resize(L.col.size());
  LT.val.resize(L.col.size());
  {
    std::vector<int> fill(LT.ptr.begin(), LT.ptr.end() - 1);
    for (int i = 0; i < n; ++i)
      for (int k = L.ptr[i]; k < L.ptr[i + 1]; ++k) {
        const int q = fill[L.col[k]]++;
        LT.col[q] = i;
        LT.val[q] = L.val[k];
      }
  }
  drop_graphs();  // captured graphs hold the previous buffers
  amg_build(Ap, prm, H);
  nnz_fine = double(Ap.nnz());
  lev.clear();
  lev.resize(H.levels.size());
  for (size_t l = 0; l < H.levels.size(); ++l) {
    const AmgLevel& hl = H.levels[l];
    DevLevel& d = lev[l];
    d.n = hl.A.nrows;
    if (l == 0) {
      SellHost S = build_sell(d.n, hl.A.ptr.data(), hl.A.col.data());
      d.A.upload(S, st);
      d.Ad.upload(sell_values<double>(S, hl.A.val.data()), st);
      d.Af.upload(sell_values<float>(S, hl.A.val.data()), st);
      {
        std::vector<double> tab{0.0};
        std::unordered_map<uint64_t, int> slot{{0ull, 0}};
        std::vector<uint8_t> code(hl.A.val.size());
        bool fits = true;
        for (size_t k = 0; k < hl.A.val.size() && fits; ++k) {
          uint64_t bits;
          std::memcpy(&bits, &hl.A.val[k], sizeof bits);
          auto it = slot.find(bits);
          if (it == slot.end()) {
            if (int(tab.size()) == kDictMax) {
              fits = false;
              break;
            }
            it = slot.emplace(bits, int(tab.size())).first;
            tab.push_back(hl.A.val[k]);
          }
          code[k] = uint8_t(it->second);
        }
        d.dict = fits;
        if (fits) {
          std::vector<uint8_t> q(S.col.size(), 0);  // padding: code 0 = 0.0
          for (size_t k = 0; k < S.map.size(); ++k) q[S.map[k]] = code[k];
          d.Aq.upload(q, st);
          d.Atab.upload(tab, st);
        }
      }
    } else {
      d.Ac.upload(hl.A, st);
      d.tA = rep >= 8 ? 1 : csr_threads_per_row(hl.A.nrows, hl.A.nnz());
    }
    d.dinv.upload(hl.dinv, st);
    d.X.alloc(size_t(d.n) * rep);
    d.R.alloc(size_t(d.n) * rep);
    if (l > 0) {
      d.b.alloc(size_t(d.n) * rep);
      d.out.alloc(size_t(d.n) * rep);
    }
    if (l + 1 < H.levels.size()) {
      d.P.upload(hl.P, st);
      d.Rop.upload(hl.R, st);
      // with 8 or more interleaved replicas a warp already covers replicas of one row
      d.tP = rep >= 8 ? 1 : csr_threads_per_row(hl.P.nrows, hl.P.nnz());
      d.tR = rep >= 8 ? 1 : csr_threads_per_row(hl.R.nrows, hl.R.nnz());
      if (l > 0 && rep == 1) {
        Csr AP;
        csr_multiply(hl.A, hl.P, AP);
        std::vector<double> pvals;
        if (values_on_pattern(AP, hl.P, pvals)) {
          d.AP.upload(AP, st);
          d.pv.upload(pvals, st);
          std::vector<float> pf(pvals.begin(), pvals.end());
          d.pvf.upload(pf, st);
          d.tAP = csr_threads_per_row(AP.nrows, AP.nnz());
          d.fused_post = true;
        }
        Csr RA;
        csr_multiply(hl.R, hl.A, RA);
        std::vector<double> rv;
        if (values_on_pattern(RA, hl.R, rv)) {
          for (int j = 0; j < RA.nrows; ++j)
            for (int k = RA.ptr[j]; k < RA.ptr[j + 1]; ++k) RA.val[k] = rv[k] - RA.val[k] * hl.dinv[RA.col[k]];
          d.M.upload(RA, st);
          d.tM = csr_threads_per_row(RA.nrows, RA.nnz());
          d.fused_pre = true;
        }
      }
    }
  }
  ncoarse = H.ncoarse;
  csubset = !H.coarse_idx.empty() || !H.coarse_diag_inv.empty();
  if (csubset) {
    cidx.upload(H.coarse_idx, st);
    cdiag.upload(H.coarse_diag_inv, st);
    cb.alloc(size_t(std::max(ncoarse, 1)) * rep);
    cx.alloc(size_t(std::max(ncoarse, 1)) * rep);
  }
  cld = ncoarse + (ncoarse & 1);  // even rows: 16-byte loads
  {
    std::vector<double> ci(size_t(ncoarse) * cld, 0.0);
    for (int i = 0; i < ncoarse; ++i)
      std::copy(H.coarse_inv.begin() + size_t(i) * ncoarse, H.coarse_inv.begin() + size_t(i + 1) * ncoarse,
                ci.begin() + size_t(i) * cld);
    cinv.upload(ci, st);
    cldf = (ncoarse + 3) & ~3;  // FP32 copy for the mixed path, rows padded to a multiple of 4
    std::vector<float> cf(size_t(ncoarse) * cldf, 0.0f);
    for (int i = 0; i < ncoarse; ++i)
      for (int k = 0; k < ncoarse; ++k) cf[size_t(i) * cldf + k] = float(H.coarse_inv[size_t(i) * ncoarse + k]);
    cinvf.upload(cf, st);
  }
  lift.upload(L, st);
  liftT.upload(LT, st);
  for (bool& h : has_xadj) h = false;
  cmask.upload(cm, st);
  const size_t nr = size_t(n) * rep;
  x.alloc(nr);
  x.zero(st);
  rbuf[0].alloc(nr);
  rbuf[1].alloc(nr);
  z.alloc(nr);
  p.alloc(nr);
  q.alloc(nr);
  bp.alloc(nr);
  partials.alloc(size_t(2) * grid_for((long long)nr) + 64);
  if (!Sd) TMB_CUDA(cudaMalloc(&Sd, sizeof(CgScalars)));
  if (!Sh) TMB_CUDA(cudaMallocHost(&Sh, sizeof(CgScalars)));
  std::memset(Sh, 0, sizeof(CgScalars));
  TMB_CUDA(cudaMemcpyAsync(Sd, Sh, sizeof(CgScalars), cudaMemcpyHostToDevice, st));
  TMB_CUDA(cudaStreamSynchronize(st));
  has_x = false;
  computed = true;
}

void Solver::vcycle(size_t l, const double* b, double* out, int precision, cudaStream_t st, int rz_mode,
                    bool presmoothed) {
  DevLevel& L = lev[l];
  const int* done = &Sd->done;
  const bool f64 = precision == TMB_FP64;
  // live profile (kernel by kernel, never inside a graph capture): algorithmic bytes per launch
  const bool prof = ctx_prof_on();
  const double sv = f64 ? 8.0 : 4.0, R = double(rep);
  auto pb = [&](int id, double bytes) {
    if (prof) ctx_prof_begin(id, st, bytes);
  };
  auto pe = [&]() {
    if (prof) ctx_prof_end(st);
  };
  if (l + 1 == lev.size()) {
    pb(14, double(ncoarse) * ncoarse * sv + 2.0 * 8.0 * ncoarse * R);
    if (csubset) {
      launch_coarse_diag(L.n, rep, cdiag.p, b, out, done, st);
      if (ncoarse > 0) {
        launch_rows_move(ncoarse, rep, cidx.p, b, cb.p, false, done, st);
        launch_coarse_solve(ncoarse, cld, rep, cinv.p, cb.p, cx.p, done, st, f64 ? nullptr : cinvf.p, cldf);
        launch_rows_move(ncoarse, rep, cidx.p, cx.p, out, true, done, st);
      }
    } else {
      launch_coarse_solve(ncoarse, cld, rep, cinv.p, b, out, done, st, f64 ? nullptr : cinvf.p, cldf);
    }
    pe();
    return;
  }
  DevLevel& C = lev[l + 1];
  const double nl = double(L.n) * R, nc = double(C.n) * R;
  const double nnz_l = l == 0 ? nnz_fine : double(L.Ac.col.n);
  const double sweep = nnz_l * ((l == 0 ? L.fine_value_bytes(f64) : sv) + 4.0) + (l == 0 ? 0.0 : 4.0 * (L.n + 1));
  if (l == 0) {
    const SellView A = L.fine_view(rep);
    if (!presmoothed) {
      pb(10, sweep + 4.0 * 8.0 * nl);
      if (L.dict) launch_jacobi0_residual<uint8_t>(A, L.Aq.p, L.dinv.p, b, L.X.p, L.R.p, done, st);
      else if (f64) launch_jacobi0_residual<double>(A, L.Ad.p, L.dinv.p, b, L.X.p, L.R.p, done, st);
      else launch_jacobi0_residual<float>(A, L.Af.p, L.dinv.p, b, L.X.p, L.R.p, done, st);
      pe();
    }
  } else if (L.fused_pre) {
    // first sweep with its residual, and the restriction as M b, in one launch
    const CsrView A = L.Ac.view(rep);
    pb(13, sweep + 4.0 * 8.0 * nl + double(L.M.col.n) * (sv + 4.0) + 4.0 * (C.n + 1) + 8.0 * nc);
    if (f64)
      launch_csr_pre_restrict<double>(A, L.Ac.v.p, L.dinv.p, b, L.X.p, L.R.p, L.tA, L.M.view(rep), L.M.v.p, C.b.p,
                                      L.tM, done, st);
    else
      launch_csr_pre_restrict<float>(A, L.Ac.vf.p, L.dinv.p, b, L.X.p, L.R.p, L.tA, L.M.view(rep), L.M.vf.p, C.b.p,
                                     L.tM, done, st);
    pe();
  } else {
    const CsrView A = L.Ac.view(rep);
    pb(13, sweep + 4.0 * 8.0 * nl);
    if (f64) launch_csr_jacobi0_residual<double>(A, L.Ac.v.p, L.dinv.p, b, L.X.p, L.R.p, done, st, L.tA);
    else launch_csr_jacobi0_residual<float>(A, L.Ac.vf.p, L.dinv.p, b, L.X.p, L.R.p, done, st, L.tA);
    pe();
  }
  if (l == 0 || !L.fused_pre) {
    pb(11, double(L.Rop.col.n) * (sv + 4.0) + 4.0 * (C.n + 1) + 8.0 * (nl + nc));
    if (f64) launch_csr_spmv<double>(L.Rop.view(rep), L.Rop.v.p, L.R.p, C.b.p, false, done, st, L.tR);
    else launch_csr_spmv<float>(L.Rop.view(rep), L.Rop.vf.p, L.R.p, C.b.p, false, done, st, L.tR);
    pe();
  }
  vcycle(l + 1, C.b.p, C.out.p, precision, st, -1);
  if (l > 0 && L.fused_post) {
    // prolongation and post-smoothing sweep in one pass over the rows of A P
    pb(13, double(L.AP.col.n) * (2.0 * sv + 4.0) + 4.0 * (L.n + 1) + 8.0 * (nc + 4.0 * nl));
    if (f64)
      launch_csr_prolong_smooth<double>(L.AP.view(rep), L.AP.v.p, L.pv.p, L.dinv.p, L.X.p, L.R.p, C.out.p, out, done,
                                        st, L.tAP);
    else
      launch_csr_prolong_smooth<float>(L.AP.view(rep), L.AP.vf.p, L.pvf.p, L.dinv.p, L.X.p, L.R.p, C.out.p, out, done,
                                       st, L.tAP);
    pe();
    return;
  }
  pb(12, double(L.P.col.n) * (sv + 4.0) + 4.0 * (L.n + 1) + 8.0 * (nc + 2.0 * nl));
  if (f64) launch_csr_spmv<double>(L.P.view(rep), L.P.v.p, C.out.p, L.X.p, true, done, st, L.tP);
  else launch_csr_spmv<float>(L.P.view(rep), L.P.vf.p, C.out.p, L.X.p, true, done, st, L.tP);
  pe();
  if (l == 0) {
    const SellView A = L.fine_view(rep);
    pb(9, sweep + 5.0 * 8.0 * nl);
    if (rz_mode >= 0) {
      // finest level: the post-smoothing sweep also reduces r.z for the next CG direction
      if (L.dict) launch_jacobi_rz<uint8_t>(A, L.Aq.p, L.dinv.p, b, L.X.p, out, Sd, partials.p, rz_mode == 1, st);
      else if (f64) launch_jacobi_rz<double>(A, L.Ad.p, L.dinv.p, b, L.X.p, out, Sd, partials.p, rz_mode == 1, st);
      else launch_jacobi_rz<float>(A, L.Af.p, L.dinv.p, b, L.X.p, out, Sd, partials.p, rz_mode == 1, st);
    } else {
      if (L.dict) launch_jacobi<uint8_t>(A, L.Aq.p, L.dinv.p, b, L.X.p, out, done, st);
      else if (f64) launch_jacobi<double>(A, L.Ad.p, L.dinv.p, b, L.X.p, out, done, st);
      else launch_jacobi<float>(A, L.Af.p, L.dinv.p, b, L.X.p, out, done, st);
    }
    pe();
  } else {
    const CsrView A = L.Ac.view(rep);
    pb(13, sweep + 4.0 * 8.0 * nl);
    if (f64) launch_csr_jacobi<double>(A, L.Ac.v.p, L.dinv.p, b, L.X.p, out, done, st, L.tA);
    else launch_csr_jacobi<float>(A, L.Ac.vf.p, L.dinv.p, b, L.X.p, out, done, st, L.tA);
    pe();
  }
}

// Preconditioner application z = M r followed by rho = r.z (first: beta = 0).
void Solver::precondition_rz(int precision, cudaStream_t st, bool first) {
  if (lev.size() > 1) {
    vcycle(0, rbuf[rc].p, z.p, precision, st, first ? 1 : 0);
  } else {
    vcycle(0, rbuf[rc].p, z.p, precision, st, -1);
    launch_cg_rz(n * rep, rbuf[rc].p, z.p, Sd, partials.p, first, st);
  }
}

// The start of a solve: b' = b_F - L b_C with x_C pinned, r = b' - A x from the warm start, and the
// first V-cycle with r.z (beta = 0).
void Solver::solve_start(const double* b_dev, int precision, cudaStream_t st) {
  const SellView A0 = lev[0].fine_view(rep);
  const bool f64 = precision == TMB_FP64;
  const bool prof = ctx_prof_on();
  const bool op64 = f64 || kCgOperatorF64;
  if (prof)
    ctx_prof_begin(15, st, double(lift.col.n) * ((op64 ? 8.0 : 4.0) + 4.0) +
                               nnz_fine * (lev[0].fine_value_bytes(op64) + 4.0) + 8.0 * 8.0 * n * rep);
  if (op64) launch_cg_init<double>(n, lift.view(rep), lift.v.p, cmask.p, b_dev, bp.p, x.p, st);
  else launch_cg_init<float>(n, lift.view(rep), lift.vf.p, cmask.p, b_dev, bp.p, x.p, st);
  rc = 0;  // graphs are captured with the residual starting in rbuf[0]
  if (lev[0].dict) launch_cg_residual<uint8_t>(A0, lev[0].Aq.p, bp.p, x.p, rbuf[0].p, Sd, partials.p, st);
  else if (op64) launch_cg_residual<double>(A0, lev[0].Ad.p, bp.p, x.p, rbuf[0].p, Sd, partials.p, st);
  else launch_cg_residual<float>(A0, lev[0].Af.p, bp.p, x.p, rbuf[0].p, Sd, partials.p, st);
  if (prof) ctx_prof_end(st);
  precondition_rz(precision, st, true);
}

void Solver::solve(const double* b_dev, int precision) {
  if (!computed) throw Error(TMB_ERR_STATE, "solver: compute() not called");
  cudaStream_t st = ctx->stream;
  Sh->tol2 = tol * tol;
  Sh->maxit = maxit;
  Sh->done = 0;
  Sh->status = 0;
  Sh->iter = 0;
  TMB_CUDA(cudaMemcpyAsync(Sd, Sh, sizeof(CgScalars), cudaMemcpyHostToDevice, st));
  solve_start(b_dev, precision, st);
  if (!ctx_prof_on()) {
    // Graph path: kGraphIters iterations per graph launch; the first batch covers the
    // previous solve's iteration count, then the done flag is polled after every launch.
    // Kernels after convergence return at once (they read the done flag).
    cudaGraphExec_t g = graph_for(precision);
    const int batches = (maxit + kGraphIters - 1) / kGraphIters;
    int first = std::max(1, (last_iters + kGraphIters - 1) / kGraphIters);
    int launched = 0;
    while (launched < batches) {
      const int nlaunch = std::min(batches - launched, launched == 0 ? first : 1);
      for (int q = 0; q < nlaunch; ++q) {
        TMB_CUDA(cudaGraphLaunch(g, st));
        note_launches(graph_nodes[precision]);
      }
      launched += nlaunch;
      TMB_CUDA(cudaMemcpyAsync(Sh, Sd, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
      TMB_CUDA(cudaStreamSynchronize(st));
      if (Sh->done) break;
    }
  } else {
    for (int it = 0; it < maxit; ++it) {
      iteration_body(precision, st, true);
      if ((it + 1) % check_every == 0 || it + 1 == maxit) {
        TMB_CUDA(cudaMemcpyAsync(Sh, Sd, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
        TMB_CUDA(cudaStreamSynchronize(st));
        if (Sh->done) break;
      }
    }
  }
  TMB_CUDA(cudaGetLastError());
  TMB_CUDA(cudaMemcpyAsync(Sh, Sd, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
  TMB_CUDA(cudaStreamSynchronize(st));
  if (Sh->status == 2) x.zero(st);
  last_iters = Sh->iter;
  last_status = Sh->status == 2 ? 0 : Sh->status;
  last_relres = (Sh->bb > 0.0) ? std::sqrt(Sh->rr / Sh->bb) : 0.0;
  has_x = true;
}

void Solver::solve_t(const double* c, double* out, int precision, int slot) {
  cudaStream_t st = ctx->stream;
  slot = (slot < 0 || slot >= kAdjSlots) ? 0 : slot;
  ct.alloc(n);
  xfwd.alloc(n);
  DevArray<double>& xa = xadj[slot];
  if (!has_xadj[slot]) {
    xa.alloc(n);
    xa.zero(st);
    has_xadj[slot] = true;
  }
  launch_mask_constrained(n, cmask.p, c, ct.p, st);
  TMB_CUDA(cudaMemcpyAsync(xfwd.p, x.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  TMB_CUDA(cudaMemcpyAsync(x.p, xa.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  solve(ct.p, precision);
  if (precision == TMB_FP64) launch_lift_t<double>(n, liftT.view(), liftT.v.p, cmask.p, c, x.p, out, st);
  else launch_lift_t<float>(n, liftT.view(), liftT.vf.p, cmask.p, c, x.p, out, st);
  TMB_CUDA(cudaMemcpyAsync(xa.p, x.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  TMB_CUDA(cudaMemcpyAsync(x.p, xfwd.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
}

// ------------------------------------------------------------------------------------------
// Context implementation
// ------------------------------------------------------------------------------------------
void Ctx::set_operators(int nx, const int* ptr, const int* col, const double* K_, const double* const* g_,
                        const double* const* tg_, const double* vol, int nb_, const int* bn, const double* area_,
                        const double* nvn_soa) {
  if (nx <= 0 || nb_ < 0) throw Error(TMB_ERR_ARG, "set_operators: bad sizes");
  cudaStream_t st = stream;
  n = nx;
  nb = nb_;
  const int nnz = ptr[nx];
  hptr.assign(ptr, ptr + nx + 1);
  hcol.assign(col, col + nnz);
  hK.assign(K_, K_ + nnz);
  hvol.assign(vol, vol + nx);
  hbnodes.assign(bn, bn + nb_);
  SellHost S = build_sell(nx, ptr, col);
  pat.upload(S, st);
  K.upload(sell_values<double>(S, K_), st);
  Kf.upload(sell_values<float>(S, K_), st);
  for (int d = 0; d < 3; ++d) {
    g[d].upload(sell_values<double>(S, g_[d]), st);
    gf[d].upload(sell_values<float>(S, g_[d]), st);
    tg[d].upload(sell_values<double>(S, tg_[d]), st);
    tgf[d].upload(sell_values<float>(S, tg_[d]), st);
  }
  // dictionary codes of the three grad and the three tGrad operators (all or none of a kind)
  auto code3 = [&](const double* const* ops, DevArray<uint8_t>* q, DevArray<double>& tab) {
    std::vector<double> t(96, 0.0);
    std::vector<std::vector<uint8_t>> codes(3);
    for (int d = 0; d < 3; ++d) {
      std::unordered_map<uint64_t, int> slot{{0ull, 0}};
      int used = 1;  // local code 0 is 0.0 (the padding)
      std::vector<uint8_t> c(nnz);
      for (int k = 0; k < nnz; ++k) {
        uint64_t bits;
        std::memcpy(&bits, &ops[d][k], sizeof bits);
        auto it = slot.find(bits);
        if (it == slot.end()) {
          if (used == 32) return false;
          it = slot.emplace(bits, used).first;
          t[32 * d + used] = ops[d][k];
          ++used;
        }
        c[k] = uint8_t(32 * d + it->second);
      }
      codes[d] = std::move(c);
    }
    for (int d = 0; d < 3; ++d) {
      std::vector<uint8_t> sc(S.col.size(), uint8_t(32 * d));  // padding: the section's 0.0
      for (size_t k = 0; k < S.map.size(); ++k) sc[S.map[k]] = codes[d][k];
      q[d].upload(sc, st);
    }
    tab.upload(t, st);
    return true;
  };
  g_coded = code3(g_, gq, gtab);
  tg_coded = code3(tg_, tgq, tgtab);
  {
    std::vector<int> xp(nx + 1, 0), xcol;
    std::vector<double> xv;
    for (int i = 0; i < nx; ++i) {
      for (int k = ptr[i]; k < ptr[i + 1]; ++k)
        if (K_[k] != 0.0 || col[k] == i) {
          xcol.push_back(col[k]);
          xv.push_back(K_[k]);
        }
      xp[i + 1] = int(xcol.size());
    }
    has_patx = double(xcol.size()) < 0.9 * double(nnz);
    nnz_x = (long long)xcol.size();
    if (has_patx) {
      SellHost SX = build_sell(nx, xp.data(), xcol.data());
      patx.upload(SX, st);
      Kx.upload(sell_values<double>(SX, xv.data()), st);
      Kxf.upload(sell_values<float>(SX, xv.data()), st);
    }
  }
  node_vol.upload(vol, nx, st);
  area.upload(area_, nx, st);
  harea.assign(area_, area_ + nx);
  hKc1.clear();
  hKs.clear();
  has_cub = has_srf = has_stt = false;
  nvn.upload(nvn_soa, size_t(3) * nx, st);
  bnodes.upload(bn, nb_, st);
  std::vector<int> bi(nx, -1);
  for (int i = 0; i < nb_; ++i) bi[bn[i]] = i;
  bindex.upload(bi, st);
  rep = 1;
  for (auto* a : {&hext, &hdem, &hfix}) {
    a->alloc(size_t(3) * nx);
    a->zero(st);
  }
  has_material = false;
  has_bem = false;
  H = HMat{};
  bem_mode = 0;
  neu.reset();
  dir.reset();
  coff = {0, n};
  cboff = {0, nb};
  shared_bem = false;
  sync();
}

// Declares the mesh a disjoint union of nc components (batched instances of tetmag's
// single-mesh problem): the operators must not couple components; each component keeps its
// own pinned Neumann node (node N_c / 2 of the component, DemagField.cpp:80) and its own BEM
// block.  shared: the components are identical copies (same operators and boundary numbering,
// checked) that share one BEM block.
void Ctx::set_components(int nc, const int* off, bool shared) {
  require_mesh();
  if (nc < 1 || !off || off[0] != 0 || off[nc] != n) throw Error(TMB_ERR_ARG, "tmb_set_components: bad offsets");
  for (int c = 0; c < nc; ++c)
    if (off[c + 1] <= off[c]) throw Error(TMB_ERR_ARG, "tmb_set_components: offsets must increase");
  std::vector<int> co(off, off + nc + 1), cb(nc + 1, 0);
  for (int c = 0; c < nc; ++c) {
    for (int i = co[c]; i < co[c + 1]; ++i)
      for (int q = hptr[i]; q < hptr[i + 1]; ++q)
        if (hcol[q] < co[c] || hcol[q] >= co[c + 1])
          throw Error(TMB_ERR_ARG, "tmb_set_components: the operators couple two components");
    cb[c] = int(std::lower_bound(hbnodes.begin(), hbnodes.end(), co[c]) - hbnodes.begin());
  }
  cb[nc] = nb;
  for (int c = 0; c < nc; ++c)
    if (cb[c + 1] - cb[c] < 3) throw Error(TMB_ERR_ARG, "tmb_set_components: a component has no boundary");
  if (shared) {
    const int n0 = co[1], nb0 = cb[1];
    for (int c = 1; c < nc; ++c) {
      if (co[c + 1] - co[c] != n0 || cb[c + 1] - cb[c] != nb0)
        throw Error(TMB_ERR_ARG, "tmb_set_components: shared BEM needs components of equal size");
      for (int k = 0; k < nb0; ++k)
        if (hbnodes[cb[c] + k] - co[c] != hbnodes[k])
          throw Error(TMB_ERR_ARG, "tmb_set_components: shared BEM needs the same boundary numbering");
      for (int i = 0; i < n0; ++i) {
        const int a = hptr[i], b = hptr[co[c] + i];
        if (hptr[i + 1] - a != hptr[co[c] + i + 1] - b)
          throw Error(TMB_ERR_ARG, "tmb_set_components: shared BEM needs identical operators");
        for (int q = 0; q < hptr[i + 1] - a; ++q)
          if (hcol[b + q] - co[c] != hcol[a + q] || hK[b + q] != hK[a + q])
            throw Error(TMB_ERR_ARG, "tmb_set_components: shared BEM needs identical operators");
      }
    }
  }
  coff = co;
  cboff = cb;
  shared_bem = shared && nc > 1;
  has_bem = false;
  Bd.reset();
  Bf.reset();
  H = HMat{};
  bem_mode = 0;
  neu.reset();
  dir.reset();
}

// Declares rep interleaved replicas of the (single) mesh: state vectors grow to 3 * n * R, the
// operators, material and BEM matrix stay those of one mesh; the boundary product becomes one
// GEMM over the replicas.  Resets the solvers and the BEM (assembled afterwards).
void Ctx::set_replicas(int R) {
  require_mesh();
  if (R < 1) throw Error(TMB_ERR_ARG, "tmb_set_replicas: R must be >= 1");
  if (ncomp() != 1) throw Error(TMB_ERR_STATE, "tmb_set_replicas: not with tmb_set_components");
  if (size_t(n) * R * 3 >= size_t(1) << 31) throw Error(TMB_ERR_ARG, "tmb_set_replicas: n * R too large");
  cudaStream_t st = stream;
  rep = R;
  for (auto* a : {&hext, &hdem, &hfix}) {
    a->alloc(size_t(3) * nr());
    a->zero(st);
  }
  has_bem = false;
  H = HMat{};
  bem_mode = 0;
  neu.reset();
  dir.reset();
  tc_split = 0;
  sync();
}

// Padded boundary layout and matvec plan of the components (after the blocks are assembled).
void Ctx::plan_components() {
  const int nc = ncomp();
  std::vector<int> pos(nb);
  bem_entries = 0.0;
  if (rep > 1) {
    // replicas: the boundary values of all replicas as a [replica][ld] panel
    xstride = int(bem_ld(nb));
    xpad64.alloc(size_t(xstride) * rep);
    xpad32.alloc(size_t(xstride) * rep);
    xhi32.alloc(size_t(xstride) * rep);
    xlo32.alloc(size_t(xstride) * rep);
    bem_entries = double(nb) * nb;
    ntiles = 0;
    return;
  }
  if (shared_bem) {
    const int nbc = cboff[1];
    xstride = int(bem_ld(nbc));
    for (int c = 0; c < nc; ++c)
      for (int k = 0; k < nbc; ++k) pos[cboff[c] + k] = c * xstride + k;
    xpad64.alloc(size_t(xstride) * nc);
    xpad32.alloc(size_t(xstride) * nc);
    xhi32.alloc(size_t(xstride) * nc);
    xlo32.alloc(size_t(xstride) * nc);
    bem_entries = double(nbc) * nbc;
    ntiles = 0;
  } else {
    // tiles of up to 4 rows when the components are large enough to fill the GPU that way
    tile_rows = (nb >= 16384 && double(nb) / nc >= 256.0) ? 4 : 1;
    std::vector<GemvTile> t;
    long long boff = 0;
    int xo = 0;
    for (int c = 0; c < nc; ++c) {
      const int nbc = cboff[c + 1] - cboff[c], ld = int(bem_ld(nbc));
      for (int k = 0; k < nbc; ++k) pos[cboff[c] + k] = xo + k;
      for (int r = 0; r < nbc; r += tile_rows)
        t.push_back(GemvTile{boff + (long long)r * ld, xo, cboff[c] + r, nbc, std::min(tile_rows, nbc - r), ld, 0});
      boff += (long long)nbc * ld;
      xo += ld;
      bem_entries += double(nbc) * nbc;
    }
    ntiles = int(t.size());
    tiles.upload(t, stream);
    xpad64.alloc(size_t(xo));
    xpad32.alloc(size_t(xo));
  }
  xpad64.zero(stream);
  xpad32.zero(stream);
  xpos.upload(pos, stream);
}

void Ctx::set_material(const double* Js, const double* A, const double* Ku, const double* axis, const double* D,
                       double alpha_) {
  require_mesh();
  cudaStream_t st = stream;
  alpha = alpha_;
  std::vector<double> ij(n), vxc(n), vku(n, 0.0), vdm(n, 0.0);
  has_uni = false;
  has_dmi = false;
  for (int i = 0; i < n; ++i) {
    const double v = 1.0 / Js[i];
    ij[i] = std::isfinite(v) ? v : 0.0;  // main/TheLLG.cpp:110
    vxc[i] = -2.0 * A[i] / hvol[i] * ij[i];
    if (Ku) {
      vku[i] = 2.0 * Ku[i] * ij[i];
      has_uni |= (Ku[i] != 0.0);
    }
    if (D) {
      vdm[i] = D[i] / hvol[i] * ij[i];
      has_dmi |= (D[i] != 0.0);
    }
  }
  js.upload(Js, n, st);
  xc.upload(vxc, st);
  ku2.upload(vku, st);
  dmi_s.upload(vdm, st);
  hD.assign(n, 0.0);
  if (D) hD.assign(D, D + n);
  hij = ij;
  upload_dmi();
  upload_extra();
  if (axis) {
    kax.upload(axis, size_t(3) * n, st);
  } else {
    kax.alloc(size_t(3) * n);
    kax.zero(st);
  }
  has_material = true;
  sync();
}

void Ctx::set_bem_rowmajor(const double* /*unused*/) {}

void Ctx::ensure_demag() {
  require_mesh();
  require_material();
  if (!has_bem) throw Error(TMB_ERR_STATE, "no BEM matrix set");
  if (neu && dir) return;
  // Neumann matrix: K with row N/2 replaced by the unit row (DemagField.cpp:80, 204-220)
  // Dirichlet matrix: K with boundary rows replaced by unit rows (FEMprocessing.cpp:329-369)
  std::vector<char> isb(n, 0), pin(n, 0);
  for (int b : hbnodes) isb[b] = 1;
  for (int c = 0; c < ncomp(); ++c) pin[coff[c] + (coff[c + 1] - coff[c]) / 2] = 1;  // N/2 per component
  auto build = [&](auto pinned) {
    std::vector<int> p(n + 1, 0), c;
    std::vector<double> v;
    c.reserve(hcol.size());
    v.reserve(hcol.size());
    for (int i = 0; i < n; ++i) {
      if (pinned(i)) {
        c.push_back(i);
        v.push_back(1.0);
      } else {
        for (int q = hptr[i]; q < hptr[i + 1]; ++q) {
          c.push_back(hcol[q]);
          v.push_back(hK[q]);
        }
      }
      p[i + 1] = int(c.size());
    }
    auto s = std::make_unique<Solver>(this);
    s->set_matrix(n, p.data(), c.data(), v.data());
    s->tol = tol;
    s->maxit = maxit;
    s->compute();
    return s;
  };
  neu = build([&](int i) { return pin[i] != 0; });
  dir = build([&](int i) { return isb[i] != 0; });
  for (auto* a : {&rhs, &u1, &u2, &bdir}) a->alloc(size_t(nr()));
  u1b.alloc(nb);
  u1bf.alloc(nb);
  u2b.alloc(size_t(nb) * rep);
}

void Ctx::demag(const double* m) {
  ensure_demag();
  cudaStream_t st = stream;
  neu->tol = dir->tol = tol;
  neu->maxit = dir->maxit = maxit;
  const SellView S = pat.view(rep);
  const bool f64 = precision == TMB_FP64;
  const double sv = f64 ? 8.0 : 4.0, z = double(hptr[n]), N = double(nr()), B = double(nb) * rep;
  prof.begin(7, st, 0.0);
  prof.begin(1, st, z * (3 * (tg_coded ? 1.0 : sv) + 4) + N * 8 * 5);
  launch_div(m, js.p, 1.0 / kMu0, rhs.p, st);
  prof.end(st);
  prof.begin(4, st, 0.0);
  neu->solve(rhs.p, precision);
  prof.end(st);
  if (bem_mode == 2) {
    // H2 matvec (nested bases) in cluster order, scattered straight into the Dirichlet load
    const int w = f64 ? 0 : 1;
    prof.begin(3, st, H2[w].bytes + B * (sv + 8 + 8));
    if (f64)
      launch_h2_matvec<double>(h2_view<double>(0), neu->x.p, H.y.p, H.xp64.p, H.pos.p, n, bdir.p, H2[0].up,
                               H2[0].down, st);
    else
      launch_h2_matvec<float>(h2_view<float>(1), neu->x.p, H.y.p, H.xp32.p, H.pos.p, n, bdir.p, H2[1].up,
                              H2[1].down, st);
    prof.end(st);
  } else if (bem_mode == 1) {
    // hierarchical matvec in cluster order, scattered straight into the Dirichlet load
    const int w = f64 ? 0 : 1;
    prof.begin(3, st, H.bytes[w] + B * (sv + 8 + 8));
    if (f64) launch_h_matvec<double>(h_view<double>(0), neu->x.p, H.y.p, H.xp64.p, H.pos.p, n, bdir.p, st);
    else launch_h_matvec<float>(h_view<float>(1), neu->x.p, H.y.p, H.xp32.p, H.pos.p, n, bdir.p, st);
    prof.end(st);
  } else if (rep > 1) {
    // interleaved replicas: the replicas' boundary values as a panel, one GEMM, then the
    // Dirichlet load of every replica from the GEMM's [replica][row] output
    if (f64) launch_gather_rep<double>(nb, rep, neu->x.p, bnodes.p, xstride, xpad64.p, st);
    else launch_gather_rep<float>(nb, rep, neu->x.p, bnodes.p, xstride, xpad32.p, st);
    prof.begin(3, st, bem_entries * sv + B * (sv + 8));
    bem_gemm(f64, st);
    prof.end(st);
    launch_dirichlet_rep(n, rep, bindex.p, u2b.p, nb, bdir.p, st);
  } else if (ncomp() > 1) {
    // batched components: padded gather, then one GEMM (shared matrix) or per-component matvecs
    if (f64) launch_gather_pad<double>(nb, neu->x.p, bnodes.p, xpos.p, xpad64.p, st);
    else launch_gather_pad<float>(nb, neu->x.p, bnodes.p, xpos.p, xpad32.p, st);
    prof.begin(3, st, bem_entries * sv + B * (sv + 8));
    if (shared_bem) {
      bem_gemm(f64, st);
    } else {
      if (f64) launch_bem_gemv_tiles<double>(ntiles, tiles.p, tile_rows, Bd.p, xpad64.p, u2b.p, st);
      else launch_bem_gemv_tiles<float>(ntiles, tiles.p, tile_rows, Bf.p, xpad32.p, u2b.p, st);
    }
    prof.end(st);
    launch_dirichlet_values(n, bindex.p, u2b.p, bdir.p, st);
  } else {
    if (f64) launch_gather<double>(nb, neu->x.p, bnodes.p, u1b.p, st);
    else launch_gather<float>(nb, neu->x.p, bnodes.p, u1bf.p, st);
    prof.begin(3, st, B * B * sv + B * (sv + 8));
    if (f64) launch_bem_gemv<double>(nb, Bd.p, u1b.p, u2b.p, st);
    else launch_bem_gemv<float>(nb, Bf.p, u1bf.p, u2b.p, st);
    prof.end(st);
    launch_dirichlet_values(n, bindex.p, u2b.p, bdir.p, st);
  }
  prof.begin(5, st, 0.0);
  dir->solve(bdir.p, precision);  // synchronises: the GEMM's time-out word is readable below
  if ((shared_bem || rep > 1) && !f64 && gemm_tc && bits_h[2] != 0)
    throw Error(TMB_ERR_CUDA, "tensor-core boundary GEMM timed out waiting on a barrier");
  prof.end(st);
  prof.begin(2, st, z * (3 * (g_coded ? 1.0 : sv) + 4) + N * 8 * 11);
  launch_grad(neu->x.p, dir->x.p, hext.p, hdem.p, hfix.p, st);
  prof.end(st);
  prof.end(st);
  TMB_CUDA(cudaGetLastError());
  if (neu->last_status == 5 || dir->last_status == 5) throw Error(TMB_ERR_NAN, "demag solve broke down (NaN)");
  if (neu->last_status == 3 || dir->last_status == 3)
    throw Error(TMB_ERR_NOCONVERGE, "demag solve did not converge within maxiter");
}

// Replicas' boundary product.  Mixed path: the 3xTF32 tensor-core GEMM (its time-out word is
// copied to the pinned bits_h[2] behind it); FP64 path: the CUDA-core GEMM.
void Ctx::bem_gemm(bool f64, cudaStream_t st) {
  const int nbc = rep > 1 ? nb : cboff[1], nc = rep > 1 ? rep : ncomp();
  if (f64 || !gemm_tc || !bem_gemm_tc_supported(nbc, bem_ld(nbc), xstride)) {
    if (f64) launch_bem_gemm<double>(nbc, nc, Bd.p, xpad64.p, xstride, u2b.p, num_sms, st);
    else launch_bem_gemm<float>(nbc, nc, Bf.p, xpad32.p, xstride, u2b.p, num_sms, st);
    return;
  }
  if (tc_split == 0) tune_gemm_tc();
  launch_bem_gemm_tc(nbc, nc, bem_ld(nbc), Bf.p, xpad32.p, xstride, xhi32.p, xlo32.p, u2b.p, tc_split, tc_stages,
                     tc_err.p, st);
  TMB_CUDA(cudaMemcpyAsync(bits_h + 2, tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
}

// Autotuner of the tensor-core GEMM's K split: every candidate that gives at least one CTA per
// SM is timed (CUDA events, three launches after one warm-up) on the current panel, the fastest
// is kept for the context.
void Ctx::tune_gemm_tc() {
  const int nbc = rep > 1 ? nb : cboff[1], nc = rep > 1 ? rep : ncomp();
  cudaStream_t st = stream;
  tc_err.alloc(1);
  tc_err.zero(st);
  const int mt = (nbc + 127) / 128 * ((nc + 63) / 64), nks = (nbc + 31) / 32;
  cudaEvent_t e0, e1;
  TMB_CUDA(cudaEventCreate(&e0));
  TMB_CUDA(cudaEventCreate(&e1));
  // candidates: K split 1..8 (while the CTAs of a split stay within two waves) x TMA ring depth
  // 2, 3, 4; tc_tune_ms[sp] keeps the best depth's time for each split
  tc_tune_ms.assign(9, 0.0);
  double best = 1e300;
  int best_split = 1, best_stages = 4;
  for (int sp = 1; sp <= 8; ++sp) {
    if (sp > nks || (sp > 1 && mt * (sp - 1) >= 2 * num_sms)) break;
    for (int stg = 2; stg <= 4; ++stg) {
      launch_bem_gemm_tc(nbc, nc, bem_ld(nbc), Bf.p, xpad32.p, xstride, xhi32.p, xlo32.p, u2b.p, sp, stg, tc_err.p,
                         st);
      TMB_CUDA(cudaEventRecord(e0, st));
      for (int r = 0; r < 3; ++r)
        launch_bem_gemm_tc(nbc, nc, bem_ld(nbc), Bf.p, xpad32.p, xstride, xhi32.p, xlo32.p, u2b.p, sp, stg,
                           tc_err.p, st);
      TMB_CUDA(cudaEventRecord(e1, st));
      TMB_CUDA(cudaEventSynchronize(e1));
      float ms = 0.0f;
      TMB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (tc_tune_ms[sp] == 0.0 || ms / 3.0 < tc_tune_ms[sp]) tc_tune_ms[sp] = ms / 3.0;
      if (ms < best) {
        best = ms;
        best_split = sp;
        best_stages = stg;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int err = 0;
  TMB_CUDA(cudaMemcpy(&err, tc_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) throw Error(TMB_ERR_CUDA, "tensor-core boundary GEMM timed out waiting on a barrier");
  tc_split = best_split;
  tc_stages = best_stages;
}

template <typename T>
HMatView<T> Ctx::h_view(int w) const {
  HMatView<T> v;
  v.nb = nb;
  v.nrows = H.nrows;
  v.ngroups = H.ngroups[w];
  v.nterms = H.terms[w];
  v.gidx = H.gidx.p;
  v.near_rows = H.rows.p;
  v.near = H.nearb.p;
  v.far = H.farb.p;
  v.rank = H.rank[w].p;
  v.uoff = H.uoff[w].p;
  v.voff = H.voff[w].p;
  v.groups = H.groups[w].p;
  v.terms = H.termd[w].p;
  v.toff = H.toff[w].p;
  v.t = H.tval.p;
  if constexpr (sizeof(T) == 8) {
    v.D = H.D64.p;
    v.U = H.U64.p;
    v.V = H.V64.p;
  } else {
    v.D = H.D32.p;
    v.U = H.U32.p;
    v.V = H.V32.p;
  }
  return v;
}

template <typename T>
HMatView<T> Ctx::ht_view(int w) const {
  HMatView<T> v = h_view<T>(w);
  v.nrows = H.ntcols;
  v.near_rows = H.tcols.p;
  v.near = H.tnearb.p;
  v.ngroups = H.ntgroups[w];
  v.groups = H.tgroups[w].p;
  v.terms = H.ttermd[w].p;
  v.toff = H.ttoff[w].p;
  v.far = nullptr;
  v.rank = nullptr;
  v.uoff = nullptr;
  v.voff = nullptr;
  std::swap(v.U, v.V);  // t = U^T x, then y += V t
  return v;
}

// The transposed hierarchical product's work lists, from the host copies of the blocks: near
// tiles grouped by leaf column cluster; per precision, the admissible blocks ordered by column
// cluster, one term per rank with U's column as the streamed vector and V's column as the
// accumulated one, cut into runs of about the same work as the forward product's.
void Ctx::h_transpose_build() {
  if (H.tbuilt) return;
  cudaStream_t st = stream;
  std::vector<int> ord(H.hnearb.size());
  std::iota(ord.begin(), ord.end(), 0);
  // near blocks pair leaf clusters, whose position ranges are disjoint: the begin names the leaf
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
    return H.hnearb[a].cb < H.hnearb[b].cb || (H.hnearb[a].cb == H.hnearb[b].cb && H.hnearb[a].rb < H.hnearb[b].rb);
  });
  std::vector<HBlockDev> tn;
  std::vector<HNearRow> cols;
  for (int q : ord) {
    const HBlockDev& b = H.hnearb[q];
    const int p = int(tn.size());
    if (cols.empty() || cols.back().rb != b.cb) cols.push_back(HNearRow{b.cb, b.n, p, p + 1});
    else cols.back().last = p + 1;
    tn.push_back(b);
  }
  long long covered = 0;
  for (const auto& c : cols) covered += c.m;
  if (covered != nb) throw Error(TMB_ERR_INTERNAL, "H-matrix: leaf columns do not cover the boundary");
  H.tnearb.upload(tn, st);
  H.tcols.upload(cols, st);
  H.ntcols = int(cols.size());
  const int nf = int(H.hfarb.size());
  std::vector<int> fo(nf);
  std::iota(fo.begin(), fo.end(), 0);
  // a column cluster is its position range: a cluster and its first child begin at the same
  // position, so the blocks are grouped by (begin, size)
  std::stable_sort(fo.begin(), fo.end(), [&](int a, int b) {
    const HBlockDev &x = H.hfarb[a], &y = H.hfarb[b];
    if (x.cb != y.cb) return x.cb < y.cb;
    if (x.n != y.n) return x.n < y.n;
    return x.rb < y.rb;
  });
  for (int w = 0; w < 2; ++w) {
    // the compact factor offsets of precision w, in the forward block order
    std::vector<long long> uo(nf), vo(nf);
    std::vector<int> rk(nf);
    long long su = 0, sv = 0;
    for (int q = 0; q < nf; ++q) {
      rk[q] = H.ranks[size_t(3) * q + w];
      uo[q] = su;
      vo[q] = sv;
      su += (long long)rk[q] * pad4(H.hfarb[q].m);
      sv += (long long)rk[q] * pad4(H.hfarb[q].n);
    }
    std::vector<HTerm> td;
    std::vector<long long> to(size_t(nf) + 1);
    long long stt = 0;
    std::vector<HFarGroup> groups;
    for (int p = 0; p < nf; ++p) {
      const int q = fo[p];
      const HBlockDev& b = H.hfarb[q];
      to[p] = stt;
      const int mp = pad4(b.m), np = pad4(b.n);
      for (int l = 0; l < rk[q]; ++l) td.push_back(HTerm{uo[q] + (long long)l * mp, vo[q] + (long long)l * np, mp, b.rb});
      stt += rk[q];
      if (groups.empty() || groups.back().rb != b.cb || groups.back().m != b.n)
        groups.push_back(HFarGroup{b.cb, b.n, p, p + 1});
      else
        groups.back().last = p + 1;
    }
    to[nf] = stt;
    if (stt != H.terms[w]) throw Error(TMB_ERR_INTERNAL, "H-matrix: transposed term count differs");
    double total = 0.0;
    for (int q = 0; q < nf; ++q) total += double(rk[q]) * (H.hfarb[q].m + H.hfarb[q].n);
    const double wmax = std::max(4096.0, total / (64.0 * num_sms));
    std::vector<HFarGroup> items;
    std::vector<double> work;
    for (const HFarGroup& g : groups) {
      HFarGroup it{g.rb, g.m, g.first, g.first};
      double wk = 0.0;
      for (int p = g.first; p < g.last; ++p) {
        const int q = fo[p];
        const double wq = double(rk[q]) * (H.hfarb[q].m + H.hfarb[q].n);
        if (wk > 0.0 && wk + wq > wmax) {
          items.push_back(it);
          work.push_back(wk);
          it.first = p;
          wk = 0.0;
        }
        it.last = p + 1;
        wk += wq;
      }
      if (wk > 0.0) {
        items.push_back(it);
        work.push_back(wk);
      }
    }
    std::vector<int> order(items.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
    std::vector<HFarGroup> sorted;
    for (int g : order) sorted.push_back(items[g]);
    H.ntgroups[w] = int(sorted.size());
    H.tgroups[w].upload(sorted, st);
    H.ttoff[w].upload(to, st);
    H.ttermd[w].upload(td, st);
  }
  H.ty.alloc(size_t(std::max(nb, 1)));
  sync();
  H.tbuilt = true;
}

// y = B x or B^T x for boundary vectors in boundary-node order (device pointers), with the
// current boundary matrix form and precision: dense (mode 0), hierarchical (1) or H2 (2, forward
// only).  One component, no replicas.
void Ctx::bem_apply(const double* xb, double* yb, bool transpose) {
  require_mesh();
  if (!has_bem) throw Error(TMB_ERR_STATE, "bem_apply: no BEM matrix set");
  if (ncomp() != 1 || rep != 1) throw Error(TMB_ERR_STATE, "bem_apply: one component, no replicas");
  if (transpose && bem_mode == 2) throw Error(TMB_ERR_STATE, "bem_apply: the H2 form has no transposed product");
  cudaStream_t st = stream;
  const bool f64 = precision == TMB_FP64;
  if (bem_mode == 0) {
    if (f64 ? !Bd.p : !Bf.p) throw Error(TMB_ERR_STATE, "bem_apply: the dense matrix was not kept");
    if (transpose) {
      const int nch = bem_gemv_t_chunks(nb, num_sms);
      bap_part.alloc(size_t(nch) * nb);
      if (f64) launch_bem_gemv_t<double>(nb, Bd.p, xb, bap_part.p, nch, yb, st);
      else launch_bem_gemv_t<float>(nb, Bf.p, xb, bap_part.p, nch, yb, st);
    } else if (f64) {
      launch_bem_gemv<double>(nb, Bd.p, xb, yb, st);
    } else {
      // the FP32 operand copy of x: scatter to a node vector, gather in FP32
      bap_u.alloc(size_t(n));
      bap_f.alloc(size_t(nb));
      bap_u.zero(st);
      launch_scatter_add(nb, bnodes.p, xb, bap_u.p, st);
      launch_gather<float>(nb, bap_u.p, bnodes.p, bap_f.p, st);
      launch_bem_gemv<float>(nb, Bf.p, bap_f.p, yb, st);
    }
    return;
  }
  bap_u.alloc(size_t(n));
  bap_w.alloc(size_t(n));
  bap_u.zero(st);
  launch_scatter_add(nb, bnodes.p, xb, bap_u.p, st);
  if (transpose) {
    h_transpose_build();
    if (f64) launch_h_matvec_t<double>(ht_view<double>(0), bap_u.p, H.ty.p, H.xp64.p, st);
    else launch_h_matvec_t<float>(ht_view<float>(1), bap_u.p, H.ty.p, H.xp32.p, st);
    bap_w.zero(st);
    launch_scatter_add(nb, H.gidx.p, H.ty.p, bap_w.p, st);
  } else if (bem_mode == 2) {
    if (f64)
      launch_h2_matvec<double>(h2_view<double>(0), bap_u.p, H.y.p, H.xp64.p, H.pos.p, n, bap_w.p, H2[0].up, H2[0].down,
                               st);
    else
      launch_h2_matvec<float>(h2_view<float>(1), bap_u.p, H.y.p, H.xp32.p, H.pos.p, n, bap_w.p, H2[1].up, H2[1].down,
                              st);
  } else {
    if (f64) launch_h_matvec<double>(h_view<double>(0), bap_u.p, H.y.p, H.xp64.p, H.pos.p, n, bap_w.p, st);
    else launch_h_matvec<float>(h_view<float>(1), bap_u.p, H.y.p, H.xp32.p, H.pos.p, n, bap_w.p, st);
  }
  launch_gather<double>(nb, bap_w.p, bnodes.p, yb, st);
}

// Compresses the device-assembled dense FP64 BEM matrix into the hierarchical form:
// dense leaf tiles plus ACA low-rank blocks, FP64 terms to eps_fp64 and FP32 terms to eps_mixed.
// With `mesh` the entries come from the boundary mesh instead (no dense matrix needed): dense
// tiles with the reference arithmetic, low-rank blocks from the accurate far-field weights.
void Ctx::h_compress(const double* bxyz, const double* bnrm, int leaf, double eta, double eps_mixed,
                     double eps_fp64, int kmax, bool keep_dense, const MeshHost* mesh) {
  require_mesh();
  if (ncomp() > 1) throw Error(TMB_ERR_STATE, "hierarchical BEM: one component per context");
  if (!mesh && (!has_bem || !Bd.p))
    throw Error(TMB_ERR_STATE, "tmb_bem_compress: needs the dense FP64 BEM matrix on the device");
  if (leaf < 2 || leaf > 32) throw Error(TMB_ERR_ARG, "tmb_bem_compress: leaf size must be in [2, 32]");
  if (!(eta > 0.0) || !(eps_mixed > 0.0) || !(eps_fp64 > 0.0) || kmax < 1 || kmax > 128)
    throw Error(TMB_ERR_ARG, "tmb_bem_compress: bad eta / tolerance / rank cap (1..128)");
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t st = stream;
  HPartition P;
  // admissible blocks above 1024 rows or columns are subdivided: bounds the ACA work per CTA
  h_partition(bxyz, bnrm, nb, leaf, eta, 1024, P);
  // dense leaf tiles, grouped by leaf row cluster
  std::vector<HBlockDev> nearb;
  std::vector<HNearRow> rows;
  long long doff = 0;
  for (size_t q = 0; q < P.near.size(); ++q) {
    const HCluster& ct = P.clusters[P.near[q].first];
    const HCluster& cs = P.clusters[P.near[q].second];
    HBlockDev b{ct.begin, ct.end - ct.begin, cs.begin, cs.end - cs.begin, doff, 0, 0, 0};
    doff += (long long)b.m * b.n;
    if (rows.empty() || rows.back().rb != b.rb) rows.push_back(HNearRow{b.rb, b.m, int(q), int(q) + 1});
    else rows.back().last = int(q) + 1;
    nearb.push_back(b);
  }
  long long covered = 0;
  for (const auto& r : rows) covered += r.m;
  if (covered != nb) throw Error(TMB_ERR_INTERNAL, "H-matrix: leaf rows do not cover the boundary");
  // admissible blocks with ACA scratch offsets, grouped by row cluster
  std::vector<HBlockDev> farb;
  std::vector<HFarGroup> groups;
  long long us = 0, vs = 0, fl = 0;
  int last_cluster = -1;
  for (size_t q = 0; q < P.far.size(); ++q) {
    const HCluster& ct = P.clusters[P.far[q].first];
    const HCluster& cs = P.clusters[P.far[q].second];
    HBlockDev b{ct.begin, ct.end - ct.begin, cs.begin, cs.end - cs.begin, 0, us, vs, fl};
    us += (long long)kmax * b.m;
    vs += (long long)kmax * b.n;
    fl += b.m;
    if (P.far[q].first != last_cluster) {
      groups.push_back(HFarGroup{b.rb, b.m, int(q), int(q) + 1});
      last_cluster = P.far[q].first;
    } else {
      groups.back().last = int(q) + 1;
    }
    farb.push_back(b);
  }
  H = HMat{};
  H2[0] = H2Mat{};
  H2[1] = H2Mat{};
  H.nnear = int(nearb.size());
  H.nfar = int(farb.size());
  H.nrows = int(rows.size());
  std::vector<int> gidx(nb), pos(n, -1);
  for (int i = 0; i < nb; ++i) {
    gidx[i] = hbnodes[P.perm[i]];
    pos[gidx[i]] = i;
  }
  H.gidx.upload(gidx, st);
  H.pos.upload(pos, st);
  H.perm.upload(P.perm, st);
  if (mesh) {
    // geometry in cluster positions: coordinates, triangles, position -> touching triangles
    const BoundaryData& Bm = mesh->bnd;
    const int nt = int(Bm.tri_tet.size());
    std::vector<int> at(nb);
    for (int i = 0; i < nb; ++i) at[P.perm[i]] = i;
    std::vector<double> gx(size_t(3) * nb), gs(nb);
    for (int i = 0; i < nb; ++i) {
      for (int d = 0; d < 3; ++d) gx[size_t(3) * i + d] = mesh->xyz[size_t(3) * Bm.bnodes[P.perm[i]] + d];
      gs[i] = Bm.solid_angle[P.perm[i]];
    }
    std::vector<int> gt(size_t(3) * nt), aptr(nb + 1, 0);
    for (size_t k = 0; k < gt.size(); ++k) {
      gt[k] = at[Bm.bindex[Bm.tri[k]]];
      ++aptr[gt[k] + 1];
    }
    for (int i = 0; i < nb; ++i) aptr[i + 1] += aptr[i];
    std::vector<int2> adj(gt.size());
    std::vector<int> fill(aptr.begin(), aptr.end() - 1);
    for (int t = 0; t < nt; ++t)
      for (int k = 0; k < 3; ++k) adj[fill[gt[size_t(3) * t + k]]++] = make_int2(t, k);
    H.from_mesh = true;
    H.ntri = nt;
    H.gx.upload(gx, st);
    H.gsolid.upload(gs, st);
    H.gtri.upload(gt, st);
    H.gadj_ptr.upload(aptr, st);
    H.gadj.upload(adj, st);
    H.garea.upload(Bm.tri_area, st);
    H.gnrm.upload(Bm.tri_normal, st);
  }
  const HSource src = h_source();
  H.hnearb = nearb;
  H.hfarb = farb;
  H.nearb.upload(nearb, st);
  H.rows.upload(rows, st);
  H.farb.upload(farb, st);
  H.D64.alloc(size_t(doff));
  H.D32.alloc(size_t(doff));
  if (mesh) launch_h_near_mesh(H.nnear, H.nearb.p, src, H.D64.p, H.D32.p, st);
  else launch_h_near_gather(H.nnear, H.nearb.p, src, H.D64.p, H.D32.p, st);
  // matrix-relative accuracy: the entry scale share * ||N||_F / Nb from the dense leaf tiles N
  // (the near field, which holds the diagonal and dominates the matrix's norm); the tiles' sums
  // of squares are added in partition order, so the scale does not depend on the thread count
  h_gscale = 0.0;
  if (h_share > 0.0 && doff > 0) {
    std::vector<double> tiles(static_cast<size_t>(doff));
    TMB_CUDA(cudaMemcpyAsync(tiles.data(), H.D64.p, sizeof(double) * tiles.size(), cudaMemcpyDeviceToHost, st));
    sync();
    std::vector<double> part(nearb.size(), 0.0);
#pragma omp parallel for schedule(dynamic, 64)
    for (long long q = 0; q < (long long)nearb.size(); ++q) {
      const HBlockDev& b = nearb[size_t(q)];
      double a = 0.0;
      for (long long t = 0; t < (long long)b.m * b.n; ++t) a += tiles[size_t(b.off + t)] * tiles[size_t(b.off + t)];
      part[size_t(q)] = a;
    }
    double ss = 0.0;
    for (double a : part) ss += a;
    h_gscale = h_share * std::sqrt(ss) / double(nb);
  }
  // adaptive cross approximation of every admissible block
  std::vector<int> ranks(size_t(3) * H.nfar, 0);
  if (H.nfar > 0) {
    DevArray<double> Us, Vs;
    DevArray<unsigned char> used;
    DevArray<int> dr;
    Us.alloc(size_t(us));
    Vs.alloc(size_t(vs));
    used.alloc(size_t(fl));
    dr.alloc(size_t(3) * H.nfar);
    launch_h_aca(H.nfar, H.farb.p, src, Us.p, Vs.p, used.p, kmax, eps_fp64, eps_mixed, h_gscale, dr.p, st);
    TMB_CUDA(cudaMemcpyAsync(ranks.data(), dr.p, sizeof(int) * ranks.size(), cudaMemcpyDeviceToHost, st));
    sync();
    for (int w = 0; w < 2; ++w) {
      std::vector<int> rk(H.nfar);
      std::vector<long long> uo(H.nfar), vo(H.nfar);
      long long su = 0, sv = 0, stt = 0;
      std::vector<long long> to(size_t(H.nfar) + 1);
      std::vector<HTerm> td;
      for (int q = 0; q < H.nfar; ++q) {
        rk[q] = ranks[size_t(3) * q + w];
        uo[q] = su;
        vo[q] = sv;
        to[q] = stt;
        const int np = pad4(farb[q].n), mp = pad4(farb[q].m);
        for (int l = 0; l < rk[q]; ++l)
          td.push_back(HTerm{sv + (long long)l * np, su + (long long)l * mp, np, farb[q].cb});
        su += (long long)rk[q] * pad4(farb[q].m);
        sv += (long long)rk[q] * np;
        stt += rk[q];
      }
      to[H.nfar] = stt;
      H.toff[w].upload(to, st);
      H.termd[w].upload(td, st);
      // matvec work items: the admissible blocks of one row cluster, cut into runs of about
      // wmax U + V entries (about 64 items per SM), largest first
      double total = 0.0;
      for (int q = 0; q < H.nfar; ++q) total += double(rk[q]) * (farb[q].m + farb[q].n);
      const double wmax = std::max(4096.0, total / (64.0 * num_sms));
      std::vector<HFarGroup> items;
      std::vector<double> work;
      for (const HFarGroup& g : groups) {
        HFarGroup it{g.rb, g.m, g.first, g.first};
        double wk = 0.0;
        for (int q = g.first; q < g.last; ++q) {
          const double wq = double(rk[q]) * (farb[q].m + farb[q].n);
          if (wk > 0.0 && wk + wq > wmax) {
            items.push_back(it);
            work.push_back(wk);
            it.first = q;
            wk = 0.0;
          }
          it.last = q + 1;
          wk += wq;
        }
        if (wk > 0.0) {
          items.push_back(it);
          work.push_back(wk);
        }
      }
      std::vector<int> order(items.size());
      std::iota(order.begin(), order.end(), 0);
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
      std::vector<HFarGroup> sorted;
      for (int g : order) sorted.push_back(items[g]);
      H.ngroups[w] = int(sorted.size());
      H.groups[w].upload(sorted, st);
      H.terms[w] = stt;
      H.rank[w].upload(rk, st);
      H.uoff[w].upload(uo, st);
      H.voff[w].upload(vo, st);
      if (w == 0) {
        H.huoff = uo;
        H.hvoff = vo;
        H.hrank = rk;
        H.hsu = su;
        H.hsv = sv;
        H.U64.alloc(size_t(std::max(su, 1LL)));
        H.V64.alloc(size_t(std::max(sv, 1LL)));
        launch_h_compact<double>(H.nfar, H.farb.p, Us.p, Vs.p, H.uoff[0].p, H.voff[0].p, H.rank[0].p, H.U64.p,
                                 H.V64.p, st);
      } else {
        H.U32.alloc(size_t(std::max(su, 1LL)));
        H.V32.alloc(size_t(std::max(sv, 1LL)));
        launch_h_compact<float>(H.nfar, H.farb.p, Us.p, Vs.p, H.uoff[1].p, H.voff[1].p, H.rank[1].p, H.U32.p,
                                H.V32.p, st);
      }
      H.bytes[w] = double(doff) * (w == 0 ? 8 : 4) + double(su + sv) * (w == 0 ? 8 : 4) +
                   double(H.nnear + H.nfar) * sizeof(HBlockDev);
    }
    sync();
  } else {
    H.bytes[0] = double(doff) * 8;
    H.bytes[1] = double(doff) * 4;
  }
  for (int q = 0; q < H.nfar; ++q) {
    H.failed += ranks[size_t(3) * q + 2] != 0;
    H.max_rank = std::max(H.max_rank, ranks[size_t(3) * q]);
  }
  H.ranks = ranks;
  H.part = std::move(P);
  H.y.alloc(nb);
  // four zero entries past the end: the padded tail of a V row meets them
  H.xp64.alloc(size_t(nb) + 4);
  H.xp32.alloc(size_t(nb) + 4);
  H.xp64.zero(st);
  H.xp32.zero(st);
  H.tval.alloc(size_t(std::max(std::max(H.terms[0], H.terms[1]), 1LL)));
  H.built = true;
  bem_mode = 1;
  if (mesh) has_bem = true;
  if (!keep_dense) {
    Bd.reset();
    Bf.reset();
  }
  H.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// H2 recompression of the hierarchical matrix's admissible blocks (FP64 factors), once per
// precision: eps_fp64 for the plain path, eps_mixed for the mixed path (stored in FP32).
void Ctx::h2_build(double eps_fp64, double eps_mixed, int kmax) {
  if (!H.built) throw Error(TMB_ERR_STATE, "tmb_bem_h2: no hierarchical matrix built");
  if (!(eps_fp64 > 0.0) || !(eps_mixed > 0.0) || kmax < 1 || kmax > 64)
    throw Error(TMB_ERR_ARG, "tmb_bem_h2: tolerances must be positive, rank cap in 1..64");
  cudaStream_t st = stream;
  const HPartition& P = H.part;
  const int nf = int(P.far.size());
  // the FP64 factors on the host
  std::vector<double> hU(size_t(std::max(H.hsu, 1LL))), hV(size_t(std::max(H.hsv, 1LL)));
  if (nf > 0) {
    TMB_CUDA(cudaMemcpyAsync(hU.data(), H.U64.p, sizeof(double) * size_t(H.hsu), cudaMemcpyDeviceToHost, st));
    TMB_CUDA(cudaMemcpyAsync(hV.data(), H.V64.p, sizeof(double) * size_t(H.hsv), cudaMemcpyDeviceToHost, st));
    sync();
  }
  H2Factors F;
  F.U.resize(nf);
  F.V.resize(nf);
  F.ldu.resize(nf);
  F.ldv.resize(nf);
  F.rank = H.hrank;
  for (int q = 0; q < nf; ++q) {
    const HCluster& ct = P.clusters[P.far[q].first];
    const HCluster& cs = P.clusters[P.far[q].second];
    F.U[q] = hU.data() + H.huoff[q];
    F.V[q] = hV.data() + H.hvoff[q];
    F.ldu[q] = pad4(ct.end - ct.begin);
    F.ldv[q] = pad4(cs.end - cs.begin);
  }
  const size_t nc = P.clusters.size();
  // depth of every cluster, leaves, non-leaf clusters by depth
  std::vector<int> depth(nc, 0), parent(nc, -1);
  for (size_t c = 0; c < nc; ++c)
    for (int ch : P.clusters[c].child)
      if (ch >= 0) parent[ch] = int(c);
  std::vector<int> order{0};
  for (size_t i = 0; i < order.size(); ++i)
    for (int ch : P.clusters[order[i]].child)
      if (ch >= 0) {
        depth[ch] = depth[order[i]] + 1;
        order.push_back(ch);
      }
  const int maxd = *std::max_element(depth.begin(), depth.end());
  std::vector<int> leaves;
  std::vector<std::vector<int>> bydepth(maxd + 1);
  for (size_t c = 0; c < nc; ++c) {
    if (P.clusters[c].child[0] < 0) leaves.push_back(int(c));
    else bydepth[depth[c]].push_back(int(c));
  }
  for (int w = 0; w < 2; ++w) {
    const auto t0 = std::chrono::steady_clock::now();
    H2Host Hh;
    h2_build_host(P, F, w == 0 ? eps_fp64 : eps_mixed, kmax, Hh);
    H2Mat& M = H2[w];
    M = H2Mat{};
    M.eps = w == 0 ? eps_fp64 : eps_mixed;
    std::vector<H2Node> nodes(nc);
    std::vector<double> rowb, colb, S;
    int xo = 0, yo = 0;
    for (size_t c = 0; c < nc; ++c) {
      const HCluster& C = P.clusters[c];
      H2Node& d = nodes[c];
      d.begin = C.begin;
      d.m = C.end - C.begin;
      d.kr = Hh.row.k[c];
      d.kc = Hh.col.k[c];
      d.parent = parent[c];
      d.child0 = C.child[0];
      d.child1 = C.child[1];
      d.xo = xo;
      d.yo = yo;
      xo += d.kc;
      yo += d.kr;
      M.max_kr = std::max(M.max_kr, d.kr);
      M.max_kc = std::max(M.max_kc, d.kc);
      d.rl = d.rt = d.cl = d.ct = -1;
      if (C.child[0] < 0) {
        d.rl = (long long)rowb.size();
        rowb.insert(rowb.end(), Hh.row.leaf_basis[c].begin(), Hh.row.leaf_basis[c].end());   // m x kr col-major
        d.cl = (long long)colb.size();
        const std::vector<double>& Wc = Hh.col.leaf_basis[c];                                  // m x kc col-major
        for (int i = 0; i < d.m; ++i)
          for (int j = 0; j < d.kc; ++j) colb.push_back(Wc[i + size_t(j) * d.m]);              // -> row-major
      }
      if (parent[c] >= 0) {
        d.rt = (long long)rowb.size();
        rowb.insert(rowb.end(), Hh.row.transfer[c].begin(), Hh.row.transfer[c].end());       // kr x kr_p
        d.ct = (long long)colb.size();
        const int kp = Hh.col.k[parent[c]];
        const std::vector<double>& Fc = Hh.col.transfer[c];                                    // kc x kp col-major
        for (int i = 0; i < d.kc; ++i)
          for (int j = 0; j < kp; ++j) colb.push_back(Fc[i + size_t(j) * d.kc]);              // -> kp x kc col-major
      }
    }
    M.ncoef_c = xo;
    M.ncoef_r = yo;
    std::vector<H2Run> runs;
    std::vector<H2Blk> blks(nf);
    for (int q = 0; q < nf; ++q) {
      blks[q].s = P.far[q].second;
      blks[q].so = (long long)S.size();
      S.insert(S.end(), Hh.coupling[q].begin(), Hh.coupling[q].end());
      if (runs.empty() || runs.back().t != P.far[q].first) runs.push_back(H2Run{P.far[q].first, q, q + 1});
      else runs.back().last = q + 1;
    }
    std::vector<int> lvl;
    for (int dd = maxd; dd >= 0; --dd) {           // upward: deepest first
      int cnt = 0;
      for (int c : bydepth[dd]) cnt += nodes[c].kc > 0;
      if (cnt > 0) M.up.emplace_back(int(lvl.size()), int(bydepth[dd].size()));
      if (cnt > 0) lvl.insert(lvl.end(), bydepth[dd].begin(), bydepth[dd].end());
    }
    for (int dd = 1; dd <= maxd; ++dd) {           // downward: root first
      int cnt = 0;
      for (int c : bydepth[dd]) cnt += nodes[c].kr > 0 && nodes[parent[c]].kr > 0;
      if (cnt > 0) M.down.emplace_back(int(lvl.size()), int(bydepth[dd].size()));
      if (cnt > 0) lvl.insert(lvl.end(), bydepth[dd].begin(), bydepth[dd].end());
    }
    M.nleaf = int(leaves.size());
    M.nruns = int(runs.size());
    M.nlevels = maxd + 1;
    M.node.upload(nodes, st);
    M.leaves.upload(leaves, st);
    M.lvl_nodes.upload(lvl, st);
    M.runs.upload(runs, st);
    M.blk.upload(blks, st);
    {
      std::vector<int> br(nf);
      for (int q = 0; q < nf; ++q) br[q] = P.far[q].first;
      M.brow.upload(br, st);
    }
    M.xh.alloc(size_t(std::max(xo, 1)));
    M.yh.alloc(size_t(std::max(yo, 1)));
    const double vs = w == 0 ? 8.0 : 4.0;
    if (w == 0) {
      M.rowb64.upload(rowb, st);
      M.colb64.upload(colb, st);
      M.S64.upload(S, st);
    } else {
      std::vector<float> r(rowb.begin(), rowb.end()), c2(colb.begin(), colb.end()), s2(S.begin(), S.end());
      M.rowb32.upload(r, st);
      M.colb32.upload(c2, st);
      M.S32.upload(s2, st);
    }
    M.coupling_bytes = double(S.size()) * vs;
    M.basis_bytes = double(rowb.size() + colb.size()) * vs;
    const double near_bytes = H.bytes[w] > 0 ? double(H.D64.n) * vs : 0.0;
    M.bytes = near_bytes + M.coupling_bytes + M.basis_bytes + double(nc) * sizeof(H2Node) +
              double(nf) * sizeof(H2Blk) + double(runs.size()) * sizeof(H2Run) + 16.0 * (xo + yo);
    sync();
    M.built = true;
    M.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  bem_mode = 2;
}

template <typename T>
H2View<T> Ctx::h2_view(int w) const {
  const H2Mat& M = H2[w];
  H2View<T> v;
  v.nb = nb;
  v.nleaf = M.nleaf;
  v.nruns = M.nruns;
  v.gidx = H.gidx.p;
  v.nrows = H.nrows;
  v.near_rows = H.rows.p;
  v.near = H.nearb.p;
  v.node = M.node.p;
  v.leaves = M.leaves.p;
  v.lvl_nodes = M.lvl_nodes.p;
  v.runs = M.runs.p;
  v.nblk = int(M.blk.n);
  v.brow = M.brow.p;
  v.blk = M.blk.p;
  v.xh = const_cast<double*>(M.xh.p);
  v.yh = const_cast<double*>(M.yh.p);
  v.nyh = M.ncoef_r;
  if constexpr (sizeof(T) == 8) {
    v.D = H.D64.p;
    v.rowb = M.rowb64.p;
    v.colb = M.colb64.p;
    v.S = M.S64.p;
  } else {
    v.D = H.D32.p;
    v.rowb = M.rowb32.p;
    v.colb = M.colb32.p;
    v.S = M.S32.p;
  }
  return v;
}

HSource Ctx::h_source() const {
  HSource s;
  s.nb = nb;
  s.perm = H.perm.p;
  if (H.from_mesh) {
    s.ntri = H.ntri;
    s.xp = H.gx.p;
    s.tri = H.gtri.p;
    s.tarea = H.garea.p;
    s.tnrm = H.gnrm.p;
    s.adj_ptr = H.gadj_ptr.p;
    s.adj = H.gadj.p;
    s.solid = H.gsolid.p;
  } else {
    s.B = Bd.p;
    s.ld = bem_ld(nb);
  }
  return s;
}

// Accuracy of the low-rank blocks against the entries they were built from (the dense FP64
// matrix, which must still be on the device, or the boundary mesh) for a fixed probe vector.  out = {relative error of the far part, FP64 terms; same,
// FP32 terms; worst block relative error, FP64; same, FP32}; block_out (may be null) holds per
// block {|A x|, |A x - U64 V64^T x|, |A x - U32 V32^T x|, tight rank, loose rank, rank-cap status}.
void Ctx::h_verify(double* block_out, double* out) {
  if (!H.built) throw Error(TMB_ERR_STATE, "tmb_bem_verify: no hierarchical matrix");
  if (!H.from_mesh && !Bd.p)
    throw Error(TMB_ERR_STATE, "tmb_bem_verify: the dense FP64 matrix was released (keep_dense = 0)");
  for (int q = 0; q < 4; ++q) out[q] = 0.0;
  if (H.nfar == 0) return;
  DevArray<double> e;
  e.alloc(size_t(3) * H.nfar);
  launch_h_verify(H.nfar, H.farb.p, h_source(), H.rank[0].p, H.uoff[0].p, H.voff[0].p, H.U64.p,
                  H.V64.p, H.rank[1].p, H.uoff[1].p, H.voff[1].p, H.U32.p, H.V32.p, e.p, stream);
  std::vector<double> h(size_t(3) * H.nfar);
  TMB_CUDA(cudaMemcpyAsync(h.data(), e.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream));
  sync();
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int q = 0; q < H.nfar; ++q) {
    const double a = h[3 * q], b = h[3 * q + 1], c = h[3 * q + 2];
    s0 += a;
    s1 += b;
    s2 += c;
    if (a > 0.0) {
      out[2] = std::max(out[2], std::sqrt(b / a));
      out[3] = std::max(out[3], std::sqrt(c / a));
    }
    if (block_out) {
      double* o = block_out + size_t(6) * q;
      o[0] = std::sqrt(a);
      o[1] = std::sqrt(b);
      o[2] = std::sqrt(c);
      o[3] = H.ranks[size_t(3) * q];
      o[4] = H.ranks[size_t(3) * q + 1];
      o[5] = H.ranks[size_t(3) * q + 2];
    }
  }
  if (s0 > 0.0) {
    out[0] = std::sqrt(s1 / s0);
    out[1] = std::sqrt(s2 / s0);
  }
}

// Interfacial-DMI per-node factors (D_j, D_i / Js_i, 1 / (V_i Js_i)) when that form is selected.
void Ctx::upload_dmi() {
  if (dmi_kind != 1 || !has_dmi) {
    idm_d.reset();
    idm_a.reset();
    idm_b.reset();
    return;
  }
  std::vector<double> a(n), b(n);
  for (int i = 0; i < n; ++i) {
    a[i] = hD[i] * hij[i];
    b[i] = hij[i] / hvol[i];
  }
  idm_d.upload(hD, stream);
  idm_a.upload(a, stream);
  idm_b.upload(b, stream);
  sync();
}

// Device arrays of the cubic / surface anisotropy for the current material (Js).
void Ctx::upload_extra() {
  cudaStream_t st = stream;
  has_cub = !hKc1.empty();
  has_srf = !hKs.empty();
  if (has_cub) {
    std::vector<double> k1(n), k2(n), ax(size_t(9) * n);
    for (int i = 0; i < n; ++i) {
      const double ij = hij.empty() ? 0.0 : hij[i];
      k1[i] = hKc1[i] * ij;
      k2[i] = hKc2[i] * ij;
      for (int q = 0; q < 9; ++q) ax[size_t(q) * n + i] = hcax[size_t(9) * i + q];
    }
    cub_k1.upload(k1, st);
    cub_k2.upload(k2, st);
    cub_ax.upload(ax, st);
    kc1_raw.upload(hKc1, st);
    kc2_raw.upload(hKc2, st);
  }
  if (has_srf) {
    std::vector<double> ks(n), ksa(n);
    for (int i = 0; i < n; ++i) {
      const double ij = hij.empty() ? 0.0 : hij[i];
      ksa[i] = hKs[i] * harea[i];
      ks[i] = ksa[i] / hvol[i] * ij;
    }
    srf_k.upload(ks, st);
    ksa_raw.upload(ksa, st);
  }
  sync();
}

LocalFieldArgs Ctx::local_args(const double* m, double* ydot, double* hout, unsigned long long* tq) const {
  LocalFieldArgs a;
  std::memset(static_cast<void*>(&a), 0, sizeof a);   // padding too: the step graphs compare these bytes
  a.n = n;
  a.m = m;
  a.hfix = hfix.p;
  a.xc = xc.p;
  a.ku2 = has_uni ? ku2.p : nullptr;
  a.kax = kax.p;
  const bool idmi = has_dmi && dmi_kind == 1;
  a.dmi_s = (has_dmi && !idmi) ? dmi_s.p : nullptr;
  a.area = area.p;
  a.nvn = nvn.p;
  a.idm_d = idmi ? idm_d.p : nullptr;
  a.idm_a = idmi ? idm_a.p : nullptr;
  a.idm_b = idmi ? idm_b.p : nullptr;
  a.cub_k1 = has_cub ? cub_k1.p : nullptr;
  a.cub_k2 = cub_k2.p;
  a.cub_ax = cub_ax.p;
  a.srf_k = has_srf ? srf_k.p : nullptr;
  a.alpha = alpha;
  a.precession = precession;
  a.ydot = ydot;
  a.hout = hout;
  a.torque_bits = tq;
  return a;
}

// Divergence (sum_d tGrad_d (js m_d) scale) and gradient (-grad u) on the shared pattern, from the
// dictionary-coded operators when they exist, else from the precision's value arrays.
void Ctx::launch_div(const double* m, const double* js_, double scale, double* out, cudaStream_t st) {
  SellView S = pat.view(rep);
  if (tg_coded) {
    S.tab = tgtab.p;
    launch_divergence<uint8_t>(S, tgq[0].p, tgq[1].p, tgq[2].p, m, js_, scale, out, st);
  } else if (precision == TMB_FP64) {
    launch_divergence<double>(S, tg[0].p, tg[1].p, tg[2].p, m, js_, scale, out, st);
  } else {
    launch_divergence<float>(S, tgf[0].p, tgf[1].p, tgf[2].p, m, js_, scale, out, st);
  }
}
void Ctx::launch_grad(const double* u1, const double* u2, const double* he, double* hd, double* hf,
                      cudaStream_t st) {
  SellView S = pat.view(rep);
  if (g_coded) {
    S.tab = gtab.p;
    launch_gradient<uint8_t>(S, gq[0].p, gq[1].p, gq[2].p, u1, u2, he, hd, hf, st);
  } else if (precision == TMB_FP64) {
    launch_gradient<double>(S, g[0].p, g[1].p, g[2].p, u1, u2, he, hd, hf, st);
  } else {
    launch_gradient<float>(S, gf[0].p, gf[1].p, gf[2].p, u1, u2, he, hd, hf, st);
  }
}

// The local-field kernel on the shared pattern, or on K's own non-zero pattern when no DMI term
// needs the gradient operators (the same sums: the dropped entries are exact zeros).
void Ctx::launch_local_kernel(const LocalFieldArgs& a, cudaStream_t st) {
  const bool compact = has_patx && !a.idm_a && !a.dmi_s;
  const SellView S = compact ? patx.view(rep) : pat.view(rep);
  if (precision == TMB_FP64)
    launch_local_field<double>(S, compact ? Kx.p : K.p, tg[0].p, tg[1].p, tg[2].p, g[0].p, g[1].p, a, st);
  else
    launch_local_field<float>(S, compact ? Kxf.p : Kf.p, tgf[0].p, tgf[1].p, tgf[2].p, gf[0].p, gf[1].p, a, st);
}

void Ctx::launch_local(const LocalFieldArgs& a, cudaStream_t st) {
  const SellView S = pat.view(rep);
  launch_local_kernel(a, st);
  if (has_stt && a.ydot) {
    if (precision == TMB_FP64)
      launch_stt_add<double>(S, g[0].p, g[1].p, g[2].p, a.m, stt_eta.p, alpha, stt_beta, stt_scale, a.ydot, st);
    else
      launch_stt_add<float>(S, gf[0].p, gf[1].p, gf[2].p, a.m, stt_eta.p, alpha, stt_beta, stt_scale, a.ydot, st);
  }
}

void Ctx::local(const double* m, double* ydot, double* hout, unsigned long long* tq) {
  require_mesh();
  require_material();
  const LocalFieldArgs a = local_args(m, ydot, hout, tq);
  const double sv = precision == TMB_FP64 ? 8.0 : 4.0, z = double(hptr[n]), N = double(nr());
  const double zx = (has_patx && !a.idm_a && !a.dmi_s) ? double(nnz_x) : z;  // entries of K read
  double bytes = zx * (sv + 4) + N * 8 * (3 + 3 + 1) + (ydot ? N * 24 : 0.0) + (hout ? N * 24 : 0.0);
  if (a.ku2) bytes += N * 8 * 4;
  if (a.dmi_s) bytes += z * 3 * sv + N * 8 * 5;
  if (a.idm_a) bytes += z * 4 * sv + N * 8 * 3;
  prof.begin(0, stream, bytes);
  launch_local(a, stream);
  prof.end(stream);
}

// Energy densities of TheSimulation::calculateEnergies (main/TheSimulation.cpp:385-396): demag
// (DemagField::getDemagEnergy, main/DemagField.cpp:97-99), exchange (calcExchangeEnergy,
// main/EffFieldCalc.cpp:65-69), uniaxial with its offset (uniaxialEnergy, :86-95), Zeeman
// (TheLLG::getZeemanEnergy, main/TheLLG.cpp:345-348), cubic (cubicAnisotropyEnergy, :232-247),
// surface with its offset (surfaceAnisotropyEnergy, :108-126), DMI (-1/2 sum V H_dmi . m), each
// divided by the total volume.  out = {total, demag, exchange, uniaxial, Zeeman, cubic, surface,
// DMI}.  The demag field is evaluated for m when a BEM matrix is set (else the frozen one is
// used).  With components or replicas the sums run over the whole batch.
void Ctx::energies(const double* m, double* out) {
  require_mesh();
  require_material();
  cudaStream_t st = stream;
  const size_t n3 = size_t(3) * nr();
  if (has_bem) demag(m);
  for (auto& b : ebuf) b.alloc(n3);
  // exchange alone, then exchange + DMI: the DMI field is the difference
  LocalFieldArgs a = local_args(m, nullptr, ebuf[0].p, nullptr);
  a.hfix = nullptr;
  a.ku2 = nullptr;
  a.dmi_s = nullptr;
  a.idm_a = a.idm_b = a.idm_d = nullptr;
  a.cub_k1 = nullptr;
  a.srf_k = nullptr;
  launch_local(a, st);
  const double* hdmi = nullptr;
  if (has_dmi) {
    LocalFieldArgs b = local_args(m, nullptr, ebuf[1].p, nullptr);
    b.hfix = nullptr;
    b.ku2 = nullptr;
    b.cub_k1 = nullptr;
    b.srf_k = nullptr;
    launch_local(b, st);
    launch_lincomb(int(n3), ebuf[1].p, 1.0, ebuf[1].p, -1.0, ebuf[0].p, 0.0, nullptr, st);
    hdmi = ebuf[1].p;
  }
  const int nblk = energy_blocks(n, rep);
  epart.alloc(size_t(kEnergyTerms) * nblk);
  EnergyExtra ex;
  if (has_cub) {
    ex.kc1 = kc1_raw.p;
    ex.kc2 = kc2_raw.p;
    ex.cax = cub_ax.p;
  }
  if (has_srf) {
    ex.ksa = ksa_raw.p;
    ex.nvn = nvn.p;
  }
  launch_energy_terms(n, rep, m, ebuf[0].p, hdmi, hext.p, hdem.p, js.p, node_vol.p, has_uni ? ku2.p : nullptr,
                      kax.p, ex, epart.p, st);
  std::vector<double> h(size_t(kEnergyTerms) * nblk);
  TMB_CUDA(cudaMemcpyAsync(h.data(), epart.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  sync();
  double sum[kEnergyTerms] = {0, 0, 0, 0, 0, 0, 0};
  for (int b = 0; b < nblk; ++b)
    for (int q = 0; q < kEnergyTerms; ++q) sum[q] += h[size_t(kEnergyTerms) * b + q];
  double vtot = 0.0, ku_vol = 0.0, ks_off = 0.0;
  for (int i = 0; i < n; ++i) vtot += hvol[i];
  if (has_uni) {
    std::vector<double> k2(n);
    TMB_CUDA(cudaMemcpy(k2.data(), ku2.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i) ku_vol += hvol[i] * 0.5 * k2[i] / (hij[i] != 0.0 ? hij[i] : 1.0);
  }
  if (has_srf)
    for (int i = 0; i < n; ++i) ks_off += hKs[i] * harea[i];  // EffFieldCalc::setSurfaceAnisotropy
  vtot *= rep;
  ku_vol *= rep;
  ks_off *= rep;
  const double e_dem = -0.5 * sum[4] / vtot, e_ex = -0.5 * sum[0] / vtot, e_uni = (ku_vol - sum[2]) / vtot;
  const double e_zee = -sum[3] / vtot, e_dmi = -0.5 * sum[1] / vtot;
  const double e_cub = sum[5] / vtot, e_srf = has_srf ? (ks_off - sum[6]) / vtot : 0.0;
  out[0] = e_dem + e_ex + e_uni + e_zee + e_dmi + e_cub + e_srf;
  out[1] = e_dem;
  out[2] = e_ex;
  out[3] = e_uni;
  out[4] = e_zee;
  out[5] = e_cub;
  out[6] = e_srf;
  out[7] = e_dmi;
}

static double bits_to_double(unsigned long long b) {
  double d;
  std::memcpy(&d, &b, sizeof d);
  return d;
}

double Ctx::max_torque(const double* m) {
  TMB_CUDA(cudaMemsetAsync(bits.p, 0, sizeof(unsigned long long), stream));
  local(m, nullptr, nullptr, bits.p);
  TMB_CUDA(cudaMemcpyAsync(bits_h, bits.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
  sync();
  return bits_to_double(bits_h[0]) * kMu0;
}

// Dormand & Prince (1980) 5(4) tableau; the stage-7 input is the 5th-order solution (FSAL).
static const double kDpA[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {1.0 / 5, 0, 0, 0, 0, 0},
    {3.0 / 40, 9.0 / 40, 0, 0, 0, 0},
    {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0, 0},
    {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0, 0},
    {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656, 0},
    {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}};
static const double kDpE[7] = {35.0 / 384 - 5179.0 / 57600, 0.0, 500.0 / 1113 - 7571.0 / 16695,
                               125.0 / 192 - 393.0 / 640, -2187.0 / 6784 + 92097.0 / 339200,
                               11.0 / 84 - 187.0 / 2100, -1.0 / 40};

// Adaptive segment with odeint's controlled_runge_kutta error control and step adjustment.
int Ctx::integrate_segment(double*& y, double*& yalt, double t0, double t1, double& dt, double eps_abs,
                           double eps_rel, double* stats) {
  const int n3 = 3 * nr();
  cudaStream_t st = stream;
  double t = t0;
  local(y, kst[0].p, nullptr, nullptr);
  stats[2] += 1;
  const long long max_steps = 50000000LL;
  long long steps = 0;
  while (t < t1) {
    if (++steps > max_steps) throw Error(TMB_ERR_STEP, "integrator step cap reached");
    bool last = false;
    double h = dt;
    if (t + h >= t1) {
      h = t1 - t;
      last = true;
    }
    if (!(h > 0.0) || h < 1e-300) throw Error(TMB_ERR_STEP, "integrator step size underflow");
    const double* kp[7];
    for (int j = 0; j < 7; ++j) kp[j] = kst[j].p;
    for (int s = 1; s < 7; ++s) {
      double* dst = (s == 6) ? yalt : ytmp.p;
      launch_rk_combine(n3, y, kp, kDpA[s], s, h, dst, st);
      local(dst, kst[s].p, nullptr, nullptr);
      stats[2] += 1;
    }
    TMB_CUDA(cudaMemsetAsync(bits.p + 1, 0, sizeof(unsigned long long), st));
    launch_rk_error(n3, y, kst[0].p, kp, kDpE, 7, h, eps_abs, eps_rel, bits.p + 1, st);
    TMB_CUDA(cudaMemcpyAsync(bits_h + 1, bits.p + 1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    sync();
    const double err = bits_to_double(bits_h[1]);
    if (!std::isfinite(err) || err > 1.0) {
      const double e = std::isfinite(err) ? err : 1e30;
      dt = h * std::max(0.9 * std::pow(e, -1.0 / 3.0), 0.2);
      stats[1] += 1;
      continue;
    }
    t = last ? t1 : t + h;
    std::swap(y, yalt);
    kst[0].swap(kst[6]);
    stats[0] += 1;
    const double dtn = (err < 0.5) ? h * 0.9 * std::pow(std::max(err, std::pow(5.0, -5.0)), -1.0 / 5.0) : h;
    if (!last) dt = dtn;
    else dt = (h < dt) ? std::max(dt, dtn) : dtn;
  }
  return TMB_OK;
}

// Signature of what a captured step graph depends on: buffers, precision, the local field's
// arguments (material arrays, DMI form, extra terms) and the spin-transfer term.
static void push_bytes(std::vector<unsigned char>& v, const void* p, size_t n) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  v.insert(v.end(), b, b + n);
}

cudaGraphExec_t Ctx::step_graph_for(double* y, double* yalt) {
  const int n3 = 3 * nr();
  std::vector<unsigned char> sig;
  LocalFieldArgs a = local_args(ytmp.p, kst[1].p, nullptr, nullptr);
  push_bytes(sig, &a, sizeof a);
  const void* ptrs[] = {y, yalt, ytmp.p, kst[0].p, kst[1].p, kst[2].p, kst[3].p, kst[4].p, kst[5].p, kst[6].p,
                        ctl_d, stt_eta.p, pat.soff.p, K.p, Kf.p, patx.soff.p, Kx.p, Kxf.p};
  push_bytes(sig, ptrs, sizeof ptrs);
  const double vals[] = {double(n3), double(precision), double(has_stt), stt_beta, stt_scale, alpha};
  push_bytes(sig, vals, sizeof vals);
  const int w = precision == TMB_FP64 ? 0 : 1;
  if (step_graph[w] && step_sig[w] == sig) return step_graph[w];
  if (step_graph[w]) {
    cudaGraphExecDestroy(step_graph[w]);
    step_graph[w] = nullptr;
  }
  cudaStream_t st = stream;
  cudaGraph_t graph = nullptr;
  const long long before = launch_count();
  TMB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    const double* kp[7];
    for (int j = 0; j < 7; ++j) kp[j] = kst[j].p;
    for (int q = 0; q < kStepAttempts; ++q) {
      launch_step_begin(ctl_d, st);
      for (int s = 1; s < 7; ++s) {
        double* dst = (s == 6) ? yalt : ytmp.p;
        launch_rk_combine_dev(n3, y, kp, kDpA[s], s, ctl_d, dst, st);
        LocalFieldArgs la = local_args(dst, kst[s].p, nullptr, nullptr);
        la.active = &ctl_d->active;
        const SellView S = pat.view(rep);
        launch_local_kernel(la, st);
        if (has_stt) {
          if (precision == TMB_FP64)
            launch_stt_add<double>(S, g[0].p, g[1].p, g[2].p, dst, stt_eta.p, alpha, stt_beta, stt_scale, kst[s].p,
                                   st, &ctl_d->active);
          else
            launch_stt_add<float>(S, gf[0].p, gf[1].p, gf[2].p, dst, stt_eta.p, alpha, stt_beta, stt_scale,
                                  kst[s].p, st, &ctl_d->active);
        }
      }
      launch_rk_error_dev(n3, y, kst[0].p, kp, kDpE, 7, ctl_d, st);
      launch_step_accept(n3, ctl_d, y, yalt, kst[0].p, kst[6].p, st);
      launch_step_update(ctl_d, 6, st);
    }
  } catch (...) {
    cudaStreamEndCapture(st, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  TMB_CUDA(cudaStreamEndCapture(st, &graph));
  step_nodes = launch_count() - before;
  note_launches(-step_nodes);  // captured, not launched
  const cudaError_t e = cudaGraphInstantiate(&step_graph[w], graph, 0);
  cudaGraphDestroy(graph);
  TMB_CUDA(e);
  step_sig[w] = sig;
  return step_graph[w];
}

void Ctx::integrate_segment_dev(double* y, double* yalt, double t0, double t1, double& dt, double eps_abs,
                                double eps_rel, double* stats) {
  cudaStream_t st = stream;
  if (!ctl_d) TMB_CUDA(cudaMalloc(&ctl_d, sizeof(StepCtl)));
  if (!ctl_h) TMB_CUDA(cudaMallocHost(&ctl_h, sizeof(StepCtl)));
  local(y, kst[0].p, nullptr, nullptr);   // first same as last: k1 of the first attempt
  stats[2] += 1;
  std::memset(ctl_h, 0, sizeof(StepCtl));
  ctl_h->t = t0;
  ctl_h->t1 = t1;
  ctl_h->dt = dt;
  ctl_h->eps_abs = eps_abs;
  ctl_h->eps_rel = eps_rel;
  ctl_h->max_attempts = 50000000LL;
  TMB_CUDA(cudaMemcpyAsync(ctl_d, ctl_h, sizeof(StepCtl), cudaMemcpyHostToDevice, st));
  cudaGraphExec_t gx = step_graph_for(y, yalt);
  for (;;) {
    TMB_CUDA(cudaGraphLaunch(gx, st));
    note_launches(step_nodes);
    TMB_CUDA(cudaMemcpyAsync(ctl_h, ctl_d, sizeof(StepCtl), cudaMemcpyDeviceToHost, st));
    sync();
    if (ctl_h->done) break;
  }
  if (ctl_h->status != 0) throw Error(TMB_ERR_STEP, "integrator step size underflow or step cap");
  stats[0] += double(ctl_h->accepted);
  stats[1] += double(ctl_h->rejected);
  stats[2] += double(ctl_h->rhs);
  dt = ctl_h->dt;
}

int Ctx::relax(double* m, double duration_ps, double segment_ps, double eps_abs, double eps_rel, double* stats) {
  require_mesh();
  require_material();
  const int n3 = 3 * nr();
  cudaStream_t st = stream;
  for (auto& b : ybuf) b.alloc(n3);
  for (auto& k : kst) k.alloc(n3);
  ytmp.alloc(n3);
  TMB_CUDA(cudaMemcpyAsync(ybuf[0].p, m, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
  double* y = ybuf[0].p;
  double* yalt = ybuf[1].p;
  launch_normalize(nr(), y, st);
  const double ts = time_scale();
  double dt = std::min(segment_ps * ts, ts);
  for (int i = 0; i < 12; ++i) stats[i] = 0.0;
  double t_ps = 0.0;
  const bool with_demag = has_bem;
  while (t_ps < duration_ps - 1e-12) {
    if (with_demag) {
      demag(y);
      stats[3] += 1;
      stats[4] += neu->last_iters;
      stats[5] += dir->last_iters;
    }
    const double seg = std::min(segment_ps, duration_ps - t_ps);
    if (device_steps && !prof.on) integrate_segment_dev(y, yalt, t_ps * ts, (t_ps + seg) * ts, dt, eps_abs, eps_rel, stats);
    else integrate_segment(y, yalt, t_ps * ts, (t_ps + seg) * ts, dt, eps_abs, eps_rel, stats);
    launch_normalize(nr(), y, st);
    t_ps += seg;
    stats[8] += 1;
  }
  if (with_demag) {
    demag(y);
    stats[3] += 1;
  }
  stats[6] = max_torque(y);
  stats[7] = dt;
  TMB_CUDA(cudaMemcpyAsync(m, y, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
  sync();
  if (!std::isfinite(stats[6])) throw Error(TMB_ERR_NAN, "torque is not finite");
  return TMB_OK;
}

// ------------------------------------------------------------------------------------------
// Fixed-step RK4 with the full effective field at every stage, and its discrete adjoint
// (no tetmag counterpart; the right-hand side is tetmag's, main/TheLLG.cpp:238-254, 670-711).
// ------------------------------------------------------------------------------------------
double Ctx::pulse_hz(double t_ps) const {
  const int ns = int(bz.size());
  if (ns == 0) return 0.0;
  double b;
  if (ns == 1 || t_ps <= bz_t0) b = bz[0];
  else if (t_ps >= bz_t1) b = bz[ns - 1];
  else {
    const double u = (t_ps - bz_t0) / (bz_t1 - bz_t0) * (ns - 1);
    const int k = std::min(int(std::floor(u)), ns - 2);
    const double f = u - k;
    b = (1.0 - f) * bz[k] + f * bz[k + 1];
  }
  return b / kMu0;
}

// The applied field in effect before a fixed-step run is kept and restored afterwards.
void Ctx::begin_timed_field() {
  const size_t n3 = size_t(3) * nr();
  ab.hbase.alloc(n3);
  TMB_CUDA(cudaMemcpyAsync(ab.hbase.p, hext.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
}

void Ctx::end_timed_field() {
  const size_t n3 = size_t(3) * nr();
  TMB_CUDA(cudaMemcpyAsync(hext.p, ab.hbase.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  launch_add(int(n3), hext.p, hdem.p, hfix.p, stream);
}

// One right-hand-side evaluation with the demag field refreshed: k = f(Y, t), H = total field.
void Ctx::stage_eval(const double* Y, double t_ps, double* k, double* H) {
  if (!bz.empty()) launch_set_hz(nr(), ab.hbase.p, pulse_hz(t_ps), hext.p, stream);
  if (has_bem) {
    demag(Y);
    cnt[3] += neu->last_iters + dir->last_iters;
  } else {
    launch_add(3 * nr(), hext.p, hdem.p, hfix.p, stream);
  }
  local(Y, k, H, nullptr);
}

// y <- y + h/6 (k1 + 2 k2 + 2 k3 + k4); with Ys / Hs (4 x 3N each) the stage states and fields
// are kept for the adjoint.
void Ctx::rk4_substep(double* y, double t_ps, double ds_ps, double* Ys, double* Hs) {
  const int n3 = 3 * nr();
  const double h = ds_ps * time_scale();
  double* K[4] = {kst[0].p, kst[1].p, kst[2].p, kst[3].p};
  if (Ys) TMB_CUDA(cudaMemcpyAsync(Ys, y, sizeof(double) * n3, cudaMemcpyDeviceToDevice, stream));
  stage_eval(y, t_ps, K[0], Hs);
  const double c[3] = {0.5 * h, 0.5 * h, h};
  const double tt[3] = {t_ps + 0.5 * ds_ps, t_ps + 0.5 * ds_ps, t_ps + ds_ps};
  for (int i = 0; i < 3; ++i) {
    double* Yi = Ys ? Ys + size_t(i + 1) * n3 : ytmp.p;
    launch_lincomb(n3, Yi, 1.0, y, c[i], K[i], 0.0, nullptr, stream);
    stage_eval(Yi, tt[i], K[i + 1], Hs ? Hs + size_t(i + 1) * n3 : nullptr);
  }
  launch_rk4_final(n3, y, K[0], K[1], K[2], K[3], h, stream);
}

// gout = (df/dm)(Y)^T abar at one stage; dku accumulates (df/dKu)^T abar, zpart gets the block
// partial sums of mu_z (the Bz gradient).  The demag part runs the chain backwards:
// w = -grad^T mu, v = A_D^-T w, a = w + (B^T v_b scattered), a1 = A_N^-T a, div^T a1.
void Ctx::vjp(const double* Y, const double* H, const double* abar, double* gout, double* zpart, int stage) {
  const bool f64 = precision == TMB_FP64;
  const SellView S = pat.view();
  AdjPreArgs pa{};
  pa.n = n;
  pa.m = Y;
  pa.H = H;
  pa.abar = abar;
  pa.alpha = alpha;
  pa.precession = precession;
  pa.js = js.p;
  pa.kax = kax.p;
  pa.mu = ab.mu.p;
  pa.g = gout;
  pa.dku = ab.dku.p;
  pa.zpart = zpart;
  launch_adj_pre(pa, stream);
  const double* q = nullptr;
  if (has_bem) {
    launch_div(ab.mu.p, ab.ninvvol.p, 1.0, ab.w.p, stream);
    dir->solve_t(ab.w.p, ab.v.p, precision, stage);
    if (bem_mode == 1) {
      // hierarchical B^T in cluster order, scattered back to the boundary nodes
      HMat& Hm = this->H;  // H is the stage field here
      if (f64) launch_h_matvec_t<double>(ht_view<double>(0), ab.v.p, Hm.ty.p, Hm.xp64.p, stream);
      else launch_h_matvec_t<float>(ht_view<float>(1), ab.v.p, Hm.ty.p, Hm.xp32.p, stream);
      launch_scatter_add(nb, Hm.gidx.p, Hm.ty.p, ab.w.p, stream);
    } else {
      launch_gather<double>(nb, ab.v.p, bnodes.p, ab.vb.p, stream);
      const int nch = bem_gemv_t_chunks(nb, num_sms);
      if (f64) launch_bem_gemv_t<double>(nb, Bd.p, ab.vb.p, ab.bpart.p, nch, ab.z.p, stream);
      else launch_bem_gemv_t<float>(nb, Bf.p, ab.vb.p, ab.bpart.p, nch, ab.z.p, stream);
      launch_scatter_add(nb, bnodes.p, ab.z.p, ab.w.p, stream);
    }
    neu->solve_t(ab.w.p, ab.a1.p, precision, stage);
    cnt[4] += neu->last_iters + dir->last_iters;
    launch_grad(ab.a1.p, nullptr, nullptr, ab.q.p, nullptr, stream);
    q = ab.q.p;
  }
  const bool idmi = has_dmi && dmi_kind == 1;
  AdjLocalArgs la{};
  la.n = n;
  la.mu = ab.mu.p;
  la.xc = xc.p;
  la.ku2 = has_uni ? ku2.p : nullptr;
  la.kax = kax.p;
  la.idm_d = idmi ? idm_d.p : nullptr;
  la.idm_b = idmi ? idm_b.p : nullptr;
  la.dmi_s = (has_dmi && !idmi) ? dmi_s.p : nullptr;
  la.area = area.p;
  la.nvn = nvn.p;
  la.vol = node_vol.p;
  la.js = js.p;
  la.q = q;
  la.inv_mu0 = 1.0 / kMu0;
  la.g = gout;
  if (f64) launch_adj_local<double>(S, K.p, tg[0].p, tg[1].p, g[0].p, g[1].p, g[2].p, la, stream);
  else launch_adj_local<float>(S, Kf.p, tgf[0].p, tgf[1].p, gf[0].p, gf[1].p, gf[2].p, la, stream);
  cnt[2] += 1;
}

void Ctx::step_rk4(double* m, int nsteps, double dt_ps, int nsub, double t0_ps, bool normalize) {
  require_mesh();
  require_material();
  const int n3 = 3 * nr();
  for (int j = 0; j < 4; ++j) kst[j].alloc(n3);
  ytmp.alloc(n3);
  ab.zn.alloc(size_t(nr()));
  begin_timed_field();
  const double ds = dt_ps / nsub;
  for (int k = 0; k < nsteps; ++k) {
    for (int s = 0; s < nsub; ++s) {
      rk4_substep(m, t0_ps + k * dt_ps + s * ds, ds, nullptr, nullptr);
      cnt[0] += 4;
    }
    if (normalize) launch_normalize_keep(nr(), m, ab.zn.p, stream);
  }
  end_timed_field();
  sync();
}

void Ctx::adjoint_rk4(const double* m0, int nsteps, double dt_ps, int nsub, int ckpt, double t0_ps, bool normalize,
                      const double* w, double* m_final, double* grad_m0, double* grad_ku, double* grad_bz) {
  require_mesh();
  require_material();
  if (has_bem && (ncomp() != 1 || (bem_mode != 0 && bem_mode != 1)))
    throw Error(TMB_ERR_STATE, "adjoint: needs one component and the dense or hierarchical BEM matrix");
  if (rep != 1) throw Error(TMB_ERR_STATE, "adjoint: not for interleaved replicas");
  if (has_cub || has_srf || has_stt)
    throw Error(TMB_ERR_STATE, "adjoint: cubic / surface anisotropy and spin-transfer torque have no transpose here");
  if (has_bem) ensure_demag();
  if (has_bem && bem_mode == 1) h_transpose_build();
  cudaStream_t st = stream;
  const size_t n3 = size_t(3) * n;
  const int nck = (nsteps + ckpt - 1) / ckpt;
  const size_t per_seg = size_t(ckpt) * nsub * 4 * n3;
  for (int j = 0; j < 4; ++j) kst[j].alloc(n3);
  ytmp.alloc(n3);
  ybuf[0].alloc(n3);
  ab.ck.alloc(std::max(1, nck) * n3);
  ab.segY.alloc(per_seg);
  ab.segH.alloc(per_seg);
  ab.segZ.alloc(size_t(ckpt) * n);
  ab.segYend.alloc(size_t(ckpt) * n3);
  ab.zn.alloc(n);
  ab.lam.alloc(n3);
  for (auto& gg : ab.g) gg.alloc(n3);
  ab.abar.alloc(n3);
  ab.mu.alloc(n3);
  ab.w.alloc(n);
  ab.v.alloc(n);
  ab.a1.alloc(n);
  ab.q.alloc(n3);
  ab.vb.alloc(std::max(nb, 1));
  ab.z.alloc(std::max(nb, 1));
  ab.bpart.alloc(size_t(bem_gemv_t_chunks(std::max(nb, 1), num_sms)) * std::max(nb, 1));
  const int nblk = adj_pre_blocks(n);
  const long long nstage = 4LL * nsteps * nsub;
  ab.zpart.alloc(size_t(std::max(1LL, nstage)) * nblk);
  ab.dku.alloc(n);
  ab.dku.zero(st);
  {
    std::vector<double> niv(n);
    for (int i = 0; i < n; ++i) niv[i] = -1.0 / hvol[i];
    ab.ninvvol.upload(niv, st);
  }
  begin_timed_field();
  const double ds = dt_ps / nsub;
  const double h = ds * time_scale();
  double* y = ybuf[0].p;
  TMB_CUDA(cudaMemcpyAsync(y, m0, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
  // forward sweep, keeping a checkpoint every `ckpt` steps
  for (int k = 0; k < nsteps; ++k) {
    if (k % ckpt == 0)
      TMB_CUDA(cudaMemcpyAsync(ab.ck.p + size_t(k / ckpt) * n3, y, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
    for (int s = 0; s < nsub; ++s) {
      rk4_substep(y, t0_ps + k * dt_ps + s * ds, ds, nullptr, nullptr);
      cnt[0] += 4;
    }
    if (normalize) launch_normalize_keep(n, y, ab.zn.p, st);
  }
  TMB_CUDA(cudaMemcpyAsync(m_final, y, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
  // backward sweep: recompute each checkpoint interval keeping its stages, then transpose it
  TMB_CUDA(cudaMemcpyAsync(ab.lam.p, w, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
  for (int seg = nck - 1; seg >= 0; --seg) {
    const int k0 = seg * ckpt, k1 = std::min(nsteps, k0 + ckpt);
    TMB_CUDA(cudaMemcpyAsync(y, ab.ck.p + size_t(seg) * n3, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
    for (int k = k0; k < k1; ++k) {
      for (int s = 0; s < nsub; ++s) {
        const size_t off = (size_t(k - k0) * nsub + s) * 4 * n3;
        rk4_substep(y, t0_ps + k * dt_ps + s * ds, ds, ab.segY.p + off, ab.segH.p + off);
        cnt[1] += 4;
      }
      if (normalize) launch_normalize_keep(n, y, ab.segZ.p + size_t(k - k0) * n, st);
      TMB_CUDA(cudaMemcpyAsync(ab.segYend.p + size_t(k - k0) * n3, y, sizeof(double) * n3, cudaMemcpyDeviceToDevice,
                               st));
    }
    for (int k = k1 - 1; k >= k0; --k) {
      if (normalize) launch_adj_normalize(n, ab.segYend.p + size_t(k - k0) * n3, ab.segZ.p + size_t(k - k0) * n,
                                          ab.lam.p, st);
      for (int s = nsub - 1; s >= 0; --s) {
        const size_t off = (size_t(k - k0) * nsub + s) * 4 * n3;
        const double* Y = ab.segY.p + off;
        const double* Hs = ab.segH.p + off;
        double* zp = ab.zpart.p + size_t((long long)(k * nsub + s) * 4) * nblk;
        double* G[4] = {ab.g[0].p, ab.g[1].p, ab.g[2].p, ab.g[3].p};
        double* lam = ab.lam.p;
        double* a = ab.abar.p;
        launch_lincomb(int(n3), a, h / 6.0, lam, 0.0, nullptr, 0.0, nullptr, st);
        vjp(Y + 3 * n3, Hs + 3 * n3, a, G[3], zp + 3 * nblk, 3);
        launch_lincomb(int(n3), a, h / 3.0, lam, h, G[3], 0.0, nullptr, st);
        vjp(Y + 2 * n3, Hs + 2 * n3, a, G[2], zp + 2 * nblk, 2);
        launch_lincomb(int(n3), a, h / 3.0, lam, 0.5 * h, G[2], 0.0, nullptr, st);
        vjp(Y + n3, Hs + n3, a, G[1], zp + nblk, 1);
        launch_lincomb(int(n3), a, h / 6.0, lam, 0.5 * h, G[1], 0.0, nullptr, st);
        vjp(Y, Hs, a, G[0], zp, 0);
        launch_lincomb(int(n3), lam, 1.0, lam, 1.0, G[0], 1.0, G[1], st);
        launch_lincomb(int(n3), lam, 1.0, lam, 1.0, G[2], 1.0, G[3], st);
      }
    }
  }
  if (grad_m0) TMB_CUDA(cudaMemcpyAsync(grad_m0, ab.lam.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
  if (grad_ku) TMB_CUDA(cudaMemcpyAsync(grad_ku, ab.dku.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  const int ns = int(bz.size());
  if (grad_bz && ns > 0) {
    std::vector<double> zp(size_t(nstage) * nblk);
    TMB_CUDA(cudaMemcpyAsync(zp.data(), ab.zpart.p, zp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    sync();
    std::fill(grad_bz, grad_bz + ns, 0.0);
    const double cst[4] = {0.0, 0.5, 0.5, 1.0};
    for (long long q = 0; q < nstage; ++q) {
      double sz = 0.0;
      for (int b = 0; b < nblk; ++b) sz += zp[size_t(q) * nblk + b];
      const long long ks = q / 4;
      const int k = int(ks / nsub), sub = int(ks % nsub), i = int(q % 4);
      const double t = t0_ps + k * dt_ps + (sub + cst[i]) * ds;
      // hat weights of the samples at t
      if (ns == 1 || t <= bz_t0) grad_bz[0] += sz / kMu0;
      else if (t >= bz_t1) grad_bz[ns - 1] += sz / kMu0;
      else {
        const double u = (t - bz_t0) / (bz_t1 - bz_t0) * (ns - 1);
        const int j = std::min(int(std::floor(u)), ns - 2);
        const double f = u - j;
        grad_bz[j] += (1.0 - f) * sz / kMu0;
        grad_bz[j + 1] += f * sz / kMu0;
      }
    }
  }
  end_timed_field();
  sync();
}

}  // namespace tmb

// ==========================================================================================
// C ABI
// ==========================================================================================
using namespace tmb;

struct tmb_ctx {
  std::unique_ptr<Ctx> c;
};
struct tmb_mesh {
  MeshHost m;
};
struct tmb_solver {
  Ctx* ctx;
  std::unique_ptr<Solver> s;
};

static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define TMB_API_BEGIN try {
#define TMB_API_END                                                  \
  }                                                                  \
  catch (const Error& e) {                                           \
    return fail(e.code, e.what());                                   \
  }                                                                  \
  catch (const std::bad_alloc&) {                                    \
    return fail(TMB_ERR_INTERNAL, "host allocation failed");         \
  }                                                                  \
  catch (const std::exception& e) {                                  \
    const std::string w = e.what();                                  \
    return fail(w.rfind("CUDA", 0) == 0 ? TMB_ERR_CUDA : TMB_ERR_INTERNAL, w); \
  }                                                                  \
  return TMB_OK;

#define TMB_CHECK_ARG(cond, msg) \
  if (!(cond)) return fail(TMB_ERR_ARG, msg);

// Device address of the allocation-free right-hand side's staging array on `device` (the
// current device), resolved once per device; defined with the array below.
namespace tmb {
static void resolve_staging_address(int device);
}

// Stages a host (or device) 3N vector into a device buffer.
static const double* stage_in(Ctx& c, DevArray<double>& buf, const double* p, size_t count, int kind) {
  if (kind == TMB_PTR_DEVICE) return p;
  buf.alloc(count);
  TMB_CUDA(cudaMemcpyAsync(buf.p, p, count * sizeof(double), cudaMemcpyHostToDevice, c.stream));
  return buf.p;
}

extern "C" {

const char* tmb_last_error(void) { return g_last_error.c_str(); }
int tmb_version(void) { return 10000; }

int tmb_kernel_launches(long long* count) {
  TMB_CHECK_ARG(count, "tmb_kernel_launches: null argument");
  *count = launch_count();
  return TMB_OK;
}

int tmb_mesh_create(int nx, int ntet, const double* xyz, const int* tets, tmb_mesh** out) {
  TMB_CHECK_ARG(out && xyz && tets && nx > 0 && ntet > 0, "tmb_mesh_create: bad arguments");
  TMB_API_BEGIN
  for (long long i = 0; i < 4LL * ntet; ++i)
    if (tets[i] < 0 || tets[i] >= nx) return fail(TMB_ERR_ARG, "tmb_mesh_create: node index out of range");
  auto* h = new tmb_mesh();
  h->m.nx = nx;
  h->m.ntet = ntet;
  h->m.xyz.assign(xyz, xyz + size_t(3) * nx);
  h->m.tets.assign(tets, tets + size_t(4) * ntet);
  try {
    fem_prepare(h->m);
    extract_boundary(h->m);
    compute_solid_angles(h->m);
  } catch (...) {
    delete h;
    throw;
  }
  *out = h;
  TMB_API_END
}

int tmb_mesh_destroy(tmb_mesh* mesh) {
  delete mesh;
  return TMB_OK;
}

int tmb_mesh_info(const tmb_mesh* mesh, long long* info) {
  TMB_CHECK_ARG(mesh && info, "tmb_mesh_info: null argument");
  info[0] = mesh->m.nx;
  info[1] = mesh->m.ntet;
  info[2] = mesh->m.fem.ptr.empty() ? 0 : mesh->m.fem.ptr.back();
  info[3] = (long long)mesh->m.bnd.bnodes.size();
  info[4] = (long long)mesh->m.bnd.tri_tet.size();
  info[5] = 0;
  return TMB_OK;
}

int tmb_mesh_get_operators(const tmb_mesh* mesh, int* rowptr, int* col, double* stiff, double* gx, double* gy,
                           double* gz, double* tgx, double* tgy, double* tgz, double* node_vol) {
  TMB_CHECK_ARG(mesh, "tmb_mesh_get_operators: null mesh");
  const FemOperators& F = mesh->m.fem;
  auto cp = [](auto* dst, const auto& src) {
    if (dst) std::copy(src.begin(), src.end(), dst);
  };
  cp(rowptr, F.ptr);
  cp(col, F.col);
  cp(stiff, F.stiff);
  cp(gx, F.grad[0]);
  cp(gy, F.grad[1]);
  cp(gz, F.grad[2]);
  cp(tgx, F.tgrad[0]);
  cp(tgy, F.tgrad[1]);
  cp(tgz, F.tgrad[2]);
  cp(node_vol, F.node_vol);
  return TMB_OK;
}

int tmb_mesh_get_boundary(const tmb_mesh* mesh, int* bnodes, int* tri, double* tri_area, double* tri_normal,
                          double* node_area, double* node_normal, double* solid_angle) {
  TMB_CHECK_ARG(mesh, "tmb_mesh_get_boundary: null mesh");
  const BoundaryData& B = mesh->m.bnd;
  const int n = mesh->m.nx;
  auto cp = [](auto* dst, const auto& src) {
    if (dst) std::copy(src.begin(), src.end(), dst);
  };
  cp(bnodes, B.bnodes);
  cp(tri, B.tri);
  cp(tri_area, B.tri_area);
  cp(tri_normal, B.tri_normal);
  cp(node_area, B.node_area);
  cp(solid_angle, B.solid_angle);
  if (node_normal)
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) node_normal[size_t(d) * n + i] = B.node_normal[size_t(i) * 3 + d];
  return TMB_OK;
}

int tmb_ctx_create(int device, tmb_ctx** out) {
  TMB_CHECK_ARG(out, "tmb_ctx_create: null out");
  TMB_API_BEGIN
  int count = 0;
  TMB_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return fail(TMB_ERR_ARG, "tmb_ctx_create: no such device");
  auto* h = new tmb_ctx();
  try {
    h->c = std::make_unique<Ctx>(device);
    // the allocation-free right-hand side's staging array: its device address is resolved here,
    // where allocating is allowed (resolving it loads the module that holds the array)
    resolve_staging_address(device);
  } catch (...) {
    delete h;
    throw;
  }
  *out = h;
  TMB_API_END
}

int tmb_ctx_destroy(tmb_ctx* ctx) {
  if (ctx) {
    cudaSetDevice(ctx->c->device);
    delete ctx;
  }
  return TMB_OK;
}

int tmb_ctx_set_stream(tmb_ctx* ctx, void* stream) {
  TMB_CHECK_ARG(ctx, "null context");
  ctx->c->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->c->own;
  return TMB_OK;
}

int tmb_set_precision(tmb_ctx* ctx, int precision) {
  TMB_CHECK_ARG(ctx, "null context");
  TMB_CHECK_ARG(precision == TMB_FP64 || precision == TMB_MIXED, "tmb_set_precision: unknown precision");
  ctx->c->precision = precision;
  return TMB_OK;
}

int tmb_set_mesh(tmb_ctx* ctx, const tmb_mesh* mesh) {
  TMB_CHECK_ARG(ctx && mesh, "tmb_set_mesh: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  TMB_CUDA(cudaSetDevice(c.device));
  const MeshHost& M = mesh->m;
  const double* g[3] = {M.fem.grad[0].data(), M.fem.grad[1].data(), M.fem.grad[2].data()};
  const double* tg[3] = {M.fem.tgrad[0].data(), M.fem.tgrad[1].data(), M.fem.tgrad[2].data()};
  std::vector<double> nvn(size_t(3) * M.nx);
  for (int i = 0; i < M.nx; ++i)
    for (int d = 0; d < 3; ++d) nvn[size_t(d) * M.nx + i] = M.bnd.node_normal[size_t(i) * 3 + d];
  c.set_operators(M.nx, M.fem.ptr.data(), M.fem.col.data(), M.fem.stiff.data(), g, tg, M.fem.node_vol.data(),
                  int(M.bnd.bnodes.size()), M.bnd.bnodes.data(), M.bnd.node_area.data(), nvn.data());
  TMB_API_END
}

int tmb_set_operators(tmb_ctx* ctx, int nx, int nnz, const int* rowptr, const int* col, const double* stiff,
                      const double* gx, const double* gy, const double* gz, const double* tgx, const double* tgy,
                      const double* tgz, const double* node_vol, int nb, const int* bnodes,
                      const double* node_area, const double* node_normal) {
  TMB_CHECK_ARG(ctx && rowptr && col && stiff && gx && gy && gz && tgx && tgy && tgz && node_vol && bnodes &&
                    node_area && node_normal,
                "tmb_set_operators: null argument");
  TMB_CHECK_ARG(nx > 0 && nnz > 0 && rowptr[nx] == nnz && nb >= 0 && nb <= nx, "tmb_set_operators: bad sizes");
  TMB_API_BEGIN
  for (int i = 0; i < nnz; ++i)
    if (col[i] < 0 || col[i] >= nx) return fail(TMB_ERR_ARG, "tmb_set_operators: column out of range");
  for (int i = 0; i < nb; ++i)
    if (bnodes[i] < 0 || bnodes[i] >= nx) return fail(TMB_ERR_ARG, "tmb_set_operators: boundary node out of range");
  TMB_CUDA(cudaSetDevice(ctx->c->device));
  const double* g[3] = {gx, gy, gz};
  const double* tg[3] = {tgx, tgy, tgz};
  ctx->c->set_operators(nx, rowptr, col, stiff, g, tg, node_vol, nb, bnodes, node_area, node_normal);
  TMB_API_END
}

int tmb_bem_assemble(tmb_ctx* ctx, const tmb_mesh* mesh) { return tmb_bem_assemble_ex(ctx, mesh, 0); }

int tmb_bem_assemble_ex(tmb_ctx* ctx, const tmb_mesh* mesh, int formula) {
  TMB_CHECK_ARG(ctx && mesh, "tmb_bem_assemble: null argument");
  TMB_CHECK_ARG(formula == 0 || formula == 1, "tmb_bem_assemble_ex: formula is 0 (reference) or 1 (accurate)");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  const MeshHost& M = mesh->m;
  const BoundaryData& B = M.bnd;
  const int nb = int(B.bnodes.size()), nt = int(B.tri_tet.size());
  if (nb != c.nb || M.nx != c.n) return fail(TMB_ERR_ARG, "tmb_bem_assemble: mesh differs from the context's");
  TMB_CUDA(cudaSetDevice(c.device));
  for (int i = 0; i < nb; ++i)
    if (B.bnodes[i] != c.hbnodes[i]) return fail(TMB_ERR_ARG, "tmb_bem_assemble: mesh differs from the context's");
  // one block per component (one shared block for replicas), each assembled from its own
  // boundary triangles in local boundary numbering
  const int nc = c.ncomp(), nstore = c.shared_bem ? 1 : nc;
  std::vector<long long> boff(nstore + 1, 0);
  for (int k = 0; k < nstore; ++k) {
    const int nbc = c.cboff[k + 1] - c.cboff[k];
    boff[k + 1] = boff[k] + (long long)bem_ld(nbc) * nbc;
  }
  c.Bd.alloc(size_t(boff[nstore]));
  std::vector<int> tcomp(nt);
  for (int t = 0; t < nt; ++t) {
    const int b0 = B.bindex[B.tri[size_t(3) * t]];
    tcomp[t] = int(std::upper_bound(c.cboff.begin(), c.cboff.end(), b0) - c.cboff.begin()) - 1;
  }
  for (int k = 0; k < nstore; ++k) {
    const int lo = c.cboff[k], nbc = c.cboff[k + 1] - lo;
    std::vector<double> bxyz(size_t(3) * nbc), area, nrm, solid(B.solid_angle.begin() + lo,
                                                                  B.solid_angle.begin() + lo + nbc);
    for (int i = 0; i < nbc; ++i)
      for (int d = 0; d < 3; ++d) bxyz[size_t(3) * i + d] = M.xyz[size_t(3) * B.bnodes[lo + i] + d];
    std::vector<int> tri;
    for (int t = 0; t < nt; ++t) {
      if (tcomp[t] != k) continue;
      for (int v = 0; v < 3; ++v) {
        const int bi = B.bindex[B.tri[size_t(3) * t + v]] - lo;
        if (bi < 0 || bi >= nbc) return fail(TMB_ERR_ARG, "tmb_bem_assemble: a boundary triangle spans components");
        tri.push_back(bi);
      }
      area.push_back(B.tri_area[t]);
      for (int d = 0; d < 3; ++d) nrm.push_back(B.tri_normal[size_t(3) * t + d]);
    }
    const int ntc = int(area.size());
    DevArray<double> dx, da, dn, ds;
    DevArray<int> dt;
    dx.upload(bxyz, c.stream);
    dt.upload(tri, c.stream);
    da.upload(area, c.stream);
    dn.upload(nrm, c.stream);
    ds.upload(solid, c.stream);
    launch_bem_assemble(nbc, ntc, dx.p, dt.p, da.p, dn.p, ds.p, c.Bd.p + boff[k], formula == 1, c.stream);
    c.sync();
  }
  c.Bf.alloc(size_t(boff[nstore]));
  launch_to_float(c.Bd.p, c.Bf.p, size_t(boff[nstore]), c.stream);
  if (nc > 1 || c.rep > 1) c.plan_components();
  c.sync();
  c.has_bem = true;
  c.H = Ctx::HMat{};
  c.bem_mode = 0;
  c.neu.reset();
  c.dir.reset();
  TMB_API_END
}

int tmb_set_components(tmb_ctx* ctx, int ncomp, const int* node_offsets, int shared_bem) {
  TMB_CHECK_ARG(ctx && node_offsets && ncomp >= 1, "tmb_set_components: bad arguments");
  TMB_API_BEGIN
  if (ctx->c->rep > 1) return fail(TMB_ERR_STATE, "tmb_set_components: the context has interleaved replicas");
  TMB_CUDA(cudaSetDevice(ctx->c->device));
  ctx->c->set_components(ncomp, node_offsets, shared_bem != 0);
  TMB_API_END
}

int tmb_set_replicas(tmb_ctx* ctx, int nrep) {
  TMB_CHECK_ARG(ctx && nrep >= 1, "tmb_set_replicas: nrep must be >= 1");
  TMB_API_BEGIN
  TMB_CUDA(cudaSetDevice(ctx->c->device));
  ctx->c->set_replicas(nrep);
  TMB_API_END
}

int tmb_set_bem_dense(tmb_ctx* ctx, int nb, const double* B_colmajor) {
  TMB_CHECK_ARG(ctx && B_colmajor, "tmb_set_bem_dense: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  if (nb != c.nb) return fail(TMB_ERR_ARG, "tmb_set_bem_dense: nb differs from the boundary node count");
  if (c.ncomp() > 1) return fail(TMB_ERR_STATE, "tmb_set_bem_dense: the context has several components");
  TMB_CUDA(cudaSetDevice(c.device));
  const size_t ld = bem_ld(nb);
  std::vector<double> rowmajor(ld * nb, 0.0);
  for (int j = 0; j < nb; ++j)
    for (int i = 0; i < nb; ++i) rowmajor[size_t(i) * ld + j] = B_colmajor[size_t(j) * nb + i];
  c.Bd.upload(rowmajor, c.stream);
  c.Bf.alloc(ld * nb);
  launch_to_float(c.Bd.p, c.Bf.p, ld * nb, c.stream);
  if (c.rep > 1) c.plan_components();
  c.sync();
  c.has_bem = true;
  c.H = Ctx::HMat{};
  c.bem_mode = 0;
  c.neu.reset();
  c.dir.reset();
  TMB_API_END
}

int tmb_get_bem_dense(tmb_ctx* ctx, double* B_colmajor) {
  TMB_CHECK_ARG(ctx && B_colmajor, "tmb_get_bem_dense: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  if (!c.has_bem || !c.Bd.p) return fail(TMB_ERR_STATE, "no dense BEM matrix on the device");
  if (c.ncomp() > 1) return fail(TMB_ERR_STATE, "tmb_get_bem_dense: the context has several components");
  const int nb = c.nb;
  const size_t ld = bem_ld(nb);
  std::vector<double> rowmajor(ld * nb);
  TMB_CUDA(cudaMemcpyAsync(rowmajor.data(), c.Bd.p, sizeof(double) * ld * nb, cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  for (int j = 0; j < nb; ++j)
    for (int i = 0; i < nb; ++i) B_colmajor[size_t(j) * nb + i] = rowmajor[size_t(i) * ld + j];
  TMB_API_END
}

int tmb_bem_compress(tmb_ctx* ctx, const double* bxyz, const double* bnormal, int leaf, double eta,
                     double eps_mixed, double eps_fp64, int kmax, int keep_dense) {
  TMB_CHECK_ARG(ctx && bxyz, "tmb_bem_compress: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  if (c.rep > 1) return fail(TMB_ERR_STATE, "tmb_bem_compress: not for interleaved replicas (dense GEMM)");
  TMB_CUDA(cudaSetDevice(c.device));
  c.h_compress(bxyz, bnormal, leaf, eta, eps_mixed, eps_fp64, kmax, keep_dense != 0);
  TMB_API_END
}

int tmb_bem_build_h(tmb_ctx* ctx, const tmb_mesh* mesh, int leaf, double eta, double eps_mixed, double eps_fp64,
                    int kmax) {
  TMB_CHECK_ARG(ctx && mesh, "tmb_bem_build_h: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  const MeshHost& M = mesh->m;
  const BoundaryData& B = M.bnd;
  const int nb = int(B.bnodes.size());
  if (nb != c.nb || M.nx != c.n) return fail(TMB_ERR_ARG, "tmb_bem_build_h: mesh differs from the context's");
  if (c.rep > 1) return fail(TMB_ERR_STATE, "tmb_bem_build_h: not for interleaved replicas (dense GEMM)");
  TMB_CUDA(cudaSetDevice(c.device));
  std::vector<double> bxyz(size_t(3) * nb), bnrm(size_t(3) * nb);
  for (int i = 0; i < nb; ++i)
    for (int d = 0; d < 3; ++d) {
      bxyz[size_t(3) * i + d] = M.xyz[size_t(3) * B.bnodes[i] + d];
      bnrm[size_t(3) * i + d] = B.node_normal[size_t(3) * B.bnodes[i] + d];
    }
  c.h_compress(bxyz.data(), bnrm.data(), leaf, eta, eps_mixed, eps_fp64, kmax, true, &M);
  TMB_API_END
}

int tmb_set_bem_accuracy(tmb_ctx* ctx, double matrix_share) {
  TMB_CHECK_ARG(ctx && matrix_share >= 0.0 && std::isfinite(matrix_share),
                "tmb_set_bem_accuracy: matrix_share is a finite number >= 0");
  ctx->c->h_share = matrix_share;
  return TMB_OK;
}

int tmb_set_bem_mode(tmb_ctx* ctx, int mode) {
  TMB_CHECK_ARG(ctx && (mode >= 0 && mode <= 2), "tmb_set_bem_mode: mode is 0 (dense), 1 (hierarchical) or 2 (H2)");
  Ctx& c = *ctx->c;
  if (mode == 1 && !c.H.built) return fail(TMB_ERR_STATE, "tmb_set_bem_mode: no hierarchical matrix built");
  if (mode == 2 && !(c.H2[0].built && c.H2[1].built))
    return fail(TMB_ERR_STATE, "tmb_set_bem_mode: no H2 matrix built (tmb_bem_h2)");
  if (mode == 0 && (!c.Bd.p || !c.Bf.p)) return fail(TMB_ERR_STATE, "tmb_set_bem_mode: the dense matrix was released");
  c.bem_mode = mode;
  return TMB_OK;
}

int tmb_bem_info(tmb_ctx* ctx, double* out) {
  TMB_CHECK_ARG(ctx && out, "tmb_bem_info: null argument");
  const Ctx& c = *ctx->c;
  const auto& H = c.H;
  out[0] = c.bem_mode;
  out[1] = H.nnear;
  out[2] = H.nfar;
  out[3] = double(H.terms[0]);
  out[4] = double(H.terms[1]);
  out[5] = H.bytes[0];
  out[6] = H.bytes[1];
  out[7] = double(c.nb) * double(c.nb);
  out[8] = H.failed;
  out[9] = H.max_rank;
  out[10] = H.ms;
  out[11] = H.built ? 1.0 : 0.0;
  return TMB_OK;
}

int tmb_bem_h2(tmb_ctx* ctx, double eps_fp64, double eps_mixed, int kmax) {
  TMB_CHECK_ARG(ctx, "tmb_bem_h2: null context");
  TMB_API_BEGIN
  ctx->c->h2_build(eps_fp64, eps_mixed, kmax);
  TMB_API_END
}

int tmb_bem_h2_info(tmb_ctx* ctx, double* out) {
  TMB_CHECK_ARG(ctx && out, "tmb_bem_h2_info: null argument");
  const Ctx& c = *ctx->c;
  for (int w = 0; w < 2; ++w) {
    const auto& M = c.H2[w];
    double* o = out + 8 * w;
    o[0] = M.built ? 1.0 : 0.0;
    o[1] = M.bytes;
    o[2] = M.coupling_bytes;
    o[3] = M.basis_bytes;
    o[4] = M.max_kr;
    o[5] = M.max_kc;
    o[6] = M.ms;
    o[7] = M.eps;
  }
  return TMB_OK;
}

int tmb_bem_verify(tmb_ctx* ctx, double* block_out, double* out) {
  TMB_CHECK_ARG(ctx && out, "tmb_bem_verify: null argument");
  TMB_API_BEGIN
  TMB_CUDA(cudaSetDevice(ctx->c->device));
  ctx->c->h_verify(block_out, out);
  TMB_API_END
}

int tmb_bem_apply(tmb_ctx* ctx, const double* x, double* y, int transpose, int ptr_kind) {
  TMB_CHECK_ARG(ctx && x && y, "tmb_bem_apply: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  TMB_CUDA(cudaSetDevice(c.device));
  c.require_mesh();
  const size_t nbv = size_t(c.nb);
  const double* xd = stage_in(c, c.in3, x, nbv, ptr_kind);
  if (ptr_kind == TMB_PTR_DEVICE) {
    c.bem_apply(xd, y, transpose != 0);
  } else {
    c.out3.alloc(nbv);
    c.bem_apply(xd, c.out3.p, transpose != 0);
    TMB_CUDA(cudaMemcpyAsync(y, c.out3.p, nbv * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
  }
  TMB_API_END
}

int tmb_set_material(tmb_ctx* ctx, const double* Js, const double* A, const double* Ku, const double* ku_axis,
                     const double* D, double alpha) {
  TMB_CHECK_ARG(ctx && Js && A, "tmb_set_material: Js and A are required");
  TMB_CHECK_ARG(std::isfinite(alpha) && alpha >= 0.0, "tmb_set_material: alpha must be finite and >= 0");
  TMB_API_BEGIN
  TMB_CUDA(cudaSetDevice(ctx->c->device));
  ctx->c->set_material(Js, A, Ku, ku_axis, D, alpha);
  TMB_API_END
}

int tmb_set_dmi_kind(tmb_ctx* ctx, int kind) {
  TMB_CHECK_ARG(ctx && (kind == 0 || kind == 1), "tmb_set_dmi_kind: kind is 0 (bulk) or 1 (interfacial)");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  TMB_CUDA(cudaSetDevice(c.device));
  c.dmi_kind = kind;
  if (c.has_material) c.upload_dmi();
  TMB_API_END
}

int tmb_set_applied_field(tmb_ctx* ctx, const double* hext, int ptr_kind) {
  TMB_CHECK_ARG(ctx && hext, "tmb_set_applied_field: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  const size_t n3 = size_t(3) * c.nr();
  TMB_CUDA(cudaMemcpyAsync(c.hext.p, hext, n3 * sizeof(double),
                           ptr_kind == TMB_PTR_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c.stream));
  launch_add(int(n3), c.hext.p, c.hdem.p, c.hfix.p, c.stream);
  c.sync();
  TMB_API_END
}

int tmb_set_llg_options(tmb_ctx* ctx, int precession) {
  TMB_CHECK_ARG(ctx, "null context");
  ctx->c->precession = precession ? 1 : 0;
  return TMB_OK;
}

int tmb_set_solver_params(tmb_ctx* ctx, double tol, int maxiter) {
  TMB_CHECK_ARG(ctx, "null context");
  TMB_CHECK_ARG(tol > 0.0 && tol < 1.0 && maxiter > 0, "tmb_set_solver_params: need 0 < tol < 1, maxiter > 0");
  ctx->c->tol = tol;
  ctx->c->maxit = maxiter;
  return TMB_OK;
}

int tmb_demag_field(tmb_ctx* ctx, const double* m, double* hdem, int ptr_kind) {
  TMB_CHECK_ARG(ctx && m, "tmb_demag_field: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  const size_t n3 = size_t(3) * c.nr();
  const double* md = stage_in(c, c.in3, m, n3, ptr_kind);
  c.demag(md);
  if (hdem)
    TMB_CUDA(cudaMemcpyAsync(hdem, c.hdem.p, n3 * sizeof(double),
                             ptr_kind == TMB_PTR_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                             c.stream));
  if (ptr_kind != TMB_PTR_DEVICE) c.sync();
  TMB_API_END
}

int tmb_field_eval(tmb_ctx* ctx, const double* m, double* ydot, double* hdem, int ptr_kind) {
  TMB_CHECK_ARG(ctx && m && ydot, "tmb_field_eval: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  const size_t n3 = size_t(3) * c.nr();
  const double* md = stage_in(c, c.in3, m, n3, ptr_kind);
  c.demag(md);
  if (ptr_kind == TMB_PTR_DEVICE) {
    c.local(md, ydot, nullptr, nullptr);
    if (hdem) TMB_CUDA(cudaMemcpyAsync(hdem, c.hdem.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
  } else {
    c.out3.alloc(n3);
    c.local(md, c.out3.p, nullptr, nullptr);
    TMB_CUDA(cudaMemcpyAsync(ydot, c.out3.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    if (hdem) TMB_CUDA(cudaMemcpyAsync(hdem, c.hdem.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
  }
  TMB_API_END
}

int tmb_set_demag_frozen(tmb_ctx* ctx, const double* hdem, int ptr_kind) {
  TMB_CHECK_ARG(ctx && hdem, "tmb_set_demag_frozen: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  const size_t n3 = size_t(3) * c.nr();
  TMB_CUDA(cudaMemcpyAsync(c.hdem.p, hdem, n3 * sizeof(double),
                           ptr_kind == TMB_PTR_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c.stream));
  launch_add(int(n3), c.hext.p, c.hdem.p, c.hfix.p, c.stream);
  if (ptr_kind != TMB_PTR_DEVICE) c.sync();
  TMB_API_END
}

int tmb_effective_field(tmb_ctx* ctx, const double* m, double* h, int ptr_kind) {
  TMB_CHECK_ARG(ctx && m && h, "tmb_effective_field: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  const size_t n3 = size_t(3) * c.nr();
  const double* md = stage_in(c, c.in3, m, n3, ptr_kind);
  if (ptr_kind == TMB_PTR_DEVICE) {
    c.local(md, nullptr, h, nullptr);
  } else {
    c.out3.alloc(n3);
    c.local(md, nullptr, c.out3.p, nullptr);
    TMB_CUDA(cudaMemcpyAsync(h, c.out3.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
  }
  TMB_API_END
}

int tmb_llg_rhs(tmb_ctx* ctx, double t, const double* y, double* ydot, int ptr_kind) {
  (void)t;  // the frozen-demag right-hand side does not depend on t explicitly
  TMB_CHECK_ARG(ctx && y && ydot, "tmb_llg_rhs: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  const size_t n3 = size_t(3) * c.nr();
  const double* yd = stage_in(c, c.in3, y, n3, ptr_kind);
  if (ptr_kind == TMB_PTR_DEVICE) {
    c.local(yd, ydot, nullptr, nullptr);
  } else {
    c.out3.alloc(n3);
    c.local(yd, c.out3.p, nullptr, nullptr);
    TMB_CUDA(cudaMemcpyAsync(ydot, c.out3.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
  }
  TMB_API_END
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Right-hand side for host vectors without any device allocation.
//
// Some callers cannot allocate device memory while they evaluate the right-hand side: a
// host-side integrator called from inside a process that runs under a fixed device-memory
// budget, a time-critical loop that must not pay cudaMalloc's implicit device-wide
// synchronisation on its first call, or code running on a stream that other work is being
// captured on.  tmb_llg_rhs with host pointers stages y and ydot through device buffers that
// it allocates on first use; this variant stages them through one file-scope device array of
// fixed size instead.  That array (2 x 3 x 65536 doubles, 3 MiB) is held by every GPU that
// loads the library, until the process exits.
// ------------------------------------------------------------------------------------------
namespace tmb {

constexpr int kNoAllocMaxNodes = 65536;
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) double g_rhs_staging[2 * 3 * kNoAllocMaxNodes];
static std::mutex g_staging_mutex;
static double* g_staging_address[kNoAllocMaxDevices] = {};

// Resolves the device address of g_rhs_staging on `device`, which must be the current device.
// Called by tmb_ctx_create, once per device.  The host-side name of the array is only a
// stand-in: kernels and copies must be given this address.  Resolving it loads the module that
// holds the array (with lazy module loading that is the moment the 3 MiB are reserved), and the
// kernels the entry point launches are loaded with it, so that both happen at context creation,
// where allocating is allowed, and never inside tmb_llg_rhs_noalloc.  Devices beyond
// kNoAllocMaxDevices are skipped (their contexts get TMB_ERR_ARG from tmb_llg_rhs_noalloc).
static void resolve_staging_address(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) return;
  std::lock_guard<std::mutex> lock(g_staging_mutex);
  if (!g_staging_address[device]) {
    void* p = nullptr;
    TMB_CUDA(cudaGetSymbolAddress(&p, g_rhs_staging));
    preload_local_kernels();
    g_staging_address[device] = static_cast<double*>(p);
  }
}

// The address resolved by tmb_ctx_create for `device`, or nullptr.
static double* staging_address(int device) {
  std::lock_guard<std::mutex> lock(g_staging_mutex);
  return g_staging_address[device];
}

}  // namespace tmb

extern "C" {

int tmb_llg_rhs_noalloc(tmb_ctx* ctx, double t, const double* y, double* ydot) {
  (void)t;  // the frozen-demag right-hand side does not depend on t explicitly
  TMB_CHECK_ARG(ctx && y && ydot, "tmb_llg_rhs_noalloc: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  c.require_material();
  if (c.nr() > kNoAllocMaxNodes)
    return fail(TMB_ERR_ARG, "tmb_llg_rhs_noalloc: nodes x replicas = " + std::to_string(c.nr()) +
                                 "; its static staging array holds at most " +
                                 std::to_string(kNoAllocMaxNodes) + " (use tmb_llg_rhs)");
  if (c.device < 0 || c.device >= kNoAllocMaxDevices)
    return fail(TMB_ERR_ARG, "tmb_llg_rhs_noalloc: device ordinal beyond the supported range");
  double* const stage = staging_address(c.device);
  if (!stage) return fail(TMB_ERR_STATE, "tmb_llg_rhs_noalloc: staging array not resolved for this device");
  TMB_CUDA(cudaSetDevice(c.device));
  double* const yd = stage;                          // y, 3N
  double* const od = stage + 3 * kNoAllocMaxNodes;   // ydot, 3N
  const size_t n3 = size_t(3) * c.nr();
  TMB_CUDA(cudaMemcpyAsync(yd, y, n3 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
  c.launch_local(c.local_args(yd, od, nullptr, nullptr), c.stream);
  TMB_CUDA(cudaMemcpyAsync(ydot, od, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  TMB_API_END
}

int tmb_max_torque(tmb_ctx* ctx, const double* m, double* out, int ptr_kind) {
  TMB_CHECK_ARG(ctx && m && out, "tmb_max_torque: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  const double* md = stage_in(c, c.in3, m, size_t(3) * c.nr(), ptr_kind);
  *out = c.max_torque(md);
  if (!std::isfinite(*out)) return fail(TMB_ERR_NAN, "tmb_max_torque: torque is not finite");
  TMB_API_END
}

int tmb_normalize(tmb_ctx* ctx, double* m, int ptr_kind) {
  TMB_CHECK_ARG(ctx && m, "tmb_normalize: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  const size_t n3 = size_t(3) * c.nr();
  if (ptr_kind == TMB_PTR_DEVICE) {
    launch_normalize(c.nr(), m, c.stream);
  } else {
    c.in3.alloc(n3);
    TMB_CUDA(cudaMemcpyAsync(c.in3.p, m, n3 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    launch_normalize(c.nr(), c.in3.p, c.stream);
    TMB_CUDA(cudaMemcpyAsync(m, c.in3.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
  }
  TMB_API_END
}

int tmb_relax(tmb_ctx* ctx, double* m, double duration_ps, double segment_ps, double eps_abs, double eps_rel,
              double* stats, int ptr_kind) {
  TMB_CHECK_ARG(ctx && m && stats, "tmb_relax: null argument");
  TMB_CHECK_ARG(duration_ps >= 0.0 && segment_ps > 0.0 && eps_abs > 0.0 && eps_rel >= 0.0,
                "tmb_relax: bad time or tolerance arguments");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  const size_t n3 = size_t(3) * c.nr();
  if (ptr_kind == TMB_PTR_DEVICE) {
    c.relax(m, duration_ps, segment_ps, eps_abs, eps_rel, stats);
  } else {
    c.in3.alloc(n3);
    TMB_CUDA(cudaMemcpyAsync(c.in3.p, m, n3 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    c.relax(c.in3.p, duration_ps, segment_ps, eps_abs, eps_rel, stats);
    TMB_CUDA(cudaMemcpyAsync(m, c.in3.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
  }
  TMB_API_END
}

int tmb_set_cubic_anisotropy(tmb_ctx* ctx, const double* Kc1, const double* Kc2, const double* axes) {
  TMB_CHECK_ARG(ctx, "tmb_set_cubic_anisotropy: null context");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  TMB_CUDA(cudaSetDevice(c.device));
  if (!Kc1) {
    c.hKc1.clear();
  } else {
    if (!Kc2 || !axes) return fail(TMB_ERR_ARG, "tmb_set_cubic_anisotropy: Kc2 and axes are required with Kc1");
    c.hKc1.assign(Kc1, Kc1 + c.n);
    c.hKc2.assign(Kc2, Kc2 + c.n);
    c.hcax.assign(axes, axes + size_t(9) * c.n);
  }
  c.upload_extra();
  TMB_API_END
}

int tmb_set_surface_anisotropy(tmb_ctx* ctx, const double* Ks) {
  TMB_CHECK_ARG(ctx, "tmb_set_surface_anisotropy: null context");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  TMB_CUDA(cudaSetDevice(c.device));
  if (!Ks) c.hKs.clear();
  else c.hKs.assign(Ks, Ks + c.n);
  c.upload_extra();
  TMB_API_END
}

int tmb_set_stt(tmb_ctx* ctx, const double* eta, double beta, double scale) {
  TMB_CHECK_ARG(ctx, "tmb_set_stt: null context");
  TMB_CHECK_ARG(std::isfinite(beta) && std::isfinite(scale), "tmb_set_stt: beta and scale must be finite");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  TMB_CUDA(cudaSetDevice(c.device));
  if (!eta) {
    c.has_stt = false;
    c.stt_eta.reset();
  } else {
    c.stt_eta.upload(eta, size_t(3) * c.n, c.stream);
    c.stt_beta = beta;
    c.stt_scale = scale;
    c.has_stt = true;
    c.sync();
  }
  TMB_API_END
}

int tmb_energies(tmb_ctx* ctx, const double* m, double* out, int ptr_kind) {
  TMB_CHECK_ARG(ctx && m && out, "tmb_energies: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  TMB_CUDA(cudaSetDevice(c.device));
  const double* md = stage_in(c, c.in3, m, size_t(3) * c.nr(), ptr_kind);
  c.energies(md, out);
  for (int i = 0; i < 8; ++i)
    if (!std::isfinite(out[i])) return fail(TMB_ERR_NAN, "tmb_energies: an energy is not finite");
  TMB_API_END
}

int tmb_write_vtu(const char* path, int nx, const double* xyz, int ntet, const int* tets, const double* m,
                  const int* material, double time_ps, const double* field, const char* field_name, int binary) {
  TMB_CHECK_ARG(path && nx > 0 && ntet >= 0 && xyz && m && (ntet == 0 || tets) && (binary == 0 || binary == 1),
                "tmb_write_vtu: null argument or bad size");
  TMB_API_BEGIN
  for (long long k = 0; k < 4LL * ntet; ++k)
    if (tets[k] < 0 || tets[k] >= nx) return fail(TMB_ERR_ARG, "tmb_write_vtu: node index out of range");
  std::string err;
  if (int rc = write_vtu(path, nx, xyz, ntet, tets, m, material, time_ps, "timeInPs", field, field_name, binary,
                         err))
    return fail(rc, err);
  TMB_API_END
}

int tmb_read_magnetization(const char* path, int nx, double* m, double* time_ps) {
  TMB_CHECK_ARG(path && nx > 0 && m && time_ps, "tmb_read_magnetization: null argument or nx <= 0");
  TMB_API_BEGIN
  std::string err;
  if (int rc = read_magnetization(path, nx, m, time_ps, err)) return fail(rc, err);
  TMB_API_END
}

static int copy_text(const std::string& t, char* buf, int cap, const char* who) {
  if (int(t.size()) + 1 > cap)
    return fail(TMB_ERR_ARG, std::string(who) + ": buffer too small (" + std::to_string(t.size() + 1) + " bytes needed)");
  std::memcpy(buf, t.c_str(), t.size() + 1);
  return TMB_OK;
}

int tmb_log_header(const char* start_time, const char* host, const char* user, char* buf, int cap) {
  TMB_CHECK_ARG(buf && cap > 0, "tmb_log_header: null buffer");
  TMB_API_BEGIN
  return copy_text(log_header(start_time, host, user), buf, cap, "tmb_log_header");
  TMB_API_END
}

int tmb_log_format(double elapsed_ps, const double* energies, double max_torque, const double* mean_m,
                   const double* mean_h_tesla, char* buf, int cap) {
  TMB_CHECK_ARG(energies && mean_m && mean_h_tesla && buf && cap > 0, "tmb_log_format: null argument");
  TMB_API_BEGIN
  return copy_text(log_row(elapsed_ps, energies, max_torque, mean_m, mean_h_tesla), buf, cap, "tmb_log_format");
  TMB_API_END
}

int tmb_log_row(tmb_ctx* ctx, const double* m, int ptr_kind, double elapsed_ps, double max_torque, char* buf,
                int cap) {
  TMB_CHECK_ARG(ctx && m && buf && cap > 0, "tmb_log_row: null argument");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  c.require_material();
  TMB_CUDA(cudaSetDevice(c.device));
  const size_t n3 = size_t(3) * c.nr();
  const double* md = stage_in(c, c.in3, m, n3, ptr_kind);
  double e[8];
  c.energies(md, e);
  if (max_torque < 0.0) max_torque = c.max_torque(md);
  // volume-weighted means (TheSimulation::getMeanM, main/TheSimulation.cpp:100-102; TheLLG::getMeanH,
  // main/TheLLG.cpp:421-423) over every node of every replica, the field in Tesla
  std::vector<double> hm(n3), hh(n3);
  TMB_CUDA(cudaMemcpyAsync(hm.data(), md, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  TMB_CUDA(cudaMemcpyAsync(hh.data(), c.hext.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  const int nrr = c.nr(), R = c.rep;
  double mm[3] = {0, 0, 0}, mh[3] = {0, 0, 0}, vt = 0.0;
  for (int g = 0; g < nrr; ++g) {
    const double v = c.hvol[g / R];
    vt += v;
    for (int d = 0; d < 3; ++d) {
      mm[d] += v * hm[size_t(d) * nrr + g];
      mh[d] += v * hh[size_t(d) * nrr + g];
    }
  }
  for (int d = 0; d < 3; ++d) {
    mm[d] /= vt;
    mh[d] = mh[d] / vt * kMu0;
  }
  mh[2] += c.pulse_hz(elapsed_ps) * kMu0;
  for (double x : e)
    if (!std::isfinite(x)) return fail(TMB_ERR_NAN, "tmb_log_row: an energy is not finite");
  return copy_text(log_row(elapsed_ps, e, max_torque, mm, mh), buf, cap, "tmb_log_row");
  TMB_API_END
}

int tmb_set_bem_gemm_kind(tmb_ctx* ctx, int tensor_cores) {
  TMB_CHECK_ARG(ctx && (tensor_cores == 0 || tensor_cores == 1), "tmb_set_bem_gemm_kind: kind is 0 or 1");
  TMB_API_BEGIN
  ctx->c->gemm_tc = tensor_cores != 0;
  TMB_API_END
}

int tmb_bem_gemm_info(tmb_ctx* ctx, double* out) {
  TMB_CHECK_ARG(ctx && out, "tmb_bem_gemm_info: null argument");
  TMB_API_BEGIN
  const Ctx& c = *ctx->c;
  for (int i = 0; i < 11; ++i) out[i] = 0.0;
  out[0] = c.gemm_tc ? 1.0 : 0.0;
  out[1] = c.tc_split;
  for (size_t i = 1; i < c.tc_tune_ms.size() && i <= 8; ++i) out[1 + i] = c.tc_tune_ms[i];
  out[10] = c.tc_split > 0 ? c.tc_stages : 0;
  TMB_API_END
}

int tmb_set_bz_pulse(tmb_ctx* ctx, int ns, const double* bz_tesla, double t0_ps, double t1_ps) {
  TMB_CHECK_ARG(ctx && ns >= 0 && (ns == 0 || bz_tesla), "tmb_set_bz_pulse: null argument or ns < 0");
  TMB_CHECK_ARG(ns <= 1 || t1_ps > t0_ps, "tmb_set_bz_pulse: t1_ps must exceed t0_ps");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.bz.assign(bz_tesla, bz_tesla + ns);
  for (double b : c.bz)
    if (!std::isfinite(b)) throw Error(TMB_ERR_ARG, "tmb_set_bz_pulse: samples must be finite");
  c.bz_t0 = t0_ps;
  c.bz_t1 = t1_ps;
  TMB_API_END
}

int tmb_step_rk4(tmb_ctx* ctx, double* m, int nsteps, double dt_ps, int nsub, double t0_ps, int normalize,
                 double* stats, int ptr_kind) {
  TMB_CHECK_ARG(ctx && m, "tmb_step_rk4: null argument");
  TMB_CHECK_ARG(nsteps >= 0 && nsub >= 1 && dt_ps > 0.0 && std::isfinite(dt_ps), "tmb_step_rk4: bad step arguments");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  TMB_CUDA(cudaSetDevice(c.device));
  const size_t n3 = size_t(3) * c.nr();
  for (double& v : c.cnt) v = 0.0;
  double* md = m;
  if (ptr_kind != TMB_PTR_DEVICE) {
    c.ab.io[0].alloc(n3);
    TMB_CUDA(cudaMemcpyAsync(c.ab.io[0].p, m, n3 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    md = c.ab.io[0].p;
  }
  c.step_rk4(md, nsteps, dt_ps, nsub, t0_ps, normalize != 0);
  if (ptr_kind != TMB_PTR_DEVICE) {
    TMB_CUDA(cudaMemcpyAsync(m, md, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
  }
  if (stats)
    for (int i = 0; i < 8; ++i) stats[i] = c.cnt[i];
  TMB_API_END
}

int tmb_adjoint_rk4(tmb_ctx* ctx, const double* m0, int nsteps, double dt_ps, int nsub, int ckpt_every, double t0_ps,
                    int normalize, const double* w, double* m_final, double* grad_m0, double* grad_ku,
                    double* grad_bz, double* J, double* stats, int ptr_kind) {
  TMB_CHECK_ARG(ctx && m0 && w && m_final, "tmb_adjoint_rk4: null argument");
  TMB_CHECK_ARG(nsteps >= 1 && nsub >= 1 && ckpt_every >= 1 && dt_ps > 0.0 && std::isfinite(dt_ps),
                "tmb_adjoint_rk4: bad step arguments");
  TMB_API_BEGIN
  Ctx& c = *ctx->c;
  c.require_mesh();
  TMB_CUDA(cudaSetDevice(c.device));
  const size_t n3 = size_t(3) * c.nr(), n = size_t(c.n);
  for (double& v : c.cnt) v = 0.0;
  const bool dev = ptr_kind == TMB_PTR_DEVICE;
  const double* m0d = stage_in(c, c.ab.io[0], m0, n3, ptr_kind);
  const double* wd = stage_in(c, c.ab.io[1], w, n3, ptr_kind);
  double* mfd = m_final;
  double* gmd = grad_m0;
  double* gkd = grad_ku;
  if (!dev) {
    c.ab.io[2].alloc(n3);
    mfd = c.ab.io[2].p;
    if (grad_m0) {
      c.ab.io[3].alloc(n3);
      gmd = c.ab.io[3].p;
    }
    if (grad_ku) {
      c.ab.io[4].alloc(n);
      gkd = c.ab.io[4].p;
    }
  }
  c.adjoint_rk4(m0d, nsteps, dt_ps, nsub, ckpt_every, t0_ps, normalize != 0, wd, mfd, gmd, gkd, grad_bz);
  std::vector<double> hm(n3), hw(n3);
  TMB_CUDA(cudaMemcpyAsync(hm.data(), mfd, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  TMB_CUDA(cudaMemcpyAsync(hw.data(), wd, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  if (!dev) {
    TMB_CUDA(cudaMemcpyAsync(m_final, mfd, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    if (grad_m0) TMB_CUDA(cudaMemcpyAsync(grad_m0, gmd, n3 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    if (grad_ku) TMB_CUDA(cudaMemcpyAsync(grad_ku, gkd, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  }
  c.sync();
  if (J) {
    double s = 0.0;
    for (size_t i = 0; i < n3; ++i) s += hw[i] * hm[i];
    *J = s;
  }
  if (stats) {
    for (int i = 0; i < 8; ++i) stats[i] = c.cnt[i];
    stats[5] = (nsteps + ckpt_every - 1) / ckpt_every;
    stats[6] = double(c.ab.segY.n + c.ab.segH.n + c.ab.ck.n) * sizeof(double);
  }
  if (!std::isfinite(J ? *J : 0.0)) throw Error(TMB_ERR_NAN, "adjoint: objective is not finite");
  TMB_API_END
}

int tmb_get_stats(tmb_ctx* ctx, double* out) {
  TMB_CHECK_ARG(ctx && out, "tmb_get_stats: null argument");
  Ctx& c = *ctx->c;
  for (int i = 0; i < 8; ++i) out[i] = 0.0;
  if (c.neu && c.dir) {
    out[0] = c.neu->last_iters;
    out[1] = c.dir->last_iters;
    out[2] = c.neu->last_relres;
    out[3] = c.dir->last_relres;
    out[4] = c.neu->last_status;
    out[5] = c.dir->last_status;
    out[6] = double(c.neu->H.levels.size());
    out[7] = c.neu->H.setup_ms + c.dir->H.setup_ms;
  }
  return TMB_OK;
}

int tmb_profile_enable(tmb_ctx* ctx, int on) {
  TMB_CHECK_ARG(ctx, "null context");
  TMB_API_BEGIN
  ctx->c->prof.reset();
  ctx->c->prof.on = on != 0;
  TMB_API_END
}

int tmb_profile_read(tmb_ctx* ctx, double* out) {
  TMB_CHECK_ARG(ctx && out, "tmb_profile_read: null argument");
  TMB_API_BEGIN
  Prof& P = ctx->c->prof;
  P.flush();
  for (int i = 0; i < kProfIds; ++i) {
    out[3 * i] = P.count[i];
    out[3 * i + 1] = P.ms[i];
    out[3 * i + 2] = P.count[i] > 0 ? P.bytes[i] / P.count[i] : 0.0;
  }
  TMB_API_END
}

int tmb_solver_create(tmb_ctx* ctx, tmb_solver** out) {
  TMB_CHECK_ARG(ctx && out, "tmb_solver_create: null argument");
  TMB_API_BEGIN
  auto* s = new tmb_solver();
  s->ctx = ctx->c.get();
  s->s = std::make_unique<Solver>(s->ctx);
  s->s->want_rep = 1;  // the plugin solves one right-hand side
  *out = s;
  TMB_API_END
}

int tmb_solver_destroy(tmb_solver* s) {
  delete s;
  return TMB_OK;
}

int tmb_solver_set_matrix(tmb_solver* s, int n, int nnz, const int* rowptr, const int* col, const double* val) {
  TMB_CHECK_ARG(s && rowptr && col && val && n > 0 && nnz > 0 && rowptr[0] == 0 && rowptr[n] == nnz,
                "tmb_solver_set_matrix: bad arguments");
  TMB_API_BEGIN
  for (int i = 0; i < n; ++i)
    if (rowptr[i + 1] < rowptr[i]) return fail(TMB_ERR_ARG, "tmb_solver_set_matrix: rowptr not monotone");
  for (int k = 0; k < nnz; ++k)
    if (col[k] < 0 || col[k] >= n) return fail(TMB_ERR_ARG, "tmb_solver_set_matrix: column out of range");
  s->s->set_matrix(n, rowptr, col, val);
  TMB_API_END
}

int tmb_solver_set_tolerance(tmb_solver* s, double tol, int maxiter) {
  TMB_CHECK_ARG(s && tol > 0.0 && tol < 1.0 && maxiter > 0, "tmb_solver_set_tolerance: bad arguments");
  s->s->tol = tol;
  s->s->maxit = maxiter;
  return TMB_OK;
}

int tmb_solver_compute(tmb_solver* s) {
  TMB_CHECK_ARG(s, "null solver");
  TMB_API_BEGIN
  TMB_CUDA(cudaSetDevice(s->ctx->device));
  s->s->compute();
  TMB_API_END
}

int tmb_solver_solve(tmb_solver* s, const double* b, double* x, int ptr_kind) {
  TMB_CHECK_ARG(s && b && x, "tmb_solver_solve: null argument");
  TMB_API_BEGIN
  Solver& S = *s->s;
  Ctx& c = *s->ctx;
  if (!S.computed) return fail(TMB_ERR_STATE, "tmb_solver_solve: compute() not called");
  const size_t n = size_t(S.n);
  DevArray<double> tmp;
  const double* bd = stage_in(c, tmp, b, n, ptr_kind);
  S.solve(bd, c.precision);
  TMB_CUDA(cudaMemcpyAsync(x, S.x.p, n * sizeof(double),
                           ptr_kind == TMB_PTR_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  if (S.last_status == 3) return fail(TMB_ERR_NOCONVERGE, "tmb_solver_solve: not converged within maxiter");
  if (S.last_status == 5) return fail(TMB_ERR_NAN, "tmb_solver_solve: breakdown (NaN or non-positive p.Ap)");
  TMB_API_END
}

int tmb_solver_info(tmb_solver* s, double* info) {
  TMB_CHECK_ARG(s && info, "tmb_solver_info: null argument");
  info[0] = s->s->last_iters;
  info[1] = s->s->last_relres;
  info[2] = s->s->last_status;
  return TMB_OK;
}

}  // extern "C"
