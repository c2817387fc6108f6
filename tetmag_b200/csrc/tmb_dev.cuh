// Device data structures and kernel launchers of the tetmag B200 library.
//
// Sparse operators are stored in SELL-32: rows are grouped in slices of 32
// consecutive rows; a slice is stored column-major with the width of its
// longest row, so thread r of a warp reads element k of row r at
// soff[slice] + 32*k + lane -- every load of a warp is one contiguous,
// 128/256-byte segment.  Padding entries point at the row itself with value 0.
// Several operators with the same pattern (K, grad_{x,y,z}, tGrad_{x,y,z})
// share one index array and keep one value array each, so a kernel that needs
// several of them (bulk DMI, divergence, gradient) reads the indices once.
//
// Values are FP64 (the plain path) or FP32 (the mixed path); vectors and all
// accumulations are FP64 in both.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace tmb {

#define TMB_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t _e = (call);                                                                    \
    if (_e != cudaSuccess)                                                                      \
      throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(_e) + " at " +   \
                               __FILE__ + ":" + std::to_string(__LINE__));                      \
  } while (0)

constexpr int kSlice = 32;
constexpr int kBlock = 256;

// rep > 1: the operator acts on rep interleaved copies of its vectors (shared-mesh replicas):
// state row g = i * rep + r is row i of the operator for replica r, and column j of row i
// gathers entry j * rep + r.  A warp then covers 32 replicas of one operator row, so the row's
// indices and values are loaded once for all of them (broadcast) and the gathers are contiguous.
struct SellView {
  int n;             // operator rows
  int nslice;
  const int* soff;   // nslice + 1 element offsets (multiples of 32)
  const int* col;    // padded column indices
  int rep;           // interleaved replicas (1: plain vectors)
  // value table of a dictionary-coded operator (values stored as one-byte indices into it, entry 0
  // is 0.0 for the padding); null for plain FP32 / FP64 values
  const double* tab;
};

// The value of one stored operator entry: the entry itself, or its table entry for one-byte codes.
template <typename V>
__device__ __forceinline__ double opval(V v, const double* /*tab*/) {
  return static_cast<double>(v);
}
template <>
__device__ __forceinline__ double opval<uint8_t>(uint8_t v, const double* tab) {
  return __ldg(tab + v);
}

struct CsrView {
  int n;
  const int* ptr;
  const int* col;
  int rep;
};

// Scalars of one PCG solve, resident on the device so that no kernel needs
// the host between iterations.
struct CgScalars {
  double rz, rz_new, pq, rr, bb, alpha, beta, tol2;
  int iter, done, maxit, status;
  unsigned int ticket[4];
};

// --- launchers (k_field.cu) --------------------------------------------------------------
struct LocalFieldArgs {
  int n;
  const double* m;          // 3N SoA state
  const double* hfix;       // 3N field added as is (applied + frozen demag), may be null
  const double* xc;         // N  exchange row scale  -2 A_i / V_i / Js_i
  const double* ku2;        // N  2 Ku_i / Js_i, null without uniaxial anisotropy
  const double* kax;        // 3N SoA easy axis
  const double* dmi_s;      // N  D_i / V_i / Js_i, null without bulk DMI
  const double* area;       // N  boundary node area (bulk DMI surface term)
  const double* nvn;        // 3N SoA node normal
  const double* idm_d;      // N  D_j (interfacial DMI), null otherwise
  const double* idm_a;      // N  D_i / Js_i (interfacial DMI), null otherwise
  const double* idm_b;      // N  1 / (V_i Js_i) (interfacial DMI)
  const double* cub_k1;     // N  Kc1 / Js (cubic anisotropy), null without it
  const double* cub_k2;     // N  Kc2 / Js
  const double* cub_ax;     // 9N SoA cubic axes: c1 (x, y, z), c2, c3, each N long
  const double* srf_k;      // N  Ks * node area / (V Js) (surface anisotropy), null without it
  double alpha;
  int precession;
  double* ydot;             // 3N out, may be null
  double* hout;             // 3N out (total field), may be null
  unsigned long long* torque_bits;  // max |m x H| (ordered bits), may be null
  const int* active = nullptr;  // device flag: the kernel does nothing while it is 0 (null: always runs)
};

// Step control of the device-side Dormand-Prince loop (one per context, device memory): the
// host sets t, t1, dt and the tolerances per segment, the graph of step attempts updates the rest.
struct StepCtl {
  double t, t1, dt, h;               // time, segment end, proposed step, step of this attempt
  double eps_abs, eps_rel;
  unsigned long long err_bits;       // scaled error of this attempt (ordered bits of a double)
  int active;                        // this attempt runs (set by k_step_begin)
  int last;                          // this attempt ends the segment
  int done;                          // the segment is finished (or failed): later attempts do nothing
  int status;                        // 0, or TMB_ERR_STEP on step-size underflow / attempt cap
  long long accepted, rejected, rhs, attempts, max_attempts;
};
// one attempt's kernels: begin (h, last), stage combination y + h sum a_j k_j (h from the control
// block), error reduction, acceptance copy (y <- y5, k1 <- k7 when accepted), update (t, dt, counts)
void launch_step_begin(StepCtl* c, cudaStream_t st);
void launch_rk_combine_dev(int n3, const double* y, const double* const* k, const double* a, int nk,
                           const StepCtl* c, double* out, cudaStream_t st);
void launch_rk_error_dev(int n3, const double* y, const double* k1, const double* const* k, const double* e, int nk,
                         StepCtl* c, cudaStream_t st);
void launch_step_accept(int n3, const StepCtl* c, double* y, const double* y5, double* k1, const double* k7,
                        cudaStream_t st);
void launch_step_update(StepCtl* c, int rhs_per_attempt, cudaStream_t st);

template <typename V>
void launch_local_field(const SellView& s, const V* K, const V* tg0, const V* tg1, const V* tg2, const V* gr0,
                        const V* gr1, const LocalFieldArgs& a, cudaStream_t st);

template <typename V>
void launch_divergence(const SellView& s, const V* tg0, const V* tg1, const V* tg2, const double* m,
                       const double* js, double inv_mu0, double* rhs, cudaStream_t st);

template <typename V>
void launch_gradient(const SellView& s, const V* g0, const V* g1, const V* g2, const double* u1,
                     const double* u2, const double* hext, double* hdem, double* hfix, cudaStream_t st);

void launch_normalize(int n, double* m, cudaStream_t st);
// Loads the code of every kernel of the local right-hand side (see k_field.cu), once per device.
void preload_local_kernels();
// Zhang-Li spin-transfer torque added to ydot (eta: 3N SoA per node)
template <typename V>
void launch_stt_add(const SellView& s, const V* g0, const V* g1, const V* g2, const double* m, const double* eta,
                    double alpha, double beta, double scale, double* ydot, cudaStream_t st,
                    const int* active = nullptr);
// energy terms, R interleaved replicas: kEnergyTerms partial sums per block (see k_field.cu);
// extra: cubic (raw Kc1, Kc2 [J/m^3], axes SoA 9N) and surface anisotropy (Ks * node area [J])
struct EnergyExtra {
  const double* kc1 = nullptr;
  const double* kc2 = nullptr;
  const double* cax = nullptr;
  const double* ksa = nullptr;
  const double* nvn = nullptr;
};
constexpr int kEnergyTerms = 7;
int energy_blocks(int n, int R);
void launch_energy_terms(int n, int R, const double* m, const double* hex, const double* hdmi, const double* hext,
                         const double* hdem, const double* js, const double* vol, const double* ku2, const double* kax,
                         const EnergyExtra& x, double* part, cudaStream_t st);
void launch_rk_combine(int n3, const double* y, const double* const* k, const double* a, int nk, double h,
                       double* out, cudaStream_t st);
void launch_rk_error(int n3, const double* y, const double* k1, const double* const* k, const double* e, int nk,
                     double h, double eps_abs, double eps_rel, unsigned long long* err_bits, cudaStream_t st);
void launch_fill(double* p, double v, size_t n, cudaStream_t st);
void launch_add(int n, const double* a, const double* b, double* out, cudaStream_t st);

// --- launchers (k_solver.cu) -------------------------------------------------------------
template <typename V>
void launch_jacobi(const SellView& s, const V* val, const double* dinv, const double* b, const double* xin,
                   double* xout, const int* done, cudaStream_t st);
// CSR kernels with tpr (1, 2, 4, 8, 16, 32) threads per row; csr_threads_per_row picks it from
// the average row length (about six entries per thread)
int csr_threads_per_row(long long nrows, long long nnz);
template <typename V>
void launch_csr_spmv(const CsrView& c, const V* val, const double* x, double* y, bool accumulate,
                     const int* done, cudaStream_t st, int tpr = 4);
template <typename V>
void launch_csr_jacobi0_residual(const CsrView& c, const V* val, const double* dinv, const double* b, double* x,
                                 double* r, const int* done, cudaStream_t st, int tpr);
// Coarse levels, one replica: the first sweep from zero with its residual, and the restriction of
// that residual as bc = M b (M = R - (R A) D_w^-1), in one launch (ta, tm threads per row).
template <typename V>
void launch_csr_pre_restrict(const CsrView& a, const V* aval, const double* dinv, const double* b, double* x,
                             double* r, int ta, const CsrView& m, const V* mval, double* bc, int tm, const int* done,
                             cudaStream_t st);
// Coarse levels: prolongation x += P c fused with the post-smoothing sweep, over the rows of A P
// (values apv) with P's values on the same pattern (pv); x0, r0 the pre-smoothed iterate and its
// residual.
template <typename V>
void launch_csr_prolong_smooth(const CsrView& m, const V* apv, const V* pv, const double* dinv, const double* x0,
                               const double* r0, const double* c, double* out, const int* done, cudaStream_t st,
                               int tpr);
template <typename V>
void launch_csr_jacobi(const CsrView& c, const V* val, const double* dinv, const double* b, const double* xin,
                       double* xout, const int* done, cudaStream_t st, int tpr);
// coarsest level with decoupled rows: x = D^-1 b, and the moves of the coupled rows to and from a
// compact vector for the dense solve
void launch_coarse_diag(int n, int rep, const double* dinv, const double* b, double* x, const int* done,
                        cudaStream_t st);
void launch_rows_move(int m, int rep, const int* idx, const double* src, double* dst, bool scatter,
                      const int* done, cudaStream_t st);
void launch_coarse_solve(int n, int ld, int rep, const double* inv, const double* b, double* x, const int* done,
                         cudaStream_t st, const float* invf = nullptr, int ldf = 0);

template <typename V>
void launch_cg_init(int n, const CsrView& lift, const V* lval, const int* cmask, const double* b,
                    double* bprime, double* x, cudaStream_t st);
template <typename V>
void launch_cg_residual(const SellView& s, const V* val, const double* bp, const double* x, double* r,
                        CgScalars* S, double* partials, cudaStream_t st);
void launch_cg_rz(int n, const double* r, const double* z, CgScalars* S, double* partials, bool first,
                  cudaStream_t st);
void launch_cg_update(int n, const double* p, const double* q, double* x, double* r, CgScalars* S,
                      double* partials, cudaStream_t st);
// fused variants used by the PCG iteration
template <typename V>
void launch_jacobi0_residual(const SellView& s, const V* val, const double* dinv, const double* b, double* x,
                             double* r, const int* done, cudaStream_t st);
template <typename V>
void launch_jacobi_rz(const SellView& s, const V* val, const double* dinv, const double* r, const double* xin,
                      double* z, CgScalars* S, double* partials, bool first, cudaStream_t st);
template <typename V>
void launch_cg_dir_spmv(const SellView& s, const V* val, const double* z, double* p, double* q, CgScalars* S,
                        double* partials, cudaStream_t st);
template <typename V>
void launch_cg_update_jacobi0(const SellView& s, const V* val, const double* dinv, const double* p, const double* q,
                              double* x, const double* r, double* r_new, double* X, double* Rres, CgScalars* S,
                              double* partials, cudaStream_t st);

// --- launchers (k_bem.cu) ----------------------------------------------------------------
void launch_bem_assemble(int nb, int ntri, const double* bxyz, const int* tri, const double* area,
                         const double* nrm, const double* solid, double* B, bool accurate, cudaStream_t st);
void launch_to_float(const double* src, float* dst, size_t n, cudaStream_t st);
template <typename V>
void launch_bem_gemv(int nb, const V* B, const V* xb, double* u2b, cudaStream_t st);
void launch_dirichlet_values(int n, const int* bindex, const double* u2b, double* b, cudaStream_t st);
// interleaved replicas (state row i * R + r): boundary panel X[r * xs + b], Dirichlet load from Y[r * nb + b]
template <typename V>
void launch_gather_rep(int nb, int R, const double* u, const int* idx, int xs, V* X, cudaStream_t st);
void launch_dirichlet_rep(int n, int R, const int* bindex, const double* Y, int nb, double* b, cudaStream_t st);
template <typename V>
void launch_gather(int nb, const double* u, const int* idx, V* out, cudaStream_t st);
size_t bem_ld(int nb);  // leading dimension (elements) of the row-major device BEM matrix
// Batched instances (disjoint components of one context): boundary values gathered to 32-element
// aligned per-component offsets, then one matvec per component's own matrix (tiles of up to R
// rows of one component: rows b + r * ld, columns x[0..ncols), results y[r]) or, for replicas
// sharing one matrix, one GEMM.
struct GemvTile {
  long long b;
  int x, y, ncols, nrows, ld, pad_;
};
template <typename V>
void launch_gather_pad(int nb, const double* u, const int* idx, const int* pos, V* out, cudaStream_t st);
template <typename V>
void launch_bem_gemv_tiles(int ntiles, const GemvTile* tiles, int rows_per_tile, const V* B, const V* x, double* y,
                           cudaStream_t st);
template <typename V>
void launch_bem_gemm(int nbc, int ncomp, const V* B, const V* X, int xs, double* Y, int num_sms, cudaStream_t st);

// 3xTF32 tensor-core GEMM of shared-mesh replicas (k_bem_tc.cu): Y = B X on FP32 B and X,
// FP64 Y ([replica][row]); Xhi / Xlo receive the TF32 split of X (same layout); split = K
// splits (partial sums added atomically into a zeroed Y);
// err is set when a barrier wait timed out.
bool bem_gemm_tc_supported(int nbc, size_t ld, int xs);
void launch_bem_gemm_tc(int nbc, int ncomp, size_t ld, const float* B, const float* X, int xs, float* Xhi,
                        float* Xlo, double* Y, int split, int stages, int* err, cudaStream_t st);

// --- hierarchical BEM matrix (k_hmatrix.cu) ---------------------------------------------
struct HBlockDev {
  int rb, m, cb, n;        // row / column range in cluster order
  long long off;           // dense tile offset (column-major m x n), near blocks
  long long uoff, voff;    // ACA scratch offsets (kmax columns each), admissible blocks
  long long used_off;      // offset of the m row flags in the ACA scratch
};
struct HNearRow {
  int rb, m, first, last;  // leaf row cluster and its near blocks [first, last)
};
struct HFarGroup {
  int rb, m, first, last;  // row cluster and its admissible blocks [first, last)
};
// Low-rank factors are stored with leading dimensions padded to a multiple of 4 entries (zero
// padding), so that every column of U and every row of V^T starts on a 16-byte boundary.
__host__ __device__ inline int pad4(int x) { return (x + 3) & ~3; }
// One term of the far-field product: t = V_l^T x[cb .. cb + n4) (n4 = pad4(n)), V_l at offset v;
// its column of U starts at offset u.
struct HTerm {
  long long v, u;
  int n4, cb;
};
template <typename T>
struct HMatView {
  int nb = 0, nrows = 0, ngroups = 0;
  long long nterms = 0;
  const int* gidx = nullptr;             // permuted position -> boundary node (mesh numbering)
  const HNearRow* near_rows = nullptr;
  const HBlockDev* near = nullptr;
  const T* D = nullptr;                  // dense tiles
  const HBlockDev* far = nullptr;
  const int* rank = nullptr;
  const long long* uoff = nullptr;       // compact U offsets (column-major pad4(m) x rank)
  const long long* voff = nullptr;       // compact V offsets (column-major pad4(n) x rank)
  const T* U = nullptr;
  const T* V = nullptr;
  const HFarGroup* groups = nullptr;     // row clusters, largest work first
  const HTerm* terms = nullptr;          // every term of every admissible block, block by block
  const long long* toff = nullptr;       // first term of each admissible block, then the term count
  double* t = nullptr;                   // the terms' values V^T x (nterms)
};
// Where the entries of the boundary matrix (in cluster order) come from: the dense FP64
// matrix (B != nullptr, row-major with leading dimension ld, rows/columns perm[i]) or the
// boundary mesh itself, evaluated on the fly.
struct HSource {
  const double* B = nullptr;
  size_t ld = 0;
  const int* perm = nullptr;
  int nb = 0, ntri = 0;
  const double* xp = nullptr;     // 3 per cluster position: node coordinates
  const int* tri = nullptr;       // 3 per triangle: cluster positions, mesh vertex order
  const double* tarea = nullptr;  // triangle areas
  const double* tnrm = nullptr;   // outward unit normals, 3 per triangle
  const int* adj_ptr = nullptr;   // position -> [adj_ptr[p], adj_ptr[p+1]) in adj
  const int2* adj = nullptr;      // (triangle, local vertex 0..2) touching the position
  const double* solid = nullptr;  // interior solid angle per position
};
// dense tiles of the inadmissible blocks: copied from B, or assembled from the mesh with the
// reference Lindholm formula (k_bem_assemble.cu)
void launch_h_near_gather(int nblk, const HBlockDev* blk, const HSource& src, double* d64, float* d32,
                          cudaStream_t st);
void launch_h_near_mesh(int nblk, const HBlockDev* blk, const HSource& src, double* d64, float* d32,
                        cudaStream_t st);
void launch_h_aca(int nblk, const HBlockDev* blk, const HSource& src, double* Us, double* Vs, unsigned char* used,
                  int kmax, double eps_tight, double eps_loose, double gscale, int* out_rank, cudaStream_t st);
// per low-rank block {|A x|^2, |A x - U64 V64^T x|^2, |A x - U32 V32^T x|^2} for a fixed probe x
// (ranks <= 128)
void launch_h_verify(int nblk, const HBlockDev* blk, const HSource& src, const int* rk64, const long long* uo64,
                     const long long* vo64, const double* U64, const double* V64, const int* rk32,
                     const long long* uo32, const long long* vo32, const float* U32, const float* V32, double* out,
                     cudaStream_t st);
template <typename T>
void launch_h_compact(int nblk, const HBlockDev* blk, const double* Us, const double* Vs, const long long* du,
                      const long long* dv, const int* rank, T* U, T* V, cudaStream_t st);
// y (cluster order, FP64) = H u[boundary]; then b[node] = y[pos[node]] (0 off the boundary)
template <typename T>
void launch_h_matvec(const HMatView<T>& H, const double* u, double* y, T* xp, const int* pos, int n, double* bdir,
                     cudaStream_t st);
// Transposed product y (cluster order, FP64) = H^T u[boundary], from a view whose near-field
// groups are the leaf column clusters (near_rows: column cluster, its blocks [first, last) of
// `near` ordered by column), whose far-field groups, terms and offsets are the admissible blocks
// ordered by column cluster with U and V exchanged (t = U^T x, then y += V t); the dense tiles are
// the forward ones, read by columns.
template <typename T>
void launch_h_matvec_t(const HMatView<T>& Ht, const double* u, double* y, T* xp, cudaStream_t st);

// --- H2 matrix (nested cluster bases, h2.cpp) -----------------------------------------------
// One cluster of the tree: position range, ranks of its row and column bases, tree links,
// offsets of its coefficients (FP64 vectors xh, yh) and of its basis data (-1: none):
//   rl  leaf row basis, m x kr column-major
//   rt  row transfer E, kr x kr_parent column-major (the parent's basis restricted to this
//       cluster is this cluster's basis times E)
//   cl  leaf column basis, m x kc row-major
//   ct  column transfer, stored transposed: kc_parent x kc column-major
struct H2Node {
  int begin, m, kr, kc;
  int parent, child0, child1;
  int xo, yo;
  long long rl, rt, cl, ct;
};
struct H2Run {              // a row cluster and its admissible blocks [first, last)
  int t, first, last;
};
struct H2Blk {              // admissible block: column cluster, coupling offset (kr_t x kc_s, column-major)
  int s;
  long long so;
};
template <typename T>
struct H2View {
  int nb = 0, nleaf = 0, nruns = 0;
  const int* gidx = nullptr;
  int nrows = 0;                           // near field: the H-matrix's dense leaf tiles
  const HNearRow* near_rows = nullptr;
  const HBlockDev* near = nullptr;
  const T* D = nullptr;
  const H2Node* node = nullptr;
  const int* leaves = nullptr;             // leaf cluster ids
  const int* lvl_nodes = nullptr;          // non-leaf cluster ids grouped by depth
  const T* rowb = nullptr;
  const T* colb = nullptr;
  const H2Run* runs = nullptr;
  int nblk = 0;
  const int* brow = nullptr;               // row cluster of every admissible block
  const H2Blk* blk = nullptr;
  const T* S = nullptr;
  double* xh = nullptr;
  double* yh = nullptr;
  long long nyh = 0;
};
// the same product through the H2 matrix: near tiles, column basis upward pass, couplings, row
// basis downward pass; up / down: host lists of the depths that have work (deepest first / root first)
// up / down: (offset into lvl_nodes, count) of the clusters of each depth with work, in launch
// order (deepest first for the upward pass, root first for the downward pass)
template <typename T>
void launch_h2_matvec(const H2View<T>& H, const double* u, double* y, T* xp, const int* pos, int n, double* bdir,
                      const std::vector<std::pair<int, int>>& up, const std::vector<std::pair<int, int>>& down,
                      cudaStream_t st);

// --- discrete adjoint of the fixed-step integration (k_adjoint.cu) -------------------------
struct AdjPreArgs {
  int n;
  const double* m;       // 3N stage state
  const double* H;       // 3N total field at the stage
  const double* abar;    // 3N adjoint weight of the stage's right-hand side
  double alpha;
  int precession;
  const double* js;      // N  Js (uniaxial gradient), with kax
  const double* kax;     // 3N easy axis
  double* mu;            // 3N out: (df/dH)^T abar
  double* g;             // 3N out: (df/dm at fixed H)^T abar
  double* dku;           // N  accumulated dJ/dKu, may be null
  double* zpart;         // one partial sum of mu_z per block, may be null
};
struct AdjLocalArgs {
  int n;
  const double* mu;      // 3N
  const double* xc;      // N  exchange row scale
  const double* ku2;     // N  2 Ku / Js, null without uniaxial anisotropy
  const double* kax;     // 3N
  const double* idm_d;   // N  D (interfacial DMI), null otherwise
  const double* idm_b;   // N  1 / (V Js), null without interfacial DMI
  const double* dmi_s;   // N  D / (V Js) (bulk DMI), null otherwise
  const double* area;    // N  boundary node areas (bulk DMI surface term)
  const double* nvn;     // 3N boundary node normals (bulk DMI surface term)
  const double* vol;     // N  node volumes
  const double* js;      // N
  const double* q;       // 3N -grad a1 of the transposed demag chain, null without demag
  double inv_mu0;
  double* g;             // 3N in/out
};
void launch_set_hz(int n, const double* hbase, double hz, double* hext, cudaStream_t st);
void launch_lincomb(int n3, double* out, double c0, const double* v0, double c1, const double* v1, double c2,
                    const double* v2, cudaStream_t st);
void launch_rk4_final(int n3, double* y, const double* k1, const double* k2, const double* k3, const double* k4,
                      double h, cudaStream_t st);
void launch_normalize_keep(int n, double* y, double* zn, cudaStream_t st);
void launch_adj_normalize(int n, const double* y, const double* zn, double* lam, cudaStream_t st);
int adj_pre_blocks(int n);
void launch_adj_pre(const AdjPreArgs& a, cudaStream_t st);
template <typename V>
void launch_adj_local(const SellView& s, const V* K, const V* tg0, const V* tg1, const V* gr0, const V* gr1, const V* gr2,
                      const AdjLocalArgs& a, cudaStream_t st);
int bem_gemv_t_chunks(int nb, int num_sms);
template <typename V>
void launch_bem_gemv_t(int nb, const V* B, const double* x, double* part, int nchunk, double* out, cudaStream_t st);
void launch_mask_constrained(int n, const int* cmask, const double* c, double* out, cudaStream_t st);
template <typename V>
void launch_lift_t(int n, const CsrView& lt, const V* lval, const int* cmask, const double* c, const double* x,
                   double* out, cudaStream_t st);
void launch_scatter_add(int nb, const int* idx, const double* z, double* a, cudaStream_t st);

// Count of kernel launches issued by this library (all contexts), for benchmarking.
long long launch_count();
void note_launch();
void note_launches(long long k);  // k kernels launched at once (a CUDA graph)

inline int grid_for(long long n, int block = kBlock) {
  long long g = (n + block - 1) / block;
  return int(g < 1 ? 1 : g);
}

// Programmatic dependent launch for chains of small dependent kernels (the CG iteration and its
// V-cycle): a kernel launched by launch_pdl may be scheduled while its predecessor in the stream
// still runs, so that its launch and CTA placement overlap the predecessor's execution instead
// of following its completion.  Such a kernel calls pdl_enter() first, in every CTA: it waits
// until the predecessor grid has completed and its writes are visible (griddepcontrol.wait),
// then lets its own successor be scheduled (griddepcontrol.launch_dependents).  Waiting before
// triggering keeps at most one pre-scheduled grid behind the running one; every CTA waits, so
// completion stays ordered along the chain.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}
template <typename... P, typename... A>
inline void launch_pdl(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  TMB_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
}

}  // namespace tmb
