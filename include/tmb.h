/*
 * tmb.h -- C ABI of the tetmag B200 library (libtmb.so).
 *
 * A drop-in replacement for the per-step effective-field and LLG
 * right-hand-side evaluation of tetmag (R-Hertel/tetmag v1.7.7), including
 * its FEM-BEM demagnetising-field chain.  Plain C types only: caller-owned
 * buffers, int status codes, an opaque context per mesh.  Every entry point
 * returns TMB_OK (0) or a positive TMB_ERR_* code; tmb_last_error() gives
 * the message of the last failure on the calling thread.
 *
 * Vectors of nodal 3-vectors use tetmag's layout: SoA / column-major
 * [x(0..N-1), y(0..N-1), z(0..N-1)], length 3N (main/TheLLG.cpp:156).  Fields
 * are in A/m, reduced time t*gamma/(1+alpha^2) (specs/SimulationData.cpp:52-57).
 * Entry points that take a `ptr_kind` accept host (TMB_PTR_HOST) or device
 * (TMB_PTR_DEVICE) pointers; device-pointer calls are ordered on the context
 * stream and do not synchronise the host except where stated.
 *
 * Threading: a context is used by one host thread at a time.
 */
#ifndef TMB_H_
#define TMB_H_

#ifdef __cplusplus
extern "C" {
#endif

#define TMB_OK 0
#define TMB_ERR_ARG 1          /* invalid argument or size */
#define TMB_ERR_CUDA 2         /* CUDA runtime error */
#define TMB_ERR_NOCONVERGE 3   /* an iterative solve hit its iteration cap */
#define TMB_ERR_STATE 4        /* call out of order (e.g. no mesh set) */
#define TMB_ERR_NAN 5          /* NaN / Inf detected (field, torque, solver breakdown) */
#define TMB_ERR_STEP 6         /* integrator step-size underflow or step cap */
#define TMB_ERR_INTERNAL 7

#define TMB_FP64 0             /* plain path: FP64 operators and vectors */
#define TMB_MIXED 1            /* FP32 operator values (the CG's own operator FP64), FP64 vectors, reductions, coarse solve, step control */

#define TMB_PTR_HOST 0
#define TMB_PTR_DEVICE 1

typedef struct tmb_ctx tmb_ctx;
typedef struct tmb_mesh tmb_mesh;
typedef struct tmb_solver tmb_solver;

const char* tmb_last_error(void);
int tmb_version(void);
/* Kernels launched by this library so far, all contexts (no reference counterpart; for benchmarking). */
int tmb_kernel_launches(long long* count);

/* ---------------------------------------------------------------------------------------
 * Host mesh preprocessing.  Replaces PreprocessMesh::prepareAllMatrices
 * (preproc/FEMprocessing.cpp:70-93), MeshBoundary::extractFeatures
 * (preproc/Boundary.cpp:47-55) and BEMprocessing::calculateSolidAngles
 * (preproc/BEMprocessing.cpp:358-372).  xyz: N x 3 row-major (mesh units);
 * tets: E x 4 node ids.
 * ------------------------------------------------------------------------------------- */
int tmb_mesh_create(int nx, int ntet, const double* xyz, const int* tets, tmb_mesh** out);
int tmb_mesh_destroy(tmb_mesh* mesh);
/* info[0..5] = nx, ntet, nnz (shared operator pattern), nb (boundary nodes), ntri (boundary triangles), 0 */
int tmb_mesh_info(const tmb_mesh* mesh, long long* info);
/* CSR arrays of the shared pattern: rowptr[N+1], col[nnz]; each value array has nnz entries.
 * tg* are tetmag's msh.tGrad* (not negated).  Any output pointer may be NULL. */
int tmb_mesh_get_operators(const tmb_mesh* mesh, int* rowptr, int* col, double* stiff, double* gx, double* gy,
                           double* gz, double* tgx, double* tgy, double* tgz, double* node_vol);
/* bnodes[nb] ascending; tri[3*ntri] global ids; tri_area[ntri]; tri_normal[3*ntri] outward (row-major);
 * node_area[N]; node_normal[3N] SoA; solid_angle[nb].  Any output pointer may be NULL. */
int tmb_mesh_get_boundary(const tmb_mesh* mesh, int* bnodes, int* tri, double* tri_area, double* tri_normal,
                          double* node_area, double* node_normal, double* solid_angle);

/* ---------------------------------------------------------------------------------------
 * Context: one mesh on one device.
 * ------------------------------------------------------------------------------------- */
int tmb_ctx_create(int device, tmb_ctx** out);       /* SetDevice::set (gpu/SetDevice.cu:41-60) */
int tmb_ctx_destroy(tmb_ctx* ctx);
int tmb_ctx_set_stream(tmb_ctx* ctx, void* cuda_stream);  /* NULL: the context's own stream */
int tmb_set_precision(tmb_ctx* ctx, int precision);   /* TMB_FP64 (default) or TMB_MIXED */

/* Operators from a preprocessed mesh, or from tetmag's own MeshData arrays
 * (main/TheLLG.cpp:88-108 uploads K; main/DemagField.cpp:65-89 keeps grad,
 * tGrad, the Dirichlet and Neumann matrices).  The caller's CSR must hold K,
 * grad* and tGrad* on one pattern; node_normal is SoA 3N. */
int tmb_set_mesh(tmb_ctx* ctx, const tmb_mesh* mesh);
int tmb_set_operators(tmb_ctx* ctx, int nx, int nnz, const int* rowptr, const int* col, const double* stiff,
                      const double* gx, const double* gy, const double* gz, const double* tgx, const double* tgy,
                      const double* tgz, const double* node_vol, int nb, const int* bnodes,
                      const double* node_area, const double* node_normal);

/* Dense double-layer BEM matrix.  tmb_bem_assemble builds it on the device from the
 * mesh boundary (BEMprocessing::assembleLaplaceBEMmatrix, preproc/BEMprocessing.cpp:375-411);
 * tmb_set_bem_dense takes tetmag's MeshData::laplaceBEM (Nb x Nb, column-major). */
int tmb_bem_assemble(tmb_ctx* ctx, const tmb_mesh* mesh);
/* formula 0: tmb_bem_assemble (tetmag's arithmetic).  formula 1: the same weights in a
 * far-field-accurate arithmetic (solid angle by atan2 of the triple product, log1p edge terms):
 * tetmag's acos form drifts from the exact weights several hundred nm from a nm-sized triangle
 * (row sums of a 500 nm film's matrix miss -1 by up to ~1e-3); this form keeps them to ~1e-13.
 * No tetmag counterpart; it is the FP64 reference for the hierarchical matrix. */
int tmb_bem_assemble_ex(tmb_ctx* ctx, const tmb_mesh* mesh, int formula);
int tmb_set_bem_dense(tmb_ctx* ctx, int nb, const double* B_colmajor);
/* Batched instances in one context: the mesh given to tmb_set_mesh / tmb_set_operators is a
 * disjoint union of ncomp meshes, component c owning nodes [node_offsets[c], node_offsets[c+1])
 * (the operators must not couple components).  Each component is one tetmag problem: its own
 * pinned Neumann node (node N_c / 2 of the component, main/DemagField.cpp:80) and its own dense
 * BEM block, assembled by tmb_bem_assemble(_ex) afterwards; the boundary matvec runs for all
 * components in one launch.  shared_bem = 1 declares the components identical copies of one
 * mesh (checked: operators and boundary numbering) that share one BEM block: the matvec is then
 * one GEMM, B times the replicas' boundary values.  Solves, step control and torques are taken
 * over all components together (one set of CG iterations and one step size for the batch).
 * No tetmag counterpart (tetmag runs one mesh per process).  Call before tmb_bem_assemble; the
 * hierarchical BEM and tmb_set_bem_dense / tmb_get_bem_dense need ncomp = 1. */
int tmb_set_components(tmb_ctx* ctx, int ncomp, const int* node_offsets, int shared_bem);
/* R interleaved replicas of the context's single mesh (same operators, material and BEM matrix;
 * own state and applied field each): every state vector (m, ydot, fields, tmb_set_applied_field)
 * then holds 3 * N * R doubles, component d of node i of replica r at d * N * R + i * R + r.
 * Every operator row is applied to the R replicas at once (a warp reads the row's indices and
 * values once for 32 replicas), the two solves are one CG over the replicas, and the boundary
 * product is one GEMM (tmb_set_bem_gemm_kind).  Call after tmb_set_mesh and before
 * tmb_bem_assemble / tmb_set_bem_dense; material arrays stay per node (N).  Not with
 * tmb_set_components, the hierarchical BEM or the adjoint.  No tetmag counterpart (tetmag runs
 * one magnetisation per process). */
int tmb_set_replicas(tmb_ctx* ctx, int nrep);
/* Boundary GEMM of shared-mesh replicas on the mixed path: 1 (default) the 3xTF32 tensor-core
 * kernel (tcgen05, FP32 accumulation per K split, FP64 sum of the splits), 0 the CUDA-core kernel
 * (FP32 products, FP64 accumulation).  The FP64 path always uses the CUDA-core kernel.  The K
 * split and the TMA ring depth of the tensor-core kernel are chosen by timing the candidates on
 * first use.  No tetmag
 * counterpart (tetmag multiplies one boundary vector at a time, main/DemagField.cpp:145-147). */
int tmb_set_bem_gemm_kind(tmb_ctx* ctx, int tensor_cores);
/* out[0..10]: tensor cores on, chosen K split, tuned ms per launch for splits 1..8 (the best TMA
 * ring depth of each; 0: not tried), chosen ring depth (2, 3 or 4 stages; 0: not tuned yet). */
int tmb_bem_gemm_info(tmb_ctx* ctx, double* out);
int tmb_get_bem_dense(tmb_ctx* ctx, double* B_colmajor);

/* Hierarchical compression of the dense matrix (replaces H2Lib's setupH2MatrixC /
 * H2_mvp_sub, main/h2interface.c:77-95, 373-399): cluster tree over bxyz (Nb x 3, boundary
 * order) with leaf size `leaf` (<= 32; tetmag uses clf = 32), admissibility
 * min(diam) <= eta * dist (tetmag: eta = 2), dense leaf tiles and adaptive-cross-approximation
 * low-rank blocks: FP32 terms to eps_mixed for the mixed path, FP64 terms to eps_fp64 for the
 * plain path (at most kmax <= 128 terms per block).  bnormal (Nb x 3 node normals, may be NULL) lets
 * the cluster tree separate faces of different orientation first, so that every low-rank block
 * couples one smooth piece of surface to another.  Needs the dense FP64 matrix on the device
 * (tmb_bem_assemble / tmb_set_bem_dense); keep_dense = 0 releases it afterwards.  The demag
 * chain then uses the hierarchical matvec (tmb_set_bem_mode switches back). */
int tmb_bem_compress(tmb_ctx* ctx, const double* bxyz, const double* bnormal, int leaf, double eta,
                     double eps_mixed, double eps_fp64, int kmax, int keep_dense);
/* Hierarchical matrix straight from the mesh boundary, without the dense matrix: same
 * partition and ranks as tmb_bem_compress (the cluster tree splits faces by node-normal
 * orientation), dense tiles with tetmag's Lindholm arithmetic, and low-rank blocks from entries
 * evaluated on the device in a far-field-accurate form of the same weights (the reference form
 * loses up to ~10% of a weight several hundred nm from a nm-sized triangle, which is noise
 * that cross approximation cannot compress).  This is the c2-sized path where H2Lib's own
 * assembly replaces the dense matrix (setupH2MatrixC, main/h2interface.c:315-399). */
int tmb_bem_build_h(tmb_ctx* ctx, const tmb_mesh* mesh, int leaf, double eta, double eps_mixed, double eps_fp64,
                    int kmax);
/* Accuracy measure of the next tmb_bem_compress / tmb_bem_build_h.  matrix_share = 0 (the
 * default): each admissible block's cross approximation stops at eps relative to the block's own
 * Frobenius norm.  matrix_share = s > 0: a block may also stop at its share of a matrix-relative
 * budget, eps * s * sqrt(m n) * ||N||_F / Nb, where N is the dense leaf tiles (the near field,
 * which holds the diagonal); blocks far from each other, whose entries are orders of magnitude
 * below the matrix's, then keep the few terms the product needs.  tetmag's recompression
 * truncates relative to each cluster's total matrix rather than per block for the same reason
 * (new_releucl_truncmode, main/h2interface.c:328, 362-369). */
int tmb_set_bem_accuracy(tmb_ctx* ctx, double matrix_share);
int tmb_set_bem_mode(tmb_ctx* ctx, int mode);  /* 0 dense, 1 hierarchical, 2 H2 */
/* H2 matrix: the hierarchical matrix's admissible blocks (its FP64 terms) recompressed into nested
 * cluster bases -- orthogonal row and column bases per cluster, leaf bases explicit and parents'
 * through transfer matrices, one small coupling matrix per admissible block -- truncated at
 * eps_fp64 (the plain path's copy) and eps_mixed (the mixed path's FP32 copy) relative to the
 * largest singular value of each cluster's total matrix, ranks at most kmax (<= 64); the near
 * field stays the hierarchical matrix's dense tiles.  Restates H2Lib's recompression
 * (compress_hmatrix_h2matrix at 1e-5, main/h2interface.c:362-369) and the H2 matvec of
 * H2_mvp_sub (:77-95).  Needs tmb_bem_build_h / tmb_bem_compress first; selects mode 2. */
int tmb_bem_h2(tmb_ctx* ctx, double eps_fp64, double eps_mixed, int kmax);
/* out[8 * w + 0..7] for w = 0 (FP64 copy), 1 (FP32 copy): built, bytes streamed per matvec
 * (near tiles + bases + couplings), coupling bytes, basis + transfer bytes, max row rank, max
 * column rank, build ms, tolerance. */
int tmb_bem_h2_info(tmb_ctx* ctx, double* out);
/* out[0..11]: mode, dense tiles, low-rank blocks, FP64 terms, FP32 terms, FP64 bytes, FP32 bytes,
 * dense entries (Nb^2), blocks at the rank cap, max FP64 rank, compression ms, built flag */
int tmb_bem_info(tmb_ctx* ctx, double* out);
/* Accuracy of the low-rank blocks against the dense FP64 matrix (still on the device:
 * keep_dense = 1) for a fixed probe vector.  out[0..3]: relative error of the low-rank part
 * with FP64 terms, with FP32 terms, worst block relative error FP64, FP32.  block_out (may be
 * NULL; 6 per low-rank block, partition order): |A x|, FP64 error, FP32 error, FP64 rank, FP32
 * rank, 1 if the block hit the rank cap.  Diagnostic only: tetmag's call path has no
 * counterpart. */
int tmb_bem_verify(tmb_ctx* ctx, double* block_out, double* out);
/* The boundary product alone, DemagField::mvp (main/DemagField.cpp:139-152: denseMVP or
 * h2MVP -> H2_mvp_sub, main/h2interface.c:77-95): y = B x (transpose = 0) or B^T x (1) for
 * boundary vectors of Nb entries in boundary-node order (tmb_mesh_get_boundary's bnodes), with
 * the context's boundary matrix form (tmb_set_bem_mode) and precision.  The transposed
 * product (the adjoint's) exists for the dense and hierarchical forms; one component, no
 * replicas.  Host pointers synchronise. */
int tmb_bem_apply(tmb_ctx* ctx, const double* x, double* y, int transpose, int ptr_kind);

/* Material per node (SimulationData, specs/SimulationData.cpp:125-163): Js [T], A [J/m]
 * already divided by scale^2, Ku [J/m^3], ku_axis 3N SoA, D [J/m^2] already divided by
 * scale (bulk DMI, main/EffFieldCalc.cpp:159-170).  Ku, ku_axis, D may be NULL. */
int tmb_set_material(tmb_ctx* ctx, const double* Js, const double* A, const double* Ku, const double* ku_axis,
                     const double* D, double alpha);
/* DMI form applied with the material's D: 0 bulk (tetmag's, main/EffFieldCalc.cpp:159-170, the
 * default), 1 interfacial (thin films with the interface normal along z; no tetmag
 * counterpart): H = -(1/V) dE/dm of E = sum_i V_i D_i [m_z div m - (m . grad) m_z]_i with
 * tetmag's nodal gradient operators, divided by Js. */
int tmb_set_dmi_kind(tmb_ctx* ctx, int kind);
/* Cubic anisotropy (EffFieldCalc::cubicAnisotropyField, main/EffFieldCalc.cpp:249-272): Kc1, Kc2
 * [J/m^3] per node, axes 9 per node (node i: the three cubic axes c1, c2, c3, each x, y, z, as
 * SimulationData::cubicAxes' columns).  H += C dE/dalpha / Js with alpha = C^T m.  Kc1 = NULL
 * removes the term.  Call after tmb_set_mesh; the 1/Js scaling follows tmb_set_material. */
int tmb_set_cubic_anisotropy(tmb_ctx* ctx, const double* Kc1, const double* Kc2, const double* axes);
/* Surface anisotropy (EffFieldCalc::surfaceAnisotropyField, main/EffFieldCalc.cpp:128-149): Ks per
 * node [J/m^2, already divided by scale as specs/SimulationData.cpp:47], multiplied by the node's
 * boundary area; H += -2 Ks a nm (nm m - n) / (V Js) with n the node normal, nm = m . n.  NULL
 * removes the term. */
int tmb_set_surface_anisotropy(tmb_ctx* ctx, const double* Ks);
/* Zhang-Li spin-transfer torque (TheLLG::sttDynamics, main/TheLLG.cpp:201-220; u term
 * calcUtermSTT, :402-415): eta = 3N SoA per node (tetmag's eta_jx, eta_jy, eta_jz: current
 * density times the spin-polarisation factor, specs/ProgramSpecs.cpp:395-420), beta the
 * non-adiabaticity, scale the current-pulse value (1 for a constant current; the caller updates
 * it for a pulse).  Adds s [-(beta - alpha) m x U - (1 + alpha beta) m x (m x U)] with
 * U = sum_d eta_d (grad_d m) to every right-hand side; the max-torque value excludes it (as
 * main/TheLLG.cpp:437).  eta = NULL removes it. */
int tmb_set_stt(tmb_ctx* ctx, const double* eta, double beta, double scale);
/* Applied field, 3N SoA in A/m (TheLLG::setZeemanField, main/TheLLG.cpp:477-483). */
int tmb_set_applied_field(tmb_ctx* ctx, const double* hext, int ptr_kind);
/* precession = 0 selects the "remove precession" dynamics (TheLLG::noPrecession, main/TheLLG.cpp:180-199). */
int tmb_set_llg_options(tmb_ctx* ctx, int precession);
/* Relative residual tolerance and iteration cap of both demag solves
 * ("CG tolerance", specs/ProgramSpecs.cpp:70; maxiter main/AMGCLSolver.cpp:42). */
int tmb_set_solver_params(tmb_ctx* ctx, double tol, int maxiter);

/* DemagField::calcField (main/DemagField.cpp:92-94): m (3N) -> H_dem (3N).  The result
 * also becomes the frozen demag field used by the right-hand side. hdem may be NULL. */
int tmb_demag_field(tmb_ctx* ctx, const double* m, double* hdem, int ptr_kind);
/* One full field evaluation: the demag chain on m, then the local field and the LLG
 * right-hand side -- TheLLG::rhs with "freeze demag = false", whose calcDemagField refreshes
 * H_dem inside the right-hand side (main/TheLLG.cpp:278-283, 458-462).  hdem may be NULL. */
int tmb_field_eval(tmb_ctx* ctx, const double* m, double* ydot, double* hdem, int ptr_kind);
/* TheLLG::setHdem (main/TheLLG.cpp:508-510). */
int tmb_set_demag_frozen(tmb_ctx* ctx, const double* hdem, int ptr_kind);
/* Total effective field with the frozen demag (TheLLG::totalEffectiveField, main/TheLLG.cpp:238-254). */
int tmb_effective_field(tmb_ctx* ctx, const double* m, double* h, int ptr_kind);
/* The CVODE right-hand side (TheLLG::rhs / rhs_d, main/TheLLG.cpp:670-711,
 * gpu/LLGWrapper.cu:213-228): ydot = -m x H - alpha m x (m x H).  t is reduced time. */
int tmb_llg_rhs(tmb_ctx* ctx, double t, const double* y, double* ydot, int ptr_kind);
/* tmb_llg_rhs for host vectors y and ydot (3N), without allocating device memory -- no
 * counterpart in the reference.  For callers that cannot allocate on the device while they
 * evaluate the right-hand side (a fixed device-memory budget, a loop that must not pay
 * cudaMalloc's device-wide synchronisation, a stream under capture by other work).  y and
 * ydot are staged through one file-scope device array of 2 x 3 x 65536 doubles (3 MiB, held by
 * every GPU that loads the library until exit); contexts with nodes x replicas above 65536 get
 * TMB_ERR_ARG.  tmb_ctx_create resolves that array's device address for its device
 * (cudaGetSymbolAddress, which also loads the module holding the array) and loads the kernels
 * this entry point launches (with lazy module loading a kernel's code is otherwise loaded at its
 * first launch), so no call of this entry point, the first included, allocates.  Every call shares the array: calls that overlap
 * on the GPU (other threads, other contexts on the same device) race, so serialise them.
 * Nothing in the array needs to start at zero: each call overwrites the 6N entries it uses.
 * Synchronises. */
int tmb_llg_rhs_noalloc(tmb_ctx* ctx, double t, const double* y, double* ydot);
/* TheLLG::getMaxTorque (main/TheLLG.cpp:426-439): mu0 * max_i |m_i x H_i| with the frozen demag.
 * Synchronises.  Returns TMB_ERR_NAN if the torque is not finite. */
int tmb_max_torque(tmb_ctx* ctx, const double* m, double* out, int ptr_kind);
/* m <- m / |m| per node (TheSimulation::normalizeMag, main/TheSimulation.cpp:404-411). */
int tmb_normalize(tmb_ctx* ctx, double* m, int ptr_kind);

/* The simulation loop of TheSimulation::start (main/TheSimulation.cpp:231-311) with frozen
 * demag: per segment of segment_ps, refresh H_dem, integrate the LLG with an adaptive
 * Dormand-Prince 5(4) stepper on the device (TheLLG::IntegrateODEINT's stepper,
 * main/TheLLG.cpp:514-572), normalise.  stats[0..11] = accepted steps, rejected steps,
 * rhs evaluations, demag evaluations, Neumann CG iterations, Dirichlet CG iterations,
 * final max torque [T], final dt (reduced), segments, 0, 0, 0.  Synchronises. */
int tmb_relax(tmb_ctx* ctx, double* m, double duration_ps, double segment_ps, double eps_abs, double eps_rel,
              double* stats, int ptr_kind);
/* Energy densities [J/m^3] of TheSimulation::calculateEnergies (main/TheSimulation.cpp:385-396):
 * out[0..7] = total, demag (DemagField::getDemagEnergy, main/DemagField.cpp:97-99), exchange
 * (EffFieldCalc::calcExchangeEnergy, main/EffFieldCalc.cpp:65-69), uniaxial with tetmag's offset
 * sum V Ku (:86-95), Zeeman (TheLLG::getZeemanEnergy, main/TheLLG.cpp:345-348), cubic
 * (cubicAnisotropyEnergy, :232-247), surface (surfaceAnisotropyEnergy, :108-126), DMI
 * (-1/2 sum V Js H_dmi . m, bulk or interfacial), each divided by the total node volume.  The
 * demag field is evaluated for m when a BEM matrix is set (the frozen one otherwise).  With
 * components or replicas the sums run over the whole batch.  Synchronises. */
int tmb_energies(tmb_ctx* ctx, const double* m, double* out, int ptr_kind);
/* Time-dependent applied field: a piecewise-linear Bz(t) through ns samples [T] spaced uniformly
 * over [t0_ps, t1_ps] (held at the end values outside), added as Bz/mu0 to the z component of the
 * applied field during tmb_step_rk4 / tmb_adjoint_rk4.  ns = 0 removes it.  Generalises tetmag's
 * field pulse (TheLLG::setPulseField, main/TheLLG.cpp:320-332). */
int tmb_set_bz_pulse(tmb_ctx* ctx, int ns, const double* bz_tesla, double t0_ps, double t1_ps);
/* Fixed-step integration: nsteps steps of dt_ps from t0_ps, each nsub classical RK4 substeps with
 * the full effective field (demag refreshed, main/TheLLG.cpp:238-254, 670-711) at every stage,
 * then m <- m/|m| if normalize (main/TheSimulation.cpp:404-411).  m (3N SoA) in / out.
 * stats (may be NULL, 8): [0] right-hand-side evaluations, [3] CG iterations.  The applied field
 * is restored afterwards.  Synchronises.  No tetmag counterpart for the fixed step (tetmag's CVODE
 * is adaptive); this is the map that tmb_adjoint_rk4 differentiates. */
int tmb_step_rk4(tmb_ctx* ctx, double* m, int nsteps, double dt_ps, int nsub, double t0_ps, int normalize,
                 double* stats, int ptr_kind);
/* Discrete adjoint of tmb_step_rk4 for the objective J = sum_k w[k] y_N[k] (w: 3N SoA, e.g. the
 * volume weights of mean m_z): runs the forward map from m0 keeping a checkpoint every ckpt_every
 * steps, then per checkpoint interval (last first) recomputes its steps keeping the stage states
 * and fields, and transposes them.  Outputs: m_final (3N), J, and the gradients dJ/dm0 (3N),
 * dJ/dKu per node (N, with the material's easy axis; Ku may be 0) and dJ/dbz (ns samples of
 * tmb_set_bz_pulse, host memory).  grad_m0, grad_ku, grad_bz, J, stats may be NULL.
 * stats (8): [0] forward evaluations, [1] recomputed evaluations, [2] transposed evaluations,
 * [3] CG iterations forward, [4] CG iterations transposed, [5] checkpoints, [6] checkpoint and
 * stage storage in bytes.  Needs the interfacial DMI form (or none), one component and the dense
 * BEM.  Synchronises.  No tetmag counterpart (tetmag has no adjoint). */
int tmb_adjoint_rk4(tmb_ctx* ctx, const double* m0, int nsteps, double dt_ps, int nsub, int ckpt_every, double t0_ps,
                    int normalize, const double* w, double* m_final, double* grad_m0, double* grad_ku,
                    double* grad_bz, double* J, double* stats, int ptr_kind);
/* Counters of the last demag evaluation: [0] Neumann iterations, [1] Dirichlet iterations,
 * [2] Neumann relative residual, [3] Dirichlet relative residual, [4] Neumann status,
 * [5] Dirichlet status, [6] AMG levels (Neumann), [7] AMG setup ms (both). Synchronises. */
int tmb_get_stats(tmb_ctx* ctx, double* out);

/* Live profiling with CUDA events on the context stream (no reference counterpart; tetmag's
 * timers are host wall clocks, main/DemagField.cpp:155-160, utils/Timer.cpp:36-81).
 * Kernel ids: 0 local field + LLG, 1 divergence, 2 gradient, 3 BEM matvec, 4 Neumann solve,
 * 5 Dirichlet solve, 6 CG fine-level SpMV, 7 whole demag chain (4, 5 and 7 span several kernels),
 * 8 fused CG update + first fine smoothing sweep, 9 fine post-smoothing sweep + r.z, 10 fine
 * pre-smoothing sweep (unfused), 11 restriction, 12 prolongation, 13 coarse-level smoothing
 * sweeps, 14 coarsest dense solve, 15 CG start (lift, initial residual), 16 CG vector update
 * (unfused).  tmb_profile_read fills out[3*id + {0,1,2}] = launches, total ms, algorithmic bytes
 * per launch, for the 17 ids (51 doubles). */
int tmb_profile_enable(tmb_ctx* ctx, int on);
int tmb_profile_read(tmb_ctx* ctx, double* out);

/* ---------------------------------------------------------------------------------------
 * Linear solver plugin (SolverFactory, main/SolverFactory.h:42-65): a "b200" solver
 * for the row-pinned Neumann and row-replaced Dirichlet matrices of the demag chain.
 * Rows whose only entry is a unit diagonal are treated as constraints and eliminated
 * symmetrically, so the remaining system is SPD and solved by PCG with a device
 * smoothed-aggregation V-cycle.  The previous solution is the initial guess
 * (as AMGCLSolver::solve, main/AMGCLSolver.cpp:97-103).
 * ------------------------------------------------------------------------------------- */
int tmb_solver_create(tmb_ctx* ctx, tmb_solver** out);
int tmb_solver_destroy(tmb_solver* s);
int tmb_solver_set_matrix(tmb_solver* s, int n, int nnz, const int* rowptr, const int* col, const double* val);
int tmb_solver_set_tolerance(tmb_solver* s, double tol, int maxiter);
int tmb_solver_compute(tmb_solver* s);                 /* setup; SolverFactory::compute */
int tmb_solver_solve(tmb_solver* s, const double* b, double* x, int ptr_kind);  /* synchronises */
/* info[0] iterations, [1] relative residual, [2] status (0 ok, 3 not converged, 5 breakdown) */
int tmb_solver_info(tmb_solver* s, double* info);

/* ---------------------------------------------------------------------------------------
 * Run artefacts (host only, no device work except where stated).
 * ------------------------------------------------------------------------------------- */
/* MeshWriter::outputVTK (io/MeshWriter.cpp:174-239; grid of defineUnstructuredVTKGrid, :69-86):
 * a VTK XML unstructured grid of tetrahedra with point vectors "Magnetization" (m, 3N SoA), point
 * scalars "Material" (material, N ints; NULL writes zeros), an optional second point vector field
 * (field, 3N SoA, named field_name; NULL: none; tetmag's final file carries "Demag",
 * main/TheSimulation.cpp:321) and the field-data value "timeInPs" (io/MeshWriter.h:60).
 * xyz: N x 3 row-major, tets: E x 4.  binary = 0 writes ASCII arrays, 1 appended raw binary. */
int tmb_write_vtu(const char* path, int nx, const double* xyz, int ntet, const int* tets, const double* m,
                  const int* material, double time_ps, const double* field, const char* field_name, int binary);
/* VTKReader::readMag + getTime (io/VTKReader.cpp:83-181): the point array "Magnetization" of a .vtu
 * (ASCII, inline base64 or appended raw / base64 arrays, optionally zlib-compressed, UInt32 or UInt64
 * headers: what VTK's XML writer produces) or of a legacy ASCII .vtk file, into m (3N SoA), and the
 * field-data value "timeInPs" into time_ps (0 when absent).  A point count other than nx is an
 * error (VTKReader::checkNodeNumber, :72-81). */
int tmb_read_magnetization(const char* path, int nx, double* m, double* time_ps);
/* writeLogFileHeader (main/TheSimulation.cpp:85-93): the header lines of tetmag's .log file, with
 * the start time as ctime() gives it (ending in a newline), host and user; NUL-terminated in buf. */
int tmb_log_header(const char* start_time, const char* host, const char* user, char* buf, int cap);
/* TheSimulation::writeLogStream (main/TheSimulation.cpp:367-372) after calculateEnergies (:385-396):
 * one .log row for state m at elapsed_ps, character for character as tetmag writes it: time,
 * the eight energy densities of tmb_energies, the max torque (computed when max_torque < 0), the
 * volume-weighted mean m and mean applied field in T (applied field plus the Bz pulse at
 * elapsed_ps).  Evaluates the demag field for m like tmb_energies; synchronises. */
int tmb_log_row(tmb_ctx* ctx, const double* m, int ptr_kind, double elapsed_ps, double max_torque, char* buf,
                int cap);
/* The formatting step of tmb_log_row alone (writeLogStream, main/TheSimulation.cpp:367-372):
 * energies[8] in tmb_energies order, mean_m[3], mean_h_tesla[3]. */
int tmb_log_format(double elapsed_ps, const double* energies, double max_torque, const double* mean_m,
                   const double* mean_h_tesla, char* buf, int cap);

#ifdef __cplusplus
}
#endif

#endif /* TMB_H_ */
