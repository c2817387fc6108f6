"""GPU parity of the CUDA path (through the C ABI) against the FP64 oracle.

Tolerances (relative L2 over all nodes and components):
  plain FP64 path   <= 1e-10  (field, demag, right-hand side)
  mixed path        <= 1e-5   (FP32 operator values, FP64 vectors / reductions)
  relaxation        |<m>_gpu - <m>_oracle| <= 1e-4
"""
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle import tetmag_oracle as O
from tetmag_b200 import _lib, meshgen, workloads
from tetmag_b200.api import Context, MeshOps, SolverFactory, TheLLG, DemagField

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).with_name("golden") / "oracle_small.npz"
FP64_TOL = 1e-10
MIXED_TOL = 1e-5


def rel(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def oracle_problem(w: workloads.Workload, with_bem=True):
    axis = None if w.ku_axis is None else O.soa_to_rows(w.ku_axis)
    return O.make_problem(w.mesh.xyz, w.mesh.tets, w.mesh.scale, Ms=w.Ms, A=w.A, alpha=w.alpha,
                          Ku=w.Ku, ku_axis=axis if axis is not None else (0, 0, 1), D=w.D, hext=w.hext,
                          with_bem=with_bem)


@pytest.fixture(scope="module")
def golden():
    g = np.load(GOLDEN)
    mo = MeshOps(g["xyz"], g["tets"])
    ctx = Context(0)
    ctx.set_mesh(mo)
    ctx.bem_assemble(mo)
    n = mo.nx
    ctx.set_material(np.full(n, O.MU0 * 8e5), np.full(n, 1.3e-11 / 1e-18), Ku=np.full(n, 5e4),
                     ku_axis=O.rows_to_soa(g["axis"]), D=np.full(n, 3e-3 / 1e-9), alpha=0.3)
    ctx.set_applied_field(np.ascontiguousarray(g["hext"]))
    return g, mo, ctx


@pytest.fixture(scope="module")
def c1():
    w = workloads.c1()
    mo, ctx = workloads.setup_context(w, tol=1e-13, maxiter=200)
    pb = oracle_problem(w)
    return w, mo, ctx, pb, O.DemagOracle(pb)


def test_bem_assembly_matches_oracle(golden, c1):
    g, mo, ctx = golden
    B = ctx.get_bem_dense()
    assert np.max(np.abs(B - g["B"])) <= 1e-12 * np.max(np.abs(g["B"]))
    w, mo1, ctx1, pb, _ = c1
    B1 = ctx1.get_bem_dense()
    assert np.max(np.abs(B1 - pb.B)) <= 1e-12 * np.max(np.abs(pb.B))
    assert np.max(np.abs(B1.sum(axis=1) + 1.0)) < 1e-9          # B.1 = -1 per row
    assert O.bem_rowsum_error(B1) < 5e-3                          # the reference's own check


def test_local_field_and_rhs_fp64(golden):
    g, mo, ctx = golden
    m = O.rows_to_soa(g["m"])
    ctx.set_demag_frozen(O.rows_to_soa(g["hdem"]))
    H = ctx.effective_field(m)
    assert rel(H, O.rows_to_soa(g["H"])) <= 1e-12
    ydot = TheLLG(ctx)(m, 0.0)
    assert rel(ydot, O.rows_to_soa(g["ydot"])) <= 1e-12
    assert abs(ctx.max_torque(m) - float(g["torque"])) <= 1e-12 * float(g["torque"])


def test_local_field_mixed(golden):
    g, mo, ctx = golden
    m = O.rows_to_soa(g["m"])
    ctx.set_demag_frozen(O.rows_to_soa(g["hdem"]))
    ctx.set_precision(True)
    try:
        H = ctx.effective_field(m)
    finally:
        ctx.set_precision(False)
    assert rel(H, O.rows_to_soa(g["H"])) <= MIXED_TOL


def test_demag_fp64_golden(golden):
    g, mo, ctx = golden
    ctx.set_solver_params(1e-13, 300)
    H = DemagField(ctx).calcField(O.rows_to_soa(g["m"]))
    assert rel(H, O.rows_to_soa(g["hdem"])) <= FP64_TOL


def test_demag_fp64_c1(c1):
    w, mo, ctx, pb, dem = c1
    ctx.set_precision(False)
    m = w.m0
    H = ctx.demag_field(m)
    Ho = dem.field(O.soa_to_rows(m))
    assert rel(H, O.rows_to_soa(Ho)) <= FP64_TOL
    st = ctx.stats()
    assert st["status_neumann"] == 0 and st["status_dirichlet"] == 0
    # a second call warm-starts from the previous solution and still matches
    H2 = ctx.demag_field(m)
    assert rel(H2, O.rows_to_soa(Ho)) <= FP64_TOL


def test_demag_mixed_c1(c1):
    w, mo, ctx, pb, dem = c1
    ctx.set_precision(True)
    ctx.set_solver_params(1e-9, 200)
    try:
        for seed in (3, 4):
            m = meshgen.random_state(w.n, seed)
            H = ctx.demag_field(m)
            Ho = dem.field(O.soa_to_rows(m))
            assert rel(H, O.rows_to_soa(Ho)) <= MIXED_TOL
    finally:
        ctx.set_precision(False)
        ctx.set_solver_params(1e-13, 200)


def test_full_rhs_with_demag_c1(c1):
    w, mo, ctx, pb, dem = c1
    m = meshgen.random_state(w.n, 9)
    ctx.demag_field(m)                     # refresh the frozen demag field
    ydot = ctx.llg_rhs(0.0, m)
    mr = O.soa_to_rows(m)
    Ho = O.local_field(pb, mr, dem.field(mr))
    assert rel(ydot, O.rows_to_soa(O.llg_rhs(pb, mr, Ho))) <= FP64_TOL
    assert abs(ctx.max_torque(m) - O.max_torque(mr, Ho)) <= 1e-9 * O.max_torque(mr, Ho)


def test_solver_plugin_on_reference_matrices(c1):
    # the row-pinned Neumann and row-replaced Dirichlet matrices of DemagField
    w, mo, ctx, pb, dem = c1
    rng = np.random.default_rng(5)
    for A in (dem.neumann, dem.dirichlet):
        s = SolverFactory.makeSolver("b200", ctx)
        s.setMatrix(A)
        s.setCGTolerance(1e-13)
        s.maxiter = 300
        assert s.compute()
        b = rng.standard_normal(A.shape[0])
        s.setLoadVector(b)
        s.solve()
        assert s.wasSuccessful()
        x_ref = spla.splu(A.tocsc()).solve(b)
        assert rel(s.result(), x_ref) <= 1e-10


def test_normalize_and_device_pointers(c1):
    torch = pytest.importorskip("torch")
    w, mo, ctx, pb, dem = c1
    m = meshgen.random_state(w.n, 12) * 1.7
    mt = torch.from_numpy(m.copy()).cuda()
    ctx.normalize(mt)
    mh = ctx.normalize(m.copy())
    assert np.allclose(mt.cpu().numpy(), mh, rtol=0, atol=1e-15)
    assert np.allclose(np.linalg.norm(O.soa_to_rows(mh), axis=1), 1.0, atol=1e-15)
    yd = ctx.llg_rhs(0.0, mt)
    torch.cuda.synchronize()
    assert rel(yd.cpu().numpy(), ctx.llg_rhs(0.0, mh)) <= 1e-14


def test_nan_is_reported(c1):
    w, mo, ctx, pb, dem = c1
    m = meshgen.random_state(w.n, 2)
    m[5] = np.nan
    with pytest.raises(_lib.TmbError) as e:
        ctx.max_torque(m)
    assert e.value.code == _lib.TMB_ERR_NAN


def test_relax_short_matches_oracle(c1):
    w, mo, ctx, pb, dem = c1
    ctx.set_precision(False)
    ctx.set_solver_params(1e-12, 200)
    m = w.m0.copy()
    st = ctx.relax(m, duration_ps=10.0, segment_ps=0.5)
    mo_, so = O.relax(pb, w.m0, 10.0, 0.5, demag=dem)
    assert st["segments"] == so["segments"] == 20
    assert np.max(np.abs(O.mean_m(pb, O.soa_to_rows(m)) - O.mean_m(pb, mo_))) <= 1e-4
    assert abs(st["accepted"] - so["accepted"]) <= max(2, 0.02 * so["accepted"])
    assert np.isfinite(st["max_torque"])


def test_full_size_c4_properties():
    # 28611 nodes / 7002 boundary nodes: size-independent checks at full size
    w = workloads.c4_replica(replica=0)
    mo, ctx = workloads.setup_context(w, tol=1e-11, maxiter=200)
    B = ctx.get_bem_dense()
    assert np.max(np.abs(B.sum(axis=1) + 1.0)) < 1e-8
    del B
    # uniform magnetisation: demag factors of the 200x200x40 nm prism (Aharoni)
    n = w.n
    Ms = w.Ms
    vol = mo.operators()["node_vol"]
    Nd = []
    for d in range(3):
        m = np.zeros(3 * n)
        m[d * n:(d + 1) * n] = 1.0
        H = ctx.demag_field(m)
        E = -(O.MU0 * Ms * vol) @ H[d * n:(d + 1) * n] / 2.0
        Nd.append(E / (0.5 * O.MU0 * Ms * Ms * vol.sum()))
    assert abs(sum(Nd) - 1.0) < 0.02
    assert abs(Nd[2] - O.aharoni_nz(100.0, 100.0, 20.0)) < 0.01
    # mixed vs FP64 on a random state
    m = w.m0
    H64 = ctx.demag_field(m)
    ctx.set_precision(True)
    ctx.set_solver_params(1e-9, 200)
    Hmx = ctx.demag_field(m)
    assert rel(Hmx, H64) <= MIXED_TOL


def test_hierarchical_bem_matches_dense_c4():
    # 7002 boundary nodes: leaf 32, eta 2; FP64 terms to 1e-7, FP32 terms to 1e-6.  On this film
    # the admissible blocks pairing top+bottom-face clusters need the ACA residual check.
    w = workloads.c4_replica(replica=1)
    mo, ctx = workloads.setup_context(w, tol=1e-12, maxiter=300, hmatrix=True, keep_dense=True)
    info = ctx.bem_info()
    assert info["built"] == 1 and info["mode"] == 1
    assert info["bytes_fp32"] < 0.5 * 4 * info["dense_entries"]
    m = w.m0
    ctx.set_bem_mode(False)
    H_dense = ctx.demag_field(m)
    ctx.set_bem_mode(True)
    H_h64 = ctx.demag_field(m)
    assert rel(H_h64, H_dense) <= 1e-6
    ctx.set_precision(True)
    ctx.set_solver_params(1e-9, 300)
    H_h32 = ctx.demag_field(m)
    assert rel(H_h32, H_dense) <= MIXED_TOL


def test_accurate_dense_assembly_c4():
    # the far-field-accurate weights keep the exact identity B.1 = -1 per row; on this 200 nm
    # cuboid the reference arithmetic is still close to them
    w = workloads.c4_replica(replica=0)
    mo = MeshOps(w.mesh.xyz, w.mesh.tets)
    ctx = Context(0)
    ctx.set_mesh(mo)
    ctx.bem_assemble(mo, accurate=True)
    Ba = ctx.get_bem_dense()
    assert np.max(np.abs(Ba.sum(axis=1) + 1.0)) < 1e-11
    ctx.bem_assemble(mo)
    Br = ctx.get_bem_dense()
    assert np.max(np.abs(Ba - Br)) < 1e-7 * np.max(np.abs(Br))


def test_hierarchical_bem_from_mesh_c4():
    # built from the mesh boundary (no dense matrix): low-rank blocks from the accurate far-field
    # weights, dense tiles with the reference arithmetic; compared with the dense path on the
    # accurate matrix
    w = workloads.c4_replica(replica=2)
    mo, ctx = workloads.setup_context(w, tol=1e-12, maxiter=300, hmatrix="mesh", keep_dense=True)
    info = ctx.bem_info()
    assert info["built"] == 1 and info["mode"] == 1
    v = ctx.bem_verify()
    assert v["rel_err_fp64"] <= 3e-6 and v["rel_err_fp32"] <= 1e-5
    m = w.m0
    ctx.set_bem_mode(False)
    H_dense = ctx.demag_field(m)
    ctx.set_bem_mode(True)
    assert rel(ctx.demag_field(m), H_dense) <= 1e-6
    ctx.set_precision(True)
    ctx.set_solver_params(1e-9, 300)
    assert rel(ctx.demag_field(m), H_dense) <= MIXED_TOL


def test_hierarchical_matrix_relative_accuracy_c4():
    # the same film built to matrix-relative accuracy (tmb_set_bem_accuracy): a low-rank block may
    # stop at its share of eps * ||N||_F, so blocks far apart keep fewer terms; the demag field
    # stays within the bounds of the block-relative build
    w = workloads.c4_replica(replica=2)
    mo, ctx = workloads.setup_context(w, tol=1e-12, maxiter=300, hmatrix="mesh", keep_dense=True)
    base = ctx.bem_info()
    ctx.set_bem_accuracy(1.0)
    ctx.bem_build_h(mo, leaf=32, eta=2.0, eps_mixed=1e-6, eps_fp64=1e-7, kmax=64)
    info = ctx.bem_info()
    assert info["built"] == 1 and info["lowrank_blocks"] == base["lowrank_blocks"]
    assert info["terms_fp64"] < base["terms_fp64"] and info["terms_fp32"] < base["terms_fp32"]
    assert info["bytes_fp32"] < base["bytes_fp32"]
    m = w.m0
    ctx.set_bem_mode(False)
    H_dense = ctx.demag_field(m)
    ctx.set_bem_mode(True)
    assert rel(ctx.demag_field(m), H_dense) <= 1e-6
    ctx.set_precision(True)
    ctx.set_solver_params(1e-9, 300)
    assert rel(ctx.demag_field(m), H_dense) <= MIXED_TOL


def test_bem_accuracy_rejects_bad_share(c1):
    w, mo, ctx, pb, dem = c1
    for bad in (-1.0, float("nan"), float("inf")):
        with pytest.raises(_lib.TmbError):
            ctx.set_bem_accuracy(bad)


def test_hierarchical_from_mesh_all_dense_tiles_equal_dense_c1(c1):
    # with a vanishing admissibility parameter every block is a dense tile assembled from the
    # mesh: the matvec must reproduce the dense assembly to round-off
    w, mo, ctx, pb, dem = c1
    ctx2 = workloads.setup_context(w, tol=1e-12, maxiter=300, mesh_ops=mo)[1]
    ctx2.bem_build_h(mo, leaf=32, eta=1e-9)
    info = ctx2.bem_info()
    assert info["lowrank_blocks"] == 0 and info["dense_tiles"] > 0
    m = meshgen.random_state(w.n, 5)
    H_tiles = ctx2.demag_field(m)
    ctx2.set_bem_mode(False)
    assert rel(H_tiles, ctx2.demag_field(m)) <= 1e-12


def test_hierarchical_from_mesh_without_dense_c1_against_oracle(c1):
    w, mo, ctx, pb, dem = c1
    ctx2 = workloads.setup_context(w, tol=1e-12, maxiter=300, hmatrix="mesh", keep_dense=False, mesh_ops=mo)[1]
    with pytest.raises(_lib.TmbError):
        ctx2.set_bem_mode(False)
    m = meshgen.random_state(w.n, 19)
    Ho = O.rows_to_soa(dem.field(O.soa_to_rows(m)))
    assert rel(ctx2.demag_field(m), Ho) <= 1e-6


def test_hierarchical_bem_c1_against_oracle(c1):
    w, mo, ctx, pb, dem = c1
    ctx2 = workloads.setup_context(w, tol=1e-12, maxiter=300, hmatrix=True, keep_dense=False, mesh_ops=mo)[1]
    assert ctx2.bem_info()["built"] == 1
    m = meshgen.random_state(w.n, 17)
    Ho = O.rows_to_soa(dem.field(O.soa_to_rows(m)))
    assert rel(ctx2.demag_field(m), Ho) <= 1e-6
    ctx2.set_precision(True)
    ctx2.set_solver_params(1e-9, 300)
    assert rel(ctx2.demag_field(m), Ho) <= MIXED_TOL


def _separate(meshes, m0s, hexts, axes, Ku, alpha, tol=1e-13):
    """Demag field and right-hand side of each instance in its own single-mesh context."""
    out = []
    for mesh, m0, hx, ax in zip(meshes, m0s, hexts, axes):
        w = workloads.Workload(name="one", mesh=mesh, Ms=8.0e5, A=1.3e-11, alpha=alpha, m0=m0, hext=hx, Ku=Ku,
                               ku_axis=ax)
        ctx = workloads.setup_context(w, tol=tol, maxiter=300)[1]
        h = ctx.demag_field(m0)
        out.append((h, ctx.llg_rhs(0.0, m0)))
    return out


def test_components_uneven_dots_match_separate_contexts():
    # three dots of different sizes as one batched context (each with its own BEM block) against
    # three single-mesh contexts; one of them also against the oracle
    meshes = [meshgen.kuhn_cuboid(6, 5, 2, 2.5), meshgen.kuhn_cuboid(9, 7, 3, 2.2), meshgen.kuhn_cuboid(4, 8, 5, 2.8)]
    m0s = [meshgen.random_state(m.nx, 40 + i) for i, m in enumerate(meshes)]
    hx = [meshgen.field_from_angles(m.nx, 0.03 * (i + 1), 30.0 * i, 50.0) for i, m in enumerate(meshes)]
    rng = np.random.default_rng(8)
    axes = []
    for m in meshes:
        a = rng.standard_normal(3)
        axes.append(np.repeat(a / np.linalg.norm(a), m.nx))
    mesh, off = meshgen.union(meshes)
    w = workloads.Workload(name="dots", mesh=mesh, Ms=8.0e5, A=1.3e-11, alpha=0.1, m0=meshgen.soa_stack(m0s),
                           hext=meshgen.soa_stack(hx), Ku=5e4, ku_axis=meshgen.soa_stack(axes), components=off)
    mo, ctx = workloads.setup_context(w, tol=1e-13, maxiter=300)
    H = meshgen.soa_split(ctx.demag_field(w.m0), off)
    Y = meshgen.soa_split(ctx.llg_rhs(0.0, w.m0), off)
    ref = _separate(meshes, m0s, hx, axes, 5e4, 0.1)
    for c in range(3):
        assert rel(H[c], ref[c][0]) <= 1e-10
        assert rel(Y[c], ref[c][1]) <= 1e-10
    pb = O.make_problem(meshes[1].xyz, meshes[1].tets, 1e-9, Ms=8e5, A=1.3e-11, alpha=0.1, Ku=5e4,
                        ku_axis=O.soa_to_rows(axes[1]), D=0.0, hext=hx[1])
    Ho = O.DemagOracle(pb).field(O.soa_to_rows(m0s[1]))
    assert rel(H[1], O.rows_to_soa(Ho)) <= FP64_TOL
    ctx.set_precision(True)
    ctx.set_solver_params(1e-9, 300)
    Hm = meshgen.soa_split(ctx.demag_field(w.m0), off)
    for c in range(3):
        assert rel(Hm[c], ref[c][0]) <= MIXED_TOL


def test_shared_bem_replicas_gemm_match_separate_contexts():
    # five replicas of one cuboid sharing one BEM matrix (boundary matvec as one GEMM), each with
    # its own m0 and applied field
    base = meshgen.kuhn_cuboid(12, 10, 3, 3.0)
    R = 5
    m0s = [meshgen.random_state(base.nx, 60 + r) for r in range(R)]
    hx = [meshgen.field_from_angles(base.nx, 0.01 * r, 20.0 * r, 10.0 * r) for r in range(R)]
    mesh, off = meshgen.union([base] * R)
    w = workloads.Workload(name="reps", mesh=mesh, Ms=8.0e5, A=1.3e-11, alpha=0.5, m0=meshgen.soa_stack(m0s),
                           hext=meshgen.soa_stack(hx), components=off, shared_bem=True)
    mo, ctx = workloads.setup_context(w, tol=1e-13, maxiter=300)
    H = meshgen.soa_split(ctx.demag_field(w.m0), off)
    ref = _separate([base] * R, m0s, hx, [None] * R, 0.0, 0.5)
    for r in range(R):
        assert rel(H[r], ref[r][0]) <= 1e-10
    ctx.set_precision(True)
    ctx.set_solver_params(1e-9, 300)
    Hm = meshgen.soa_split(ctx.demag_field(w.m0), off)
    for r in range(R):
        assert rel(Hm[r], ref[r][0]) <= MIXED_TOL
    # identical replicas must give identical fields
    mesh2, off2 = meshgen.union([base] * 3)
    w2 = workloads.Workload(name="same", mesh=mesh2, Ms=8.0e5, A=1.3e-11, alpha=0.5,
                            m0=meshgen.soa_stack([m0s[0]] * 3), hext=meshgen.soa_stack([hx[1]] * 3),
                            components=off2, shared_bem=True)
    ctx2 = workloads.setup_context(w2, tol=1e-13, maxiter=300)[1]
    H2 = meshgen.soa_split(ctx2.demag_field(w2.m0), off2)
    assert rel(H2[2], H2[0]) <= 1e-12


def test_components_reject_coupled_operators(c1):
    w, mo, ctx, pb, dem = c1
    ctx2 = Context(0)
    ctx2.set_mesh(mo)
    with pytest.raises(_lib.TmbError):
        ctx2.set_components([0, w.n // 2, w.n])       # splits one connected mesh


def test_interfacial_dmi_local_field(golden):
    # interfacial DMI (no reference counterpart) against the oracle's exact energy gradient,
    # both precisions; then back to the bulk form
    g, mo, ctx = golden
    m = O.rows_to_soa(g["m"])
    pb = O.make_problem(g["xyz"], g["tets"], 1e-9, Ms=8e5, A=1.3e-11, alpha=0.3, Ku=5e4, ku_axis=g["axis"],
                        D=3e-3, hext=np.ascontiguousarray(g["hext"]), with_bem=False, dmi_kind="interfacial")
    Ho = O.local_field(pb, g["m"], g["hdem"])
    ctx.set_demag_frozen(O.rows_to_soa(g["hdem"]))
    ctx.set_dmi_kind(True)
    try:
        H = ctx.effective_field(m)
        assert rel(H, O.rows_to_soa(Ho)) <= 1e-12
        assert rel(TheLLG(ctx)(m, 0.0), O.rows_to_soa(O.llg_rhs(pb, g["m"], Ho))) <= 1e-12
        ctx.set_precision(True)
        assert rel(ctx.effective_field(m), O.rows_to_soa(Ho)) <= MIXED_TOL
    finally:
        ctx.set_precision(False)
        ctx.set_dmi_kind(False)
    assert rel(ctx.effective_field(m), O.rows_to_soa(g["H"])) <= 1e-12


@pytest.mark.parametrize("replicas", [64, 70])
def test_tensor_core_replica_gemm_matches_cuda_cores(replicas):
    # the 3xTF32 tcgen05 boundary GEMM against the CUDA-core GEMM on the mixed path: one full
    # 64-replica tile, and 70 replicas (a second, mostly empty tile); plus the FP64 reference
    base = meshgen.kuhn_cuboid(14, 12, 3, 3.0)
    m0s = [meshgen.random_state(base.nx, 300 + r) for r in range(replicas)]
    mesh, off = meshgen.union([base] * replicas)
    w = workloads.Workload(name="reps", mesh=mesh, Ms=8.0e5, A=1.3e-11, alpha=0.5, m0=meshgen.soa_stack(m0s),
                           hext=np.zeros(3 * mesh.nx), components=off, shared_bem=True)
    mo, ctx = workloads.setup_context(w, tol=1e-12, maxiter=300)
    H64 = ctx.demag_field(w.m0)
    ctx.set_precision(True)
    ctx.set_solver_params(1e-11, 300)
    ctx.set_bem_gemm_kind(False)
    Hcc = ctx.demag_field(w.m0)
    ctx.set_bem_gemm_kind(True)
    Htc = ctx.demag_field(w.m0)
    info = ctx.bem_gemm_info()
    assert info["tensor_cores"] and info["split"] >= 1 and info["tuned_ms"]
    assert rel(Htc, Hcc) <= 2e-6
    assert rel(Htc, H64) <= MIXED_TOL
    Htc2 = ctx.demag_field(w.m0)           # second call: tuned split, warm solves
    assert rel(Htc2, Htc) <= 1e-8


@pytest.mark.parametrize("R", [5, 40])
def test_interleaved_replicas_match_separate_contexts(R):
    # R interleaved replicas of one cuboid (operators applied to all replicas at once, the boundary
    # product one GEMM) against R single-mesh contexts: FP64 to 1e-10, mixed to 1e-5; R = 5 mixes
    # operator rows inside a warp, R = 40 gives warps of one row and warps that straddle two rows
    base = meshgen.kuhn_cuboid(10, 9, 3, 3.0)
    m0s = [meshgen.random_state(base.nx, 500 + r) for r in range(R)]
    hx = [meshgen.field_from_angles(base.nx, 0.002 * r, 13.0 * r, 7.0 * r) for r in range(R)]
    w = workloads.Workload(name="irep", mesh=base, Ms=8.0e5, A=1.3e-11, alpha=0.5, m0=meshgen.interleave(m0s),
                           hext=meshgen.interleave(hx), replicas=R)
    mo, ctx = workloads.setup_context(w, tol=1e-13, maxiter=300)
    H = meshgen.deinterleave(ctx.demag_field(w.m0), R)
    Y = meshgen.deinterleave(ctx.llg_rhs(0.0, w.m0), R)
    torque = ctx.max_torque(w.m0)
    ref = _separate([base] * R, m0s, hx, [None] * R, 0.0, 0.5)
    for r in range(R):
        assert rel(H[r], ref[r][0]) <= 1e-10
        assert rel(Y[r], ref[r][1]) <= 1e-10
    assert torque > 0.0
    ctx.set_precision(True)
    ctx.set_solver_params(1e-10, 300)
    Hm = meshgen.deinterleave(ctx.demag_field(w.m0), R)
    for r in range(R):
        assert rel(Hm[r], ref[r][0]) <= MIXED_TOL
    # a short relaxation of the batch stays normalised and finite
    m = w.m0.copy()
    st = ctx.relax(m, duration_ps=0.5, segment_ps=0.25)
    assert np.isfinite(st["max_torque"])
    nrm = np.linalg.norm(m.reshape(3, -1), axis=0)
    assert np.max(np.abs(nrm - 1.0)) < 1e-12


def _golden_problem(g, dmi_kind="bulk"):
    return O.make_problem(g["xyz"], g["tets"], 1e-9, Ms=8e5, A=1.3e-11, alpha=0.3, Ku=5e4, ku_axis=g["axis"],
                          D=3e-3, hext=np.ascontiguousarray(g["hext"]), with_bem=False, dmi_kind=dmi_kind)


def _check_energies(e, eo, tol):
    scale = max(abs(v) for v in eo.values())
    for k, v in eo.items():
        assert abs(e[k] - v) <= tol * scale, (k, e[k], v)


def test_energies_match_oracle(golden):
    # the energy densities of TheSimulation::calculateEnergies (demag evaluated for m through the
    # solves) against the oracle's sums, bulk and interfacial DMI, FP64 and mixed
    g, mo, ctx = golden
    m = O.rows_to_soa(g["m"])
    try:
        for kind in ("bulk", "interfacial"):
            ctx.set_dmi_kind(kind == "interfacial")
            eo = O.energies(_golden_problem(g, kind), g["m"], g["hdem"])
            assert eo["dmi"] != 0.0 and eo["uniaxial"] > 0.0
            ctx.set_solver_params(1e-13, 300)
            _check_energies(ctx.energies(m), eo, 1e-10)
            ctx.set_precision(True)
            ctx.set_solver_params(1e-10, 300)
            _check_energies(ctx.energies(m), eo, MIXED_TOL)
            ctx.set_precision(False)
    finally:
        ctx.set_precision(False)
        ctx.set_dmi_kind(False)
        ctx.set_solver_params(1e-13, 300)


def test_energies_uniform_state_and_replicas():
    # a uniform state along the easy axis has no exchange, anisotropy or DMI energy and a positive
    # demag energy below (1/2) Js Ms; R interleaved replicas give the mean of R single contexts
    base = meshgen.kuhn_cuboid(10, 9, 3, 3.0)
    R = 3
    axis = np.concatenate([np.zeros(2 * base.nx), np.ones(base.nx)])
    up = np.concatenate([np.zeros(2 * base.nx), np.ones(base.nx)])
    w = workloads.Workload(name="up", mesh=base, Ms=8.0e5, A=1.3e-11, alpha=0.5, m0=up, hext=np.zeros(3 * base.nx),
                           Ku=5e4, ku_axis=axis, D=2e-3)
    ctx = workloads.setup_context(w, tol=1e-13, maxiter=300)[1]
    e = ctx.energies(up)
    ed = 0.5 * O.MU0 * 8.0e5 ** 2
    assert 0.0 < e["demag"] < ed
    for k in ("exchange", "uniaxial", "dmi", "zeeman", "cubic", "surface"):
        assert abs(e[k]) <= 1e-9 * ed, (k, e[k])
    m0s = [meshgen.random_state(base.nx, 900 + r) for r in range(R)]
    hx = [meshgen.field_from_angles(base.nx, 0.01 * (r + 1), 20.0 * r, 5.0 * r) for r in range(R)]
    singles = []
    for r in range(R):
        wr = workloads.Workload(name="one", mesh=base, Ms=8.0e5, A=1.3e-11, alpha=0.5, m0=m0s[r], hext=hx[r],
                                Ku=5e4, ku_axis=axis, D=2e-3)
        singles.append(workloads.setup_context(wr, tol=1e-13, maxiter=300)[1].energies(m0s[r]))
    wR = workloads.Workload(name="rep", mesh=base, Ms=8.0e5, A=1.3e-11, alpha=0.5, m0=meshgen.interleave(m0s),
                            hext=meshgen.interleave(hx), Ku=5e4, ku_axis=axis, D=2e-3, replicas=R)
    eR = workloads.setup_context(wR, tol=1e-13, maxiter=300)[1].energies(wR.m0)
    mean = {k: np.mean([s[k] for s in singles]) for k in singles[0]}
    _check_energies(eR, mean, 1e-10)


def _random_cubic_axes(n, seed):
    q, _ = np.linalg.qr(np.random.default_rng(seed).standard_normal((n, 3, 3)))
    return np.ascontiguousarray(np.transpose(q, (0, 2, 1)))   # rows: the three cubic axes


def test_cubic_and_surface_anisotropy_match_oracle(golden):
    # cubic anisotropy with per-node axes (EffFieldCalc::cubicAnisotropyField) and surface
    # anisotropy (surfaceAnisotropyField): field, right-hand side and energies against the oracle
    # in both precisions; removing them gives back the golden field
    g, mo, ctx = golden
    m = O.rows_to_soa(g["m"])
    n = mo.nx
    cax = _random_cubic_axes(n, 21)
    k1 = np.random.default_rng(5).uniform(2e4, 6e4, n)
    pb = _golden_problem(g)
    pb.extra.update(Kc1=k1, Kc2=np.full(n, -1.5e4), cax=cax, Ks=np.full(n, 8e-4 / 1e-9))
    Ho = O.local_field(pb, g["m"], g["hdem"])
    ctx.set_cubic_anisotropy(k1, -1.5e4, cax)
    ctx.set_surface_anisotropy(8e-4 / 1e-9)
    try:
        ctx.set_demag_frozen(O.rows_to_soa(g["hdem"]))
        assert rel(ctx.effective_field(m), O.rows_to_soa(Ho)) <= 1e-12
        assert rel(TheLLG(ctx)(m, 0.0), O.rows_to_soa(O.llg_rhs(pb, g["m"], Ho))) <= 1e-12
        ctx.set_solver_params(1e-13, 300)
        eo = O.energies(pb, g["m"], g["hdem"])
        assert eo["cubic"] != 0.0 and eo["surface"] != 0.0
        _check_energies(ctx.energies(m), eo, 1e-10)
        ctx.set_precision(True)
        ctx.set_demag_frozen(O.rows_to_soa(g["hdem"]))
        assert rel(ctx.effective_field(m), O.rows_to_soa(Ho)) <= MIXED_TOL
    finally:
        ctx.set_precision(False)
        ctx.set_cubic_anisotropy(None)
        ctx.set_surface_anisotropy(None)
    ctx.set_demag_frozen(O.rows_to_soa(g["hdem"]))
    assert rel(ctx.effective_field(m), O.rows_to_soa(g["H"])) <= 1e-12


def test_spin_transfer_torque_rhs_matches_oracle(golden):
    # Zhang-Li term of TheLLG::sttDynamics with per-node eta, beta and a pulse scale, against the
    # oracle; the max torque ignores it (TheLLG::getMaxTorque); removing it gives the golden rhs
    g, mo, ctx = golden
    m = O.rows_to_soa(g["m"])
    eta = np.random.default_rng(8).standard_normal((mo.nx, 3)) * 4e6
    pb = _golden_problem(g)
    pb.extra.update(eta=eta, beta=0.05, stt_scale=0.7)
    Ho = O.local_field(pb, g["m"], g["hdem"])
    ref = O.rows_to_soa(O.llg_rhs(pb, g["m"], Ho))
    assert rel(ref, O.rows_to_soa(g["ydot"])) > 1e-2          # the term matters at this size
    ctx.set_demag_frozen(O.rows_to_soa(g["hdem"]))
    ctx.set_stt(O.rows_to_soa(eta), beta=0.05, scale=0.7)
    try:
        assert rel(TheLLG(ctx)(m, 0.0), ref) <= 1e-12
        assert abs(ctx.max_torque(m) - float(g["torque"])) <= 1e-12 * float(g["torque"])
        ctx.set_precision(True)
        assert rel(TheLLG(ctx)(m, 0.0), ref) <= MIXED_TOL
    finally:
        ctx.set_precision(False)
        ctx.set_stt(None)
    assert rel(TheLLG(ctx)(m, 0.0), O.rows_to_soa(g["ydot"])) <= 1e-12
