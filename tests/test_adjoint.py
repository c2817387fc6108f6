"""Adjoint of the fixed-step LLG integration (the interfacial-DMI disk workload).

CPU: the FP64 oracle's discrete adjoint against central finite differences of its own forward
map.  GPU (marked): the device adjoint through the C ABI against the oracle's gradient, against
central finite differences of the device forward map, and its cost against a forward run.

Tolerances: FP64 device gradient vs oracle gradient <= 1e-8 relative (CG tolerance 1e-13);
directional finite differences <= 1e-4 relative (FP64 and mixed paths).
"""
import numpy as np
import pytest

from oracle import adjoint_oracle as A
from oracle import tetmag_oracle as O
from tetmag_b200 import meshgen


def small_disk_problem(seed=5, diameter=30.0, thickness=6.0, D=1.58e-3):
    mesh = meshgen.jittered_disk(diameter, thickness, 3.0, seed=seed)
    pb = O.make_problem(mesh.xyz, mesh.tets, 1e-9, Ms=3.84e5, A=8.78e-12, alpha=0.3, Ku=0.0, ku_axis=(0, 0, 1),
                        D=D, dmi_kind="interfacial")
    # a C-contiguous copy: rows_to_soa of a transposed view would alias it, and the device
    # integrators work in place
    m0 = np.ascontiguousarray(O.soa_to_rows(meshgen.skyrmion_state(mesh.xyz, 3, radius=diameter / 4,
                                                                   wall=diameter / 15)))
    return mesh, pb, m0


def test_pulse_weights():
    w = A.pulse_weights(5, 0.0, 4.0, 1.25)
    assert np.allclose(w, [0, 0.75, 0.25, 0, 0])
    assert np.allclose(A.pulse_weights(5, 0.0, 4.0, -1.0), [1, 0, 0, 0, 0])
    assert np.allclose(A.pulse_weights(5, 0.0, 4.0, 9.0), [0, 0, 0, 0, 1])
    assert np.allclose(A.pulse_weights(5, 0.0, 4.0, 4.0), [0, 0, 0, 0, 1])


def test_oracle_adjoint_matches_finite_differences():
    mesh, pb, m0 = small_disk_problem()
    dem = O.DemagOracle(pb)
    rng = np.random.default_rng(1)
    n = mesh.nx
    bz = 0.05 * rng.standard_normal(7)
    ku = 2e4 * rng.uniform(0, 1, n)
    nsteps, dt, nsub = 2, 1.0, 8
    w = A.mean_mz_weights(pb)

    def J(ku_, bz_, m_=m0):
        d = A.Dynamics(A.problem_with_ku(pb, ku_), dem, bz_, 0.0, nsteps * dt)
        return float(np.sum(w * A.rk4_forward(d, m_, nsteps, dt, nsub)))

    d = A.Dynamics(A.problem_with_ku(pb, ku), dem, bz, 0.0, nsteps * dt)
    Jv, yN, gm, gku, gbz = A.rk4_adjoint(d, m0, nsteps, dt, w, nsub)
    assert abs(Jv - J(ku, bz)) <= 1e-14
    v = rng.standard_normal(n)
    fd = (J(ku + 10 * v, bz) - J(ku - 10 * v, bz)) / 20
    assert abs(fd - gku @ v) <= 1e-7 * abs(gku @ v)
    v = rng.standard_normal(bz.size)
    fd = (J(ku, bz + 1e-4 * v) - J(ku, bz - 1e-4 * v)) / 2e-4
    assert abs(fd - gbz @ v) <= 1e-7 * abs(gbz @ v)
    v = rng.standard_normal(m0.shape)
    fd = (J(ku, bz, m0 + 1e-5 * v) - J(ku, bz, m0 - 1e-5 * v)) / 2e-5
    assert abs(fd - np.sum(gm * v)) <= 1e-7 * abs(np.sum(gm * v))


def bulk_disk_problem(seed=5):
    """The small disk with tetmag's bulk DMI form (EffFieldCalc::dmiField, main/EffFieldCalc.cpp:159-170)."""
    import dataclasses
    mesh, pb, m0 = small_disk_problem(seed=seed, D=3e-3)
    return mesh, dataclasses.replace(pb, dmi_kind="bulk"), m0


def test_oracle_bulk_dmi_adjoint_matches_finite_differences():
    mesh, pb, m0 = bulk_disk_problem()
    dem = O.DemagOracle(pb)
    rng = np.random.default_rng(2)
    n = mesh.nx
    ku = 2e4 * rng.uniform(0, 1, n)
    nsteps, dt, nsub = 2, 1.0, 8
    w = A.mean_mz_weights(pb)

    def J(m_):
        d = A.Dynamics(A.problem_with_ku(pb, ku), dem, None)
        return float(np.sum(w * A.rk4_forward(d, m_, nsteps, dt, nsub)))

    d = A.Dynamics(A.problem_with_ku(pb, ku), dem, None)
    # the bulk form is what the forward map uses
    assert np.abs(O.dmi_field(pb, m0)).max() > 0.0
    Jv, yN, gm, gku, gbz = A.rk4_adjoint(d, m0, nsteps, dt, w, nsub)
    assert abs(Jv - J(m0)) <= 1e-14
    for k in range(2):
        v = rng.standard_normal(m0.shape)
        fd = (J(m0 + 1e-5 * v) - J(m0 - 1e-5 * v)) / 2e-5
        assert abs(fd - np.sum(gm * v)) <= 1e-7 * abs(np.sum(gm * v)), k
    # the DMI part of the transpose alone: <H_dmi(m), mu> = <m, H_dmi^T(mu)>
    mu = rng.standard_normal(m0.shape)
    lhs = np.sum(O.dmi_field(pb, m0) * O.inv_js(pb)[:, None] * mu)
    rhs = np.sum(m0 * d.bulk_dmi_t(mu))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


# ------------------------------------------------------------------------------------------
# GPU: the device adjoint through the C ABI
# ------------------------------------------------------------------------------------------
def _device_setup(mesh, tol=1e-13, mixed=False, Ku=None, D=1.58e-3, interfacial=True):
    from tetmag_b200.api import Context, MeshOps
    n = mesh.nx
    mo = MeshOps(mesh.xyz, mesh.tets)
    ctx = Context(0)
    ctx.set_mesh(mo)
    ctx.bem_assemble(mo)
    Js = np.full(n, O.MU0 * 3.84e5)
    A_ = np.full(n, 8.78e-12 / 1e-18)
    D = np.full(n, D / 1e-9)
    axis = np.concatenate([np.zeros(2 * n), np.ones(n)])
    ctx.set_material(Js, A_, Ku=Ku, ku_axis=axis, D=D, alpha=0.3)
    ctx.set_dmi_kind(interfacial)
    ctx.set_applied_field(np.zeros(3 * n))
    ctx.set_precision(mixed)
    ctx.set_solver_params(tol, 400)
    return mo, ctx, (Js, A_, axis, D)


def _relerr(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.gpu
def test_device_adjoint_matches_oracle_fp64():
    mesh, pb, m0 = small_disk_problem()
    dem = O.DemagOracle(pb)
    rng = np.random.default_rng(11)
    n = mesh.nx
    bz = 0.05 * rng.standard_normal(7)
    ku = 2e4 * rng.uniform(0, 1, n)
    nsteps, dt, nsub = 3, 1.0, 8
    w = A.mean_mz_weights(pb)
    d = A.Dynamics(A.problem_with_ku(pb, ku), dem, bz, 0.0, nsteps * dt)
    Jo, yo, gmo, gko, gbo = A.rk4_adjoint(d, m0, nsteps, dt, w, nsub)
    mo, ctx, _ = _device_setup(mesh, Ku=ku)
    ctx.set_bz_pulse(bz, 0.0, nsteps * dt)
    # forward map alone
    m = O.rows_to_soa(m0).copy()
    ctx.step_rk4(m, nsteps, dt, nsub)
    assert _relerr(m, O.rows_to_soa(yo)) <= 1e-10
    # checkpoint every 2 steps: one full interval and one partial
    r = ctx.adjoint_rk4(O.rows_to_soa(m0), O.rows_to_soa(w), nsteps, dt, nsub, ckpt_every=2, n_bz=bz.size)
    assert abs(r["J"] - Jo) <= 1e-12
    assert _relerr(r["m_final"], O.rows_to_soa(yo)) <= 1e-10
    assert _relerr(r["grad_m0"], O.rows_to_soa(gmo)) <= 1e-8
    assert _relerr(r["grad_ku"], gko) <= 1e-8
    assert _relerr(r["grad_bz"], gbo) <= 1e-8
    st = r["stats"]
    assert st["fwd_evals"] == 4 * nsteps * nsub and st["vjp_evals"] == 4 * nsteps * nsub
    assert st["checkpoints"] == 2


@pytest.mark.gpu
def test_device_adjoint_finite_differences_and_autograd():
    # directional central differences of the device forward map (FP64 and mixed paths), and the
    # torch.autograd wrapper returning the same gradient
    import torch
    from tetmag_b200.autograd import LLGObjective
    mesh = meshgen.jittered_disk(60.0, 9.0, 3.0, seed=8)
    n = mesh.nx
    m0 = meshgen.skyrmion_state(mesh.xyz, 4, radius=15.0, wall=4.0)
    nsteps, dt, nsub = 4, 1.0, 8
    rng = np.random.default_rng(5)
    bz0 = 0.02 + 0.01 * rng.standard_normal(9)
    ku0 = np.zeros(n)
    wv = np.zeros(3 * n)
    mo0 = MeshOpsForWeights(mesh)
    wv[2 * n:] = mo0 / mo0.sum()
    results = {}
    for mixed in (False, True):
        mo, ctx, (Js, A_, axis, D) = _device_setup(mesh, tol=1e-13 if not mixed else 1e-10, mixed=mixed, Ku=ku0)
        prob = LLGObjective(ctx, Js, A_, axis, D, 0.3, m0, wv, nsteps, dt, nsub=nsub, ckpt_every=3)
        ku_t = torch.zeros(n, dtype=torch.float32, requires_grad=True)
        bz_t = torch.tensor(bz0, dtype=torch.float64, requires_grad=True)
        J = prob.objective(ku_t, bz_t)
        J.backward()
        gku, gbz = ku_t.grad.double().numpy(), bz_t.grad.numpy()
        assert np.allclose(gku, prob.last["grad_ku"].astype(np.float32), rtol=1e-6, atol=0)
        assert np.array_equal(gbz, prob.last["grad_bz"])
        assert abs(prob.forward_only(ku0, bz0) - J.item()) <= (1e-8 if mixed else 1e-12)
        v = rng.standard_normal(n)
        eps = 200.0
        fd = (prob.forward_only(ku0 + eps * v, bz0) - prob.forward_only(ku0 - eps * v, bz0)) / (2 * eps)
        assert abs(fd - gku @ v) <= 1e-4 * abs(gku @ v), (mixed, fd, gku @ v)
        v = rng.standard_normal(bz0.size)
        eps = 1e-3
        fd = (prob.forward_only(ku0, bz0 + eps * v) - prob.forward_only(ku0, bz0 - eps * v)) / (2 * eps)
        assert abs(fd - gbz @ v) <= 1e-4 * abs(gbz @ v), (mixed, fd, gbz @ v)
        results[mixed] = (gku, gbz)
    assert _relerr(results[True][0], results[False][0]) <= 1e-4
    assert _relerr(results[True][1], results[False][1]) <= 1e-4


def MeshOpsForWeights(mesh):
    """Node volumes of the mesh (the weights of the volume-averaged mean m_z)."""
    from tetmag_b200.api import MeshOps
    return MeshOps(mesh.xyz, mesh.tets).operators()["node_vol"]


@pytest.mark.gpu
def test_device_bulk_dmi_adjoint_matches_oracle_fp64():
    # tetmag's bulk DMI form (surface term and curl, main/EffFieldCalc.cpp:159-170, 280-298) through
    # the device adjoint against the oracle's explicit transposes
    mesh, pb, m0 = bulk_disk_problem()
    dem = O.DemagOracle(pb)
    rng = np.random.default_rng(12)
    n = mesh.nx
    bz = 0.05 * rng.standard_normal(5)
    ku = 2e4 * rng.uniform(0, 1, n)
    nsteps, dt, nsub = 2, 1.0, 8
    w = A.mean_mz_weights(pb)
    d = A.Dynamics(A.problem_with_ku(pb, ku), dem, bz, 0.0, nsteps * dt)
    Jo, yo, gmo, gko, gbo = A.rk4_adjoint(d, m0, nsteps, dt, w, nsub)
    mo, ctx, _ = _device_setup(mesh, Ku=ku, D=3e-3, interfacial=False)
    ctx.set_bz_pulse(bz, 0.0, nsteps * dt)
    r = ctx.adjoint_rk4(O.rows_to_soa(m0), O.rows_to_soa(w), nsteps, dt, nsub, ckpt_every=1, n_bz=bz.size)
    assert abs(r["J"] - Jo) <= 1e-12
    assert _relerr(r["m_final"], O.rows_to_soa(yo)) <= 1e-10
    assert _relerr(r["grad_m0"], O.rows_to_soa(gmo)) <= 1e-8
    assert _relerr(r["grad_ku"], gko) <= 1e-8
    assert _relerr(r["grad_bz"], gbo) <= 1e-8


def _hier_disk_context(mixed=False):
    """A disk large enough for admissible boundary blocks: dense matrix kept, hierarchical form
    (leaf 32, eta 2, ACA to 1e-10 / 1e-6) selected."""
    mesh = meshgen.jittered_disk(90.0, 9.0, 3.0, seed=8)
    mo, ctx, mat = _device_setup(mesh, tol=1e-13 if not mixed else 1e-10, mixed=mixed)
    ctx.bem_assemble(mo, accurate=True)   # far-field-accurate weights: compressible to 1e-10
    bd = mo.boundary()
    bn = bd["bnodes"]
    ctx.bem_compress(mesh.xyz[bn], leaf=32, eta=2.0, eps_mixed=1e-6, eps_fp64=1e-10, kmax=64, keep_dense=True)
    assert ctx.bem_info()["lowrank_blocks"] > 0
    return mesh, mo, ctx, mat, bn


@pytest.mark.gpu
def test_hierarchical_transposed_product():
    # B^T through the hierarchical form (transposed tiles, U and V exchanged, column-cluster work
    # lists) against the dense B^T, and <y, H x> = <H^T y, x> for the hierarchical matrix itself
    mesh, mo, ctx, _, bn = _hier_disk_context()
    nb = bn.size
    rng = np.random.default_rng(3)
    x, y = rng.standard_normal(nb), rng.standard_normal(nb)
    for mixed, tol_dense, tol_sym in ((False, 1e-8, 1e-13), (True, 2e-5, 1e-6)):
        ctx.set_precision(mixed)
        ctx.set_bem_mode(0)
        bx, bty = ctx.bem_apply(x), ctx.bem_apply(y, transpose=True)
        ctx.set_bem_mode(1)
        hx, hty = ctx.bem_apply(x), ctx.bem_apply(y, transpose=True)
        assert _relerr(hx, bx) <= tol_dense, mixed
        assert _relerr(hty, bty) <= tol_dense, mixed
        assert abs(y @ hx - hty @ x) <= tol_sym * abs(y @ hx), mixed
        if not mixed:
            assert abs(y @ bx - bty @ x) <= 1e-13 * abs(y @ bx)
    ctx.set_precision(False)
    # the dense B^T against the dense matrix itself
    B = ctx.get_bem_dense()
    ctx.set_bem_mode(0)
    assert _relerr(ctx.bem_apply(y, transpose=True), B.T @ y) <= 1e-14


@pytest.mark.gpu
def test_device_adjoint_hierarchical_bem():
    # the adjoint through the hierarchical boundary matrix: directional finite differences of the
    # same forward map, and the dense-matrix adjoint within the compression error
    mesh, mo, ctx, (Js, A_, axis, D), bn = _hier_disk_context()
    n = mesh.nx
    m0 = meshgen.skyrmion_state(mesh.xyz, 4, radius=22.0, wall=5.0)
    nsteps, dt, nsub = 2, 1.0, 6
    rng = np.random.default_rng(9)
    bz0 = 0.02 + 0.01 * rng.standard_normal(5)
    ku0 = 1e4 * rng.uniform(0, 1, n)
    ctx.set_material(Js, A_, Ku=ku0, ku_axis=axis, D=D, alpha=0.3)
    ctx.set_dmi_kind(True)
    ctx.set_bz_pulse(bz0, 0.0, nsteps * dt)
    vol = mo.operators()["node_vol"]
    wv = np.zeros(3 * n)
    wv[2 * n:] = vol / vol.sum()
    res = {}
    for mode in (1, 0):
        ctx.set_bem_mode(mode)
        res[mode] = ctx.adjoint_rk4(m0.copy(), wv, nsteps, dt, nsub, ckpt_every=1, n_bz=bz0.size)
    g1, g0 = res[1], res[0]
    assert _relerr(g1["grad_m0"], g0["grad_m0"]) <= 1e-7
    assert _relerr(g1["grad_ku"], g0["grad_ku"]) <= 1e-7
    assert _relerr(g1["grad_bz"], g0["grad_bz"]) <= 1e-7
    ctx.set_bem_mode(1)

    def J(m_):
        m = m_.copy()
        ctx.step_rk4(m, nsteps, dt, nsub)
        return float(wv @ m)

    assert abs(J(m0) - g1["J"]) <= 1e-11
    for k in range(2):
        v = rng.standard_normal(3 * n)
        fd = (J(m0 + 1e-5 * v) - J(m0 - 1e-5 * v)) / 2e-5
        assert abs(fd - g1["grad_m0"] @ v) <= 1e-6 * abs(g1["grad_m0"] @ v), k
