"""Run-length and full-size parity against the FP64 oracle (fixtures by tests/golden/make_parity.py).

* c1, the whole configured run: 1 ns of frozen-demag Dormand-Prince relaxation (0.5 ps segments)
  of the 1,323-node cuboid from its seeded random state; the mean magnetisation after the run
  within 1e-4 of the oracle's (the bound the workloads state for the mean magnetisation), on the plain
  FP64 path and the mixed path.
* c4 at full size (28,611 nodes, 7,002 boundary nodes, dense BEM): demag field and LLG right-hand
  side of a seeded random state against the oracle's direct solves, 1e-10 on the plain FP64 path
  and 1e-5 on the mixed path.
* c4's whole configured run for replica 0 (1 ns at alpha = 0.5 from its seeded random state in its
  applied field) and c3's whole 0.5 ns run for three dots of the 256-dot batch (the batch stepped in
  one context, each dot run alone by the oracle): the mean magnetisation after every 100 ps within
  1e-4 of the oracle's, on both paths.  c3's dots precess for the whole run (alpha = 0.1), so both
  integrators run at tolerance 1e-8 there: at tetmag's 1e-6 the step control alone moves a dot's
  mean m by up to 1e-3 within 200 ps.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import tetmag_oracle as O
from tetmag_b200 import meshgen, workloads

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).with_name("golden")
FP64_TOL = 1e-10
MIXED_TOL = 1e-5
MEAN_M_TOL = 1e-4


def rel(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _mean_m(m_soa, vol):
    return m_soa.reshape(3, -1) @ vol / vol.sum()


@pytest.mark.parametrize("mixed", [False, True])
def test_c1_relaxation_1ns_mean_m(mixed):
    g = np.load(GOLDEN / "c1_relax_1ns.npz")
    w = workloads.c1()
    mo, ctx = workloads.setup_context(w, mixed=mixed, tol=1e-12 if not mixed else 1e-8, maxiter=300)
    m = w.m0.copy()
    st = ctx.relax(m, duration_ps=1000.0, segment_ps=0.5)
    vol = mo.operators()["node_vol"]
    got = _mean_m(m, vol)
    assert st["segments"] == int(g["segments"]) == 2000
    assert np.max(np.abs(got - g["mean_m"])) <= MEAN_M_TOL, (got, g["mean_m"])
    # the step counts of the two Dormand-Prince loops agree closely
    assert abs(st["accepted"] - int(g["accepted"])) <= max(5, 0.02 * int(g["accepted"]))
    assert abs(st["max_torque"] - float(g["max_torque"])) <= 1e-2 * float(g["max_torque"])


@pytest.fixture(scope="module")
def c4():
    g = np.load(GOLDEN / "c4_field.npz")
    w = workloads.c4_replica(replica=0)
    mo, ctx = workloads.setup_context(w, tol=1e-13, maxiter=400)
    m = meshgen.random_state(w.n, int(g["state_seed"]))
    return g, w, mo, ctx, m


def test_c4_full_size_fp64_against_oracle(c4):
    g, w, mo, ctx, m = c4
    ctx.set_precision(False)
    ctx.set_solver_params(1e-13, 400)
    h = np.empty(3 * w.n)
    y = ctx.field_eval(m, hdem=h)
    assert rel(h, g["hdem"]) <= FP64_TOL
    assert rel(y, g["ydot"]) <= FP64_TOL
    assert abs(ctx.max_torque(m) - float(g["torque"])) <= 1e-9 * float(g["torque"])


def test_c4_full_size_mixed_against_oracle(c4):
    g, w, mo, ctx, m = c4
    ctx.set_precision(True)
    ctx.set_solver_params(1e-8, 400)
    try:
        h = np.empty(3 * w.n)
        y = ctx.field_eval(m, hdem=h)
        assert rel(h, g["hdem"]) <= MIXED_TOL
        assert rel(y, g["ydot"]) <= MIXED_TOL
    finally:
        ctx.set_precision(False)
        ctx.set_solver_params(1e-13, 400)


def test_c4_full_size_hierarchical_against_oracle(c4):
    # the hierarchical BEM built from the mesh (no dense matrix), plain FP64 terms: field error
    # against the oracle's dense-matrix field within the compression's accuracy
    g, w, _, _, m = c4
    mo, ctx = workloads.setup_context(w, tol=1e-13, maxiter=400, hmatrix="mesh", keep_dense=False)
    h = np.empty(3 * w.n)
    ctx.field_eval(m, hdem=h)
    assert rel(h, g["hdem"]) <= 1e-6
    ctx.set_precision(True)
    ctx.set_solver_params(1e-8, 400)
    ctx.field_eval(m, hdem=h)
    assert rel(h, g["hdem"]) <= MIXED_TOL


@pytest.mark.parametrize("mixed", [False, True])
def test_c4_run_1ns_mean_m(mixed):
    g = np.load(GOLDEN / "c4_relax_1ns.npz")
    w = workloads.c4_replica(replica=0)
    mo, ctx = workloads.setup_context(w, mixed=mixed, tol=1e-12 if not mixed else 1e-8, maxiter=300)
    vol = mo.operators()["node_vol"]
    m = w.m0.copy()
    for k in range(len(g["mean_m"])):
        ctx.relax(m, duration_ps=float(g["chunk_ps"]), segment_ps=float(g["segment_ps"]))
        got = _mean_m(m, vol)
        assert np.max(np.abs(got - g["mean_m"][k])) <= MEAN_M_TOL, (k, got, g["mean_m"][k])


@pytest.mark.parametrize("mixed", [False, True])
def test_c3_batch_run_sampled_dots_mean_m(mixed):
    g = np.load(GOLDEN / "c3_dots_run.npz")
    w = workloads.c3_dots(256, 3)
    mo, ctx = workloads.setup_context(w, mixed=mixed, tol=1e-12 if not mixed else 1e-8, maxiter=300)
    vol = mo.operators()["node_vol"]
    off = np.asarray(w.components)
    m = w.m0.copy()
    eps = float(g["eps"])
    for k in range(g["mean_m"].shape[1]):
        ctx.relax(m, duration_ps=float(g["chunk_ps"]), segment_ps=float(g["segment_ps"]), eps_abs=eps, eps_rel=eps)
        mm = m.reshape(3, -1)
        for i, c in enumerate(g["dots"]):
            lo, hi = int(off[c]), int(off[c + 1])
            assert hi - lo == int(g["nodes"][i])
            got = mm[:, lo:hi] @ vol[lo:hi] / vol[lo:hi].sum()
            assert np.max(np.abs(got - g["mean_m"][i, k])) <= MEAN_M_TOL, (int(c), k, got, g["mean_m"][i, k])
