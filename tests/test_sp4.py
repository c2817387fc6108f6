"""Parity pin against the reference's own output: muMAG standard problem 4 on its mesh.

The reference documents one run of its own (examples/example2, doc/examples/example2.rst):

1. the zero-field "s-state" of the 500 x 125 x 3 nm Permalloy platelet (mesh sp4_.vtk, 16,602
   nodes) by a hysteresis branch from 1000 mT to 0 mT in 200 mT steps at theta = phi = 45 deg,
   alpha = 1, precession removed, demag refreshed every 0.5 ps, each field relaxed until the
   maximum torque is below 5e-4 T (simulation.cfg_static; the loop of TheSimulation::start,
   main/TheSimulation.cpp:231-341);
2. the switching under 25 mT at theta = 90, phi = 170 deg with alpha = 0.02 and demag refreshed
   every 0.1 ps (simulation.cfg_dyn), whose .log rows at t = 132 .. 140 ps are quoted in the
   documentation (example2.rst:113-120; tests/golden/make_sp4.py extracts them with the mesh).

This test runs both stages through the C ABI on the plain FP64 path (dense BEM assembled on the
device with tetmag's Lindholm arithmetic; the reference's default used its H2 approximation of
the same matrix) and compares the volume-weighted mean magnetisation with those rows.  Measured:
the trajectory runs 3.1 ps (2.3 %) ahead of the reference's -- the first zero crossing of <m_x>
comes at 134.0 ps where the rows place it at 137.0 ps -- and once shifted by that time it agrees
with every row to 5e-3; at those shifted times the total and demag energy densities agree to
0.6 % and 0.9 %, the exchange energy is 8 % lower.  The s-state is defined by a torque threshold
rather than a unique end point, and the reference integrated with CVODE (Adams,
rtol = atol = 1e-6, a weighted RMS error
norm, main/TheLLG.cpp:605-618) where this path uses Dormand-Prince 5(4) with a max-norm error at
the same tolerances; over 140 ps of low-damping dynamics such differences shift the switching
time.  So the test pins the trajectory up to a small time shift: the best shift within +-4 ps,
the rows within 1e-2 after it, and the energy densities at the shifted times (ENERGY_TOL).
"""
from pathlib import Path

import numpy as np
import pytest

from tetmag_b200 import meshgen
from tetmag_b200.api import Context, MeshOps

GOLDEN = Path(__file__).with_name("golden")
MU0 = 1.256637061435917295376e-6
JS = 1.00530964914872800000                 # examples/example2/material001.dat
A_EX = 1.3e-11

MAX_SHIFT_PS = 4.0     # |time shift| of the best alignment with the reference's rows
SHIFTED_TOL = 1e-2     # |<m>_here(t + shift) - <m>_reference(t)| per component, t = 132 .. 140 ps
# relative energy densities at the shifted times: total and demag agree closely (measured 0.6 %
# and <= 0.9 %); the exchange energy of this run's switching texture is systematically lower
# (measured 8.2-8.5 %), which the tolerance records rather than hides
ENERGY_TOL = {"total": 0.02, "demag": 0.02, "exchange": 0.10}


def sp4_context(mixed: bool = False):
    g = np.load(GOLDEN / "sp4_mesh.npz")
    mo = MeshOps(g["xyz"], g["tets"])
    ctx = Context(0)
    ctx.set_mesh(mo)
    ctx.bem_assemble(mo)
    ctx.set_precision(mixed)
    ctx.set_solver_params(1e-10 if not mixed else 1e-7, 300)
    return mo, ctx


def set_material(ctx, n, alpha):
    ctx.set_material(np.full(n, JS), np.full(n, A_EX / 1e-18), alpha=alpha)


def mean_m(m, vol):
    return m.reshape(3, -1) @ vol / vol.sum()


def s_state(ctx, mo, torque_limit=5e-4, cap_ps=5000.0):
    """Hysteresis branch 1000 -> 0 mT (200 mT steps, 45 / 45 deg), alpha = 1, no precession,
    0.5 ps segments, each field relaxed until the max torque is below the limit."""
    n = mo.nx
    set_material(ctx, n, 1.0)
    ctx.set_llg_options(precession=False)
    m = meshgen.uniform_state(n, (1.0, 0.0, 0.0))      # homogeneous_x
    segments = []
    for b_mt in (1000, 800, 600, 400, 200, 0):
        ctx.set_applied_field(meshgen.field_from_angles(n, b_mt * 1e-3, 45.0, 45.0))
        ctx.demag_field(m)
        torque = ctx.max_torque(m)
        t, k = 0.0, 0
        while t < cap_ps - 1e-9 and torque > torque_limit:
            st = ctx.relax(m, duration_ps=0.5, segment_ps=0.5)
            torque = st["max_torque"]
            t += 0.5
            k += 1
        segments.append(k)
    ctx.set_llg_options(precession=True)
    return m, segments


def switching(ctx, mo, m, until_ps=150.0, log_ps=1.0):
    """25 mT at 90 / 170 deg, alpha = 0.02, 0.1 ps segments; the state logged every log_ps."""
    n = mo.nx
    set_material(ctx, n, 0.02)
    ctx.set_applied_field(meshgen.field_from_angles(n, 0.025, 90.0, 170.0))
    vol = mo.operators()["node_vol"]
    log = {}
    t = 0.0
    while True:
        log[round(t, 6)] = (mean_m(m, vol), ctx.energies(m))
        if t >= until_ps - 1e-9:
            break
        ctx.relax(m, duration_ps=log_ps, segment_ps=0.1)
        t += log_ps
    return log


def align(log, rows):
    """Best time shift (0.05 ps grid within MAX_SHIFT_PS) of the logged trajectory against the
    reference rows, and the largest component difference after it."""
    t = np.array(sorted(log))
    m = np.array([log[k][0] for k in t])

    def at(tt):
        return np.array([np.interp(tt, t, m[:, d]) for d in range(3)])

    best = (0.0, np.inf)
    for sh in np.arange(-MAX_SHIFT_PS, MAX_SHIFT_PS + 1e-9, 0.05):
        r = max(float(np.abs(at(row[0] + sh) - row[10:13]).max()) for row in rows)
        if r < best[1]:
            best = (float(sh), r)
    return best


@pytest.mark.gpu
def test_sp4_against_reference_log_rows():
    mo, ctx = sp4_context()
    rows = np.load(GOLDEN / "sp4_log_rows.npz")["rows"]
    m, segs = s_state(ctx, mo)
    assert all(0 < k < 10000 for k in segs[1:]), segs     # every field step converged below the cap
    vol = mo.operators()["node_vol"]
    ms = mean_m(m, vol)
    # the s-state: magnetisation along +x on average, small +y from the 45 deg history
    assert ms[0] > 0.9 and 0.05 < ms[1] < 0.2 and abs(ms[2]) < 0.05, ms
    log = switching(ctx, mo, m, until_ps=float(rows[-1, 0]) + MAX_SHIFT_PS + 1.0)
    shift, resid = align(log, rows)
    assert abs(shift) < MAX_SHIFT_PS and resid <= SHIFTED_TOL, (shift, resid)
    # energies at the shifted times (linear between the logged times)
    times = np.array(sorted(log))
    for r in rows:
        for key, col in (("total", 1), ("demag", 2), ("exchange", 3)):
            e = np.interp(r[0] + shift, times, [log[k][1][key] for k in times])
            assert abs(e - r[col]) <= ENERGY_TOL[key] * abs(r[col]), (r[0], key, e, r[col])
    # <m_x> crosses zero once in this window, a few ps from the reference's 136 .. 138 ps
    mx = np.array([log[k][0][0] for k in times])
    i = next(i for i in range(1, len(mx)) if mx[i - 1] > 0.0 >= mx[i])
    assert abs(times[i] - 137.0) <= MAX_SHIFT_PS + 1.0, times[i]
    print(f"sp4: s-state <m> = {ms}, field-step segments {segs}, shift {shift:+.2f} ps, "
          f"residual after shift {resid:.2e}")
