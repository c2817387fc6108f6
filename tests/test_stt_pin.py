"""Parity pin against the reference's own output: the spin-transfer-torque standard problem.

The reference documents one run of its own (examples/example3, doc/examples/example3.rst):

1. a vortex ("vortex_xy": core of radius 2 nm along +z at the origin, in-plane curl
   m = (-y, x, 0)/r around it, specs/InitMag.cpp:203-225) in the 100 x 100 x 10 nm Permalloy
   square of mesh sp_stt.vtk (10,269 nodes), relaxed with alpha = 1, precession removed and the
   demag field refreshed every 2 ps until the maximum torque is below 1e-4 T (simulation.cfg_static;
   the loop of TheSimulation::start, main/TheSimulation.cpp:231-341);
2. 14 ns of Zhang-Li dynamics (TheLLG::sttDynamics and calcUtermSTT, main/TheLLG.cpp:201-220,
   402-415) under a dc current of 1e12 A/m^2 along x with polarisation 1 and beta = 0.05, alpha =
   0.1, the demag field refreshed every 0.1 ps (simulation.cfg_dynamic).

Its documentation quotes the mean magnetisation of the equilibrium reached after 14 ns:
<M_x> = -1.7009e5 A/m, <M_y> = 1.566e4 A/m (example3.rst:68; tests/golden/make_stt.py extracts
them with the mesh).  This test runs both stages through the C ABI on the plain FP64 path and
compares the volume-weighted mean magnetisation with them (measured: -170,097.4 and 15,660.6 A/m;
the static stage ends after 1,336 ps; 160 s on one B200).  The STT coefficients are the reference's
(STT::setEta and the constructor's btimesMs, specs/ProgramSpecs.cpp:405-421): per node
eta_d = j_d P mu_B mu0 / (gamma0 e (1 + beta^2) scale Js).
"""
from pathlib import Path

import numpy as np
import pytest

from tetmag_b200.api import Context, MeshOps

GOLDEN = Path(__file__).with_name("golden")
MU0 = 1.256637061435917295376e-6
GAMMA0 = 221276.14886372426        # rad m / (A s)
MU_B = 9.274009994e-24             # J/T
E_CHARGE = 1.6021766208e-19        # C
SCALE = 1e-9

# |<M>_here - <M>_reference| per component, in A/m (Ms = 8e5 A/m).  Measured: 7.4 A/m (x) and
# 0.6 A/m (y) on both precision paths, within the rounding of the quoted values (5 A/m); the
# vortex still circles the equilibrium at 14 ns (the last nanosecond moves <M_y> by 84 A/m), so
# the bound allows for a small phase difference of that residual motion.
MEAN_M_TOL = 100.0
SETTLE_TOL = 250.0    # |<M>(14 ns) - <M>(13 ns)| per component


def vortex_xy(xyz):
    """specs/InitMag.cpp:203-225: +z inside radius 2 (mesh units), (-y, x, 0)/r outside."""
    d = xyz[:, :2]
    r = np.linalg.norm(d, axis=1)
    m = np.zeros_like(xyz)
    core = r < 2.0
    m[core, 2] = 1.0
    rs = np.where(core, 1.0, r)
    m[~core, 0] = -d[~core, 1] / rs[~core]
    m[~core, 1] = d[~core, 0] / rs[~core]
    return np.ascontiguousarray(m.T.ravel())


def stt_eta(g, n):
    """STT::setEta: the current direction times P mu_B mu0 / (gamma0 e (1 + beta^2) scale) / Js."""
    th, ph = np.radians(float(g["current_theta"])), np.radians(float(g["current_phi"]))
    jc = 1e12 * float(g["current_density"]) * np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph),
                                                          np.cos(th)])
    beta = float(g["beta"])
    btimes_ms = float(g["polarization"]) * MU_B * MU0 / (GAMMA0 * E_CHARGE * (1.0 + beta * beta)) / SCALE
    js = MU0 * float(g["Ms"])
    return np.repeat(jc * btimes_ms / js, n)


def mean_m(m, vol):
    return m.reshape(3, -1) @ vol / vol.sum()


def run_stt_problem(mixed=False, log=None):
    g = np.load(GOLDEN / "stt_reference.npz")
    mesh = np.load(GOLDEN / "stt_mesh.npz")
    mo = MeshOps(mesh["xyz"], mesh["tets"])
    n = mo.nx
    ctx = Context(0)
    ctx.set_mesh(mo)
    ctx.bem_assemble(mo)
    ctx.set_precision(mixed)
    ctx.set_solver_params(1e-10 if not mixed else 1e-7, 300)
    js = np.full(n, MU0 * float(g["Ms"]))
    a = np.full(n, float(g["A"]) / SCALE ** 2)
    vol = mo.operators()["node_vol"]
    # static stage: alpha = 1, no precession, demag refreshed every 2 ps, torque below the limit
    ctx.set_material(js, a, alpha=float(g["static_alpha"]))
    ctx.set_applied_field(np.zeros(3 * n))
    ctx.set_llg_options(precession=False)
    m = vortex_xy(mesh["xyz"])
    ctx.demag_field(m)
    torque, t, seg = ctx.max_torque(m), 0.0, float(g["static_segment_ps"])
    while t < float(g["static_duration_ps"]) - 1e-9 and torque > float(g["torque_limit"]):
        torque = ctx.relax(m, duration_ps=seg, segment_ps=seg)["max_torque"]
        t += seg
    static = (t, torque, mean_m(m, vol))
    # dynamic stage: Zhang-Li torque under the dc current, demag refreshed every 0.1 ps
    ctx.set_llg_options(precession=True)
    ctx.set_material(js, a, alpha=float(g["alpha"]))
    ctx.set_stt(stt_eta(g, n), beta=float(g["beta"]), scale=1.0)
    total, chunk = float(g["duration_ps"]), 1000.0
    done = 0.0
    while done < total - 1e-9:
        ctx.relax(m, duration_ps=min(chunk, total - done), segment_ps=float(g["segment_ps"]))
        done += min(chunk, total - done)
        if log is not None:
            log.append((done, mean_m(m, vol) * float(g["Ms"])))
    return g, static, mean_m(m, vol) * float(g["Ms"])


@pytest.mark.gpu
def test_stt_standard_problem_against_reference_mean_m():
    log = []
    g, static, M = run_stt_problem(mixed=False, log=log)
    t_static, torque, m_static = static
    # the relaxed vortex: centred, so the in-plane mean is small, the core along +z
    assert torque <= float(g["torque_limit"]) and np.abs(m_static[:2]).max() < 0.02 and m_static[2] > 0.0, static
    assert abs(M[0] - float(g["mean_Mx"])) <= MEAN_M_TOL, (M, log[-3:])
    assert abs(M[1] - float(g["mean_My"])) <= MEAN_M_TOL, (M, log[-3:])
    # nearly settled: the last nanosecond moves the mean by little
    assert np.abs(log[-1][1] - log[-2][1]).max() <= SETTLE_TOL, log[-3:]
    print(f"stt: static {t_static:g} ps, <M> after {log[-1][0]:g} ps = {M} A/m")
