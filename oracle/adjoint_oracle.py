"""FP64 CPU oracle of the fixed-step LLG integration and its discrete adjoint.

TEST INFRASTRUCTURE ONLY (the checker): tests/ and bench.py's CPU legs import it,
the product never does.

tetmag has no adjoint; what is differentiated here is tetmag's right-hand side
(TheLLG::rhs, main/TheLLG.cpp:670-711, with the full effective field of
TheLLG::totalEffectiveField, main/TheLLG.cpp:238-254, and the demag field of
DemagField::calcField, main/DemagField.cpp:92-113, refreshed at every stage)
integrated with the classical fixed-step Runge-Kutta 4 scheme (nsub substeps
per time step) and renormalised after every time step like
TheSimulation::start (main/TheSimulation.cpp:404-411).  The applied field is the
static field plus a piecewise-linear Bz(t) pulse sampled uniformly in time
(a generalisation of tetmag's pulse field, main/TheLLG.cpp:320-332).

The objective is linear in the final state, J = sum_k w_k y_N[k]; the
gradients are taken with respect to the initial state, the per-node uniaxial
constant Ku (main/EffFieldCalc.cpp:71-84) and the Bz samples.  Every
transpose is an explicit sparse / dense transpose of the oracle's own
matrices, and the two pinned linear systems are solved transposed with their
SuperLU factors, so this is an independent reference for the device adjoint.
"""
from __future__ import annotations

import numpy as np

from oracle import tetmag_oracle as O


def pulse_weights(ns: int, t0_ps: float, t1_ps: float, t_ps: float):
    """Hat-function weights of the ns uniformly spaced samples at time t (held outside)."""
    w = np.zeros(ns)
    if ns == 0:
        return w
    if ns == 1 or t_ps <= t0_ps:
        w[0] = 1.0
        return w
    if t_ps >= t1_ps:
        w[-1] = 1.0
        return w
    u = (t_ps - t0_ps) / (t1_ps - t0_ps) * (ns - 1)
    k = min(int(np.floor(u)), ns - 2)
    f = u - k
    w[k] = 1.0 - f
    w[k + 1] = f
    return w


class Dynamics:
    """Field, right-hand side and their transposes for one problem (bulk, interfacial or no DMI)."""

    def __init__(self, pb: O.Problem, dem: O.DemagOracle, bz=None, t0_ps=0.0, t1_ps=0.0):
        if np.any(pb.D != 0.0) and pb.dmi_kind not in ("bulk", "interfacial"):
            raise ValueError(f"unknown DMI form {pb.dmi_kind!r}")
        self.pb, self.dem = pb, dem
        self.bz = np.zeros(0) if bz is None else np.asarray(bz, np.float64)
        self.t0, self.t1 = t0_ps, t1_ps
        self.ij = O.inv_js(pb)
        V = pb.fem.node_vol
        self.W = V * pb.Js
        self.xcK = (-2.0 * pb.A / V * self.ij)                 # row scale of the exchange operator

    def hz(self, t_ps):
        if self.bz.size == 0:
            return 0.0
        return float(pulse_weights(self.bz.size, self.t0, self.t1, t_ps) @ self.bz) / O.MU0

    def field(self, m, t_ps):
        pb = self.pb
        H = O.local_field(pb, m, self.dem.field(m))
        H[:, 2] += self.hz(t_ps)
        return H

    def rhs(self, m, t_ps):
        H = self.field(m, t_ps)
        return O.llg_rhs(self.pb, m, H), H

    # ---- transposes of the linear field operator ----------------------------------------
    def demag_t(self, mu):
        """Transpose of m -> H_dem (divergence, pinned Neumann solve, BEM, Dirichlet solve, -grad)."""
        pb, dem = self.pb, self.dem
        g = pb.fem.grad
        w = -(g[0].T @ mu[:, 0] + g[1].T @ mu[:, 1] + g[2].T @ mu[:, 2])
        v = dem.lu_dir.solve(w, trans="T")
        bn = pb.bnd.bnodes
        a = w.copy()
        a[bn] += pb.B.T @ v[bn]
        a1 = dem.lu_neu.solve(a, trans="T")
        tg = pb.fem.tgrad
        return np.stack([tg[d].T @ a1 for d in range(3)], axis=1) * (pb.Js / O.MU0)[:, None]

    def field_t(self, mu):
        """Transpose of the linear part of m -> H (exchange, uniaxial, interfacial DMI, demag)."""
        pb = self.pb
        out = pb.fem.stiff.T @ (self.xcK[:, None] * mu)
        km = np.sum(pb.ku_axis * mu, axis=1)
        out += (2.0 * pb.Ku * self.ij * km)[:, None] * pb.ku_axis
        if np.any(pb.D != 0.0) and pb.dmi_kind == "interfacial":
            out += self.W[:, None] * O.interfacial_dmi_field(pb, mu / self.W[:, None]) * self.ij[:, None]
        elif np.any(pb.D != 0.0):
            out += self.bulk_dmi_t(mu)
        return out + self.demag_t(mu)

    def bulk_dmi_t(self, mu):
        """Transpose of m -> H_dmi / Js for the bulk form (EffFieldCalc::dmiField, surfIntDMI and
        curlM, main/EffFieldCalc.cpp:159-170, 280-298): H = ds (a m x n - 2 curl m) with
        ds = D / (V Js) and curl m built from -tGrad; the transpose is ds a (n x mu) plus the
        explicit transposes of the tGrad matrices applied to ds mu."""
        pb = self.pb
        ds = pb.D / pb.fem.node_vol * self.ij
        v = ds[:, None] * mu
        tx, ty, tz = pb.fem.tgrad
        out = (ds * pb.bnd.node_area)[:, None] * np.cross(pb.bnd.node_normal, mu)
        # -2 curl m = 2 [ty mz - tz my, tz mx - tx mz, tx my - ty mx] (tGrad itself, not -tGrad)
        out[:, 0] += 2.0 * (tz.T @ v[:, 1] - ty.T @ v[:, 2])
        out[:, 1] += 2.0 * (tx.T @ v[:, 2] - tz.T @ v[:, 0])
        out[:, 2] += 2.0 * (ty.T @ v[:, 0] - tx.T @ v[:, 1])
        return out

    def vjp(self, m, H, abar, t_ps):
        """(df/dm)^T abar and the parameter pieces (dKu per node, dJ/dHz scalar) at one stage."""
        al = self.pb.alpha
        mu = np.cross(m, abar) - al * np.cross(m, np.cross(m, abar))
        mH = np.sum(m * H, axis=1, keepdims=True)
        ma = np.sum(m * abar, axis=1, keepdims=True)
        Ha = np.sum(H * abar, axis=1, keepdims=True)
        g = np.cross(abar, H) - al * (mH * abar + ma * H - 2.0 * Ha * m)
        g += self.field_t(mu)
        pb = self.pb
        dku = 2.0 * self.ij * np.sum(pb.ku_axis * m, axis=1) * np.sum(pb.ku_axis * mu, axis=1)
        dhz = float(np.sum(mu[:, 2]))
        return g, dku, dhz


def _rk4_substep(dyn: Dynamics, y, t, dt_ps, h, keep=None):
    k1, H1 = dyn.rhs(y, t)
    Y2 = y + 0.5 * h * k1
    k2, H2 = dyn.rhs(Y2, t + 0.5 * dt_ps)
    Y3 = y + 0.5 * h * k2
    k3, H3 = dyn.rhs(Y3, t + 0.5 * dt_ps)
    Y4 = y + h * k3
    k4, H4 = dyn.rhs(Y4, t + dt_ps)
    if keep is not None:
        keep.append(([y, Y2, Y3, Y4], [H1, H2, H3, H4]))
    return y + h / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4)


def rk4_forward(dyn: Dynamics, m0, nsteps, dt_ps, nsub=1, normalize=True, t0_ps=0.0):
    """nsteps steps of dt_ps, each nsub classical RK4 substeps in reduced time, then (normalize)
    m -> m / |m| per node as tetmag does after every time step (main/TheSimulation.cpp:404-411)."""
    ds = dt_ps / nsub
    h = ds * dyn.pb.time_scale()
    y = np.array(m0, np.float64)
    for k in range(nsteps):
        for s in range(nsub):
            y = _rk4_substep(dyn, y, t0_ps + k * dt_ps + s * ds, ds, h)
        if normalize:
            y = y / np.linalg.norm(y, axis=1, keepdims=True)
    return y


def rk4_adjoint(dyn: Dynamics, m0, nsteps, dt_ps, w, nsub=1, normalize=True, t0_ps=0.0):
    """J = sum(w * y_N) of rk4_forward and its gradients: (J, y_N, dJ/dm0, dJ/dKu, dJ/dbz).

    Discrete adjoint, store-all (the device checkpoints instead).  One RK4 substep
    y' = y + h/6 (k1 + 2 k2 + 2 k3 + k4), stages Y1..Y4 at t, t+h/2, t+h/2, t+h, maps the
    adjoint lam' to lam = lam' + g1 + g2 + g3 + g4 with g_i = (df/dy)(Y_i)^T a_i and
    a4 = h/6 lam', a3 = h/3 lam' + h g4, a2 = h/3 lam' + h/2 g3, a1 = h/6 lam' + h/2 g2;
    the parameter gradients collect (df/dp)(Y_i)^T a_i.  The normalisation y = z/|z| maps
    lam to (lam - y (y . lam)) / |z| per node.
    """
    ds = dt_ps / nsub
    h = ds * dyn.pb.time_scale()
    y = np.array(m0, np.float64)
    steps = []
    for k in range(nsteps):
        y0 = y
        subs = []
        for s in range(nsub):
            y = _rk4_substep(dyn, y, t0_ps + k * dt_ps + s * ds, ds, h, keep=subs)
        zn = np.linalg.norm(y, axis=1, keepdims=True)
        if normalize:
            y = y / zn
        steps.append((y0, subs, zn, y))
    lam = np.array(w, np.float64)
    n = dyn.pb.nx
    dku = np.zeros(n)
    dbz = np.zeros(dyn.bz.size)
    for k in range(nsteps - 1, -1, -1):
        _, subs, zn, yk = steps[k]
        if normalize:
            lam = (lam - yk * np.sum(yk * lam, axis=1, keepdims=True)) / zn
        for s in range(nsub - 1, -1, -1):
            Y, Hs = subs[s]
            t = t0_ps + k * dt_ps + s * ds
            times = [t, t + 0.5 * ds, t + 0.5 * ds, t + ds]
            a4 = h / 6.0 * lam
            g4, p4, z4 = dyn.vjp(Y[3], Hs[3], a4, times[3])
            a3 = h / 3.0 * lam + h * g4
            g3, p3, z3 = dyn.vjp(Y[2], Hs[2], a3, times[2])
            a2 = h / 3.0 * lam + 0.5 * h * g3
            g2, p2, z2 = dyn.vjp(Y[1], Hs[1], a2, times[1])
            a1 = h / 6.0 * lam + 0.5 * h * g2
            g1, p1, z1 = dyn.vjp(Y[0], Hs[0], a1, times[0])
            lam = lam + g1 + g2 + g3 + g4
            dku += p1 + p2 + p3 + p4
            for zi, ti in zip((z1, z2, z3, z4), times):
                dbz += zi / O.MU0 * pulse_weights(dyn.bz.size, dyn.t0, dyn.t1, ti)
    yN = steps[-1][3] if steps else np.array(m0, np.float64)
    return float(np.sum(w * yN)), yN, lam, dku, dbz


def problem_with_ku(pb: O.Problem, Ku):
    """A copy of the problem with a new per-node Ku (the differentiated parameter)."""
    import dataclasses
    return dataclasses.replace(pb, Ku=np.broadcast_to(np.asarray(Ku, np.float64), (pb.nx,)).copy())


def mean_mz_weights(pb: O.Problem):
    """dJ/dy of J = mean m_z (volume-weighted, TheSimulation::getMeanM) in node-row layout."""
    V = pb.fem.node_vol
    w = np.zeros((pb.nx, 3))
    w[:, 2] = V / V.sum()
    return w
