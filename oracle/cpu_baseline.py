"""Timed CPU baseline of one full field evaluation, from bounded samples.

TEST / BENCH INFRASTRUCTURE ONLY (the cpu_baseline leg and the reference arm
of bench.py).  One field evaluation is the oracle's

    local field + LLG right-hand side          (main/TheLLG.cpp:150-254)
  + divergence, gradient                        (main/DemagField.cpp:102-136)
  + Neumann and Dirichlet solves                (main/DemagField.cpp:223-240)
  + dense BEM matvec                            (main/DemagField.cpp:145-147)

on the host cores.  Solves are conjugate gradients with a Jacobi
preconditioner to the reference's relative tolerance (1e-7, 100-iteration cap
of AMGCLSolver lifted), on the same symmetric-eliminated systems; the dense
BEM matvec is timed on a row sample of an Nb x Nb FP64 matrix and scaled to Nb
rows (a GEMV costs the same whatever the values; assembling the dense c2
matrix on the CPU would take hours).  Large meshes cannot afford the
reference's default SparseLU here (115 s and 3 GB of factors for 363k nodes).
"""
from __future__ import annotations

import os
import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import tetmag_oracle as O


def _eliminate(K: sp.csr_matrix, fixed: np.ndarray):
    """Symmetric elimination of the unit-row constraints of the reference's
    Neumann / Dirichlet matrices: returns (A_FF, A_FC, free, fixed)."""
    n = K.shape[0]
    mask = np.zeros(n, bool)
    mask[fixed] = True
    free = np.flatnonzero(~mask)
    Kc = K.tocsc()
    A_ff = Kc[free][:, free].tocsr()
    A_fc = Kc[free][:, fixed].tocsr()
    return A_ff, A_fc, free, np.flatnonzero(mask)


class CpuFieldEval:
    def __init__(self, pb: O.Problem, tol: float = 1e-7, bem_rows: int = 400, seed: int = 0):
        self.pb = pb
        self.tol = tol
        n = pb.nx
        self.k = n // 2
        self.neu = _eliminate(pb.fem.stiff, np.array([self.k]))
        self.dir = _eliminate(pb.fem.stiff, pb.bnd.bnodes)
        for A in (self.neu[0], self.dir[0]):
            A.sort_indices()
        self.nb = pb.bnd.bnodes.size
        rows = min(bem_rows, self.nb)
        rng = np.random.default_rng(seed)
        self.bem_sample = rng.standard_normal((rows, self.nb)) if pb.B is None else pb.B[:rows]
        self.threads = os.cpu_count() or 1
        self.iters = None

    def _solve(self, sysm, b_full, x0=None, maxiter=None):
        A_ff, A_fc, free, fixed = sysm
        rhs = b_full[free] - A_fc @ b_full[fixed]
        d = A_ff.diagonal()
        M = sp.diags(1.0 / d)
        it = [0]

        def cb(_):
            it[0] += 1

        x, info = spla.cg(A_ff, rhs, x0=x0, rtol=self.tol, maxiter=maxiter, M=M, callback=cb)
        return x, it[0]

    def _iterations_to_tol(self, sysm, b_full, cap: int) -> int:
        """CG iterations to reach tol: run at most `cap` iterations; if not converged,
        extrapolate geometrically from the residual reduction reached."""
        A_ff, A_fc, free, fixed = sysm
        rhs = b_full[free] - A_fc @ b_full[fixed]
        x, it = self._solve(sysm, b_full, maxiter=cap)
        rel = np.linalg.norm(rhs - A_ff @ x) / np.linalg.norm(rhs)
        if rel <= self.tol or it < cap:
            return it
        return int(np.ceil(cap * np.log(self.tol) / np.log(max(rel, 1e-300))))

    def calibrate(self, m_rows: np.ndarray, cap: int = 400):
        """One cold demag evaluation: Jacobi-PCG iteration counts to tol (capped run,
        geometric extrapolation beyond the cap)."""
        pb = self.pb
        tg = pb.fem.tgrad
        rhs = (tg[0] @ (m_rows[:, 0] * pb.Js) + tg[1] @ (m_rows[:, 1] * pb.Js) + tg[2] @ (m_rows[:, 2] * pb.Js)) / O.MU0
        t = time.perf_counter()
        it1 = self._iterations_to_tol(self.neu, rhs, cap)
        b2 = np.zeros(pb.nx)
        b2[pb.bnd.bnodes] = np.random.default_rng(1).standard_normal(self.nb) * np.abs(rhs).mean()
        it2 = self._iterations_to_tol(self.dir, b2, cap)
        self.iters = (it1, it2)
        return time.perf_counter() - t

    def sample(self, m_rows: np.ndarray, cg_iters_sample: int = 25) -> dict:
        """Seconds per full field evaluation, from bounded component samples."""
        pb = self.pb
        if self.iters is None:
            self.calibrate(m_rows)
        out = {}
        t = time.perf_counter()
        H = O.local_field(pb, m_rows, np.zeros_like(m_rows))
        O.llg_rhs(pb, m_rows, H)
        out["local_s"] = time.perf_counter() - t
        t = time.perf_counter()
        tg, g = pb.fem.tgrad, pb.fem.grad
        rhs = (tg[0] @ (m_rows[:, 0] * pb.Js) + tg[1] @ (m_rows[:, 1] * pb.Js) + tg[2] @ (m_rows[:, 2] * pb.Js)) / O.MU0
        u = rhs
        _ = -np.stack([g[0] @ u, g[1] @ u, g[2] @ u], axis=1)
        out["div_grad_s"] = time.perf_counter() - t
        t = time.perf_counter()
        self._solve(self.neu, rhs, maxiter=cg_iters_sample)
        per_it = (time.perf_counter() - t) / cg_iters_sample
        out["cg_iter_s"] = per_it
        out["solves_s"] = per_it * (self.iters[0] + self.iters[1])
        x = np.random.default_rng(2).standard_normal(self.nb)
        t = time.perf_counter()
        self.bem_sample @ x
        out["bem_s"] = (time.perf_counter() - t) * self.nb / self.bem_sample.shape[0]
        out["total_s"] = out["local_s"] + out["div_grad_s"] + out["solves_s"] + out["bem_s"]
        out["cg_iters"] = list(self.iters)
        return out

    def describe(self) -> str:
        return (f"oracle field evaluation on the full mesh (N={self.pb.nx}, Nb={self.nb}): local field + LLG, "
                f"divergence and gradient timed in full; Neumann/Dirichlet Jacobi-PCG at tol {self.tol} timed "
                f"over 25 iterations and scaled to the iteration counts to tol {self.iters} (a run capped at 400 "
                f"iterations, extrapolated geometrically past the cap); dense BEM GEMV timed on "
                f"{self.bem_sample.shape[0]} of {self.nb} rows and scaled")
