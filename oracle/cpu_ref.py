"""ctypes wrapper and build recipe of the C++ CPU restatement (oracle/cpu_field.cpp).

TEST / BENCH INFRASTRUCTURE ONLY: the reference arm and cpu_baseline leg of bench.py and the
tests use it; the library never loads it.  It times one full field evaluation of the
reference's CPU path on the host cores: GMRES(30) + smoothed-aggregation AMG with ILU(0)
relaxation for both solves (tetmag's AMGCL configuration), the dense or hierarchical boundary
matrix, and the field / LLG kernels, all FP64 with OpenMP.

    python -m oracle.cpu_ref          # builds oracle/_build/liborc_cpu.so
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "cpu_field.cpp"
OUT = HERE / "_build"
LIB = OUT / "liborc_cpu.so"

_lib = None


def build(force: bool = False) -> Path:
    """g++ -O3 -fopenmp; rebuilt when the source is newer than the library."""
    OUT.mkdir(exist_ok=True)
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    cxx = shutil.which("g++") or os.environ.get("CXX") or "g++"
    cmd = [cxx, "-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", str(SRC), "-o", str(LIB)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building the CPU oracle failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        P, D, I = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.c_int, I, I, D, D, D, D, D, D, D, D, C.c_int, I, D, D, D, D, D, C.c_double,
                                 C.c_double, C.c_int]
        L.orc_destroy.argtypes = [P]
        L.orc_destroy.restype = None
        L.orc_set_bem_dense.argtypes = [P, D]
        L.orc_build_hmatrix.argtypes = [P, D, C.c_int, I, D, D, D, D, C.c_int, C.c_double, C.c_double, C.c_int, D]
        L.orc_bem_matvec.argtypes = [P, D, D]
        L.orc_field_eval.argtypes = [P, D, D, D]
        L.orc_info.argtypes = [P, D]
        L.orc_reset_timers.argtypes = [P]
        L.orc_reset_timers.restype = None
        L.orc_last_error.restype = C.c_char_p
        L.orc_threads.restype = C.c_int
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_threads.restype = None
        _lib = L
    return _lib


def _d(a):
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    return np.ascontiguousarray(a, np.int32).ctypes.data_as(C.POINTER(C.c_int))


class CpuField:
    """One problem on the host cores: operators of the oracle's preprocessing (tetmag's FEM
    restated), material per node, the reference's row-pinned / row-replaced systems."""

    def __init__(self, pb, tol: float = 1e-7, maxiter: int = 100, threads: int | None = None):
        L = lib()
        if threads:
            L.orc_set_threads(int(threads))
        self.threads = int(L.orc_threads())
        f = pb.fem
        n = pb.nx
        self.n, self.nb = n, int(pb.bnd.bnodes.size)
        self._keep = [f.stiff.indptr.astype(np.int32), f.stiff.indices.astype(np.int32)]
        axis = np.ascontiguousarray(pb.ku_axis.T.ravel())
        hext = np.ascontiguousarray(pb.hext.T.ravel())
        A = np.ascontiguousarray(pb.A)
        self.h = L.orc_create(n, _i(self._keep[0]), _i(self._keep[1]), _d(f.stiff.data), _d(f.grad[0].data),
                              _d(f.grad[1].data), _d(f.grad[2].data), _d(f.tgrad[0].data), _d(f.tgrad[1].data),
                              _d(f.tgrad[2].data), _d(f.node_vol), self.nb, _i(pb.bnd.bnodes), _d(pb.Js), _d(A),
                              _d(pb.Ku), _d(axis), _d(hext), float(pb.alpha), float(tol), int(maxiter))
        if not self.h:
            raise RuntimeError(L.orc_last_error().decode())
        self.pb = pb
        self.bem = None

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_destroy(h)
            self.h = None

    def set_bem_dense(self, B):
        lib().orc_set_bem_dense(self.h, _d(np.ascontiguousarray(B, np.float64)))
        self.bem = "dense"

    def build_hmatrix(self, solid_angle, leaf=32, eta=2.0, eps=1e-6, kmax=64) -> dict:
        pb = self.pb
        bnd = pb.bnd
        bx = np.ascontiguousarray(pb.xyz[bnd.bnodes], np.float64)
        tri_b = np.ascontiguousarray(bnd.bindex[bnd.tri], np.int32)
        nn = np.ascontiguousarray(bnd.node_normal[bnd.bnodes], np.float64)
        out = (C.c_double * 4)()
        rc = lib().orc_build_hmatrix(self.h, _d(bx), int(tri_b.shape[0]), _i(tri_b), _d(bnd.tri_area),
                                     _d(np.ascontiguousarray(bnd.tri_normal)), _d(nn), _d(solid_angle), int(leaf),
                                     float(eta), float(eps), int(kmax), out)
        if rc != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        self.bem = "hierarchical"
        return dict(dense_tiles=out[0], lowrank_blocks=out[1], bytes=out[2], build_s=out[3])

    def bem_matvec(self, x):
        y = np.empty(self.nb)
        lib().orc_bem_matvec(self.h, _d(x), y.ctypes.data_as(C.POINTER(C.c_double)))
        return y

    def field_eval(self, m_soa, hdem=None):
        y = np.empty(3 * self.n)
        m = np.ascontiguousarray(m_soa, np.float64)
        hp = hdem.ctypes.data_as(C.POINTER(C.c_double)) if hdem is not None else None
        rc = lib().orc_field_eval(self.h, _d(m), y.ctypes.data_as(C.POINTER(C.c_double)), hp)
        if rc != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return y

    def info(self) -> dict:
        out = (C.c_double * 12)()
        lib().orc_info(self.h, out)
        lv = int(out[10])
        return dict(evals=int(out[0]), div_s=out[1], neumann_s=out[2], bem_s=out[3], dirichlet_s=out[4],
                    local_s=out[5], it_neumann=int(out[6]), it_dirichlet=int(out[7]), relres_neumann=out[8],
                    relres_dirichlet=out[9], amg_levels=(lv % 1000, lv // 1000), amg_setup_s=out[11])

    def reset_timers(self):
        lib().orc_reset_timers(self.h)


if __name__ == "__main__":
    print(build(force=True))
