"""The allocation-free right-hand side (tmb_llg_rhs_noalloc) against tmb_llg_rhs.

tmb_llg_rhs_noalloc serves callers that cannot allocate device memory while they evaluate
the right-hand side: it stages the host vectors through a fixed file-scope device array
instead of buffers allocated on first use.  Its results must equal the regular host-pointer
entry point's, call after call (the array keeps the previous call's contents).  This file is
collected last so that a failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import tetmag_oracle as O
from tetmag_b200 import _lib, meshgen
from tetmag_b200.api import Context, MeshOps

pytestmark = pytest.mark.gpu

TOL = 1e-12  # same kernel, same inputs: the two paths agree to rounding (in practice bit for bit)


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@pytest.fixture(scope="module")
def ctx():
    mesh = meshgen.kuhn_cuboid(12, 10, 4, 3.0)
    mo = MeshOps(mesh.xyz, mesh.tets)
    c = Context(0)
    c.set_mesh(mo)
    n = mo.nx
    rng = np.random.default_rng(21)
    axis = rng.standard_normal((n, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    c.set_material(np.full(n, O.MU0 * 8e5), np.full(n, 1.3e-11 / 1e-18), Ku=np.full(n, 5e4),
                   ku_axis=O.rows_to_soa(axis), D=np.full(n, 3e-3 / 1e-9), alpha=0.3)
    c.set_applied_field(meshgen.field_from_angles(n, 0.04, 30.0, 60.0))
    c.set_demag_frozen(1e4 * rng.standard_normal(3 * n))
    return mo, c


def noalloc_rhs(c, y):
    out = np.full_like(y, np.nan)
    code = _lib.lib().tmb_llg_rhs_noalloc(c.h, 0.0, _ptr(y), _ptr(out))
    _lib.check(code)
    return out


@pytest.mark.parametrize("mixed", [False, True])
def test_noalloc_matches_llg_rhs_twice(ctx, mixed):
    mo, c = ctx
    c.set_precision(mixed)
    try:
        for seed in (31, 32):  # two calls in a row, different states
            y = meshgen.random_state(mo.nx, seed)
            ref = c.llg_rhs(0.0, y)
            got = noalloc_rhs(c, y)
            assert np.all(np.isfinite(got))
            assert np.linalg.norm(got - ref) <= TOL * np.linalg.norm(ref)
    finally:
        c.set_precision(False)


def test_noalloc_rejects_meshes_beyond_its_array():
    mesh = meshgen.kuhn_cuboid(40, 40, 41, 2.0)  # 41 * 41 * 42 = 70602 nodes > 65536
    mo = MeshOps(mesh.xyz, mesh.tets)
    c = Context(0)
    c.set_mesh(mo)
    n = mo.nx
    c.set_material(np.full(n, O.MU0 * 8e5), np.full(n, 1.3e-11 / 1e-18), alpha=0.5)
    y = meshgen.random_state(n, 1)
    out = np.zeros_like(y)
    code = _lib.lib().tmb_llg_rhs_noalloc(c.h, 0.0, _ptr(y), _ptr(out))
    assert code == _lib.TMB_ERR_ARG
    assert b"65536" in _lib.lib().tmb_last_error()
