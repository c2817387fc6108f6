"""The allocation-free right-hand side (tmb_llg_rhs_noalloc) against tmb_llg_rhs.

tmb_llg_rhs_noalloc serves callers that cannot allocate device memory while they evaluate
the right-hand side (a host-side integrator under a fixed device-memory budget, a loop that
must not pay cudaMalloc's device-wide synchronisation, code that shares a stream with a
capture): it stages the host vectors through a fixed file-scope device array, whose address
tmb_ctx_create resolves, instead of buffers allocated on first use.  Its results must equal
the regular host-pointer entry point's, call after call (the array keeps the previous call's
contents), and no call of it may change the device's free memory.  This file is collected
last so that a failure here comes after every other test has run.
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


def _material(c, n, seed):
    rng = np.random.default_rng(seed)
    axis = rng.standard_normal((n, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    c.set_material(np.full(n, O.MU0 * 8e5), np.full(n, 1.3e-11 / 1e-18), Ku=np.full(n, 5e4),
                   ku_axis=O.rows_to_soa(axis), D=np.full(n, 3e-3 / 1e-9), alpha=0.3)
    c.set_applied_field(meshgen.field_from_angles(n, 0.04, 30.0, 60.0))
    c.set_demag_frozen(1e4 * rng.standard_normal(3 * n))


@pytest.fixture(scope="module")
def ctx():
    mesh = meshgen.kuhn_cuboid(12, 10, 4, 3.0)
    mo = MeshOps(mesh.xyz, mesh.tets)
    c = Context(0)
    c.set_mesh(mo)
    _material(c, mo.nx, 21)
    return mo, c


def noalloc_rhs(c, y):
    out = np.full_like(y, np.nan)
    code = _lib.lib().tmb_llg_rhs_noalloc(c.h, 0.0, _ptr(y), _ptr(out))
    _lib.check(code)
    return out


def _extra_terms(c, n, on):
    """Cubic and surface anisotropy and the spin-transfer torque (all in the same local launch)."""
    if not on:
        c.set_cubic_anisotropy(None)
        c.set_surface_anisotropy(None)
        c.set_stt(None)
        return
    rng = np.random.default_rng(9)
    q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    c.set_cubic_anisotropy(rng.uniform(2e4, 6e4, n), -1.5e4, q)
    c.set_surface_anisotropy(8e-4 / 1e-9)
    c.set_stt(O.rows_to_soa(rng.standard_normal((n, 3)) * 4e6), beta=0.05, scale=0.7)


@pytest.mark.parametrize("extra", [False, True])
@pytest.mark.parametrize("mixed", [False, True])
def test_noalloc_matches_llg_rhs_twice(ctx, mixed, extra):
    mo, c = ctx
    c.set_precision(mixed)
    _extra_terms(c, mo.nx, extra)
    try:
        for seed in (31, 32):  # two calls in a row, different states
            y = meshgen.random_state(mo.nx, seed)
            ref = c.llg_rhs(0.0, y)
            got = noalloc_rhs(c, y)
            assert np.all(np.isfinite(got))
            assert np.linalg.norm(got - ref) <= TOL * np.linalg.norm(ref)
    finally:
        c.set_precision(False)
        _extra_terms(c, mo.nx, False)


def test_noalloc_leaves_device_memory_unchanged():
    # A fresh context on a mesh near the array's limit (3N doubles = 1.5 MB per vector): the
    # allocation-free calls come before any host-pointer right-hand side of this context, and
    # the device's free memory is the same before and after them.  The regular host-pointer
    # call afterwards allocates its two staging vectors, which shows the measurement sees
    # allocations of this size.
    import torch

    mesh = meshgen.kuhn_cuboid(40, 40, 36, 2.0)  # 41 * 41 * 37 = 62197 nodes
    mo = MeshOps(mesh.xyz, mesh.tets)
    c = Context(0)
    c.set_mesh(mo)
    n = mo.nx
    _material(c, n, 23)
    y0 = meshgen.random_state(n, 41)
    y1 = meshgen.random_state(n, 42)
    # load the local-field kernel with a device-pointer call (no staging buffers involved)
    yd = torch.from_numpy(y0).cuda()
    ref_dev = c.llg_rhs(0.0, yd).cpu().numpy()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    got0 = noalloc_rhs(c, y0)
    got1 = noalloc_rhs(c, y1)
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"tmb_llg_rhs_noalloc changed free device memory by {free0 - free1} bytes"
    ref1 = c.llg_rhs(0.0, y1)                  # host pointers: allocates the context's staging
    free2, _ = torch.cuda.mem_get_info(0)
    assert free2 < free1, "the free-memory probe did not see the regular path's 3 MB of staging"
    assert np.linalg.norm(got0 - ref_dev) <= TOL * np.linalg.norm(ref_dev)
    assert np.linalg.norm(got1 - ref1) <= TOL * np.linalg.norm(ref1)


_FRESH_PROCESS = r"""
import ctypes as C, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import torch
from oracle import tetmag_oracle as O
from tetmag_b200 import _lib, meshgen
from tetmag_b200.api import Context, MeshOps

mesh = meshgen.kuhn_cuboid(24, 20, 8, 3.0)
mo = MeshOps(mesh.xyz, mesh.tets)
c = Context(0)
c.set_mesh(mo)
n = mo.nx
rng = np.random.default_rng(5)
axis = rng.standard_normal((n, 3))
axis /= np.linalg.norm(axis, axis=1, keepdims=True)
c.set_material(np.full(n, O.MU0 * 8e5), np.full(n, 1.3e-11 / 1e-18), Ku=np.full(n, 5e4),
               ku_axis=O.rows_to_soa(axis), D=np.full(n, 3e-3 / 1e-9), alpha=0.3)
c.set_demag_frozen(1e4 * rng.standard_normal(3 * n))
c.set_stt(O.rows_to_soa(rng.standard_normal((n, 3)) * 4e6), beta=0.05, scale=0.7)
c.set_precision(int(sys.argv[2]))
ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
torch.cuda.mem_get_info(0)
torch.cuda.synchronize()
free0, _ = torch.cuda.mem_get_info(0)
outs = []
for seed in (1, 2):
    y = meshgen.random_state(n, seed)
    out = np.full_like(y, np.nan)
    _lib.check(_lib.lib().tmb_llg_rhs_noalloc(c.h, 0.0, ptr(y), ptr(out)))
    outs.append((y, out))
free1, _ = torch.cuda.mem_get_info(0)
err = max(float(np.linalg.norm(o - c.llg_rhs(0.0, y)) / np.linalg.norm(o)) for y, o in outs)
print(free0 - free1, err)
"""


@pytest.mark.parametrize("mixed", [0, 1])
def test_noalloc_first_call_of_a_fresh_process(mixed):
    # In a process whose only earlier work on the device is the context's set-up, the first two
    # calls (local field with uniaxial anisotropy, bulk DMI and the spin-transfer term) leave the
    # device's free memory unchanged: tmb_ctx_create has resolved the array and loaded the
    # kernels the entry point launches.  Their results equal the regular entry point's.
    import subprocess
    import sys
    from pathlib import Path

    root = str(Path(__file__).resolve().parents[1])
    r = subprocess.run([sys.executable, "-c", _FRESH_PROCESS, root, str(mixed)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    delta, err = r.stdout.split()[-2:]
    assert int(delta) == 0, f"the first calls changed free device memory by {delta} bytes"
    assert float(err) <= TOL


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


def test_noalloc_counts_replicas_against_its_array():
    # the limit is on nodes x replicas: 4 replicas of a 20,000-node mesh exceed it
    mesh = meshgen.kuhn_cuboid(30, 30, 20, 2.0)  # 31 * 31 * 21 = 20181 nodes
    mo = MeshOps(mesh.xyz, mesh.tets)
    c = Context(0)
    c.set_mesh(mo)
    c.set_replicas(4)
    n = mo.nx
    c.set_material(np.full(n, O.MU0 * 8e5), np.full(n, 1.3e-11 / 1e-18), alpha=0.5)
    y = np.zeros(3 * n * 4)
    out = np.zeros_like(y)
    code = _lib.lib().tmb_llg_rhs_noalloc(c.h, 0.0, _ptr(y), _ptr(out))
    assert code == _lib.TMB_ERR_ARG
    assert b"replicas" in _lib.lib().tmb_last_error()
