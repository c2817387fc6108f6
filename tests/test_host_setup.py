"""CPU tests of the library's host side: the C ABI exports, argument checks,
and the C++ mesh preprocessing against the oracle (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import tetmag_oracle as O
from tetmag_b200 import _lib, meshgen
from tetmag_b200.api import MeshOps

HEADER = Path(__file__).resolve().parents[1] / "include" / "tmb.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(tmb_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.SIGNATURES) | {"tmb_last_error"}


def test_version_and_error_channel():
    lib = _lib.lib()
    assert lib.tmb_version() >= 10000
    h = C.c_void_p()
    xyz = np.zeros((4, 3))
    tets = np.array([[0, 1, 2, 7]], dtype=np.int32)  # node 7 does not exist
    code = lib.tmb_mesh_create(4, 1, xyz.ctypes.data_as(C.POINTER(C.c_double)),
                               tets.ctypes.data_as(C.POINTER(C.c_int)), C.byref(h))
    assert code == _lib.TMB_ERR_ARG
    assert b"out of range" in lib.tmb_last_error()
    assert lib.tmb_ctx_create(0, None) == _lib.TMB_ERR_ARG


@pytest.mark.parametrize("kind", ["cuboid", "disk"])
def test_cpp_preprocessing_matches_oracle(kind):
    if kind == "cuboid":
        mesh = meshgen.kuhn_cuboid(7, 5, 3, 3.0)
    else:
        mesh = meshgen.jittered_disk(30.0, 6.0, 3.0, seed=5)
    mo = MeshOps(mesh.xyz, mesh.tets)
    ops, bd = mo.operators(), mo.boundary()
    fem = O.fem_prepare(mesh.xyz, mesh.tets)
    bnd = O.extract_boundary(mesh.xyz, mesh.tets)
    n = mesh.nx
    assert mo.nnz == fem.stiff.nnz and mo.nb == bnd.bnodes.size and mo.ntri == bnd.tri.shape[0]

    def csr(v):
        return sp.csr_matrix((v, ops["col"], ops["rowptr"]), shape=(n, n))

    def rel(a, b):
        return abs(a - b).max() / abs(b).max()

    assert rel(csr(ops["stiff"]), fem.stiff) < 1e-13
    for d, k in enumerate("xyz"):
        assert rel(csr(ops["g" + k]), fem.grad[d]) < 1e-13
        assert rel(csr(ops["tg" + k]), fem.tgrad[d]) < 1e-13
    assert np.allclose(ops["node_vol"], fem.node_vol, rtol=1e-14, atol=0)
    assert np.array_equal(bd["bnodes"], bnd.bnodes)
    assert np.allclose(bd["node_area"], bnd.node_area, rtol=1e-13, atol=1e-13)
    assert np.allclose(bd["node_normal"].reshape(3, n).T, bnd.node_normal, atol=1e-13)
    sub = O.solid_angles(mesh.xyz, mesh.tets, bnd)
    assert np.allclose(bd["solid_angle"], sub, atol=1e-12)
    # same triangles (as sets of sorted node triples) with the same outward normals
    tri = bd["tri"].reshape(-1, 3)
    key = {tuple(t): i for i, t in enumerate(bnd.tri)}
    idx = np.array([key[tuple(t)] for t in tri])
    assert np.allclose(bd["tri_normal"].reshape(-1, 3), bnd.tri_normal[idx], atol=1e-13)
    assert np.allclose(bd["tri_area"], bnd.tri_area[idx], rtol=1e-13)


def test_union_and_soa_round_trip():
    a, b = meshgen.kuhn_cuboid(3, 2, 2, 2.0), meshgen.kuhn_cuboid(2, 4, 1, 3.0)
    u, off = meshgen.union([a, b])
    assert list(off) == [0, a.nx, a.nx + b.nx]
    assert u.tets.max() == a.nx + b.nx - 1 and u.tets[len(a.tets):].min() == a.nx
    va, vb = np.arange(3.0 * a.nx), 1000 + np.arange(3.0 * b.nx)
    s = meshgen.soa_stack([va, vb])
    assert np.array_equal(s[:a.nx], va[:a.nx]) and np.array_equal(s[a.nx:a.nx + b.nx], vb[:b.nx])
    ra, rb = meshgen.soa_split(s, off)
    assert np.array_equal(ra, va) and np.array_equal(rb, vb)
    # the preprocessing of the union is the union of the preprocessing
    mu, ma = MeshOps(u.xyz, u.tets), MeshOps(a.xyz, a.tets)
    assert mu.nb == ma.nb + MeshOps(b.xyz, b.tets).nb
    Ku, Ka = mu.operators(), ma.operators()
    assert np.allclose(Ku["stiff"][:Ka["rowptr"][-1]], Ka["stiff"], rtol=0, atol=0)


def test_interleave_roundtrip():
    rng = np.random.default_rng(0)
    vs = [rng.standard_normal(3 * 7) for _ in range(4)]
    v = meshgen.interleave(vs)
    assert v.shape == (3 * 7 * 4,)
    assert v[1 * 7 * 4 + 2 * 4 + 3] == vs[3][1 * 7 + 2]      # y of node 2, replica 3
    for a, b in zip(meshgen.deinterleave(v, 4), vs):
        assert np.array_equal(a, b)
