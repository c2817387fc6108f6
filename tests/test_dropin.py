"""The drop-in boundary as tetmag would call it.

* tmb_set_operators / tmb_set_bem_dense take tetmag's MeshData arrays (specs/MeshData.h:41-63:
  K, grad*, tGrad* on one CSR pattern, node volumes, boundary nodes, areas, normals, and the
  column-major dense BEM matrix; consumed at main/DemagField.cpp:65-71).  Fed the library's own
  preprocessing output they give bit-equal results to tmb_set_mesh; fed the oracle's restatement
  of tetmag's preprocessing they give the oracle's field.
* The "remove precession" dynamics (TheLLG::noPrecession, main/TheLLG.cpp:180-199).
* A C++ translation unit that includes include/tmb.h and implements INTEGRATION.md's
  B200Solver and CVODE right-hand-side adapters against stand-in base classes, linked to
  libtmb.so: compiled here (CPU), run on the GPU.
"""
import os
import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle import tetmag_oracle as O
from tetmag_b200 import meshgen, workloads
from tetmag_b200.api import Context, MeshOps

ROOT = Path(__file__).resolve().parents[1]
SHIM = Path(__file__).with_name("shim") / "tetmag_shims.cpp"
LIBDIR = ROOT / "tetmag_b200"
FP64_TOL = 1e-10
MIXED_TOL = 1e-5


def rel(a, b):
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _cuda_home():
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and Path(c, "include", "cuda_runtime.h").exists():
            return Path(c)
    return None


def build_shim(outdir: Path) -> Path:
    """g++ on the shim translation unit, linked to the in-tree libtmb.so and the CUDA runtime."""
    cxx = shutil.which("g++")
    cuda = _cuda_home()
    if cxx is None or cuda is None:
        pytest.skip("g++ or the CUDA headers are not available")
    if not (LIBDIR / "libtmb.so").exists():
        pytest.fail("libtmb.so is not built (python -m tetmag_b200.build)")
    exe = outdir / "tetmag_shims"
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}",
           f"-I{cuda / 'include'}", str(SHIM), "-o", str(exe), f"-L{LIBDIR}", "-ltmb", f"-Wl,-rpath,{LIBDIR}",
           f"-L{cuda / 'lib64'}", "-lcudart", f"-Wl,-rpath,{cuda / 'lib64'}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, f"shim build failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return exe


def test_shim_translation_unit_builds_against_the_header(tmp_path):
    exe = build_shim(tmp_path)
    assert exe.exists()


@pytest.fixture(scope="module")
def small():
    mesh = meshgen.kuhn_cuboid(8, 6, 3, 4.0)
    n = mesh.nx
    m = meshgen.random_state(n, 77)
    pb = O.make_problem(mesh.xyz, mesh.tets, 1e-9, Ms=8e5, A=1.3e-11, alpha=0.5)
    return mesh, m, pb, O.DemagOracle(pb)


def _material(ctx, n, alpha):
    ctx.set_material(np.full(n, O.MU0 * 8e5), np.full(n, 1.3e-11 / 1e-18), alpha=alpha)


@pytest.mark.gpu
def test_set_operators_and_bem_dense_bit_equal_to_set_mesh(small):
    # MeshData arrays of the library's own preprocessing through tmb_set_operators, the device-
    # assembled matrix copied out and handed back through tmb_set_bem_dense (column-major, as
    # Eigen's MatrixXd): the same operators and matrix, so the same bits
    mesh, m, pb, dem = small
    mo = MeshOps(mesh.xyz, mesh.tets)
    n = mo.nx
    a = Context(0)
    a.set_mesh(mo)
    a.bem_assemble(mo)
    ops, bd = mo.operators(), mo.boundary()
    b = Context(0)
    b.set_operators(ops["rowptr"], ops["col"], ops["stiff"], [ops["gx"], ops["gy"], ops["gz"]],
                    [ops["tgx"], ops["tgy"], ops["tgz"]], ops["node_vol"], bd["bnodes"], bd["node_area"],
                    bd["node_normal"])
    b.set_bem_dense(a.get_bem_dense())
    for c in (a, b):
        _material(c, n, 0.5)
        c.set_solver_params(1e-12, 300)
    for mixed in (False, True):
        ha, hb = np.empty(3 * n), np.empty(3 * n)
        for c in (a, b):
            c.set_precision(mixed)
        ya = a.field_eval(m, hdem=ha)
        yb = b.field_eval(m, hdem=hb)
        assert np.array_equal(ha, hb) and np.array_equal(ya, yb)


@pytest.mark.gpu
def test_set_operators_from_oracle_meshdata(small):
    # tetmag's MeshData restated by the oracle (FEMprocessing / Boundary / BEMprocessing): K and
    # the six gradient operators share one pattern, B is the oracle's dense Lindholm matrix
    mesh, m, pb, dem = small
    f, bnd = pb.fem, pb.bnd
    for op in f.grad + f.tgrad:
        assert np.array_equal(op.indptr, f.stiff.indptr) and np.array_equal(op.indices, f.stiff.indices)
    n = pb.nx
    ctx = Context(0)
    ctx.set_operators(f.stiff.indptr, f.stiff.indices, f.stiff.data, [g.data for g in f.grad],
                      [t.data for t in f.tgrad], f.node_vol, bnd.bnodes, bnd.node_area,
                      O.rows_to_soa(bnd.node_normal))
    ctx.set_bem_dense(pb.B)
    _material(ctx, n, 0.5)
    ctx.set_solver_params(1e-13, 300)
    mr = O.soa_to_rows(m)
    Hd = dem.field(mr)
    ref = O.rows_to_soa(O.llg_rhs(pb, mr, O.local_field(pb, mr, Hd)))
    h = np.empty(3 * n)
    y = ctx.field_eval(m, hdem=h)
    assert rel(h, O.rows_to_soa(Hd)) <= FP64_TOL
    assert rel(y, ref) <= FP64_TOL
    ctx.set_precision(True)
    ctx.set_solver_params(1e-8, 300)
    y = ctx.field_eval(m, hdem=h)
    assert rel(h, O.rows_to_soa(Hd)) <= MIXED_TOL
    assert rel(y, ref) <= MIXED_TOL


@pytest.mark.gpu
def test_no_precession_matches_oracle(small):
    # TheLLG::noPrecession: -alpha m x (m x H), the precession term removed; also through a short
    # frozen-demag relaxation against the oracle's loop with the same dynamics
    mesh, m, pb, dem = small
    mo = MeshOps(mesh.xyz, mesh.tets)
    n = mo.nx
    ctx = Context(0)
    ctx.set_mesh(mo)
    ctx.bem_assemble(mo)
    _material(ctx, n, 0.5)
    ctx.set_solver_params(1e-13, 300)
    mr = O.soa_to_rows(m)
    Hd = dem.field(mr)
    ctx.set_demag_frozen(O.rows_to_soa(Hd))
    H = O.local_field(pb, mr, Hd)
    with_prec = ctx.llg_rhs(0.0, m)
    ctx.set_llg_options(precession=False)
    try:
        got = ctx.llg_rhs(0.0, m)
        ref = O.rows_to_soa(O.llg_rhs(pb, mr, H, precession=False))
        assert rel(got, ref) <= 1e-12
        assert rel(with_prec, ref) > 1e-2            # the precession term matters here
        # the remaining term is the damping one: orthogonal to m and to m x H
        g = O.soa_to_rows(got)
        assert np.max(np.abs(np.sum(g * mr, axis=1))) <= 1e-9 * np.max(np.abs(g))
        assert np.max(np.abs(np.sum(g * np.cross(mr, H), axis=1))) <= 1e-9 * np.max(np.abs(g) * np.abs(H))
        mg = m.copy()
        st = ctx.relax(mg, duration_ps=5.0, segment_ps=0.5)
        mo_, so = O.relax(pb, m, 5.0, 0.5, demag=dem, precession=False)
        assert st["segments"] == so["segments"] == 10
        assert np.max(np.abs(O.mean_m(pb, O.soa_to_rows(mg)) - O.mean_m(pb, mo_))) <= 1e-4
    finally:
        ctx.set_llg_options(precession=True)


@pytest.mark.gpu
def test_cpp_shims_through_the_header(tmp_path, small):
    # the compiled B200Solver / DemagField / CVODE rhs and rhs_d adapters, run on the GPU, against
    # the oracle (demag field, right-hand side) and a direct solve (the Neumann system)
    mesh, m, pb, dem = small
    exe = build_shim(tmp_path)
    n = pb.nx
    rng = np.random.default_rng(4)
    bload = rng.standard_normal(n)
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([n, mesh.tets.shape[0]], np.int32).tofile(f)
        np.ascontiguousarray(mesh.xyz, np.float64).tofile(f)
        np.ascontiguousarray(mesh.tets, np.int32).tofile(f)
        np.ascontiguousarray(m, np.float64).tofile(f)
        bload.tofile(f)
    r = subprocess.run([str(exe), str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, f"shim program failed ({r.returncode}):\n{r.stdout}\n{r.stderr}"
    assert "b200 PCG+AMG" in r.stdout
    d = np.fromfile(out, np.float64)
    H, yh, yd, x, info = np.split(d, np.cumsum([3 * n, 3 * n, 3 * n, n]))
    mr = O.soa_to_rows(m)
    Hd = dem.field(mr)
    assert rel(H, O.rows_to_soa(Hd)) <= FP64_TOL
    # the right-hand side uses the demag field frozen by the calcField call above
    ref = O.rows_to_soa(O.llg_rhs(pb, mr, O.local_field(pb, mr, Hd)))
    assert rel(yh, ref) <= FP64_TOL
    assert np.array_equal(yh, yd)
    xr = spla.splu(dem.neumann.tocsc()).solve(bload)
    assert rel(x, xr) <= FP64_TOL
    assert info[2] == 0 and info[0] >= 1
