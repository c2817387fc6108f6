"""Run artefacts: .vtu writer, magnetisation reader (VTKReader::readMag), .log columns.

CPU tests call the host-only C-ABI entry points (no device work); the .log row of a live
context is checked on the GPU against the oracle's energies.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import output_oracle as OO
from tetmag_b200 import _lib, api, meshgen


@pytest.fixture(scope="module")
def small():
    mesh = meshgen.kuhn_cuboid(4, 3, 2, 2.5)
    return mesh, meshgen.random_state(mesh.nx, 3)


@pytest.mark.parametrize("binary", [False, True])
def test_vtu_roundtrip(tmp_path, small, binary):
    # MeshWriter::outputVTK layout, read back by the VTKReader restatement: exact in both encodings
    mesh, m = small
    p = tmp_path / "m.vtu"
    api.write_vtu(p, mesh.xyz, mesh.tets, m, material=np.arange(mesh.nx) % 3, time_ps=123.25, field=-m,
                  field_name="Demag", binary=binary)
    m2, t = api.read_magnetization(p, mesh.nx)
    assert np.array_equal(m2, m) and t == 123.25
    text = p.read_bytes()
    for tag in (b'Name="Magnetization"', b'Name="Material"', b'Name="Demag"', b'Name="timeInPs"',
                b'Name="connectivity"', b'Name="offsets"', b'Name="types"'):
        assert tag in text
    if not binary:
        assert f'NumberOfPoints="{mesh.nx}" NumberOfCells="{mesh.tets.shape[0]}"'.encode() in text


@pytest.mark.parametrize("mode", ["ascii", "binary", "appended-base64", "appended-raw"])
@pytest.mark.parametrize("header", ["UInt32", "UInt64"])
@pytest.mark.parametrize("compress", [False, True])
def test_read_vtk_xml_encodings(tmp_path, small, mode, header, compress):
    # the encodings VTK's XML writer produces (tetmag writes through vtkXMLUnstructuredGridWriter)
    if mode == "ascii" and (compress or header == "UInt32"):
        pytest.skip("ASCII arrays have no header or compression")
    mesh, m = small
    p = tmp_path / "v.vtu"
    # a block size that splits the magnetisation array into several zlib blocks
    p.write_bytes(OO.vtk_xml(mesh.xyz, mesh.tets, m, time_ps=4.5, mode=mode, header=header, compress=compress,
                             block=200))
    m2, t = api.read_magnetization(p, mesh.nx)
    assert np.array_equal(m2, m) and t == 4.5


def test_read_vtk_xml_float32_and_joint_base64(tmp_path, small):
    mesh, m = small
    p = tmp_path / "f.vtu"
    p.write_bytes(OO.vtk_xml(mesh.xyz, mesh.tets, m, time_ps=None, mode="binary", compress=False, dtype="Float32",
                             joint_base64=True))
    m2, t = api.read_magnetization(p, mesh.nx)
    assert np.array_equal(m2, m.astype(np.float32).astype(np.float64)) and t == 0.0


@pytest.mark.parametrize("layout", ["v4", "v5"])
def test_read_legacy_vtk(tmp_path, small, layout):
    mesh, m = small
    p = tmp_path / "l.vtk"
    p.write_text(OO.vtk_legacy(mesh.xyz, mesh.tets, m, time_ps=7.0, layout=layout))
    m2, t = api.read_magnetization(p, mesh.nx)
    assert np.array_equal(m2, m) and t == 7.0


def test_reader_errors(tmp_path, small):
    # VTKReader's checks: point count (checkNodeNumber), missing magnetisation, unknown extension
    mesh, m = small
    p = tmp_path / "m.vtu"
    api.write_vtu(p, mesh.xyz, mesh.tets, m)
    with pytest.raises(_lib.TmbError, match="inconsistent number of points"):
        api.read_magnetization(p, mesh.nx + 1)
    q = tmp_path / "nom.vtu"
    q.write_bytes(p.read_bytes().replace(b'Name="Magnetization"', b'Name="Other"'))
    with pytest.raises(_lib.TmbError, match="no data on the magnetization"):
        api.read_magnetization(q, mesh.nx)
    r = tmp_path / "m.gmv"
    r.write_text("gmvinput ascii\n")
    with pytest.raises(_lib.TmbError, match="not supported"):
        api.read_magnetization(r, mesh.nx)
    with pytest.raises(_lib.TmbError, match="not found"):
        api.read_magnetization(tmp_path / "absent.vtu", mesh.nx)


def test_log_header_text():
    start = "Thu Dec  3 10:00:00 2026\n"
    assert api.log_header(start, "node7", "alice") == OO.log_header(start, "node7", "alice")


def test_log_row_format_matches_restatement():
    # writeLogStream's column formats, on values that exercise signs, widths and exponents
    rng = np.random.default_rng(0)
    cases = [(0.0, np.zeros(8), 0.0, [0.0, 0.0, 1.0], [0.0, 0.0, 0.0]),
             (1500.0, [-3.2e3, 1.1e5, 2.2e4, 0.0, -1.0e-3, 0.0, 0.0, 12.5], 4.5e-7, [-0.5, 1e-5, 0.8660254037844],
              [0.02, -0.0, 1e-9])]
    for _ in range(40):
        cases.append((rng.uniform(0, 5000), rng.standard_normal(8) * 10.0 ** rng.integers(-3, 7, 8),
                      10.0 ** rng.uniform(-8, 3), rng.uniform(-1, 1, 3) * 10.0 ** rng.integers(-12, 1, 3),
                      rng.standard_normal(3) * 10.0 ** rng.integers(-4, 1, 3)))
    for t, e, tq, mm, hh in cases:
        assert api.log_format(t, e, tq, mm, hh) == OO.log_row(t, e, tq, mm, hh)


@pytest.mark.gpu
def test_log_row_of_a_context_matches_oracle():
    # tmb_log_row on a live context: energies, torque, mean m and mean applied field against the
    # oracle, parsed back from the columns
    from oracle import tetmag_oracle as O
    g = np.load(Path(__file__).with_name("golden") / "oracle_small.npz")
    mo = api.MeshOps(g["xyz"], g["tets"])
    ctx = api.Context(0)
    ctx.set_mesh(mo)
    ctx.bem_assemble(mo)
    n = mo.nx
    ctx.set_material(np.full(n, O.MU0 * 8e5), np.full(n, 1.3e-11 / 1e-18), Ku=np.full(n, 5e4),
                     ku_axis=O.rows_to_soa(g["axis"]), D=np.full(n, 3e-3 / 1e-9), alpha=0.3)
    ctx.set_applied_field(np.ascontiguousarray(g["hext"]))
    ctx.set_solver_params(1e-13, 300)
    m = O.rows_to_soa(g["m"])
    row = ctx.log_row(m, 250.0)
    cols = row.rstrip("\n").split("\t")
    assert len(cols) == 12 and cols[0] == "250.0000"
    pb = O.make_problem(g["xyz"], g["tets"], 1e-9, Ms=8e5, A=1.3e-11, alpha=0.3, Ku=5e4, ku_axis=g["axis"],
                        D=3e-3, hext=np.ascontiguousarray(g["hext"]), with_bem=False)
    eo = O.energies(pb, g["m"], g["hdem"])
    scale = max(abs(v) for v in eo.values())
    for k, c in zip(OO.ENERGY_KEYS, cols[1:9]):
        assert abs(float(c) - eo[k]) <= 1e-9 * scale + 1e-4
    assert abs(float(cols[9]) - float(g["torque"])) <= 1e-3 * float(g["torque"])
    V = pb.fem.node_vol
    mm = V @ g["m"] / V.sum()
    assert np.allclose([float(x) for x in cols[10].split()], mm, atol=1e-9)
    hm = V @ pb.hext / V.sum() * O.MU0
    assert np.allclose([float(x) for x in cols[11].split()], hm, atol=1e-6)
