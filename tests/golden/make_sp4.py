"""Generates tests/golden/sp4_mesh.npz and tests/golden/sp4_log_rows.npz from the reference.

The reference ships one trajectory of its own: the muMAG standard problem 4 example
(examples/example2: mesh sp4_.vtk, 16,602 nodes and 48,569 tetrahedra of a 500 x 125 x 3 nm
Permalloy platelet), with five rows of the .log file it wrote, t = 132 .. 140 ps, quoted in
doc/examples/example2.rst:113-120.  This script reads both files from the reference tree:

* the legacy VTK mesh (POINTS as 32-bit floats, as tetmag's VTK reader gets them; cells from
  OFFSETS / CONNECTIVITY), stored as float64 coordinates (exact copies of the float32 values)
  and int32 tetrahedra;
* the log rows, column by column as TheSimulation::writeLogStream writes them
  (main/TheSimulation.cpp:367-372): time [ps], total, demag, exchange, uniaxial, Zeeman, cubic,
  surface and DMI energy densities [J/m^3], max torque [T], mean m (3), mean applied field [T] (3).

Run once where the reference tree is mounted (it is not available when the tests run):

    python tests/golden/make_sp4.py [path/to/tetmag]
"""
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def read_legacy_vtk_tets(path: Path):
    toks = path.read_text().split()
    i = toks.index("POINTS")
    npts, dtype = int(toks[i + 1]), toks[i + 2]
    if dtype != "float":
        raise ValueError(f"expected float points, got {dtype}")
    xyz = np.array(toks[i + 3:i + 3 + 3 * npts], dtype=np.float32).astype(np.float64).reshape(npts, 3)
    i = toks.index("CELLS")
    noff = int(toks[i + 1])
    j = toks.index("OFFSETS")
    off = np.array(toks[j + 2:j + 2 + noff], dtype=np.int64)
    k = toks.index("CONNECTIVITY")
    conn = np.array(toks[k + 2:k + 2 + int(off[-1])], dtype=np.int64)
    t = toks.index("CELL_TYPES")
    ntypes = int(toks[t + 1])
    types = np.array(toks[t + 2:t + 2 + ntypes], dtype=np.int64)
    if ntypes != noff - 1 or np.any(types != 10) or np.any(np.diff(off) != 4):
        raise ValueError("expected tetrahedra only (VTK cell type 10)")
    return xyz, conn.reshape(-1, 4).astype(np.int32)


def read_log_rows(rst: Path):
    rows = []
    for line in rst.read_text().splitlines():
        f = line.split()
        if len(f) == 16 and re.fullmatch(r"\d+\.\d{4}", f[0]):
            rows.append([float(v) for v in f])
    if not rows:
        raise ValueError("no log rows found")
    return np.array(rows)


def main():
    ref = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")
    xyz, tets = read_legacy_vtk_tets(ref / "examples" / "example2" / "sp4_.vtk")
    rows = read_log_rows(ref / "doc" / "examples" / "example2.rst")
    np.savez_compressed(HERE / "sp4_mesh.npz", xyz=xyz, tets=tets)
    np.savez_compressed(HERE / "sp4_log_rows.npz", rows=rows,
                        columns=np.array(["t_ps", "E_total", "E_demag", "E_exchange", "E_uniaxial", "E_zeeman",
                                          "E_cubic", "E_surface", "E_dmi", "max_torque_T", "mx", "my", "mz",
                                          "Bx_T", "By_T", "Bz_T"]))
    print(f"mesh: {xyz.shape[0]} nodes, {tets.shape[0]} tets; {rows.shape[0]} log rows "
          f"(t = {rows[0, 0]:g} .. {rows[-1, 0]:g} ps)")


if __name__ == "__main__":
    main()
