"""Generates tests/golden/stt_mesh.npz and tests/golden/stt_reference.npz from the reference.

The reference's example 3 is the spin-transfer-torque standard problem (examples/example3: mesh
sp_stt.vtk, a 100 x 100 x 10 nm Permalloy square, A = 1.3e-11 J/m, Ms = 8e5 A/m): a vortex
relaxed with simulation.cfg_static, then 14 ns of Zhang-Li dynamics under a dc current along x
(1e12 A/m^2, P = 1, beta = 0.05, alpha = 0.1; simulation.cfg_dynamic).  Its documentation quotes
the mean magnetisation of the equilibrium reached after 14 ns (doc/examples/example3.rst:68):
<M_x> = -1.7009e5 A/m and <M_y> = 1.566e4 A/m.  This script reads the mesh (as make_sp4.py does)
and those two values, with the run parameters from the two configuration files.

Run once where the reference tree is mounted (it is not available when the tests run):

    python tests/golden/make_stt.py [path/to/tetmag]
"""
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_sp4 import read_legacy_vtk_tets  # noqa: E402


def read_cfg(path: Path) -> dict:
    out = {}
    for line in path.read_text().splitlines():
        line = line.split("#", 1)[0].strip()
        if "=" in line:
            k, v = (s.strip() for s in line.split("=", 1))
            out[k] = v
    return out


def read_mean_m(rst: Path):
    text = rst.read_text()
    mx = re.search(r"langle M_x\\rangle = (-?[\d.]+)\\times 10\^(\d+)", text)
    my = re.search(r"langle M_y\\rangle = (-?[\d.]+)\s*\\times 10\^(\d+)", text)
    if not (mx and my):
        raise ValueError("mean magnetisation not found")
    return float(mx.group(1)) * 10.0 ** int(mx.group(2)), float(my.group(1)) * 10.0 ** int(my.group(2))


def main():
    ref = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")
    ex = ref / "examples" / "example3"
    xyz, tets = read_legacy_vtk_tets(ex / "sp_stt.vtk")
    static, dyn = read_cfg(ex / "simulation.cfg_static"), read_cfg(ex / "simulation.cfg_dynamic")
    mat = read_cfg(ex / "material001.dat")
    mx, my = read_mean_m(ref / "doc" / "examples" / "example3.rst")
    np.savez_compressed(HERE / "stt_mesh.npz", xyz=xyz, tets=tets)
    np.savez_compressed(
        HERE / "stt_reference.npz",
        mean_Mx=mx, mean_My=my, A=float(mat["A"]), Ms=float(mat["Ms"]),
        static_alpha=float(static["alpha"]), static_segment_ps=float(static["time step"]),
        static_duration_ps=float(static["duration"]), torque_limit=float(static["torque limit"]),
        alpha=float(dyn["alpha"]), segment_ps=float(dyn["time step"]), duration_ps=float(dyn["duration"]),
        polarization=float(dyn["spin polarization"]), current_density=float(dyn["current density"]),
        beta=float(dyn["beta"]), current_theta=float(dyn["current theta"]), current_phi=float(dyn["current phi"]))
    print(f"mesh: {xyz.shape[0]} nodes, {tets.shape[0]} tets; <M> = ({mx:g}, {my:g}) A/m after "
          f"{dyn['duration']} ps")


if __name__ == "__main__":
    main()
