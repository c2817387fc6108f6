"""Generates tests/golden/oracle_small.npz from the FP64 oracle.

The reference binary cannot be built here (Eigen, Boost, SUNDIALS, AMGCL and
H2Lib are absent), so these vectors pin the oracle restatement against drift;
the oracle itself is pinned by the reference's own known-answer checks
(tests/test_oracle.py).  Re-run only when the oracle changes on purpose:

    python tests/golden/make_golden.py
"""
from pathlib import Path
import sys

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import tetmag_oracle as O  # noqa: E402
from tetmag_b200 import meshgen  # noqa: E402


def main():
    mesh = meshgen.kuhn_cuboid(6, 5, 4, 3.0)
    n = mesh.nx
    rng = np.random.default_rng(7)
    axis = rng.standard_normal((n, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    hext = meshgen.field_from_angles(n, 0.03, 60.0, 20.0)
    pb = O.make_problem(mesh.xyz, mesh.tets, 1e-9, Ms=8e5, A=1.3e-11, alpha=0.3, Ku=5e4, ku_axis=axis,
                        D=3e-3, hext=hext)
    m = O.soa_to_rows(meshgen.random_state(n, 11))
    dem = O.DemagOracle(pb)
    hdem = dem.field(m)
    H = O.local_field(pb, m, hdem)
    ydot = O.llg_rhs(pb, m, H)
    out = Path(__file__).with_name("oracle_small.npz")
    np.savez_compressed(out, xyz=mesh.xyz, tets=mesh.tets, axis=axis, hext=hext, m=m, B=pb.B, hdem=hdem, H=H,
                        ydot=ydot, torque=O.max_torque(m, H))
    print("wrote", out, "N =", n, "Nb =", pb.bnd.bnodes.size)


if __name__ == "__main__":
    main()
