"""Generates the oracle fixtures of the run-length and full-size parity tests.

* c1_relax_1ns.npz -- the c1 configuration (100 x 100 x 10 nm permalloy cuboid, 5 nm Kuhn cells,
  1,323 nodes, alpha = 1, zero field, seeded random initial state) relaxed for 1 ns by the
  oracle's restatement of TheSimulation::start with frozen demag per 0.5 ps segment
  (main/TheSimulation.cpp:231-311) and the Dormand-Prince stepper at eps 1e-6
  (main/TheLLG.cpp:514-572): final state, mean m, step statistics.
* c4_field.npz -- the c4 cuboid (200 x 200 x 40 nm at 4 nm, 28,611 nodes, 7,002 boundary nodes,
  dense BEM) with replica 0's applied field and a seeded random state: the oracle's demag field
  (direct solves of the reference's row-pinned / row-replaced systems) and LLG right-hand side.

The oracle runs on the CPU in minutes; the GPU tests compare against these files.  Re-run only
when the oracle changes on purpose:

    python tests/golden/make_parity.py [c1] [c4]
"""
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import tetmag_oracle as O  # noqa: E402
from tetmag_b200 import meshgen, workloads  # noqa: E402

HERE = Path(__file__).resolve().parent
C4_STATE_SEED = 404


def problem(w, with_bem=True):
    axis = None if w.ku_axis is None else O.soa_to_rows(w.ku_axis)
    return O.make_problem(w.mesh.xyz, w.mesh.tets, w.mesh.scale, Ms=w.Ms, A=w.A, alpha=w.alpha, Ku=w.Ku,
                          ku_axis=axis if axis is not None else (0, 0, 1), D=w.D, hext=w.hext, with_bem=with_bem)


def make_c1():
    w = workloads.c1()
    pb = problem(w)
    dem = O.DemagOracle(pb)
    t = time.time()
    m, st = O.relax(pb, w.m0, 1000.0, 0.5, demag=dem)
    print(f"c1 relax 1 ns: {time.time() - t:.1f} s, {st}")
    np.savez_compressed(HERE / "c1_relax_1ns.npz", m=O.rows_to_soa(m), mean_m=O.mean_m(pb, m),
                        accepted=st["accepted"], rejected=st["rejected"], rhs=st["rhs"], segments=st["segments"],
                        max_torque=st["max_torque"])


def make_c4():
    w = workloads.c4_replica(replica=0)
    t = time.time()
    pb = problem(w)
    print(f"c4 problem (dense BEM {pb.B.shape}): {time.time() - t:.1f} s")
    t = time.time()
    dem = O.DemagOracle(pb)
    m = O.soa_to_rows(meshgen.random_state(w.n, C4_STATE_SEED))
    hdem = dem.field(m)
    H = O.local_field(pb, m, hdem)
    ydot = O.llg_rhs(pb, m, H)
    print(f"c4 field: {time.time() - t:.1f} s; row-sum error {O.bem_rowsum_error(pb.B):.2e}")
    np.savez_compressed(HERE / "c4_field.npz", state_seed=C4_STATE_SEED, hdem=O.rows_to_soa(hdem),
                        ydot=O.rows_to_soa(ydot), torque=O.max_torque(m, H))


if __name__ == "__main__":
    which = sys.argv[1:] or ["c1", "c4"]
    if "c1" in which:
        make_c1()
    if "c4" in which:
        make_c4()
