"""Generates the oracle fixtures of the run-length and full-size parity tests.

* c1_relax_1ns.npz -- the c1 configuration (100 x 100 x 10 nm permalloy cuboid, 5 nm Kuhn cells,
  1,323 nodes, alpha = 1, zero field, seeded random initial state) relaxed for 1 ns by the
  oracle's restatement of TheSimulation::start with frozen demag per 0.5 ps segment
  (main/TheSimulation.cpp:231-311) and the Dormand-Prince stepper at eps 1e-6
  (main/TheLLG.cpp:514-572): final state, mean m, step statistics.
* c4_field.npz -- the c4 cuboid (200 x 200 x 40 nm at 4 nm, 28,611 nodes, 7,002 boundary nodes,
  dense BEM) with replica 0's applied field and a seeded random state: the oracle's demag field
  (direct solves of the reference's row-pinned / row-replaced systems) and LLG right-hand side.
* c3_dots_run.npz -- three dots of the c3 batch (256 seeded nanodots; dots 36, 120 and 189 with
  513, 1,496 and 4,032 nodes), each run alone for the configuration's 0.5 ns by the same loop in
  five calls of 100 ps, with the Dormand-Prince tolerances at 1e-8: mean m after each call.  At
  alpha = 0.1 the dots precess for the whole run, and at the reference's 1e-6 the integrator alone
  moves dot 189's mean m by 1.6e-4 at 100 ps and 8.6e-4 at 200 ps (against 1e-8), more than the
  1e-4 that the comparison asks of the field evaluation.
* c4_relax_1ns.npz -- replica 0 of c4 (its seeded initial state and applied field, alpha = 0.5)
  run for the configuration's 1 ns by the same relaxation loop as c1 (frozen demag per 0.5 ps
  segment), in ten calls of 100 ps: mean m, accepted steps and torque after each call, final state.

The oracle runs on the CPU in minutes; the GPU tests compare against these files.  Re-run only
when the oracle changes on purpose:

    python tests/golden/make_parity.py [c1] [c4] [c4run] [c3run]
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


def make_c4_run():
    w = workloads.c4_replica(replica=0)
    t = time.time()
    pb = problem(w)
    dem = O.DemagOracle(pb)
    print(f"c4 problem: {time.time() - t:.1f} s", flush=True)
    m = w.m0.copy()
    means, acc, torque = [], [], []
    for k in range(10):
        t = time.time()
        mr, st = O.relax(pb, m, 100.0, 0.5, demag=dem)
        m = O.rows_to_soa(mr)
        means.append(O.mean_m(pb, mr))
        acc.append(st["accepted"])
        torque.append(st["max_torque"])
        print(f"c4 run {100 * (k + 1)} ps: {time.time() - t:.1f} s, mean m {means[-1]}, {st}", flush=True)
    np.savez_compressed(HERE / "c4_relax_1ns.npz", m=m, mean_m=np.array(means), accepted=np.array(acc),
                        max_torque=np.array(torque), chunk_ps=100.0, segment_ps=0.5)


C3_DOTS = (36, 120, 189)
C3_EPS = 1e-8


def make_c3_run():
    w = workloads.c3_dots(256, 3)
    ctl = O.StepControl(eps_abs=C3_EPS, eps_rel=C3_EPS)
    means = np.zeros((len(C3_DOTS), 5, 3))
    sizes = []
    for i, c in enumerate(C3_DOTS):
        wc = workloads.component(w, c)
        pb = problem(wc)
        dem = O.DemagOracle(pb)
        m = wc.m0.copy()
        t = time.time()
        for k in range(5):
            mr, st = O.relax(pb, m, 100.0, 0.5, demag=dem, ctl=ctl)
            m = O.rows_to_soa(mr)
            means[i, k] = O.mean_m(pb, mr)
        sizes.append(wc.mesh.nx)
        print(f"c3 dot {c} ({wc.mesh.nx} nodes): {time.time() - t:.1f} s, mean m {means[i]}", flush=True)
    np.savez_compressed(HERE / "c3_dots_run.npz", dots=np.array(C3_DOTS), nodes=np.array(sizes), mean_m=means,
                        chunk_ps=100.0, segment_ps=0.5, eps=C3_EPS)


if __name__ == "__main__":
    which = sys.argv[1:] or ["c1", "c4", "c4run", "c3run"]
    if "c1" in which:
        make_c1()
    if "c4" in which:
        make_c4()
    if "c4run" in which:
        make_c4_run()
    if "c3run" in which:
        make_c3_run()
