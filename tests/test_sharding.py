"""Sharding of batched workloads across ranks (tetmag_b200.sharding), on CPU.

Partition balance and determinism, the per-instance work estimate against the library's own
preprocessing, sub-batches, and two world-size-2 runs as child processes: a gloo gather of
per-instance results, and a rank that leaves between steps (made on the host) noticed by the
other through the heartbeat before its next step.
"""
import json
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from tetmag_b200 import meshgen, sharding, workloads

WORKER = Path(__file__).with_name("shard_worker.py")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("nranks", [1, 2, 3, 8])
def test_partition_covers_and_balances(nranks):
    rng = np.random.default_rng(nranks)
    work = rng.uniform(1.0, 100.0, 256)
    parts = sharding.partition(work, nranks)
    allidx = np.concatenate(parts)
    assert np.array_equal(np.sort(allidx), np.arange(256))
    loads = np.array([work[p].sum() for p in parts])
    # longest-processing-time-first: every rank within one instance's work of the others
    assert loads.max() - loads.min() <= work.max() + 1e-9
    assert all(np.all(np.diff(p) > 0) for p in parts)
    again = sharding.partition(work, nranks)
    assert all(np.array_equal(a, b) for a, b in zip(parts, again))


def test_partition_more_ranks_than_instances_and_errors():
    parts = sharding.partition([3.0, 1.0], 4)
    assert [p.tolist() for p in parts] == [[0], [1], [], []]
    with pytest.raises(ValueError):
        sharding.partition([1.0, np.nan], 2)
    with pytest.raises(ValueError):
        sharding.partition([1.0], 0)


def test_mesh_work_matches_library_preprocessing():
    from tetmag_b200.api import MeshOps

    for dims in ((3, 4, 2, 2.5), (7, 2, 1, 3.0)):
        m = meshgen.kuhn_cuboid(*dims)
        nnz, nb = sharding.mesh_work(m.tets, m.nx)
        mo = MeshOps(m.xyz, m.tets)
        assert (nnz, nb) == (mo.nnz, mo.nb)


def test_select_components_and_replicas():
    w = workloads.c3_dots(ndots=5, seed=2, h_range=(4.0, 4.0))
    sub = sharding.select(w, [1, 3])
    a, b = workloads.component(w, 1), workloads.component(w, 3)
    assert sub.n == a.n + b.n
    assert np.array_equal(sub.components, [0, a.n, a.n + b.n])
    assert np.array_equal(sub.m0.reshape(3, -1)[:, :a.n], a.m0.reshape(3, -1))
    assert np.array_equal(sub.hext.reshape(3, -1)[:, a.n:], b.hext.reshape(3, -1))
    mesh = meshgen.kuhn_cuboid(3, 2, 1, 2.0)
    n = mesh.nx
    reps = [meshgen.random_state(n, s) for s in range(4)]
    wr = workloads.Workload(name="r", mesh=mesh, Ms=8e5, A=1.3e-11, alpha=0.5, m0=meshgen.interleave(reps),
                            hext=meshgen.interleave([np.full(3 * n, float(s)) for s in range(4)]), replicas=4)
    sr = sharding.select(wr, [0, 2, 3])
    assert sr.replicas == 3
    back = meshgen.deinterleave(sr.m0, 3)
    assert all(np.array_equal(x, reps[i]) for x, i in zip(back, [0, 2, 3]))
    one = sharding.select(wr, [2])
    assert one.replicas == 1 and np.array_equal(one.m0, reps[2])
    mm = sharding.per_instance_mean_m(sr, sr.m0, np.ones(n))
    assert np.allclose(mm, [reps[i].reshape(3, -1).mean(axis=1) for i in (0, 2, 3)])


def _run_ranks(mode, world, tmp_path, timeout=120):
    port = _free_port()
    outs = [tmp_path / f"{mode}{r}.out" for r in range(world)]
    procs = [subprocess.Popen([sys.executable, str(WORKER), "--rank", str(r), "--world", str(world), "--port",
                               str(port), "--mode", mode, "--out", str(outs[r])],
                              stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True) for r in range(world)]
    logs = []
    for p in procs:
        try:
            logs.append(p.communicate(timeout=timeout)[0])
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
    for p, log in zip(procs, logs):
        assert p.returncode == 0, log
    return outs


def test_world_size_2_gloo_gather(tmp_path):
    outs = _run_ranks("gather", 2, tmp_path)
    w = workloads.c3_dots(ndots=6, seed=11, h_range=(4.0, 4.0))
    work = sharding.instance_work(w)
    parts = sharding.partition(work, 2)
    assert all(len(p) > 0 for p in parts)
    want = np.array([workloads.component(w, c).m0.reshape(3, -1).mean(axis=1) for c in range(6)])
    nodes = np.diff(w.components)
    for o in outs:
        g = np.load(o)
        assert np.allclose(g["mean_m"], want, rtol=0, atol=1e-15)
        assert np.array_equal(g["nodes"], nodes)
        assert np.array_equal(g["work"], work)
        for r, p in enumerate(parts):
            assert np.all(g["rank"][p] == r)


def test_world_size_2_rank_leaving_between_steps(tmp_path):
    outs = _run_ranks("leave", 2, tmp_path)
    r0, r1 = (json.loads(o.read_text()) for o in outs)
    assert r1["left_at"] == 2 and r1["steps_done"] == 2
    assert r0["steps_done"] == 2
    assert r0["lost"] == {"step": 2, "missing": [1]}
