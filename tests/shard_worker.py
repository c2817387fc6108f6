"""One rank of the world-size-2 sharding tests (run as a child process by tests/test_sharding.py).

    python tests/shard_worker.py --rank R --world W --port P --mode gather|leave --out FILE

gather: partition a small batch of uneven dots by work, build this rank's sub-batch, compute
        each instance's mean m and node count from its initial state (host only), gather them
        over a gloo process group and write the assembled arrays to FILE (npz).
leave:  step a heartbeat over a TCPStore; the last rank leaves after step 1 (between steps,
        nothing in flight); the others record the RankLost they get at step 2 in FILE (json).
"""
import argparse
import datetime
import json
import os
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402


def small_batch():
    from tetmag_b200 import workloads

    # six dots, sides 8-20 nm at 4 nm cells: tens to a few hundred nodes each
    w = workloads.c3_dots(ndots=6, seed=11, h_range=(4.0, 4.0))
    return w


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--rank", type=int, required=True)
    p.add_argument("--world", type=int, required=True)
    p.add_argument("--port", type=int, required=True)
    p.add_argument("--mode", choices=["gather", "leave"], required=True)
    p.add_argument("--out", required=True)
    a = p.parse_args()
    import torch.distributed as dist

    from tetmag_b200 import sharding

    if a.mode == "gather":
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{a.port}", rank=a.rank, world_size=a.world,
                                timeout=datetime.timedelta(seconds=60))
        w = small_batch()
        work = sharding.instance_work(w)
        parts = sharding.partition(work, a.world)
        mine = parts[a.rank]
        sub = sharding.select(w, mine)
        # node volumes of the sub-batch: uniform weights are enough for the gather check
        vol = np.ones(sub.n)
        mean_m = sharding.per_instance_mean_m(sub, sub.m0, vol)
        nodes = (np.diff(sub.components) if sub.components is not None else np.array([sub.n]))
        got = sharding.gather({"mean_m": mean_m, "nodes": nodes, "rank": np.full(len(mine), a.rank)}, mine,
                              len(work))
        with open(a.out, "wb") as f:
            np.savez(f, **got, work=work)
        dist.barrier()
        dist.destroy_process_group()
        return 0

    store = dist.TCPStore("127.0.0.1", a.port, world_size=a.world, is_master=(a.rank == 0),
                          timeout=datetime.timedelta(seconds=30))
    hb = sharding.Heartbeat(store, a.rank, a.world, timeout_s=2.0)
    leaver = a.world - 1
    result = {"rank": a.rank, "steps_done": 0, "lost": None}
    for step in range(4):
        if a.rank == leaver and step == 2:
            result["left_at"] = step
            break                        # leaves between steps: posts nothing for step 2
        try:
            hb.step(step)
        except sharding.RankLost as e:
            result["lost"] = {"step": e.step, "missing": e.missing}
            break
        result["steps_done"] = step + 1
    Path(a.out).write_text(json.dumps(result))
    return 0


if __name__ == "__main__":
    sys.exit(main())
