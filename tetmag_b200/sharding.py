"""Sharding of batched workloads across ranks (one process per GPU).

tetmag runs one mesh on one device (gpu/SetDevice.cu:41-60); a batch of independent instances
-- uneven dots, each its own tetmag problem, or replicas of one mesh with their own initial
state and applied field -- has no exchange step, so it shards without any data-path
collective:

* ``instance_work`` estimates the bytes one mixed field evaluation of each instance streams:
  its sparse operators (nnz of the shared FEM pattern, read about ``SPARSE_PASSES`` times per
  evaluation by the two preconditioned solves and the field kernels, at 8 bytes per entry) plus
  its dense boundary block (Nb^2 FP32 entries).
* ``partition`` assigns instances to ranks by longest-processing-time-first: instances in
  decreasing work, each to the least-loaded rank (ties to the lower rank), so every rank's
  load is within one instance's work of the mean.
* ``select`` builds a rank's sub-batch as a workload of its own (union of its components, or
  its subset of the interleaved replicas), which the rank steps in one context on its GPU.
* ``gather`` collects per-instance results (mean m, energies, ...) in the original instance
  order on every rank, with one object all-gather after the run (host side; the data path
  has none).
* ``Heartbeat`` lets ranks notice, between steps and before their next launch, that a rank has
  left: each rank posts its step number to the process group's key-value store and waits, with
  a short time limit, for every other rank's post.  A missing rank raises ``RankLost`` on the
  others instead of a collective that would wait for it.
"""
from __future__ import annotations

import datetime
from dataclasses import dataclass
from typing import Dict, List, Sequence

import numpy as np

from . import meshgen
from .workloads import Workload, component, instances

# operator passes of one field evaluation: two solves of about ten PCG iterations, each a fine
# product and two smoothing sweeps on the fine level, plus divergence, gradient and local field
SPARSE_PASSES = 64


def mesh_work(tets: np.ndarray, nx: int) -> tuple:
    """(nnz, nb) of a tetrahedral mesh: nnz of the node-pair pattern every FEM operator shares
    (the diagonal plus both directions of every edge) and the number of boundary nodes (nodes of
    faces that belong to one tetrahedron)."""
    t = np.asarray(tets, np.int64)
    if t.size == 0:
        return nx, 0
    pairs = np.concatenate([t[:, [a, b]] for a, b in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))])
    pairs.sort(axis=1)
    edges = np.unique(pairs[:, 0] * nx + pairs[:, 1]).size
    faces = np.concatenate([t[:, [0, 1, 2]], t[:, [0, 1, 3]], t[:, [0, 2, 3]], t[:, [1, 2, 3]]])
    faces.sort(axis=1)
    key = (faces[:, 0] * nx + faces[:, 1]) * nx + faces[:, 2]
    uniq, cnt = np.unique(key, return_counts=True)
    bf = uniq[cnt == 1]
    bnodes = np.unique(np.concatenate([bf // (nx * nx), (bf // nx) % nx, bf % nx]))
    return nx + 2 * edges, int(bnodes.size)


def instance_work(w: Workload) -> np.ndarray:
    """Estimated bytes of one mixed field evaluation per instance of a batched workload."""
    if w.replicas > 1:
        nnz, nb = mesh_work(w.mesh.tets, w.mesh.nx)
        return np.full(w.replicas, SPARSE_PASSES * 8.0 * nnz + 4.0 * nb * nb)
    if w.components is None:
        nnz, nb = mesh_work(w.mesh.tets, w.mesh.nx)
        return np.array([SPARSE_PASSES * 8.0 * nnz + 4.0 * nb * nb])
    out = np.empty(instances(w))
    for c in range(out.size):
        wc = component(w, c)
        nnz, nb = mesh_work(wc.mesh.tets, wc.mesh.nx)
        out[c] = SPARSE_PASSES * 8.0 * nnz + 4.0 * nb * nb
    return out


def partition(work: Sequence[float], nranks: int) -> List[np.ndarray]:
    """Longest-processing-time-first assignment of instances to nranks ranks.  Returns, per rank,
    its instance indices in increasing order.  Deterministic: every rank computes the same
    partition from the same work vector."""
    work = np.asarray(work, np.float64)
    if nranks < 1:
        raise ValueError("partition: nranks must be >= 1")
    if work.ndim != 1 or np.any(~np.isfinite(work)) or np.any(work < 0):
        raise ValueError("partition: work must be a 1-D array of finite non-negative values")
    order = sorted(range(work.size), key=lambda i: (-work[i], i))
    load = np.zeros(nranks)
    owner = np.empty(work.size, np.int64)
    for i in order:
        r = int(np.argmin(load))          # least loaded; argmin takes the lowest rank on ties
        owner[i] = r
        load[r] += work[i]
    return [np.flatnonzero(owner == r) for r in range(nranks)]


def select(w: Workload, idx: Sequence[int]) -> Workload:
    """Sub-batch of instances idx (increasing) as a workload: the union of those components, or
    those interleaved replicas."""
    idx = [int(i) for i in idx]
    if not idx:
        raise ValueError("select: empty instance list")
    if w.replicas > 1:
        m0 = meshgen.deinterleave(w.m0, w.replicas)
        he = meshgen.deinterleave(w.hext, w.replicas)
        info = dict(w.info, instances=idx)
        if len(idx) == 1:
            return Workload(name=f"{w.name}[{idx[0]}]", mesh=w.mesh, Ms=w.Ms, A=w.A, alpha=w.alpha, m0=m0[idx[0]],
                            hext=he[idx[0]], Ku=w.Ku, ku_axis=w.ku_axis, D=w.D, duration_ps=w.duration_ps,
                            segment_ps=w.segment_ps, dmi_kind=w.dmi_kind, info=info)
        return Workload(name=f"{w.name}/shard{len(idx)}", mesh=w.mesh, Ms=w.Ms, A=w.A, alpha=w.alpha,
                        m0=meshgen.interleave([m0[i] for i in idx]), hext=meshgen.interleave([he[i] for i in idx]),
                        Ku=w.Ku, ku_axis=w.ku_axis, D=w.D, duration_ps=w.duration_ps, segment_ps=w.segment_ps,
                        dmi_kind=w.dmi_kind, replicas=len(idx), info=info)
    if w.components is None:
        if idx != [0]:
            raise ValueError("select: a single-mesh workload has one instance")
        return w
    parts = [component(w, i) for i in idx]
    if len(parts) == 1:
        p = parts[0]
        p.info = dict(instances=idx)
        return p
    mesh, off = meshgen.union([p.mesh for p in parts], name=f"{w.name}/shard{len(idx)}")
    stack = lambda vs: None if vs[0] is None else meshgen.soa_stack(vs)  # noqa: E731
    return Workload(name=mesh.name, mesh=mesh, Ms=w.Ms, A=w.A, alpha=w.alpha, m0=stack([p.m0 for p in parts]),
                    hext=stack([p.hext for p in parts]), Ku=w.Ku, ku_axis=stack([p.ku_axis for p in parts]), D=w.D,
                    duration_ps=w.duration_ps, segment_ps=w.segment_ps, components=off, shared_bem=w.shared_bem,
                    dmi_kind=w.dmi_kind, info=dict(instances=idx))


def per_instance_mean_m(w: Workload, m: np.ndarray, node_vol: np.ndarray) -> np.ndarray:
    """Volume-weighted mean magnetisation of every instance of (sub-)batch w for state m (3N SoA
    of the batch): (instances, 3).  node_vol: the mesh's node volumes (N of the union or of the
    replicated mesh)."""
    if w.replicas > 1:
        out = []
        for mr in meshgen.deinterleave(m, w.replicas):
            v = mr.reshape(3, -1)
            out.append(v @ node_vol / node_vol.sum())
        return np.array(out)
    off = w.components if w.components is not None else np.array([0, w.n])
    v = m.reshape(3, -1)
    out = []
    for c in range(len(off) - 1):
        lo, hi = int(off[c]), int(off[c + 1])
        vol = node_vol[lo:hi]
        out.append(v[:, lo:hi] @ vol / vol.sum())
    return np.array(out)


def gather(local: Dict[str, np.ndarray], idx: Sequence[int], total: int, group=None) -> Dict[str, np.ndarray]:
    """Every rank's per-instance arrays (first axis: the rank's instances, in the order of idx)
    assembled in global instance order, on every rank.  One all_gather_object over the process
    group (gloo or nccl); with no initialised process group the local arrays are the result."""
    import torch.distributed as dist

    idx = np.asarray(idx, np.int64)
    payload = {"idx": idx, **{k: np.asarray(v) for k, v in local.items()}}
    if dist.is_available() and dist.is_initialized():
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, payload, group=group)
    else:
        parts = [payload]
    seen = np.concatenate([p["idx"] for p in parts])
    if seen.size != total or np.unique(seen).size != total or seen.min() < 0 or seen.max() >= total:
        raise RuntimeError("gather: the ranks' instance lists do not cover every instance exactly once")
    out = {}
    for k in local:
        first = np.asarray(parts[0][k])
        arr = np.empty((total,) + first.shape[1:], dtype=first.dtype)
        for p in parts:
            arr[p["idx"]] = p[k]
        out[k] = arr
    return out


class RankLost(RuntimeError):
    """A rank did not reach a step within the heartbeat's time limit."""

    def __init__(self, step: int, missing: List[int]):
        super().__init__(f"rank(s) {missing} did not reach step {step}")
        self.step = step
        self.missing = missing


@dataclass
class Heartbeat:
    """Step-level liveness check over a c10d key-value store (TCPStore, FileStore, ...).

    arrive(step) posts this rank's step; check(step) waits at most `timeout_s` for every rank's
    post of that step and raises RankLost listing the ranks that did not post.  Call both between
    steps, with no kernel or collective of this rank in flight, before the next launch."""
    store: object
    rank: int
    world: int
    timeout_s: float = 2.0
    prefix: str = "tmb_hb"

    def _key(self, step: int, r: int) -> str:
        return f"{self.prefix}/{step}/{r}"

    def arrive(self, step: int) -> None:
        self.store.set(self._key(step, self.rank), "1")

    def check(self, step: int) -> None:
        keys = [self._key(step, r) for r in range(self.world)]
        try:
            self.store.wait(keys, datetime.timedelta(seconds=self.timeout_s))
        except Exception:  # the store raises on its time limit (RuntimeError / DistStoreError)
            missing = [r for r, k in enumerate(keys) if not self.store.check([k])]
            if not missing:      # every post arrived just after the limit
                return
            raise RankLost(step, missing) from None

    def step(self, step: int) -> None:
        self.arrive(step)
        self.check(step)
