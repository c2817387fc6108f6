#!/usr/bin/env python3
"""Benchmark of tetmag's full field evaluation (demag chain + local field + LLG
right-hand side) on B200.

Default run: one JSON line for c2 -- a step is one full field evaluation of the 363,609-node
permalloy film (500x500x20 nm at 2.5 nm, seeded vortex, 20 mT in-plane): divergence, Neumann
PCG+AMG, hierarchical (leaf 32, eta 2) double-layer BEM matvec, Dirichlet PCG+AMG, gradient,
fused local field + LLG right-hand side, on the mixed path (FP32 operator values except the CG's
own operator, FP64 vectors / reductions / coarse solve).  The plain FP64 paths are measured in the same run as the speed bar,
with the relative error between them.  The same line carries, under "workloads", the other
configurations measured in the same run: c3 (256 uneven dots in one batched context), c4x64
(64 replicas of one mesh sharing one dense BEM, the boundary product a tensor-core GEMM) and c5
(the interfacial-DMI disk: fixed-step RK4 and its discrete adjoint).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload all|c1|c2|c3|c4|c4x64|c5|cuboid:NXxNYxNZxH]

Under torchrun: c2 runs one replica per rank (independent seeds, no data-path collective; value
= all ranks' evaluations / max-over-ranks time); c3 and c4x64 shard their fixed batch across the
ranks by estimated work (tetmag_b200.sharding); c5 (one mesh) is measured at N = 1 only.

The reference arm (--impl reference) and the cpu_baseline leg time the C++ CPU restatement of the
reference's CPU path (oracle/cpu_field.cpp: GMRES + smoothed-aggregation AMG with ILU(0), the
dense or hierarchical boundary matrix, FP64, OpenMP on every host core) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "field evals/s & simulated ns/hour vs plain FP64 GPU path at <=1e-5 rel. err"
UNIT = "field evals/s"
FALLBACK_HBM_GBS = 6650.0
EXTRAS = ("c3", "c4x64", "c5")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="all",
                   help="all (c2 line with c3, c4x64, c5 under 'workloads'), c1, c2, c3, c4, c4x64, c5, or "
                        "cuboid:NXxNYxNZxH (Kuhn cuboid of NX*NY*NZ cells of edge H nm)")
    p.add_argument("--tol", type=float, default=1e-7)
    p.add_argument("--sim-ps", type=float, default=2.0, help="simulated ps for the ns/hour figure")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--c5-steps", type=int, default=500, help="time steps of the adjoint workload (c5)")
    p.add_argument("--c5-h", type=float, default=3.0,
                   help="lattice spacing of the c5 disk in nm (3.0: 8,188 nodes; 1.75: 41,328 nodes, the "
                        "configuration's 'about 40k')")
    p.add_argument("--bem", default="auto", choices=["auto", "h2", "hmatrix", "hmatrix-only", "hmatrix-dense", "dense"],
                   help="BEM form of the timed paths (the dense FP64 path is measured too, except with "
                        "hmatrix-only: the hierarchical matrix built from the mesh with no dense copy on the "
                        "device, for profiling captures that must stay a few GB); h2: the hierarchical "
                        "matrix built from the mesh, recompressed into nested cluster bases; auto: h2 for c2 "
                        "(its configuration names the H2-compressed BEM), the dense matrix otherwise")
    p.add_argument("--matrix-share", type=float, default=0.0,
                   help="accuracy measure of the hierarchical matrix: 0 block-relative cross approximation, "
                        "s > 0 also a matrix-relative budget per block (tmb_set_bem_accuracy)")
    return p.parse_args()


H2_EPS = (1e-7, 1e-6)     # recompression tolerances of the FP64 and FP32 H2 copies


def bem_for(args, workload: str) -> str:
    if args.bem != "auto":
        return args.bem
    return "hmatrix" if workload == "c2" else "dense"


def peak_hbm():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region (read only)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = ROOT / f"_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.fh = open(self.out, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        self.out.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_workload(name: str, rank: int):
    """The named configuration.  c2 and the single meshes get a seed per rank (independent
    replicas); the batched c3 / c4x64 are the same fixed batch on every rank (sharded later)."""
    from tetmag_b200 import workloads

    if name == "c4":
        return workloads.c4_replica(replica=rank)
    if name == "c4x64":
        return workloads.c4_batch(replicas=64, seed=4)
    if name == "c3":
        return workloads.c3_dots(ndots=256, seed=3)
    if name.startswith("cuboid:"):
        nx, ny, nz, h = name.split(":", 1)[1].split("x")
        return workloads.cuboid_random(int(nx), int(ny), int(nz), float(h), seed=7 + rank, alpha=0.5,
                                       name=f"cuboid_{nx}x{ny}x{nz}_h{h}")
    return workloads.WORKLOADS[name](seed=2 + 17 * rank)


def config_for(w, bem: str, tol: float, world: int, sharded: bool) -> dict:
    """The workload's identity: shared by the GPU arm and the reference arm (same keys, same values)."""
    from tetmag_b200 import sharding, workloads

    nnz, nb = sharding.mesh_work(w.mesh.tets, w.mesh.nx)
    ninst = workloads.instances(w)
    cfg = {"workload": w.name, "nodes": int(w.m0.size // 3), "mesh_nodes": int(w.mesh.nx), "boundary_nodes": nb,
           "nnz": nnz, "instances": ninst,
           "bem": ("H2, leaf 32, eta 2 (tetmag's H2 parameters)" if bem == "h2" else
                "hierarchical, leaf 32, eta 2 (tetmag's H2 parameters)" if bem.startswith("hmatrix")
                else "dense double-layer (Lindholm)"),
           "cg_tol": tol, "states": "W+K distinct seeded perturbed states, warm-started solves",
           "l2": "inputs larger than L2 (c2's boundary matrix alone streams over 1 GB per step)",
           "parallelism": (("instances sharded over %d ranks" % world) if sharded else
                           ("replicas x%d" % world)) if world > 1 else "single"}
    return cfg


# ------------------------------------------------------------------------------------------
# CPU restatement of the reference's path (reference arm and cpu_baseline leg)
# ------------------------------------------------------------------------------------------
def cpu_problem(w):
    """The oracle's problem for one instance of w (the median-sized one of a batch)."""
    from oracle import tetmag_oracle as O
    from tetmag_b200 import workloads

    if w.replicas > 1:
        w = workloads.component(w, 0)
    elif w.components is not None:
        sizes = np.diff(w.components)
        w = workloads.component(w, int(np.argsort(sizes)[len(sizes) // 2]))
    axis = None if w.ku_axis is None else O.soa_to_rows(w.ku_axis)
    pb = O.make_problem(w.mesh.xyz, w.mesh.tets, w.mesh.scale, Ms=w.Ms, A=w.A, alpha=w.alpha, Ku=w.Ku,
                        ku_axis=axis if axis is not None else (0, 0, 1), D=w.D, hext=w.hext, with_bem=False)
    return w, pb


def cpu_field(w, bem: str, tol: float):
    """The C++ CPU restatement set up for (one instance of) w: its AMG hierarchies, and the dense
    boundary matrix (oracle assembly, tetmag's arithmetic) or the hierarchical one (ACA to 1e-6)."""
    from oracle import cpu_ref, tetmag_oracle as O

    wi, pb = cpu_problem(w)
    t = time.perf_counter()
    cf = cpu_ref.CpuField(pb, tol=tol, maxiter=100)
    sa = O.solid_angles(pb.xyz, pb.tets, pb.bnd)
    if bem.startswith("hmatrix") or bem == "h2":
        info = cf.build_hmatrix(sa, leaf=32, eta=2.0, eps=1e-6, kmax=64)
        desc = (f"hierarchical boundary matrix (ACA to 1e-6, {info['bytes'] / 1e9:.2f} GB FP64, built in "
                f"{info['build_s']:.1f} s)")
    else:
        cf.set_bem_dense(O.dense_bem(pb.xyz, pb.tets, pb.bnd, sub=sa))
        desc = "dense boundary matrix"
    return wi, cf, desc, time.perf_counter() - t


def cpu_states(wi, count: int, seed: int):
    rng = np.random.default_rng(seed)
    base = wi.m0.reshape(3, -1)
    out = []
    for _ in range(count):
        s = base + 0.05 * rng.standard_normal(base.shape)
        s /= np.linalg.norm(s, axis=0, keepdims=True)
        out.append(np.ascontiguousarray(s.ravel()))
    return out


def cpu_describe(cf, wi, desc: str, evals: int) -> str:
    inf = cf.info()
    return (f"C++ FP64 restatement of the reference's CPU path on {cf.threads} OpenMP threads "
            f"(instance {wi.name}, N={cf.n}, Nb={cf.nb}): {evals} full field evaluations, each timed whole "
            f"(divergence, Neumann and Dirichlet GMRES(30) with smoothed-aggregation AMG / ILU(0) at the "
            f"reference's tolerance, warm-started, AMG levels {inf['amg_levels']}; {desc}; gradient, local "
            f"field and LLG right-hand side); no extrapolation")


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    name = "c2" if args.workload == "all" else args.workload
    bem = bem_for(args, name)
    w = make_workload(name, 0)
    wi, cf, desc, setup_s = cpu_field(w, bem, args.tol)
    states = cpu_states(wi, args.warmup + args.steps, 1000)
    for k in range(args.warmup):
        cf.field_eval(states[k])
    cf.reset_timers()
    t = time.perf_counter()
    for k in range(args.steps):
        cf.field_eval(states[args.warmup + k])
    tot = time.perf_counter() - t
    inf = cf.info()
    value = args.steps / tot
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_for(w, bem, args.tol, world, name in ("c3", "c4x64")),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cf.threads, "kind": "port",
                         "sample": cpu_describe(cf, wi, desc, args.steps)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "components_s_per_eval": {k: inf[k] / args.steps for k in
                                  ("div_s", "neumann_s", "bem_s", "dirichlet_s", "local_s")},
        "iterations_last_eval": [inf["it_neumann"], inf["it_dirichlet"]],
        "setup_s": setup_s,
    }
    if w.replicas > 1 or w.components is not None:
        line["note"] = "value is per instance (one instance of the batch, the reference runs one mesh per process)"
    print(json.dumps(line), flush=True)


def cpu_baseline_leg(w, bem: str, tol: float, evals: int = 3) -> dict:
    wi, cf, desc, setup_s = cpu_field(w, bem, tol)
    states = cpu_states(wi, evals + 1, 2000)
    cf.field_eval(states[0])
    cf.reset_timers()
    t = time.perf_counter()
    for k in range(evals):
        cf.field_eval(states[1 + k])
    tot = time.perf_counter() - t
    inf = cf.info()
    return {"value": evals / tot, "unit": UNIT + (" (one instance)" if wi is not w else ""), "cores": cf.threads,
            "kind": "port", "sample": cpu_describe(cf, wi, desc, evals),
            "components_s_per_eval": {k: inf[k] / evals for k in
                                      ("div_s", "neumann_s", "bem_s", "dirichlet_s", "local_s")},
            "setup_s": setup_s}


# ------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world, self.rank, self.local = dist_env()
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg is not None:
            self.pg.barrier()

    def max(self, x: float, dev) -> float:
        if self.pg is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg is not None:
            self.pg.destroy_process_group()


def roofline_of(prof: dict) -> tuple:
    """The single kernel with the largest total time in the profiled pass (solver kernels included;
    the ids that group several kernels -- the boundary product, the per-level transfer and coarse
    sweeps, the containers -- are reported under `kernels` but are not one kernel) and its achieved
    algorithmic bandwidth."""
    from tetmag_b200.api import PROFILE_SINGLE

    cands = {k: v for k, v in prof.items() if k in PROFILE_SINGLE and v["launches"] > 0}
    dom = max(cands, key=lambda k: cands[k]["total_ms"])
    d = cands[dom]
    avg_ms = d["total_ms"] / d["launches"]
    achieved = d["bytes_per_launch"] / (avg_ms / 1e3) / 1e9
    return dom, d, avg_ms, achieved


def measure(args, name: str, dist: Dist, full: bool) -> dict:
    """Field evaluations of workload `name` on this rank's GPU.  full: the headline extras too
    (dense FP64 reference path, frozen-demag local rate, relaxation rate)."""
    import torch
    from tetmag_b200 import api, sharding, workloads

    world, rank, local = dist.world, dist.rank, dist.local
    dev = torch.device("cuda", local)
    bem = bem_for(args, name)
    w_all = make_workload(name, rank)
    sharded = name in ("c3", "c4x64") and world > 1
    w = w_all
    if sharded:
        parts = sharding.partition(sharding.instance_work(w_all), world)
        w = sharding.select(w_all, parts[rank])
    ninst = workloads.instances(w)
    ninst_all = workloads.instances(w_all) if sharded else world * ninst
    t0 = time.perf_counter()
    hier = bem != "dense"
    dense_ref = bem != "hmatrix-only"
    mo, ctx = workloads.setup_context(w, device=local, mixed=True, tol=args.tol, maxiter=100,
                                      hmatrix={"hmatrix": "mesh", "hmatrix-only": "mesh", "h2": "mesh",
                                               "hmatrix-dense": True}.get(bem, False),
                                      keep_dense=dense_ref, h2=H2_EPS if bem == "h2" else None,
                                      matrix_share=args.matrix_share if hier else 0.0)
    hier_mode = 2 if bem == "h2" else 1
    bem_info = ctx.bem_info() if hier else None
    if hier:
        bem_info["matrix_share"] = args.matrix_share
    if hier and dense_ref:
        bem_info["verify"] = ctx.bem_verify()
    if bem == "h2":
        bem_info["h2"] = ctx.bem_h2_info()
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.Stream(dev)
    ctx.set_stream(stream.cuda_stream)
    torch.cuda.set_stream(stream)
    n = w.m0.size // 3
    K, W = args.steps, args.warmup
    rng = np.random.default_rng(1000 + rank)
    base = w.m0.reshape(3, n)
    states = []
    for _ in range(W + K):
        s = base + 0.05 * rng.standard_normal((3, n))
        s /= np.linalg.norm(s, axis=0, keepdims=True)
        states.append(s.ravel())
    S = torch.from_numpy(np.stack(states)).to(dev)
    ydot = torch.empty(3 * n, dtype=torch.float64, device=dev)
    hdem = torch.empty(3 * n, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)

    def timed(mixed: bool, profile: bool, dense: bool = False):
        ctx.set_precision(mixed)
        if hier:
            ctx.set_bem_mode(0 if dense else hier_mode)
        for k in range(W):
            ctx.field_eval(S[k], ydot, hdem)
        torch.cuda.synchronize(dev)
        dist.barrier()
        torch.cuda.synchronize(dev)
        if profile:
            api.profile_enable(ctx, True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = api.kernel_launches()
        its = [0, 0]
        tag = f"timed_{name}_{'mixed' if mixed else 'fp64'}{'_dense' if dense else ''}{'_prof' if profile else ''}"
        torch.cuda.nvtx.range_push(tag)
        e0.record(stream)
        for k in range(K):
            ctx.field_eval(S[W + k], ydot, hdem)
            st = ctx.stats()
            its[0] += st["it_neumann"]
            its[1] += st["it_dirichlet"]
        e1.record(stream)
        torch.cuda.synchronize(dev)
        torch.cuda.nvtx.range_pop()
        dist.barrier()
        ms = e0.elapsed_time(e1)
        launches = api.kernel_launches() - l0
        prof = api.profile_read(ctx) if profile else None
        if profile:
            api.profile_enable(ctx, False)
        return dist.max(ms, dev), launches, prof, its, ms

    clocks = Clocks(local)
    clocks.start()
    ms_mx, launches, _, its_mx, _ = timed(True, False)
    clk = clocks.stop()
    ms_64, _, _, its_64, _ = timed(False, False)
    ms_64d = timed(False, False, dense=True)[0] if hier and dense_ref else None
    # per-kernel CUDA-event timing in a separate pass over the same K states (with the profiler
    # on, the PCG runs kernel by kernel instead of from CUDA graphs)
    _, _, prof, _, ms_prof = timed(True, True)

    # relative error of the mixed path against FP64 (dense BEM where present), solved to 1e-12
    probe = S[W + K - 1]
    ctx.set_precision(False)
    if hier and dense_ref:
        ctx.set_bem_mode(False)
    ctx.set_solver_params(1e-12, 300)
    h64 = hdem.clone()
    y64 = ctx.field_eval(probe, torch.empty_like(ydot), h64)
    err64 = None
    if hier:
        ctx.set_bem_mode(hier_mode)
        h64h = hdem.clone()
        y64h = ctx.field_eval(probe, torch.empty_like(ydot), h64h)
    ctx.set_precision(True)
    ctx.set_solver_params(args.tol, 100)
    hmx = hdem.clone()
    ymx = ctx.field_eval(probe, torch.empty_like(ydot), hmx)
    torch.cuda.synchronize(dev)

    def relerr(a, b):
        return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))

    err = {"hdem": relerr(hmx, h64), "ydot": relerr(ymx, y64),
           "reference": "FP64, " + ("dense" if (dense_ref or not hier) else "hierarchical") + " BEM, CG to 1e-12"}
    if hier and dense_ref:
        err64 = {"hdem": relerr(h64h, h64), "ydot": relerr(y64h, y64)}

    # end to end through the public API with host buffers (H2D of m from pinned host memory, D2H
    # of ydot into pinned host memory, per step)
    host_states = [torch.from_numpy(np.ascontiguousarray(st)).pin_memory() for st in states]
    yh = torch.empty(3 * n, dtype=torch.float64).pin_memory()
    for k in range(W):
        ctx.field_eval(host_states[k], yh)
    dist.barrier()
    t = time.perf_counter()
    for k in range(K):
        ctx.field_eval(host_states[W + k], yh)
    e2e_s = dist.max(time.perf_counter() - t, dev)

    # simulated time: the frozen-demag relaxation loop (0.5 ps segments), mixed; one untimed
    # segment first, then the best of three runs from the same state
    ctx.relax(S[0].clone(), duration_ps=0.5, segment_ps=0.5)
    sim_runs = []
    for _ in range(3):
        mrun = S[0].clone()
        torch.cuda.synchronize(dev)
        dist.barrier()
        t = time.perf_counter()
        rs = ctx.relax(mrun, duration_ps=args.sim_ps, segment_ps=0.5)
        sim_runs.append(dist.max(time.perf_counter() - t, dev))
    sim_s = min(sim_runs)
    ns_per_hour = ninst_all * (args.sim_ps * 1e-3) / (sim_s / 3600.0)

    local_per_s = None
    if full:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for k in range(3):
            ctx.llg_rhs(0.0, S[k], ydot)
        e0.record(stream)
        nloc = 50
        for k in range(nloc):
            ctx.llg_rhs(0.0, S[k % (W + K)], ydot)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        local_per_s = ninst_all * nloc / (dist.max(e0.elapsed_time(e1), dev) / 1e3)

    # batched workloads: the plain FP64 path one instance at a time (one single-mesh context per
    # instance, as the reference runs one mesh per process) on a sample of this rank's instances
    unbatched = None
    if ninst > 1:
        if w.replicas > 1 or w.shared_bem:
            sample = [0]
        else:
            sizes = np.diff(w.components)
            sample = sorted(set(int(i) for i in
                                np.argsort(sizes)[np.linspace(0, ninst - 1, min(ninst, 8)).astype(int)]))
        t_tot, n_ev = 0.0, 0
        for c in sample:
            wc = workloads.component(w, c)
            _, cx = workloads.setup_context(wc, device=local, mixed=False, tol=args.tol, maxiter=100)
            cx.set_stream(stream.cuda_stream)
            mc = torch.from_numpy(np.ascontiguousarray(wc.m0)).to(dev)
            yc = torch.empty_like(mc)
            for _ in range(W):
                cx.field_eval(mc, yc)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(K):
                cx.field_eval(mc, yc)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            t_tot += e0.elapsed_time(e1) / 1e3
            n_ev += K
            del cx
        unbatched = {"value": n_ev / t_tot, "unit": "instance field evals/s (one GPU)",
                     "instances_sampled": len(sample),
                     "path": "plain FP64, one single-mesh context per instance, dense BEM, same CG tolerance"}

    value = ninst_all * K / (ms_mx / 1e3)
    fp64_value = ninst_all * K / (ms_64 / 1e3)
    peak, peak_kind = peak_hbm()
    dom, d, avg_ms, achieved = roofline_of(prof)
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        traffic = json.loads(tf.read_text()).get(w_all.name + ("/" + bem if hier else ""), {}).get(dom)
    kshare = {k: round(v["total_ms"] / ms_prof, 4) for k, v in prof.items()
              if v["launches"] > 0 and k not in ("demag_chain",)}
    out = {
        "name": name, "w": w_all, "bem": bem, "value": value, "ms_per_step": ms_mx / K, "fp64_value": fp64_value,
        "launches": launches, "clocks": clk, "ninst": ninst_all, "sharded": sharded,
        "e2e": {"value": ninst_all * K / e2e_s, "unit": UNIT if ninst_all == 1 else "instance field evals/s",
                "h2d_bytes_per_step": 3 * n * 8, "d2h_bytes_per_step": 3 * n * 8},
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "bytes_per_launch": d["bytes_per_launch"], "avg_ms": avg_ms, "launches": d["launches"]},
        "rel_err_vs_fp64": err, "rel_err_fp64_hier_vs_dense": err64,
        "fp64_dense_value": ninst_all * K / (ms_64d / 1e3) if ms_64d else None,
        "bem_info": bem_info, "bem_gemm": ctx.bem_gemm_info() if (w.shared_bem or w.replicas > 1) else None,
        "local_rhs_evals_per_s": local_per_s, "sim_ns_per_hour": ns_per_hour,
        "relax": {"sim_ps": args.sim_ps, "wall_s": sim_s, "steps": rs["accepted"], "rejected": rs["rejected"],
                  "rhs": rs["rhs"]},
        "cg_iters_per_eval": {"mixed": [i / K for i in its_mx], "fp64": [i / K for i in its_64]},
        "kernel_time_share": kshare,
        "kernels": {k: {"launches": v["launches"], "avg_us": 1e3 * v["total_ms"] / v["launches"],
                        "gbs": (v["bytes_per_launch"] / (v["total_ms"] / v["launches"] / 1e3) / 1e9)
                        if v["total_ms"] > 0 and v["bytes_per_launch"] > 0 else None,
                        "frac": (v["bytes_per_launch"] / (v["total_ms"] / v["launches"] / 1e3) / 1e9 / peak)
                        if v["total_ms"] > 0 and v["bytes_per_launch"] > 0 else None}
                    for k, v in prof.items() if v["launches"] > 0 and k not in api.PROFILE_CONTAINERS},
        "profiled_pass_ms_per_step": ms_prof / K,
        "plain_fp64_unbatched": unbatched,
        "speedup_vs_plain_fp64_unbatched": (value / world / unbatched["value"]) if unbatched else None,
        "setup_s": setup_s,
        "config": config_for(w_all, bem, args.tol, world, sharded),
    }
    del ctx, mo
    return out


def extra_summary(r: dict) -> dict:
    """Compact record of a secondary workload for the headline line."""
    keys = ("value", "ms_per_step", "fp64_value", "e2e", "roofline", "rel_err_vs_fp64", "sim_ns_per_hour",
            "cg_iters_per_eval", "kernel_time_share", "plain_fp64_unbatched", "speedup_vs_plain_fp64_unbatched",
            "bem_gemm", "launches", "clocks", "setup_s", "config")
    out = {k: r[k] for k in keys if k in r}
    out["unit"] = "instance field evals/s" if r["ninst"] > 1 else UNIT
    out["speedup_vs_fp64_same_path"] = r["value"] / r["fp64_value"]
    return out


def headline_line(args, r: dict, world: int) -> dict:
    line = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
        "scaling": "strong" if r["sharded"] else "weak", "vs_baseline": None,
        "dtype": "f32 operators / f64 vectors+reductions", "data": "synthetic", "config": r["config"],
        "path": "mixed precision (FP32 operator values except the CG's own operator; FP64 vectors, reductions, coarse solve, step control)",
        "e2e": r["e2e"], "gpu_launches": r["launches"], "roofline": r["roofline"], "clocks": r["clocks"],
    }
    for k in ("fp64_value", "fp64_dense_value", "rel_err_vs_fp64", "rel_err_fp64_hier_vs_dense", "bem_info",
              "bem_gemm", "local_rhs_evals_per_s", "sim_ns_per_hour", "relax", "cg_iters_per_eval",
              "kernel_time_share", "kernels", "profiled_pass_ms_per_step", "plain_fp64_unbatched",
              "speedup_vs_plain_fp64_unbatched", "setup_s"):
        line[k] = r.get(k)
    line["speedup_vs_fp64"] = r["value"] / r["fp64_value"]
    if r.get("fp64_dense_value"):
        line["speedup_vs_fp64_dense"] = r["value"] / r["fp64_dense_value"]
    return line


def run_gpu(args):
    import torch

    dist = Dist()
    torch.cuda.set_device(dist.local)
    main_name = "c2" if args.workload == "all" else args.workload
    r = measure(args, main_name, dist, full=True)
    line = headline_line(args, r, dist.world)
    if args.workload == "all":
        extras = {}
        for name in EXTRAS:
            if name == "c5":
                if dist.world == 1:
                    extras[name] = run_adjoint(args, dist)
                else:
                    extras[name] = {"skipped": "one mesh: measured at N = 1 only (replicas only)"}
            else:
                extras[name] = extra_summary(measure(args, name, dist, full=False))
        line["workloads"] = extras
        # every kernel launched in the timed regions of the run, all workloads
        line["gpu_launches_all_workloads"] = r["launches"] + sum(
            v.get("launches", 0) or 0 for v in extras.values() if isinstance(v, dict))
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_leg(r["w"], r["bem"], args.tol)
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    dist.close()


def run_adjoint(args, dist: Dist | None = None) -> dict:
    """c5: the interfacial-DMI disk integrated with fixed-step RK4 (full field at every stage) and
    the discrete adjoint of that map.  value = field evaluations / s of the mixed forward run;
    the adjoint's cost is reported as (forward + backward sweep time) / forward time."""
    import torch
    from tetmag_b200 import api, workloads
    from tetmag_b200.autograd import LLGObjective

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    nsteps = args.c5_steps
    w = workloads.c5_disk(nsteps=nsteps, h=args.c5_h)
    info = w.info
    t0 = time.perf_counter()
    mo, ctx = workloads.setup_context(w, device=local, mixed=True, tol=args.tol, maxiter=200)
    nsub = workloads.stable_substeps(w, mo, info["dt_ps"])
    setup_s = time.perf_counter() - t0
    n = w.n
    node_vol = mo.operators()["node_vol"]
    wv = np.zeros(3 * n)
    wv[2 * n:] = node_vol / node_vol.sum()                  # J = volume-weighted mean m_z
    Js, A_, _, axis, D = w.material_arrays()
    ku0 = np.zeros(n)
    bz0 = np.asarray(info["bz"])
    ckpt = info["ckpt_every"]
    prob = LLGObjective(ctx, Js, A_, axis, D, w.alpha, w.m0, wv, nsteps, info["dt_ps"], nsub=nsub, ckpt_every=ckpt,
                        bz_t0=info["bz_t0"], bz_t1=info["bz_t1"])

    def sync():
        torch.cuda.synchronize()

    def timed_forward(tag):
        sync()
        torch.cuda.nvtx.range_push(f"timed_forward_{tag}")
        t = time.perf_counter()
        J = prob.forward_only(ku0, bz0)
        sync()
        torch.cuda.nvtx.range_pop()
        return J, time.perf_counter() - t

    def timed_adjoint(tag):
        sync()
        torch.cuda.nvtx.range_push(f"timed_adjoint_{tag}")
        t = time.perf_counter()
        r = prob.run(ku0, bz0)
        sync()
        torch.cuda.nvtx.range_pop()
        return r, time.perf_counter() - t

    out = {}
    clocks = Clocks(local)
    clk = None
    for mixed in (True, False):
        ctx.set_precision(mixed)
        ctx.set_solver_params(args.tol if mixed else 1e-12, 200)
        if args.warmup > 0:
            prob.forward_only(ku0, bz0)
        if mixed:
            clocks.start()
        l0 = api.kernel_launches()
        tag = "mixed" if mixed else "fp64"
        Jf, tf = timed_forward(tag)
        launches = api.kernel_launches() - l0
        r, ta = timed_adjoint(tag)
        if mixed:
            clk = clocks.stop()
        out[mixed] = dict(J=Jf, forward_s=tf, adjoint_s=ta, r=r, launches=launches)
    mx, f64 = out[True], out[False]
    evals = 4.0 * nsteps * nsub
    rng = np.random.default_rng(17)
    ctx.set_precision(True)
    ctx.set_solver_params(args.tol, 200)
    fd = {}
    v = rng.standard_normal(n)
    eps = 200.0
    d_ku = (prob.forward_only(ku0 + eps * v, bz0) - prob.forward_only(ku0 - eps * v, bz0)) / (2 * eps)
    g = float(mx["r"]["grad_ku"] @ v)
    fd["ku"] = {"fd": d_ku, "adjoint": g, "rel_err": abs(d_ku - g) / abs(g)}
    v = rng.standard_normal(bz0.size)
    eps = 1e-3
    d_bz = (prob.forward_only(ku0, bz0 + eps * v) - prob.forward_only(ku0, bz0 - eps * v)) / (2 * eps)
    g = float(mx["r"]["grad_bz"] @ v)
    fd["bz"] = {"fd": d_bz, "adjoint": g, "rel_err": abs(d_bz - g) / abs(g)}

    def rel(a, b):
        return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))

    value = evals / mx["forward_s"]
    res = {
        "value": value, "unit": UNIT, "ms_per_step": 1e3 * mx["forward_s"] / evals,
        "config": {"workload": w.name, "nodes": n, "boundary_nodes": mo.nb, "nnz": mo.nnz, "dmi": "interfacial",
                   "steps": nsteps, "dt_ps": info["dt_ps"], "rk4_substeps": nsub, "checkpoint_every": ckpt,
                   "bz_samples": int(bz0.size), "objective": "volume-weighted mean m_z after the run",
                   "parameters": "per-node Ku (FP32 tensor, baseline 0, easy axis z) and the Bz(t) samples",
                   "cg_tol": args.tol, "parallelism": "single",
                   "timing": "host wall clock around synchronous library calls (one stream)"},
        "launches": mx["launches"], "clocks": clk,
        "fp64_value": evals / f64["forward_s"],
        "sim_ns_per_hour": nsteps * info["dt_ps"] * 1e-3 / (mx["forward_s"] / 3600.0),
        "adjoint": {
            "forward_s": mx["forward_s"], "forward_plus_adjoint_s": mx["adjoint_s"],
            "cost_ratio": mx["adjoint_s"] / mx["forward_s"],
            "cost_ratio_fp64": f64["adjoint_s"] / f64["forward_s"],
            "fd_check_mixed": fd,
            "grad_rel_err_mixed_vs_fp64": {"ku": rel(mx["r"]["grad_ku"], f64["r"]["grad_ku"]),
                                           "bz": rel(mx["r"]["grad_bz"], f64["r"]["grad_bz"])},
            "J": {"mixed": mx["J"], "fp64": f64["J"]},
            "mean_m_diff_mixed_vs_fp64": abs(mx["J"] - f64["J"]),
            "stats_mixed": mx["r"]["stats"], "stats_fp64": f64["r"]["stats"]},
        "setup_s": setup_s,
    }
    del ctx, mo
    return res


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c5":
        res = run_adjoint(args)
        world, rank, _ = dist_env()
        line = {"metric": METRIC, "n_gpus": world, "steps": 1, "warmup": args.warmup, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 operators / f64 vectors+reductions",
                "data": "synthetic", "gpu_launches": res["launches"], **res}
        if rank == 0:
            print(json.dumps(line), flush=True)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
