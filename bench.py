#!/usr/bin/env python3
"""Benchmark of tetmag's full field evaluation (demag chain + local field + LLG
right-hand side) on B200.

Default (c2): a step is one full field evaluation of the 363,609-node permalloy
film (500x500x20 nm at 2.5 nm, seeded vortex, 20 mT in-plane): divergence,
Neumann PCG+AMG, hierarchical (leaf 32, eta 2) double-layer BEM matvec,
Dirichlet PCG+AMG, gradient, fused local field + LLG right-hand side.  The
headline path is the mixed one (FP32 operator values, FP64 vectors /
reductions / coarse solve); the plain FP64 paths (hierarchical and dense BEM)
are measured in the same run as the speed bar, with the relative error between
them.  Other workloads: c1, c3 (256 uneven dots in one batched context), c4 /
c4x64 (replicas sharing one dense BEM, the boundary product a GEMM), c5 (the
interfacial-DMI disk: fixed-step RK4 and its discrete adjoint).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload c2]

Under torchrun each rank evaluates its own replica (independent seed): no
data-path collective; value = all ranks' evaluations / max-over-ranks time.
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


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="c2",
                   help="c1, c2, c4, or cuboid:NXxNYxNZxH (Kuhn cuboid of NX*NY*NZ cells of edge H nm)")
    p.add_argument("--tol", type=float, default=1e-7)
    p.add_argument("--sim-ps", type=float, default=2.0, help="simulated ps for the ns/hour figure")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--c5-steps", type=int, default=500, help="time steps of the adjoint workload (c5)")
    p.add_argument("--bem", default="auto", choices=["auto", "hmatrix", "hmatrix-only", "hmatrix-dense", "dense"],
                   help="BEM form of the timed paths (the dense FP64 path is measured too, except with "
                        "hmatrix-only: the hierarchical matrix built from the mesh with no dense copy on the "
                        "device, for profiling captures that must stay a few GB); auto: the hierarchical "
                        "matrix built from the mesh for c2 (its configuration names the H2-compressed BEM), "
                        "the dense matrix otherwise")
    a = p.parse_args()
    if a.bem == "auto":
        a.bem = "hmatrix" if a.workload == "c2" else "dense"
    return a


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


def make_workload(name: str, rank: int):
    """The named configuration; each rank gets its own seed (independent replicas)."""
    from tetmag_b200 import workloads

    if name == "c4":
        return workloads.c4_replica(replica=rank)
    if name == "c4x64":
        return workloads.c4_batch(replicas=64, seed=4 + 1000 * rank)
    if name == "c3":
        return workloads.c3_dots(ndots=256, seed=3 + 1000 * rank)
    if name.startswith("cuboid:"):
        nx, ny, nz, h = name.split(":", 1)[1].split("x")
        w = workloads.cuboid_random(int(nx), int(ny), int(nz), float(h), seed=7 + rank, alpha=0.5,
                                    name=f"cuboid_{nx}x{ny}x{nz}_h{h}")
        return w
    return workloads.WORKLOADS[name](seed=2 + 17 * rank)


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline_sample(w, samples: int = 1):
    """Oracle field evaluation on the host cores (bounded sample).  For a batched workload the
    sample is one instance (the median-sized one) and the rate is per instance."""
    from oracle import cpu_baseline, tetmag_oracle as O
    from tetmag_b200 import workloads

    if w.replicas > 1:
        w = workloads.component(w, 0)
    elif w.components is not None:
        sizes = np.diff(w.components)
        w = workloads.component(w, int(np.argsort(sizes)[len(sizes) // 2]))
    axis = None if w.ku_axis is None else O.soa_to_rows(w.ku_axis)
    pb = O.make_problem(w.mesh.xyz, w.mesh.tets, w.mesh.scale, Ms=w.Ms, A=w.A, alpha=w.alpha, Ku=w.Ku,
                        ku_axis=axis if axis is not None else (0, 0, 1), D=w.D, hext=w.hext, with_bem=False)
    ev = cpu_baseline.CpuFieldEval(pb)
    m = O.soa_to_rows(w.m0)
    ev.calibrate(m)
    res = [ev.sample(m) for _ in range(samples)]
    return ev, res, m


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from tetmag_b200 import workloads

    w = make_workload(args.workload, 0)
    ev, res, m = cpu_baseline_sample(w, samples=0)
    for _ in range(args.warmup):
        ev.sample(m)
    tot = 0.0
    parts = []
    for _ in range(args.steps):
        r = ev.sample(m)
        tot += r["total_s"]
        parts.append(r)
    value = args.steps / tot
    cores = ev.threads
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w.name, "nodes": w.n, "impl": "oracle port on host cores"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": ev.describe()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "components_s": {k: float(np.mean([p[k] for p in parts])) for k in
                         ("local_s", "div_grad_s", "solves_s", "bem_s")},
    }
    print(json.dumps(line), flush=True)


def run_gpu(args):
    import torch
    from tetmag_b200 import api, workloads

    world, rank, local = dist_env()
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    w = make_workload(args.workload, rank)
    ninst = workloads.instances(w)         # batched instances in the context (field evals per call)
    t0 = time.perf_counter()
    hier = args.bem != "dense"
    dense_ref = args.bem != "hmatrix-only"          # a dense matrix is on the device
    mo, ctx = workloads.setup_context(w, device=local, mixed=True, tol=args.tol, maxiter=100,
                                      hmatrix={"hmatrix": "mesh", "hmatrix-only": "mesh",
                                               "hmatrix-dense": True}.get(args.bem, False),
                                      keep_dense=dense_ref)
    bem_info = ctx.bem_info() if hier else None
    if hier:
        bem_info["verify"] = ctx.bem_verify()
    setup_s = time.perf_counter() - t0
    # one non-default stream for the library's kernels and the timing events
    stream = torch.cuda.Stream(dev)
    ctx.set_stream(stream.cuda_stream)
    torch.cuda.set_stream(stream)
    n = w.m0.size // 3          # state nodes (all instances)
    K, W = args.steps, args.warmup

    # W + K distinct states: the seeded initial state with seeded perturbations
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

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(mixed: bool, profile: bool, dense: bool = False):
        ctx.set_precision(mixed)
        if hier:
            ctx.set_bem_mode(not dense)
        for k in range(W):
            ctx.field_eval(S[k], ydot, hdem)
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        if profile:
            api.profile_enable(ctx, True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = api.kernel_launches()
        its = [0, 0]
        tag = f"timed_{'mixed' if mixed else 'fp64'}{'_dense' if dense else ''}{'_prof' if profile else ''}"
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
        barrier()
        ms = e0.elapsed_time(e1)
        launches = api.kernel_launches() - l0
        prof = api.profile_read(ctx) if profile else None
        if profile:
            api.profile_enable(ctx, False)
        return max_over_ranks(ms), launches, prof, its

    clocks = Clocks(local)
    clocks.start()
    ms_mx, launches, _, its_mx = timed(True, False)
    clk = clocks.stop()
    ms_64, _, _, its_64 = timed(False, False)
    ms_64d = timed(False, False, dense=True)[0] if hier and dense_ref else ms_64
    # per-kernel CUDA-event timing in a separate pass over the same K states (with the
    # profiler on, the PCG runs kernel by kernel instead of from CUDA graphs)
    _, _, prof, _ = timed(True, True)

    # relative error of the mixed path against the FP64 path, on one state
    # reference: plain FP64 with the dense BEM (the hierarchical one with hmatrix-only), solved to 1e-12
    probe = S[W + K - 1]
    ctx.set_precision(False)
    if hier and dense_ref:
        ctx.set_bem_mode(False)
    ctx.set_solver_params(1e-12, 300)
    h64 = hdem.clone()
    y64 = ctx.field_eval(probe, torch.empty_like(ydot), h64)
    if hier:
        ctx.set_bem_mode(True)
    h64h = hdem.clone()
    y64h = ctx.field_eval(probe, torch.empty_like(ydot), h64h)
    ctx.set_precision(True)
    ctx.set_solver_params(args.tol, 100)
    hmx = hdem.clone()
    ymx = ctx.field_eval(probe, torch.empty_like(ydot), hmx)
    torch.cuda.synchronize(dev)

    def relerr(a, b):
        return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))

    err_h, err_y = relerr(hmx, h64), relerr(ymx, y64)
    err_h64, err_y64 = relerr(h64h, h64), relerr(y64h, y64)

    # local right-hand side only (frozen demag), mixed
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for k in range(3):
        ctx.llg_rhs(0.0, S[k], ydot)
    e0.record(stream)
    nloc = 50
    for k in range(nloc):
        ctx.llg_rhs(0.0, S[k % (W + K)], ydot)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    local_per_s = ninst * nloc / (max_over_ranks(e0.elapsed_time(e1)) / 1e3)

    # end to end through the public API with host buffers (H2D of m from pinned host memory, D2H
    # of ydot into pinned host memory, per step)
    host_states = [torch.from_numpy(np.ascontiguousarray(st)).pin_memory() for st in states]
    yh = torch.empty(3 * n, dtype=torch.float64).pin_memory()
    for k in range(W):
        ctx.field_eval(host_states[k], yh)
    barrier()
    t = time.perf_counter()
    for k in range(K):
        ctx.field_eval(host_states[W + k], yh)
    e2e_s = max_over_ranks(time.perf_counter() - t)

    # simulated time: the frozen-demag relaxation loop (0.5 ps segments), mixed; one untimed
    # segment first (first-call allocations), then the best of three runs from the same state
    # (each run is tens of ms of wall clock with host polls between steps, so a single sample jitters)
    ctx.relax(S[0].clone(), duration_ps=0.5, segment_ps=0.5)
    sim_runs = []
    for _ in range(3):
        mrun = S[0].clone()
        torch.cuda.synchronize(dev)
        barrier()
        t = time.perf_counter()
        rs = ctx.relax(mrun, duration_ps=args.sim_ps, segment_ps=0.5)
        sim_runs.append(max_over_ranks(time.perf_counter() - t))
    sim_s = min(sim_runs)
    ns_per_hour = ninst * (args.sim_ps * 1e-3) / (sim_s / 3600.0)

    # batched workloads: the plain FP64 path one instance at a time (one single-mesh context per
    # instance, as the reference runs one mesh per process) on a sample of the instances
    unbatched = None
    if ninst > 1:
        if w.replicas > 1 or w.shared_bem:
            sample = [0]                 # identical meshes: one instance's rate
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
        per_inst_s = t_tot / n_ev          # mean time of one instance evaluation
        unbatched = {"value": 1.0 / per_inst_s, "unit": "instance field evals/s", "instances_sampled": len(sample),
                     "path": "plain FP64, one single-mesh context per instance, dense BEM, same CG tolerance"}

    value = world * ninst * K / (ms_mx / 1e3)
    fp64_value = world * ninst * K / (ms_64 / 1e3)
    peak, peak_kind = peak_hbm()
    kernels = ["local_llg", "divergence", "gradient", "bem_matvec", "cg_spmv"]
    dom = max(kernels, key=lambda k: prof[k]["total_ms"])
    d = prof[dom]
    avg_ms = d["total_ms"] / max(d["launches"], 1)
    achieved = d["bytes_per_launch"] / (avg_ms / 1e3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        key = w.name + ("/" + args.bem if hier else "")
        traffic = json.loads(tf.read_text()).get(key, {}).get(dom)
    kshare = {k: round(prof[k]["total_ms"] / ms_mx, 4) for k in prof if k != "demag_chain"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms_mx / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 operators / f64 vectors+reductions", "data": "synthetic",
        "config": {"workload": w.name, "nodes": n, "boundary_nodes": mo.nb, "nnz": mo.nnz, "instances": ninst,
                   "batched": (None if ninst == 1 else
                               ("interleaved replicas of one mesh: every operator row applied to all replicas "
                                "at once, the boundary product one GEMM (3xTF32 tensor cores on the mixed path)"
                                if w.replicas > 1 else
                                "replicas of one mesh sharing one BEM matrix (boundary matvec = one GEMM)"
                                if w.shared_bem else "uneven meshes, one BEM block each, one batched matvec")
                               + "; one CG and one step size for the batch; value counts instance evals"),
                   "bem": ("hierarchical (leaf 32, eta 2, ACA: FP32 terms to 1e-6 on the mixed path, FP64 "
                           "terms to 1e-7 on the plain path), " +
                           ("built from the mesh boundary" if args.bem in ("hmatrix", "hmatrix-only") else
                            "compressed from the device-assembled dense matrix")
                           if hier else "dense, device-assembled, FP32 on the mixed path"),
                   "precision": "mixed",
                   "cg_tol": args.tol, "states": "W+K distinct seeded perturbed states, warm-started solves",
                   "l2": "inputs larger than L2 (dense BEM alone is 4*Nb^2 bytes)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single"},
        "e2e": {"value": world * ninst * K / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 3 * n * 8,
                "d2h_bytes_per_step": 3 * n * 8},
        "gpu_launches": launches,
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "bytes_per_launch": d["bytes_per_launch"], "avg_ms": avg_ms},
        "clocks": clk,
        "fp64_value": fp64_value, "speedup_vs_fp64": value / fp64_value,
        "plain_fp64_unbatched": unbatched,
        "speedup_vs_plain_fp64_unbatched": (value / world / unbatched["value"]) if unbatched else None,
        "fp64_dense_value": world * ninst * K / (ms_64d / 1e3) if dense_ref else None,
        "speedup_vs_fp64_dense": ms_64d / ms_mx if dense_ref else None,
        "rel_err_vs_fp64": {"hdem": err_h, "ydot": err_y,
                            "reference": "FP64, " + ("dense" if dense_ref else "hierarchical") + " BEM, CG to 1e-12"},
        "rel_err_fp64_hier_vs_dense": {"hdem": err_h64, "ydot": err_y64} if dense_ref else None,
        "bem_info": bem_info,
        "bem_gemm": ctx.bem_gemm_info() if (w.shared_bem or w.replicas > 1) else None,
        "local_rhs_evals_per_s": world * local_per_s,
        "sim_ns_per_hour": world * ns_per_hour,
        "relax": {"sim_ps": args.sim_ps, "wall_s": sim_s, "steps": rs["accepted"], "rejected": rs["rejected"],
                  "rhs": rs["rhs"]},
        "cg_iters_per_eval": {"mixed": [i / K for i in its_mx], "fp64": [i / K for i in its_64]},
        "kernel_time_share": kshare,
        "kernels": {k: {"launches": prof[k]["launches"],
                        "avg_us": 1e3 * prof[k]["total_ms"] / max(prof[k]["launches"], 1),
                        "gbs": (prof[k]["bytes_per_launch"] / (prof[k]["total_ms"] / max(prof[k]["launches"], 1) / 1e3)
                                / 1e9) if prof[k]["total_ms"] > 0 and prof[k]["bytes_per_launch"] > 0 else None}
                    for k in kernels},
        "setup_s": setup_s,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ev, res, _ = cpu_baseline_sample(w, samples=1)
        line["cpu_baseline"] = {"value": 1.0 / res[0]["total_s"], "unit": UNIT, "cores": ev.threads,
                                "kind": "port", "sample": ev.describe(),
                                "components_s": {k: res[0][k] for k in
                                                 ("local_s", "div_grad_s", "solves_s", "bem_s")}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del ctx, mo
    if dist is not None:
        dist.destroy_process_group()


def run_adjoint(args):
    """c5: the interfacial-DMI disk integrated with fixed-step RK4 (full field at every stage) and
    the discrete adjoint of that map.  value = field evaluations / s of the mixed forward run;
    the adjoint's cost is reported as (forward + backward sweep time) / forward time."""
    import torch
    from tetmag_b200 import api, workloads
    from tetmag_b200.autograd import LLGObjective

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    nsteps = args.c5_steps
    w = workloads.c5_disk(nsteps=nsteps)
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
    # directional central differences of the mixed forward map
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
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": 1, "warmup": args.warmup,
        "ms_per_step": 1e3 * mx["forward_s"] / evals, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 operators / f64 vectors+reductions", "data": "synthetic",
        "config": {"workload": w.name, "nodes": n, "boundary_nodes": mo.nb, "nnz": mo.nnz, "dmi": "interfacial",
                   "steps": nsteps, "dt_ps": info["dt_ps"], "rk4_substeps": nsub, "checkpoint_every": ckpt,
                   "bz_samples": int(bz0.size), "objective": "volume-weighted mean m_z after the run",
                   "parameters": "per-node Ku (FP32 tensor, baseline 0, easy axis z) and the Bz(t) samples",
                   "cg_tol": args.tol, "parallelism": "single",
                   "timing": "host wall clock around synchronous library calls (one stream)"},
        "gpu_launches": mx["launches"],
        "clocks": clk,
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
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c5":
        run_adjoint(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
