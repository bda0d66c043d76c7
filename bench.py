#!/usr/bin/env python
"""LPs/sec to 1e-6 relative KKT on B200 (one JSON line on rank 0).

Default workload (refinery_learned): the parametric multi-site refinery planning
family (fixed 2000 x 8000 structure, 6 nnz/col, 256-dim parameter vector).  Set
up untimed: 20,000 training instances solved by the batched engine to 1e-8
relative KKT, the MLP 256 -> 1024 -> 1024 -> 10,001 trained on them on the
tensor cores.  Timed: 2,000 held-out instances solved to 1e-6 relative KKT by
(a) learned-warm mixed-precision batched PDHG (the value), (b) cold mixed
precision, (c) plain FP64 cold start -- same GPU, same instances.  A "step" is
one batched solve of all held-out instances; N GPUs run N replicas on their own
held-out seeds (weak scaling).

Other workloads: block_angular (single 204k x 1M LP), random_sparse (300 x 1000),
uneven_batch (4096 independent LPs), refinery (random-structure family, cold),
ill_conditioned (single 1M x 5M LP, 50M nonzeros, badly scaled; to 1e-8 by default,
each solve takes minutes: use --steps 1 --e2e-steps 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload refinery_learned|block_angular|uneven_batch|refinery|random_sparse|ill_conditioned]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# Iterations the FP64 Halpern engine needs to reach 1e-6 relative KKT on each
# single-LP workload (measured on B200).  The reference arm's LPs/sec
# extrapolates the reference CPU solver's per-iteration cost over this many
# iterations -- generous to the CPU: the reference's own vanilla PDHG needs far
# more iterations and never reaches 1e-6 on these LPs.
HALPERN_ITERS = {"block_angular": 6784, "random_sparse": 5056, "refinery_learned": 110744, "uneven_batch": 6379,
                 # mixed engine to 1e-8 (the FP64 leg of this workload was not run)
                 "ill_conditioned": 1230784}

METRIC = "LPs/sec to 1e-6 rel KKT"

# Copy bandwidth (STREAM-style) and sustained BF16 GEMM throughput (cuBLAS loop under the
# power cap) measured on B200 in an earlier run; the roofline denominators when no
# MEASURED_PEAKS.json sits beside this file.
EARLIER_PEAKS = {"hbm_gbs": 6558.7, "bf16_tflops_sustained": 1371.5}


def peaks():
    """(measured peaks, label of their source)."""
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        return json.loads(f.read_text()), "MEASURED_PEAKS.json (of measured)"
    return dict(EARLIER_PEAKS), "B200 copy / BF16 GEMM measured in an earlier run; MEASURED_PEAKS.json absent (of measured)"

# Seconds of each part of the refinery_learned run on one B200 (2,000 held-out
# instances; labels to 1e-8, legs to 1e-6 relative KKT with the answer's objective
# within 1e-6), used to plan the run's wall time from its leg counts.
LEARNED_LEG_S = {"start": 20.0, "label_per_instance": 0.0156, "epoch": 0.015, "warmup_step": 1.5,
                 "learned": 29.2, "mixed_cold": 30.3, "fp64_cold": 45.9, "e2e": 29.4, "cpu_sample": 12.0,
                 "single_lp": 0.6}


def metric_for(args):
    return f"LPs/sec to {args.eps:g} rel KKT"
METRIC_LEARNED = "LPs/sec to 1e-6 rel KKT: learned-warm mixed-prec PDHG vs plain FP64, one B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default 1 for refinery_learned, else 5)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="refinery_learned",
                    choices=["refinery_learned", "block_angular", "random_sparse", "uneven_batch", "refinery",
                             "ill_conditioned"])
    ap.add_argument("--train-count", type=int, default=20000, help="refinery_learned: training instances")
    ap.add_argument("--label-eps", type=float, default=1e-8, help="refinery_learned: label accuracy")
    ap.add_argument("--epochs", type=int, default=600, help="refinery_learned: MLP training epochs")
    ap.add_argument("--heldout", type=int, default=2000, help="refinery_learned: held-out instances per GPU")
    ap.add_argument("--batch-count", type=int, default=4096, help="instances of the batched workloads")
    ap.add_argument("--eps", type=float, default=None,
                    help="relative KKT tolerance (default 1e-8 for ill_conditioned, else 1e-6)")
    ap.add_argument("--eps-objective", type=float, default=1e-6,
                    help="an answer also needs its objective within this relative distance of the optimum (FP64 "
                         "bound on the device); 0 = relative KKT alone")
    ap.add_argument("--check-every", type=int, default=256,
                    help="refinery_learned: iterations between restart checks in every leg (measured on 2,000 "
                         "cold planning instances: 70.8 LPs/s at the library default 64, 75.1 at 128, 77.0 at "
                         "256 -- the checks cost less and the family needs slightly fewer iterations)")
    ap.add_argument("--compare-steps", type=int, default=1,
                    help="refinery_learned: steps of each comparison leg (cold mixed, cold FP64)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison leg")
    ap.add_argument("--single-sample", type=int, default=8,
                    help="refinery_learned: held-out instances solved one LP per solve by the single-LP FP64 "
                         "engine (the GPU without the batched engine); 0 skips that comparison")
    ap.add_argument("--time-limit", type=float, default=None,
                    help="single-LP workloads: seconds per solve before it stops as INTERRUPTED "
                         "(default 1200 for ill_conditioned, else none)")
    ap.add_argument("--e2e-steps", type=int, default=None,
                    help="end-to-end steps (default 1 for refinery_learned, else = --steps; 0 skips the e2e leg)")
    ap.add_argument("--cpu-sample-iters", type=int, default=20)
    ap.add_argument("--profile-scale", type=float, default=1.0,
                    help="--profile with ill_conditioned: rows and columns scaled by this factor (0.4 keeps each "
                         "matrix orientation above L2 while the device holds a few GB)")
    ap.add_argument("--profile", action="store_true",
                    help="profiling case: one short solve, then the two iteration kernels once each inside the "
                         "NVTX range 'kernel_timing' (for ncu --nvtx-include kernel_timing/)")
    a = ap.parse_args()
    if a.steps is None:
        a.steps = 1 if a.workload in ("refinery_learned", "ill_conditioned") else 5
    if a.eps is None:
        a.eps = 1e-8 if a.workload == "ill_conditioned" else 1e-6
    if a.time_limit is None:
        a.time_limit = 1200.0 if a.workload == "ill_conditioned" else 0.0
    if a.e2e_steps is None:
        a.e2e_steps = 1 if a.workload == "refinery_learned" else a.steps
    return a


def profile_learned(args):
    """Profiling case of refinery_learned (for ncu, NVTX range 'timed'): a small
    training run (1024 labels to 1e-6, 20 epochs), then the three legs on 1024
    held-out instances capped at 100k iterations -- per-instance vectors of the
    held-out batch (~240 MB) exceed L2 like the full workload's."""
    import torch
    torch.cuda.set_device(0)
    torch.cuda.set_stream(torch.cuda.Stream())
    b2p, fam, _ = learned_setup(args, 0)
    P = fam.sample_params(1024, seed=20001)
    with b2p.Context(0) as ctx:
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        ws = b2p.warmstart.LearnedWarmStart(ctx, fam)
        ws.fit(n_train=1024, label_eps=1e-6, epochs=20, max_iterations=100000)
        b2p.warmstart.upload_family(ctx, fam, P)
        F = P.astype(np.float32)
        stop = dict(eps=args.eps, eps_objective=args.eps_objective, check_every=args.check_every)
        legs = {
            "learned": lambda it: ctx.batch_solve_learned(F, precision="fp32", max_iterations=it, outputs=False,
                                                          **stop),
            "mixed_cold": lambda it: ctx.batch_solve(precision="fp32", max_iterations=it, outputs=False, **stop),
            "fp64_cold": lambda it: ctx.batch_solve(precision="fp64", max_iterations=it, outputs=False, **stop),
        }
        for fn in legs.values():
            fn(2048)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("timed")
        out = {}
        for name, fn in legs.items():
            summ, per, _, _ = fn(100000)
            out[name] = {"kernel_ms": summ["kernel_time_ms"], "iterations_mean": float(per["iterations"].mean()),
                         "instance_iterations": int(per["iterations"].sum()), "launches": summ["kernel_launches"]}
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps(out), flush=True)


def profile_case(args):
    import torch
    torch.cuda.set_device(0)
    torch.cuda.set_stream(torch.cuda.Stream())
    b2p, lp, _ = make_lp(args.workload, args.profile_scale)
    with b2p.Context(0) as ctx:
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        ctx.upload(lp.standard())
        for prec in ("fp32", "fp64"):
            ctx.solve(engine="halpern", precision=prec, eps=args.eps, max_iterations=256)
            torch.cuda.nvtx.range_push("kernel_timing")
            kt = ctx.kernel_timing(reps=1, engine="halpern", precision=prec, eps=args.eps)
            torch.cuda.nvtx.range_pop()
            print(json.dumps({"precision": prec, **kt}), flush=True)


def make_lp(workload, scale=1.0):
    import __graft_entry__ as g
    b2p = g.load_package()
    if workload == "block_angular":
        lp = b2p.lpgen.block_angular()
        cfg = {"workload": "block_angular_multiperiod_blending", "m": lp.m, "n": lp.n, "nnz": lp.nnz,
               "periods": 50, "block": "4000x20000", "nnz_per_col": 8, "link_rows": 4000, "seed": 1}
    elif workload == "ill_conditioned":
        lp = b2p.lpgen.ill_conditioned(m=int(round(1_000_000 * scale)), n=int(round(5_000_000 * scale)))
        cfg = {"workload": "ill_conditioned_stress", "m": lp.m, "n": lp.n, "nnz": lp.nnz, "nnz_per_col": 10,
               "row_scales": "10^U(-4,4)", "col_scales": "10^U(-3,3)", "box": "[0, 10^U(0,3)]", "seed": 4}
    else:
        lp = b2p.lpgen.random_sparse()
        cfg = {"workload": "random_sparse_300x1000", "m": lp.m, "n": lp.n, "nnz": lp.nnz, "seed": 0}
    return b2p, lp, cfg


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="b2p_clocks_", suffix=".csv")
        os.close(fd)
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(v, world, op):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(v, world):
    """Slowest rank's time: the whole job's time (one scalar all-reduce)."""
    import torch.distributed as dist
    return _reduce(v, world, dist.ReduceOp.MAX if world > 1 else None)


def sum_over_ranks(v, world):
    import torch.distributed as dist
    return _reduce(v, world, dist.ReduceOp.SUM if world > 1 else None)


def timed_solves(ctx, torch, steps, world, **params):
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    results = []
    for _ in range(steps):
        res, _, _ = ctx.solve(**params)
        results.append(res)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1)
    return ms, results


def cpu_reference_sample(lp, sample_iters, iters_needed):
    """Reference CPUFirstOrderSolver (compiled from the reference sources) on this host:
    setup time from a 1-iteration run, per-iteration time from the difference to a run
    of 1 + k iterations, k starting at `sample_iters` and doubled until that difference
    is at least 50 ms (timer noise would otherwise dominate on small LPs); LPs/sec
    extrapolated over `iters_needed` iterations.  Falls back to the oracle's C port if
    the reference library is absent."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_lib import REF_DIR, OracleLib, RefLib  # oracle: CPU baseline leg only
    if (REF_DIR / "libbharatopt_ref.so").exists():
        ref = RefLib()
        kind = "reference"

        def run(iters):
            r = ref.fo_solve(lp, max_iterations=iters)
            return r["solve_time_ms"] / 1e3, int(r.get("iterations", iters)), r["status"]
    else:
        orc = OracleLib()
        std = lp.standard()
        kind = "port"

        def run(iters):
            t = time.perf_counter()
            orc.ref_pdhg(std, max_iterations=iters)
            return time.perf_counter() - t, iters, "MAX_ITERATIONS"
    t0 = time.perf_counter()
    setup, _, _ = run(1)
    k = max(1, sample_iters)
    while True:
        t_k, it_k, status = run(1 + k)
        ran = max(1, it_k - 1)  # the reference may stop early
        diff = t_k - setup
        if diff >= 0.05 or ran < k or k >= (1 << 22):
            break
        k *= 2
    per_iter = max(diff, 1e-9) / ran
    wall = time.perf_counter() - t0
    seconds = setup + per_iter * iters_needed
    return {"value": 1.0 / seconds, "unit": "LPs/s", "cores": 1, "kind": kind,
            "sample": (f"reference CPUFirstOrderSolver, 1 thread: runs of 1 and {1 + ran} PDHG iterations "
                       f"on the same LP ({wall:.1f} s wall; setup {setup:.3f} s incl. validate+presolve+CSR, "
                       f"{per_iter * 1e3:.4f} ms/iteration, status {status}); LPs/s = 1/(setup + {iters_needed} x "
                       f"per-iteration), {iters_needed} = iterations the GPU engine needs to the benchmark's "
                       f"tolerance; the reference's own PDHG does not reach it on this LP"),
            "per_iteration_ms": per_iter * 1e3, "setup_s": setup}


def _batch_ref_worker(task):
    """One bounded reference CPUFirstOrderSolver sample on instance i of a batched workload."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_lib import RefLib  # oracle: reference arm only
    workload, count, i, sample = task
    args = argparse.Namespace(workload=workload, batch_count=count)
    _, lps, _, _, _ = batch_lps(args)
    ref = RefLib()
    r1 = ref.fo_solve(lps[i], max_iterations=1)
    r2 = ref.fo_solve(lps[i], max_iterations=1 + sample)
    ran = max(1, int(r2.get("iterations", 1 + sample)) - 1)
    return r1["solve_time_ms"] / 1e3, (r2["solve_time_ms"] - r1["solve_time_ms"]) / ran / 1e3


def run_reference_batch(args):
    """Reference arm of the batched workloads: the reference's CPU PDHG on the workload's
    instances, one per host core in parallel; per-LP time = setup + per-iteration cost x the
    iterations the FP64 engine needs (an extrapolation: the reference's own vanilla PDHG has
    no relative-KKT stop and does not reach the tolerance on these LPs)."""
    import multiprocessing as mp
    _, lps, stds, _, cfg = batch_lps(args)
    cores = os.cpu_count() or 1
    iters = HALPERN_ITERS.get(args.workload, 6207)
    sample = 4000
    vals = []
    t0 = time.perf_counter()
    stride = max(1, len(lps) // (cores * max(1, args.steps)))
    with mp.get_context("spawn").Pool(cores) as pool:
        pool.map(_batch_ref_worker, [(args.workload, args.batch_count, 0, 10)] * cores)  # warm-up
        for step in range(args.steps):
            idx = [((step * cores + c) * stride) % len(lps) for c in range(cores)]
            out = pool.map(_batch_ref_worker, [(args.workload, args.batch_count, i, sample) for i in idx])
            per_lp = [a + b * iters for a, b in out]
            vals.append(len(out) / max(per_lp))
    wall = time.perf_counter() - t0
    v = statistics.median(vals)
    cb = {"value": v, "unit": "LPs/s", "cores": cores, "kind": "reference",
          "sample": (f"reference CPUFirstOrderSolver, {cores} processes x 1 instance each: runs of 1 and {1 + sample} "
                     f"iterations; per-LP time = setup + {iters} x per-iteration; {wall:.1f} s wall"),
          "extrapolation": {"iterations": iters, "source": "mean iterations of this engine's plain FP64 solve of the "
                            "workload (a different algorithm: restarted Halpern PDHG with scaling)"}}
    line = {"metric": metric_for(args), "value": v, "unit": "LPs/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, no dataset)", "config": cfg,
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "LPs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    _, lp, cfg = make_lp(args.workload)
    iters = HALPERN_ITERS.get(args.workload, 5000)
    for _ in range(args.warmup):  # untimed warm-up samples
        cpu_reference_sample(lp, max(1, args.cpu_sample_iters // 4), iters)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cb = cpu_reference_sample(lp, args.cpu_sample_iters, iters)
        vals.append(cb)
    wall = time.perf_counter() - t0
    v = statistics.median([c["value"] for c in vals])
    cb = dict(vals[-1])
    cb["value"] = v
    line = {"metric": metric_for(args), "value": v, "unit": "LPs/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, no dataset)",
            "config": cfg, "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "LPs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


def batch_lps(args, seed_offset=0):
    """(standard-form instances, shared matrix or None, config) of a batched workload."""
    import __graft_entry__ as g
    b2p = g.load_package()
    if args.workload == "uneven_batch":
        lps = b2p.lpgen.uneven_batch(args.batch_count, seed=2 + seed_offset)
        stds = [lp.standard() for lp in lps]
        cfg = {"workload": "uneven_batch", "count": len(stds), "m": "logU(50,2000)", "n": "m*U(2,5)",
               "nnz_per_col": "4-10", "seed": 2, "nnz_total": int(sum(s.nnz for s in stds))}
        return b2p, lps, stds, None, cfg
    fam = b2p.lpgen.RefineryFamily()
    p = fam.sample_params(args.batch_count, seed=20001 + seed_offset)
    lps = [fam.instance(q) for q in p]
    stds = [lp.standard() for lp in lps]
    cfg = {"workload": "refinery_family_cold", "count": len(stds), "m": fam.m, "n": fam.n,
           "nnz": int(fam.rowptr[-1]), "shared_matrix": True, "seed": 3}
    return b2p, lps, stds, stds[0], cfg


def upload_batch(ctx, stds, shared):
    if shared is not None:
        mats = [(shared.m, shared.n, shared.rowptr, shared.colidx, shared.vals)]
        inst = np.zeros(len(stds), np.int32)
    else:
        mats = [(s.m, s.n, s.rowptr, s.colidx, s.vals) for s in stds]
        inst = np.arange(len(stds), dtype=np.int32)
    ctx.batch_upload(mats, inst, np.concatenate([s.b for s in stds]), np.concatenate([s.c for s in stds]),
                     np.concatenate([s.lb for s in stds]), np.concatenate([s.ub for s in stds]),
                     np.concatenate([s.is_eq for s in stds]))


def run_batch_workload(args):
    """The uneven batch (4096 LPs of uneven size, each its own matrix) or the
    random-structure refinery family (one shared matrix), cold start: mixed precision
    timed for --steps, plain FP64 for --compare-steps, end to end for --e2e-steps; one
    replica per GPU on its own seed (weak scaling)."""
    import torch
    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    torch.cuda.set_stream(torch.cuda.Stream())
    b2p, lps, stds, shared, cfg = batch_lps(args, seed_offset=1000 * rank)
    ctx = b2p.Context(local)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    upload_batch(ctx, stds, shared)
    stop = dict(eps=args.eps, eps_objective=args.eps_objective)
    cap = 400000
    for _ in range(args.warmup):
        for prec in ("fp32", "fp64"):
            ctx.batch_solve(precision=prec, max_iterations=2048, outputs=False, **stop)
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    res, clocks = {}, None
    for prec, k in (("fp32", args.steps), ("fp64", args.compare_steps)):
        if k <= 0:
            continue
        sampler = ClockSampler(uuid) if prec == "fp32" else None
        if sampler:
            sampler.start()
        ms, (summ, per, _, _) = timed_leg(ctx, torch, world, k,
                                          lambda: ctx.batch_solve(precision=prec, max_iterations=cap, outputs=False,
                                                                  **stop))
        if sampler:
            clocks = sampler.stop()
        solved = sum_over_ranks(float((per["status"] == 0).sum()), world)
        res[prec] = {"value": solved * k / (ms / 1e3), "unit": "LPs/s", "steps": k, "ms_per_step": ms / k,
                     "solved": int(solved), "instances": len(stds) * world,
                     "iterations_mean": float(per["iterations"].mean()), "iterations_max": int(per["iterations"].max()),
                     "worst_rel_kkt": float(per["rel_kkt"].max()), "kernel_ms": summ["kernel_time_ms"],
                     "kernel_launches": summ["kernel_launches"], "tuned_threads_chunk": summ["step_size"],
                     "trace": trace_summary(*ctx.batch_trace(), len(stds))}
        if prec == "fp32":
            it_total = float(per["iterations"].sum())
            per_inst_iters = per["iterations"].astype(float)
            kern_ms = summ["kernel_time_ms"]
            launches = int(summ["kernel_launches"]) * k
    # end to end: pinned host instance data -> batch upload -> mixed solve -> x, y to host
    pin = {k: torch.from_numpy(np.ascontiguousarray(np.concatenate([getattr(s_, k) for s_ in stds]))).pin_memory()
           for k in ("b", "c", "lb", "ub", "is_eq")}
    h2d = sum(t.numel() * t.element_size() for t in pin.values())
    mats = ([(shared.m, shared.n, shared.rowptr, shared.colidx, shared.vals)] if shared is not None
            else [(s_.m, s_.n, s_.rowptr, s_.colidx, s_.vals) for s_ in stds])
    h2d += sum(q[2].nbytes + q[3].nbytes + q[4].nbytes for q in mats)
    inst = np.zeros(len(stds), np.int32) if shared is not None else np.arange(len(stds), dtype=np.int32)
    d2h = 8 * sum(s_.n + s_.m for s_ in stds)

    def e2e_step():
        ctx.batch_upload(mats, inst, pin["b"].numpy(), pin["c"].numpy(), pin["lb"].numpy(), pin["ub"].numpy(),
                         pin["is_eq"].numpy())
        return ctx.batch_solve(precision="fp32", max_iterations=cap, **stop)

    e2e = {"value": None, "skipped": "--e2e-steps 0", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
    if args.e2e_steps > 0:
        e2e_ms, (_, eper, _, _) = timed_leg(ctx, torch, world, args.e2e_steps, e2e_step)
        esolved = sum_over_ranks(float((eper["status"] == 0).sum()), world)
        e2e = {"value": esolved * args.e2e_steps / (e2e_ms / 1e3), "unit": "LPs/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": args.e2e_steps, "ms_per_step": e2e_ms / args.e2e_steps,
               "solved": int(esolved)}
    # roofline of k_batch_chunk<float>: algorithmic bytes of every instance-iteration (12 B per
    # nonzero, 24 B per column, 16 B per row) over its kernel time; the bound is HBM when the
    # matrices and vectors the resident instances stream exceed L2, else L2
    per_iter = np.array([12.0 * s_.nnz + 24.0 * s_.n + 16.0 * s_.m for s_ in stds])
    alg = float((per_inst_iters * per_iter).sum())
    pk, pk_src = peaks()
    peak = pk["hbm_gbs"]
    achieved = alg / (kern_ms / 1e3) / 1e9
    resident = 2 * 148  # two CTAs per SM, one instance each
    vec = np.array([24.0 * s_.n + 16.0 * s_.m for s_ in stds])
    mat = np.array([12.0 * s_.nnz for s_ in stds])
    top = np.argsort(-(vec + mat))[:resident]
    hot = float(vec[top].sum() + (mat[0] if shared is not None else mat[top].sum()))
    bound = "hbm" if hot > 126e6 else "l2"
    roofline = {"bound": bound, "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": "k_batch_chunk<float>",
                "algorithmic_bytes_per_instance_iteration_mean": float(per_iter.mean()),
                "resident_working_set_bytes": hot, "peak_source": "hbm_gbs: " + pk_src}
    cpu = None
    if rank == 0 and world == 1 and "fp64" in res:
        cpu = cpu_reference_sample(lps[0], 2000, int(res["fp64"]["iterations_mean"]))
    if rank == 0:
        line = {"metric": metric_for(args), "value": res["fp32"]["value"], "unit": "LPs/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["fp32"]["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 (SpMV, vectors) + f64 (scaling, KKT, re-centring)",
                "data": "synthetic (seeded generator, no dataset)",
                "config": dict(cfg, parallelism=f"replicas x{world}", eps_rel_kkt=args.eps,
                               eps_objective=args.eps_objective,
                               steps={"mixed (value)": args.steps, "fp64": args.compare_steps, "e2e": args.e2e_steps}),
                "mixed": res["fp32"], "fp64": res.get("fp64"), "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu,
                "gpu_launches": launches, "clocks": clocks}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def learned_setup(args, rank):
    """Family, trained warm-start model and held-out parameter vectors of this rank."""
    import __graft_entry__ as g
    b2p = g.load_package()
    fam = b2p.lpgen.RefineryPlanningFamily()
    P = fam.sample_params(args.heldout, seed=20001 + 1000 * rank)
    return b2p, fam, P


def learned_cfg(args, fam, world):
    return {"workload": "refinery_planning_learned_warm_start", "m": fam.m, "n": fam.n, "nnz": int(fam.rowptr[-1]),
            "params": fam.N_PARAM, "train_instances": args.train_count, "label_eps": args.label_eps,
            "heldout_instances": args.heldout, "mlp": f"{fam.N_PARAM}->1024->1024->{fam.n + fam.m + 1} GELU bf16/fp32acc",
            "epochs": args.epochs, "eps_rel_kkt": args.eps, "eps_objective": args.eps_objective,
            "shared_matrix": True, "family_seed": 3,
            "heldout_seed": 20001, "parallelism": f"replicas x{world}",
            "l2": "per-instance vectors of 2000 instances (~300 MB) exceed L2; the shared matrix is L2-resident",
            "warmup": "warm-up steps run the same solves capped at 2048 iterations (autotuning, graphs, allocations)",
            "steps": {"learned (value)": args.steps, "mixed_cold": args.compare_steps, "fp64_cold": args.compare_steps,
                      "e2e": args.e2e_steps, "fp64_single_lp (instances)": args.single_sample},
            "mlp_training": "batch 1024, Adam lr 2e-3 -> 2e-5 cosine", "check_every": args.check_every}


def timed_leg(ctx, torch, world, steps, fn):
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    out = None
    for _ in range(steps):
        out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    return max_over_ranks(e0.elapsed_time(e1), world), out


def planned_wall_s(args):
    """Planned wall time (s) of the refinery_learned run from its leg counts and the
    per-leg times measured on one B200 (LEARNED_LEG_S): untimed labels and training,
    warm-up solves, the value leg x --steps, the comparison legs x --compare-steps,
    the e2e leg x --e2e-steps and the CPU sample."""
    t = LEARNED_LEG_S
    scale = args.heldout / 2000.0
    return (t["start"] + t["label_per_instance"] * args.train_count + t["epoch"] * args.epochs
            + args.warmup * t["warmup_step"]
            + scale * (args.steps * t["learned"] + args.compare_steps * (t["mixed_cold"] + t["fp64_cold"])
                       + args.e2e_steps * t["e2e"])
            + args.single_sample * t["single_lp"] + t["cpu_sample"])


def run_learned_workload(args):
    import torch
    t_wall0 = time.perf_counter()
    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    torch.cuda.set_stream(torch.cuda.Stream())  # CUDA graphs need a non-default stream
    b2p, fam, P = learned_setup(args, rank)
    ctx = b2p.Context(local)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    plan = planned_wall_s(args)
    if rank == 0:
        print(f"[bench] planned wall time {plan:.0f} s", file=sys.stderr, flush=True)
    ws = b2p.warmstart.LearnedWarmStart(ctx, fam)
    fit = ws.fit(n_train=args.train_count, label_eps=args.label_eps, epochs=args.epochs)
    s0 = b2p.warmstart.upload_family(ctx, fam, P)
    F = P.astype(np.float32)
    # every leg stops on the same rule: relative KKT <= eps and the answer's objective
    # within eps_objective of the optimum (FP64 bound evaluated on the device)
    stop = dict(eps=args.eps, eps_objective=args.eps_objective, check_every=args.check_every)
    cap = 400000
    legs = {
        "learned": lambda it: ctx.batch_solve_learned(F, fallback=True, precision="fp32", max_iterations=it,
                                                      outputs=False, **stop),
        "mixed_cold": lambda it: ctx.batch_solve(precision="fp32", max_iterations=it, outputs=False, **stop),
        "fp64_cold": lambda it: ctx.batch_solve(precision="fp64", max_iterations=it, outputs=False, **stop),
    }
    for _ in range(args.warmup):
        for fn in legs.values():
            fn(2048)
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    res = {}
    clocks = None
    steps_of = {"learned": args.steps, "mixed_cold": args.compare_steps, "fp64_cold": args.compare_steps}
    for name, fn in legs.items():
        k = steps_of[name]
        if k <= 0:
            continue
        sampler = ClockSampler(uuid) if name == "learned" else None
        if sampler:
            sampler.start()
        ms, (summ, per, _, _) = timed_leg(ctx, torch, world, k, lambda: fn(cap))
        if sampler:
            clocks = sampler.stop()
        objs = ctx.batch_objectives()
        ok = per["status"] == 0
        solved = sum_over_ranks(float(ok.sum()), world)
        res[name] = {"value": solved * k / (ms / 1e3), "unit": "LPs/s", "steps": k, "ms_per_step": ms / k,
                     "solved": int(solved), "instances": args.heldout * world,
                     "iterations_mean": float(per["iterations"].mean()),
                     "iterations_max": int(per["iterations"].max()), "worst_rel_kkt": float(per["rel_kkt"].max()),
                     "worst_obj_err_solved": float(objs["obj_err"][ok].max()) if ok.any() else None,
                     "statuses": {str(v): int((per["status"] == v).sum()) for v in np.unique(per["status"])},
                     "kernel_ms": summ["kernel_time_ms"], "kernel_launches": summ["kernel_launches"]}
        if name in ("learned", "fp64_cold"):
            res[name]["trace"] = trace_summary(*ctx.batch_trace(), args.heldout)
        if name == "learned":
            res[name]["fallbacks"] = summ["fallbacks"]
            res[name]["warm_used"] = int(per["warm_used"].sum())
            launches = int(summ["kernel_launches"]) * k
            it_total = float(per["iterations"].sum())
            kern_ms = summ["kernel_time_ms"]
            ni = max(1, int(round(summ["used_average"])) // 10)  # instances per CTA of the tuned shape
    # end to end through the public API: pinned host parameter vectors and instance
    # data -> upload -> learned solve -> answers to host
    _, B, Cc, LB, UB, EQ = fam.standard_batch(P)
    pin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory()
           for k, v in (("b", B.ravel()), ("c", Cc.ravel()), ("lb", LB.ravel()), ("ub", UB.ravel()),
                        ("is_eq", EQ.ravel().astype(np.uint8)), ("f", F))}
    h2d = sum(t.numel() * t.element_size() for t in pin.values())
    d2h = 8 * args.heldout * (fam.n + fam.m)

    def e2e_step():
        ctx.batch_upload([(s0.m, s0.n, s0.rowptr, s0.colidx, s0.vals)], np.zeros(args.heldout, np.int32),
                         pin["b"].numpy(), pin["c"].numpy(), pin["lb"].numpy(), pin["ub"].numpy(), pin["is_eq"].numpy())
        return ctx.batch_solve_learned(pin["f"].numpy(), fallback=True, precision="fp32", max_iterations=cap, **stop)

    e2e = {"value": None, "skipped": "--e2e-steps 0", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
    if args.e2e_steps > 0:
        e2e_ms, (esumm, eper, ex, ey) = timed_leg(ctx, torch, world, args.e2e_steps, e2e_step)
        esolved = sum_over_ranks(float((eper["status"] == 0).sum()), world)
        e2e = {"value": esolved * args.e2e_steps / (e2e_ms / 1e3), "unit": "LPs/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": args.e2e_steps, "ms_per_step": e2e_ms / args.e2e_steps,
               "solved": int(esolved),
               "note": "batch upload (host CSR checks, renumbering, device transpose, scaling) + learned solve + x, y"}
    # plain FP64 cold-start PDHG one LP per solve -- the single-LP engine on the same GPU, the
    # held-out instances one after another -- on the first --single-sample instances: what the
    # GPU gives without the batched engine (each solve timed with CUDA events on the stream)
    single = None
    if args.single_sample > 0:
        cnt = min(args.single_sample, args.heldout)
        tot_ms, ok1, its1 = 0.0, 0, []
        stream = torch.cuda.current_stream()
        for i in range(cnt):
            ctx.upload(b2p.lpgen.StdLP(s0.m, s0.n, s0.rowptr, s0.colidx, s0.vals, B[i], Cc[i], LB[i], UB[i], EQ[i]))
            if i == 0:  # autotune the single-LP kernels for this shape outside the timing
                ctx.solve(engine="halpern", precision="fp64", max_iterations=2048, **stop)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            r1, _, _ = ctx.solve(engine="halpern", precision="fp64", max_iterations=cap, **stop)
            e1.record(stream)
            torch.cuda.synchronize()
            tot_ms += e0.elapsed_time(e1)
            ok1 += int(r1["status"] == "OPTIMAL")
            its1.append(r1["iterations"])
        lps = sum_over_ranks(ok1 / (max_over_ranks(tot_ms, world) / 1e3), world)
        single = {"value": lps, "unit": "LPs/s", "instances": cnt, "solved": ok1, "ms_per_lp": tot_ms / cnt,
                  "iterations_mean": float(np.mean(its1)),
                  "engine": "single-LP Halpern engine, FP64, cold start, one LP per solve (same stop rule)"}
    # roofline of the dominant kernel (the batched chunk kernel of the tuned shape):
    # algorithmic bytes of every instance-iteration of the value leg over its kernel time --
    # the SELL matrix (12 B per nonzero, both orientations) once per CTA-iteration, so once
    # per ni instances, plus each instance's vectors.  The shared matrix and the vectors are
    # served from L2 and shared memory, so the bound that applies is the on-chip one; the
    # DRAM share comes from the committed ncu capture.
    nnz = int(fam.rowptr[-1])
    per_iter = 12 * nnz / ni + 24 * fam.n + 16 * fam.m
    pk, pk_src = peaks()
    peak = pk["hbm_gbs"]
    achieved = it_total * per_iter / (kern_ms / 1e3) / 1e9
    kname = "k_batch_pair" if ni == 2 else "k_batch_chunk"
    prof = read_profile(ROOT / "profiles" / f"{kname[2:]}_refinery_planning.txt")
    roofline = {"bound": "l2", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": prof.get("dram_bytes_per_instance_iteration"),
                "traffic_unit": "DRAM bytes per instance-iteration (ncu dram__bytes_read.sum + write.sum)",
                "dram_frac": (prof["dram_bytes_per_instance_iteration"] / per_iter
                              if "dram_bytes_per_instance_iteration" in prof else None),
                "l2_bytes_per_instance_iteration": prof.get("l2_bytes_per_instance_iteration"),
                "lts_throughput_pct": prof.get("lts_throughput_pct"),
                "kernel": f"{kname}<float> (SELL, {ni} instance(s) per CTA, learned leg)",
                "algorithmic_bytes_per_instance_iteration": per_iter,
                "peak_source": "hbm_gbs: " + pk_src + "; no measured L2 peak exists, so the fraction is against HBM",
                "note": f"12 B per nonzero (FP32 value + 16-bit index, both orientations) shared by the {ni} "
                        "instance(s) of a CTA, 24 B per column, 16 B per row; bound 'l2': the shared matrix and "
                        "the instances' vectors stay in L2 / shared memory (ncu: DRAM carries dram_frac of these "
                        "bytes)"}
    # training on the tensor cores: GEMM FLOPs of all epochs (per sample: layer 1 forward +
    # weight gradient, layers 2 and 3 forward + weight gradient + input gradient) over the
    # training time, against the sustained BF16 peak
    hid, outp = 1024, (fam.n + fam.m + 1 + 7) // 8 * 8
    flop = (4.0 * fam.N_PARAM * hid + 6.0 * hid * hid + 6.0 * hid * outp) * args.train_count * args.epochs
    bf16 = pk.get("bf16_tflops_sustained") or pk.get("bf16_tflops")
    fit["train_tflops"] = flop / max(fit["train_s"], 1e-9) / 1e12
    fit["train_frac_of_bf16_sustained"] = fit["train_tflops"] / bf16
    fit["train_peak_source"] = "bf16_tflops_sustained: " + pk_src
    fit["train_flop"] = flop
    cpu = None
    if rank == 0 and world == 1:
        lp0 = fam.instance(P[0])
        # ~10 s of one host core: 120k reference iterations on a held-out instance
        cpu = cpu_reference_sample(lp0, 120000, int(res["fp64_cold"]["iterations_mean"])
                                   if "fp64_cold" in res else HALPERN_ITERS["refinery_learned"])
    if rank == 0:
        ratio = (res["learned"]["value"] / res["fp64_cold"]["value"]) if "fp64_cold" in res else None
        ratio1 = (res["learned"]["value"] / single["value"]) if single and single["value"] > 0 else None
        line = {"metric": METRIC_LEARNED, "value": res["learned"]["value"], "unit": "LPs/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["learned"]["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 (SpMV, vectors) + f64 (scaling, KKT, re-centring); bf16 MLP",
                "data": "synthetic (seeded refinery planning family, no dataset)",
                "config": learned_cfg(args, fam, world), "learned_vs_fp64_cold": ratio,
                "learned_vs_fp64_single_lp": ratio1,
                "stop_rule": {"eps_rel_kkt": args.eps, "eps_objective": args.eps_objective,
                          "counted": "status OPTIMAL: FP64 relative KKT <= eps on the original instance and the "
                                     "FP64 objective-error bound <= eps_objective, both on the device"},
                "learned": res["learned"], "mixed_cold": res.get("mixed_cold"), "fp64_cold": res.get("fp64_cold"),
                "fp64_single_lp": single,
                "training": fit, "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": launches,
                "clocks": clocks, "wall_s": time.perf_counter() - t_wall0, "planned_wall_s": plan}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def trace_summary(t_ms, active, count, sm_count=148):
    """Where the time of one batched solve goes, from its active-instance trace: the
    time by which 50 / 90 / 99 / 100 % of the instances had finished, and the share of
    the solve spent with fewer active instances than SMs (the tail, where most SMs idle)."""
    t = np.asarray(t_ms, float)
    a = np.asarray(active, float)
    out = {"points": int(len(t)), "total_ms": float(t[-1]) if len(t) else 0.0}
    for q in (50, 90, 99, 100):
        left = count * (1 - q / 100.0)
        hit = np.nonzero(a <= left)[0]
        out[f"t{q}_ms"] = float(t[hit[0]]) if len(hit) else None
    if len(t) > 1 and t[-1] > 0:
        dt = np.diff(t)
        out["tail_share"] = float(dt[a[:-1] < sm_count].sum() / t[-1])
    return out


def read_profile(path):
    """`name: value` lines of a committed ncu summary (numbers only)."""
    out = {}
    if path.exists():
        for ln in path.read_text().splitlines():
            if ":" in ln:
                k, v = ln.split(":", 1)
                try:
                    out[k.strip()] = float(v.split()[0])
                except (ValueError, IndexError):
                    pass
    return out


def _ref_worker(q):
    """One bounded reference CPUFirstOrderSolver sample on the instance of parameter vector q."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import __graft_entry__ as g
    from oracle_lib import RefLib  # oracle: reference arm only
    b2p = g.load_package()
    fam = b2p.lpgen.RefineryPlanningFamily()
    lp = fam.instance(q)
    ref = RefLib()
    r1 = ref.fo_solve(lp, max_iterations=1)
    r2 = ref.fo_solve(lp, max_iterations=1 + _ref_worker.sample)
    ran = max(1, int(r2.get("iterations", 1 + _ref_worker.sample)) - 1)
    return r1["solve_time_ms"] / 1e3, (r2["solve_time_ms"] - r1["solve_time_ms"]) / ran / 1e3


_ref_worker.sample = 20000  # ~2 s of one core per sample


def run_reference_learned(args):
    """Reference arm of refinery_learned: the reference's CPU PDHG on held-out instances,
    one instance per host core in parallel; per-LP time = setup + per-iteration cost x
    the iterations the FP64 engine needs (the reference's own PDHG has no 1e-6 stop
    rule and does not reach it; extrapolating is generous to the CPU)."""
    import multiprocessing as mp
    _, fam, P = learned_setup(args, 0)
    cores = os.cpu_count() or 1
    iters = HALPERN_ITERS["refinery_learned"]
    vals = []
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(cores) as pool:
        pool.map(_ref_worker, list(P[:cores]))  # warm-up (loads, page-in)
        for step in range(args.steps):
            out = pool.map(_ref_worker, list(P[(step * cores) % len(P):][:cores]))
            per_lp = [s + it * iters for s, it in out]
            vals.append(len(out) / max(per_lp))
    wall = time.perf_counter() - t0
    v = statistics.median(vals)
    cb = {"value": v, "unit": "LPs/s", "cores": cores, "kind": "reference", "extrapolated": True,
          "sample": (f"reference CPUFirstOrderSolver (compiled from its sources), {cores} processes x 1 held-out "
                     f"instance each: runs of 1 and {1 + _ref_worker.sample} iterations; per-LP time = setup + "
                     f"{iters} x per-iteration; {wall:.1f} s wall"),
          "extrapolation": (f"the reference's plain PDHG does not reach 1e-6 relative KKT on these LPs (it stops at "
                            f"its iteration limit); its measured per-iteration cost is multiplied by {iters}, the "
                            f"mean iteration count of the B200 FP64 Halpern engine (a different, restarted "
                            f"algorithm) on the 2,000 held-out instances -- generous to the CPU")}
    line = {"metric": METRIC_LEARNED, "value": v, "unit": "LPs/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded refinery planning family, no dataset)",
            "config": learned_cfg(args, fam, 1), "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "LPs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.profile:
        profile_learned(args) if args.workload == "refinery_learned" else profile_case(args)
        return
    if args.impl == "reference":
        if int(os.environ.get("RANK", 0)) != 0:
            return
        if args.workload == "refinery_learned":
            run_reference_learned(args)
        elif args.workload in ("uneven_batch", "refinery"):
            run_reference_batch(args)
        else:
            run_reference(args)
        return
    if args.workload == "refinery_learned":
        run_learned_workload(args)
        return
    if args.workload in ("uneven_batch", "refinery"):
        run_batch_workload(args)
        return
    import torch
    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    # the engine captures CUDA graphs, which the legacy default stream does not allow
    work_stream = torch.cuda.Stream()
    torch.cuda.set_stream(work_stream)
    b2p, lp, cfg = make_lp(args.workload)
    std = lp.standard()
    ctx = b2p.Context(local)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    ctx.upload(std)
    common = dict(engine="halpern", eps=args.eps, max_iterations=2_000_000, time_limit_s=args.time_limit)
    # warm-up (also fills the autotune / allocation caches); on the stress LP, whose
    # solve takes minutes, warm-up solves stop after 4096 iterations
    warm = dict(common, max_iterations=4096) if args.workload == "ill_conditioned" else common
    for _ in range(args.warmup):
        ctx.solve(precision="fp32", **warm)
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    sampler.start()
    ms, results = timed_solves(ctx, torch, args.steps, world, precision="fp32", **common)
    clocks = sampler.stop()
    ms_max = max_over_ranks(ms, world)
    solved = sum_over_ranks(float(sum(r["status"] == "OPTIMAL" for r in results)), world)
    value = solved / (ms_max / 1e3)  # LPs that reached the tolerance, per second
    launches = int(sum(r["kernel_launches"] for r in results))
    iters = results[-1]["iterations"]
    # plain FP64 PDHG on the same LP and GPU
    fp64 = None
    if not args.no_fp64:
        for _ in range(1):
            ctx.solve(precision="fp64", **warm)
        ms64, res64 = timed_solves(ctx, torch, args.steps, world, precision="fp64", **common)
        ms64 = max_over_ranks(ms64, world)
        solved64 = sum_over_ranks(float(sum(r["status"] == "OPTIMAL" for r in res64)), world)
        fp64 = {"value": solved64 / (ms64 / 1e3), "unit": "LPs/s", "iterations": res64[-1]["iterations"],
                "ms_per_step": ms64 / args.steps, "rel_kkt": res64[-1]["rel_kkt"], "solved": int(solved64)}
    # roofline of the dominant kernel (mixed precision), timed live with CUDA events
    # after a (capped) mixed solve has set up the tuned kernels
    ctx.solve(precision="fp32", **warm)
    kt = ctx.kernel_timing(reps=20, precision="fp32", **common)
    pk, pk_src = peaks()
    peak = pk["hbm_gbs"]
    dom = "primal" if kt["primal_ms"] >= kt["dual_ms"] else "dual"
    achieved = kt[f"{dom}_bytes"] / (kt[f"{dom}_ms"] / 1e3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / f"halpern_{dom}_{args.workload}.txt"
    if tfile.exists():
        for ln in tfile.read_text().splitlines():
            if ln.startswith("dram_bytes_per_launch:"):
                traffic = float(ln.split(":")[1])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": f"k_iter<{dom}> (mixed)", "kernel_ms": kt[f"{dom}_ms"],
                "algorithmic_bytes": kt[f"{dom}_bytes"],
                "iteration": {"ms": kt["primal_ms"] + kt["dual_ms"],
                              "GB/s": (kt["primal_bytes"] + kt["dual_bytes"]) / ((kt["primal_ms"] + kt["dual_ms"]) / 1e3) / 1e9},
                "peak_source": "hbm_gbs: " + pk_src}
    # end to end through the public API: pinned host buffers -> upload (H2D + transpose) -> solve -> x, y to host
    pin = {k: torch.from_numpy(np.ascontiguousarray(getattr(std, k))).pin_memory()
           for k in ("rowptr", "colidx", "vals", "b", "c", "lb", "ub", "is_eq")}

    class PinnedLP:
        pass

    plp = PinnedLP()
    for k, t in pin.items():
        setattr(plp, k, t.numpy())
    plp.m, plp.n = std.m, std.n
    h2d = sum(t.numel() * t.element_size() for t in pin.values())
    d2h = 8 * (std.m + std.n)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    up_s = solve_s = 0.0
    e2e_status = []
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        ctx.upload(plp)
        t1 = time.perf_counter()
        res, x, y = ctx.solve(precision="fp32", **common)
        t2 = time.perf_counter()
        up_s += t1 - t0
        solve_s += t2 - t1
        e2e_status.append(res["status"])
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    if args.e2e_steps > 0:
        e2e_solved = sum_over_ranks(float(sum(r == "OPTIMAL" for r in e2e_status)), world)
        e2e = {"value": e2e_solved / (e2e_ms / 1e3), "unit": "LPs/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": args.e2e_steps,
               "upload_ms_per_step": 1e3 * up_s / args.e2e_steps, "solve_ms_per_step": 1e3 * solve_s / args.e2e_steps,
               "iterations": res["iterations"], "solved": int(e2e_solved)}
    else:
        e2e = {"value": None, "skipped": "--e2e-steps 0 (each solve of this workload takes minutes)",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_reference_sample(lp, args.cpu_sample_iters, fp64["iterations"] if fp64 else iters)
    if rank == 0:
        line = {"metric": metric_for(args), "value": value, "unit": "LPs/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 values + f64 iterates/KKT",
                "data": "synthetic (seeded generator, no dataset)",
                "config": dict(cfg, parallelism=f"replicas x{world}", eps_rel_kkt=args.eps,
                               l2=f"inputs larger than L2 (scaled A and A^T: ~{16 * lp.nnz / 1e6:.0f} MB)",
                               engine="halpern/mixed"),
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": launches,
                "clocks": clocks, "iterations": iters, "solved": int(solved), "status": results[-1]["status"],
                "fp64": fp64, "rel_kkt": results[-1]["rel_kkt"],
                "time_limit_s": args.time_limit or None}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
