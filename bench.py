"""Benchmark: time to relative KKT 1e-6 on the SOC-constrained QP workload.

Workload (the configuration the headline metric is quoted on): n = 1e6
variables in 20000 standard SOC blocks of 50 slots, m = 5e5 equality rows
with 10 nnz/row N(0,1), diagonal Q ~ U(0.01, 1), c ~ N(0,1), b = A x0 with
x0 strictly inside the cones; seeded synthetic data (no public dataset).

One step = one complete solve to relative KKT 1e-6 (eps_opt = eps_feas =
1e-6).  ``value`` is seconds per solve with the problem already resident in
HBM; ``e2e`` is the same solve through the C entry point solve_qp_problem
from host buffers (host->device copies and the device->host copy of the
solution inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from pdhcg_b200 import capi, instances, native  # noqa: E402

EPS = 1e-6
METRIC = "time-to-1e-6 KKT (s) & SpMV GB/s: mixed/warm-start vs plain FP64, 1 B200"
WORKLOAD = "soc_qp: n=1e6 (20000 SOC blocks x 50), m=5e5 eq rows, 10 nnz/row, diag Q, eps 1e-6"

# DRAM read + write bytes of one step of the SOC-QP workload (both
# kernels), from an ncu capture of the two step kernels on it
STEP_TRAFFIC = {"f64": 202.5e6, "f32": 121.4e6}
# random 4- / 8-byte gathers per second of one B200 through L1TEX, measured
# by pdhcg_b200/csrc/probes/gather_ceiling.cu
GATHER_RATE = 1.95e11

# Single-instance workloads: the generator, whether the mixed form is timed
# beside FP64, and what keeps the timed solves out of L2.

WORKLOADS = {
    "soc_qp": {"make": lambda scale, r: instances.soc_qp(seed=2 + r, scale=scale), "desc": WORKLOAD,
               "mixed": True, "l2": "working set (>=134 MB) larger than L2"},
    "sparse_qp": {"make": lambda scale, r: instances.sparse_qp(seed=1 + r, scale=scale),
                  "desc": "sparse_qp: n=1e4, m=5e3, 8 nnz/row, Q = B'B + 0.1 I (B 2000 x 1e4, 4 nnz/row; "
                          "sparse Q, inner BB solve), box [-10, 10], eps 1e-6",
                  "mixed": True, "l2": "L2-resident working set (< 3 MB): latency-bound, time to tolerance"},
    "portfolio": {"make": lambda scale, r: instances.portfolio(seed=3 + r, scale=scale),
                  "desc": "portfolio: n=2e5 assets, R 100 x 2e5 dense N(0, 1/sqrt n), D diag U(0.5, 2), "
                          "Q diag U(1e-4, 1e-2), budget + 500 sector + 100 exposure rows, RSOC tracking-error "
                          "block, x in [0, 0.02], eps 1e-6",
                  "mixed": True, "l2": "working set (A, R and R^T, >700 MB) larger than L2"},
    "fixed_soc": {"make": lambda scale, r: instances.fixed_cone_qp(seed=21 + r, nsoc=400, soc_len=50),
                  "desc": "fixed_soc: conic LP with 400 SOC blocks of 50, 4 RSOC, 6 EXP and 6 POW blocks and "
                          "slots of about half the blocks fixed by set_cone_fixed (n=20128), eps 1e-6",
                  "mixed": False, "l2": "L2-resident working set: time to tolerance"},
}


def _h2d_bytes(p) -> int:
    """Bytes of the problem arrays a host-buffer solve copies to the device."""
    n, m = p.n, (p.A.m if p.A is not None else 0)
    b = 3 * n * 8 + 2 * m * 8
    for M in (p.A, p.Q):
        if M is not None:
            b += M.nnz * 12 + (M.m + 1) * 4
    if getattr(p, "R_dense", None) is not None:
        b += p.R_dense.size * 8
    if getattr(p, "D", None) is not None:
        b += p.D.nnz * 12 + (p.D.m + 1) * 4
    b += 12 * len(p.cones or [])
    return int(b)


def _params(lib, iters=None):
    over = {"termination_criteria.eps_optimal_relative": EPS, "termination_criteria.eps_feasible_relative": EPS,
            "termination_criteria.time_sec_limit": 600.0}
    if iters:
        over["termination_criteria.iteration_limit"] = iters
    return capi.default_params(lib, **over)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu: int = 0):
        self.samples = []
        self._stop = threading.Event()
        self.gpu = gpu
        self._t = None

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                f = [x.strip() for x in out.stdout.strip().split(",")]
                if len(f) >= 7:
                    self.samples.append(f)
            except Exception:
                pass
            self._stop.wait(0.2)

    def stop(self) -> dict:
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(self.samples[0][1]) if self.samples[0][1].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(self.samples)}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(problem, n_iter_ref: int, budget_s: float = 20.0) -> dict:
    """The oracle (single-threaded FP64 port of the same iteration) timed on
    a bounded sample: a fixed number of iterations on the full workload,
    extrapolated to the GPU's iteration count to tolerance."""
    oracle = C.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    oracle.oracle_solve.restype = C.POINTER(capi.PdhcgResult)
    oracle.oracle_solve.argtypes = [C.POINTER(capi.QpProblem), C.POINTER(capi.PdhgParameters)]
    lib = native.load()
    prob, keep = capi.build(lib, problem)
    sample_iters = 20
    t0 = time.perf_counter()
    r = oracle.oracle_solve(prob, C.byref(_params(lib, sample_iters)))
    dt = time.perf_counter() - t0
    oracle.oracle_result_free(r)
    # second sample to separate per-iteration time from setup (rescaling, power method)
    sample2 = max(sample_iters + 1, int(sample_iters * min(8.0, max(2.0, budget_s / max(dt, 1e-3)))))
    t0 = time.perf_counter()
    r = oracle.oracle_solve(prob, C.byref(_params(lib, sample2)))
    dt2 = time.perf_counter() - t0
    oracle.oracle_result_free(r)
    lib.qp_problem_free(prob)
    per_iter = (dt2 - dt) / (sample2 - sample_iters)
    setup = max(dt - per_iter * sample_iters, 0.0)
    est = setup + per_iter * n_iter_ref
    return {"value": est, "unit": "s", "cores": 1, "kind": "port", "cpu_model": _cpu_model(),
            "sample": f"oracle FP64 on the full workload: {sample_iters} and {sample2} iterations "
                      f"({dt:.1f}s, {dt2:.1f}s), extrapolated to {n_iter_ref} iterations "
                      f"(setup {setup:.2f}s + {per_iter * 1e3:.1f} ms/iter)"}


def run_ours(args):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
    lib = native.load()
    W = WORKLOADS[args.workload]
    # one instance does not shard (its products would need an exchange each
    # step): with several ranks every rank solves the same instance, a replica
    problem = W["make"](args.scale, 0)
    prob, keep = capi.build(lib, problem)
    prm = _params(lib, args.iters)
    forms = {"fp64": 0, "mixed": 1} if W["mixed"] else {"fp64": 0}
    handle = lib.pdhcg_b200_upload(prob)
    if not handle:
        raise RuntimeError("pdhcg_b200_upload failed")

    def solve(precision, device, time_steps=0):
        opts = native.default_options(precision=precision, time_steps=time_steps, solution_on_device=int(device))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if device:
            r = lib.pdhcg_b200_solve_device(handle, C.byref(prm), C.byref(opts))
        else:
            r = lib.pdhcg_b200_solve(prob, C.byref(prm), C.byref(opts))
        e1.record()
        torch.cuda.synchronize()
        if not r:
            raise RuntimeError("solve failed")
        if device:
            rr = r.contents
            d = {"status": capi.TERMINATION_REASONS[rr.termination_reason], "total_count": rr.total_count,
                 "rel_kkt": max(rr.relative_primal_residual, rr.relative_dual_residual, rr.relative_objective_gap),
                 "primal_objective_value": rr.primal_objective_value, "total_inner_count": rr.total_inner_count}
        else:
            d = capi.result_dict(r, problem.n, problem.A.m)
        lib.pdhcg_result_free(r)
        return e0.elapsed_time(e1) / 1e3, d, native.last_stats()

    def time_form(precision):
        res = {}
        for device in (True, False):
            for _ in range(args.warmup):
                solve(precision, device)
            sampler = ClockSampler(local)
            sampler.start()
            times, r1, st = [], None, None
            for _ in range(args.steps):
                if world > 1:
                    torch.distributed.barrier()
                t, r1, st = solve(precision, device)
                times.append(t)
            clocks = sampler.stop()
            if world > 1:
                tt = torch.tensor([max(times)], device="cuda")
                torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
                worst = tt.item()
            else:
                worst = max(times)
            res["device" if device else "host"] = (sum(times) / len(times), worst, r1, st, clocks)
        # kernel-level timing in a separate run (events around each fused step)
        _, _, tstats = solve(precision, True, time_steps=1)
        res["tstats"] = tstats
        return res

    out = {name: time_form(pr) for name, pr in forms.items()}
    lib.pdhcg_b200_device_problem_free(handle)
    if world > 1:
        torch.distributed.barrier()
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    peak, peak_kind = _peaks()

    def roof(tstats):
        step_ms = tstats["step_kernel_ms"] / max(1, tstats["step_kernel_launches"])
        ach = tstats["step_bytes"] / (step_ms * 1e-3) / 1e9 if step_ms > 0 else None
        # DRAM bytes (read + write) of one step's kernels, from the ncu
        # capture of the step kernels, weighted like the timed steps
        traffic = None
        if args.workload == "soc_qp" and args.scale == 1.0 and tstats["step_kernel_launches"] > 0:
            f32 = tstats["fp32_iterations"] / tstats["step_kernel_launches"]
            traffic = f32 * STEP_TRAFFIC["f32"] + (1.0 - f32) * STEP_TRAFFIC["f64"]
        return {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": (ach / peak) if ach else None, "traffic": traffic, "peak_kind": peak_kind,
                "bytes_per_step": tstats["step_bytes"], "step_kernel_ms": step_ms,
                "kernels": "the two launches of a step: primal_cone_kernel (A^T y, prox, SOC projection, "
                           "Halpern) and dual_kernel (A x_refl, dual prox, Halpern)",
                # each product gathers one vector entry per nonzero; the B200's
                # random-gather rate bounds the step below HBM speed
                "gather_bound": {"gathers_per_step": 2 * problem.A.nnz, "measured_ceiling_per_s": GATHER_RATE,
                                 "floor_ms": 2 * problem.A.nnz / GATHER_RATE * 1e3,
                                 "frac_of_floor": (2 * problem.A.nnz / GATHER_RATE * 1e3) / step_ms
                                 if step_ms > 0 else None,
                                 "source": "profiles/spmv_gather_ceiling_b200.md"}}

    head = out["mixed"] if W["mixed"] else out["fp64"]
    fp64 = out["fp64"]
    per_solve, _, res, stats, clocks = head["device"]
    e2e_solve, _, e2e_res, e2e_stats, _ = head["host"]
    rl = roof(head["tstats"])
    line = {
        "metric": METRIC, "value": per_solve, "unit": "s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_solve * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if W["mixed"] else "f64", "data": "synthetic",
        "config": {"workload": W["desc"],
                   "parallelism": "replicas: every rank solves the same instance" if world > 1 else "single",
                   "eps": EPS, "form": "mixed: FP32 bulk, FP64 polish below 1e-5" if W["mixed"] else "FP64",
                   "l2_flush": W["l2"],
                   "inputs": "value: problem resident in HBM (pdhcg_b200_upload once), solution left on device; "
                             "e2e: host buffers through pdhcg_b200_solve"},
        "status": res["status"], "iterations": res["total_count"], "rel_kkt": res["rel_kkt"],
        "objective": res["primal_objective_value"], "fp32_iterations": stats["fp32_iterations"],
        "spmv_gbs": rl["achieved"],
        "roofline": rl,
        "e2e": {"value": e2e_solve, "unit": "s",
                "h2d_bytes_per_step": _h2d_bytes(problem),
                "d2h_bytes_per_step": int(8 * (2 * problem.n + problem.A.m)),
                "status": e2e_res["status"], "iterations": e2e_res["total_count"]},
        "gpu_launches": int(stats["kernel_launches"]) * args.steps,
        "clocks": clocks,
        "breakdown_ms": {k: stats[k] for k in ("host_copy_ms", "upload_ms", "setup_ms", "loop_ms", "result_ms",
                                               "total_ms")},
        "e2e_breakdown_ms": {k: e2e_stats[k] for k in ("host_copy_ms", "upload_ms", "setup_ms", "loop_ms",
                                                       "result_ms", "total_ms")},
    }
    if W["mixed"]:
        line["fp64_form"] = {"value": fp64["device"][0], "e2e": fp64["host"][0],
                             "status": fp64["device"][2]["status"], "iterations": fp64["device"][2]["total_count"],
                             "rel_kkt": fp64["device"][2]["rel_kkt"],
                             "objective": fp64["device"][2]["primal_objective_value"],
                             "roofline": roof(fp64["tstats"])}
        line["speedup_mixed_vs_fp64"] = fp64["device"][0] / per_solve
    else:
        line["inner_iterations"] = res.get("total_inner_count")
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(problem, res["total_count"])
    if world == 1 and not args.no_extras and args.workload == "soc_qp":
        # the other patterns and workloads on the same line (one GPU): the
        # batched solver on the full 4096-instance batch, the learned warm
        # start at a reduced training count, and the inner-BB workloads
        # beside the reference's own build
        line["batched"] = measure_batch(4096, steps=3, warmup=1)
        line["warm_start"] = measure_warm_start(50000, train=256, epochs=60, heldout=24)
        for name in ("sparse_qp", "portfolio"):
            line[name] = measure_single(name)
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


BATCH_METRIC = "batched instance throughput (instances/s) at 1e-5 KKT, vs sequential plain solves, 1 B200"
BATCH_WORKLOAD = ("mpc_batch: 4096 MPC QPs, horizon T ~ U{10..100}, n = 12 T, m = 8 T, 13 nnz/row, "
                  "diag Q ~ U(0.1, 1), inputs in [-1, 1], eps 1e-5")
BATCH_EPS = 1e-5


def _batch_params(lib):
    return capi.default_params(lib, **{"termination_criteria.eps_optimal_relative": BATCH_EPS,
                                       "termination_criteria.eps_feasible_relative": BATCH_EPS,
                                       "termination_criteria.time_sec_limit": 600.0})


def measure_batch(count: int, steps: int, warmup: int, rank: int = 0, world: int = 1, seq_sample: int = 16) -> dict:
    """One batch of ``count`` MPC instances split across the ranks by
    nonzero count (pdhcg_b200.shard): every rank builds only its bin and
    solves it with pdhcg_b200_solve_batch on its own GPU; the results come
    back to rank 0 once at the end.  Times are the max over ranks; the
    throughputs are the whole batch over that time (strong scaling: the
    batch is the same for every rank count).  Rank 0 also times one
    solve_qp_problem per instance on a sample, the way the reference would
    solve them."""
    import torch
    from pdhcg_b200 import shard
    lib = native.load()
    weights = [instances.mpc_nnz(int(t)) for t in instances.mpc_horizons(4, count)]
    mine = shard.partition(weights, world)[rank]
    probs = instances.mpc_batch(seed=4, count=count, indices=mine)
    built = [capi.build(lib, p) for p in probs]
    k = len(built)
    arr = (C.POINTER(capi.QpProblem) * max(k, 1))(*[b[0] for b in built])
    prm = _batch_params(lib)
    opts = native.BatchOptions()
    lib.pdhcg_b200_default_batch_options(C.byref(opts))
    shape_ms = (C.c_double * native.BATCH_SHAPES)()
    if k and lib.pdhcg_b200_batch_autotune(min(k, 512), arr, C.byref(prm), C.byref(opts), shape_ms) != 0:
        raise RuntimeError("batch autotune failed")
    res = (C.POINTER(capi.PdhcgResult) * max(k, 1))()
    launches = [0]
    copies = [(0, 0, 0.0)]

    def solve():
        if not k:
            return 0.0, 0.0, {}
        t0 = time.perf_counter()
        if lib.pdhcg_b200_solve_batch(k, arr, C.byref(prm), C.byref(opts), res) != 0:
            raise RuntimeError("batch solve failed")
        wall = time.perf_counter() - t0
        bst = native.BatchStats()
        lib.pdhcg_b200_last_batch_stats(C.byref(bst))
        launches[0] += bst.launches
        copies[0] = (int(bst.h2d_bytes), int(bst.d2h_bytes), bst.pack_ms)
        out = {}
        for i, r in zip(mine, res[:k]):
            out[i] = (capi.TERMINATION_REASONS[r.contents.termination_reason], r.contents.total_count)
            lib.pdhcg_result_free(r)
        return wall, bst.kernel_ms * 1e-3, out

    for _ in range(warmup):
        solve()
    launches[0] = 0
    walls, kerns, last = [], [], {}
    for _ in range(steps):
        if world > 1:
            torch.distributed.barrier()
        w, kt, last = solve()
        walls.append(w)
        kerns.append(kt)
    wall, kern = max(walls), max(kerns)
    if world > 1:
        t = torch.tensor([wall, kern], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        wall, kern = t[0].item(), t[1].item()
        b = torch.tensor([float(copies[0][0]), float(copies[0][1])], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(b)  # copies of all ranks
        copies[0] = (int(b[0].item()), int(b[1].item()), copies[0][2])
    allres = shard.gather_results(last, rank, world, count)
    nnz_mine = int(sum(weights[i] for i in mine))
    out = None
    if rank == 0:
        stat = {}
        for st, _ in allres:
            stat[st] = stat.get(st, 0) + 1
        t0 = time.perf_counter()
        for i in range(min(seq_sample, k)):
            r = lib.solve_qp_problem(arr[i], C.byref(prm))
            lib.pdhcg_result_free(r)
        seq = min(seq_sample, k) / (time.perf_counter() - t0)
        out = {"value": count / kern, "unit": "instances/s", "ms_per_step": kern * 1e3, "instances": count,
               "statuses": stat, "mean_iterations": float(np.mean([it for _, it in allres])),
               "e2e": {"value": count / wall, "unit": "instances/s", "h2d_bytes_per_step": copies[0][0],
                       "d2h_bytes_per_step": copies[0][1], "pack_ms_rank0": copies[0][2]},
               "sequential_plain_solves": {"value": seq, "unit": "instances/s", "sample": min(seq_sample, k),
                                           "call": "solve_qp_problem per instance, one GPU"},
               "speedup_vs_sequential": (count / wall) / seq,
               "shape": int(opts.shape), "band_shapes": [int(b) - 1 for b in opts.band_shape],
               "autotune_ms": list(shape_ms), "gpu_launches": launches[0],
               "partition": {"ranks": world, "instances_on_rank0": k, "nnz_on_rank0": nnz_mine,
                             "nnz_total": int(sum(weights))}}
    for b in built:
        lib.qp_problem_free(b[0])
    return out


def run_batch(args):
    """The batched workload on its own line (--workload mpc_batch)."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
    count = max(1, int(4096 * args.scale))
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    m = measure_batch(count, args.steps, args.warmup, rank, world)
    clocks = sampler.stop()
    if rank == 0:
        line = {"metric": BATCH_METRIC, "value": m["value"], "unit": "instances/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms_per_step"],
                "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
                "dtype": "f32+f64", "data": "synthetic",
                "config": {"workload": BATCH_WORKLOAD, "instances": count,
                           "parallelism": "one batch partitioned across ranks by nonzeros" if world > 1 else "single",
                           "l2_flush": "not needed: each instance lives in shared memory for its whole solve",
                           "inputs": "value: kernel time, problem arrays already on the device; e2e: the whole "
                                     "pdhcg_b200_solve_batch call from host problems"},
                **{k: v for k, v in m.items() if k not in ("value", "unit", "ms_per_step")},
                "clocks": clocks}
        if not args.no_cpu_baseline:
            lib = native.load()
            oracle = C.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
            oracle.oracle_solve.restype = C.POINTER(capi.PdhcgResult)
            oracle.oracle_solve.argtypes = [C.POINTER(capi.QpProblem), C.POINTER(capi.PdhgParameters)]
            prm = _batch_params(lib)
            t0, done = time.perf_counter(), 0
            for p in instances.mpc_batch(seed=4, count=count, indices=range(min(count, 2000))):
                if time.perf_counter() - t0 >= 10.0:
                    break
                prob, keep = capi.build(lib, p)
                r = oracle.oracle_solve(prob, C.byref(prm))
                oracle.oracle_result_free(r)
                lib.qp_problem_free(prob)
                done += 1
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": done / dt, "unit": "instances/s", "cores": 1, "kind": "port",
                                    "sample": f"oracle FP64 on the first {done} instances ({dt:.1f}s)"}
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


WS_METRIC = "learned warm start: time-to-1e-6 KKT (s) per held-out instance, warm vs cold start, 1 B200"
WS_EPS = 1e-6


def measure_warm_start(n: int, train: int, epochs: int, heldout: int, warmup: int = 2) -> dict:
    """The parametric family: cold solves of ``train`` parameters, the MLP
    trained on the GPU, then ``heldout`` new instances solved three ways --
    cold, from the training targets' mean, and from the network's
    prediction -- all with the family's cached step size (no power method in
    any of them), each timed as a whole call (the prediction included).
    Every answer must meet the same tolerance."""
    from pdhcg_b200 import warmstart
    fam = warmstart.ParametricQP(seed=5, n=n)
    params = {"termination_criteria.eps_optimal_relative": WS_EPS,
              "termination_criteria.eps_feasible_relative": WS_EPS, "termination_criteria.time_sec_limit": 600.0}
    ws = warmstart.WarmStart(fam, hidden=512, rank=64, seed=1)
    try:
        t0 = time.perf_counter()
        thetas = fam.thetas(train, seed=1)
        X, lw, train_its = ws.collect(thetas, params)
        t_collect = time.perf_counter() - t0
        batch = min(64, train)
        t0 = time.perf_counter()
        loss = ws.fit(thetas, X, lw, epochs=epochs, batch=batch, lr=1e-3)
        t_fit = time.perf_counter() - t0
        held = fam.thetas(heldout + warmup, seed=2)
        for th in held[:warmup]:
            for f in ("cold", "mean", "net"):
                ws.solve(th, params, start=f)
        forms = {f: {"t": [], "it": [], "ok": 0} for f in ("cold", "mean", "net")}
        for th in held[warmup:]:
            res = {f: ws.solve(th, params, start=f) for f in forms}
            ref = res["cold"]["primal_objective_value"]
            for f, d in res.items():
                forms[f]["t"].append(d["wall_s"])
                forms[f]["it"].append(d["total_count"])
                forms[f]["ok"] += int(d["status"] == "OPTIMAL" and
                                      abs(d["primal_objective_value"] - ref) <= 10 * WS_EPS * (1 + abs(ref)))
    finally:
        ws.close()
    summ = {f: {"value": float(np.mean(v["t"])), "unit": "s", "mean_iterations": float(np.mean(v["it"])),
                "passing_same_tolerance": f"{v['ok']}/{heldout}"} for f, v in forms.items()}
    steps = epochs * (train // batch)
    return {"value": summ["net"]["value"], "unit": "s", "forms": summ,
            "speedup_net_vs_cold": summ["cold"]["value"] / summ["net"]["value"],
            "speedup_net_vs_mean": summ["mean"]["value"] / summ["net"]["value"],
            "iterations_cold_over_net": summ["cold"]["mean_iterations"] / summ["net"]["mean_iterations"],
            "iterations_mean_over_net": summ["mean"]["mean_iterations"] / summ["net"]["mean_iterations"],
            "equal_setup": "every form reuses the family's cached step size (no power method); times are whole "
                           "calls, the network's prediction included",
            "training": {"solves": train, "epochs": epochs, "collect_s": t_collect, "fit_s": t_fit,
                         "fit_ms_per_step": t_fit / max(1, steps) * 1e3, "final_loss": loss,
                         "mean_training_iterations": float(np.mean(train_its))},
            "config": {"workload": f"parametric QP family: n={n}, m={n // 2}, A 6 nnz/row, diag Q, theta in R^32, "
                                   f"c = c0 + C theta, row bounds + L theta, eps 1e-6",
                       "network": "32-512-512 MLP, rank-64 output head to n + m, log primal-weight head; "
                                  "BF16 tensor-core products, FP32 accumulation"}}


def run_warm_start(args):
    """The learned warm start on its own line (--workload warm_start)."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if rank != 0:  # one family, one GPU: the other ranks idle
        return
    n = max(1000, int(50000 * args.scale))
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    m = measure_warm_start(n, args.train, args.epochs, args.heldout, args.warmup)
    clocks = sampler.stop()
    line = {"metric": WS_METRIC, "value": m["value"], "unit": "s", "n_gpus": 1, "steps": args.heldout,
            "warmup": args.warmup, "ms_per_step": m["value"] * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 solve, bf16/f32 network", "data": "synthetic",
            "config": {**m["config"], "training_solves": args.train, "heldout_solves": args.heldout,
                       "epochs": args.epochs},
            **{k: v for k, v in m.items() if k not in ("value", "unit", "config")},
            "e2e": {"value": m["value"], "unit": "s",
                    "h2d_bytes_per_step": int(n // 2 * 6 * 12 + n * 8 * 6 + (n // 2) * 8 * 3),
                    "d2h_bytes_per_step": int(8 * (2 * n + n // 2))},
            "clocks": clocks}
    print(json.dumps(line))


def measure_single(name: str, steps: int = 2, warmup: int = 1) -> dict:
    """Time to 1e-6 of one single-instance workload: the problem resident
    (pdhcg_b200_upload, then solves) and from host buffers, in FP64 and,
    where the workload has one, the mixed form (FP32 bulk phase, FP64
    polish), beside the reference's own build on the same instance when it
    is present."""
    import torch
    lib = native.load()
    W = WORKLOADS[name]
    problem = W["make"](1.0, 0)
    prob, keep = capi.build(lib, problem)
    prm = _params(lib)
    handle = lib.pdhcg_b200_upload(prob)
    forms = {"fp64": 0, "mixed": 1} if W["mixed"] else {"fp64": 0}
    res = {}
    for form, precision in forms.items():
        for device in (True, False):
            opts = native.default_options(precision=precision, solution_on_device=int(device))
            ts = []
            for i in range(warmup + steps):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                r = lib.pdhcg_b200_solve_device(handle, C.byref(prm), C.byref(opts)) if device else \
                    lib.pdhcg_b200_solve(prob, C.byref(prm), C.byref(opts))
                torch.cuda.synchronize()
                dt = time.perf_counter() - t0
                rr = r.contents
                d = {"status": capi.TERMINATION_REASONS[rr.termination_reason], "total_count": rr.total_count,
                     "primal_objective_value": rr.primal_objective_value,
                     "total_inner_count": rr.total_inner_count,
                     "rel_kkt": max(rr.relative_primal_residual, rr.relative_dual_residual,
                                    rr.relative_objective_gap),
                     "fp32_iterations": native.last_stats()["fp32_iterations"]}
                lib.pdhcg_result_free(r)
                if i >= warmup:
                    ts.append(dt)
            res[(form, device)] = (float(np.mean(ts)), d)
    lib.pdhcg_b200_device_problem_free(handle)
    lib.qp_problem_free(prob)
    (tv, d), (te, _) = res[("fp64", True)], res[("fp64", False)]
    out = {"value": tv, "unit": "s", "e2e": te, "status": d["status"], "iterations": d["total_count"],
           "inner_iterations": d.get("total_inner_count"), "objective": d["primal_objective_value"],
           "rel_kkt": d["rel_kkt"], "form": "FP64", "workload": W["desc"]}
    if "mixed" in forms:
        (mv, md), (me, _) = res[("mixed", True)], res[("mixed", False)]
        out["mixed"] = {"value": mv, "unit": "s", "e2e": me, "status": md["status"], "iterations": md["total_count"],
                        "fp32_iterations": md["fp32_iterations"], "inner_iterations": md.get("total_inner_count"),
                        "objective": md["primal_objective_value"], "rel_kkt": md["rel_kkt"],
                        "objective_rel_diff_vs_fp64": abs(md["primal_objective_value"] - d["primal_objective_value"]) /
                                                      (1 + abs(d["primal_objective_value"])),
                        "form": "FP32 values of Q, R, R^T and of A's long rows with FP64 iterates and accumulation "
                                "until the relative KKT error is below 1e-5, then FP64"}
        out["speedup_mixed_vs_fp64"] = tv / mv
    path = os.path.join(ROOT, "oracle", "_ref", "libpdhcg_ref.so")
    if os.path.exists(path):
        ref = capi.bind_api(C.CDLL(path))
        rprob, rkeep = capi.build(ref, problem)
        rprm = _params(ref)
        ts = []
        for i in range(1 + 1):
            t0 = time.perf_counter()
            r = ref.solve_qp_problem(rprob, C.byref(rprm))
            dt = time.perf_counter() - t0
            rd = capi.result_dict(r, problem.n, problem.A.m)
            ref.pdhcg_result_free(r)
            if i >= 1:
                ts.append(dt)
        ref.qp_problem_free(rprob)
        out["reference"] = {"value": float(np.mean(ts)), "unit": "s", "status": rd["status"],
                            "iterations": rd["total_count"],
                            "objective_rel_diff": abs(d["primal_objective_value"] - rd["primal_objective_value"]) /
                                                  (1 + abs(rd["primal_objective_value"])),
                            "call": "the reference's own build, solve_qp_problem from host buffers"}
        out["speedup_e2e_vs_reference"] = out["reference"]["value"] / te
    return out


def run_reference(args):
    """The reference's own solver (built from its sources into oracle/_ref)
    on the same instance through its C API; falls back to the oracle port
    when that build is absent."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    path = os.path.join(ROOT, "oracle", "_ref", "libpdhcg_ref.so")
    W = WORKLOADS.get(args.workload, WORKLOADS["soc_qp"])
    problem = W["make"](args.scale, 0)
    if not os.path.exists(path):
        lib = native.load(build=False)
        cb = cpu_baseline(problem, 3000)
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "s",
                          "higher_is_better": False, "n_gpus": 1, "steps": 1, "warmup": 0,
                          "config": {"workload": W["desc"]}, "cpu_baseline": cb,
                          "e2e": {"value": cb["value"], "unit": "s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return
    ref = capi.bind_api(C.CDLL(path))
    prob, keep = capi.build(ref, problem)
    prm = _params(ref, args.iters)
    times = []
    res = None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        r = ref.solve_qp_problem(prob, C.byref(prm))
        dt = time.perf_counter() - t0
        if not r:
            print(json.dumps({"impl": "reference", "unavailable": "reference solve returned NULL"}))
            return
        res = capi.result_dict(r, problem.n, problem.A.m)
        ref.pdhcg_result_free(r)
        if i >= args.warmup:
            times.append(dt)
    per = sum(times) / len(times)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": per, "unit": "s", "higher_is_better": False,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3, "dtype": "f64",
        "data": "synthetic", "config": {"workload": W["desc"], "eps": EPS},
        "status": res["status"], "iterations": res["total_count"], "rel_kkt": res["rel_kkt"],
        "objective": res["primal_objective_value"], "reference_loop_s": res["cumulative_time_sec"],
        "cpu_baseline": {"value": per, "unit": "s", "cores": 1, "kind": "reference",
                         "sample": "reference single-GPU build (cuSPARSE/cuBLAS) via its C API, full solve"},
        "e2e": {"value": per, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="workload scale (1.0 = the benchmark size)")
    ap.add_argument("--iters", type=int, default=None, help="iteration cap (profiling only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="soc_qp",
                    choices=["soc_qp", "sparse_qp", "portfolio", "fixed_soc", "mpc_batch", "warm_start"],
                    help="soc_qp: the headline single-instance workload; sparse_qp: sparse-Q QP (inner BB "
                         "solve); portfolio: low-rank portfolio QP; mpc_batch: the batched workload; "
                         "warm_start: the learned warm start on the parametric family")
    ap.add_argument("--train", type=int, default=2000, help="warm_start: training solves")
    ap.add_argument("--heldout", type=int, default=200, help="warm_start: held-out solves")
    ap.add_argument("--epochs", type=int, default=100, help="warm_start: training epochs")
    ap.add_argument("--no-extras", action="store_true",
                    help="soc_qp: leave out the batched, warm-start, sparse_qp and portfolio measurements")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: start them (the driver launches torchrun itself)
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
        sys.exit(subprocess.call(cmd))
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "mpc_batch":
        run_batch(args)
    elif args.workload == "warm_start":
        run_warm_start(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
