#!/usr/bin/env python
"""Benchmark: kriged targets/s on one B200 for the 2-D anisotropic sector-search
ordinary-kriging workload (200 000 clustered observations, 2000 x 2000 targets).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config C]

``--config`` picks one of the five workloads of bench_workloads.py at its full
size (default 2, the benchmark); the JSON line has the same keys for each.

Prints one JSON line.  ``value`` is device throughput of the FP32-factor +
FP64-refinement form with inputs resident in HBM (CUDA events on the solve
stream, L2 flushed between timed steps, max over ranks); ``fp64_plain`` is the
same measurement for the FP64 form and ``auto_default`` for the library's
default precision (per neighbour-count list the faster form, as timed by the
kernel tuner); ``replay`` times the weight-store re-estimate (store_weight
solve once, then update_obs_value + solve per step: one gather-dot kernel);
``sgsim`` times a sequential Gaussian simulation (four realisations on a
200 x 200 grid) against the oracle's sequential run; ``e2e`` is the same
metric through the
public ``Kriging`` API with host inputs/outputs copied every step.  The
reference arm (``--impl reference``) times the CPU restatement of the
reference engine (oracle/kk_oracle.c, OpenMP over all host threads) on a
bounded contiguous sample of the same targets.
"""
from __future__ import annotations

import argparse
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

import bench_workloads as bw  # noqa: E402

METRIC = "kriged targets/s on 1 B200: FP32+refine batched vs FP64 plain at <=1e-6 rel err"

# DRAM bytes per target of the dominant kernels, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of the same workload on its
# 400 x 400 target grid: the factorisation launch covers one 65 536-target
# chunk (its traffic is the chunk's K64 read back, 16.6 KB per target), the
# search launch all 160 000 targets (coordinates and neighbour lists); both
# grow in proportion to the targets.
NCU_DRAM_BYTES_PER_TARGET = {"solve_fp32_refine": (1098.960e6 + 30.646e6) / 65536,
                             "search": (8.722e6 + 1.375e6) / 160000}


def solve_flops(n, p=1, q=1):
    """Algorithmic FLOPs of one target system (Cholesky n^3/3, solves, Schur, variance)."""
    n = np.asarray(n, dtype=np.float64)
    return (n ** 3 / 3 + n ** 2 / 2 + n / 6 + 2 * n ** 2 * (p + q) + 2 * n * p ** 2 + 4 * n * p * q
            + p ** 3 / 3 + 2 * p ** 2 * q + 2 * (n + p) * q ** 2 + 2 * n * q)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks(torch, device):
    """Live cuBLAS SGEMM (FP32 CUDA cores, TF32 off) and DGEMM throughput, TFLOP/s."""
    out = {}
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    for name, dt, n in (("fp32", torch.float32, 8192), ("fp64", torch.float64, 8192)):
        a = torch.randn(n, n, device=device, dtype=dt)
        b = torch.randn(n, n, device=device, dtype=dt)
        for _ in range(2):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        out[name] = 2.0 * n ** 3 / best / 1e12
        del a, b
    torch.backends.cuda.matmul.allow_tf32 = old
    torch.cuda.empty_cache()
    return out


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def cpu_sample_run(W, nthread, target_seconds):
    """Time the CPU oracle on a contiguous slab of targets (all observations)."""

    def run(lo, hi):
        o = W.oracle(idx=np.arange(lo, hi))
        t0 = time.perf_counter()
        o.solve(nthread=nthread)
        return time.perf_counter() - t0, o

    n_all = W.ntarget
    pilot = min(n_all, 4000)
    lo0 = (n_all // 2) - (n_all // 2) % 2000
    lo0 = min(lo0, n_all - pilot)
    dt, _ = run(lo0, lo0 + pilot)
    rate = pilot / max(dt, 1e-6)
    n = int(min(n_all - lo0, max(pilot, rate * target_seconds)))
    dt, o = run(lo0, lo0 + n)
    return dict(rate=n / dt, seconds=dt, lo=lo0, hi=lo0 + n, oracle=o)


def workload_config(W):
    w = W.w
    vg = "; ".join(f"{i}{j} {s['vtype']} nug{s.get('nugget', 0)} sill{s.get('sill', 0)} a{s.get('a_major', '')}"
                   for (i, j, s) in w["vgm"])
    return {"workload": W.name, "ntargets": W.ntarget, "nobs": W.nobs, "ndim": w["ndim"], "nvar": w["nvar"],
            "search": W.describe(), "variogram": vg}


def run_reference(args, W):
    nthread = os.cpu_count() or 1
    step_rates = []
    for _ in range(args.warmup):
        cpu_sample_run(W, nthread, args.cpu_seconds / 4)
    last = None
    for _ in range(args.steps):
        r = cpu_sample_run(W, nthread, args.cpu_seconds)
        step_rates.append(r["rate"])
        last = r
    value = statistics.median(step_rates)
    sample = (f"targets {last['lo']}..{last['hi']} of the {W.ntarget} targets with all "
              f"{W.nobs} observations; {last['seconds']:.1f} s per step")
    cfg = workload_config(W)
    cfg["precision"] = "fp64"
    line = {
        "metric": METRIC, "value": value, "unit": "targets/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": last["seconds"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, see bench_workloads.py)",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": "targets/s", "cores": nthread, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "targets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def neighbours(k, nvar):
    """[(nnear, inear)] of each variable of the last solve."""
    return [k.get_neighbours(iv) for iv in range(1, nvar + 1)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2, choices=[1, 2, 3, 4, 5],
                    help="workload: 1 OK 2-D, 2 anisotropic sector OK (the benchmark), 3 KED 3-D, "
                         "4 LMC cokriging, 5 space-time product-sum with block support")
    ap.add_argument("--grid", type=int, default=None,
                    help="targets per axis (default: the workload's own size, 2000 for the benchmark)")
    ap.add_argument("--nmax", type=int, default=None,
                    help="neighbours per variable (per sector), overriding the workload's own")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-auto", action="store_true", help="skip the leg of the default precision (auto)")
    ap.add_argument("--no-replay", action="store_true", help="skip the weight-store re-estimate leg")
    ap.add_argument("--no-sgsim", action="store_true", help="skip the sequential-simulation leg")
    ap.add_argument("--autotune", type=int, default=None, choices=[0, 1, 2],
                    help="kernel plan: 0 fixed (use under a profiler, whose serialised launches distort the "
                         "tuner's timings), 1 tuned once per signature (the library default)")
    ap.add_argument("--precision", default="fp32_refine", choices=["fp32_refine", "fp64"],
                    help="form of the timed leg (fp64 is for profiling the plain form alone)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        run_reference(args, bw.Workload(args.config, args.grid, args.nmax))
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    W = bw.Workload(args.config, args.grid, args.nmax)
    W.autotune = args.autotune
    w = W.w
    nvar = w["nvar"]
    ntarget = W.ntarget
    nobs = W.nobs
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def time_steps(k, steps, warmup, sampler=None):
        for _ in range(warmup):
            k.solve()
        barrier()
        times = []
        ctx = sampler if sampler is not None else _Null()
        with ctx:
            for _ in range(steps):
                flush.fill_(1.0)  # L2 flush between timed steps (256 MiB write, outside the timed region)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                k.solve()
                e1.record()
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
        barrier()
        tot = sum(times) / 1e3
        if dist is not None:
            t = torch.tensor([tot], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            tot = float(t.item())
        return tot, times

    # targets are sharded, never exchanged: rank r solves slab r of a global
    # target set of world copies of the targets (weak scaling, fixed work per GPU)
    from krigekit_b200.shard import target_slab
    lo, hi = target_slab(world * ntarget, rank, world)
    slab = np.arange(lo, hi) % ntarget

    # ---- FP32 + refinement (the measured form)
    k32 = W.product(args.precision, idx=slab)
    sampler = ClockSampler(dev)
    tot32, times32 = time_steps(k32, args.steps, args.warmup, sampler)
    value = ntarget * world * args.steps / tot32
    clocks = sampler.summary()
    # per-phase device times from one extra profiled solve
    k32.profile(True)
    flush.fill_(1.0)
    k32.solve()
    ph32 = k32.phases()
    k32.profile(False)
    gst = k32.gpu_stats()
    k32_plan = k32.kernel_plan()
    e32, v32 = k32.get_results()
    nb32 = neighbours(k32, nvar)
    nnear = sum(nn.astype(np.int64) for nn, _ in nb32)

    # ---- FP64 plain
    fp64 = None
    if not args.no_fp64 and args.precision != "fp64":
        k64 = W.product("fp64", idx=slab)
        tot64, _ = time_steps(k64, args.steps, args.warmup)
        k64.profile(True)
        flush.fill_(1.0)
        k64.solve()
        ph64 = k64.phases()
        e64, v64 = k64.get_results()
        fp64 = {"value": ntarget * world * args.steps / tot64, "ms_per_step": tot64 / args.steps * 1e3,
                "phases_ms": ph64}
        ee = bw.rel_err(e32, e64, 1e-3 * w["zstd"])
        ve = bw.rel_err(v32, v64, 1e-3 * w["sill"])
        fin = np.isfinite(np.asarray(e64, dtype=np.float64))
        fp64["fp32_vs_fp64_rel_err"] = {
            "est_max": float(ee[fin].max()), "est_p99": float(np.percentile(ee[fin], 99)),
            "var_max": float(ve[fin].max()), "var_p99": float(np.percentile(ve[fin], 99))}
        del k64

    # ---- the product default: per list the form the kernel tuner timed faster
    auto = None
    if not args.no_auto and args.precision != "fp64":
        ka = W.product("auto", idx=slab)
        tota, _ = time_steps(ka, args.steps, args.warmup)
        auto = {"value": ntarget * world * args.steps / tota, "ms_per_step": tota / args.steps * 1e3,
                "plan": ka.kernel_plan()}
        del ka

    # ---- weight-store re-estimate: solve once with store_weight, then new
    # observation values per step (update_obs_value + solve = one k_replay)
    replay = None
    if not args.no_replay and not W.st:
        kr = W.product("fp64", idx=slab, store_weight=True)
        kr.solve()
        rng = np.random.default_rng(7)
        vals = [np.asarray(o["value"]) * (1.0 + 0.01 * rng.standard_normal(len(o["value"]))) for o in w["obs"]]
        for _ in range(args.warmup):
            for iv, v in enumerate(vals, start=1):
                kr.update_obs_value(iv, v)
            kr.solve()
        barrier()
        rtimes = []
        for _ in range(args.steps):
            for iv, v in enumerate(vals, start=1):
                kr.update_obs_value(iv, v)
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            kr.solve()
            e1.record()
            e1.synchronize()
            rtimes.append(e0.elapsed_time(e1))
        barrier()
        rt = sum(rtimes) / 1e3
        if dist is not None:
            t = torch.tensor([rt], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            rt = float(t.item())
        rnn = sum(kr.get_neighbours(iv)[0].astype(np.int64) for iv in range(1, nvar + 1))
        # HBM bytes per re-estimate: per target and variable the weight rows
        # (8 B per neighbour of every variable), the neighbour lists (4 B),
        # nnear, and the estimate written; the observation values (a few MB)
        # are served from L2 and not counted
        rbytes = float(len(slab)) * (nvar * 8 * 1 + 4 * nvar) + float(rnn.sum()) * (8 * nvar + 4)
        rgbs = rbytes / (rt / args.steps) / 1e9
        hbm_gbs_r, hbm_src_r = hbm_peak()
        replay = {"value": ntarget * world * args.steps / rt, "unit": "targets/s", "ms_per_step": rt / args.steps * 1e3,
                  "launches_per_step": kr.phases()["launches"],
                  "roofline": {"bound": "hbm", "achieved": rgbs, "peak": hbm_gbs_r, "unit": "GB/s",
                               "frac": rgbs / hbm_gbs_r, "bytes_per_step": rbytes, "kernel": "k_replay",
                               "peak_source": hbm_src_r}}
        kr.close()
        del kr

    # ---- sequential Gaussian simulation: config 1's observations, a 200 x 200
    # grid, nmax 24, four realisations along a seeded path (rank 0, one GPU)
    sgsim = None
    if not args.no_sgsim and rank == 0 and not W.st:
        from krigekit_b200 import Kriging
        w1 = bw.config1(grid_n=200)
        ob = w1["obs"][0]
        rng = np.random.default_rng(9)
        sg = w1["grid"]
        path = rng.permutation(len(sg)) + 1
        nsim_b = 4
        smp = rng.normal(0, 1, (len(sg), nsim_b))
        spec = w1["vgm"][0][2]

        def sg_setup(k):
            k.set_obs(1, ob["coord"], ob["value"], nmax=24)
            k.set_vgm(1, 1, **spec)
            k.set_grid(sg)
            k.set_search(1)
            k.set_sim(path, smp)
            return k

        ks = sg_setup(Kriging(ndim=2, nvar=1, nsim=nsim_b, seed=3))
        ks.solve()
        ks.profile(True)
        sg_ms = []
        for _ in range(max(1, args.steps)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ks.solve()
            e1.record()
            e1.synchronize()
            sg_ms.append(e0.elapsed_time(e1))
        sims_g, _ = ks.get_results()
        sgsim = {"value": len(sg) * nsim_b / (statistics.median(sg_ms) / 1e3), "unit": "simulated values/s",
                 "ms_per_solve": statistics.median(sg_ms), "targets": len(sg), "nsim": nsim_b, "nmax": 24,
                 "phases_ms": ks.phases(), "workload": "config-1 observations, 200 x 200 grid, sph, seeded path"}
        if not args.no_cpu:
            from oracle.oracle import OracleKriging
            ko = sg_setup(OracleKriging(ndim=2, nvar=1, nsim=nsim_b))
            t0 = time.perf_counter()
            ko.solve()
            tcpu = time.perf_counter() - t0
            so, _ = ko.get_results()
            sgsim["cpu_oracle"] = {"value": len(sg) * nsim_b / tcpu, "seconds": tcpu, "cores": 1,
                                   "kind": "port (sequential, as the reference runs SGSIM)"}
            sgsim["max_abs_diff_vs_oracle"] = float(np.nanmax(np.abs(np.asarray(sims_g) - so)))
        ks.close()
        del ks

    # ---- roofline of the dominant kernel (the factorisation kernels)
    peaks = measured_peaks(torch, dev)
    p_aug, q_rhs = W.pq()
    nn = nnear[nnear >= 2].astype(np.float64)
    flops = float(solve_flops(nn, p_aug, q_rhs).sum())
    # the factorisation launches alone (CUDA events around each launch in the
    # profiled solve), not the whole solve phase with the assembly
    factor_ms = ph32["factor_ms"] if ph32.get("factor_ms", 0.0) > 0 else ph32["solve_ms"]
    achieved = flops / (factor_ms / 1e3) / 1e12
    hbm_gbs, hbm_src = hbm_peak()
    # search: algorithmic bytes = target coords + neighbour gathers (8*(coords+1) per neighbour) + list write
    ncoord = w["ndim"] + (1 if W.st else 0)
    search_bytes = len(slab) * 8 * ncoord + float(nn.sum()) * (8 * (ncoord + 1) + 4) + len(slab) * 4 * nvar
    search_gbs = search_bytes / (ph32["search_ms"] / 1e3) / 1e9
    ncu_known = args.config == 2 and args.grid in (None, 2000) and args.nmax is None

    # ---- CPU baseline (oracle on a bounded sample) + accuracy against it
    cpu = None
    acc = None
    if rank == 0 and not args.no_cpu:
        r = cpu_sample_run(W, os.cpu_count() or 1, args.cpu_seconds)
        o = r["oracle"]
        lo, hi = r["lo"], r["hi"]
        oe, ov = o.get_results()
        ee = bw.rel_err(np.asarray(e32)[lo:hi], oe, 1e-3 * w["zstd"])
        ve = bw.rel_err(np.asarray(v32)[lo:hi], ov, 1e-3 * w["sill"])
        same = True
        for iv, (nn_g, in_g) in enumerate(nb32):
            same = same and bool(np.array_equal(nn_g[lo:hi], o.nnear[:, iv]))
            if same:
                m = min(in_g.shape[1], o.inear.shape[2])
                same = bool(np.array_equal(in_g[lo:hi, :m], o.inear[:, iv, :m]))
        acc = {"vs_oracle_sample": f"targets {lo}..{hi}", "est_max": float(ee.max()),
               "est_p99": float(np.percentile(ee, 99)), "var_max": float(ve.max()),
               "var_p99": float(np.percentile(ve, 99)), "neighbour_sets_identical": same}
        cpu = {"value": r["rate"], "unit": "targets/s", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"targets {lo}..{hi} of the {ntarget} targets, all {nobs} observations, "
                         f"{r['seconds']:.1f} s (oracle/kk_oracle.c, OpenMP dynamic,1, 64-slot factor cache)"}

    # ---- end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        k = W.product("fp32_refine", idx=slab)
        io = {}

        def e2e_step():
            io["h2d"] = W.set_data(k, slab)
            k.solve()
            est, var = k.get_results()
            io["d2h"] = np.asarray(est).nbytes + np.asarray(var).nbytes
            return est, var

        for _ in range(max(1, args.warmup - 1)):
            e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        torch.cuda.synchronize()
        te = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([te], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            te = float(t.item())
        e2e = {"value": ntarget * world * args.steps / te, "unit": "targets/s",
               "h2d_bytes_per_step": int(io["h2d"]), "d2h_bytes_per_step": int(io["d2h"]),
               "ms_per_step": te / args.steps * 1e3,
               "note": "pageable numpy inputs through set_obs/set_grid/set_search/solve/get_results"}
        del k

    if rank == 0:
        cfg = workload_config(W)
        cfg.update({"precision": args.precision, "l2": "flushed (256 MiB write) between timed steps",
                    "parallelism": f"targets sharded per rank, {ntarget} per GPU (weak), {world} GPU(s)"})
        line = {
            "metric": METRIC, "value": value, "unit": "targets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot32 / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 factor + f64 refinement" if args.precision == "fp32_refine" else "f64",
            "data": "synthetic (seeded, see bench_workloads.py)",
            "config": cfg,
            "fp64_plain": fp64,
            "speedup_fp32r_vs_fp64": (value / fp64["value"]) if fp64 else None,
            "auto_default": auto,
            "replay": replay,
            "sgsim": sgsim,
            "kernel_plan": k32_plan,
            "accuracy": acc,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peaks["fp32"], "unit": "TFLOP/s",
                         "frac": achieved / peaks["fp32"],
                         "traffic": NCU_DRAM_BYTES_PER_TARGET["solve_fp32_refine"] * ntarget if ncu_known else None,
                         "traffic_note": ("ncu DRAM bytes per target (400x400 grid) x targets of the solve"
                                          if ncu_known else "no ncu capture of this workload"),
                         "kernel": "factorisation launches of the plan (k_solve_warp / k_solve_block), "
                                   "CUDA-core arithmetic",
                         "peak_source": "cuBLAS SGEMM 8192^3, TF32 off, measured live",
                         "flops_per_solve": flops, "factor_ms": factor_ms,
                         "frac_of_fp64_peak": achieved / peaks["fp64"],
                         "solve_ms": ph32["solve_ms"]},
            "roofline_search": {"bound": "hbm", "achieved": search_gbs, "peak": hbm_gbs, "unit": "GB/s",
                                "frac": search_gbs / hbm_gbs,
                                "traffic": NCU_DRAM_BYTES_PER_TARGET["search"] * ntarget if ncu_known else None,
                                "kernel": "k_search<768>", "peak_source": hbm_src,
                                "search_ms": ph32["search_ms"]},
            "peaks_measured_tflops": peaks,
            "phases_ms": ph32, "gpu_stats": gst,
            "gpu_launches": int(ph32["launches"] * args.steps),
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


if __name__ == "__main__":
    main()
