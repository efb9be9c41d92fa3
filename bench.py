#!/usr/bin/env python3
"""Benchmark of the batched RADM2 ROS-3 chemistry solve on B200.

Metric: chem cell-steps/s -- one cell advanced through one 600 s operator-split
chemistry step.  A benchmark "step" is one such split over every cell of the
workload (default: 1,048,576 cells, 30% night, plain FP64 method, the
operator-split loop replayed as one CUDA graph).  K timed steps are K
consecutive splits (K = 6 is one simulated hour).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one process per GPU; each rank integrates its own
contiguous shard of the global cell index space (weak scaling, no collective on
the data path); time is the max over ranks.  `--impl reference` times the CPU
restatement of the reference's per-cell Rosenbrock on the host cores (the
reference itself does not build with CUDA 12.9) on a bounded sample.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "radm2-solver-multi-gpu_b200"))

import numpy as np  # noqa: E402

# Algorithmic FP64 flops, counted from the emitted mechanism code (radm2_gen.h):
# per step attempt Jac 1272 + diagonal shift 59 + LU 3588 + 3 solves 3777 + stage-2 RHS 1085
# + stage/err-norm vector work 24 x 59; per accepted step the new Fcn0 (1085).
FLOPS_PER_ATTEMPT = 1272 + 59 + 3588 + 3 * 1259 + 1085 + 24 * 59
FLOPS_PER_ACCEPT = 1085
# FP32-LU variant: each stage solve adds `refine` sweeps of Jv (880, FP64) + solve (1259) + 3 x 59.
FLOPS_PER_SWEEP = 3 * (880 + 1259 + 3 * 59)

WORKLOADS = {
    # name: (cells per GPU, seed, generator workload, night fraction, dt)
    "plain-1m": (1048576, 1, "plain", 0.3, 600.0),
    "plain-4k": (4096, 0, "plain", 0.0, 600.0),
    "plain-64k": (65536, 1, "plain", 0.3, 600.0),  # profiling case (same distributions as plain-1m)
    "mixed-4m": (4194304, 2, "mixed", 0.4, 600.0),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain-1m", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32lu"])
    ap.add_argument("--schedule", default="persistent", choices=["static", "persistent"])
    ap.add_argument("--block-threads", type=int, default=0)
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def flops_of(stats, precision, refine):
    att = stats["n_accepted"] + stats["n_rejected"]
    f = att * FLOPS_PER_ATTEMPT + stats["n_accepted"] * FLOPS_PER_ACCEPT
    if precision == "fp32lu":
        f += att * refine * FLOPS_PER_SWEEP
    return float(f)


def cpu_baseline(cells, dt, target_s=12.0, nthreads=0):
    """The oracle (CPU restatement of the reference's per-cell Rosenbrock) on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import radm2b200
    nthreads = nthreads or os.cpu_count() or 1
    atol, rtol = np.ones(59), np.full(59, 1e-3)
    ipar, rpar = radm2b200.default_params(hstart=0.01 * dt)
    ok, p = oracle.params(0.0, dt, atol, rtol, rpar, ipar)
    rc_all = None

    def run(n):
        nonlocal rc_all
        sl = slice(0, n)
        rc = oracle.rconst(cells["JV"][sl], cells["TEMP"][sl], cells["FIX"][sl], cells["RC_N2O5"][sl], nthreads)
        t = time.perf_counter()
        oracle.integrate(cells["VAR"][sl], cells["FIX"][sl], rc, p, nthreads)
        return time.perf_counter() - t

    probe = min(len(cells["TEMP"]), max(256, 8 * nthreads))
    tp = run(probe)
    n = int(min(len(cells["TEMP"]), 65536, max(probe, probe * target_s / max(tp, 1e-3))))
    t = run(n)
    return {"value": n / t, "unit": "cell-steps/s", "cores": nthreads, "kind": "port",
            "sample": "first %d cells of the workload, one %g s split, %d OpenMP threads" % (n, dt, nthreads),
            "seconds": t}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from radm2b200 import inputs
    ncell, seed, wl, night, dt = WORKLOADS[args.workload]
    sample = min(ncell, 65536)
    cells = inputs.make_cells(sample, seed, wl, night)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import radm2b200
    nthreads = os.cpu_count() or 1
    atol, rtol = np.ones(59), np.full(59, 1e-3)
    ipar, rpar = radm2b200.default_params(hstart=0.01 * dt)
    ok, p = oracle.params(0.0, dt, atol, rtol, rpar, ipar)
    rc = oracle.rconst(cells["JV"], cells["TEMP"], cells["FIX"], cells["RC_N2O5"], nthreads)
    # size each step to ~8 s of work on this host
    t = time.perf_counter()
    oracle.integrate(cells["VAR"][:512], cells["FIX"][:512], rc[:512], p, nthreads)
    per_cell = (time.perf_counter() - t) / 512
    n = int(min(sample, max(512, 8.0 / max(per_cell, 1e-9))))
    y = cells["VAR"][:n]
    for _ in range(args.warmup):
        y, _ = oracle.integrate(y, cells["FIX"][:n], rc[:n], p, nthreads)
    t = time.perf_counter()
    for _ in range(args.steps):
        y, _ = oracle.integrate(y, cells["FIX"][:n], rc[:n], p, nthreads)
    el = time.perf_counter() - t
    v = n * args.steps / el
    line = {"impl": "reference", "metric": "chem cell-steps/s", "value": v, "unit": "cell-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "cells": n, "split_s": dt, "method": "ROS-3 FP64, rtol 1e-3"},
            "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": nthreads, "kind": "port",
                             "sample": "first %d cells of %s, %d consecutive %g s splits per step" %
                                       (n, args.workload, args.steps, dt)},
            "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import radm2b200
    from radm2b200 import inputs

    ncell, seed, wl, night, dt = WORKLOADS[args.workload]
    cells = inputs.make_cells(ncell, seed, wl, night, first_cell=rank * ncell)
    prec = radm2b200.PREC_FP32LU if args.precision == "fp32lu" else radm2b200.PREC_FP64
    sched = radm2b200.SCHED_PERSISTENT if args.schedule == "persistent" else radm2b200.SCHED_STATIC
    refine = 1
    solver = radm2b200.Solver(precision=prec, schedule=sched, refine_sweeps=refine, device=local,
                              block_threads=args.block_threads, blocks_per_sm=args.blocks_per_sm)
    stream = torch.cuda.Stream()
    solver.set_stream(stream.cuda_stream)
    atol, rtol = np.ones(59), np.full(59, 1e-3)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    # ---- device-resident leg: inputs in HBM, K splits as one CUDA graph
    solver.set_cells(cells)
    ld = (ncell + 31) // 32 * 32
    y0 = torch.empty((59, ld), dtype=torch.float64, device="cuda")
    solver.update_rconst()
    solver.get_state_device(y0.data_ptr(), ld)
    for _ in range(args.warmup):
        ipar, rpar = radm2b200.default_params()
        ierr = solver.run_split(1, dt, atol, rtol, rpar, ipar)
        assert ierr == 1, "warm-up IERR %d" % ierr
    solver.set_state_device(y0.data_ptr(), ld)
    solver.set_kernel_timing(True)
    ipar, rpar = radm2b200.default_params()
    solver.run_split(args.steps, dt, atol, rtol, rpar, ipar)  # capture + first replay of the K-split graph
    solver.set_state_device(y0.data_ptr(), ld)
    solver.kernel_time()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ipar, rpar = radm2b200.default_params()
    barrier()
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        ierr = solver.run_split(args.steps, dt, atol, rtol, rpar, ipar)
        ev1.record(stream)
        barrier()
    assert ierr == 1, "IERR %d" % ierr
    el_ms = ev0.elapsed_time(ev1)
    kms, klaunch = solver.kernel_time()
    st = solver.stats()  # last split; totals come from IPAR
    tot = {"n_accepted": int(ipar[13]), "n_rejected": int(ipar[14])}
    flops = flops_of(tot, args.precision, refine)
    if dist:
        t = torch.tensor([el_ms, kms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        el_ms, kms = float(t[0]), float(t[1])
    value = ncell * world * args.steps / (el_ms * 1e-3)

    # ---- end to end through the C ABI with host buffers (pinned)
    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
        hv, hf, ht, hr, hj = (pin(cells[k]) for k in ("VAR", "FIX", "TEMP", "RC_N2O5", "JV"))
        hout = pin(np.empty_like(cells["VAR"]))
        bi = sum(a.nbytes for a in (hv, hf, ht, hr, hj))
        bo = hout.nbytes
        ipar, rpar = radm2b200.default_params()
        solver.set_inputs(hv, hf, ht, hr, hj)
        solver.run_split(1, dt, atol, rtol, rpar, ipar)
        solver.get_state(hout)
        barrier()
        t0 = time.perf_counter()
        cur = hv
        for _ in range(args.steps):
            solver.set_inputs(cur, hf, ht, hr, hj)
            ipar, rpar = radm2b200.default_params()
            ierr = solver.run_split(1, dt, atol, rtol, rpar, ipar)
            solver.get_state(hout)
            assert ierr == 1
            cur = hout
        barrier()
        e2e_s = time.perf_counter() - t0
        if dist:
            t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t[0])
        e2e = {"value": ncell * world * args.steps / e2e_s, "unit": "cell-steps/s",
               "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
               "path": "radm2_set_inputs + radm2_run_split + radm2_get_state, pinned host AoS buffers"}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    fp64_peak, fp32_peak = radm2b200.fma_peak(local)
    per_launch_flops = flops / max(klaunch, 1)
    achieved = per_launch_flops / (kms / max(klaunch, 1) * 1e-3) * 1e-12 if kms > 0 else None
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "solver_dram_traffic.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            tr = json.load(f)
        key = "%s-%s" % (args.precision, args.schedule)
        if key in tr:
            # DRAM bytes per step attempt from one ncu capture (small case), scaled to the
            # attempts of an average launch here: traffic grows with attempts, not cells
            att = (tot["n_accepted"] + tot["n_rejected"]) / max(klaunch, 1)
            traffic = tr[key]["dram_bytes_per_attempt"] * att
    line = {
        "metric": "chem cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-LU/f64",
        "data": "synthetic (seeded per-cell distributions; reference WRF inputs not shipped)",
        "config": {"workload": args.workload, "cells_per_gpu": ncell, "split_s": dt,
                   "method": "ROS-3, rtol 1e-3, atol 1 molec/cm^3, Hstart 0.01*dt",
                   "precision": args.precision, "schedule": args.schedule,
                   "parallelism": "cells sharded over %d GPU(s), no collective" % world,
                   "l2": "inputs (%.1f GB per GPU) larger than L2" % (ncell * 91 * 8 / 1e9),
                   "steps_are": "consecutive 600 s operator splits (K=6 is one simulated hour)"},
        "gpu_launches": 3 * args.steps,
        "roofline": {"bound": "fp64" if args.precision == "fp64" else "fp64+fp32", "achieved": achieved,
                     "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": (achieved / fp64_peak) if achieved else None, "traffic": traffic,
                     "peak_source": "measured CUDA-core FMA microbenchmark (radm2_fma_peak), FP32 %.1f" % fp32_peak,
                     "kernel_ms_per_launch": kms / max(klaunch, 1), "flops_per_launch": per_launch_flops},
        "steps_per_cell": {"accepted": tot["n_accepted"] / ncell / args.steps,
                           "rejected": tot["n_rejected"] / ncell / args.steps},
        "clocks": clocks.summary(),
        "e2e": e2e,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cells, dt)
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
