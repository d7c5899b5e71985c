#!/usr/bin/env python
"""Benchmark: batched stiff-chemistry BDF on B200, cells/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload gri_1m]
                    [--precision mixed|fp64] [--form persistent|step]
                    [--scaling weak|strong] [--impl reference] [--serving-only]

A "step" integrates one full batch of the workload (every cell from t=0 to dt)
from the same seeded initial state.  Default workload: GRI-Mech 3.0,
1,048,576 cells, P ~ U[1,40] atm, T0 ~ U[900,2400] K, phi ~ U[0.4,2.5],
dt = 1e-4 s, rtol 1e-6 / atol 1e-10, mixed precision, persistent kernel
(the 1M-cell mixed-precision configuration whose target is >= 2x the plain
FP64 one-launch-per-step form on the same GPU).

Beside the device-timed value the line carries: the same metric end to end
through the C ABI with host buffers (e2e); the plain FP64 one-launch-per-step
form on the same cells; the error against the FP64 oracle and the GPU/CPU
agreement at the same tolerances; the CPU integrator (reference pyJac C
chemistry + CVODE-semantics BDF) timed serially and with OpenMP on the host
cores; the FP64/FP32-pipe roofline of the BDF kernel; the serving loop on a
stream of small requests; SM clocks during the timed region.

Multi-GPU (torchrun): --scaling weak (default): every rank integrates its own
seeded batch of the same size; --scaling strong: the one workload is split
into cost-balanced contiguous ranges (hpc_ode_b200.shard), one per rank.  No
collective on the data path; the timed region is bracketed by a barrier and
the max over ranks is reported.

``--impl reference`` times the reference-semantics CPU integrator (the
oracle's CVODE-semantics BDF with the reference's own pyJac C kernels when they
were compiled into oracle/_ref, else the oracle's restated chemistry) on the
host cores, rank 0 only.  ``--serving-only`` runs the serving loop alone at
the offered loads given (p50/p99 over many small requests).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from hpc_ode_b200 import shard, workloads as W  # noqa: E402

L2_FLUSH_BYTES = 256 << 20
# DRAM bytes per cell of one k_bdf launch, from ncu (dram__bytes_read.sum +
# dram__bytes_write.sum of one mixed-precision capture, divided by its cells):
# the traffic is the compulsory T/P/Y in + T/Y/status out, the mechanism tables
# once and register-spill write-backs, taken to scale with the cell count (the
# kerosene capture, one cell per SM, is table-dominated and is not scaled).
# Values: (bytes, summary file).
NCU_DRAM_BYTES_PER_CELL = {
    "gri30": (1157.0, "profiles/k_bdf_gri8k_mixed_full.txt"),
    "h2o2": (148.0, "profiles/k_bdf_h2_32k_mixed_sections.txt"),
    "nDodecane_Reitz": (3934.0, "profiles/k_bdf_nc12_1k_mixed_sections.txt"),
}
# Warp instructions per cell-step of the same captures (smsp__inst_executed.sum /
# (cells x BDF steps per cell)): scaled by the run's own step count, issued
# instructions against the SMs' peak issue rate.
NCU_WARP_INSTR_PER_CELL_STEP = {
    ("gri30", "mixed"): (25.293e9 / (8192 * 132.98), "profiles/k_bdf_gri8k_mixed_full.txt"),
    ("h2o2", "mixed"): (122.29e9 / (32768 * 558.06), "profiles/k_bdf_h2_32k_mixed_sections.txt"),
    ("nDodecane_Reitz", "mixed"): (22.700e9 / (1024 * 551.23), "profiles/k_bdf_nc12_1k_mixed_sections.txt"),
    (W.ESTIMATE, "mixed"): (27.519e9 / (148 * 662.09), "profiles/k_bdf_kero148_mixed_sections.txt"),
}
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
CPU_SAMPLE = {"gri_1m": 4096, "gri_bimodal": 8192, "gri_32k": 8192, "h2_1024": 1024, "h2li_grid": 4096,
              "nc12_8k": 512, "kero_2k": 64}


def _dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def sample_index(n: int, ncells: int) -> np.ndarray:
    """Stratified sample: every (n // ncells)-th cell, ncells of them."""
    stride = max(1, n // max(1, ncells))
    return np.arange(0, n, stride)[:ncells]


def cpu_reference(batch: W.Batch, ncells: int, threads: int, conv: bool = False):
    """One timed pass of the reference-semantics CPU integrator over a
    stratified sample of the batch."""
    from oracle import pyoracle
    o = pyoracle.get()
    idx = sample_index(batch.ncells, ncells)
    sub = batch.subset(idx)
    use_ref = o.has_ref() and batch.mech == "gri30" and not conv   # the reference pyJac is CONP
    t0 = time.perf_counter()
    _, st = o.bdf(sub.mech, sub.state_rows(), sub.P, sub.dt, rtol=W.RTOL, atol=W.ATOL,
                  threads=threads, use_ref_kernels=use_ref, conv=conv)
    el = time.perf_counter() - t0
    kind = "reference" if use_ref else "port"
    what = ("CVODE-semantics BDF (oracle/bdf_oracle.c) + reference pyJac C RHS/Jacobian"
            if use_ref else "CVODE-semantics BDF + restated chemistry (oracle)")
    return len(idx), el, kind, what, st


def cpu_baseline_block(batch: W.Batch, sample: int, conv: bool = False, passes: int = 5) -> dict:
    """The CPU integrator on the host cores: OpenMP over all cores (schedule
    dynamic, 1; the reference's CVodeIntegratorOMP) as the baseline value, and
    serial (one core; the reference's CVodeIntegrator) beside it.  Each a
    warm-up pass then the median of `passes` timed passes over the same
    stratified sample."""
    threads = os.cpu_count() or 1
    cpu_reference(batch, max(64, sample // 8), threads, conv=conv)          # warm-up
    runs = [cpu_reference(batch, sample, threads, conv=conv) for _ in range(passes)]
    n, kind, what = runs[0][0], runs[0][2], runs[0][3]
    omp = n / float(np.median([r[1] for r in runs]))
    ser_n = max(32, sample // 16)
    cpu_reference(batch, 16, 1, conv=conv)
    sruns = [cpu_reference(batch, ser_n, 1, conv=conv) for _ in range(passes)]
    serial = sruns[0][0] / float(np.median([r[1] for r in sruns]))
    return {"value": omp, "unit": "cells/s", "cores": threads, "kind": kind,
            "sample": f"{n} of {batch.ncells} cells (every {max(1, batch.ncells // sample)}th), {what}; "
                      f"OpenMP dynamic,1 on {threads} threads, warm-up + median of {passes} passes",
            "serial": {"value": serial, "unit": "cells/s", "cores": 1,
                       "sample": f"{sruns[0][0]} cells, one thread, warm-up + median of {passes} passes"}}


def run_reference_arm(args):
    ws, rank, _ = _dist_env()
    if rank != 0:
        return 0
    batch = W.make(args.workload)
    threads = os.cpu_count() or 1
    sample = args.cpu_sample or CPU_SAMPLE.get(args.workload, 4096)
    conv = args.formulation == "conv"
    for _ in range(args.warmup):
        cpu_reference(batch, max(64, sample // 8), threads, conv=conv)
    times = []
    n_done = 0
    kind = what = None
    for _ in range(args.steps):
        n, el, kind, what, _ = cpu_reference(batch, sample, threads, conv=conv)
        times.append(el)
        n_done += n
    total = sum(times)
    val = n_done / total
    line = {
        "impl": "reference", "metric": "cells_per_sec", "value": val, "unit": "cells/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "ncells": batch.ncells, "mechanism": batch.mech,
                   "dt": batch.dt, "rtol": W.RTOL, "atol": W.ATOL, "sample_cells_per_step": sample},
        "cpu_baseline": {"value": val, "unit": "cells/s", "cores": threads, "kind": kind,
                         "sample": f"{sample} of {batch.ncells} cells per step (every "
                                   f"{max(1, batch.ncells // sample)}th), {what}, OpenMP dynamic,1"},
        "e2e": {"value": val, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def accuracy_block(batch: W.Batch, T_gpu: np.ndarray, Y_gpu: np.ndarray, nsample: int = 256,
                   conv: bool = False) -> dict:
    """On a stratified sample of cells: the GPU result's error against the FP64
    oracle (the CVODE-semantics BDF at rtol 1e-10 / atol 1e-14) beside the CPU
    integrator's at the same rtol/atol as the GPU, and the GPU against that CPU
    integrator (the agreement the parity gates judge)."""
    from oracle import pyoracle
    o = pyoracle.get()
    idx = sample_index(batch.ncells, nsample)
    sub = batch.subset(idx)
    threads = os.cpu_count() or 1
    ytrue, st_true = o.bdf(sub.mech, sub.state_rows(), sub.P, sub.dt, rtol=1e-10, atol=1e-14, threads=threads,
                           conv=conv)
    ycpu, st_cpu = o.bdf(sub.mech, sub.state_rows(), sub.P, sub.dt, rtol=W.RTOL, atol=W.ATOL, threads=threads,
                         conv=conv)
    Tg, Yg = T_gpu[idx], Y_gpu[:-1, idx].T

    def gate(Ya, Yb):
        return np.abs(Ya - Yb) <= np.maximum(1e-4 * np.abs(Yb), 1e-10)

    eT = np.abs(Tg - ytrue[:, 0]) / ytrue[:, 0]
    eTc = np.abs(ycpu[:, 0] - ytrue[:, 0]) / ytrue[:, 0]
    eTgc = np.abs(Tg - ycpu[:, 0]) / ycpu[:, 0]
    eY = np.abs(Yg - ytrue[:, 1:])
    eYc = np.abs(ycpu[:, 1:] - ytrue[:, 1:])
    return {"oracle": "CVODE-semantics BDF, FP64, rtol 1e-10 atol 1e-14", "cells": int(idx.size),
            "gate": "|dT|/T <= 1e-5; |dY| <= max(1e-4 |Y|, 1e-10)",
            "gpu_T_rel_max": float(eT.max()), "gpu_T_rel_p99": float(np.quantile(eT, 0.99)),
            "gpu_Y_within_gate": float(gate(Yg, ytrue[:, 1:]).mean()),
            "gpu_Y_abs_max": float(eY.max()),
            "cpu_T_rel_max": float(eTc.max()), "cpu_Y_within_gate": float(gate(ycpu[:, 1:], ytrue[:, 1:]).mean()),
            "cpu_Y_abs_max": float(eYc.max()),
            "gpu_vs_cpu_same_tol": {"T_rel_max": float(eTgc.max()), "T_rel_p99": float(np.quantile(eTgc, 0.99)),
                                    "Y_within_gate": float(gate(Yg, ycpu[:, 1:]).mean()),
                                    "T_within_gate": float((eTgc <= 1e-5).mean())},
            "oracle_failed": int((st_true["status"] != 0).sum()), "cpu_failed": int((st_cpu["status"] != 0).sum())}


def serving_block(native, device: int, n_requests: int, load: float, seed: int = 4,
                  chunk_cells: int = 32768, min_cells: int = 1024, max_cells: int = 4096,
                  calib: int = 64) -> dict:
    """Serving loop under Poisson arrivals: requests of the serving workload
    (log-uniform [min_cells, max_cells] cells, 60 % H2 / 40 % GRI, dt in
    {1e-5, 1e-4}) are submitted at exponential inter-arrival times with rate
    load x the measured saturation request rate; latency is submit -> results in
    the caller's host buffers (measured by the library's dispatcher thread).
    Requests larger than chunk_cells run as consecutive launches of at most
    that many cells."""
    cal = list(W.serving_requests(calib, seed=seed + 1, min_cells=min_cells, max_cells=max_cells))
    reqs = list(W.serving_requests(n_requests, seed=seed, min_cells=min_cells, max_cells=max_cells))
    srv = native.Server(max_inflight=4, device=device, chunk_cells=chunk_cells)
    try:
        # saturation: the calibration requests submitted at once, twice; the first
        # pass warms the server's handles and staging, the second is timed
        for _ in range(2):
            t0 = time.perf_counter()
            ids = [srv.submit(b.mech, b.T.copy(), np.ascontiguousarray(b.Y.copy()), b.P, b.dt) for b in cal]
            for r in ids:
                srv.poll(r, -1)
            sat = len(cal) / (time.perf_counter() - t0)
        rate = load * sat
        rng = np.random.default_rng(seed + 7)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
        bufs = [(b.T.copy(), np.ascontiguousarray(b.Y.copy())) for b in reqs]
        pending, infos = [], []
        start = time.perf_counter()
        for b, (T, Y), ta in zip(reqs, bufs, arrivals):
            while True:
                now = time.perf_counter() - start
                pending = [r for r in pending if not _take(srv, r, infos)]
                if now >= ta:
                    break
                time.sleep(min(0.002, ta - now))
            pending.append(srv.submit(b.mech, T, Y, b.P, b.dt))
        for r in pending:
            st, info = srv.poll(r, -1)
            infos.append(info)
        span = time.perf_counter() - start
        lat = np.array([i["latency_ms"] for i in infos])
        cells = int(sum(i["n_cells"] for i in infos))
        rep = srv.report()
        return {"requests": len(infos), "offered_load": load, "saturation_req_per_s": sat,
                "p50_latency_ms": float(np.percentile(lat, 50)), "p99_latency_ms": float(np.percentile(lat, 99)),
                "max_latency_ms": float(lat.max()), "mean_queue_ms": float(np.mean([i["queue_ms"] for i in infos])),
                "cells_per_sec": cells / span, "cells": cells, "max_concurrent": rep["max_concurrent"],
                "failed_cells": int(sum(i["n_failed"] for i in infos)),
                "chunk_cells": chunk_cells,
                "workload": f"log-uniform {min_cells}-{max_cells} cells, 60 % H2 (h2_1024 dists) / 40 % GRI "
                            "(gri_32k dists), dt in {1e-5, 1e-4} s, Poisson arrivals, host buffers"}
    finally:
        srv.close()


def _take(srv, rid, infos) -> bool:
    r = srv.poll(rid, 0)
    if r is None:
        return False
    infos.append(r[1])
    return True


def pipe_roofline(native, mech: str, precision: str, st: dict, kernel_ms: float, dev: int, peaks: dict) -> dict:
    """The governing roofline of the BDF kernel: its algorithmic FP64 and FP32
    work (the op counts of hpc_ode_b200.roofline times the run's own counters)
    against the measured FP64 and FP32 FMA peaks.  frac = (time the two pipes
    would need at peak) / (measured kernel time); achieved and peak are the
    corresponding flop rates (peak = the two-pipe rate for this mix)."""
    from hpc_ode_b200.roofline import flops_by_pipe
    f64, f32 = flops_by_pipe(mech, st, mixed=(precision == "mixed"))
    p64 = native.fp64_peak_gflops(dev) * 1e9
    p32 = native.fp32_peak_gflops(dev) * 1e9
    t_s = kernel_ms * 1e-3
    t_pipes = f64 / p64 + f32 / p32
    achieved = (f64 + f32) / t_s / 1e12
    peak = (f64 + f32) / t_pipes / 1e12
    return {"bound": "fp64+fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": None,
            "fp64": {"flops_per_step": f64, "achieved_tflops": f64 / t_s / 1e12, "peak_tflops": p64 / 1e12,
                     "frac": f64 / t_s / p64},
            "fp32": {"flops_per_step": f32, "achieved_tflops": f32 / t_s / 1e12, "peak_tflops": p32 / 1e12,
                     "frac": f32 / t_s / p32},
            "peak_source": "measured FMA microkernels on this GPU (b200ode_fp64_peak, b200ode_fp32_peak)",
            "work": "per-cell counters x op counts of the generated code (exp/log/pow as one op each)"}


def serving_only(args) -> int:
    from hpc_ode_b200 import native
    out = []
    for load in args.serving_loads:
        out.append(serving_block(native, 0, args.serving_requests, load, chunk_cells=args.serving_chunk,
                                 min_cells=args.serving_min_cells, max_cells=args.serving_max_cells))
        print(json.dumps(out[-1]), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="gri_1m", choices=sorted(W.WORKLOADS))
    ap.add_argument("--ncells", type=int, default=None, help="override cells per GPU (weak) or in all (strong)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--form", default="persistent", choices=["persistent", "step"])
    ap.add_argument("--formulation", default="conp", choices=["conp", "conv"],
                    help="constant pressure (the reference's) or constant volume")
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"])
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="cells of the workload the CPU baseline integrates per pass (0 = per-workload default)")
    ap.add_argument("--e2e-steps", type=int, default=2, help="timed end-to-end calls (after one warm-up call)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the autotuner (launch shape, threads per cell, queue chunk) before warm-up")
    ap.add_argument("--accuracy-cells", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-fp64-step", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serving-only", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=1000)
    ap.add_argument("--serving-load", type=float, default=0.8)
    ap.add_argument("--serving-loads", type=float, nargs="+", default=[0.5, 0.8, 0.95])
    ap.add_argument("--serving-min-cells", type=int, default=1024)
    ap.add_argument("--serving-max-cells", type=int, default=4096)
    ap.add_argument("--serving-chunk", type=int, default=32768,
                    help="cells per launch of a serving request (larger requests run in chunks)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.serving_only:
        return serving_only(args)

    import torch
    ws, rank, local = _dist_env()
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    else:
        dist = None
    dev = torch.device("cuda", local if ws > 1 else 0)
    from hpc_ode_b200 import native

    cfg = W.WORKLOADS[args.workload]
    if args.scaling == "strong":
        # one workload for the whole job; this rank's cost-balanced contiguous range
        full = W.make(args.workload, args.ncells or cfg["ncells"], seed=cfg["seed"])
        a, b_ = shard.rank_range(full.T, ws, rank)
        batch = full.subset(np.arange(a, b_))
        total_cells = full.ncells
    else:
        batch = W.make(args.workload, args.ncells or cfg["ncells"], seed=cfg["seed"] + 1000 * rank)
        total_cells = ws * batch.ncells
    n = batch.ncells
    # the CPU baseline first, in a process that has not yet touched the GPU
    # (as the reference arm's process)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_block(batch, args.cpu_sample or CPU_SAMPLE.get(args.workload, 4096),
                                 conv=args.formulation == "conv")
    prec = native.B200ODE_MIXED if args.precision == "mixed" else native.B200ODE_FP64
    form = native.B200ODE_CONV if args.formulation == "conv" else native.B200ODE_CONP
    solver = native.Solver(batch.mech, precision=prec, persistent=int(args.form == "persistent"),
                           device=dev.index, formulation=form)
    nsp = solver.nsp
    T0 = torch.from_numpy(batch.T).to(dev)
    Y0 = torch.from_numpy(np.ascontiguousarray(batch.Y)).to(dev)
    P = torch.from_numpy(batch.P).to(dev)
    T = torch.empty_like(T0)
    Y = torch.empty_like(Y0)
    status = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    tuned = None
    if not args.no_autotune and args.form == "persistent" and n > 0:
        # the autotuner times its candidates on a sample of these cells (left
        # unmodified) and keeps the fastest in the solver's options
        t_at = time.perf_counter()
        solver.autotune(n, P.data_ptr(), 0.0, T0.data_ptr(), Y0.data_ptr(), batch.dt)
        o = solver.options()
        tuned = {"warps_per_block": o.warps_per_block,
                 "blocks_per_sm": o.blocks_per_sm, "queue_chunk": o.queue_chunk, "cta_helpers": o.cta_helpers,
                 "seconds": time.perf_counter() - t_at}
    opts_used = solver.options()

    def one_step(stats=False):
        T.copy_(T0)
        Y.copy_(Y0)
        return solver.integrate_device(n, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), batch.dt,
                                       dstatus=status.data_ptr(), stream=stream.cuda_stream,
                                       want_stats=stats)

    for _ in range(args.warmup):
        one_step()
        flush.zero_()
    st = one_step(stats=True)   # counters for the roofline
    torch.cuda.synchronize(dev)
    n_fail = int((status[:n] != 0).sum().item())

    clocks = ClockSampler(dev.index)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    ev0.record(stream)
    for k in range(args.steps):
        flush.zero_()                      # L2 flush between timed steps
        T.copy_(T0)
        Y.copy_(Y0)
        kev[k][0].record(stream)
        solver.integrate_device(n, P.data_ptr(), 0.0, T.data_ptr(), Y.data_ptr(), batch.dt,
                                dstatus=status.data_ptr(), stream=stream.cuda_stream,
                                want_stats=False)
        kev[k][1].record(stream)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    elapsed_ms = ev0.elapsed_time(ev1)
    kernel_ms = float(np.mean([a.elapsed_time(b) for a, b in kev]))
    if dist:
        t = torch.tensor([elapsed_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    ms_per_step = elapsed_ms / args.steps
    value = total_cells / (ms_per_step * 1e-3)

    # ---- end-to-end through the C ABI with pinned host buffers (one warm-up call)
    e2e = None
    if not args.no_e2e:
        hT = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
        hY = torch.empty((nsp, n), dtype=torch.float64, pin_memory=True).numpy()
        hP = torch.from_numpy(batch.P.copy()).pin_memory().numpy()
        hst = torch.empty(max(n, 1), dtype=torch.int32, pin_memory=True).numpy()
        e2e_steps = max(1, min(args.steps, args.e2e_steps))
        for it in range(e2e_steps + 1):
            hT[:] = batch.T
            hY[:] = batch.Y
            if it == 1:
                if dist:
                    dist.barrier()
                torch.cuda.synchronize(dev)
                w0 = time.perf_counter()
            native._check(solver.lib.b200ode_integrate(
                solver.h, n, native._ptr(hP), 0.0, native._ptr(hT), native._ptr(hY), 0.0, batch.dt,
                hst.ctypes.data_as(native._i32p), None))
        w1 = time.perf_counter()
        e2e_ms = (w1 - w0) * 1e3 / e2e_steps
        if dist:
            t = torch.tensor([e2e_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": total_cells / (e2e_ms * 1e-3), "unit": "cells/s",
               "h2d_bytes_per_step": int(n * (nsp + 2) * 8),
               "d2h_bytes_per_step": int(n * (nsp + 1) * 8 + n * 4),
               "ms_per_step": e2e_ms, "steps": f"1 warm-up + {e2e_steps} timed calls"}

    # ---- rooflines of the dominant kernel (the persistent BDF kernel)
    peaks = {}
    if os.path.exists(PEAKS_PATH):
        with open(PEAKS_PATH) as f:
            peaks = json.load(f)
    try:
        roofline = pipe_roofline(native, batch.mech, args.precision, st, kernel_ms, dev.index, peaks)
    except Exception as e:  # noqa: BLE001
        roofline = {"bound": "fp64+fp32", "error": str(e)}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    alg_bytes = n * ((nsp + 1) * 8 + 8) + n * ((nsp + 1) * 8 + 4)   # T,Y,P in; T,Y,status out
    per_cell, dram_src = NCU_DRAM_BYTES_PER_CELL.get(batch.mech, (None, None))
    traffic = per_cell * n if per_cell else None
    roofline["traffic"] = traffic
    roofline["hbm"] = {"achieved_gbs": alg_bytes / (kernel_ms * 1e-3) / 1e9, "peak_gbs": hbm_peak,
                       "frac": alg_bytes / (kernel_ms * 1e-3) / 1e9 / hbm_peak, "alg_bytes": alg_bytes,
                       "traffic_bytes": traffic,
                       "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_bdf "
                                          "launch (%s), per cell, scaled by cells" % dram_src
                                          if per_cell else None),
                       "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks
                                       else "fallback 6,650 GB/s (MEASURED_PEAKS.json absent)")}
    issue = None
    ipcs, ipcs_src = NCU_WARP_INSTR_PER_CELL_STEP.get((batch.mech, args.precision), (None, None))
    if ipcs and st:
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
        peak_issue = 4 * sms * mhz * 1e6            # one warp instruction per scheduler per cycle
        ach = ipcs * st["total_nst"] / (kernel_ms * 1e-3)
        issue = {"achieved_warp_inst_per_s": ach, "peak_warp_inst_per_s": peak_issue, "frac": ach / peak_issue,
                 "source": "warp instructions per cell-step from ncu smsp__inst_executed.sum "
                           "(%s) x this run's BDF steps / CUDA-event kernel "
                           "time; peak = 4 schedulers x SMs x median SM clock" % ipcs_src}

    # ---- the plain FP64 one-launch-per-step form on the same cells (the
    # comparison the mixed persistent form is measured against); one GPU only
    fp64_step = None
    ref = None
    if ws == 1 and not args.no_fp64_step and args.precision == "mixed" and args.form == "persistent":
        try:
            ref = native.Solver(batch.mech, precision=native.B200ODE_FP64, persistent=0, device=dev.index,
                                formulation=form)
        except native.B200Error as e:   # e.g. a Newton matrix too large for FP64 in shared memory
            fp64_step = {"unavailable": str(e)}
    if ref is not None:
        Ts, Ys = torch.empty_like(T0), torch.empty_like(Y0)
        m = min(n, 8192)   # warm-up on the first cells (loads the kernels, sizes the records)
        Ts[:m].copy_(T0[:m])
        Ys2 = Y0[:, :m].contiguous()
        ref.integrate_device(m, P.data_ptr(), 0.0, Ts.data_ptr(), Ys2.data_ptr(), batch.dt,
                             stream=stream.cuda_stream, want_stats=False)
        Ts.copy_(T0)
        Ys.copy_(Y0)
        flush.zero_()
        torch.cuda.synchronize(dev)
        a = torch.cuda.Event(enable_timing=True)
        bev = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ref.integrate_device(n, P.data_ptr(), 0.0, Ts.data_ptr(), Ys.data_ptr(), batch.dt,
                             stream=stream.cuda_stream, want_stats=False)
        bev.record(stream)
        torch.cuda.synchronize(dev)
        fp64_ms = a.elapsed_time(bev)
        ref.close()
        fp64_step = {"value": n / (fp64_ms * 1e-3), "unit": "cells/s", "ms_per_step": fp64_ms,
                     "form": "FP64 Newton matrix, one launch per BDF step, state in HBM between launches",
                     "steps": f"warm-up on {m} cells + 1 timed pass", "mixed_persistent_speedup": fp64_ms / kernel_ms}

    serving = None
    if ws == 1 and not args.no_serving:
        try:
            serving = serving_block(native, dev.index, args.serving_requests, args.serving_load,
                                    chunk_cells=args.serving_chunk, min_cells=args.serving_min_cells,
                                    max_cells=args.serving_max_cells)
        except Exception as e:  # noqa: BLE001
            serving = {"error": str(e)}

    acc = None
    if rank == 0 and not args.no_accuracy:
        try:
            acc = accuracy_block(batch, T.cpu().numpy(), Y.cpu().numpy(), nsample=args.accuracy_cells,
                                 conv=args.formulation == "conv")
        except Exception as e:  # noqa: BLE001
            acc = {"error": str(e)}

    line = {
        "metric": "cells_per_sec", "value": value, "unit": "cells/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": args.scaling, "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f64+f32",
        "data": "synthetic (seeded; stands in for the reference's missing 55,076-cell flame dataset)",
        "config": {"workload": args.workload, "mechanism": batch.mech, "cells_per_gpu": n,
                   "cells_total": total_cells, "dt": batch.dt, "rtol": W.RTOL, "atol": W.ATOL,
                   "precision": args.precision, "form": args.form, "formulation": args.formulation,
                   "l2": "256 MiB memset between timed steps",
                   "parallelism": f"cell shards x{ws} ({args.scaling}), no collective",
                   "launch": {"warps_per_block": opts_used.warps_per_block,
                              "blocks_per_sm": opts_used.blocks_per_sm, "queue_chunk": opts_used.queue_chunk,
                              "autotuned": tuned}},
        "kernel_ms_per_step": kernel_ms,
        "cell_steps_per_sec": (ws if args.scaling == "weak" else 1) * st["total_nst"] / (kernel_ms * 1e-3)
        if st else None,
        "counters_per_cell": {k: st[f"total_{k}"] / max(n, 1) for k in
                              ("nst", "nfe", "nje", "nsetups", "nni", "ncfn", "netf")},
        "failed_cells": n_fail,
        "e2e": e2e,
        "gpu_launches": args.steps * int(st["gpu_launches"]),
        "roofline": roofline,
        "issue_roofline": issue,
        "cpu_baseline": cpu,
        "fp64_step_form": fp64_step,
        "serving": serving,
        "accuracy": acc,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    solver.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
