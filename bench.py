#!/usr/bin/env python
"""Benchmark of the B200 Smith-Waterman hot path (banded seed extension).

Workload (one step): config 1 -- the left (reversed prefix) and right
extensions of 5M synthetic 150 bp reads per GPU off a seeded 100 Mbp
reference with 20% of reads from tandem-repeat blocks (~10M extension
tasks), every task bit-exact with BandedSWScalar.align.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value    extensions/s with inputs resident in HBM (swb_ext_batch_device),
         timed with CUDA events on the launching stream, max over ranks.
e2e      the same metric through the C ABI's host entry point
         (swb_ext_batch) from pinned host buffers: H2D of reads + tasks,
         the kernels, D2H of results, every step.
roofline the dominant kernel's algorithmic int ops (13 per DP cell) per
         launch / its average launch time, against the measured int32
         add/max rate of the same GPU (swb_int_alu_peak).
For N > 1 the driver launches one process per GPU (torchrun); each rank
extends its own shard (weak scaling, no data-path collective).
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

OPS_PER_CELL_EXT = 13   # add q, select M!=0, 2 max for H, 2x{sub,max0,sub,max} for E/F, 1 row-max


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n-reads", type=int, default=5_000_000)
    ap.add_argument("--ref-len", type=int, default=100_000_000)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample time")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- helpers
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def traffic_per_launch(kernel: str):
    """Per-launch DRAM bytes (read + write) of `kernel` from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p))
        return d.get(kernel, {}).get("dram_bytes_per_launch_full_workload")
    except Exception:
        return None


def cpu_baseline(wl, sc, seconds: float, gpu_out=None):
    """The oracle (C++ restatement of the reference's CPU code) on a bounded
    sample of the same tasks, all host threads."""
    from oracle import oracle
    threads = os.cpu_count() or 1
    n = len(wl.tasks)
    probe = min(n, 20_000)
    t0 = time.perf_counter()
    oracle.ext_batch(sc, wl.bases, wl.tasks[:probe], pac=wl.ref.pac, ref_bases=wl.ref.n, n_threads=threads)
    rate = probe / max(time.perf_counter() - t0, 1e-6)
    s = int(min(n, max(probe, rate * seconds)))
    t0 = time.perf_counter()
    res, cells = oracle.ext_batch(sc, wl.bases, wl.tasks[:s], pac=wl.ref.pac, ref_bases=wl.ref.n,
                                  n_threads=threads)
    dt = time.perf_counter() - t0
    out = {"value": s / dt, "unit": "ext/s", "cores": threads, "kind": "port",
           "sample": f"first {s} of {n} config-1 extension tasks ({cells} DP cells, {dt:.1f} s)",
           "gcups": cells / dt / 1e9}
    if gpu_out is not None:
        same = int(np.sum(np.all(np.stack([gpu_out[f][:s] == res[f] for f in res.dtype.names]), axis=0)))
        out["bitexact_sample"] = f"{same}/{s}"
    return out


# --------------------------------------------------------- reference arm
def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from swiftbwa_b200 import workloads as W
    from swiftbwa_b200.abi import Scoring
    from oracle import oracle
    sc = Scoring.default()
    wl = W.config1(rank=0, n_reads=args.n_reads, ref_len=args.ref_len)
    threads = os.cpu_count() or 1
    n = len(wl.tasks)
    probe = min(n, 20_000)
    t0 = time.perf_counter()
    oracle.ext_batch(sc, wl.bases, wl.tasks[:probe], pac=wl.ref.pac, ref_bases=wl.ref.n, n_threads=threads)
    rate = probe / max(time.perf_counter() - t0, 1e-6)
    total_budget = 150.0
    s = int(min(n, max(probe, rate * total_budget / max(args.steps + args.warmup, 1))))
    times, cells_tot = [], 0
    for it in range(args.warmup + args.steps):
        lo = (it * s) % max(n - s, 1)
        t0 = time.perf_counter()
        _, cells = oracle.ext_batch(sc, wl.bases, wl.tasks[lo:lo + s], pac=wl.ref.pac, ref_bases=wl.ref.n,
                                    n_threads=threads)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt)
            cells_tot += cells
    tot = sum(times)
    value = s * len(times) / tot
    line = {"impl": "reference", "metric": "extensions/s (bit-exact banded SW extension, config 1)",
            "value": value, "unit": "ext/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded config-1 generator)",
            "config": {"workload": wl.name, "sample_tasks_per_step": s},
            "gcups": cells_tot / tot / 1e9,
            "cpu_baseline": {"value": value, "unit": "ext/s", "cores": threads, "kind": "port",
                             "sample": f"{s} of {n} config-1 tasks per step, C++ restatement of BandedSWScalar.align, {threads} threads"},
            "e2e": {"value": value, "unit": "ext/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- our arm
def run_ours(args):
    ws, rank, local = dist_env()
    import torch
    dist = None
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    else:
        torch.cuda.set_device(local)
    from swiftbwa_b200 import workloads as W
    from swiftbwa_b200.abi import EXT_RESULT_DTYPE, Scoring
    from swiftbwa_b200.alignment import Engine
    from swiftbwa_b200.build import build
    build()

    sc = Scoring.default()
    t_gen = time.perf_counter()
    wl = W.config1(rank=rank, n_reads=args.n_reads, ref_len=args.ref_len)
    t_gen = time.perf_counter() - t_gen
    n = len(wl.tasks)
    eng = Engine(local)
    eng.upload_reference(wl.ref.pac, wl.ref.n)
    alu_peak = eng.int_alu_peak()

    # HBM-resident inputs (torch only allocates; the library computes).
    dev = torch.device("cuda", local)
    d_bases = torch.from_numpy(wl.bases).to(dev)
    d_tasks = torch.from_numpy(wl.tasks.view(np.uint8)).to(dev)
    d_out = torch.empty(n * EXT_RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    # A dedicated stream: the library's kernels and the timing events both go
    # on it (a NULL handle would select the library's own context stream).
    stream = torch.cuda.Stream(dev)
    torch.cuda.synchronize()

    def step():
        eng.ext_batch_device(sc, d_bases.data_ptr(), d_tasks.data_ptr(), n, d_out.data_ptr(), stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    eng.profile(True)
    eng.profile_reset()
    launches0 = eng.kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - w0) * 1e3 / args.steps
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()
    launches = eng.kernel_launches() - launches0
    prof = eng.profile_read()
    eng.profile(False)
    ms_max = ms
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    gpu_out = d_out.cpu().numpy().view(EXT_RESULT_DTYPE)

    cells_step = sum(v[2] for v in prof.values()) / args.steps
    # The length bins run concurrently on their own streams, so the unit the
    # roofline measures is the whole extension pass: fork to join on the
    # launching stream (one "ext_pass" launch per step), all bins' cells.
    pass_launches, pass_ms, _ = prof["ext_pass"]
    bin_cells = sum(v[2] for k, v in prof.items() if k.startswith("ext_"))
    dom_name = "ext_pass (ext_fast_q32..q256 + ext_global_i32, concurrent bins)"
    achieved = (bin_cells / pass_launches) * OPS_PER_CELL_EXT / (pass_ms / pass_launches * 1e-3)
    step_ms_sum = sum(v[1] for k, v in prof.items() if k in ("ext_keys", "cub_radix_sort", "bin_bounds", "ext_pass"))
    kernels = {k: {"launches": v[0], "ms_per_step": v[1] / args.steps,
                   "share_of_step": (v[1] / step_ms_sum) if k in ("ext_keys", "cub_radix_sort", "bin_bounds", "ext_pass") else None,
                   "cells_per_step": v[2] / args.steps,
                   "gcups_in_own_window": (v[2] / (v[1] * 1e-3) / 1e9) if v[2] else None} for k, v in prof.items()}

    # End to end through the host entry point, pinned host buffers.
    e2e = None
    if not args.no_e2e:
        hb = torch.from_numpy(wl.bases).pin_memory().numpy()
        ht = torch.from_numpy(wl.tasks.view(np.uint8)).pin_memory().numpy().view(wl.tasks.dtype)
        ho = torch.empty(n * EXT_RESULT_DTYPE.itemsize, dtype=torch.uint8).pin_memory().numpy().view(EXT_RESULT_DTYPE)
        eng.ext_batch(sc, hb, ht, out=ho)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            eng.ext_batch(sc, hb, ht, out=ho)
        wall = (time.perf_counter() - t0) / args.steps
        if dist:
            t = torch.tensor([wall], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            wall = float(t.item())
        assert np.array_equal(ho, gpu_out), "host and device entry points disagree"
        e2e = {"value": n * ws / wall, "unit": "ext/s", "h2d_bytes_per_step": int(hb.nbytes + ht.nbytes),
               "d2h_bytes_per_step": int(ho.nbytes), "ms_per_step": wall * 1e3}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(wl, sc, args.cpu_seconds, gpu_out)

    if rank == 0:
        line = {
            "metric": "extensions/s (bit-exact banded SW extension, config 1)",
            "value": n * ws / (ms_max * 1e-3), "unit": "ext/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "wall_ms_per_step": wall_ms,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded config-1 generator: reads, errors, tandem repeats)",
            "config": {"workload": wl.name, "tasks_per_gpu": n, "reads_per_gpu": args.n_reads, "read_len": 150,
                       "ref_bases": wl.ref.n, "w": 100, "h0": 19, "end_bonus": 5,
                       "l2": f"inputs larger than L2 ({(wl.bases.nbytes + wl.tasks.nbytes) / 1e6:.0f} MB read per step)",
                       "parallelism": f"replicas x{ws} (task shards, no collective)"},
            "gcups": cells_step * ws / (ms_max * 1e-3) / 1e9,
            "cells_per_step_per_gpu": cells_step,
            "roofline": {"bound": "alu", "kernel": dom_name, "achieved": achieved / 1e12,
                         "avg_launch_ms": pass_ms / pass_launches,
                         "peak": alu_peak / 1e12, "unit": "Tops/s (int32 add/max)",
                         "frac": achieved / alu_peak, "traffic": traffic_per_launch("ext_pass"),
                         "ops_per_cell": OPS_PER_CELL_EXT,
                         "peak_source": "measured in this run: swb_int_alu_peak (int32 add/max probe); "
                                        "MEASURED_PEAKS.json has no integer figure"},
            "kernels": kernels,
            "gpu_launches": int(launches),
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gen_seconds": t_gen,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
