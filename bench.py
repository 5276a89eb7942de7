#!/usr/bin/env python
"""Benchmark of the B200 Stokes hot path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the level-6 thick spherical shell (10 diamonds x 65 x 65 lateral
nodes x 65 radial nodes, r in [0.55, 1]), viscosity exp of a seeded smooth
field with 10^2 contrast, Dirichlet inner / free-slip outer boundary, seeded
synthetic velocity. One step = one epsilon-div-div operator apply (kernel plus
interface sum) in FP64 over the whole shell. Inputs (154 MB FP64) exceed the
126 MB L2; the L2 is also flushed between timed steps.

With N > 1 (torchrun) each rank runs an independent replica (the path does not
shard); value = all ranks' work / max-over-ranks device time.

--impl reference times the CPU restatement of the reference's fast-path apply
(oracle/, all host threads) on a bounded number of level-6 applies.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "terra-ng_b200"))

METRIC = "L6 Stokes solve time to 1e-8 (FP32-MG vs FP64); op-apply HBM GB/s"
LEVEL = 6
BYTES_PER_NODE = {"f64": 56, "f32": 28}  # src 3 + k 1 read, dst 3 written


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="f64", choices=["f64", "f32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic(name):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(name)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=2)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _cpu_baseline(nthreads=None, budget_s=12.0):
    """Oracle port of the reference's fast-path apply on the host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import oracle as O

    threads = O.set_threads(nthreads or os.cpu_count() or 1)
    sh = O.Shell(LEVEL)
    rng = np.random.default_rng(1)
    k = np.exp(rng.uniform(-1, 1, sh.scalar_shape))
    u = rng.standard_normal(sh.vec_shape)
    op = O.EpsDivDiv(sh, k=k, bc_cmb=O.DIRICHLET, bc_surface=O.FREESLIP)
    op.apply(u, path="fast")  # warm-up
    n, t0 = 0, time.perf_counter()
    while True:
        op.apply(u, path="fast")
        n += 1
        if time.perf_counter() - t0 > budget_s or n >= 40:
            break
    dt = (time.perf_counter() - t0) / n
    nodes = 10 * sh.nl * sh.nl * sh.nr
    gbs = BYTES_PER_NODE["f64"] * nodes / dt / 1e9
    return {"value": gbs, "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"{n} level-6 FP64 applies (oracle fast path, OpenMP), {dt * 1e3:.1f} ms each"}, dt


def run_reference(a):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    cb, dt = _cpu_baseline(budget_s=20.0)
    steps = max(1, min(a.steps, 20))
    line = {"metric": METRIC, "value": cb["value"], "unit": "GB/s", "n_gpus": a.gpus, "steps": steps,
            "warmup": a.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "L6 epsilon-div-div FP64 operator apply (10x65x65x65 nodes), Dirichlet/free-slip"},
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(a):
    import numpy as np
    import torch

    import terra_b200 as T

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    prec = a.precision
    dt_t = torch.float64 if prec == "f64" else torch.float32
    shell = T.Shell(LEVEL)
    nl, nr = shell.dims()
    nodes = 10 * nl * nl * nr
    g = torch.Generator(device=dev).manual_seed(1234 + rank)
    coords = torch.tensor(shell.coords(), device=dev)
    radii = torch.tensor(shell.radii(), device=dev)
    X = coords[:, :, :, None, :] * radii[None, None, None, :, None]
    field = torch.zeros((10, nl, nl, nr), device=dev, dtype=torch.float64)
    for _ in range(6):
        kv = torch.randn(3, generator=g, device=dev, dtype=torch.float64) * 3.0
        ph = torch.rand(1, generator=g, device=dev, dtype=torch.float64) * 6.283185307179586
        field += torch.sin(X @ kv + ph)
    field /= field.abs().max()
    k = torch.exp(np.log(100.0) * 0.5 * field).to(dt_t)
    op = T.EpsDivDiv(shell, k=k, bc_cmb=T.DIRICHLET, bc_surface=T.FREESLIP)
    src = torch.randn((3, 10, nl, nl, nr), generator=g, device=dev, dtype=torch.float64).to(dt_t)
    shell.interface_sum(src)
    dst = torch.zeros_like(src)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    for _ in range(max(a.warmup, 3)):
        op.apply(src, dst)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    for i in range(a.steps):
        flush.zero_()
        ev[i][0].record(stream)
        op.apply(src, dst)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    ck = clocks.stop()
    times = [s.elapsed_time(e) / 1e3 for s, e in ev]
    t_step = sum(times) / len(times)
    t_tensor = torch.tensor([t_step], device=dev, dtype=torch.float64)
    if ws > 1:
        torch.distributed.all_reduce(t_tensor, op=torch.distributed.ReduceOp.MAX)
    t_step = float(t_tensor.item())
    alg_bytes = BYTES_PER_NODE[prec] * nodes
    value = ws * alg_bytes / t_step / 1e9

    # end-to-end through the public API: pinned host input -> device -> apply -> host result
    h_src = src.cpu().pin_memory()
    h_dst = torch.empty_like(h_src).pin_memory()
    e2e_steps = max(3, min(a.steps, 10))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d_src = torch.empty_like(src)
    e0.record(stream)
    for _ in range(e2e_steps):
        d_src.copy_(h_src, non_blocking=True)
        op.apply(d_src, dst)
        h_dst.copy_(dst, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = e0.elapsed_time(e1) / 1e3 / e2e_steps
    io_bytes = src.numel() * src.element_size()

    peak, peak_kind = _peaks()
    kname = f"epsdivdiv_{prec}_L6"
    traffic = _profile_traffic(kname)
    cpu = None
    if rank == 0 and not a.no_cpu_baseline and ws == 1:
        cpu, _ = _cpu_baseline()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": ws, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": prec, "data": "synthetic",
            "config": {"workload": f"L6 epsilon-div-div {prec.upper()} operator apply (10x65x65x65 nodes, "
                                   "Dirichlet inner / free-slip outer, 1e2 viscosity contrast); interface sum included",
                       "l2": "flushed between timed steps (inputs also exceed L2 in FP64)",
                       "replicas": ws},
            "roofline": {"bound": "hbm", "achieved": alg_bytes / t_step / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg_bytes / t_step / 1e9 / peak, "traffic": traffic,
                         "peak_kind": peak_kind, "kernel": "epsdivdiv_kernel + iface_kernel",
                         "algorithmic_bytes_per_launch": alg_bytes},
            "cpu_baseline": cpu,
            "clocks": ck,
            "e2e": {"value": ws * alg_bytes / t_e2e / 1e9, "unit": "GB/s", "h2d_bytes_per_step": io_bytes,
                    "d2h_bytes_per_step": io_bytes, "ms_per_step": t_e2e * 1e3},
            "gpu_launches": 2 * a.steps,
            "mdof_per_s": 3 * (10 * (nl - 1) ** 2 + 2) * nr / t_step / 1e6,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()


def main():
    a = _args()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
