#!/usr/bin/env python
"""Benchmark of the B200 Stokes hot path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the level-6 Stokes solve of the reference's mantle-convection app):
thick spherical shell, 10 diamonds x 65 x 65 lateral x 65 radial velocity
nodes (levels 2..6 form the multigrid hierarchy, pressure on level 5), r in
[0.55, 1]; no-slip inner / free-slip outer boundary; viscosity exp(ln 10 *
s(x) * cos(pi (r - 0.55) / 0.45)) from 8 seeded real spherical harmonics of
degree <= 4 (10^2 contrast); buoyancy right-hand side from a seeded
temperature field (harmonics plus N(0, 0.01) noise). FGMRES(30) with the
block-triangular preconditioner (Schur = inverse lumped 1/eta pressure mass,
velocity = one GMG V(2,2) cycle with Chebyshev smoothing of order 3 (the degree
configuration 0 of the workload description names; the application's default
is order 2, which takes 355 iterations here instead of 235), Galerkin coarse operators,
coarsest level 2 solved directly with its inverse formed once at set-up
(--coarse dense; --coarse pcg: the reference's 50-iteration / 1e-6 CG, the
other one is timed once beside it)), relative tolerance 1e-8 with constant
pressure treated as a null vector (see the solver's project_pressure_mean).

One step = one solve from a zero initial guess. value = seconds per solve of
the mixed-precision solver (FP32 V-cycle inside FP64 FGMRES); the plain FP64
solve is timed the same way and reported beside it. The solve reads and
writes well over the 126 MB L2 per iteration (the level-6 vectors alone are
66 MB each). The operator-apply line (roofline) times the dominant kernel,
the FP32 epsilon-div-div apply of the fine level, standalone with an L2 flush
between launches.

With N > 1 (torchrun) each rank solves its own replica (the path has no
exchange step); value = max over ranks of the per-solve time.

--impl reference times the reference's own FP64 code, compiled from its
sources into oracle/_ref (Kokkos OpenMP, all host threads), on a bounded
sample: set-up, one warm-up and five timed FGMRES iterations of the same
level-6 solve, extrapolated to the FP64 iteration count, plus five
fine-level applies.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "terra-ng_b200"))

METRIC = "L6 Stokes solve time to 1e-8 (FP32-MG vs FP64); op-apply HBM GB/s"
LEVEL, NUM_LEVELS = 6, 5
BCS = (1, 2)  # no-slip CMB, free-slip surface
SEED_ETA, SEED_TEMP = 1, 2
BYTES_PER_NODE = {"f64": 56, "f32": 28}  # src 3 + k 1 read, dst 3 written
# FGMRES iterations the FP64 solve of this workload takes to 1e-8 (the bench line's iterations.fp64); the
# reference arm, which runs without the GPU solve, extrapolates its per-iteration time with it, while the
# main arm's cpu_baseline uses the count it has just measured.
FP64_ITERATIONS = 235
# Chebyshev order of the V(2,2) smoother, both arms
CHEB_ORDER = 3
WORKLOAD = ("L6 Stokes solve (10x65x65x65 velocity nodes, pressure on L5, hierarchy L2..L6), no-slip CMB / "
            "free-slip surface, 1e2 viscosity contrast from 8 seeded SH (l<=4) x radial cosine, seeded buoyancy "
            "RHS; FGMRES(30) + block-triangular GMG V(2,2) Chebyshev(3) preconditioner, GCA coarse operators, "
            "FP64 coarsest solve on L2, rtol 1e-8")


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--coarse", default="dense", choices=["dense", "pcg"],
                    help="coarsest-level solve of the timed solvers: dense (the assembled level-2 operator inverted "
                         "once, an exact solve per V-cycle) or pcg (the reference's 50-iteration CG); the other "
                         "one is timed once beside it")
    ap.add_argument("--workload", default="solve", choices=["solve", "apply-f32", "apply-f64", "coupling",
                                                             "precondition", "adjoint-L5", "solve-L7", "gca-build",
                                                             "gca-modes", "solve-profile"],
                    help="solve: the L6 Stokes solve (default); apply-*: the standalone L6 fine-level operator "
                         "apply; coupling: the L6 B and B^T applies (FP64); precondition: one application of the "
                         "L6 mixed-precision block preconditioner; gca-build: the L6 Galerkin hierarchy build, fast "
                         "against plain scalar and adaptive against full; gca-modes: the L6 solve with full, "
                         "adaptive and no GCA; solve-profile: one mixed and one FP64 L6 solve inside NVTX ranges; "
                         "adjoint-L5: the L5 misfit gradient at 1e4 contrast with a finite-difference check; "
                         "solve-L7: the L7 mixed and FP64 solves plus one adjoint gradient")
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
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
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


# ---------------------------------------------------------------------------
# CPU: the reference's own FP64 solve (compiled from its sources into oracle/_ref)
# ---------------------------------------------------------------------------
class _HostShell:
    """coords / radii accessor of an oracle shell for synthetic.viscosity."""

    def __init__(self, sh):
        self.sh = sh

    def coords(self, level):
        return self.sh.coords

    def radii(self, level):
        return self.sh.radii


def _host_temperature(sh, seed=SEED_TEMP, noise=0.01):
    """synthetic.temperature on the host: the same harmonics, and the same seeded uniform pairs (the library's
    SplitMix64 stream, restated in oracle.seeded_uniform) through the same Box-Muller transform."""
    import numpy as np

    import oracle as O
    import synthetic as S

    s = S._harmonic_sum(sh.coords, seed)
    rad = np.sin(math.pi * (sh.radii - sh.radii[0]) / (sh.radii[-1] - sh.radii[0]))
    t = s[..., None] * rad[None, None, None, :]
    u = O.seeded_uniform(sh, 2, seed * 1000003 + 17)
    u1 = np.maximum(0.5 * (u[0] + 1.0), 1e-300)
    u2 = 0.5 * (u[1] + 1.0)
    return t + noise * np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def _reference_sample(iterations, warm=1, applies=5):
    """Times the reference's own FP64 code on the host cores (oracle/_ref, Kokkos OpenMP, every host thread):
    the level-6 Stokes solve of this workload (its set-up, then `warm` FGMRES iterations, in which the
    smoothers estimate their spectra, then `iterations` timed iterations from a zero guess) and `applies`
    fine-level operator applies after one warm-up (median). The right-hand side is assembled by the reference
    (VectorMass, then its boundary treatment) from the same seeded temperature."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import oracle as O
    import ref as R
    import synthetic as S

    if not R.available():
        raise RuntimeError("the compiled reference (oracle/_ref/libterra_ref.so) is not present")
    R.lib()
    sh = O.Shell(LEVEL)
    shp = sh.coarser()
    eta = S.viscosity(_HostShell(sh), 0, seed=SEED_ETA)
    X = sh.physical_coords()
    rhat = X / np.linalg.norm(X, axis=-1, keepdims=True)
    f = R.vector_mass(LEVEL, np.moveaxis(_host_temperature(sh)[..., None] * rhat, -1, 0))
    b = R.rhs_enforce(LEVEL, np.concatenate([f.ravel(), np.zeros(shp.scalar_shape).ravel()]), *BCS)
    shells = [sh]
    for _ in range(NUM_LEVELS - 1):
        shells.insert(0, shells[0].coarser())
    starts = [O.seeded_uniform(shells[l], 3, 12345 + 7919 * l) for l in range(NUM_LEVELS)]
    st = R.StokesRef(LEVEL, NUM_LEVELS, eta, 1.0 / O.inject(shp, eta), start=starts, bc_cmb=BCS[0],
                     bc_surface=BCS[1], cheb_order=CHEB_ORDER)
    _, _, t_warm = st.solve(b, rtol=1e-8, atol=0.0, max_it=warm)
    _, hist, t_solve = st.solve(b, rtol=1e-8, atol=0.0, max_it=iterations)
    st.close()
    t_apply = R.epsdivdiv_time(LEVEL, eta, O.seeded_normal(sh.vec_shape, 3), reps=applies, bc_cmb=BCS[0],
                               bc_surface=BCS[1])
    return {"per_iteration_s": t_solve / iterations, "setup_s": st.setup_seconds, "warm_s": t_warm,
            "apply_s": float(np.median(t_apply)), "threads": R.num_threads(), "iterations": iterations,
            "history": [float(v) for v in hist]}


def _reference_baseline(fp64_iterations, samples=5):
    r = _reference_sample(samples)
    value = r["per_iteration_s"] * fp64_iterations
    sample = (f"reference FP64 code (oracle/_ref: the reference's own operators, GCA, Chebyshev multigrid, PCG, "
              f"block preconditioner and FGMRES, Kokkos OpenMP, {r['threads']} threads): {samples} FGMRES "
              f"iterations of this level-6 solve after set-up ({r['setup_s']:.1f} s) and one warm-up iteration, "
              f"{r['per_iteration_s']:.2f} s each, extrapolated to the {fp64_iterations} iterations the FP64 "
              f"solve of this workload takes to 1e-8 (the reference has no pressure-mean projection; unprojected, "
              f"its residual floors near 3e-8 on this free-slip system, so a full run never reaches 1e-8); "
              f"fine-level apply {r['apply_s'] * 1e3:.0f} ms (median of 5)")
    return {"value": value, "unit": "s/solve", "cores": r["threads"], "kind": "reference", "sample": sample,
            "per_iteration_s": r["per_iteration_s"], "apply_s": r["apply_s"], "setup_s": r["setup_s"]}


def run_reference(a):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    samples = max(5, min(a.steps, 10))
    try:
        cpu = _reference_baseline(FP64_ITERATIONS, samples)
    except Exception as e:  # the library did not travel with the tree
        print(json.dumps({"impl": "reference", "unavailable": f"{type(e).__name__}: {e}"}), flush=True)
        return
    value = cpu["value"]
    line = {"metric": METRIC, "value": value, "unit": "s/solve", "n_gpus": a.gpus, "steps": samples, "warmup": 1,
            "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": {"workload": WORKLOAD}, "impl": "reference",
            "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "reference_per_iteration_s": cpu["per_iteration_s"], "reference_apply_s": cpu["apply_s"],
            "reference_setup_s": cpu["setup_s"], "iterations_extrapolated": FP64_ITERATIONS,
            "e2e": {"value": value, "unit": "s/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _time_apply(T, torch, shell, eta, dtype, steps, flush, level=None, eta_cell=None):
    """Average device time of the standalone fine-level apply (kernel + interface sum)."""
    level = NUM_LEVELS - 1 if level is None else level
    nl, nr = shell.dims(level)
    if eta_cell is not None:
        op = T.EpsDivDiv(shell, level, k_cell=eta_cell.to(dtype), bc_cmb=BCS[0], bc_surface=BCS[1])
    else:
        op = T.EpsDivDiv(shell, level, k=eta.to(dtype), bc_cmb=BCS[0], bc_surface=BCS[1])
    src = T.random_vector(shell, level, 3, 77, dtype=dtype)
    dst = torch.zeros_like(src)
    for _ in range(3):
        op.apply(src, dst)
    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        op.apply(src, dst)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    t = sum(s.elapsed_time(e) for s, e in ev) / steps / 1e3
    nodes = 10 * nl * nl * nr
    return t, nodes


def run_apply(a):
    """The L6 fine-level epsilon-div-div apply alone (the top kernel of the solve), one JSON line."""
    import torch

    import synthetic as S
    import terra_b200 as T

    prec = "f32" if a.workload == "apply-f32" else "f64"
    dt = torch.float32 if prec == "f32" else torch.float64
    shell = T.Shell(LEVEL, num_levels=NUM_LEVELS)
    eta = torch.tensor(S.viscosity(shell, NUM_LEVELS - 1, seed=SEED_ETA), device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(max(3, a.warmup)):
        _time_apply(T, torch, shell, eta, dt, 1, flush)
    t, nodes = _time_apply(T, torch, shell, eta, dt, max(1, a.steps), flush)
    peak, peak_kind = _peaks()
    ach = BYTES_PER_NODE[prec] * nodes / t / 1e9
    print(json.dumps({"metric": "L6 epsilon-div-div apply algorithmic HBM GB/s", "value": ach, "unit": "GB/s",
                      "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": t * 1e3,
                      "higher_is_better": True, "dtype": prec, "data": "synthetic",
                      "config": {"workload": f"L6 epsilon-div-div {prec.upper()} apply + interface sum, no-slip / "
                                             "free-slip, L2 flushed between launches"},
                      "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                   "traffic": _profile_traffic(f"epsdivdiv_{prec}_L6"), "peak_kind": peak_kind}}),
          flush=True)


def _time_device(torch, fn, steps, flush):
    """Mean device seconds of fn() over `steps` launches, L2 flushed before each."""
    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    for s0, s1 in ev:
        flush.zero_()
        s0.record(stream)
        fn()
        s1.record(stream)
    torch.cuda.synchronize()
    return sum(s0.elapsed_time(s1) for s0, s1 in ev) / steps / 1e3


def run_coupling(a):
    """The L6 divergence B (velocity -> L5 pressure) and gradient B^T, FP64, each with its interface sum."""
    import torch

    import terra_b200 as T

    shell = T.Shell(LEVEL, num_levels=NUM_LEVELS)
    fine = NUM_LEVELS - 1
    u = T.random_vector(shell, fine, 3, 5)
    p = T.random_vector(shell, fine - 1, 1, 6)[0].contiguous()
    po, uo = torch.zeros_like(p), torch.zeros_like(u)
    B = T.Divergence(shell, fine, bc_cmb=BCS[0], bc_surface=BCS[1])
    BT = T.Gradient(shell, fine, bc_cmb=BCS[0], bc_surface=BCS[1])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    steps = max(1, a.steps)
    for _ in range(max(3, a.warmup)):
        B.apply(u, po)
        BT.apply(p, uo)
    tb = _time_device(torch, lambda: B.apply(u, po), steps, flush)
    tg = _time_device(torch, lambda: BT.apply(p, uo), steps, flush)
    nl, nr = shell.dims(fine)
    nodes = 10 * nl * nl * nr
    nlp, nrp = shell.dims(fine - 1)
    cells = 10 * (nl - 1) ** 2 * (nr - 1)
    # algorithmic bytes: velocity read or written once (24 B/node), pressure once, the per-wedge scratch
    # written and read back once (2 x 16 B per cell)
    bytes_b = 24 * nodes + 8 * 10 * nlp * nlp * nrp + 32 * cells
    peak, peak_kind = _peaks()
    print(json.dumps({"metric": "L6 B and B^T apply time (FP64)", "value": (tb + tg) * 1e3, "unit": "ms",
                      "n_gpus": 1, "steps": steps, "warmup": a.warmup, "higher_is_better": False, "dtype": "f64",
                      "data": "synthetic",
                      "config": {"workload": "L6 divergence and gradient (10x65x65x65 velocity nodes, pressure on L5), "
                                             "no-slip / free-slip, L2 flushed between launches"},
                      "divergence_ms": tb * 1e3, "gradient_ms": tg * 1e3,
                      "roofline": {"bound": "hbm", "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                                   "algorithmic_bytes": bytes_b,
                                   "divergence_frac": bytes_b / tb / 1e9 / peak,
                                   "gradient_frac": bytes_b / tg / 1e9 / peak}}), flush=True)


# nodal viscosity of the adaptive-GCA comparisons: the benchmark field with log-amplitude ln(1000), contrast 1e6
# (GCAElementsCollector's absolute threshold of 10 on the reference-coordinate gradient marks 71 of the 640
# level-2 cells at level 6; at contrast 1e4 it marks none)
GCA_MODES_LOG_AMPLITUDE = math.log(1000.0)


def run_gca_build(a):
    """TwoGridGCA down the level-6 hierarchy (Neumann L6 operator -> L5 -> L4 -> L3 -> L2).

    Full GCA on the benchmark viscosity: the fast build (L5 from the on-the-fly L6 matrices in the rank form
    P^T g; L4..L2 from stored matrices with the 18 x 18 triple products on the FP64 tensor cores) against the
    plain scalar build (one fine wedge at a time, fine matrix then P^T A P), per level and in total, and the
    level-2 matrices of both. Adaptive GCA on a viscosity of contrast 1e6: the marked coarsest cells, the
    stored cells and bytes of every coarse level against full GCA, and its build time."""
    import numpy as np
    import torch

    import synthetic as S
    import terra_b200 as T

    shell = T.Shell(LEVEL, num_levels=NUM_LEVELS)
    fine = NUM_LEVELS - 1
    eta = torch.tensor(S.viscosity(shell, fine, seed=SEED_ETA), device="cuda")

    def chain(k, mode):
        ops = {fine: T.EpsDivDiv(shell, fine, k=k, bc_cmb=0, bc_surface=0)}
        kl = k
        for l in range(fine - 1, -1, -1):
            nl, nr = shell.dims(l)
            kl = kl[:, ::2, ::2, ::2].contiguous()
            ops[l] = T.EpsDivDiv(shell, l, k=kl, bc_cmb=0, bc_surface=0)
        marks = T.gca_mark_elements(shell, fine, fine, k) if mode == "adaptive" else None
        if marks is not None:
            for l in range(fine - 1, -1, -1):
                ops[l].set_selective_matrices(l, marks)
        return ops, marks

    def build_times(ops, tc):
        per = []
        for l in range(fine - 1, -1, -1):
            T.gca_build(ops[l + 1], ops[l], tensor_cores=tc)  # warm-up (also the input of the next level)
            dt, _ = _timed(torch, lambda: T.gca_build(ops[l + 1], ops[l], tensor_cores=tc))
            per.append({"coarse_level": l + (LEVEL - fine), "ms": dt * 1e3})
        return per

    times, mats = {}, {}
    for tc in (True, False):
        ops, _ = chain(eta, "full")
        times["fast" if tc else "scalar"] = build_times(ops, tc)
        mats[tc] = ops[0].local_matrices()
        del ops
    diff = float(np.abs(mats[True] - mats[False]).max() / np.abs(mats[False]).max())
    tot = {k: sum(p["ms"] for p in v) for k, v in times.items()}

    eta4 = torch.tensor(S.viscosity(shell, fine, seed=SEED_ETA, log_amplitude=GCA_MODES_LOG_AMPLITUDE), device="cuda")
    storage = {}
    for mode in ("adaptive", "full"):
        ops, marks = chain(eta4, mode)
        per = build_times(ops, True)
        storage[mode] = {"build_ms": sum(p["ms"] for p in per), "per_level": [
            dict(zip(("stored_cells", "bytes"), ops[l].stored_cells()), level=l + (LEVEL - fine),
                 cells=10 * (shell.dims(l)[0] - 1) ** 2 * (shell.dims(l)[1] - 1)) for l in range(fine - 1, -1, -1)]}
        if marks is not None:
            storage[mode]["marked_coarsest_cells"] = int(marks.sum().item())
            storage[mode]["coarsest_cells"] = int(marks.numel())
        del ops
    for mode in storage:
        storage[mode]["bytes"] = sum(p["bytes"] for p in storage[mode]["per_level"])
    print(json.dumps({"metric": "L6 GCA hierarchy build time", "value": tot["fast"], "unit": "ms",
                      "n_gpus": 1, "higher_is_better": False, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": "TwoGridGCA chain of the L6 hierarchy (Neumann L6 operator with the "
                                             "benchmark viscosity, coarse levels 5..2)"},
                      "per_level": times, "scalar_total_ms": tot["scalar"],
                      "speedup_fast_vs_scalar": tot["scalar"] / tot["fast"],
                      "level2_max_rel_diff_fast_vs_scalar": diff,
                      "adaptive_vs_full": {"viscosity": "benchmark field with log-amplitude ln(1000) (contrast 1e6)",
                                           **storage}}), flush=True)


def run_gca_modes(a):
    """The L6 mixed-precision Stokes solve with full (gca = 1), adaptive (gca = 2) and no GCA (gca = 0) on a
    nodal viscosity of contrast 1e6: set-up time, iterations and time to 1e-8, the time of one preconditioner
    application (one FP32 V-cycle), and the bytes of stored coarse-level matrices of each hierarchy."""
    import torch

    import synthetic as S
    import terra_b200 as T

    shell = T.Shell(LEVEL, num_levels=NUM_LEVELS)
    fine = NUM_LEVELS - 1
    eta = torch.tensor(S.viscosity(shell, fine, seed=SEED_ETA, log_amplitude=GCA_MODES_LOG_AMPLITUDE), device="cuda")
    temp = S.temperature(shell, fine, seed=SEED_TEMP)
    f = S.buoyancy_rhs(shell, fine, temp, *BCS)
    x = _stokes_vectors(torch, shell, fine, "cuda")
    b = [f[c].contiguous() for c in range(3)] + [torch.zeros_like(x[3])]
    out = {}
    # one solver built and dropped first, so that no mode's set-up time includes the process's first use of the
    # library's kernels
    del_me = T.StokesSolver(shell, eta=eta, bc_cmb=BCS[0], bc_surface=BCS[1], mixed_precision=1, gca=1,
                            chebyshev_order=CHEB_ORDER,
                            coarse_solver=T.COARSE_DENSE)
    del del_me
    for gca in (1, 2, 0):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sol = T.StokesSolver(shell, eta=eta, bc_cmb=BCS[0], bc_surface=BCS[1], mixed_precision=1, gca=gca,
                             chebyshev_order=CHEB_ORDER, coarse_solver=T.COARSE_DENSE, relative_tolerance=1e-8, absolute_tolerance=0.0,
                             max_iterations=3000, project_pressure_mean=1)
        torch.cuda.synchronize()
        setup = time.perf_counter() - t0
        for t in x:
            t.zero_()
        sol.solve(x, b)  # warm-up
        dt, _ = _timed(torch, lambda: ([t.zero_() for t in x], sol.solve(x, b)))
        its, rr, conv = sol.result()
        # one preconditioner application (Schur step, B^T, one FP32 V-cycle), L2 flushed before each
        z = [torch.zeros_like(t) for t in b]
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        for _ in range(3):
            sol.precondition(b, z)
        t_prec = _time_device(torch, lambda: sol.precondition(b, z), 10, flush)
        out[f"gca{gca}"] = {"setup_s": setup, "solve_s": dt, "iterations": its, "relative_residual": rr,
                            "converged": conv, "precondition_ms": t_prec * 1e3,
                            "stored_bytes": sum(sol.level_storage(l)[1] for l in range(fine)),
                            "stored_cells": [sol.level_storage(l)[0] for l in range(fine)]}
        del sol
    print(json.dumps({"metric": "L6 mixed-precision Stokes solve time by GCA mode", "value": out["gca2"]["solve_s"],
                      "unit": "s/solve", "n_gpus": 1, "higher_is_better": False, "dtype": "f32+f64",
                      "data": "synthetic",
                      "config": {"workload": "L6 Stokes (no-slip CMB, free-slip surface), buoyancy rhs, viscosity "
                                             "of contrast 1e6 (benchmark field, log-amplitude ln(1000)), FGMRES(30) "
                                             "to 1e-8 with the FP32 V-cycle and the dense coarsest solve"},
                      "modes": out}), flush=True)


def run_solve_profile(a):
    """The level-6 benchmark solve for launch lists: after one warm-up solve each, one mixed-precision and one FP64
    solve inside the NVTX ranges "mixed_solve" and "fp64_solve" (ncu --nvtx --nvtx-include "mixed_solve/")."""
    import torch

    import synthetic as S
    import terra_b200 as T

    shell = T.Shell(LEVEL, num_levels=NUM_LEVELS)
    fine = NUM_LEVELS - 1
    eta = torch.tensor(S.viscosity(shell, fine, seed=SEED_ETA), device="cuda")
    f = S.buoyancy_rhs(shell, fine, S.temperature(shell, fine, seed=SEED_TEMP), *BCS)
    x = _stokes_vectors(torch, shell, fine, "cuda")
    b = [f[c].contiguous() for c in range(3)] + [torch.zeros_like(x[3])]
    out = {}
    for name, mixed in (("mixed", 1), ("fp64", 0)):
        sol = T.StokesSolver(shell, eta=eta, bc_cmb=BCS[0], bc_surface=BCS[1], mixed_precision=mixed,
                             chebyshev_order=CHEB_ORDER,
                             coarse_solver=T.COARSE_DENSE if a.coarse == "dense" else T.COARSE_PCG,
                             relative_tolerance=1e-8, absolute_tolerance=0.0, max_iterations=3000,
                             project_pressure_mean=1)
        for t in x:
            t.zero_()
        sol.solve(x, b)
        for t in x:
            t.zero_()
        torch.cuda.synchronize()
        l0 = T.kernel_launch_count()
        torch.cuda.nvtx.range_push(f"{name}_solve")
        dt, _ = _timed(torch, lambda: sol.solve(x, b))
        torch.cuda.nvtx.range_pop()
        its, rr, conv = sol.result()
        out[name] = {"s": dt, "iterations": its, "relative_residual": rr, "converged": conv,
                     "launches": T.kernel_launch_count() - l0}
        del sol
    print(json.dumps({"metric": "L6 Stokes solve (launch-list workload)", "unit": "s/solve", "n_gpus": 1,
                      "higher_is_better": False, "data": "synthetic", "config": {"workload": WORKLOAD},
                      "solves": out}), flush=True)


def run_precondition(a):
    """One application of the L6 block-triangular preconditioner of the mixed-precision solver
    (Schur diagonal, B^T, one FP32 V-cycle with the FP64 coarsest CG)."""
    import torch

    import synthetic as S
    import terra_b200 as T

    shell = T.Shell(LEVEL, num_levels=NUM_LEVELS)
    fine = NUM_LEVELS - 1
    eta = torch.tensor(S.viscosity(shell, fine, seed=SEED_ETA), device="cuda")
    sol = T.StokesSolver(shell, eta=eta, bc_cmb=BCS[0], bc_surface=BCS[1], mixed_precision=1,
                         chebyshev_order=CHEB_ORDER,
                         project_pressure_mean=1)
    u = T.random_vector(shell, fine, 3, 5)
    p = T.random_vector(shell, fine - 1, 1, 6)[0].contiguous()
    v = [u[c].contiguous() for c in range(3)] + [p]
    z = [torch.zeros_like(t) for t in v]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(max(3, a.warmup)):
        sol.precondition(v, z)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("precondition")  # one application, for per-kernel captures (ncu --nvtx)
    sol.precondition(v, z)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    steps = max(1, a.steps)
    t = _time_device(torch, lambda: sol.precondition(v, z), steps, flush)
    its, init, final = sol.coarse_stats()
    print(json.dumps({"metric": "L6 mixed-precision block preconditioner apply time", "value": t * 1e3, "unit": "ms",
                      "n_gpus": 1, "steps": steps, "warmup": a.warmup, "higher_is_better": False,
                      "dtype": "f32+f64", "data": "synthetic",
                      "config": {"workload": "L6 block-triangular preconditioner: lumped 1/eta Schur, B^T, one FP32 "
                                             "V(2,2) Chebyshev(3) cycle over L2..L6 with GCA coarse operators and the "
                                             "FP64 coarsest CG (50 iterations / 1e-6)"},
                      "coarse_cg": {"iterations": its, "initial_residual": init, "final_residual": final}}),
          flush=True)


def run_ours(a):
    import torch

    import synthetic as S
    import terra_b200 as T

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    steps, warmup = max(1, a.steps), max(3, a.warmup)

    shell = T.Shell(LEVEL, num_levels=NUM_LEVELS)
    fine = NUM_LEVELS - 1
    eta = torch.tensor(S.viscosity(shell, fine, seed=SEED_ETA), device=dev)
    temp = S.temperature(shell, fine, seed=SEED_TEMP)
    f = S.buoyancy_rhs(shell, fine, temp, *BCS)
    nlp, nrp = shell.dims(fine - 1)
    coarse = {"dense": T.COARSE_DENSE, "pcg": T.COARSE_PCG}
    other = "pcg" if a.coarse == "dense" else "dense"
    opts = dict(bc_cmb=BCS[0], bc_surface=BCS[1], relative_tolerance=1e-8, absolute_tolerance=0.0,
                max_iterations=3000, restart=30, project_pressure_mean=1, normalize_pressure=1,
                chebyshev_order=CHEB_ORDER)
    solvers, setup_s = {}, {}
    for name, mixed in (("mixed", 1), ("fp64", 0)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solvers[name] = T.StokesSolver(shell, eta=eta, mixed_precision=mixed, coarse_solver=coarse[a.coarse],
                                       **opts)
        torch.cuda.synchronize()
        setup_s[name] = time.perf_counter() - t0

    b = [f[c].contiguous() for c in range(3)] + [torch.zeros((10, nlp, nlp, nrp), dtype=torch.float64, device=dev)]
    x = [torch.zeros_like(t) for t in b]
    stream = torch.cuda.current_stream()

    def solve(name):
        for t in x:
            t.zero_()
        solvers[name].solve(x, b)

    for name in ("mixed", "fp64"):
        for _ in range(warmup):
            solve(name)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    results = {}
    if ws > 1:
        torch.distributed.barrier()
    for name in ("mixed", "fp64"):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.synchronize()
        l0 = T.kernel_launch_count()
        for i in range(steps):
            ev[i][0].record(stream)
            solve(name)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        launches = T.kernel_launch_count() - l0
        its, rr, conv = solvers[name].result()
        results[name] = {"s": sum(s.elapsed_time(e) for s, e in ev) / steps / 1e3, "iterations": its,
                         "relres": rr, "full_relres": solvers[name].full_residual(), "converged": conv,
                         "launches": launches, "x": [t.clone() for t in x]}
    if ws > 1:
        torch.distributed.barrier()
    ck = clocks.stop()
    # the other coarsest-level solve, timed once after one warm-up solve
    alt = {}
    for name, mixed in (("mixed", 1), ("fp64", 0)):
        s_alt = T.StokesSolver(shell, eta=eta, mixed_precision=mixed, coarse_solver=coarse[other], **opts)
        for t in x:
            t.zero_()
        s_alt.solve(x, b)
        dt_alt, _ = _timed(torch, lambda: ([t.zero_() for t in x], s_alt.solve(x, b)))
        its_alt, rr_alt, conv_alt = s_alt.result()
        alt[name] = {"s": dt_alt, "iterations": its_alt, "relative_residual": rr_alt, "converged": conv_alt}
        del s_alt
    t_mixed = results["mixed"]["s"]
    t_tensor = torch.tensor([t_mixed, results["fp64"]["s"]], device=dev, dtype=torch.float64)
    if ws > 1:
        torch.distributed.all_reduce(t_tensor, op=torch.distributed.ReduceOp.MAX)
    t_mixed, t_fp64 = (float(v) for v in t_tensor.tolist())

    # mixed vs FP64 solution (owned-node relative L2; pressure mean-free)
    own_u = torch.tensor(shell.ownership(fine), device=dev).double()
    own_p = torch.tensor(shell.ownership(fine - 1), device=dev).double()
    xm, xd = results["mixed"]["x"], results["fp64"]["x"]
    du = sum(((xm[c] - xd[c]) ** 2 * own_u).sum() for c in range(3))
    nu = sum((xd[c] ** 2 * own_u).sum() for c in range(3))
    pm = xm[3] - (xm[3] * own_p).sum() / own_p.sum()
    pd = xd[3] - (xd[3] * own_p).sum() / own_p.sum()
    err_u = float(torch.sqrt(du / nu))
    err_p = float(torch.sqrt(((pm - pd) ** 2 * own_p).sum() / (pd ** 2 * own_p).sum()))

    # end to end through the public solve call with host buffers
    h_b = [t.cpu().pin_memory() for t in b]
    h_x = [torch.empty_like(t, device="cpu").pin_memory() for t in x]
    d_b = [torch.empty_like(t) for t in b]
    e2e_steps = max(1, min(steps, 3))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        for d, h in zip(d_b, h_b):
            d.copy_(h, non_blocking=True)
        for t in x:
            t.zero_()
        solvers["mixed"].solve(x, d_b)
        for h, t in zip(h_x, x):
            h.copy_(t, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = e0.elapsed_time(e1) / 1e3 / e2e_steps
    io_bytes = sum(t.numel() * t.element_size() for t in b)

    # operator apply roofline: the FP32 fine-level apply dominates the mixed solve
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    t32, nodes = _time_apply(T, torch, shell, eta, torch.float32, 20, flush)
    t64, _ = _time_apply(T, torch, shell, eta, torch.float64, 20, flush)
    peak, peak_kind = _peaks()
    ach32 = BYTES_PER_NODE["f32"] * nodes / t32 / 1e9
    ach64 = BYTES_PER_NODE["f64"] * nodes / t64 / 1e9

    cpu = None
    if rank == 0 and not a.no_cpu_baseline and ws == 1:
        try:
            cpu = _reference_baseline(results["fp64"]["iterations"])
        except Exception as e:
            cpu = {"value": None, "unavailable": f"{type(e).__name__}: {e}"}
    if rank == 0:
        dofs_u = 3 * (10 * (shell.dims(fine)[0] - 1) ** 2 + 2) * shell.dims(fine)[1]
        line = {
            "metric": METRIC, "value": t_mixed, "unit": "s/solve", "n_gpus": ws, "steps": steps, "warmup": warmup,
            "ms_per_step": t_mixed * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "l2": "inputs exceed L2 (66 MB per velocity vector, 0.45-0.9 GB of "
                                                  "level-5 Galerkin matrices streamed per V-cycle)",
                       "replicas": ws, "velocity_dofs": dofs_u},
            "fp64_solve_s": t_fp64, "speedup_mixed_vs_fp64": t_fp64 / t_mixed,
            "coarse_solver": a.coarse, f"coarse_{other}": alt,
            "iterations": {"mixed": results["mixed"]["iterations"], "fp64": results["fp64"]["iterations"]},
            "relative_residual": {k: results[k]["relres"] for k in results},
            "relative_residual_without_projection": {k: results[k]["full_relres"] for k in results},
            "converged": {k: results[k]["converged"] for k in results},
            "mixed_vs_fp64_rel_l2": {"velocity": err_u, "pressure": err_p},
            "setup_s": setup_s,
            "roofline": {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s", "frac": ach32 / peak,
                         "traffic": _profile_traffic("epsdivdiv_f32_L6"), "peak_kind": peak_kind,
                         "kernel": "epsdivdiv_kernel<float> + iface_kernel (L6 fine-level apply)",
                         "algorithmic_bytes_per_launch": BYTES_PER_NODE["f32"] * nodes, "ms": t32 * 1e3,
                         "fp64": {"achieved": ach64, "frac": ach64 / peak, "ms": t64 * 1e3,
                                  "traffic": _profile_traffic("epsdivdiv_f64_L6")}},
            "cpu_baseline": cpu,
            "clocks": ck,
            "e2e": {"value": t_e2e, "unit": "s/solve", "h2d_bytes_per_step": io_bytes,
                    "d2h_bytes_per_step": io_bytes},
            "gpu_launches": results["mixed"]["launches"] + results["fp64"]["launches"],
            "gpu_launches_per_solve": {k: results[k]["launches"] / steps for k in results},
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()


def _stokes_vectors(torch, shell, level, dev):
    nl, nr = shell.dims(level)
    nlp, nrp = shell.dims(level - 1)
    x = [torch.zeros((10, nl, nl, nr), dtype=torch.float64, device=dev) for _ in range(3)]
    x.append(torch.zeros((10, nlp, nlp, nrp), dtype=torch.float64, device=dev))
    return x


def _timed(torch, fn):
    """Device seconds of fn() on the current stream (synchronised on both sides)."""
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3, out


# FGMRES restart of the configuration-3 solves: with 1e4 jumps between cells, FGMRES(30) stalls near 1e-6, while
# FGMRES(128) reaches 1e-8 in about 1250 iterations and 1e-13 in about 1100-1400 from a good Schur coefficient
ADJOINT_RESTART = 128
TIMED_MAX_ITERATIONS = 4000


def run_adjoint_l5(a):
    """Misfit gradient at level 5 (configuration 3: 10 x 33 x 33 x 33 velocity nodes, hierarchy L2..L5) with per-cell
    viscosity from seeded log-uniform [1, 1e4] lateral blocks in a smooth background (contrast 8e4), no-slip CMB /
    free-slip surface, J = 1/2 ||u - u_obs||^2 over owned nodes, u_obs from a seeded perturbation of log-viscosity.

    Timed: one forward solve, one adjoint solve and the backward kernel (mixed precision, rtol 1e-8). Checked on the
    same viscosity: the gradient of solves to 1e-13 against central differences along 32 seeded element directions
    at step 1e-6 (and 8 at step 1e-5), and against the gradient of the FP64 solver. The perturbed solves start from
    the unperturbed solution and reduce their residual by 2e-9; J(+) - J(-) is summed as 1/2 (u+ - u-).(u+ + u- -
    2 u_obs) with exact rounding (math.fsum). All solves: FGMRES(ADJOINT_RESTART), dense coarsest solve, Schur
    coefficient 1/mean(eta) of the cells around each pressure node."""
    import numpy as np
    import torch

    import synthetic as S
    import terra_b200 as T

    level, nlev, bcs = 5, 4, BCS
    dev = torch.device("cuda", 0)
    g = T.Shell(level, num_levels=nlev)
    fine = nlev - 1
    f = S.buoyancy_rhs(g, fine, S.temperature(g, fine, seed=SEED_TEMP), *bcs)
    own = torch.tensor(g.ownership(fine), device=dev).bool()
    eta = S.cell_viscosity_blocks(g, fine, seed=3, tiles=4, fraction=0.3, max_log10=4.0,
                                  background_log_amplitude=0.5 * math.log(10.0))
    ks = torch.tensor(S.schur_coefficient_from_cells(g, fine, eta), device=dev)
    theta = np.log(eta)
    rng = np.random.default_rng(5)
    theta_obs = theta + 0.1 * rng.standard_normal(theta.shape)

    def solver(th, rtol, mixed=1, max_iterations=TIMED_MAX_ITERATIONS):
        return T.StokesSolver(g, eta_cell=torch.tensor(np.exp(th), device=dev), k_schur=ks, bc_cmb=bcs[0],
                              bc_surface=bcs[1], relative_tolerance=rtol, absolute_tolerance=0.0,
                              max_iterations=max_iterations, restart=ADJOINT_RESTART, coarse_solver=T.COARSE_DENSE,
                              project_pressure_mean=1, normalize_pressure=0, mixed_precision=mixed)

    def forward(s, x0=None):
        x = _stokes_vectors(torch, g, fine, dev)
        if x0 is not None:
            for t, t0 in zip(x, x0):
                t.copy_(t0)
        rhs = [f[c].contiguous() for c in range(3)] + [torch.zeros_like(x[3])]
        ok = s.solve(x, rhs)
        return x, ok

    s_obs = solver(theta_obs, 1e-10)
    x_obs, _ = forward(s_obs)
    u_obs = [x_obs[c].clone() for c in range(3)]
    del s_obs

    # --- timed gradient at rtol 1e-8
    s8 = solver(theta, 1e-8)
    grad8 = torch.zeros(theta.shape, dtype=torch.float64, device=dev)
    for _ in range(max(1, a.warmup)):
        x8, _ = forward(s8)
        s8.misfit_gradient(x8, u_obs, grad8)
    steps = max(1, a.steps)
    t_fwd = t_adj = 0.0
    conv_fwd = conv_adj = True
    for _ in range(steps):
        dt, (x8, ok) = _timed(torch, lambda: forward(s8))
        t_fwd += dt / steps
        conv_fwd = conv_fwd and bool(ok)
        its_fwd, res_fwd, _ = s8.result()
        dt, ok = _timed(torch, lambda: s8.misfit_gradient(x8, u_obs, grad8))
        t_adj += dt / steps
        conv_adj = conv_adj and bool(ok)
        its_adj, res_adj, _ = s8.result()
    del s8

    # --- gradient check at the same viscosity, solves to 1e-13
    grads, base = {}, {}
    x_base = None
    for name, mixed in (("mixed", 1), ("fp64", 0)):
        s = solver(theta, 1e-13, mixed=mixed, max_iterations=8000)
        x, ok = forward(s)
        fwd = s.result()
        if mixed:
            x_base = [t.clone() for t in x]
        gr = torch.zeros(theta.shape, dtype=torch.float64, device=dev)
        ok_adj = s.misfit_gradient(x, u_obs, gr)
        adj = s.result()
        base[name] = {"forward": {"iterations": fwd[0], "relative_residual": fwd[1], "converged": bool(ok)},
                      "adjoint": {"iterations": adj[0], "relative_residual": adj[1], "converged": bool(ok_adj)}}
        grads[name] = gr.cpu().numpy()
        del s
    gm, gd = grads["mixed"], grads["fp64"]
    mixed_vs_fp64 = float(np.linalg.norm(gm - gd) / np.linalg.norm(gd))

    def delta_j(up, um):
        terms = [((up[c] - um[c]) * (up[c] + um[c] - 2 * u_obs[c]))[own].cpu().numpy() for c in range(3)]
        return 0.5 * math.fsum(np.concatenate(terms))

    drng = np.random.default_rng(6)
    dirs = [drng.standard_normal(theta.shape) for _ in range(32)]
    fd_err, fd_its = {}, []
    t0 = time.perf_counter()
    for h, nd in ((1e-6, 32), (1e-5, 8)):
        errs = []
        for d in dirs[:nd]:
            xs = []
            for sgn in (1.0, -1.0):
                s = solver(theta + sgn * h * d, 2e-9, max_iterations=3000)
                x, _ = forward(s, x_base)
                fd_its.append(s.result()[0])
                xs.append(x)
                del s
            fd = delta_j(xs[0], xs[1]) / (2 * h)
            ad = math.fsum((gm * d).ravel())
            errs.append(abs(fd - ad) / abs(ad))
        fd_err[f"{h:g}"] = {"directions": nd, "max": max(errs), "median": float(np.median(errs))}
    t_fd = time.perf_counter() - t0
    line = {"metric": "L5 adjoint log-viscosity gradient time (forward + adjoint solve + VJP, rtol 1e-8)",
            "value": t_fwd + t_adj, "unit": "s/gradient", "n_gpus": 1, "steps": steps, "warmup": a.warmup,
            "ms_per_step": (t_fwd + t_adj) * 1e3, "higher_is_better": False, "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": "L5 adjoint gradient (10x33x33x33 velocity nodes, hierarchy L2..L5), no-slip / "
                                   "free-slip, per-cell viscosity: log-uniform [1, 1e4] 8x8-cell lateral blocks in "
                                   "a smooth SH background (factor 10), J = 1/2||u - u_obs||^2, u_obs from log-eta "
                                   "+ 0.1 N(0,1); FGMRES(128), dense coarsest solve, Schur 1/mean(eta)",
                       "viscosity_contrast": float(eta.max() / eta.min())},
            "forward_s": t_fwd, "adjoint_and_vjp_s": t_adj,
            "iterations": {"forward": its_fwd, "adjoint": its_adj, "limit": TIMED_MAX_ITERATIONS},
            "relative_residual": {"forward": res_fwd, "adjoint": res_adj},
            "converged": {"forward": conv_fwd, "adjoint": conv_adj},
            "ms_per_iteration": {"forward": t_fwd / max(its_fwd, 1) * 1e3, "adjoint": t_adj / max(its_adj, 1) * 1e3},
            "gradient_check": {"viscosity": "the timed one", "base_solves": base,
                               "fd_rel_err_by_step": fd_err, "perturbed_solve_reduction": 2e-9,
                               "perturbed_iterations": {"min": min(fd_its), "max": max(fd_its)},
                               "mixed_vs_fp64_gradient_rel": mixed_vs_fp64, "fd_seconds": t_fd}}
    print(json.dumps(line), flush=True)


def run_solve_l7(a):
    """Level 7: 10 x 129 x 129 x 129 velocity nodes (64M velocity dofs), pressure on L6, hierarchy L2..L7,
    per-cell viscosity with contrast 1e3 including a x30 jump below r = 0.9, seeded buoyancy right-hand side.
    Times the mixed and the FP64 solve to 1e-8 and one adjoint gradient with the mixed solver."""
    import gc

    import numpy as np
    import torch

    import synthetic as S
    import terra_b200 as T

    level, nlev, bcs = 7, 6, BCS
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = T.Shell(level, num_levels=nlev)
    fine = nlev - 1
    t0 = time.perf_counter()
    eta = S.cell_viscosity_radial_jump(g, fine, seed=SEED_ETA, contrast=1e3, jump=30.0, r_jump=0.9)
    ks = torch.tensor(S.schur_coefficient_from_cells(g, fine, eta), device=dev)
    eta_d = torch.tensor(eta, device=dev)
    f = S.buoyancy_rhs(g, fine, S.temperature(g, fine, seed=SEED_TEMP), *bcs)
    t_inputs = time.perf_counter() - t0
    opts = dict(k_schur=ks, bc_cmb=bcs[0], bc_surface=bcs[1], relative_tolerance=1e-8, absolute_tolerance=0.0,
                max_iterations=2000, restart=30, project_pressure_mean=1, normalize_pressure=0,
                chebyshev_order=CHEB_ORDER, coarse_solver=T.COARSE_DENSE)
    free0 = torch.cuda.mem_get_info(dev)[0]

    # observations from a perturbed viscosity (one mixed solve, solver released before the timed ones)
    rng = np.random.default_rng(7)
    s_obs = T.StokesSolver(g, eta_cell=torch.tensor(eta * np.exp(0.1 * rng.standard_normal(eta.shape)),
                                                    device=dev), mixed_precision=1, **opts)
    x_obs = _stokes_vectors(torch, g, fine, dev)
    b = [f[c].contiguous() for c in range(3)] + [torch.zeros_like(x_obs[3])]
    s_obs.solve(x_obs, b)
    u_obs = [x_obs[c] for c in range(3)]
    del s_obs
    gc.collect()

    res, setup = {}, {}
    steps = max(1, a.steps)
    for name, mixed in (("mixed", 1), ("fp64", 0)):
        dt, s = _timed(torch, lambda: T.StokesSolver(g, eta_cell=eta_d, mixed_precision=mixed, **opts))
        setup[name] = dt
        used = free0 - torch.cuda.mem_get_info(dev)[0]
        x = _stokes_vectors(torch, g, fine, dev)
        for _ in range(max(1, a.warmup)):
            for t in x:
                t.zero_()
            s.solve(x, b)
        ts = []
        for _ in range(steps):
            for t in x:
                t.zero_()
            dt, _ = _timed(torch, lambda: s.solve(x, b))
            ts.append(dt)
        its, rr, conv = s.result()
        r = {"s": sum(ts) / steps, "iterations": its, "relres": rr, "converged": conv,
             "device_bytes_with_solver": used}
        if mixed:
            grad = torch.zeros(eta.shape, dtype=torch.float64, device=dev)
            dt, ok = _timed(torch, lambda: s.misfit_gradient(x, u_obs, grad))
            r["adjoint_gradient_s"] = dt
            r["adjoint_converged"] = ok
            r["gradient_finite"] = bool(torch.isfinite(grad).all())
        res[name] = r
        del s, x
        gc.collect()

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    peak, peak_kind = _peaks()
    nl, nr = g.dims(fine)
    nodes = 10 * nl * nl * nr
    apply = {}
    for prec, dt in (("f32", torch.float32), ("f64", torch.float64)):
        t, _ = _time_apply(T, torch, g, None, dt, 10, flush, level=fine, eta_cell=eta_d)
        ach = BYTES_PER_NODE[prec] * nodes / t / 1e9
        apply[prec] = {"ms": t * 1e3, "achieved_gbs": ach, "frac": ach / peak}
    line = {"metric": "L7 Stokes solve time to 1e-8 (FP32-MG vs FP64)", "value": res["mixed"]["s"],
            "unit": "s/solve", "n_gpus": 1, "steps": steps, "warmup": a.warmup,
            "ms_per_step": res["mixed"]["s"] * 1e3, "higher_is_better": False, "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": "L7 Stokes solve (10x129x129x129 velocity nodes, pressure on L6, hierarchy "
                                   "L2..L7), no-slip / free-slip, per-cell viscosity contrast 1e3 with a x30 jump "
                                   "below r = 0.9, seeded buoyancy RHS, FGMRES(30) + block-triangular GMG "
                                   "preconditioner, rtol 1e-8", "viscosity_contrast": float(eta.max() / eta.min())},
            "fp64_solve_s": res["fp64"]["s"], "speedup_mixed_vs_fp64": res["fp64"]["s"] / res["mixed"]["s"],
            "solves": res, "setup_s": setup, "inputs_s": t_inputs,
            "apply_roofline": {"peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                               "bytes_per_node": BYTES_PER_NODE, **apply}}
    print(json.dumps(line), flush=True)


def main():
    a = _args()
    if a.impl == "reference":
        run_reference(a)
    elif a.workload.startswith("apply"):
        run_apply(a)
    elif a.workload == "coupling":
        run_coupling(a)
    elif a.workload == "precondition":
        run_precondition(a)
    elif a.workload == "gca-build":
        run_gca_build(a)
    elif a.workload == "gca-modes":
        run_gca_modes(a)
    elif a.workload == "solve-profile":
        run_solve_profile(a)
    elif a.workload == "adjoint-L5":
        run_adjoint_l5(a)
    elif a.workload == "solve-L7":
        run_solve_l7(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
