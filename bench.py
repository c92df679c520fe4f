#!/usr/bin/env python
"""Benchmark of the MiniFS iteration hot path on B200.

One step = one iteration of the reference's main loop (main.cpp:201-291:
Roe flux + residual, local time step, LU-SGS forward/backward sweeps with
the update, node-based Green-Gauss gradient, residual norm) over the whole
mesh.  Metric: cell-updates/s = cells x steps / device time.

Workload (N=1): the 64^3 x 6 = 1,572,864-tet cube (interior jitter 0.15h,
seed 1), Mach 0.5, alpha 2 deg, CFL 10, far field on all sides, freestream
plus a 5% Gaussian density bump; FP64.  The working set (~1.2 GB) is far
larger than the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
  python bench.py --form batched [--ncase 64]
  python bench.py --form mixed [--mixed-size 128] [--converge 3000]
  python bench.py --form channel [--converge 20000]
  python bench.py --form batched --precision mixed
  python bench.py --form partition [--parts K]

--form batched: 64 cube cases with n^3 x 6 tets, n uniform in [8, 48], Mach
U(0.3, 0.8), alpha U(-5, 5) deg, jitter U(0, 0.2)h, all in one context (one
launch per kernel covers every case), against the same cases run one after
another in their own contexts.

--form mixed: the 128^3 x 6 cube (jitter 0.1h, Mach 0.8, alpha 1.25 deg, CFL
20) in the FP64 and the mixed-precision forms: throughput of each, the
mixed state's error against FP64, and with --converge the iterations and
time each form needs for a 1e-6 residual drop.

--form channel: the 4x1x1 channel (192x48x48 hexes x 6 tets, slip wall with
a bump at the bottom, Mach 0.7, CFL 30) in both forms, as --form mixed, to a
1e-8 residual drop with --converge, and the mixed form's wall pressure
against FP64.

--precision mixed (batched form): the batch and its sequential per-case
reference both in the mixed form.

--form partition: the fp64 workload's cube split into K parts (recursive
coordinate bisection; K = --parts, default the number of GPUs), each part
its own context iterating through the halo phases with the reference's
MPI-mode exchanges between them: device copies between the parts of one
process, NCCL point-to-point and all-reduce between processes (part z on
rank z mod N).  Strong scaling: the whole mesh's cells per step.

Before the warm-up the launch parameters (sweep kernels, chunk assignment,
sweep mode, face-kernel register caps, gradient block sizes) are chosen by
measurement on the workload's own grid (mfg_autotune) and reported.

With --gpus N > 1 (one process per GPU under torchrun) every rank runs its
own replica of the workload (the path has no exchange step) and rank 0
prints the aggregate.  --impl reference times the reference's own CPU code
(oracle/_ref, all host cores) on the same workload.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s on 1 B200: FP64 vs mixed vs batched at equal residual drop"
UNIT = "cell-updates/s"


def workload(n: int) -> dict:
    return dict(name=f"cube{n}x6_M0.5_a2_cfl10_fp64", n=n, jitter=0.15, seed=1, mach=0.5,
                alpha=2.0, cfl=10.0, bump_amp=0.05, bump_sigma=0.1)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mfgpu", choices=["mfgpu", "reference"])
    ap.add_argument("--size", type=int, default=64, help="hexes per cube edge (64 = 1.57M tets)")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the reference's CPU runs (baseline and parity)")
    ap.add_argument("--parity-iters", type=int, default=10,
                    help="iterations of the parity check against the reference's serial build")
    ap.add_argument("--no-forms", action="store_true",
                    help="fp64 form only: skip the mixed, channel and batched legs")
    ap.add_argument("--form-iters", type=int, default=1500,
                    help="iteration cap of the mixed form's run to its drop (x3 for the channel)")
    ap.add_argument("--form-batch-steps", type=int, default=10,
                    help="timed iterations of the batched form and of its sequential runs")
    ap.add_argument("--form-cpu-iters", type=int, default=2,
                    help="iteration cap of the reference's CPU sample on the channel workload")
    ap.add_argument("--form-cpu", default="serial", choices=["serial", "tdtree"],
                    help="the reference build timed on the 128^3 mixed workload (its TDTree "
                         "set-up takes minutes there)")
    ap.add_argument("--form", default="fp64",
                    choices=["fp64", "batched", "mixed", "channel", "partition"],
                    help="fp64: the single-grid workload; batched: 64 uneven cases in one "
                         "context against the same cases run one after another; mixed: the "
                         "mixed-precision form against FP64 on the 128^3 x 6 cube")
    ap.add_argument("--mixed-size", type=int, default=128)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="batched form: the precision of the batch and of its sequential "
                         "per-case reference")
    ap.add_argument("--converge", type=int, default=0,
                    help="mixed form: also iterate both forms to a 1e-6 residual drop "
                         "(at most this many iterations) and time it")
    ap.add_argument("--ncase", type=int, default=64)
    ap.add_argument("--tune-trials", type=int, default=3,
                    help="timed iterations per autotuner trial (0: no autotuning)")
    ap.add_argument("--parts", type=int, default=0,
                    help="partition form: parts of the mesh (default: one per GPU)")
    ap.add_argument("--profile-region", action="store_true",
                    help="bracket the timed iterations with cudaProfilerStart/Stop (for ncu "
                         "--profile-from-start off)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# algorithmic bytes per iteration (each input array element counted once per
# kernel that needs it, each output once)
# ---------------------------------------------------------------------------

def algorithmic_bytes(C, G, F, N, K):
    n = C + G
    S = 2 * F - G
    csr = 4 * (C + 1) + 4 * S
    return {
        # flux + res, time step + CellIsMG + limit, Diag: one fused gather
        "face_gather": F * (32 + 8) + F * 24 + 40 * n + 24 * n + 8 * C + csr +
                       40 * C + 8 * C + 8 * C,
        "sweep_fwd": F * 40 + csr + 40 * n + 40 * C + 8 * C + 40 * C,
        # backward sweep with the update fused: + the new state
        "sweep_bwd_update": F * 40 + csr + 40 * n + 40 * C + 8 * C + 40 * C + 40 * C,
        "node_values": 40 * n + 12 * K + 8 * K + 8 * N + 40 * N,
        "grad_faces": 40 * N + F * (12 + 32 + 8) + 8 * C + 120 * n,
        "norm": 0,
    }


def kernel_of_phase(phase: str, sweep_mode: int) -> str:
    persistent = {"sweep_fwd": "k_sweep_fwd_chunk", "sweep_bwd_update": "k_sweep_bwd_chunk"}
    per_level = {"sweep_fwd": "k_sweep_fwd", "sweep_bwd_update": "k_sweep_bwd"}
    other = {"face_gather": "k_face_flux+k_face_gather", "node_values": "k_node_values",
             "grad_faces": "k_grad_faces", "norm": "k_norm_final"}
    return (persistent if sweep_mode == 1 else per_level).get(phase, other.get(phase, phase))


def read_traffic(kernel: str, workload_name: str):
    """DRAM bytes per launch of `kernel` (a "+"-joined phase of several
    kernels: their sum) from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    if "+" in kernel:
        parts = [read_traffic(k, workload_name) for k in kernel.split("+")]
        return None if any(p is None for p in parts) else sum(parts)
    for line in open(path):
        parts = line.split()
        if len(parts) >= 3 and not line.startswith("#") and parts[0] == kernel and \
                parts[1] == workload_name:
            try:
                return float(parts[2])
            except ValueError:
                return None
    return None


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own code (oracle/_ref), else the C oracle
# ---------------------------------------------------------------------------

def cpu_reference_run(mesh, wl, iters, threads=None, tdtree=True):
    from oracle import refrun
    x0, y0, z0 = wl.get("bump_center", (0.5, 0.5, 0.5))
    flow = dict(mach=wl["mach"], alpha=wl["alpha"], cfl_start=wl["cfl"], cfl_end=wl["cfl"],
                n_steps=iters, bump_amp=wl["bump_amp"], bump_sigma=wl["bump_sigma"],
                bump_x0=x0, bump_y0=y0, bump_z0=z0)
    threads = threads or os.cpu_count()
    if tdtree and refrun.available(tdtree=True):
        r = refrun.run(mesh, flow, tdtree=True, threads=threads, light=True, dump=False)
        kind, desc = "reference", f"reference TDTree build (OpenMP, {threads} threads)"
    elif refrun.available():
        r = refrun.run(mesh, flow, light=True, dump=False)
        threads, kind, desc = 1, "reference", "reference serial build (1 thread)"
    else:
        return None
    return dict(iter_times=list(r["iter_times"]), threads=threads, kind=kind, desc=desc)


def cpu_port_run(pg, params, iters):
    from oracle import oracle_py
    o = oracle_py.OracleSolver(pg.arrays, params.as_dict(), pg.q0,
                               (pg.n_node, pg.n_face, pg.n_cell, pg.n_bface))
    times = []
    for _ in range(iters):
        t = time.perf_counter()
        o.step()
        times.append(time.perf_counter() - t)
    return dict(iter_times=times, threads=1, kind="port", desc="C restatement (1 thread)")


def ref_flow(wl, iters):
    return dict(mach=wl["mach"], alpha=wl["alpha"], cfl_start=wl["cfl"], cfl_end=wl["cfl"],
                n_steps=iters, bump_amp=wl["bump_amp"], bump_sigma=wl["bump_sigma"],
                bump_x0=0.5, bump_y0=0.5, bump_z0=0.5)


def cpu_baseline(mesh, pg, params, wl, iters=16):
    """The reference's threaded build on all host cores over `iters` full
    iterations (a sample of a few seconds at 64^3), timed per iteration."""
    r = cpu_reference_run(mesh, wl, iters)
    if r is None:
        r = cpu_port_run(pg, params, max(2, iters // 8))
    t = sum(r["iter_times"])
    return {"value": pg.n_cell * len(r["iter_times"]) / t, "unit": UNIT, "cores": r["threads"],
            "kind": r["kind"],
            "sample": f"{wl['name']}, {len(r['iter_times'])} full iterations after setup, "
                      f"{r['desc']}, {t:.2f} s"}


def parity_vs_reference(mesh, pg, params, wl, device, iters):
    """The bench's own workload run `iters` iterations by the reference's
    serial build (oracle/_ref/minifs_ref, the unmodified kernels on one core)
    and by a fresh GPU context from the same seeded mesh and initial state:
    entries of the final state, residual, gradient and dt extrema that
    differ, and the largest relative difference of the per-iteration
    residual norms (a reduction of its own order on the GPU).  The serial
    run's iteration times are the one-core baseline."""
    from oracle import refrun
    from minifs_b200.solver import Solver
    if not refrun.available():
        return None, None
    t0 = time.perf_counter()
    ref = refrun.run(mesh, ref_flow(wl, iters), dump=True, dump_iters="-1")
    ref_s = time.perf_counter() - t0
    s = Solver(pg, params, device=device)
    s.calculate_gradient()
    norms = s.iterate(iters)
    fields = {"q": ("final.q", s.download("q")), "res": ("final.res", s.download("res")),
              "dqdx": ("final.dqdx", s.download("dqdx")),
              "dqdy": ("final.dqdy", s.download("dqdy")),
              "dqdz": ("final.dqdz", s.download("dqdz"))}
    ext = np.array(s.dt_extrema)
    s.close()
    out = {"against": "reference serial build (oracle/_ref/minifs_ref: the unmodified MiniFS "
                      "kernels), same seeded mesh, parameters and initial state",
           "iterations": iters, "fields": {}}
    total = 0
    for name, (key, got) in fields.items():
        want = ref[key]
        diff = got.view(np.int64) != want.view(np.int64)
        nd = int(np.count_nonzero(diff))
        total += nd
        out["fields"][name] = {"entries": int(want.size), "differing": nd,
                               "max_abs_diff": float(np.max(np.abs(got - want))) if nd else 0.0}
    dex = int(np.count_nonzero(ext.view(np.int64) != ref["final.dt_extrema"].view(np.int64)))
    out["fields"]["dt_extrema"] = {"entries": 2, "differing": dex}
    total += dex
    rn = ref["norms"].reshape(iters, 5)
    out["norms_max_rel_diff"] = float(np.max(np.abs(norms - rn) / np.abs(rn)))
    out["differing_total"] = total
    out["bitwise_equal"] = total == 0
    ts = float(sum(ref["iter_times"]))
    serial = {"value": pg.n_cell * iters / ts, "unit": UNIT, "cores": 1,
              "sample": f"reference serial build, {iters} iterations, {ts:.2f} s "
                        f"(run with its set-up and dumps {ref_s:.1f} s)"}
    return out, serial


# ---------------------------------------------------------------------------

def build_case(wl):
    """(mesh, params, prepared grid, seconds of the host preprocessing)."""
    from minifs_b200 import grid as gr, meshgen
    mesh = meshgen.cube_mesh(wl["n"], jitter=wl["jitter"], seed=wl["seed"])
    params = gr.make_params(mach=wl["mach"], alpha=wl["alpha"], cfl_start=wl["cfl"])
    t = time.perf_counter()
    pg = gr.prepare(mesh, params, bump_amp=wl["bump_amp"], bump_sigma=wl["bump_sigma"])
    return mesh, params, pg, time.perf_counter() - t


def prep_on_gpu(mesh, params, wl, pg, host_s, device):
    """The same preprocessing with metrics and node weights on the GPU: wall
    seconds from the raw host mesh to host arrays (copies included; the
    second of two runs), device time of its kernels, and whether every array
    matches the host result bit for bit."""
    from minifs_b200 import grid as gr
    kw = dict(bump_amp=wl["bump_amp"], bump_sigma=wl["bump_sigma"], device=device)
    gr.prepare(mesh, params, **kw)
    st = {}
    t = time.perf_counter()
    pgd = gr.prepare(mesh, params, stats=st, **kw)
    gpu_s = time.perf_counter() - t
    same = all(np.asarray(pgd.arrays[k]).tobytes() == np.asarray(pg.arrays[k]).tobytes()
               for k in pg.arrays) and pgd.q0.tobytes() == pg.q0.tobytes()
    return {"host_s": host_s, "gpu_s": gpu_s, "gpu_kernels_ms": st["gpu_kernels_s"] * 1e3,
            "gpu_upload_and_kernels_s": st["gpu_run_s"], "gpu_download_s": st["gpu_download_s"],
            "init_flow_on_host_s": st["init_flow_s"], "speedup": host_s / gpu_s,
            "bitwise_equal": bool(same),
            "steps": "SpecifyBC, ComputeMetrics, AllocAndInitFlowfield + SetGhostVariables, "
                     "CalC2N, ComputeWeight3D_Node, FindNodeSYMM"}


def setup_on_device(mesh, params, wl, device):
    """Raw host mesh to a ready context with the grid kept on the device:
    the GPU preprocessing, the initial state on the host from the device's
    centroids and normals, and the context built on the device
    (mfg_create_from_prep).  Seconds of each part."""
    from minifs_b200 import grid as gr
    from minifs_b200.solver import Solver
    t0 = time.perf_counter()
    prep = gr.DevicePrep(mesh, device=device)
    t1 = time.perf_counter()
    q0 = prep.init_flow(params, bump_amp=wl["bump_amp"], bump_sigma=wl["bump_sigma"])
    t2 = time.perf_counter()
    s = Solver.from_device_prep(prep, params, q0)
    t3 = time.perf_counter()
    s.close()
    prep.close()
    return {"total_s": t3 - t0, "prep_s": t1 - t0, "init_flow_s": t2 - t1,
            "create_s": t3 - t2}


def run_reference_arm(args, rank, world):
    wl = workload(args.size)
    if rank != 0:
        return
    from minifs_b200 import meshgen
    mesh = meshgen.cube_mesh(wl["n"], jitter=wl["jitter"], seed=wl["seed"])
    total = args.warmup + args.steps
    r = cpu_reference_run(mesh, wl, total)
    if r is None:
        from minifs_b200 import grid as gr
        params = gr.make_params(mach=wl["mach"], alpha=wl["alpha"], cfl_start=wl["cfl"])
        pg = gr.prepare(mesh, params, bump_amp=wl["bump_amp"], bump_sigma=wl["bump_sigma"])
        r = cpu_port_run(pg, params, total)
    timed = r["iter_times"][args.warmup:]
    t = sum(timed)
    value = mesh.n_cell * len(timed) / t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t / len(timed), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl["name"], "cells": mesh.n_cell, "parallelism": "cpu"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["threads"],
                             "kind": r["kind"],
                             "sample": f"{wl['name']}: {args.warmup} warm-up + {args.steps} "
                                       f"timed full iterations, {r['desc']}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batched_workload(ncase=64, seed=2024):
    """64 cube cases, n uniform in [8, 48] hexes per edge (n^3 x 6 tets), Mach
    U(0.3, 0.8), alpha U(-5, 5) deg, jitter U(0, 0.2)h, CFL 10."""
    rng = np.random.default_rng(seed)
    cases = []
    for k in range(ncase):
        cases.append(dict(n=int(rng.integers(8, 49)), mach=float(rng.uniform(0.3, 0.8)),
                          alpha=float(rng.uniform(-5.0, 5.0)),
                          jitter=float(rng.uniform(0.0, 0.2)), seed=1000 + k, cfl=10.0,
                          bump_amp=0.05, bump_sigma=0.1))
    return dict(name=f"batched{ncase}_cube_n8-48_fp64", cases=cases)


def batched_cells(bw):
    return [6 * c["n"] ** 3 for c in bw["cases"]]


def build_batched(bw, which=None):
    """Grids and parameters of the cases `which` (default: all)."""
    from minifs_b200 import grid as gr, meshgen
    grids, params = [], []
    for k, c in enumerate(bw["cases"]):
        if which is not None and k not in which:
            continue
        m = meshgen.cube_mesh(c["n"], jitter=c["jitter"], seed=c["seed"])
        p = gr.make_params(mach=c["mach"], alpha=c["alpha"], cfl_start=c["cfl"])
        grids.append(gr.prepare(m, p, bump_amp=c["bump_amp"], bump_sigma=c["bump_sigma"]))
        params.append(p)
    return grids, params


def measure(s, counts, args, stream, dist, world, local, total_cells=None):
    """Timed fused iterations of a context, its phase breakdown, roofline and
    the end-to-end host-buffer run.  counts = (C, G, F, N, K, n) of this
    rank; total_cells: cells of the whole job (default: world replicas of
    C).  Device times are the max over the ranks."""
    import torch
    from minifs_b200 import _lib, shard
    C, G, F, N, K, n = counts
    total = world * C if total_cells is None else total_cells
    info = s.info()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(ms):
        return shard.reduce_max(ms, dist, "cuda")

    # launch parameters chosen by measurement on this grid (the state is left
    # as it was), then the warm-up (builds the CUDA graphs)
    s.calculate_gradient()
    tuned = s.autotune(args.tune_trials) if args.tune_trials > 0 else None
    info = s.info()
    s.iterate(max(args.warmup, 3), norms=False)
    barrier()
    launches0 = _lib.kernel_launches()
    with ClockSampler(local) as clk:
        barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        if args.profile_region:
            torch.cuda.cudart().cudaProfilerStart()
        ev0.record(stream)
        s.iterate(args.steps, norms=False)
        ev1.record(stream)
        ev1.synchronize()
        if args.profile_region:
            torch.cuda.cudart().cudaProfilerStop()
        barrier()
    launches = _lib.kernel_launches() - launches0
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    out = {"ms": ms, "value": total * args.steps / (ms / 1e3), "launches": int(launches),
           "clocks": clk.summary(), "info": info,
           "autotuned": None if tuned is None else dict(
               tuned, sweep_chunks=info["sweep_chunks"], sweep_kernel=info["sweep_kernel"],
               sweep_chunking=info["sweep_chunking"], sweep_model_us=info["sweep_model_us"])}

    # phase breakdown with CUDA events on the same stream (same fused kernels)
    phase_iters = max(3, min(args.steps, 10))
    phases = s.profile_phases(phase_iters)
    alg = algorithmic_bytes(C, G, F, N, K)
    peak, peak_kind = measured_peak()
    per_level = info["sweep_mode"] == 0
    nl = {"face_gather": 2, "sweep_fwd": info["fw_levels"] if per_level else 1,
          "sweep_bwd_update": info["bw_levels"] if per_level else 1,
          "node_values": 1, "grad_faces": 1, "norm": 1}
    phase_out = {}
    for ph, tot in phases.items():
        per_it = tot / phase_iters
        phase_out[ph] = {"ms_per_iter": per_it, "launches_per_iter": nl[ph],
                         "alg_bytes": alg[ph],
                         "gbs": (alg[ph] / (per_it / 1e3) / 1e9) if per_it > 0 else None}
    dom = max(phases, key=lambda k: phases[k])
    dom_ms_launch = phases[dom] / phase_iters / nl[dom]
    dom_bytes_launch = alg[dom] / nl[dom]
    achieved = dom_bytes_launch / (dom_ms_launch / 1e3) / 1e9
    dom_kernel = kernel_of_phase(dom, info["sweep_mode"])
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                       "frac": achieved / peak, "traffic": None, "kernel": dom_kernel,
                       "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                       "alg_bytes_per_launch": dom_bytes_launch,
                       "ms_per_launch": dom_ms_launch}
    fg_ms = sum(phases[p] for p in ("face_gather", "node_values", "grad_faces")) / phase_iters
    fg_bytes = alg["face_gather"] + alg["node_values"] + alg["grad_faces"]
    out["flux_plus_gradient"] = {"gbs": fg_bytes / (fg_ms / 1e3) / 1e9,
                                 "frac": fg_bytes / (fg_ms / 1e3) / 1e9 / peak}
    out["phases"] = phase_out

    # end to end through the C ABI with host buffers (pinned), every step:
    # host state in, one iteration, host state and the step's residual norms
    # out; then the same with the residual field copied out as well
    qh = torch.empty(5 * n, dtype=torch.float64, pin_memory=True).numpy()
    qo = torch.empty(5 * n, dtype=torch.float64, pin_memory=True).numpy()
    rh = torch.empty(5 * C, dtype=torch.float64, pin_memory=True).numpy()
    ncase = int(info.get("ncase", 1))
    nh = torch.empty(5 * ncase, dtype=torch.float64, pin_memory=True).numpy()

    def e2e_run(res_field):
        nonlocal qh, qo
        qh[:] = s.download("q")
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            s.iterate_host(1, qh, qo, rh if res_field else None, nh)
            qh, qo = qo, qh
        e1.record(stream)
        e1.synchronize()
        return max_over_ranks(e0.elapsed_time(e1))

    e2e_ms = e2e_run(False)
    e2e_res_ms = e2e_run(True)
    out["e2e"] = {"value": total * args.e2e_steps / (e2e_ms / 1e3), "unit": UNIT,
                  "h2d_bytes_per_step": 8 * 5 * n, "d2h_bytes_per_step": 8 * 5 * n + 8 * 5 * ncase,
                  "steps": args.e2e_steps,
                  "api": "mfg_iterate_host (C ABI, pinned host buffers): state in, state and "
                         "residual norms out",
                  "with_residual_field": {
                      "value": total * args.e2e_steps / (e2e_res_ms / 1e3),
                      "d2h_bytes_per_step": 8 * 5 * n + 8 * 5 * C + 8 * 5 * ncase}}
    return out


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    # a dedicated (capturable) stream shared by the library and the events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    if args.form == "batched":
        run_batched(args, rank, world, local, stream, dist)
    elif args.form in ("mixed", "channel"):
        run_mixed(args, rank, world, local, stream, dist)
    elif args.form == "partition":
        run_partition(args, rank, world, local, dist)
    else:
        run_single(args, rank, world, local, stream, dist)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_single(args, rank, world, local, stream, dist):
    from minifs_b200.solver import Solver
    wl = workload(args.size)
    mesh, params, pg, host_prep_s = build_case(wl)
    prep = prep_on_gpu(mesh, params, wl, pg, host_prep_s, local)
    t = time.perf_counter()
    s = Solver(pg, params, device=local)
    prep["solver_create_s"] = time.perf_counter() - t
    prep["device_path"] = setup_on_device(mesh, params, wl, local)
    prep["host_path_setup_s"] = host_prep_s + prep["solver_create_s"]
    s.set_stream(stream.cuda_stream)
    C, G, F, N = pg.n_cell, pg.n_bface, pg.n_face, pg.n_node
    K = int(pg.arrays["nnpc"].sum())
    r = measure(s, (C, G, F, N, K, pg.n), args, stream, dist, world, local)
    r["roofline"]["traffic"] = read_traffic(r["roofline"]["kernel"], wl["name"])
    norms = s.residual_norm()
    info = r["info"]
    s.close()
    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(mesh, pg, params, wl)
        except Exception as e:  # reported, never silently replaced
            cpu = {"error": str(e)[:200]}
        try:
            parity, serial = parity_vs_reference(mesh, pg, params, wl, local, args.parity_iters)
            if serial is not None and isinstance(cpu, dict) and "value" in cpu:
                cpu["serial_1core"] = serial
        except Exception as e:
            parity = {"error": str(e)[:300]}
    if rank == 0:
        line = {
            "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": wl["name"], "form": "fp64", "cells": C, "faces": F,
                       "nodes": N, "ghosts": G, "precision": "fp64 (bit-faithful)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single",
                       "l2": "no flush: working set "
                             f"{info['device_bytes'] / 2**20:.0f} MiB > 126 MB L2",
                       "lusgs_levels": {"forward": info["fw_levels"],
                                        "backward": info["bw_levels"]},
                       "sweeps": "persistent chunked" if info["sweep_mode"] == 1 else
                                 "one launch per level"},
            "autotuned": r["autotuned"],
            "roofline": r["roofline"],
            "flux_plus_gradient": r["flux_plus_gradient"],
            "phases": r["phases"],
            "cpu_baseline": cpu,
            "parity": parity,
            "e2e": r["e2e"],
            "gpu_launches": r["launches"],
            "clocks": r["clocks"],
            "residual_norm": [float(x) for x in norms],
            "prep": prep,
        }
        if world == 1 and not args.no_forms:
            line["forms"] = run_forms(args, local, stream, not args.no_cpu_baseline)
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# the metric's other legs in the default run: mixed precision, batched cases
# and the channel, each to its residual drop (bounded) with clocks sampled
# ---------------------------------------------------------------------------

def _drop_runs(prep, q0, params, C, stream, drop, max_iter, precisions, fp64_flux_below):
    """Each precision from the same device-prepared grid and initial state to
    `drop` (at most max_iter iterations): iterations, device ms, throughput,
    final state."""
    from minifs_b200.solver import Solver
    out, states = {}, {}
    for prec in precisions:
        s = Solver.from_device_prep(prep, params, q0, precision=prec)
        s.set_stream(stream.cuda_stream)
        s.calculate_gradient()
        tail = fp64_flux_below if prec == "mixed" else None
        it, ms, reached, switched = to_drop(s, stream, drop, max_iter, fp64_flux_below=tail)
        info = s.info()
        out[prec] = {"iterations": it, "ms": ms, "drop": reached, "reached": reached <= drop,
                     "cell_updates_per_s": C * it / (ms / 1e3),
                     "sweep_chunking": info["sweep_chunking"],
                     "sweep_model_us": info["sweep_model_us"]}
        if tail is not None:
            out[prec]["fp64_flux_from_iteration"] = switched
        states[prec] = s.download("q")
        s.close()
    return out, states


def _form_errors(states, n, p_bar):
    from minifs_b200.compare import state_component_err, state_rel_err
    return {"physical_scales": state_rel_err(states["mixed"], states["fp64"], n, p_bar),
            "per_component": state_component_err(states["mixed"], states["fp64"], n)}


def form_mixed(args, local, stream, with_cpu):
    """Configuration 3: the 128^3 x 6 cube (Mach 0.8, alpha 1.25 deg, CFL 20),
    FP64 and mixed forms each to a 1e-6 residual drop."""
    from minifs_b200 import grid as gr, meshgen
    wl = mixed_workload(args.mixed_size)
    mesh = meshgen.cube_mesh(wl["n"], jitter=wl["jitter"], seed=wl["seed"])
    params = gr.make_params(mach=wl["mach"], alpha=wl["alpha"], cfl_start=wl["cfl"])
    prep = gr.DevicePrep(mesh, device=local)
    q0 = prep.init_flow(params, bump_amp=wl["bump_amp"], bump_sigma=wl["bump_sigma"])
    C, n = prep.n_cell, prep.n
    with ClockSampler(local) as clk:
        runs, states = _drop_runs(prep, q0, params, C, stream, 1e-6, args.form_iters,
                                  ("fp64", "mixed"), None)
    prep.close()
    f, m = runs["fp64"], runs["mixed"]
    out = {"workload": wl["name"], "cells": C, "drop_target": 1e-6, "fp64": f, "mixed": m,
           "mixed_over_fp64": m["cell_updates_per_s"] / f["cell_updates_per_s"],
           "time_to_drop_ratio": f["ms"] / m["ms"] if m["reached"] and f["reached"] else None,
           "state_rel_err_vs_fp64_at_drop": _form_errors(states, n, params.p_bar),
           "clocks": clk.summary()}
    if with_cpu:
        # the TDTree build's own set-up (METIS on the cell graph) takes minutes
        # at 12.6M cells: the serial build by default, the threaded one on
        # request
        out["cpu_baseline"] = _cpu_sample(mesh, wl, 1, tdtree=args.form_cpu == "tdtree")
    return out


def form_channel(args, local, stream, with_cpu):
    """Configuration 5: the 4x1x1 channel with a wall bump (Mach 0.7, CFL 30),
    FP64 and mixed forms each to a 1e-8 residual drop (the mixed form's flux
    goes FP64 below a 1e-6 drop), and the mixed wall pressure against FP64."""
    from minifs_b200 import grid as gr, meshgen
    wl = channel_workload()
    mesh = meshgen.channel_mesh(jitter=wl["jitter"], seed=wl["seed"])
    params = gr.make_params(mach=wl["mach"], alpha=wl["alpha"], cfl_start=wl["cfl"])
    prep = gr.DevicePrep(mesh, device=local)
    q0 = prep.init_flow(params, bump_amp=wl["bump_amp"], bump_sigma=wl["bump_sigma"],
                        bump_center=wl["bump_center"])
    C, n, G = prep.n_cell, prep.n, prep.n_bface
    with ClockSampler(local) as clk:
        runs, states = _drop_runs(prep, q0, params, C, stream, wl["drop"], args.form_iters * 3,
                                  ("fp64", "mixed"), 1e-6)
    bct = np.asarray(prep.bctype)[:G]
    prep.close()
    wf = np.nonzero(bct == 3)[0]
    c1 = np.asarray(mesh.f2c).reshape(-1, 2)[wf, 0]
    pa, pb = states["mixed"][4 * n + c1], states["fp64"][4 * n + c1]
    d = np.abs(pa - pb) / (np.abs(pb) + params.p_bar)
    f, m = runs["fp64"], runs["mixed"]
    out = {"workload": wl["name"], "cells": C, "drop_target": wl["drop"], "fp64": f, "mixed": m,
           "mixed_over_fp64": m["cell_updates_per_s"] / f["cell_updates_per_s"],
           "time_to_drop_ratio": f["ms"] / m["ms"] if m["reached"] and f["reached"] else None,
           "state_rel_err_vs_fp64_at_drop": _form_errors(states, n, params.p_bar),
           "wall_pressure_rel_err_vs_fp64": {"max": float(d.max()),
                                             "rms": float(np.sqrt(np.mean(d * d))),
                                             "faces": int(wf.size),
                                             "scale": "p + p_bar"},
           "clocks": clk.summary()}
    if with_cpu:
        out["cpu_baseline"] = _cpu_sample(mesh, wl, args.form_cpu_iters, tdtree=True)
    return out


def _cpu_sample(mesh, wl, iters, tdtree):
    """The reference's threaded build on all host cores (tdtree) or its serial
    build on one core, capped at `iters` iterations of the form's workload
    (its set-up time stated apart)."""
    t0 = time.perf_counter()
    r = cpu_reference_run(mesh, wl, iters, tdtree=tdtree)
    if r is None:
        return None
    t = sum(r["iter_times"])
    return {"value": mesh.n_cell * len(r["iter_times"]) / t, "unit": UNIT, "cores": r["threads"],
            "kind": r["kind"],
            "sample": f"{wl['name']}: {len(r['iter_times'])} full iterations (iteration-capped) "
                      f"after set-up, {r['desc']}, {t:.2f} s; run with its set-up "
                      f"{time.perf_counter() - t0:.1f} s"}


def cpu_sample_batched(bw, ncase=8, iters=5, seed=7):
    """The reference's threaded build on all host cores over a seeded subset
    of the batch's cases, one case after another (its per-case runs), capped
    at `iters` iterations each: cell-updates over the summed iteration times
    (each case's set-up stated apart)."""
    from minifs_b200 import meshgen
    rng = np.random.default_rng(seed)
    pick = sorted(int(i) for i in rng.choice(len(bw["cases"]), size=min(ncase, len(bw["cases"])),
                                             replace=False))
    t0 = time.perf_counter()
    updates, t, r, cells = 0, 0.0, None, 0
    for i in pick:
        c = bw["cases"][i]
        mesh = meshgen.cube_mesh(c["n"], jitter=c["jitter"], seed=c["seed"])
        r = cpu_reference_run(mesh, c, iters, tdtree=True)
        if r is None:
            return None
        updates += mesh.n_cell * len(r["iter_times"])
        t += sum(r["iter_times"])
        cells += mesh.n_cell
    return {"value": float(updates / t), "unit": UNIT, "cores": r["threads"], "kind": r["kind"],
            "sample": f"{bw['name']}: cases {pick} ({cells} cells) one after another, "
                      f"{iters} full iterations each (iteration-capped) after set-up, "
                      f"{r['desc']}, {t:.2f} s; run with its set-ups "
                      f"{time.perf_counter() - t0:.1f} s"}


def form_batched(args, local, stream, with_cpu=False):
    """Configuration 4: 64 cube cases (n uniform in 8..48, Mach U(0.3, 0.8),
    alpha U(-5, 5) deg, jitter U(0, 0.2)h) in one context against the same
    cases one after another in their own contexts, FP64 and mixed, each over
    the same timed iterations."""
    import torch
    from minifs_b200.solver import BatchSolver, Solver
    bw = batched_workload(args.ncase)
    grids, params = build_batched(bw)
    cells = int(sum(g.n_cell for g in grids))
    steps = args.form_batch_steps
    out = {"workload": bw["name"], "ncase": len(grids), "cells": cells, "steps": steps}
    with ClockSampler(local) as clk:
        for prec in ("fp64", "mixed"):
            seq_ms = 0.0
            for pg, p in zip(grids, params):
                s = Solver(pg, p, device=local, precision=prec)
                s.set_stream(stream.cuda_stream)
                s.calculate_gradient()
                s.iterate(3, norms=False)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                s.iterate(steps, norms=False)
                e1.record(stream)
                e1.synchronize()
                seq_ms += e0.elapsed_time(e1)
                s.close()
            b = BatchSolver(grids, params, device=local, precision=prec)
            b.set_stream(stream.cuda_stream)
            b.calculate_gradient()
            # the batch's sweep kernels and chunks as chosen at creation (a
            # rebuild of 12M cells takes seconds); the other knobs timed
            tuned = b.autotune(2, rebuild=False) if args.tune_trials > 0 else None
            b.iterate(3, norms=False)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.iterate(steps, norms=False)
            e1.record(stream)
            e1.synchronize()
            bms = e0.elapsed_time(e1)
            info = b.info()
            b.close()
            bv, sv = cells * steps / (bms / 1e3), cells * steps / (seq_ms / 1e3)
            out[prec] = {"value": bv, "unit": UNIT, "ms_per_step": bms / steps,
                         "sequential": {"value": sv, "ms_per_step": seq_ms / steps,
                                        "how": "each case in its own context, graph-captured "
                                               "fused iterations, one after another; device "
                                               "time summed"},
                         "batched_over_sequential": bv / sv,
                         "autotuned": tuned,
                         "sweep_kernel": info["sweep_kernel"],
                         "sweep_chunks": info["sweep_chunks"],
                         "sweep_chunking": info["sweep_chunking"],
                         "sweep_model_us": info["sweep_model_us"]}
    out["clocks"] = clk.summary()
    if with_cpu:
        try:
            out["cpu_baseline"] = cpu_sample_batched(bw)
        except Exception as e:  # reported beside the GPU figures
            out["cpu_baseline"] = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
    return out


def run_forms(args, local, stream, with_cpu):
    """The metric's mixed, batched and channel legs (configurations 3-5)."""
    forms = {}
    for name, fn in (("mixed", lambda: form_mixed(args, local, stream, with_cpu)),
                     ("channel", lambda: form_channel(args, local, stream, with_cpu)),
                     ("batched", lambda: form_batched(args, local, stream, with_cpu))):
        t0 = time.perf_counter()
        try:
            forms[name] = fn()
        except Exception as e:  # reported, never silently replaced
            forms[name] = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
        forms[name]["wall_s"] = time.perf_counter() - t0
    return forms


def run_partition(args, rank, world, local, dist):
    """The fp64 workload's mesh as K parts iterated in step (the reference's
    MPI mode), part z on rank z mod world."""
    import torch
    from minifs_b200 import _lib, grid as gr, meshgen, shard
    from minifs_b200 import partition as pa
    wl = workload(args.size)
    mesh = meshgen.cube_mesh(wl["n"], jitter=wl["jitter"], seed=wl["seed"])
    params = gr.make_params(mach=wl["mach"], alpha=wl["alpha"], cfl_start=wl["cfl"])
    K = args.parts or world
    t = time.perf_counter()
    part_of = pa.rcb_parts(mesh, K)
    zones = [z for z in range(K) if z % world == rank]
    parts, whole, held = pa.build_parts(mesh, params, K, part_of=part_of, zones=zones,
                                        device_of=lambda z: local, bump_amp=wl["bump_amp"],
                                        bump_sigma=wl["bump_sigma"])
    ex = pa.DistExchange() if world > 1 else pa.LocalExchange()
    d = pa.Decomposed(held, ex)
    setup_s = time.perf_counter() - t
    stream = next(iter(held.values())).stream
    d.iterate(max(args.warmup, 3))

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    launches0 = _lib.kernel_launches()
    with ClockSampler(local) as clk:
        barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        norms = d.iterate(args.steps)
        ev1.record(stream)
        ev1.synchronize()
        barrier()
    launches = _lib.kernel_launches() - launches0
    ms = shard.reduce_max(ev0.elapsed_time(ev1), dist, "cuda")
    C = whole.n_cell
    cut = sum(len(p.interfaces.nbz) for p in parts) // 2
    if rank == 0:
        line = {
            "metric": METRIC, "value": C * args.steps / (ms / 1e3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl["name"], "form": "partition", "cells": C, "parts": K,
                       "part_cells": [int(p.cells.size) for p in parts], "cut_faces": cut,
                       "partitioner": "recursive coordinate bisection",
                       "parallelism": f"{K} parts on {world} GPU(s)",
                       "exchange": "NCCL p2p + all-reduce" if world > 1 else "device copies",
                       "l2": "no flush: working set far above the 126 MB L2"},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "residual_norm": [float(x) for x in norms[-1]],
            "setup_s": setup_s,
        }
        print(json.dumps(line), flush=True)
    d.close()


def mixed_workload(n: int) -> dict:
    """Cube n^3 x 6 tets, jitter 0.1h, Mach 0.8, alpha 1.25 deg, CFL 20,
    far field on all sides, 5% density bump."""
    return dict(name=f"cube{n}x6_M0.8_a1.25_cfl20", n=n, jitter=0.1, seed=1, mach=0.8,
                alpha=1.25, cfl=20.0, bump_amp=0.05, bump_sigma=0.1)


def channel_workload() -> dict:
    """Box 4x1x1 of 192x48x48 hexes x 6 tets (2,654,208 cells), jitter 0.1h,
    a slip wall at the bottom carrying a Gaussian bump (height 0.05, width
    0.2, at x = 1.5), far field on the other faces; Mach 0.7, alpha 0, CFL
    30, 5% density bump; converged to a 1e-8 residual drop."""
    return dict(name="channel192x48x48x6_M0.7_a0_cfl30", jitter=0.1, seed=5, mach=0.7,
                alpha=0.0, cfl=30.0, bump_amp=0.05, bump_sigma=0.1, drop=1e-8,
                bump_center=(2.0, 0.5, 0.5))


def to_drop(s, stream, target, max_iter, chunk=100, fp64_flux_below=None):
    """Iterate until the rho residual norm falls below target x its first
    value; returns (iterations, device ms, drop reached, iterations at the
    switch to the FP64 flux or None).  With ``fp64_flux_below`` (mixed form)
    the flux switches to FP64 once the drop is below that value."""
    import torch
    first, it, ms, drop, switched = None, 0, 0.0, 1.0, None
    while it < max_iter:
        if fp64_flux_below is not None and switched is None and drop <= fp64_flux_below:
            s.set_flux_fp64(True)
            switched = it
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nrm = s.iterate(chunk)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        if first is None:
            first = nrm[0, 0]
        hit = np.nonzero(nrm[:, 0] <= target * first)[0]
        if hit.size:
            it += int(hit[0]) + 1
            drop = float(nrm[hit[0], 0] / first)
            break
        it += chunk
        drop = float(nrm[-1, 0] / first)
    return it, ms, drop, switched


def run_mixed(args, rank, world, local, stream, dist):
    """FP64 and mixed forms on the same grid: throughput of each, the mixed
    state's error against FP64 after the same iterations, and (--converge)
    the iterations and time each needs for a 1e-6 residual drop."""
    from minifs_b200 import grid as gr, meshgen
    from minifs_b200.solver import Solver
    if args.form == "channel":
        wl = channel_workload()
        mesh = meshgen.channel_mesh(jitter=wl["jitter"], seed=wl["seed"])
    else:
        wl = mixed_workload(args.mixed_size)
        wl["drop"] = 1e-6
        mesh = meshgen.cube_mesh(wl["n"], jitter=wl["jitter"], seed=wl["seed"])
    params = gr.make_params(mach=wl["mach"], alpha=wl["alpha"], cfl_start=wl["cfl"])
    pg = gr.prepare(mesh, params, bump_amp=wl["bump_amp"], bump_sigma=wl["bump_sigma"],
                    bump_center=wl.get("bump_center", (0.5, 0.5, 0.5)))
    drop_key = f"to_drop_{wl['drop']:.0e}".replace("e-0", "e-")
    C, G, F, N = pg.n_cell, pg.n_bface, pg.n_face, pg.n_node
    K = int(pg.arrays["nnpc"].sum())
    res = {}
    states = {}
    for prec in ("fp64", "mixed"):
        s = Solver(pg, params, device=local, precision=prec)
        s.set_stream(stream.cuda_stream)
        r = measure(s, (C, G, F, N, K, pg.n), args, stream, dist, world, local)
        states[prec] = s.download("q")
        r["residual_norm"] = [float(x) for x in s.residual_norm()]
        if args.converge:
            s2 = Solver(pg, params, device=local, precision=prec)
            s2.set_stream(stream.cuda_stream)
            s2.calculate_gradient()
            # below a 1e-6 drop the mixed form's FP32 dissipation would hold the
            # residual at its rounding floor: the flux goes FP64 from there
            tail = 1e-6 if (prec == "mixed" and wl["drop"] < 1e-6) else None
            it, ms, drop, switched = to_drop(s2, stream, wl["drop"], args.converge,
                                             fp64_flux_below=tail)
            r[drop_key] = {"iterations": it, "ms": ms, "drop": drop,
                           "cell_updates_per_s": C * it / (ms / 1e3)}
            if prec == "mixed" and tail is not None:
                r[drop_key]["fp64_flux_from_iteration"] = switched
            states[prec + "_conv"] = s2.download("q")
            s2.close()
        res[prec] = r
        s.close()
    n = pg.n

    from minifs_b200.compare import state_rel_err

    def rel_err(a, b):
        return state_rel_err(a, b, n, params.p_bar)
    # same number of iterations in both forms: the warm-up, the timed steps
    # and the phase-profile iterations of measure()
    err_same_iters = rel_err(states["mixed"], states["fp64"])
    err_conv = rel_err(states["mixed_conv"], states["fp64_conv"]) if args.converge else None
    wall = None
    bct = np.asarray(pg.arrays["bctype"])[:G]
    wf = np.nonzero(bct == 3)[0]
    if wf.size:
        # pressure on the wall faces (the inner cell's, which the mirror ghost
        # copies): the mixed form against FP64, relative to p + p_bar
        c1 = np.asarray(pg.arrays["f2c"])[2 * wf]

        def wall_err(a, b):
            pa, pb = a[4 * n + c1], b[4 * n + c1]
            d = np.abs(pa - pb) / (np.abs(pb) + params.p_bar)
            return {"max": float(d.max()), "rms": float(np.sqrt(np.mean(d * d))),
                    "faces": int(wf.size)}
        wall = {"same_iterations": wall_err(states["mixed"], states["fp64"]),
                "at_drop": wall_err(states["mixed_conv"], states["fp64_conv"])
                if args.converge else None}
    if rank == 0:
        m, d = res["mixed"], res["fp64"]
        info = m["info"]
        line = {
            "metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": wl["name"], "form": args.form, "cells": C, "faces": F,
                       "precision": "mixed: FP32 Roe averages/dissipation, LU-SGS off-diagonal "
                                    "products and gradient; FP64 central flux, residual, "
                                    "Diag, norm, update",
                       "parallelism": f"replicas x{world}" if world > 1 else "single",
                       "l2": "no flush: working set "
                             f"{info['device_bytes'] / 2**20:.0f} MiB > 126 MB L2",
                       "lusgs_levels": {"forward": info["fw_levels"],
                                        "backward": info["bw_levels"]}},
            "fp64": {"value": d["value"], "ms_per_step": d["ms"] / args.steps,
                     "autotuned": d["autotuned"],
                     "phases": d["phases"], drop_key: d.get(drop_key)},
            "mixed_over_fp64": m["value"] / d["value"],
            "state_rel_err_vs_fp64": {"same_iterations": err_same_iters,
                                      "at_" + drop_key[len("to_drop_"):] + "_drop": err_conv},
            "wall_pressure_rel_err_vs_fp64": wall,
            "autotuned": m["autotuned"],
            "roofline": m["roofline"],
            "flux_plus_gradient": m["flux_plus_gradient"],
            "phases": m["phases"],
            drop_key: m.get(drop_key),
            "cpu_baseline": None,
            "e2e": m["e2e"],
            "gpu_launches": m["launches"],
            "clocks": m["clocks"],
        }
        print(json.dumps(line), flush=True)


def run_batched(args, rank, world, local, stream, dist):
    """64 uneven cases in one context against the same cases run one after
    another, each in its own context (sequential per-case launches).  Under
    N ranks the cases are sharded by cell count (no collective during the
    iterations); both figures are whole-job: all cells over the slowest
    rank's device time."""
    import torch
    from minifs_b200 import shard
    from minifs_b200.solver import BatchSolver, Solver
    bw = batched_workload(args.ncase)
    cells = batched_cells(bw)
    if world > len(cells):
        raise SystemExit("more ranks than cases")
    mine = shard.rank_cases(cells, world, rank)
    grids, params = build_batched(bw, set(mine))
    counts = [0] * 6
    for pg in grids:
        for i, v in enumerate((pg.n_cell, pg.n_bface, pg.n_face, pg.n_node,
                               int(pg.arrays["nnpc"].sum()), pg.n)):
            counts[i] += v
    # sequential per-case launches: each case alone, timed on the device
    seq_ms, seq_cells = 0.0, 0
    for pg, p in zip(grids, params):
        s = Solver(pg, p, device=local, precision=args.precision)
        s.set_stream(stream.cuda_stream)
        s.calculate_gradient()
        s.iterate(max(args.warmup, 3), norms=False)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.iterate(args.steps, norms=False)
        e1.record(stream)
        e1.synchronize()
        seq_ms += e0.elapsed_time(e1)
        seq_cells += pg.n_cell
        s.close()
    total_cells = int(shard.reduce_sum(counts[0], dist, "cuda"))
    seq_ms = shard.reduce_max(seq_ms, dist, "cuda")
    b = BatchSolver(grids, params, device=local, precision=args.precision)
    b.set_stream(stream.cuda_stream)
    r = measure(b, tuple(counts), args, stream, dist, world, local, total_cells=total_cells)
    norms = b.residual_norm()
    info = r["info"]
    seq_value = total_cells * args.steps / (seq_ms / 1e3)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_sample_batched(bw)
        except Exception as e:  # reported beside the GPU figures
            cpu = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
    if rank == 0:
        ns = [c["n"] for c in bw["cases"]]
        line = {
            "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": bw["name"] + ("" if args.precision == "fp64" else "_mixed"),
                       "form": "batched", "ncase": len(ns),
                       "n_min": min(ns), "n_max": max(ns), "cells": total_cells,
                       "cells_rank0": counts[0], "cases_rank0": len(mine),
                       "precision": ("fp64 (bit-faithful per case)" if args.precision == "fp64"
                                     else "mixed (each case as its own mixed run)"),
                       "parallelism": (f"cases sharded over {world} ranks by cell count"
                                       if world > 1 else "single"),
                       "l2": "no flush: working set "
                             f"{info['device_bytes'] / 2**20:.0f} MiB > 126 MB L2",
                       "lusgs_levels": {"forward": info["fw_levels"],
                                        "backward": info["bw_levels"]},
                       "sweeps": "persistent chunked" if info["sweep_mode"] == 1 else
                                 "one launch per level"},
            "sequential": {"value": seq_value, "unit": UNIT, "ms_per_step": seq_ms / args.steps,
                           "how": "each case in its own context, graph-captured fused "
                                  "iterations, cases one after another; device time summed"},
            "batched_over_sequential": r["value"] / seq_value,
            "autotuned": r["autotuned"],
            "roofline": r["roofline"],
            "flux_plus_gradient": r["flux_plus_gradient"],
            "phases": r["phases"],
            "cpu_baseline": cpu,
            "e2e": r["e2e"],
            "gpu_launches": r["launches"],
            "clocks": r["clocks"],
            "residual_norm_max": [float(x) for x in norms.max(axis=0)],
        }
        print(json.dumps(line), flush=True)
    b.close()


if __name__ == "__main__":
    main()
