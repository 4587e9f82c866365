"""Benchmark of the gtdgl ladder cycle on B200: ladder cell-updates/s and HBM GB/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload ramp256|parity12|sweep|serve|bilayer]

Workload ``ramp256`` (default): one ladder run of a three-band KWT sample, 256×128×32 cells at h = 0.5ξ with an
8-cell insulating padding (σvac = 0.01: the PCG field solve with the FP32 separable preconditioner, tolerance 1e-10),
a WEDGE notch 40 cells deep on the y1 face, the open-boundary FFT self-field (recomputed every 1 t_GL), κ = 25,
H = 0.03 and the transport current ramped as Jx = ±0.06·step/20000 (HJ updated every step), built by
juliatdgl_b200.workloads.  Synthetic state: the Meissner seed of the model.  ``parity12`` is the 12×8×4 two-band
parity case.

A bench step is one ladder cycle: the lMax = 40 calls of gtdgl's step! that one call of the accelerator hook makes
(gtdgl/src/protocol.jl:306-316, :409), so the timed steps hold the open-boundary recomputations in their proportion
(one every 51 steps).  ``value`` is device time (CUDA events on the library's stream) for K cycles with the state
resident in HBM; ``e2e`` is the same K cycles through the C-ABI with the state in pinned host buffers copied up and
down around each cycle, as the hook does.  ``roofline`` is the dominant kernel's algorithmic bytes per launch over its
event-timed duration, from a profiled pass.  ``cpu_baseline`` times the C++ restatement of gtdgl's CPU step (the
oracle) on the same full-size workload, all host threads and one thread.  ``sweep`` and ``serve`` summarise the
batched and served forms (configurations 3 and 4) measured in the same run.  With --gpus N each rank runs an
independent replica (replicas only: a grid does not shard), polarity alternating by rank; time is the max over
ranks.  ``--impl reference`` times the oracle alone on the same full-size workload, one step! per bench step.
"""
from __future__ import annotations

import argparse
import copy
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import juliatdgl_b200 as T  # noqa: E402
from juliatdgl_b200 import abi, workloads  # noqa: E402
from juliatdgl_b200.state import LINK_FIELDS, State  # noqa: E402

LMAX = 40


# ---------------------------------------------------------------------------------------------- workloads
def build_workload(name, bar_tables=None):
    if name == "parity12":
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import cases
        st, s, H, HJ = cases.config1()
        return st, s, H, (lambda q: HJ)
    st, s, H = workloads.ramp(bar_tables=bar_tables)
    return st, s, H, None


def oracle_bar_tables():
    """The bar-field tables of the full-size grid from the oracle's own restatement (field.jl:151-180), so that the
    CPU arms load no part of the CUDA library."""
    from juliatdgl_b200.scheme import BarField
    from oracle import pyoracle
    gr = T.Grid.make(256, 128, 32, dx=0.5, buf=8)
    return BarField(*pyoracle.bar_field(gr))


# ---------------------------------------------------------------------------------------------- CUDA helpers
class Cudart:
    def __init__(self):
        for name in ("libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so.12"):
            try:
                self.rt = C.CDLL(name)
                break
            except OSError:
                continue
        self.rt.cudaEventElapsedTime.argtypes = [C.POINTER(C.c_float), C.c_void_p, C.c_void_p]
        self.rt.cudaEventRecord.argtypes = [C.c_void_p, C.c_void_p]
        self.rt.cudaEventSynchronize.argtypes = [C.c_void_p]
        self.rt.cudaHostAlloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t, C.c_uint]

    def set_device(self, d):
        assert self.rt.cudaSetDevice(int(d)) == 0

    def sync(self):
        assert self.rt.cudaDeviceSynchronize() == 0

    def event(self):
        e = C.c_void_p()
        assert self.rt.cudaEventCreate(C.byref(e)) == 0
        return e

    def record(self, e, stream):
        assert self.rt.cudaEventRecord(e, C.c_void_p(stream)) == 0

    def elapsed_ms(self, a, b):
        self.rt.cudaEventSynchronize(b)
        ms = C.c_float()
        assert self.rt.cudaEventElapsedTime(C.byref(ms), a, b) == 0
        return float(ms.value)

    def pinned_like(self, a: np.ndarray) -> np.ndarray:
        p = C.c_void_p()
        assert self.rt.cudaHostAlloc(C.byref(p), a.nbytes, 0) == 0
        buf = (C.c_byte * a.nbytes).from_address(p.value)
        out = np.frombuffer(buf, dtype=a.dtype).reshape(a.shape, order="F")
        out[...] = a
        return out


def pinned_state(cu, s: State) -> State:
    return State([cu.pinned_like(g) for g in s.G], [cu.pinned_like(f) for f in s.F],
                 *(cu.pinned_like(getattr(s, k)) for k in LINK_FIELDS))


class Clocks:
    """nvidia-smi samples during the timed region (clocks, power, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None
        self.lines = []

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.p = None

    def _read(self):
        for line in self.p.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------------------------- arms
# DRAM bytes (read + write) per launch of the kernels of ramp256, one `ncu --set full --clock-control none` capture
# per kernel of `python bench.py --quick --no-graphs --steps 1 --warmup 1` (summaries under profiles/): the
# roofline's `traffic`, to set against the algorithmic bytes the live run measures.
NCU_TRAFFIC = {"precond_transform_f32": 22.24e6, "pcg_apply": 110.3e6, "band_stage": 176.0e6, "open_fft": 482.8e6}
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # SMs × FP32 lanes × 2 × max SM clock


def transform_flops(gr):
    """Algorithmic FP32 flops of one plane-transform launch (the mirror-halved y and z products of the x, y and z
    components' planes, which one launch takes together): per plane 2·[(h_S1² + h_D1²)·n2 + n1·(h_S2² + h_D2²)]."""
    ny, nz, nx = gr.Ny - 1, gr.Nz - 1, gr.Nx - 1
    tot = 0.0
    for n1, n2, planes in ((ny, nz, nx - 1), (ny - 1, nz, nx), (ny, nz - 1, nx)):
        h = lambda n: ((n + 1) // 2) ** 2 + (n // 2) ** 2
        tot += planes * 2.0 * (h(n1) * n2 + n1 * h(n2))
    return tot


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_pass(gs, steps, H, hj, q0):
    gpu_lib = gs_lib()
    gpu_lib.tdgl_profile(gs.h, 1)
    gs.steps_ramp(H, [hj(q0 + q) for q in range(steps)])
    n = gpu_lib.tdgl_profile_read(gs.h, -1, None, None, None, None)
    rows = []
    for cat in range(n):
        name = C.c_char_p()
        launches = C.c_int64()
        ms = C.c_double()
        by = C.c_double()
        gpu_lib.tdgl_profile_read(gs.h, cat, C.byref(name), C.byref(launches), C.byref(ms), C.byref(by))
        if launches.value:
            rows.append({"kernel": name.value.decode(), "launches": launches.value, "ms": ms.value, "bytes": by.value})
    gpu_lib.tdgl_profile(gs.h, 0)
    return rows


def gs_lib():
    from juliatdgl_b200 import gpu
    L = gpu.lib()
    L.tdgl_profile.argtypes = [C.c_void_p, C.c_int32]
    L.tdgl_profile_read.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_int64),
                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]
    return L


def oracle_threads(n):
    from oracle import pyoracle
    pyoracle.lib().oracle_set_threads(int(n))


def cpu_sample(workload, steps=2, single=1):
    """The oracle on the same workload: (value with all host threads, value on one thread, description, threads).
    One untimed step first (it holds the cold PCG start and the first open-boundary computation); then `steps` steps
    on every host thread and `single` step on one."""
    from oracle import pyoracle
    threads = os.cpu_count() or 1
    bar = oracle_bar_tables() if workload == "ramp256" else None
    st, s, H, hj = build_workload(workload, bar_tables=bar)
    if hj is None:
        hj = workloads.ramp_hj(st, +1)
    if workload == "parity12":
        steps, single = 200, 200
    o = pyoracle.OracleStepper(st)
    o.upload(s)
    oracle_threads(threads)
    o.steps_ramp(H, [hj(0)])
    t = time.perf_counter()
    o.steps_ramp(H, [hj(1 + q) for q in range(steps)])
    v_all = st.grid.sample_cells * steps / (time.perf_counter() - t)
    v_one = None
    if single:
        oracle_threads(1)
        t = time.perf_counter()
        o.steps_ramp(H, [hj(1 + steps + q) for q in range(single)])
        v_one = st.grid.sample_cells * single / (time.perf_counter() - t)
        oracle_threads(threads)
    desc = (f"the full {workload} workload: {steps} steps on {threads} threads and {single} on one, after one "
            "untimed step (C++ restatement of gtdgl's CPU step! with OpenMP over planes; the reference is Julia)")
    return v_all, v_one, desc, threads


def run_reference(args, rank, world):
    """The reference arm: the C++ restatement of gtdgl's CPU step (this project's oracle: the reference is Julia and
    cannot run here) on the same full-size workload, every host thread; one bench step is one step! (a bounded sample
    of the 40-step ladder cycle the B200 arm's step holds).  Bar tables from the oracle: no CUDA library is loaded."""
    if rank != 0:
        return
    from oracle import pyoracle
    threads = os.cpu_count() or 1
    bar = oracle_bar_tables() if args.workload == "ramp256" else None
    st, s, H, hj = build_workload(args.workload, bar_tables=bar)
    if hj is None:
        hj = workloads.ramp_hj(st, +1)
    o = pyoracle.OracleStepper(st)
    o.upload(s)
    oracle_threads(threads)
    o.steps_ramp(H, [hj(q) for q in range(args.warmup)])
    t = time.perf_counter()
    o.steps_ramp(H, [hj(args.warmup + q) for q in range(args.steps)])
    dt = time.perf_counter() - t
    v = st.grid.sample_cells * args.steps / dt
    sample = (f"the full {args.workload} workload, one step! per bench step ({args.steps} timed after {args.warmup}), "
              f"{threads} threads")
    line = {"impl": "reference", "metric": "ladder cell-updates/s", "value": v, "unit": "cell-updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "step_unit": "one step! of the workload", "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": _config(args),
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "pcg_iters_per_step": o.stats().pcg_total_iters / max(1, o.stats().steps)}
    print(json.dumps(line), flush=True)


WORKLOADS = {
    "ramp256": ("ramp256: 256x128x32 three-band KWT, WEDGE notch, insulating buffer 8 (PCG, FP32 preconditioner, "
                "tol 1e-10), open-boundary FFT self-field, Jx ramp", 256 * 128 * 32),
    "parity12": ("parity12: 12x8x4 two-band KWT, SepSolver, bar field", 12 * 8 * 4)}


def _config(args):
    desc, cells = WORKLOADS[args.workload]
    return {"workload": desc, "sample_cells": cells, "parallelism": f"replicas{args.gpus}",
            "l2": "state and workspaces exceed the 126 MB L2 (no flush needed)"}


def max_over_ranks(dist, x):
    """The largest of every rank's x (the job's time is its slowest replica's); x itself without a process group."""
    if not dist:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_b200(args, rank, world, local_rank, dist):
    from juliatdgl_b200 import gpu
    cu = Cudart()
    cu.set_device(local_rank)
    st, s, H, hj = build_workload(args.workload)
    if hj is None:
        hj = workloads.ramp_hj(st, +1 if rank % 2 == 0 else -1)
    cyc = LMAX                              # step! calls per bench step (one ladder cycle)
    peak, peak_kind = measured_peak()
    gs = gpu.GPUStepper(st)
    if args.no_graphs:
        gs.set_graphs(False)
    gs.upload(s)
    q = 0
    for _ in range(args.warmup):
        gs.steps_ramp(H, [hj(q + i) for i in range(cyc)])
        q += cyc
    stream = gs.stream
    e0, e1 = cu.event(), cu.event()
    clocks = Clocks(local_rank)
    # snapshot of the state and the carry at the start of the timed cycles: the end-to-end run below replays the
    # same cycles from it, so the two numbers time identical work (same PCG iterations, same open recomputes)
    host = pinned_state(cu, s)
    snap = None
    if not args.quick:
        gs.download(host)
        snap = copy.deepcopy(gs.get_carry())
    q0 = q
    st0 = gs.stats()
    n_steps = args.steps * cyc
    # ---- device-resident timed region: K cycles, the state resident in HBM
    cu.sync()
    if dist:
        dist.barrier()
    clocks.start()
    cu.record(e0, stream)
    gs.steps_ramp(H, [hj(q + i) for i in range(n_steps)])
    cu.record(e1, stream)
    cu.sync()
    ms = cu.elapsed_ms(e0, e1)
    clk = clocks.stop()
    q += n_steps
    stats = gs.stats()
    launches = stats.kernel_launches_last_call
    iters = (stats.pcg_total_iters - st0.pcg_total_iters) / n_steps
    recomputes = stats.open_recomputes - st0.open_recomputes
    ms = max_over_ranks(dist, ms)
    if args.quick:
        rows = profile_pass(gs, min(args.steps, 2) * cyc, H, hj, q) if (args.kernels and rank == 0) else []
        gs.close()
        if rank == 0:
            out = {"quick": True, "ms_per_step": ms / args.steps, "ms_per_tdgl_step": ms / n_steps,
                   "pcg_iters_per_tdgl_step": iters, "open_recomputes": recomputes, "gpu_launches": launches}
            if rows:
                out["kernels"] = [{"kernel": r["kernel"], "launches": r["launches"], "ms": round(r["ms"], 4),
                                   "us_per_launch": round(1e3 * r["ms"] / r["launches"], 2),
                                   "gbs": round(r["bytes"] / (r["ms"] * 1e6), 1)} for r in rows]
            print(json.dumps(out), flush=True)
        return
    # ---- end to end over the same cycles: each uploads the pinned host state, steps and downloads it, through the
    # C-ABI, as the ladder hook does once per cycle
    gs.set_carry(snap)
    cu.sync()
    if dist:
        dist.barrier()
    e2, e3 = cu.event(), cu.event()
    cu.record(e2, stream)
    qe = q0
    for _ in range(args.steps):
        gs.upload(host)
        gs.steps_ramp(H, [hj(qe + i) for i in range(cyc)])
        gs.download(host)
        qe += cyc
    cu.record(e3, stream)
    cu.sync()
    e2e_s = max_over_ranks(dist, cu.elapsed_ms(e2, e3)) / 1e3
    state_bytes = sum(a.nbytes for _, a in host.fields())
    # ---- profiled pass (per-kernel events) over two cycles
    n_prof = min(args.steps, 2) * cyc
    rows = profile_pass(gs, n_prof, H, hj, q) if rank == 0 else []
    gs.close()
    if rank != 0:
        return
    cells = st.grid.sample_cells
    value = world * cells * n_steps / (ms / 1e3)
    tot_ms = sum(r["ms"] for r in rows) or 1.0
    # the dominant kernel: the preconditioner transform's two directions are one kernel (k_half32, forward and
    # inverse instances) and count together
    merged = {}
    for r in rows:
        k = "precond_transform_f32" if r["kernel"] in ("precond_transform_f32", "precond_inverse_f32") else r["kernel"]
        m = merged.setdefault(k, {"kernel": k, "launches": 0, "ms": 0.0, "bytes": 0.0})
        m["launches"] += r["launches"]
        m["ms"] += r["ms"]
        m["bytes"] += r["bytes"]
    dom = max(merged.values(), key=lambda r: r["ms"]) if rows else None
    step_bytes = sum(r["bytes"] for r in rows) / n_prof if rows else None
    roof = None
    if dom:
        per_launch_bytes = dom["bytes"] / dom["launches"]
        per_launch_s = dom["ms"] / dom["launches"] / 1e3
        ach = per_launch_bytes / per_launch_s / 1e9
        roof = {"kernel": dom["kernel"], "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_kind": peak_kind, "traffic": NCU_TRAFFIC.get(dom["kernel"]),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch (profiles/)",
                "algorithmic_bytes_per_launch": per_launch_bytes, "share_of_step": dom["ms"] / tot_ms}
        if dom["kernel"] == "precond_transform_f32":
            roof["kernel"] = "precond_transform_f32 (k_half32, forward and inverse)"
        if dom["kernel"] == "precond_transform_f32" and args.workload == "ramp256":
            fl = transform_flops(st.grid)
            roof.update(flops_per_launch=fl, achieved_tflops=fl / per_launch_s / 1e12)
    cpu_v = cpu_one = None
    cpu_desc, cpu_threads = "skipped", 0
    if not args.no_cpu:
        cpu_v, cpu_one, cpu_desc, cpu_threads = cpu_sample(args.workload)
    line = {"metric": "ladder cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "step_unit": f"one ladder cycle: {cyc} step! calls (the accelerator hook's lMax)",
            "ms_per_tdgl_step": ms / n_steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config(args),
            "hbm_gbs_step": (step_bytes / (ms / n_steps / 1e3) / 1e9) if step_bytes else None,
            "roofline": roof,
            "cpu_baseline": {"value": cpu_v, "unit": "cell-updates/s", "cores": cpu_threads, "kind": "port",
                             "sample": cpu_desc, "single_thread_value": cpu_one},
            "e2e": {"value": world * cells * n_steps / e2e_s, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                    "path": "GPUStepper.upload / steps_ramp / download per cycle (tdgl_upload_state, "
                            "tdgl_steps_ramp, tdgl_download_state), pinned host State"},
            "gpu_launches": launches, "clocks": clk,
            "pcg_iters_per_tdgl_step": iters, "open_recomputes_timed": recomputes,
            "kernels": [{"kernel": r["kernel"], "launches": r["launches"], "ms": round(r["ms"], 4),
                         "share": round(r["ms"] / tot_ms, 4), "gbs": round(r["bytes"] / (r["ms"] / 1e3) / 1e9, 1)}
                        for r in sorted(rows, key=lambda r: -r["ms"])]}
    if args.workload == "ramp256" and not args.no_extras:
        line["sweep"] = sweep_measure(100, 3)
        line["serve"] = serve_measure(32)
    print(json.dumps(line), flush=True)


def sweep_measure(K, W, quick=False):
    """The batched sweep: 64 two-band runs of mixed sizes (juliatdgl_b200/sweep.py) stepped as one batch, against the
    plain drop-in path (one run at a time, state up and down every lMax-step cycle).  Both are timed over the same
    K steps per run after W warm-up steps and reported as runs per hour of 10000-step runs."""
    from juliatdgl_b200 import sweep
    runs = sweep.sweep_instances(64, seed=2)
    info = {}
    t_b, ctxs = sweep.run_batched(runs, K, warm=W, info=info)
    launches = sum(g.stats().kernel_launches_last_call for g in ctxs)
    for g in ctxs:
        g.close()
    t_p = sweep.run_plain(runs, K, warm=W) if not quick else None   # quick: the batched arm alone
    per_run = 10000 / K
    cells = sum(r.cells for r in runs)
    rph_b = 3600.0 / (t_b * per_run) * len(runs)
    rph_p = 3600.0 / (t_p * per_run) * len(runs) if t_p else None
    return {"runs_per_h": rph_b, "plain_runs_per_h": rph_p, "batched_over_plain": rph_b / rph_p if rph_p else None,
            "steps_timed_per_run": K, "warmup": W, "cells": cells,
            "cell_updates_per_s": cells * K / t_b, "plain_cell_updates_per_s": cells * K / t_p if t_p else None,
            "gpu_launches": launches,
            "merge": {"contexts": info.get("contexts"), "chains": info.get("chains"),
                      "launches_per_step": info.get("launches"),
                      "autotune_s_by_blocks_per_sm": {str(k): round(v, 5) for k, v in info.get("tune_s", {}).items()}},
            "workload": "sweep64: 64 two-band runs (mgb2 model II, kappa 25), grids {64,96,128,192}x{32,48,64}"
                        "x{8,12,16} seed 2, WEDGE depth 10-40%, Jx in [0.01,0.05] both polarities, Hz 0.2; runs/h of "
                        "10000-step runs from the timed steps"}


def run_sweep(args, rank, world):
    K, W = args.steps, max(3, args.warmup)
    m = sweep_measure(K, W, quick=args.quick)
    line = {"metric": "batched runs/h", "value": m["runs_per_h"], "unit": "runs/h (10000-step runs)", "n_gpus": 1,
            "steps": K, "warmup": W, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": m["workload"], "cells": m["cells"],
                       "parallelism": "one batch graph per step, runs with the same kernels merged into one launch per kernel"},
            "gpu_launches": m["gpu_launches"], **{k: v for k, v in m.items() if k not in ("workload", "gpu_launches")}}
    print(json.dumps(line), flush=True)


def bilayer_workload(nx=512, ny=256, nz=64, buf=16, seed=4):
    """The large noisy bilayer: a lower three-band layer and an upper two-band layer (band 3 absent, a <= T) joined by
    a 2-node barrier material of transparency 0.3 to both; per material the masses (through ξ), Γ and σn drawn from
    U[0.8, 1.2] of their unit values (seed 4); masses per axis (1, 1, 4); bath T = 0.5 (ε = a − T); Langevin noise
    T̃ = 0.005 on every band and the field (device Philox, seed 4); 16-cell insulating buffer (σvac = 0.01: PCG, FP32
    preconditioner, tol 1e-10); open-boundary FFT self-field; H = 0.03, Jx = 0.02."""
    from juliatdgl_b200.grid import with_materials
    rng = np.random.default_rng(seed)
    u = lambda: float(rng.uniform(0.8, 1.2))
    Tb = 0.5

    def bands(sm, sg, three):
        ax = lambda m: (m, m, 4 * m)
        return (T.Band.make(m_axes=ax(1.0 * sm), Γ=1.0 * sg, a=1.0),
                T.Band.make(m_axes=ax(sm / (16 * 0.59)), Γ=1.0 * sg, a=0.59),
                T.Band.make(m_axes=ax(2.0 * sm), Γ=1.2 * sg, a=0.8 if three else 0.4))

    lower = T.Model.make(bands(u(), u(), True), [[0.0, 1e-3, -0.02], [1e-3, 0.0, -0.02], [-0.02, -0.02, 0.0]],
                         κ=25.0, σn=u(), T=Tb)
    upper = T.Model.make(bands(u(), u(), False), [[0.0, 1e-3, 0.0], [1e-3, 0.0, 0.0], [0.0, 0.0, 0.0]],
                         κ=25.0, σn=u(), T=Tb)
    barrier = T.Model.make(lower.bands, lower.γ, κ=25.0, σn=u(), T=Tb)
    gr = T.Grid.make(nx, ny, nz, dx=0.5, buf=buf)
    kmid = gr.z1 + nz // 2 - 1
    k = np.arange(1, gr.Nz + 2)
    layer = np.where(k <= kmid, 1, np.where(k <= kmid + 2, 3, 2)).astype(np.uint8)
    mat = np.broadcast_to(layer[None, None, :], gr.node)
    mk = with_materials(T.box_masks(gr), gr, np.asfortranarray(mat))
    st = T.Stepper.make(lower, gr, mk, materials=[upper, barrier],
                        transparency=[[1.0, 1.0, 0.3], [1.0, 1.0, 0.3], [0.3, 0.3, 1.0]], absent=[[], [3], []],
                        σvac=0.01, selffield_bc="open", pcg_tol=1e-10, noise=0.005, noise_seed=seed, noise_field=True)
    H = 0.03
    s = T.initial_state(lower, gr, mk, H, materials=st.mt.models)
    return st, s, H, T.selffield(st, 0.02)


def run_bilayer(args, rank, world):
    """The large noisy bilayer (512x256x64, buffer 16): device-timed steps with the state resident, the PCG
    iterations, the device memory, and a profiled pass's per-kernel table."""
    from juliatdgl_b200 import gpu
    t0 = time.perf_counter()
    st, s, H, HJ = bilayer_workload()
    t_setup = time.perf_counter() - t0
    gs = gpu.GPUStepper(st)
    gs.upload(s)
    rt = Cudart()
    W, K = max(3, args.warmup), args.steps
    gs.steps(W, H, HJ)
    it0 = gs.stats().pcg_total_iters
    a, b = rt.event(), rt.event()
    rt.record(a, gs.stream)
    gs.steps(K, H, HJ)
    rt.record(b, gs.stream)
    ms = rt.elapsed_ms(a, b)
    its = (gs.stats().pcg_total_iters - it0) / K
    gs.profile(True)
    gs.steps(2, H, HJ)
    rows = gs.profile_read()
    gs.profile(False)
    tot = sum(r["ms"] for r in rows)
    table = [{"kernel": r["kernel"], "share": round(r["ms"] / tot, 4), "gbs": round(r["bytes"] / r["ms"] / 1e6, 1)}
             for r in sorted(rows, key=lambda r: -r["ms"])[:10]]
    cells = st.grid.sample_cells
    line = {"metric": "ladder cell-updates/s", "value": cells * K / (ms / 1e3), "unit": "cell-updates/s", "n_gpus": 1,
            "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "bilayer512: 512x256x64, buffer 16, two materials + 2-node barrier (t 0.3), masses "
                                   "(1,1,4), bath T 0.5, noise 0.005 on bands and field (Philox seed 4), PCG FP32 "
                                   "preconditioner tol 1e-10, open boundary, H 0.03, Jx 0.02",
                       "cells": cells, "nodes": (st.grid.Nx + 1) * (st.grid.Ny + 1) * (st.grid.Nz + 1)},
            "pcg_iters_per_step": its, "device_gb": gs.device_bytes / 1e9, "host_setup_s": t_setup,
            "seconds_for_5000_steps": 5000 * ms / K / 1e3, "kernels": table}
    gs.close()
    print(json.dumps(line), flush=True)


def serve_key(r):
    nan = lambda x: "none" if math.isnan(x) else x
    return (r.id, nan(r.onset_J), nan(r.delay), r.rungs, r.steps)


def serve_measure(n):
    """The served stream: Poisson arrivals at 4 runs/s (seed 3) of two- and three-band onset searches on grids from
    32x16x4 to 256x128x32 (juliatdgl_b200/serve.py), served with continuous batching against a 150 GB budget; the
    plain drop-in path serves the same runs one at a time (first come, first served, the state on the host between
    cycles).  p50/p99 time-to-onset (arrival to result) and runs/h of both, and the capacity (every run submitted at
    once)."""
    from juliatdgl_b200 import serve
    reqs = serve.served_requests(n, seed=3, rate=4.0)
    srv = serve.Server(serve.OnsetSpec(), budget_bytes=150e9)
    res = srv.run(reqs, realtime=True)
    tto = sorted(r.time_to_onset for r in res)
    services = []
    plain = []
    for r in reqs:
        p, secs = serve.plain_service(r, srv.spec)
        services.append(secs)
        plain.append(p)
    sat = serve.Server(serve.OnsetSpec(), budget_bytes=150e9)
    res_sat = sat.run(reqs, realtime=False)
    same_sat = sum(1 for a, b in zip(res, res_sat) if serve_key(a) == serve_key(b))
    fin = serve.fifo([r.arrival for r in reqs], services)
    tto_p = sorted(f - r.arrival for f, r in zip(fin, reqs))
    same = sum(1 for a, b in zip(res, plain) if (a.onset_J == b.onset_J) or (math.isnan(a.onset_J) and math.isnan(b.onset_J)))
    pct = lambda v, q: float(np.percentile(v, q))
    return {"p50_s": pct(tto, 50), "p99_s": pct(tto, 99), "runs_per_h": 3600.0 * n / srv.makespan,
            "plain_p50_s": pct(tto_p, 50), "plain_p99_s": pct(tto_p, 99), "plain_runs_per_h": 3600.0 * n / sum(services),
            "served_over_plain_runs_per_h": (n / srv.makespan) / (n / sum(services)),
            "capacity_runs_per_h": 3600.0 * n / sat.makespan, "capacity_over_plain": sum(services) / sat.makespan,
            "results_same_streamed_and_all_at_once": same_sat, "peak_active_runs": srv.peak_active,
            "onsets_found": sum(1 for r in res if not math.isnan(r.onset_J)), "onsets_same_as_plain": same, "runs": n,
            "workload": f"serve{n}: Poisson 4 runs/s seed 3, 2/3-band onset searches on 32x16x4..256x128x32 "
                        "(log-uniform), WEDGE, H 0.03, J ladder 0.1..1.0 step 0.1, 5 tGL rungs, 10 tGL delay "
                        "confirmation, 150 GB budget; plain = one run at a time, first come first served"}


def run_serve(args, rank, world):
    n = args.steps if args.steps != 40 else 32
    m = serve_measure(n)
    line = {"metric": "served p50/p99 time-to-onset", "value": m["p50_s"], "unit": "s", "n_gpus": 1, "steps": n,
            "warmup": 0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": m["workload"], "parallelism": "continuous batching, one stream per run, cycles pipelined"},
            **{k: v for k, v in m.items() if k != "workload"}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--workload", default="ramp256", choices=("ramp256", "parity12", "sweep", "serve", "bilayer"))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-extras", action="store_true", help="ramp256: skip the sweep and serve summaries")
    ap.add_argument("--quick", action="store_true", help="device-timed steps only (no e2e, profile pass or CPU sample)")
    ap.add_argument("--kernels", action="store_true", help="with --quick: add the per-kernel table of a profiled pass")
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch every kernel from the host (the same kernels; for profilers that cannot see graph nodes)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    if args.workload in ("sweep", "serve", "bilayer") and args.impl == "b200":
        if rank == 0:
            {"sweep": run_sweep, "serve": run_serve, "bilayer": run_bilayer}[args.workload](args, rank, world)
    elif args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_b200(args, rank, world, local_rank, dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
