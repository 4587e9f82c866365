"""Batched sweeps: many independent uneven grids stepped together on one GPU (the batched form of the ladder's
fixed-current runs).

`sweep_instances` draws the mixed-size onset sweep: two-band runs (the model of the diode studies,
gtdgl/materials/mgb2_model_II.toml: two_band(ξ_π/ξ_σ = 4, κ = 25)), grids from {64, 96, 128, 192} × {32, 48, 64} ×
{8, 12, 16} cells, a WEDGE notch of depth 10–40 % of the width, fixed Jx on a uniform grid of [0.01, 0.05] in both
polarities, Hz = 0.2.  `run_batched` steps them as one batch (tdgl_batch_*: one graph launch per step for all runs);
`run_plain` is the drop-in path the reference's accelerator takes, one run at a time, copying every field of the
state up before and down after each protocol cycle of lMax steps (TDGLGPU.jl:2114-2144).
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import gpu
from .grid import GeomSpec, Grid, build_masks
from .model import two_band
from .scheme import Stepper, selffield
from .state import State, initial_state

SIZES = ((64, 96, 128, 192), (32, 48, 64), (8, 12, 16))


@dataclass
class Run:
    st: Stepper
    s: State
    H: float
    HJ: float
    J: float

    @property
    def cells(self) -> int:
        g = self.st.grid
        return (g.x2 - g.x1) * (g.y2 - g.y1) * (g.z2 - g.z1)


def sweep_instances(n: int = 64, seed: int = 2, H: float = 0.2, kappa: float = 25.0) -> list[Run]:
    """The n runs of the sweep (n/2 currents × 2 polarities), drawn with numpy's generator of `seed`."""
    rng = np.random.default_rng(seed)
    md = two_band(xi_ratio=4.0, κ=kappa)
    half = max(1, n // 2)
    Js = np.linspace(0.01, 0.05, half)
    runs = []
    for i in range(n):
        nx, ny, nz = (int(rng.choice(a)) for a in SIZES)
        depth = float(rng.uniform(0.10, 0.40))
        gr = Grid.make(nx, ny, nz, dx=0.5, buf=1)
        mk = build_masks(GeomSpec(GEOM_MODE="WEDGE", wedge_depth=depth), gr)
        st = Stepper.make(md, gr, mk)
        J = float(Js[i % half]) * (1.0 if i < half else -1.0)
        runs.append(Run(st, initial_state(md, gr, mk, H), H, selffield(st, J), J))
    return runs


def run_batched(runs: list[Run], steps: int, *, cycle: int = 40, warm: int = 8, tune: bool = True, info=None):
    """Steps every run `steps` times as one batch (after `warm` untimed steps, and the autotuning of the merged
    launch shape with tune: a few more untimed steps per candidate); returns (seconds, contexts).  The caller closes
    the contexts.  `info` (a dict) receives the tuning times and the merge of the timed steps."""
    ctxs = []
    for r in runs:
        gs = gpu.GPUStepper(r.st)
        gs.upload(r.s.copy())
        ctxs.append(gs)
    bt = gpu.Batch(ctxs)
    H = [r.H for r in runs]
    HJ = [r.HJ for r in runs]
    bt.steps(warm, H, HJ)
    if tune:
        t = bt.tune(H, HJ)
        if info is not None:
            info["tune_s"] = t
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        k = min(cycle, steps - done)
        bt.steps(k, H, HJ, wait=False)
        done += k
    for g in ctxs:
        g.sync()
    dt = time.perf_counter() - t0
    if info is not None:
        info.update(bt.merge_info)
    bt.close()
    return dt, ctxs


def run_plain(runs: list[Run], steps: int, *, cycle: int = 40, warm: int = 8):
    """The drop-in path, one run after the other: per protocol cycle, upload the state, lMax steps, download it
    (the hook contract: every State field on the host after each cycle).  Returns seconds for all runs."""
    total = 0.0
    for r in runs:
        gs = gpu.GPUStepper(r.st)
        s = r.s.copy()
        gs.upload(s)
        gs.steps(warm, r.H, r.HJ)
        gs.download(s)
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            k = min(cycle, steps - done)
            gs.upload(s)
            gs.steps(k, r.H, r.HJ)
            gs.download(s)
            done += k
        total += time.perf_counter() - t0
        gs.close()
    return total
