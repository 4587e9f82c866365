"""The voltmeter of gtdgl's ladder and the onset integration on the device (gtdgl/src/protocol.jl).

The ladder (protocol.jl:325) measures, after every protocol cycle, quantities that `GPUStepper.measure()` now
computes on the resident state (meter.cu): this module holds the host side that the reference keeps on the host as
well — the voltmeter's planes and masks (protocol.jl:340-351), the unwrapping of the path phases against the
previous cycle (`_unwrap!`, :181-189), the line averages — and `crossing_times` (:271-296), the onset delay at
fixed current, stepping on the device and reading back only the path phases every `every` steps.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .grid import Grid, Masks
from .scheme import Stepper, selffield

TWO_PI = 2 * math.pi


@dataclass
class Voltmeter:
    """Planes vi < vo and the line masks over (y1..y2+1) × (z1..z2+1) (protocol.jl:340-351)."""
    vi: int
    vo: int
    Min: np.ndarray        # live x links on plane vi
    Mou: np.ndarray        # live x links on plane vo
    line_ok: np.ndarray    # every x link live between the planes
    line_f1: np.ndarray    # line_ok and f = 1 on every node of the line

    @property
    def nin(self) -> int:
        return int(self.Min.sum())

    @property
    def nou(self) -> int:
        return int(self.Mou.sum())

    @property
    def nlin(self) -> int:
        return int(self.line_ok.sum())


def voltmeter(gr: Grid, mk: Masks, delta_v: int = 8) -> Voltmeter:
    """protocol.jl:340-351: vi = x1 + δv, vo = x2 − δv; the masks from τx > 0.5 and f ≥ 1 − 1e-12."""
    vi, vo = gr.x1 + delta_v, gr.x2 - delta_v
    if not vi < vo:
        raise ValueError(f"delta_v = {delta_v} leaves no voltmeter")
    ys, zs = slice(gr.y1 - 1, gr.y2 + 1), slice(gr.z1 - 1, gr.z2 + 1)
    tx = mk.τx
    Min = np.asfortranarray(tx[vi - 1, ys, zs] > 0.5)
    Mou = np.asfortranarray(tx[vo - 1, ys, zs] > 0.5)
    line_ok = np.asfortranarray(np.all(tx[vi - 1:vo - 1, ys, zs] > 0.5, axis=0))
    f1 = np.all(mk.f[vi - 1:vo, ys, zs] >= 1 - 1e-12, axis=0)
    vm = Voltmeter(vi, vo, Min, Mou, line_ok, np.asfortranarray(line_ok & f1))
    if vm.nin == 0 or vm.nou == 0:
        raise ValueError(f"no live links on the voltmeter planes (delta_v = {delta_v})")
    if vm.nlin == 0:
        raise ValueError("no complete line between the voltmeter planes")
    return vm


def oround_f(x):
    """round(x, RoundNearestTiesAway), elementwise (geometry.jl:13)."""
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


def unwrap(T: np.ndarray, Dl: np.ndarray, Dprev: np.ndarray) -> np.ndarray:
    """_unwrap! (protocol.jl:181-189): T += the change of Dl since Dprev brought into (−π, π]; Dprev ← Dl."""
    d = Dl - Dprev
    d = d - TWO_PI * oround_f(d / TWO_PI)
    T += d
    Dprev[...] = Dl
    return T


def line_mean(a: np.ndarray, mask: np.ndarray) -> float:
    """sumlin over the masked lines in the reference's order (column-major) ÷ their count."""
    v = a.ravel(order="F")[mask.ravel(order="F")]
    s = 0.0
    for x in v:
        s += float(x)
    return s / len(v)


def path_phase_host(G: np.ndarray, Vx: np.ndarray, gr: Grid, vi: int, vo: int) -> np.ndarray:
    """_path_phase! (protocol.jl:168-179) on a host State: per line (j, k) over y1..y2+1 × z1..z2+1 the sum over
    vi ≤ i < vo of angle((conj(G[i]) Vx[i]) G[i+1]), i in order (the host side of the drop-in path; the device
    computes the same in tdgl_measure)."""
    ys, zs = slice(gr.y1 - 1, gr.y2 + 1), slice(gr.z1 - 1, gr.z2 + 1)
    acc = np.zeros((gr.y2 - gr.y1 + 2, gr.z2 - gr.z1 + 2), order="F")
    for i in range(vi, vo):
        w = (np.conj(G[i - 1, ys, zs]) * Vx[i - 1, ys, zs]) * G[i, ys, zs]
        acc += np.arctan2(w.imag, w.real)
    return acc


def voltage(obs: dict, vm: Voltmeter) -> float:
    """Vser (protocol.jl:412) from the device plane sums."""
    return obs["vsum_out"] / vm.nou - obs["vsum_in"] / vm.nin


def crossing_times(gs, st: Stepper, J: float, *, H: float, T: float, stop: int = 3, delta_v: int = 8,
                   every: int = 10, trace: list | None = None):
    """protocol.jl:271-296 on the device: integrates the state resident in `gs` at fixed current J and field H for up
    to T t_GL and returns (times, t, diverged): the times at which the line-averaged band-1 phase across the
    voltmeter passes a further multiple of 2π, sampled every `every` steps, stopping after `stop` crossings
    (0: never).  Only the path phases of band 1 cross to the host per sample.  `trace`, when given, receives the
    line-averaged phase of every sample."""
    vm = voltmeter(st.grid, st.masks, delta_v)
    gs.meter_set(vm, nphase=1)
    HJ = selffield(st, J)
    Dp = gs.measure()["D"][0].copy()
    acc = np.zeros_like(Dp)
    n = vm.nlin
    times, nxt, nst, q = [], 1, int(round(T / st.dt)), 0
    while q < nst:
        gs.steps(every, H, HJ)
        q += every
        D = gs.measure()["D"][0]
        unwrap(acc, D, Dp)
        ph = line_mean(acc, vm.line_ok) if n else 0.0
        if trace is not None:
            trace.append(ph)
        if not math.isfinite(ph):
            return times, q * st.dt, True
        if abs(ph) >= nxt * TWO_PI:
            times.append(q * st.dt)
            nxt += 1
        if stop > 0 and len(times) >= stop:
            break
    return times, q * st.dt, False
