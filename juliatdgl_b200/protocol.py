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


# ---------------------------------------------------------------------------------------------- close rules
def slope(t, y) -> float:
    """The least-squares slope of y against t (pendiente, observables.jl:23-26)."""
    A = np.column_stack([np.asarray(t, dtype=np.float64), np.ones(len(t))])
    return float(np.linalg.lstsq(A, np.asarray(y, dtype=np.float64), rcond=None)[0][0])


def crossings_now(T1, Tm1, line_ok, m: int, dt_cyc: float) -> float:
    """_crossings_now (protocol.jl:193-199): the 2π crossings the second half's phase slope projects over the whole
    point (m cycles of dt_cyc); 0 while the lines' accumulated phase (Tm1) stays below one crossing, or the second
    half holds fewer than 3 cycles.  T1: the line-mean phase per cycle (T1[q − 1] is cycle q)."""
    acc = 0.0
    for v, ok in zip(np.ravel(Tm1, order="F"), np.ravel(line_ok, order="F")):
        if ok:
            acc += abs(float(v))
    if acc / TWO_PI < 1:
        return 0.0
    lo = m - m // 2 + 1
    if m - lo + 1 < 3:
        return 0.0
    th = (np.arange(lo, m + 1) - lo) * dt_cyc
    return abs(slope(th, np.asarray(T1[lo - 1:m]))) * m * dt_cyc / TWO_PI


def late_crossings(T1, m: int) -> float:
    """_late_crossings (protocol.jl:204-207): the crossings since the first quarter of the point, over the whole
    point (the first quarter is left out: the static phase change of a current step is not a slip)."""
    q = max(1, m // 4)
    return abs(float(T1[m - 1]) - float(T1[q - 1])) * m / (m - q) / TWO_PI if m > q else 0.0


def silent_now(T1, Tm1, line_ok, m: int, dt_cyc: float, lim: float) -> bool:
    """_silent_now (protocol.jl:208-209): neither the slope nor the late crossings reach lim."""
    return max(crossings_now(T1, Tm1, line_ok, m, dt_cyc), late_crossings(T1, m)) < lim


@dataclass
class CloseRules:
    """The parameters of a point's close rules (the Protocol defaults, protocol.jl:38-48)."""
    f_strict: bool = True     # 'F' only below f_margin crossings, 'V' only at ≥ 10 by the slope
    f_margin: float = 0.5
    use_Vconv: bool = True    # the resistive route
    v_margin: float = 1.1
    any_band: bool = False    # slip_band_mode :any_band (else band 1)


def close_point(m: int, Tser, Tmat, line_ok, dif, diffh: float, J: float, *, dt_cyc: float, iter_min: int,
                it_res_min: int, nwin: int, eps: float, noisy: bool, rules: CloseRules = CloseRules()):
    """Whether a ladder point closes at cycle m (protocol.jl:466-490), from the device's cycle observables: 'F' (a
    fixed point, or with noise a silent rung), 'V' (a resistive plateau), or None to go on; with the band that met
    the resistive criterion ('V', else None).  Tser[µ]: the line-mean unwrapped phase of band µ per cycle (Tser[µ][q −
    1] is cycle q); Tmat[µ]: its per-line accumulation at cycle m; dif[µ]: max ||Ψ_µ| − |Ψ_µ|prev|| of the cycle;
    diffh: max |h_z − h_z prev|."""
    N = len(Tser)
    bands = range(N) if rules.any_band else range(1)
    silent = lambda: all(silent_now(Tser[µ], Tmat[µ], line_ok, m, dt_cyc, rules.f_margin) for µ in bands)
    half = max(1, m // 2)
    if noisy:
        # with noise the state never reaches a fixed point: a rung is silent when it held it_res_min cycles without a
        # phase slip on any band
        if m >= it_res_min and max(abs(float(Tser[µ][m - 1])) for µ in range(N)) < TWO_PI and \
                (not rules.f_strict or silent()):
            return "F", None
    elif m >= iter_min and max(dif) < eps and diffh < eps:
        if m < 2 or max(abs(float(Tser[µ][m - 1]) - float(Tser[µ][half - 1])) for µ in range(N)) < TWO_PI:
            if not rules.f_strict or silent():
                return "F", None
    if rules.use_Vconv and abs(J) > 0 and m >= max(it_res_min, 2 * nwin):
        for µ in bands:
            plateau = abs(float(Tser[µ][m - 1]) - float(Tser[µ][half - 1])) * 2 >= rules.v_margin * 10 * TWO_PI
            if plateau and (not rules.f_strict or crossings_now(Tser[µ], Tmat[µ], line_ok, m, dt_cyc) >= 10):
                return "V", µ
    return None, None


def normal_verdict(conv: str, J: float, psi2: float, lastF: float, n_frac: float = 0.02):
    """The 'N' verdict (protocol.jl:529-536): a point that closed 'F' with ⟨|Ψ₁|²⟩ over the block (psi2) below
    n_frac of the largest of the 'F' points so far (lastF) has gone normal.  Returns (verdict, lastF after it)."""
    if conv == "F" and n_frac > 0:
        if abs(J) > 0 and lastF > 0 and psi2 < n_frac * lastF:
            return "N", lastF
        return "F", max(lastF, psi2)
    return conv, lastF
