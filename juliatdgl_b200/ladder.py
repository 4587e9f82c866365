"""The current ladder of gtdgl (gtdgl/src/protocol.jl:325-601, run_ladders :842-861, brackets :809-817) on the device.

Each point of the ladder starts from the state the previous one left and is integrated in cycles of lMax steps (one
call of the accelerator hook per cycle) until it closes: 'F' a fixed point, 'V' a resistive plateau, '*' the
ceiling mMax, and 'N' a fixed point gone normal.  After every cycle the voltmeter's observables are read from the
device (GPUStepper.measure: the per-line path phases of every band, the plane sums of φx, θ_A, the residuals of
|Ψ_µ| and h_z against the previous cycle, the mid-plane current; meter.cu), so only the path phases and a few
scalars cross to the host per cycle; the state itself is read back once per point, for the point's summary
(magnetisation, ⟨|Ψ|²⟩) and the final state.  The close rules are protocol.py's (protocol.jl:466-490).

A backend is any object with reset(s) (take the state and start cold: the PCG warm start off, the open boundary
without ramp, as run_ladders starts each polarity), meter_set(vm), cycle(n, H, HJ), measure(), download(s) and
vortices(band, kc): `DeviceLadder` steps on the B200; the tests drive the same protocol over the oracle.
Not restated: the output files, STOP.txt, resume, the heat cut and the delay confirmation (t_confirm_GL, which the
served onset search of serve.py runs on device snapshots).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .grid import Grid, dl, slab_thickness
from .protocol import (CloseRules, TWO_PI, close_point, line_mean, normal_verdict, oround_f, slope, unwrap,
                       voltmeter)
from .scheme import Stepper, selffield
from .state import State, initial_state


@dataclass
class Protocol:
    """gtdgl's Protocol (protocol.jl:26-70), the fields the ladder reads."""
    lMax: int = 40
    iter_min: int = 40
    mMax: int = 500_000
    t_min_GL: float = 400.0
    t_min_GL_res: float = 1584.0
    eps_conv: float = 1e-4
    eps_rate: float = 0.0
    eps_seed: float = 5e-4
    delta_v: int = 8
    V_win: int = 40
    V_win_min_res: int = 400
    use_Vconv: bool = True
    slip_band_mode: str = "band1"
    v_margin: float = 1.1
    f_strict: bool = True
    f_margin: float = 0.5
    guard_psi: float = 5.0
    stop_after_V: int = 0
    n_frac: float = 0.02


def dt_release10(st: Stepper) -> float:
    """protocol.jl:78-86: the step release 1.0 would take (to turn a tolerance per 1.0 cycle into physical time)."""
    md, gr = st.model, st.grid
    l = dl(gr)
    dt1 = 5.79 * l / (4 * math.sqrt(1 + 10.0 ** 2))
    bands = [dt1 if µ == 0 else dt1 * md.bands[µ].m * md.bands[µ].Γ for µ in range(md.N)]
    dt2 = 1.00 * l / (4 * md.κ ** 2)
    dt3 = 0.03 * l / (4 * 0.50 ** 2)
    return 0.99 * min(*bands, dt2, dt2, dt3)


def eps_cycle(pr: Protocol, st: Stepper) -> float:
    """protocol.jl:88-89."""
    return pr.eps_rate * (pr.lMax * st.dt) if pr.eps_rate > 0 else pr.eps_conv * (st.dt / dt_release10(st))


def sumlin(values) -> float:
    s = 0.0
    for x in values:
        s += float(x)
    return s


def meanlin(values) -> float:
    v = list(values)
    return sumlin(v) / len(v)


def oround(x: float) -> int:
    a = math.floor(abs(x) + 0.5)
    return int(a if x >= 0 else -a)


def magnetization(hz: np.ndarray, H: float, gr: Grid) -> float:
    """observables.jl:34-37: the mean of h_z over x1:x2−1, y1:y2−1, z1:z2 (column-major order) minus H."""
    v = hz[gr.x1 - 1:gr.x2 - 1, gr.y1 - 1:gr.y2 - 1, gr.z1 - 1:gr.z2]
    return meanlin(v.ravel(order="F")) - H


@dataclass
class Ladder:
    """What a ladder of one polarity returns (protocol.jl:92-125), the fields restated here."""
    label: str
    J: np.ndarray
    H: np.ndarray
    V: np.ndarray
    Vb: np.ndarray
    Vh: np.ndarray
    Vstatic: np.ndarray
    m: np.ndarray
    conv: str
    res: np.ndarray
    nslip: np.ndarray
    M: np.ndarray
    Nv: np.ndarray
    psi2: np.ndarray
    Itot: np.ndarray
    Isam: np.ndarray
    dmax: np.ndarray
    nbig: np.ndarray
    Vf1: np.ndarray
    VA: np.ndarray
    t_cycle: float
    state: State
    slip_band_mode: str = "band1"
    slip_band: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=int))


def ladder(run, st: Stepper, s: State, Js, *, H, label: str = "J+", pr: Protocol = Protocol()) -> Ladder:
    """protocol.jl:325-601 without output files, resume, heat or the delay confirmation; `run` is the backend, `s`
    the starting state (advanced in place: it holds the final state on return)."""
    gr, mk, N = st.grid, st.masks, st.N
    any_band = pr.slip_band_mode == "any_band"
    bands = list(range(N)) if any_band else [0]
    Js = np.asarray(Js, dtype=np.float64)
    npt = len(Js)
    Hs = np.full(npt, float(H)) if np.ndim(H) == 0 else np.asarray(H, dtype=np.float64)
    lMax, mMax, dt = pr.lMax, pr.mMax, st.dt
    dt_cyc = lMax * dt
    iter_min = pr.iter_min
    if pr.t_min_GL > 0:
        iter_min = max(iter_min, math.ceil(pr.t_min_GL / dt_cyc))
    eps_c = eps_cycle(pr, st)
    vm = voltmeter(gr, mk, pr.delta_v)
    nin, nou, nlin = vm.nin, vm.nou, vm.nlin
    nlin_f1 = int(vm.line_f1.sum())
    nwin = max(2, pr.V_win)
    rules = CloseRules(f_strict=pr.f_strict, f_margin=pr.f_margin, use_Vconv=pr.use_Vconv, v_margin=pr.v_margin,
                       any_band=any_band)
    out = dict(V=np.zeros(npt), Vb=np.full((npt, N), np.nan), Vh=np.full((npt, N), np.nan), Vst=np.zeros(npt),
               m=np.zeros(npt, dtype=int), conv=[" "] * npt, res=np.zeros((npt, N)), nslip=np.zeros(npt),
               M=np.zeros(npt), Nv=np.zeros((npt, N), dtype=int), psi2=np.zeros((npt, N)), Itot=np.full(npt, np.nan),
               Isam=np.full(npt, np.nan), dmax=np.zeros(npt), nbig=np.zeros(npt, dtype=int), Vf1=np.full(npt, np.nan),
               VA=np.full(npt, np.nan), slip_band=np.zeros(npt, dtype=int))
    lastF = 0.0
    kc = oround((gr.z1 + gr.z2) / 2)
    nV = 0
    run.reset(s)                 # _pcg_reset! (protocol.jl:376); the open boundary starts afresh (:852)
    run.meter_set(vm)            # Cooper0 and fieldOld from the starting state (:370-371)
    line_ok = vm.line_ok
    for jp in range(npt):
        if pr.stop_after_V > 0 and nV >= pr.stop_after_V:
            break
        J, Hc = float(Js[jp]), float(Hs[jp])
        HJ = selffield(st, J)
        Vser, TAser, Tf1 = [], [], []
        Tser = [[] for _ in range(N)]
        ItSer, IsSer = [], []
        Tmat = [np.zeros(line_ok.shape, order="F") for _ in range(N)]
        Dprev = [None] * N
        m, conv, dmax_cur, nbig_cur = 1, "*", 0.0, 0
        it_res_min = max(iter_min, math.ceil(pr.t_min_GL_res / dt_cyc))
        while m <= mMax:
            run.cycle(lMax, Hc, HJ)
            o = run.measure()
            Vser.append(o["vsum_out"] / nou - o["vsum_in"] / nin)
            TAser.append(o["ta_sum"] / nlin if nlin > 0 else 0.0)
            Dl = o["D"]
            if m == 1:
                for µ in range(N):
                    Dprev[µ] = Dl[µ].copy()
                    Tmat[µ][...] = 0.0
                    Tser[µ].append(0.0)
                Tf1.append(0.0)
                dmax_cur, nbig_cur = 0.0, 0
            else:
                d = (Dl[0] - Dprev[0])[line_ok]
                d = d - TWO_PI * oround_f(d / TWO_PI)
                if d.size:
                    dmax_cur = max(dmax_cur, float(np.max(np.abs(d))))
                    nbig_cur += int(np.sum(np.abs(d) > 2.0))
                for µ in range(N):
                    unwrap(Tmat[µ], Dl[µ], Dprev[µ])
                Tf1.append(line_mean(Tmat[0], vm.line_f1) if nlin_f1 > 0 else 0.0)
                for µ in range(N):
                    Tser[µ].append(line_mean(Tmat[µ], line_ok))
            ItSer.append(o["Itot"])
            IsSer.append(o["Isam"])
            eps_here = pr.eps_seed if jp == 0 else eps_c
            dif = list(o["res"])
            amax = o["amax"]
            if pr.guard_psi > 0 and (not math.isfinite(amax) or amax > pr.guard_psi):
                raise RuntimeError(f"ladder {label}: the scheme diverged at point {jp + 1} (J = {J}), cycle {m}: "
                                   f"max|Ψ| = {amax}; dt = {st.dt} ({st.limit})")
            out["res"][jp, :] = dif
            verdict, band = close_point(m, Tser, Tmat, line_ok, dif, o["diffh"], J, dt_cyc=dt_cyc, iter_min=iter_min,
                                        it_res_min=it_res_min, nwin=nwin, eps=eps_here,
                                        noisy=st.noise_T is not None, rules=rules)
            if verdict is not None:
                conv = verdict
                if verdict == "V" and any_band:
                    out["slip_band"][jp] = band + 1
                break
            m += 1
        mlast = min(m, mMax)
        nav = min(nwin, mlast)
        out["Vst"][jp] = meanlin(Vser[mlast - nav:mlast])
        if conv == "V":
            nav = min(max(pr.V_win_min_res, mlast // 2), mlast)
        w0 = mlast - nav + 1                  # the window wq = w0:mlast (1-based cycles)
        nslip, Vc = 0.0, 0.0
        if nav >= 3:
            tq = np.arange(nav) * dt_cyc
            for µ in range(N):
                out["Vb"][jp, µ] = -slope(tq, Tser[µ][w0 - 1:mlast])
            Vc = out["Vb"][jp, 0]
            if nlin_f1 > 0:
                out["Vf1"][jp] = -slope(tq, Tf1[w0 - 1:mlast])
            out["VA"][jp] = (TAser[mlast - 1] - TAser[w0 - 1]) / ((mlast - w0) * dt_cyc)
            nslip = sumlin(np.abs(Tmat[0]).ravel(order="F")[line_ok.ravel(order="F")]) / TWO_PI
            if nslip < 1:
                Vc = 0.0
        h0 = mlast - mlast // 2 + 1
        if mlast - h0 + 1 >= 3:
            th = np.arange(mlast - h0 + 1) * dt_cyc
            for µ in range(N):
                ns = sumlin(np.abs(Tmat[µ]).ravel(order="F")[line_ok.ravel(order="F")]) / TWO_PI
                out["Vh"][jp, µ] = 0.0 if ns < 1 else -slope(th, Tser[µ][h0 - 1:mlast])
        out["V"][jp] = Vc
        out["nslip"][jp] = nslip
        out["m"][jp] = mlast if any_band else m
        out["dmax"][jp] = dmax_cur
        out["nbig"][jp] = nbig_cur
        run.download(s)
        out["M"][jp] = magnetization(s.hz, Hc, gr)
        for µ in range(N):
            out["Nv"][jp, µ] = run.vortices(µ, kc)
            blk = s.F[µ][gr.x1 - 1:gr.x2 + 1, gr.y1 - 1:gr.y2 + 1, gr.z1 - 1:gr.z2 + 1]
            if mk.vac is None:
                out["psi2"][jp, µ] = meanlin((np.abs(blk) ** 2).ravel(order="F"))
            else:
                keep = ~np.asarray(mk.vac[gr.x1 - 1:gr.x2 + 1, gr.y1 - 1:gr.y2 + 1, gr.z1 - 1:gr.z2 + 1], dtype=bool)
                a = (np.abs(blk) ** 2).ravel(order="F")[keep.ravel(order="F")]
                out["psi2"][jp, µ] = sumlin(a) / len(a)
        conv, lastF = normal_verdict(conv, J, out["psi2"][jp, 0], lastF, pr.n_frac)
        out["conv"][jp] = conv
        if mlast >= 2:
            r0 = mlast // 2                   # the second half: cycles mlast÷2+1 .. mlast
            It = sum(ItSer[r0:mlast]) / (mlast - r0)
            Is = sum(IsSer[r0:mlast]) / (mlast - r0)
            Inom = J * slab_thickness(gr) * ((gr.y2 - gr.y1 + 1) * gr.dy)
            if abs(Inom) > 0:
                out["Itot"][jp] = abs(It) / abs(Inom)
                out["Isam"][jp] = abs(Is) / max(abs(It), np.finfo(float).eps)
        nV = nV + 1 if conv in ("V", "N") else 0
    return Ladder(label, Js, Hs, out["V"], out["Vb"], out["Vh"], out["Vst"], out["m"], "".join(out["conv"]),
                  out["res"], out["nslip"], out["M"], out["Nv"], out["psi2"], out["Itot"], out["Isam"], out["dmax"],
                  out["nbig"], out["Vf1"], out["VA"], dt_cyc, s, pr.slip_band_mode, out["slip_band"])


def rung_rate(L: Ladder) -> np.ndarray:
    """protocol.jl:130-144: the rate a rung is judged by (band 1: Vh, else V)."""
    return np.array([L.V[q] if math.isnan(L.Vh[q, 0]) else L.Vh[q, 0] for q in range(len(L.V))])


def rung_class(crossings: float, conv: str, require_silence: bool) -> str:
    """observables.jl:148-151."""
    if conv == "N" or crossings >= 10:
        return "D"
    return "S" if crossings < 1 and (not require_silence or conv in ("F", "D")) else "U"


def bracket_ic(J, V, tint, conv=None, require_silence=False):
    """observables.jl:132-146: (lo, hi, ok) of the critical current from the rungs' crossings."""
    idx = [q for q in range(len(J)) if abs(J[q]) > 1e-12]
    Ja = [abs(float(J[q])) for q in idx]
    cr = [abs(V[q]) * tint[q] / TWO_PI for q in idx]
    cls = [rung_class(cr[k], " " if conv is None else conv[idx[k]], require_silence) for k in range(len(cr))]
    d = cls.index("D") if "D" in cls else None
    hi = math.inf if d is None else Ja[d]
    below = list(range(len(Ja))) if d is None else list(range(d))
    s = [q for q in below if cls[q] == "S"]
    lo = math.nan if not s else Ja[s[-1]]
    und = [Ja[q] for q in below if cls[q] == "U" and (math.isnan(lo) or Ja[q] > lo)]
    return lo, hi, (not math.isnan(lo)) and math.isfinite(hi) and not und


def brackets(pos: Ladder, neg: Ladder):
    """protocol.jl:809-817 without the delay brackets: {'pos': (lo, hi, ok), 'neg': (lo, hi, ok)}."""
    req = pos.slip_band_mode == "any_band"
    return {"pos": bracket_ic(pos.J, rung_rate(pos), pos.m * pos.t_cycle, pos.conv, req),
            "neg": bracket_ic(neg.J, rung_rate(neg), neg.m * neg.t_cycle, neg.conv, req)}


def run_ladders(make_run, st: Stepper, Jl, *, H: float, pr: Protocol = Protocol()):
    """protocol.jl:842-861: both polarities over 0 and |Jl| (sorted), each from the Meissner seed with a fresh
    backend (make_run(st)); returns (pos, neg, brackets)."""
    Jp = np.array(sorted(set([0.0] + [abs(float(x)) for x in Jl])))
    res = []
    for label, Js in (("J+", Jp), ("J-", -Jp)):
        s0 = initial_state(st.model, st.grid, st.masks, H,
                           materials=st.mt.models if st.mt is not None else None)
        res.append(ladder(make_run(st), st, s0, Js, H=H, label=label, pr=pr))
    return res[0], res[1], brackets(res[0], res[1])


class DeviceLadder:
    """The ladder's backend on the B200: the state resident in one context, a protocol cycle = tdgl_steps."""

    def __init__(self, st: Stepper):
        from . import gpu
        self.gs = gpu.GPUStepper(st)

    def reset(self, s: State):
        self.gs.upload(s)
        c = self.gs.carry
        c.pcg_warm, c.pcg_have2, c.open_count = 0, 0, -1
        self.gs.set_carry(c)

    def meter_set(self, vm):
        self.gs.meter_set(vm)

    def cycle(self, n: int, H: float, HJ: float):
        self.gs.steps(n, H, HJ)

    def measure(self):
        return self.gs.measure()

    def download(self, s: State):
        self.gs.download(s)

    def vortices(self, band: int, kc: int) -> int:
        return self.gs.vortices(band, kc)[0]

    def close(self):
        self.gs.close()
