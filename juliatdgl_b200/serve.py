"""The served onset search: runs of different grids arrive as a stream, are admitted against an HBM budget as memory
frees up, and step together on one GPU, each keeping its fields, links, PCG state and snapshots resident; only the
path phases of the voltmeter cross to the host per cycle.

Each run is an onset search at field H: a current ladder J_k = J0 + k·dJ (with the run's polarity), each rung held
for `t_rung` in protocol cycles of lMax steps; a rung slips when the line-averaged phase across the voltmeter
(gtdgl/src/protocol.jl:168-189, as `crossing_times` :271-296) passes 2π since the rung started.  The first slip is
then confirmed by the reference's delay rule (`_continue_rung`, protocol.jl:238-258): the previous rung is continued
from its own start (a device snapshot: state, carry, step count) for up to `t_confirm`; if it slips within that time
the onset is that rung's current with that delay, otherwise the slipping rung's.  (The reference keeps a ring of the
closed rungs for this; here the one below the slip.)

`Server.run` is continuous batching.  By default each run has its own stream and the runs' cycles are pipelined:
every admitted run has a cycle in flight; the host takes the oldest, waits for that cycle alone while the others keep
the device busy, reads its phases, moves its search on and enqueues its next cycle at once; new runs are admitted
as they arrive and the budget allows (the contexts of finished runs are closed when their memory is needed, since
freeing device memory waits for the whole device).  With merged=True the active runs instead step each cycle
together as one batch (tdgl_batch_*: runs with the same kernels share merged launches), formed again when a run joins
or leaves, and the host reads every run's phases between cycles.  `plain_service` is the drop-in path for comparison: one run at a time, the state on the host
between cycles (up, lMax steps, down, phases on the host), as the reference's accelerator hook works.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import gpu
from .grid import GeomSpec, Grid, build_masks
from .model import Band, Model, two_band
from .protocol import line_mean, path_phase_host, unwrap, voltmeter
from .scheme import Stepper, selffield
from .state import State, initial_state

TWO_PI = 2 * math.pi


@dataclass
class OnsetSpec:
    J0: float = 0.1
    dJ: float = 0.1
    nrung: int = 10
    t_rung: float = 5.0       # t_GL per rung
    t_confirm: float = 10.0   # t_GL of the delay confirmation
    lmax: int = 40            # steps per protocol cycle
    delta_v: int = 8


@dataclass
class Request:
    id: int
    st: Stepper
    s: State
    H: float
    sign: float
    arrival: float = 0.0


@dataclass
class Result:
    id: int
    onset_J: float            # NaN: no slip up to the last rung
    delay: float              # t_GL from the start of the onset rung to its first slip
    rungs: int                # rungs stepped (confirmation excluded)
    steps: int
    arrival: float = 0.0
    admitted: float = 0.0
    finished: float = 0.0

    @property
    def time_to_onset(self) -> float:
        return self.finished - self.arrival


def served_requests(n: int, seed: int = 3, rate: float = 4.0, H: float = 0.03):
    """The served stream: Poisson arrivals at `rate` runs/s; two- or three-band runs (50/50) on grids drawn
    log-uniformly per axis from 32×16×4 to 256×128×32 cells, a WEDGE notch, polarity 50/50."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate))
        nx, ny, nz = (int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
                      for lo, hi in ((32, 256), (16, 128), (4, 32)))
        three = bool(rng.random() < 0.5)
        sign = 1.0 if rng.random() < 0.5 else -1.0
        md = two_band(xi_ratio=4.0, κ=25.0)
        if three:
            b1, b2 = md.bands
            md = Model.make((b1, b2, Band.make(m=2.0, Γ=1.2, a=0.8)),
                            [[0.0, 1e-3, -0.02], [1e-3, 0.0, -0.02], [-0.02, -0.02, 0.0]], κ=25.0)
        gr = Grid.make(nx, ny, nz, dx=0.5, buf=1)
        mk = build_masks(GeomSpec(GEOM_MODE="WEDGE"), gr)
        st = Stepper.make(md, gr, mk)
        out.append(Request(i, st, initial_state(md, gr, mk, H), H, sign, t))
    return out


class Search:
    """The onset search of one run on its context: a small state machine driven once per cycle."""

    def __init__(self, req: Request, spec: OnsetSpec, gs):
        self.req, self.spec, self.gs = req, spec, gs
        st = req.st
        self.dv = max(1, min(spec.delta_v, (st.grid.x2 - st.grid.x1) // 4))
        self.vm = voltmeter(st.grid, st.masks, self.dv)
        gs.meter_set(self.vm, nphase=1)
        self.cyc = int(math.ceil(spec.t_rung / (spec.lmax * st.dt)))
        self.cyc_conf = int(math.ceil(spec.t_confirm / (spec.lmax * st.dt)))
        self.k = 0
        self.mode = "ladder"       # ladder → confirm → done
        self.steps = 0
        self.result = None
        self._start_rung(0)

    def J(self, k):
        return self.req.sign * (self.spec.J0 + k * self.spec.dJ)

    def _start_rung(self, k):
        self.k = k
        self.gs.snapshot(k % 2)            # the start of this rung, for the confirmation of the next
        self._begin(selffield(self.req.st, self.J(k)))

    def _begin(self, HJ):
        self.HJ = HJ
        self.Dp = self.gs.measure()["D"][0].copy()
        self.acc = np.zeros_like(self.Dp)
        self.q = 0

    def enqueue(self):
        self.gs.steps(self.spec.lmax, self.req.H, self.HJ, wait=False)
        self.steps += self.spec.lmax

    def poll(self) -> bool:
        """After the enqueued cycle: reads the phases and moves on; True when the search is done."""
        self.q += 1
        D = self.gs.measure()["D"][0]
        unwrap(self.acc, D, self.Dp)
        ph = line_mean(self.acc, self.vm.line_ok)
        slip = abs(ph) >= TWO_PI or not math.isfinite(ph)
        t = self.q * self.spec.lmax * self.req.st.dt
        if self.mode == "ladder":
            if slip:
                self.slip_k, self.slip_t = self.k, t
                if self.k == 0:
                    return self._done(self.J(0), t)
                self.mode = "confirm"
                self.gs.restore((self.k - 1) % 2)
                self._begin(selffield(self.req.st, self.J(self.k - 1)))
                return False
            if self.q >= self.cyc:
                if self.k + 1 >= self.spec.nrung:
                    return self._done(float("nan"), float("nan"))
                self._start_rung(self.k + 1)
            return False
        # confirm: the rung below, continued from its start
        if slip:
            return self._done(self.J(self.slip_k - 1), t)
        if self.q >= self.cyc_conf:
            return self._done(self.J(self.slip_k), self.slip_t)
        return False

    def _done(self, J, delay):
        self.mode = "done"
        self.result = Result(self.req.id, J, delay, self.k + 1, self.steps, self.req.arrival)
        return True


def estimate_bytes(st: Stepper) -> int:
    """Device memory of a run before it is admitted: the state and workspaces per node (bands, links, the separable
    or PCG solve), and two snapshots of the state."""
    g = st.grid
    nn = (g.Nx + 1) * (g.Ny + 1) * (g.Nz + 1)
    N = st.model.N
    state = nn * (32 * N + 3 * (4 * 8 + 2 * 16))
    work = nn * (2 * 16 + 3 * (2 * 16 + 8) + 2 * 8 + 24)
    solve = nn * (3 * 8 * (12 if st.solver == 3 else 4))
    return int(state * 3 + work + solve)


class Server:
    """Continuous batching of onset searches on one GPU (see the module docstring)."""

    def __init__(self, spec: OnsetSpec | None = None, budget_bytes: float = 150e9, merged: bool = False,
                 branches: bool = False):
        self.spec = spec or OnsetSpec()
        self.budget = budget_bytes
        self.merged = merged
        # the parallel branches inside each run's step (tdgl_set_branches): off by default, since the runs in flight
        # already fill the device and each run's chain of launches then keeps to its own stream
        self.branches = branches

    def run(self, requests, *, realtime: bool = True):
        """Serves `requests` (arrival times relative to the call with realtime; all at once without) and returns the
        results by id.  Sets peak_active, makespan, batches and t_phase (host seconds by phase)."""
        self._pending = sorted(requests, key=lambda r: r.arrival)
        self._results, self._parked = [], []
        self._used = 0
        self._t0 = time.perf_counter()
        self._realtime = realtime
        self.peak_active = 0
        self.batches = 0
        # host seconds by phase: admitting runs, forming batches, enqueuing cycles (captures included), waiting for
        # the device, reading the phases and moving the searches on, closing finished runs
        self.t_phase = {"admit": 0.0, "form": 0.0, "enqueue": 0.0, "wait": 0.0, "poll": 0.0, "close": 0.0}
        if self.merged:
            self._run_merged()
        else:
            self._run_streams()
        # the makespan ends with the last result; closing the finished runs' contexts after it is cleanup
        self.makespan = max((r.finished for r in self._results), default=self._now())
        c = time.perf_counter()
        self._close_parked()
        self.cleanup = time.perf_counter() - c
        return sorted(self._results, key=lambda r: r.id)

    def _now(self):
        return time.perf_counter() - self._t0

    def _admit(self, active, started=None) -> list:
        """Admits the runs that have arrived while the budget allows (at least one when none is active); closes the
        parked contexts of finished runs first when their memory is needed.  `started(search)` is called on each at
        once (its first cycle can run while the next is set up).  Returns the new searches."""
        c = time.perf_counter()
        new = []
        while self._pending and (not self._realtime or self._pending[0].arrival <= self._now()):
            r = self._pending[0]
            est = estimate_bytes(r.st)
            if active + len(new) and self._used + est > self.budget:
                if not self._parked:
                    break
                self._close_parked()
                continue
            self._pending.pop(0)
            gs = gpu.GPUStepper(r.st)
            if not self.branches:
                gs.set_branches(False)
            gs.upload(r.s.copy())
            srch = Search(r, self.spec, gs)
            srch.admitted = self._now()
            srch.bytes = gs.device_bytes
            self._used += srch.bytes
            new.append(srch)
            if started:
                started(srch)
        self.t_phase["admit"] += time.perf_counter() - c
        return new

    def _finish(self, a):
        """Records a finished search; its context is parked (closing frees memory, which waits for the whole device,
        so it is left for when the memory is needed or the end)."""
        res = a.result
        res.admitted, res.finished = a.admitted, self._now()
        self._results.append(res)
        self._parked.append(a)

    def _close_parked(self):
        c = time.perf_counter()
        for a in self._parked:
            a.gs.close()
            self._used -= a.bytes
        self._parked = []
        self.t_phase["close"] += time.perf_counter() - c

    def _wait_for_arrival(self):
        if self._pending:
            time.sleep(max(0.0, self._pending[0].arrival - self._now()))

    def _run_streams(self):
        """Each run on its own stream, pipelined: the runs' cycles are in flight in arrival order; the host takes the
        oldest, waits for its cycle alone (the others' keep the device busy), reads its phases and enqueues its next
        cycle at once."""
        ring = deque()
        clock = time.perf_counter
        def started(a):
            a.enqueue()
            ring.append(a)

        while self._pending or ring:
            self._admit(len(ring), started)
            self.peak_active = max(self.peak_active, len(ring))
            if not ring:
                self._wait_for_arrival()
                continue
            a = ring.popleft()
            c0 = clock()
            a.gs.sync()
            c1 = clock()
            fin = a.poll()
            c2 = clock()
            if fin:
                self._finish(a)
            else:
                a.enqueue()
                ring.append(a)
            c3 = clock()
            for k, v in zip(("wait", "poll", "enqueue"), (c1 - c0, c2 - c1, c3 - c2)):
                self.t_phase[k] += v

    def _run_merged(self):
        """The active runs step each cycle together as one batch (merged launches), formed again when a run joins or
        leaves; then each reads its phases."""
        active = []
        batch, members = None, []
        clock = time.perf_counter
        while self._pending or active:
            active += self._admit(len(active))
            self.peak_active = max(self.peak_active, len(active))
            if not active:
                self._wait_for_arrival()
                continue
            c0 = clock()
            if [id(a) for a in active] != members:   # a run joined or left: the batch is formed again
                if batch:
                    batch.close()
                batch = gpu.Batch([a.gs for a in active])
                members = [id(a) for a in active]
                self.batches += 1
            c1 = clock()
            batch.steps(self.spec.lmax, [a.req.H for a in active], [a.HJ for a in active], wait=False)
            for a in active:
                a.steps += self.spec.lmax
            c2 = clock()
            for a in active:
                a.gs.sync()
            c3 = clock()
            done = [a.poll() for a in active]
            c4 = clock()
            for k, v in zip(("form", "enqueue", "wait", "poll"), (c1 - c0, c2 - c1, c3 - c2, c4 - c3)):
                self.t_phase[k] += v
            if any(done):   # the batch goes before the finished runs' contexts
                batch.close()
                batch, members = None, []
            for a, fin in zip(active, done):
                if fin:
                    self._finish(a)
            active = [a for a, fin in zip(active, done) if not fin]
        if batch:
            batch.close()


def plain_service(req: Request, spec: OnsetSpec):
    """The same search through the drop-in path, alone: the state on the host between cycles (up, lMax steps, down),
    the phases computed on the host, host copies for the confirmation.  Returns (Result, seconds)."""
    st = req.st
    gs = gpu.GPUStepper(st)
    s = req.s.copy()
    gr = st.grid
    dv = max(1, min(spec.delta_v, (gr.x2 - gr.x1) // 4))
    vm = voltmeter(gr, st.masks, dv)
    vi, vo = vm.vi, vm.vo
    cyc = int(math.ceil(spec.t_rung / (spec.lmax * st.dt)))
    cyc_conf = int(math.ceil(spec.t_confirm / (spec.lmax * st.dt)))
    t0 = time.perf_counter()
    steps = 0

    def cycle(s, HJ):
        nonlocal steps
        gs.upload(s)
        gs.steps(spec.lmax, req.H, HJ)
        gs.download(s)
        steps += spec.lmax
        return path_phase_host(s.G[0], s.Vx, gr, vi, vo)

    def hold(s, J, ncyc, carry):
        gs.set_carry(carry)
        HJ = selffield(st, J)
        Dp = path_phase_host(s.G[0], s.Vx, gr, vi, vo)
        acc = np.zeros_like(Dp)
        for q in range(1, ncyc + 1):
            D = cycle(s, HJ)
            unwrap(acc, D, Dp)
            ph = line_mean(acc, vm.line_ok)
            if abs(ph) >= TWO_PI or not math.isfinite(ph):
                return q * spec.lmax * st.dt
        return None

    J = lambda k: req.sign * (spec.J0 + k * spec.dJ)
    prev = None
    res = None
    for k in range(spec.nrung):
        start = (s.copy(), gs.get_carry())        # the rung's start, for the confirmation of the next rung
        start = (start[0], _copy_carry(start[1]))
        t = hold(s, J(k), cyc, start[1])
        if t is not None:
            if k == 0 or prev is None:
                res = Result(req.id, J(k), t, k + 1, steps, req.arrival)
                break
            s2 = prev[0].copy()
            t2 = hold(s2, J(k - 1), cyc_conf, prev[1])
            res = Result(req.id, J(k - 1) if t2 is not None else J(k), t2 if t2 is not None else t, k + 1, steps,
                         req.arrival)
            break
        prev = start
    if res is None:
        res = Result(req.id, float("nan"), float("nan"), spec.nrung, steps, req.arrival)
    dt = time.perf_counter() - t0
    gs.close()
    return res, dt


def _copy_carry(c):
    import copy
    return copy.deepcopy(c)


def fifo(arrivals, services):
    """Finish times of a single first-come-first-served server."""
    out, t = [], 0.0
    for a, s in zip(arrivals, services):
        t = max(t, a) + s
        out.append(t)
    return out
