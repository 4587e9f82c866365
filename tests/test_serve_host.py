"""The serving engine's host logic (juliatdgl_b200/serve.py) without a GPU: the contexts are replaced by a fake whose
voltmeter phase advances at a rate set by the applied current, so that each run's onset rung is known in advance.
Covers the onset search with its delay confirmation, admission against the HBM budget (one run at a time when the
budget holds one, the finished runs' memory released first), and the pipelined per-run streams and the merged batch
giving the same results."""
import math

import numpy as np
import pytest

import cases
from juliatdgl_b200 import serve
from juliatdgl_b200.scheme import selffield

SPEC = serve.OnsetSpec(J0=0.1, dJ=0.1, nrung=6, t_rung=2.0, t_confirm=4.0, lmax=40, delta_v=2)


class FakeStepper:
    """A context whose voltmeter phase grows by rate(HJ) per step once |J| passes the run's critical current."""

    live = 0
    closed = 0

    def __init__(self, st):
        self.st = st
        self.phase = 0.0
        self.steps_done = 0
        self.snaps = {}
        self.device_bytes = serve.estimate_bytes(st)
        FakeStepper.live += 1

    def set_branches(self, on=True):
        self.branches = on

    def upload(self, s):
        pass

    def meter_set(self, vm, nphase=1):
        self.shape = vm.Min.shape

    def _rate(self, HJ):
        J = abs(HJ / selffield(self.st, 1.0)) if selffield(self.st, 1.0) else 0.0
        jc = getattr(self.st, "_fake_jc")
        return 0.0 if J < jc - 1e-12 else 0.05 * (1 + 10 * (J - jc))

    def steps(self, n, H, HJ, wait=True):
        self.phase += n * self._rate(HJ)
        self.steps_done += n

    def sync(self):
        return 0

    def measure(self):
        wrapped = (self.phase + math.pi) % (2 * math.pi) - math.pi
        return {"D": [np.full(self.shape, wrapped, order="F")]}

    def snapshot(self, slot=0):
        self.snaps[slot] = self.phase

    def restore(self, slot=0):
        self.phase = self.snaps[slot]

    def close(self):
        FakeStepper.live -= 1
        FakeStepper.closed += 1


class FakeBatch:
    def __init__(self, steppers):
        self.gs = list(steppers)

    def steps(self, n, H, HJ, wait=True):
        for g, h, hj in zip(self.gs, H, HJ):
            g.steps(n, h, hj)

    def close(self):
        pass


@pytest.fixture
def fake(monkeypatch):
    monkeypatch.setattr(serve.gpu, "GPUStepper", FakeStepper)
    monkeypatch.setattr(serve.gpu, "Batch", FakeBatch)
    FakeStepper.live = FakeStepper.closed = 0
    return FakeStepper


def requests(jcs):
    out = []
    for i, jc in enumerate(jcs):
        st, s, H, HJ = cases.small("rkl_bar")
        object.__setattr__(st, "_fake_jc", jc)
        out.append(serve.Request(i, st, s, H, 1.0 if i % 2 == 0 else -1.0, 0.0))
    return out


def test_onsets_follow_the_critical_currents(fake):
    # jc 0.25: rung 0.3 slips; the rung below (0.2) does not within the confirmation, so the onset is 0.3
    # jc 0.05: the first rung slips: the onset is J0 itself; jc 9: no rung slips
    res = serve.Server(SPEC).run(requests([0.25, 0.05, 9.0]), realtime=False)
    assert res[0].onset_J == pytest.approx(0.3) and res[0].rungs == 3
    assert res[1].onset_J == pytest.approx(-0.1) and res[1].rungs == 1
    assert math.isnan(res[2].onset_J) and res[2].rungs == SPEC.nrung
    assert fake.live == 0 and fake.closed == 3   # every context closed by the end


def test_a_budget_for_one_run_serialises_admission(fake):
    reqs = requests([0.25, 0.05, 0.45, 9.0])
    one = serve.estimate_bytes(reqs[0].st)
    srv = serve.Server(SPEC, budget_bytes=one * 1.5)
    res = srv.run(reqs, realtime=False)
    assert srv.peak_active == 1
    ref = serve.Server(SPEC).run(reqs, realtime=False)
    key = lambda r: (r.id, r.onset_J if not math.isnan(r.onset_J) else None, r.rungs, r.steps)
    assert [key(r) for r in res] == [key(r) for r in ref]


def test_streams_and_merged_batches_agree(fake):
    reqs = requests([0.25, 0.05, 0.45, 9.0, 0.15])
    key = lambda r: (r.id, r.onset_J if not math.isnan(r.onset_J) else None, r.delay if not math.isnan(r.delay) else None,
                     r.rungs, r.steps)
    a = serve.Server(SPEC).run(reqs, realtime=False)
    srv = serve.Server(SPEC, merged=True)
    b = srv.run(reqs, realtime=False)
    assert [key(r) for r in a] == [key(r) for r in b]
    assert srv.batches >= 2   # formed again as runs finished
