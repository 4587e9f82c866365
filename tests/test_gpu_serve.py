"""The served onset search (juliatdgl_b200/serve.py): runs admitted into a stream overlap on the device, and each
run's result — onset current, delay, rungs and steps — is the same alone and in the mix (each run keeps its own
context, stream and snapshots); the drop-in path (state on the host between cycles, phases on the host) finds the
same onsets.  An HBM budget smaller than two runs serialises admission without changing any result.
"""
import math

import pytest

import juliatdgl_b200 as T
from juliatdgl_b200 import serve
from juliatdgl_b200.grid import GeomSpec, build_masks

pytestmark = pytest.mark.gpu

SPEC = serve.OnsetSpec(J0=0.2, dJ=0.15, nrung=5, t_rung=3.0, t_confirm=6.0)


def requests():
    out = []
    for i, (nx, ny, nz, three, sign) in enumerate([(64, 32, 8, False, 1.0), (48, 24, 6, True, -1.0),
                                                   (96, 40, 10, False, -1.0), (32, 16, 4, False, 1.0)]):
        md = T.two_band(xi_ratio=4.0, κ=25.0)
        if three:
            b1, b2 = md.bands
            md = T.Model.make((b1, b2, T.Band.make(m=2.0, Γ=1.2, a=0.8)),
                              [[0.0, 1e-3, -0.02], [1e-3, 0.0, -0.02], [-0.02, -0.02, 0.0]], κ=25.0)
        gr = T.Grid.make(nx, ny, nz, dx=0.5, buf=1)
        mk = build_masks(GeomSpec(GEOM_MODE="WEDGE"), gr)
        st = T.Stepper.make(md, gr, mk)
        out.append(serve.Request(i, st, T.initial_state(md, gr, mk, 0.03), 0.03, sign, 0.0))
    return out


def key(r):
    return (r.id, r.onset_J if not math.isnan(r.onset_J) else "none", r.delay if not math.isnan(r.delay) else "none",
            r.rungs, r.steps)


def test_each_result_is_the_same_alone_and_in_the_mix():
    reqs = requests()
    mix = serve.Server(SPEC).run(reqs, realtime=False)
    assert any(not math.isnan(r.onset_J) for r in mix)
    for r in reqs:
        alone = serve.Server(SPEC).run([r], realtime=False)
        assert key(alone[0]) == key(mix[r.id])


def test_a_small_budget_serialises_admission_with_the_same_results():
    reqs = requests()
    srv = serve.Server(SPEC, budget_bytes=1.0)
    res = srv.run(reqs, realtime=False)
    assert srv.peak_active == 1
    ref = serve.Server(SPEC).run(reqs, realtime=False)
    assert [key(r) for r in res] == [key(r) for r in ref]


def test_the_drop_in_path_finds_the_same_onsets():
    reqs = requests()[:2]
    served = serve.Server(SPEC).run(reqs, realtime=False)
    for r in reqs:
        plain, secs = serve.plain_service(r, SPEC)
        a, b = served[r.id], plain
        assert (a.rungs, a.steps) == (b.rungs, b.steps)
        assert (math.isnan(a.onset_J) and math.isnan(b.onset_J)) or a.onset_J == b.onset_J
        assert (math.isnan(a.delay) and math.isnan(b.delay)) or a.delay == pytest.approx(b.delay)


def test_merged_batches_and_per_run_streams_give_the_same_results():
    """The active runs stepped as one merged batch per cycle, and each on its own stream: the same searches."""
    reqs = requests()
    srv = serve.Server(SPEC, merged=True)
    merged = srv.run(reqs, realtime=False)
    assert srv.batches >= 1
    streams = serve.Server(SPEC).run(reqs, realtime=False)
    assert [key(r) for r in merged] == [key(r) for r in streams]
