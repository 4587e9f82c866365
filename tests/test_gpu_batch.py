"""Batches (tdgl_batch_*): contexts of uneven grids and different paths stepped in lockstep, one graph launch per
step.  Each run in the batch gives exactly the bits it gives alone (the branches share no memory), and the batch
advances every context by the requested steps with its own H and HJ.
"""
import pytest

import cases
from juliatdgl_b200 import gpu

pytestmark = pytest.mark.gpu

MEMBERS = [("small", "euler_substeps", {}), ("small", "rkl_bar", {}), ("small", "rkc_kwt_rotframe", {}), ("small", "pcg_f32", {}),
           ("small", "three_bands", cases.NOISY["three_bands"]), ("material", "mat_two", {}),
           ("material", "mat_sigma", {})]


def build(builder, kind, kw):
    return getattr(cases, builder)(kind, **kw)


@pytest.mark.parametrize("members", [MEMBERS])
def test_a_run_in_a_batch_is_the_run_alone(members):
    runs = [build(*m) for m in members]
    alone = []
    for st, s, H, HJ in runs:
        gs = gpu.GPUStepper(st)
        b = s.copy()
        gs.upload(b)
        gs.steps(11, H, HJ)
        gs.steps(14, H, 1.5 * HJ)
        alone.append(gs.download(b))
        gs.close()
    ctxs = []
    for st, s, H, HJ in runs:
        gs = gpu.GPUStepper(st)
        gs.upload(s.copy())
        ctxs.append(gs)
    bt = gpu.Batch(ctxs)
    try:
        Hs = [r[2] for r in runs]
        HJs = [r[3] for r in runs]
        bt.steps(11, Hs, HJs)
        assert bt.one_graph
        bt.steps(14, Hs, [1.5 * h for h in HJs])
        for gs, (st, s, H, HJ), a in zip(ctxs, runs, alone):
            assert gs.stats().steps == 25
            if st.selffield_bc == 2:   # the open boundary
                assert gs.stats().open_recomputes >= 3
            assert cases.compare_states(gs.download(s.copy()), a)[0] == 0.0
    finally:
        bt.close()
        for gs in ctxs:
            gs.close()


def test_open_boundary_runs_in_a_batch_are_each_run_alone():
    """Open-boundary runs (their ramps and recomputations, with and without the PCG padding) batched with a run
    without it: the bits of each run alone, over steps that cross several recomputations and a change of HJ."""
    members = [("small", "open", {}), ("small", "open_pcg", {}), ("small", "rkl_bar", {})]
    test_a_run_in_a_batch_is_the_run_alone(members)


def test_a_batch_of_an_open_run_and_a_noisy_run_keeps_both_streams():
    members = [("small", "open", {}), ("small", "three_bands", cases.NOISY["three_bands"])]
    test_a_run_in_a_batch_is_the_run_alone(members)


def test_sweep_subset_in_a_batch_is_each_run_alone():
    """Eight runs of the mixed-size sweep (contexts of different sizes created before any steps, so one context's
    set-up must not change another's launches): batched against alone, to the bit."""
    from juliatdgl_b200 import sweep
    runs = sweep.sweep_instances(64, seed=2)[:8]
    ctxs = []
    for r in runs:
        gs = gpu.GPUStepper(r.st)
        gs.upload(r.s.copy())
        ctxs.append(gs)
    bt = gpu.Batch(ctxs)
    try:
        bt.steps(30, [r.H for r in runs], [r.HJ for r in runs])
        assert bt.one_graph
        info = bt.merge_info
        # the sweep's runs launch the same kernels: all eight share one chain of merged launches
        assert info["contexts"] == 8 and info["chains"] == 1, info
        got = [g.download(r.s.copy()) for g, r in zip(ctxs, runs)]
    finally:
        bt.close()
        for g in ctxs:
            g.close()
    for r, b in zip(runs, got):
        gs = gpu.GPUStepper(r.st)
        a = r.s.copy()
        gs.upload(a)
        gs.steps(30, r.H, r.HJ)
        gs.download(a)
        gs.close()
        assert cases.compare_states(b, a)[0] == 0.0


def _alone(st, s, H, HJ, n1, n2):
    gs = gpu.GPUStepper(st)
    b = s.copy()
    gs.upload(b)
    gs.steps(n1, H, HJ)
    gs.steps(n2, H, 1.5 * HJ)
    gs.download(b)
    gs.close()
    return b


UNEVEN = [(16, 8, 4), (20, 8, 4), (16, 12, 6), (24, 10, 5), (18, 8, 4)]


@pytest.mark.parametrize("blocks_per_sm", [0.0, 0.25, 64.0])
def test_merged_launches_of_uneven_grids_give_each_run_alone(blocks_per_sm):
    """Five bar-field runs of different grids (one group of merged launches; the plane transforms' x-grids resized
    by blocks_per_sm), two noisy three-band runs of different grids, and a PCG run (its loop keeps its own
    launches): each run to the bit as alone, with fewer launches than the runs' own."""
    runs = [cases.small("rkl_bar", grid=g) for g in UNEVEN]
    runs += [cases.small("three_bands", grid=g, **cases.NOISY["three_bands"]) for g in ((16, 8, 4), (20, 10, 4))]
    runs += [cases.small("pcg_f32")]
    alone = [_alone(*r, 9, 12) for r in runs]
    ctxs = []
    for st, s, H, HJ in runs:
        gs = gpu.GPUStepper(st)
        gs.upload(s.copy())
        ctxs.append(gs)
    bt = gpu.Batch(ctxs, blocks_per_sm=blocks_per_sm)
    try:
        Hs = [r[2] for r in runs]
        HJs = [r[3] for r in runs]
        bt.steps(9, Hs, HJs)
        info = bt.merge_info
        assert info["contexts"] >= len(UNEVEN) and info["chains"] >= 1, info
        bt.steps(12, Hs, [1.5 * h for h in HJs])
        for gs, (st, s, H, HJ), a in zip(ctxs, runs, alone):
            assert gs.stats().steps == 21
            assert cases.compare_states(gs.download(s.copy()), a)[0] == 0.0
        bt.set_merge(False)
        bt.steps(2, Hs, HJs)
        own = bt.merge_info["launches"]
        assert bt.merge_info["contexts"] == 0 and own > info["launches"], (own, info)
    finally:
        bt.close()
        for gs in ctxs:
            gs.close()


def test_autotuned_launch_shape_keeps_each_run_alone():
    """The autotuner steps the runs with each candidate launch shape and keeps the fastest; the runs' states are
    those of the same steps alone."""
    runs = [cases.small("rkl_bar", grid=g) for g in UNEVEN]
    alone = []
    for st, s, H, HJ in runs:
        gs = gpu.GPUStepper(st)
        b = s.copy()
        gs.upload(b)
        gs.steps(15, H, HJ)
        alone.append(gs.download(b))
        gs.close()
    ctxs = []
    for st, s, H, HJ in runs:
        gs = gpu.GPUStepper(st)
        gs.upload(s.copy())
        ctxs.append(gs)
    bt = gpu.Batch(ctxs)
    try:
        Hs = [r[2] for r in runs]
        HJs = [r[3] for r in runs]
        bt.steps(3, Hs, HJs)
        times = bt.tune(Hs, HJs, candidates=(0.5, 4.0), steps=2)   # 2 × (2 + 2) steps
        assert set(times) == {0.5, 4.0}
        bt.steps(4, Hs, HJs)
        assert bt.merge_info["contexts"] == len(UNEVEN)
        for gs, (st, s, H, HJ), a in zip(ctxs, runs, alone):
            assert gs.stats().steps == 15
            assert cases.compare_states(gs.download(s.copy()), a)[0] == 0.0
    finally:
        bt.close()
        for gs in ctxs:
            gs.close()


def test_a_group_larger_than_one_launch_holds_is_cut_into_chains():
    """60 runs with the same kernels: more than the parameters of one merged launch hold (about 54 records of the
    largest kernel), so the group runs as two chains; every run keeps its bits."""
    grids = [(16 + (q % 5), 8 + 2 * (q % 3), 4) for q in range(60)]
    runs = [cases.small("rkl_bar", grid=g) for g in grids]
    alone = []
    for st, s, H, HJ in runs:
        gs = gpu.GPUStepper(st)
        b = s.copy()
        gs.upload(b)
        gs.steps(6, H, HJ)
        alone.append(gs.download(b))
        gs.close()
    ctxs = []
    for st, s, H, HJ in runs:
        gs = gpu.GPUStepper(st)
        gs.upload(s.copy())
        ctxs.append(gs)
    bt = gpu.Batch(ctxs)
    try:
        bt.steps(6, [r[2] for r in runs], [r[3] for r in runs])
        info = bt.merge_info
        assert info["contexts"] == 60 and info["chains"] >= 2, info
        for gs, (st, s, H, HJ), a in zip(ctxs, runs, alone):
            assert cases.compare_states(gs.download(s.copy()), a)[0] == 0.0
    finally:
        bt.close()
        for gs in ctxs:
            gs.close()
