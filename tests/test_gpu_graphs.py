"""The step as a CUDA graph (tdgl_set_graphs): the captured step launches the same kernels in the same order as the
step launched from the host, with H, HJ, the open boundary's ramp fraction and the noise index read from device
memory and the PCG loop as a conditional node, so the results must be identical to the bit — over ramps of HJ, the
recomputations of the open boundary (launched outside the graph), noise, materials and the PCG of the padding,
across both θ/φ parities and several calls.
"""
import numpy as np
import pytest

import cases
from juliatdgl_b200 import gpu

pytestmark = pytest.mark.gpu

CASES = [("small", "euler_substeps", {}), ("small", "rkc_kwt_rotframe", {}), ("small", "pcg_f32", {}),
         ("small", "pcg", {}), ("small", "open_pcg", {}), ("small", "three_bands", cases.NOISY["three_bands"]),
         ("small", "pcg_f32", cases.NOISY["pcg_f32"]), ("material", "mat_sigma", {}),
         ("material", "mat_three_kwt", cases.MATERIAL_NOISY["mat_three_kwt"]), ("small", "qp_pcg", {}),
         ("vacuum", "vac_qp", {}), ("vacuum", "vac_qpn", {})]


def run(st, s, H, HJ, graphs):
    gs = gpu.GPUStepper(st)
    try:
        gs.set_graphs(graphs)
        b = s.copy()
        gs.upload(b)
        gs.steps(7, H, HJ)                                    # odd: the next call starts on the other parity
        ramp = HJ * (1 + 0.01 * np.arange(13))
        gs.steps_ramp(H, ramp)
        gs.steps(20, H, HJ)
        st_ = gs.stats()
        return gs.download(b), gs.get_carry(), (st_.steps, st_.pcg_total_iters, st_.pcg_last_iters)
    finally:
        gs.close()


@pytest.mark.parametrize("builder,kind,kw", CASES, ids=[f"{k}{'_noise' if kw else ''}" for _, k, kw in CASES])
def test_graph_steps_are_the_eager_steps(builder, kind, kw):
    st, s, H, HJ = getattr(cases, builder)(kind, **kw)
    a, ca, sa = run(st, s, H, HJ, graphs=False)
    b, cb, sb = run(st, s, H, HJ, graphs=True)
    assert sa == sb
    assert cases.compare_states(b, a)[0] == 0.0
    assert np.array_equal(ca.pcg_x, cb.pcg_x) and np.array_equal(ca.pcg_xprev, cb.pcg_xprev)
    assert (ca.pcg_warm, ca.pcg_have2, ca.open_count) == (cb.pcg_warm, cb.pcg_have2, cb.open_count)


@pytest.mark.parametrize("kind", ["pcg_f32", "pcg", "open_pcg"])
def test_pcg_work_beside_the_preconditioner_keeps_the_bits(kind):
    """x += αP and r·z_old run on a second stream beside the preconditioner, except when the launches are timed one
    by one (profiling on), which runs the same kernels in order on one stream: both give the same bits."""
    st, s, H, HJ = cases.small(kind)
    out = []
    for prof in (False, True):
        gs = gpu.GPUStepper(st)
        try:
            gs.profile(prof)
            b = s.copy()
            gs.upload(b)
            gs.steps(12, H, HJ)
            st_ = gs.stats()
            out.append((gs.download(b), gs.get_carry().pcg_x.copy(), (st_.steps, st_.pcg_total_iters)))
        finally:
            gs.close()
    (a, xa, sa), (b, xb, sb) = out
    assert sa == sb
    assert cases.compare_states(b, a)[0] == 0.0
    assert np.array_equal(xa, xb)


@pytest.mark.parametrize("kind,kw", [("three_bands", {}), ("pcg_f32", {}), ("rkc_kwt_rotframe", cases.NOISY["rkc_kwt_rotframe"])])
def test_branches_inside_a_step_keep_the_bits(kind, kw):
    """The bands side by side and the PCG's work beside its preconditioner (tdgl_set_branches, on by default) give
    the bits of the same kernels in one chain."""
    st, s, H, HJ = cases.small(kind, **kw)
    out = []
    for on in (True, False):
        gs = gpu.GPUStepper(st)
        try:
            gs.set_branches(on)
            b = s.copy()
            gs.upload(b)
            gs.steps(9, H, HJ)
            gs.steps(12, H, 1.2 * HJ)
            out.append(gs.download(b))
        finally:
            gs.close()
    assert cases.compare_states(out[0], out[1])[0] == 0.0
