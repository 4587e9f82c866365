"""Parity of the benchmark's scheme as a whole: the three-band KWT ramp (RKC stages with the rotating frame, the PCG
with the FP32 preconditioner at tolerance 1e-10, the open boundary with its recomputations and ramps, the WEDGE
notch, a current ramp) stepped by the device and by the oracle from the same state.

* On a bounded sample of the scheme (64×32×8 cells, 2-cell insulating padding) for 120 steps, two open-boundary
  recomputations included, compared every 10 steps at 1e-7 of each whole vector (the reference's CPU-versus-device
  bar for the PCG paths, gpu/TDGLGPU/test/compare_cpu.jl:69); PCG iterations within one per solve on average.
* At the full 256×128×32 size (8-cell padding) for 3 steps: the large-size code paths (the persistent two-plane
  transform staging, the smooth-size FFT padding, the wide reductions) against the oracle at the same bar.
* The 12×8×4 two-band parity case for 2000 steps at 1e-11, every 100 steps.
* The device's bar-field tables against the host's and the oracle's on a section of 256 cells or more.
"""
import numpy as np
import pytest

import cases
import juliatdgl_b200 as T
from juliatdgl_b200 import gpu, workloads
from juliatdgl_b200.scheme import BarField, _bar_field_device, _bar_field_host
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def oracle_bar(gr):
    return BarField(*pyoracle.bar_field(gr))


def run_pair(st, s, H, hj, q0, n, every):
    o = pyoracle.OracleStepper(st)
    o.upload(s)
    g = gpu.GPUStepper(st)
    g.upload(s)
    a, b = s.copy(), s.copy()
    worst = 0.0
    try:
        for c in range(0, n, every):
            m = min(every, n - c)
            hjs = [hj(q0 + c + i) for i in range(m)]
            assert o.steps_ramp(H, hjs) == 0
            g.steps_ramp(H, hjs)
            o.download(a)
            g.download(b)
            w, per = cases.compare_states(b, a)
            worst = max(worst, w)
            assert w <= 1e-7, (c + m, per)
        so, sg = o.stats(), g.stats()
        return worst, so, sg
    finally:
        g.close()


def test_ramp_sample_matches_the_oracle():
    """The scheme of the 256×128×32 benchmark on 64×32×8 cells, 120 steps from the middle of the ramp (Jx = 0.03 on
    a Meissner seed: the current switches on at once)."""
    st, s, H = workloads.ramp(64, 32, 8, 2, bar_tables=None, bar_backend="numpy")
    hj = workloads.ramp_hj(st, +1)
    assert st.open.every < 60                      # two recomputations fall inside 120 steps
    worst, so, sg = run_pair(st, s, H, hj, 10000, 120, 10)
    assert so.open_recomputes == sg.open_recomputes >= 3
    a, b = so.pcg_total_iters, sg.pcg_total_iters
    assert a > 120 and abs(a - b) <= max(2, a // 50), (a, b)


def test_ramp_sample_negative_polarity_matches_the_oracle():
    st, s, H = workloads.ramp(64, 32, 8, 2, bar_backend="numpy")
    worst, so, sg = run_pair(st, s, H, workloads.ramp_hj(st, -1), 10000, 60, 20)
    assert abs(so.pcg_total_iters - sg.pcg_total_iters) <= max(2, so.pcg_total_iters // 50)


def test_ramp_full_size_matches_the_oracle():
    """3 steps of the full 256×128×32 benchmark scheme (the oracle's bar tables for both sides)."""
    gr = T.Grid.make(256, 128, 32, dx=0.5, buf=8)
    st, s, H = workloads.ramp(bar_tables=oracle_bar(gr))
    hj = workloads.ramp_hj(st, +1)
    worst, so, sg = run_pair(st, s, H, hj, 10000, 3, 1)
    assert so.open_recomputes == sg.open_recomputes
    assert abs(so.pcg_total_iters - sg.pcg_total_iters) <= 1, (so.pcg_total_iters, sg.pcg_total_iters)


def test_config1_2000_steps():
    """The two-band parity case (12×8×4, KWT, RKC + frame, SepSolver, bar field) for the 2000 steps of its
    specification, every 100 steps at 1e-11."""
    st, s, H, HJ = cases.config1()
    o = pyoracle.OracleStepper(st)
    o.upload(s)
    g = gpu.GPUStepper(st)
    g.upload(s)
    a, b = s.copy(), s.copy()
    try:
        for c in range(20):
            o.steps(100, H, HJ)
            g.steps(100, H, HJ)
            o.download(a)
            g.download(b)
            w, per = cases.compare_states(b, a)
            assert w <= 1e-11, ((c + 1) * 100, per)
    finally:
        g.close()


@pytest.mark.parametrize("dims", [(64, 32, 8, 2), (256, 128, 32, 8)])
def test_bar_field_kernel_matches_the_host(dims):
    """tdgl_bar_field (one warp per face point) against the oracle's restatement of field.jl:151-180, and on the
    smaller section against the vectorised host mirror: the same sums in another order."""
    nx, ny, nz, buf = dims
    gr = T.Grid.make(nx, ny, nz, dx=0.5, buf=buf)
    assert (gr.y2 - gr.y1 + 1) * (gr.z2 - gr.z1 + 1) >= 256
    d = _bar_field_device(gr, 8)
    refs = [oracle_bar(gr)] + ([_bar_field_host(gr, 8)] if nx <= 64 else [])
    for ref in refs:
        for name in ("hy_z", "hy_y", "hz_z", "hz_y", "hz_x", "hy_x"):
            x, y = getattr(d, name), getattr(ref, name)
            assert x.shape == y.shape
            assert np.max(np.abs(x - y)) <= 1e-12 * np.max(np.abs(y)), name
