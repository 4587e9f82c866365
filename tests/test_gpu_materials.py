"""Material per region on the device (the material variants of the band stage, the supercurrent and the noise kick)
against the oracle through the C-ABI, and the reference's bit-identity property on the device itself: two regions
of one material step exactly as the uniform run (test_materials.jl:10-21), so the material kernels reduce to the
uniform ones bit for bit.

Tolerances as the uniform paths: 1e-11 whole-vector relative for the exact field solves, 1e-7 for the PCG (σn per
region), 1e-10 with noise.
"""
import numpy as np
import pytest

import cases
import juliatdgl_b200 as T
from juliatdgl_b200 import gpu
from juliatdgl_b200.state import initial_state
from oracle import pyoracle
from test_materials_oracle import same, wedge24

pytestmark = pytest.mark.gpu


def tol_for(st, noisy=False):
    return 1e-7 if st.solver == 3 else (1e-10 if noisy else 1e-11)


def gpu_run(st, s, n, H, HJ):
    gs = gpu.GPUStepper(st)
    try:
        b = s.copy()
        gs.upload(b)
        gs.steps(n, H, HJ)
        return gs.download(b)
    finally:
        gs.close()


@pytest.mark.parametrize("kind", cases.MATERIAL_KINDS)
def test_material_cases(kind):
    st, s, H, HJ = cases.material(kind)
    s = pyoracle.run(st, s, 5, H, HJ)
    a = pyoracle.run(st, s, 20, H, HJ)
    b = gpu_run(st, s, 20, H, HJ)
    worst, per = cases.compare_states(b, a)
    assert worst <= tol_for(st), per


@pytest.mark.parametrize("kind", list(cases.MATERIAL_NOISY))
def test_noisy_material_cases(kind):
    st, s, H, HJ = cases.material(kind, **cases.MATERIAL_NOISY[kind])
    s = pyoracle.run(st, s, 5, H, HJ)
    a = pyoracle.run(st, s, 20, H, HJ)
    b = gpu_run(st, s, 20, H, HJ)
    worst, per = cases.compare_states(b, a)
    assert worst <= tol_for(st, noisy=True), per


def test_absent_band_stays_zero_on_the_device():
    st, s, H, HJ = cases.material("mat_absent")
    b = gpu_run(st, s, 100, H, HJ)
    inN = (st.masks.mat == 2) & (st.masks.τψ > 0)
    assert np.all(b.G[1][inN] == 0) and np.abs(b.G[0][inN]).max() > 0.1


@pytest.mark.parametrize("model,kw", [("plain", {}), ("kwt", {}), ("kwt", dict(noise=1e-3, noise_seed=5))])
def test_one_material_in_two_regions_is_the_uniform_run_on_the_device(model, kw):
    md = {"plain": T.two_band(xi_ratio=4.0, κ=2.0), "kwt": T.two_band(xi_ratio=4.0, κ=2.0, gamma_kwt=10.0)}[model]
    gr, mk, mk2 = wedge24()
    a = T.Stepper.make(md, gr, mk, **kw)
    b = T.Stepper.make(md, gr, mk2, materials=[cases.copy_model(md)], **kw)
    HJ = T.selffield(a, 0.5)
    sa = gpu_run(a, initial_state(md, gr, mk, 0.03), 60, 0.03, HJ)
    sb = gpu_run(b, initial_state(md, gr, mk2, 0.03, materials=b.mt.models), 60, 0.03, HJ)
    assert same(sa, sb)


def test_small_bilayer_matches_the_oracle():
    """The large bilayer's scheme on a small grid: two materials and a barrier, an absent band, masses per axis,
    noise on the bands and the field, the open boundary and the PCG of the insulating buffer, all at once."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    st, s, H, HJ = bench.bilayer_workload(24, 16, 8, 2)
    s = pyoracle.run(st, s, 3, H, HJ)
    a = pyoracle.run(st, s, 12, H, HJ)
    b = gpu_run(st, s, 12, H, HJ)
    worst, per = cases.compare_states(b, a)
    assert worst <= 1e-7, per


# ---- two normal fluids per material (exchange.jl:193-290, QPVar): test_materials.jl:192-219 on the device


def test_two_fluids_with_a_copy_of_the_material_keep_the_bits_on_the_device():
    """test_materials.jl:193-201: with a copy of the material the separable δ solve runs, bit for bit the uniform run."""
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr, mk, mk2 = wedge24()
    a = T.Stepper.make(md, gr, mk, qp_exchange=1.0)
    b = T.Stepper.make(md, gr, mk2, materials=[cases.copy_model(md)], qp_exchange=1.0)
    assert b.qpx.var is None
    HJ = T.selffield(a, 0.5)
    sa = gpu_run(a, initial_state(md, gr, mk, 0.03), 60, 0.03, HJ)
    sb = gpu_run(b, initial_state(md, gr, mk2, 0.03, materials=b.mt.models), 60, 0.03, HJ)
    assert same(sa, sb)


@pytest.mark.parametrize("which", ["rates", "metal"])
def test_two_fluids_per_material_match_the_oracle(which):
    """test_materials.jl:202-219: another exchange rate in one material, or a one-band metal (band 2 absent, δ = 0
    there), take the variable-coefficient δ solve (conjugate gradients, its loop a conditional node of the captured
    step); the device follows the oracle to the PCG tolerance of the other iterative paths."""
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr, mk, mk2 = wedge24()
    if which == "rates":
        st = T.Stepper.make(md, gr, mk2, qp_exchange=1.0, materials=[cases.copy_model(md)], qp_rates=[1.0, 10.0])
        H, J = 0.03, 0.5
    else:
        metal = T.Model.make((T.Band.make(a=-0.5), T.Band.make(m=md.bands[1].m, a=-1.0)), [[0.0, 0.0], [0.0, 0.0]],
                             κ=2.0)
        st = T.Stepper.make(md, gr, mk2, materials=[metal], absent=[[], [2]], qp_exchange=1.0)
        H, J = 0.03, 0.2
    assert st.qpx.var is not None
    HJ = T.selffield(st, J)
    s = pyoracle.run(st, initial_state(md, gr, mk2, H, materials=st.mt.models), 5, H, HJ)
    a = pyoracle.run(st, s, 20, H, HJ)
    gs = gpu.GPUStepper(st)
    try:
        b = s.copy()
        gs.upload(b)
        gs.steps(20, H, HJ)
        gs.download(b)
        it = gs.stats().qp_cg_total_iters
    finally:
        gs.close()
    worst, per = cases.compare_states(b, a)
    assert worst <= 1e-7, per
    assert 20 <= it < 20 * st.qpx.maxit
