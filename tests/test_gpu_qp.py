"""Normal fluids per band (qp_exchange, gtdgl/src/exchange.jl) on the device: the reference's physical checks of
gtdgl/test/test_physics.jl:338-381 through the C-ABI (the device's steps against the oracle's are in
test_gpu_parity.py's small cases qp_*).

* a fast exchange (ν = 1e6) is the one-fluid step to O(1/ν): 1e-4 after 300 steps;
* in a long strip without Josephson the σ share of the converted current follows the 1D two-fluid law: 0.5664 with
  one fluid, 0.5484 and 0.4567 with ν = 10 and 1.
"""
import numpy as np
import pytest

import juliatdgl_b200 as T
from juliatdgl_b200 import gpu
from juliatdgl_b200.grid import GeomSpec, build_masks
from juliatdgl_b200.state import initial_state
from test_qp_oracle import band_currents, wedge_case

pytestmark = pytest.mark.gpu


def run(st, s, n, H, HJ):
    gs = gpu.GPUStepper(st)
    try:
        gs.upload(s)
        gs.steps(n, H, HJ)
        return gs.download(s)
    finally:
        gs.close()


def test_fast_exchange_is_one_fluid_on_the_device():
    md, gr, mk = wedge_case()
    H = 0.03
    st0 = T.Stepper.make(md, gr, mk)
    HJ = T.selffield(st0, 0.5)
    sa = run(st0, initial_state(md, gr, mk, H), 300, H, HJ)
    sb = run(T.Stepper.make(md, gr, mk, qp_exchange=1e6), initial_state(md, gr, mk, H), 300, H, HJ)
    for mu in range(2):
        assert np.max(np.abs(sa.G[mu] - sb.G[mu])) < 1e-4


def test_strip_follows_the_two_fluid_law_on_the_device():
    md = T.two_band(xi_ratio=4.0, κ=25.0, gamma12=0.0, gamma_kwt=10.0)

    def strip(ν):
        g2 = T.Grid.make(80, 4, 2, dx=0.5)
        m2 = build_masks(GeomSpec(GEOM_MODE="SIM"), g2)
        st = T.Stepper.make(md, g2, m2, qp_exchange=ν)
        s = run(st, initial_state(md, g2, m2, 0.0), int(np.floor(300 / st.dt + 0.5)), 0.0, T.selffield(st, 0.05))
        Ib = band_currents(s, st)
        return Ib[0] / (Ib[0] + Ib[1])

    f_inf, f10, f1 = strip(None), strip(10.0), strip(1.0)
    assert abs(f_inf - 0.5664) <= 0.003 and abs(f10 - 0.5484) <= 0.01 and abs(f1 - 0.4567) <= 0.02, (f_inf, f10, f1)


def test_two_fluids_as_a_matrix_are_the_two_band_model_on_the_device():
    """test_physics.jl:387-395: QPExchangeN with two bands steps as QPExchange (200 steps, 1e-10)."""
    from test_qp_oracle import stiffness
    md, gr, mk = wedge_case()
    H = 0.03
    st0 = T.Stepper.make(md, gr, mk)
    HJ = T.selffield(st0, 0.5)
    s0 = run(st0, initial_state(md, gr, mk, H), 300, H, HJ)
    sa = T.Stepper.make(md, gr, mk, qp_exchange=1.0)
    q2 = sa.qpx
    χ = [q2.s[µ] * md.σn * md.bands[µ].Γ / stiffness(md.bands[µ]) for µ in range(2)]
    sb = T.Stepper.make(md, gr, mk, qp_exchange=[[0.0, 1.0], [χ[0] / χ[1], 0.0]])
    a = run(sa, s0.copy(), 200, H, HJ)
    b = run(sb, s0.copy(), 200, H, HJ)
    for mu in range(2):
        assert np.max(np.abs(a.G[mu] - b.G[mu])) < 1e-10


def test_joule_heat_of_the_fluids_on_the_device():
    """test_physics.jl:672-693 (T8) on the device, and its temperature fields against the oracle's."""
    from test_qp_oracle import heated, matrix_of
    θ0, _ = heated(None, "device")
    θ6, _ = heated(1e6, "device")
    θ1, st1 = heated(1.0, "device")
    assert np.max(np.abs(θ6 - θ0)) < 1e-5 * np.max(θ0)
    assert np.max(θ1) > 1.2 * np.max(θ0)
    θn, _ = heated(matrix_of(st1), "device")
    assert np.max(np.abs(θn - θ1)) < 1e-9 * np.max(θ1)
    θo, _ = heated(1.0, "oracle")
    assert np.max(np.abs(θ1 - θo)) < 1e-10 * np.max(θo)


def test_two_fluids_with_the_insulating_padding_on_the_device():
    """test_physics.jl:633-640 on the device: the strip with the insulating padding, σ share 0.4427 ± 0.01."""
    md = T.two_band(xi_ratio=4.0, κ=25.0, gamma12=0.0, gamma_kwt=10.0)
    g2 = T.Grid.make(80, 4, 2, dx=0.5)
    k2 = build_masks(GeomSpec(GEOM_MODE="SIM"), g2)
    st = T.Stepper.make(md, g2, k2, qp_exchange=1.0, σvac=0.01)
    s = run(st, initial_state(md, g2, k2, 0.0), int(np.floor(300 / st.dt + 0.5)), 0.0, T.selffield(st, 0.05))
    Ib = band_currents(s, st)
    assert abs(Ib[0] / (Ib[0] + Ib[1]) - 0.4427) <= 0.01, Ib


def test_sculpted_sample_counts_its_conjugate_gradients():
    """The δ solve over the cut links of a sculpted sample (QPSolve) runs on the device, its loop a conditional node
    of the captured step: the iterations are counted and stay under the limit."""
    import cases
    st, s, H, HJ = cases.vacuum("vac_qp")
    gs = gpu.GPUStepper(st)
    try:
        gs.upload(s)
        gs.steps(12, H, HJ)
        it = gs.stats().qp_cg_total_iters
    finally:
        gs.close()
    assert 12 <= it < 12 * st.qpx.maxit
