"""The cycle observables on the device (tdgl_meter_set / tdgl_measure / tdgl_vortices) against the oracle's restatement
of gtdgl's measurement functions (oracle/observables.py), on states stepped on the GPU and downloaded.

Maxima are taken in exact arithmetic in any order: max|Δh_z| must agree to the bit, and the per-band residual
max| |Ψ| − |Ψ|prev | and max|Ψ| to the few ulps of |Ψ| ≈ 1 by which CUDA's hypot may differ from the host's (1e-15
absolute); sums (plane sums, θ_A, the midplane current) and path phases to 1e-12 relative (fixed-order device
reductions against sequential sums, CUDA's atan2 against the host's); vortex counts exactly.
"""
import math

import numpy as np
import pytest

import cases
from juliatdgl_b200 import gpu, protocol
from oracle import observables as ob

pytestmark = pytest.mark.gpu


def _close(a, b, rtol=1e-12, atol=1e-14):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.all(np.abs(a - b) <= atol + rtol * np.maximum(1.0, np.abs(b)))


@pytest.mark.parametrize("kind", ["three_bands", "open_pcg", "rkc_kwt_rotframe"])
def test_cycle_observables_match_the_oracle(kind):
    st, s, H, HJ = cases.small(kind)
    gr, mk, N = st.grid, st.masks, st.model.N
    gs = gpu.GPUStepper(st)
    try:
        gs.upload(s)
        gs.steps(8, H, HJ)
        vm = protocol.voltmeter(gr, mk, delta_v=2)
        gs.meter_set(vm)
        s0 = gs.download(s.copy())
        cooper0 = [ob.block_abs(s0.G[mu], gr) for mu in range(N)]
        hz0 = s0.hz.copy()
        for cyc in range(2):
            gs.steps(5, H, HJ)
            o = gs.measure()
            s1 = gs.download(s.copy())
            for mu in range(N):
                D = ob.path_phase(s1.G[mu], s1.Vx, gr, vm.vi, vm.vo)
                assert _close(o["D"][mu], D), (cyc, mu)
                r, a = ob.cooper_residual(s1.F[mu], cooper0[mu], gr)
                assert o["res"][mu] == pytest.approx(r, rel=0, abs=1e-15)
                cooper0[mu] = a
            assert o["amax"] == pytest.approx(max(ob.nanmax(ob.block_abs(s1.F[mu], gr)) for mu in range(N)), rel=1e-15)
            assert all(math.isfinite(r) for r in o["res"]) and math.isfinite(o["amax"])
            assert o["diffh"] == ob.nanmax(np.abs(s1.hz - hz0))
            hz0 = s1.hz.copy()
            assert _close(o["vsum_in"], ob.plane_sum(s1.φx, gr, vm.vi, vm.Min))
            assert _close(o["vsum_out"], ob.plane_sum(s1.φx, gr, vm.vo, vm.Mou))
            assert _close(o["ta_sum"], ob.theta_A_sum(s1.φx, gr, vm.vi, vm.vo, vm.line_ok))
            it, isam = ob.midplane_current(s1.hy, s1.hz, gr, st.model.κ ** 2)
            assert _close(o["Itot"], it) and _close(o["Isam"], isam)
            kc = int(math.floor((gr.z1 + gr.z2) / 2 + 0.5))
            for mu in range(N):
                Nv, nmap, Nl, lok = gs.vortices(mu, kc, with_map=True)
                eNv, emap, eNl, elok = ob.count_vortices(s1.F[mu], s1.Vx, s1.Vy, s1.hz, mk.f, gr, kc)
                assert (Nv, Nl, lok) == (eNv, eNl, elok)
                assert np.array_equal(nmap, emap)
    finally:
        gs.close()


def test_crossing_times_follow_the_host_replay():
    """crossing_times on the device against the same integration replayed (fresh context) with the path phases
    computed on the host from downloaded states."""
    st, s, H, HJ = cases.small("three_bands")
    J = 0.3
    gs = gpu.GPUStepper(st)
    try:
        gs.upload(s)
        trace = []
        times, t, div = protocol.crossing_times(gs, st, J, H=H, T=60 * st.dt, stop=0, delta_v=2, every=10,
                                                trace=trace)
        assert not div and t == pytest.approx(60 * st.dt) and len(trace) == 6
    finally:
        gs.close()
    gs = gpu.GPUStepper(st)
    try:
        gs.upload(s)
        vm = protocol.voltmeter(st.grid, st.masks, 2)
        HJ = protocol.selffield(st, J)
        Dp = ob.path_phase(s.G[0], s.Vx, st.grid, vm.vi, vm.vo)
        acc = np.zeros_like(Dp)
        for q in range(6):
            gs.steps(10, H, HJ)
            s1 = gs.download(s.copy())
            protocol.unwrap(acc, ob.path_phase(s1.G[0], s1.Vx, st.grid, vm.vi, vm.vo), Dp)
            assert trace[q] == pytest.approx(protocol.line_mean(acc, vm.line_ok), rel=1e-10, abs=1e-12)
    finally:
        gs.close()


def test_meter_refuses_a_bad_voltmeter():
    st, s, H, HJ = cases.small("euler_substeps")
    gs = gpu.GPUStepper(st)
    try:
        gs.upload(s)
        vm = protocol.voltmeter(st.grid, st.masks, delta_v=2)
        vm.vo = st.grid.x2 + 3
        with pytest.raises(gpu.TDGLError):
            gs.meter_set(vm)
    finally:
        gs.close()
