"""The reference's analytic checks of the KWT relaxation and the three-band ground state, on the oracle and on the
device.

* gtdgl/test/test_physics.jl:50-59: kwt_update solves w + γ²ψ Re(ψ* w) = √(1+γ²|ψ|²) R/Γ (a 2×2 real system), also
  near ψ = 0, to 1e-12.
* :60-72: a uniform amplitude perturbation decays at 2ψ₀²/(u√(1+γ²ψ₀²)), u = Γ/σn: 2.000, 0.3454, 0.03437 for
  (u, γ) = (1, 0), (5.79, 0), (5.79, 10), within 2e-3 (explicit Euler: a factor 1 − λ dt per step).
* :325-338: three identical bands with equal repulsive couplings break time reversal: phases 0, ±2π/3 of one
  chirality and |Ψ|² = 1 + |γ| in each band, to 1e-6, after 200 t_GL from unequal starting phases.
These pin the KWT, RKC and three-band branches of the step that the 256×128×32 ramp runs, which have no stored
golden state in the reference.
"""
import cmath
import math

import numpy as np
import pytest

import juliatdgl_b200 as T
from oracle import pyoracle


def test_kwt_local_step_solves_the_linear_system():
    for psi, R, γ in ((0.7 + 0.2j, 0.3 - 0.1j, 10.0), (1e-9 + 0j, 0.2 + 0.4j, 10.0), (0.4 - 0.9j, -0.5 + 0.05j, 2.0)):
        dt = 0.01
        w = (pyoracle.kwt_update(psi, dt * R, γ ** 2) - psi) / dt
        q = 1 + γ ** 2 * abs(psi) ** 2
        M = np.array([[1 + γ ** 2 * psi.real ** 2, γ ** 2 * psi.real * psi.imag],
                      [γ ** 2 * psi.real * psi.imag, 1 + γ ** 2 * psi.imag ** 2]])
        x = np.linalg.solve(M, math.sqrt(q) * np.array([R.real, R.imag]))
        assert abs(w - complex(x[0], x[1])) <= 1e-12 * abs(complex(x[0], x[1]))


class _Oracle:
    def __init__(self, st):
        self.c = pyoracle.OracleStepper(st)

    def step(self, s, n, H=0.0, HJ=0.0):
        self.c.upload(s)
        assert self.c.steps(n, H, HJ) == 0
        return self.c.download(s)


class _Device:
    def __init__(self, st):
        from juliatdgl_b200 import gpu
        self.c = gpu.GPUStepper(st)

    def step(self, s, n, H=0.0, HJ=0.0):
        self.c.upload(s)
        self.c.steps(n, H, HJ)
        return self.c.download(s)


def _decay_rates(Impl):
    for u, γ, rate in ((1.0, 0.0, 2.0), (5.79, 0.0, 0.3454), (5.79, 10.0, 0.03437)):
        md = T.Model.make((T.Band.make(Γ=u, γkwt=γ),), [[0.0]], κ=2.0)
        gr = T.Grid.make(8, 6, 4, dx=0.5)
        mk = T.box_masks(gr)
        st = T.Stepper.make(md, gr, mk, rkl=False)
        s = T.initial_state(md, gr, mk, 0.0)
        s.G[0][...] *= (1 + 1e-6)
        i, j, k = 5, 4, 3                 # Julia's (6, 5, 4)
        impl = Impl(st)
        impl.step(s, 1)
        d1 = abs(s.G[0][i, j, k]) - 1
        impl.step(s, 1)
        d2 = abs(s.G[0][i, j, k]) - 1
        assert math.isclose((1 - d2 / d1) / st.dt, rate, rel_tol=2e-3), (u, γ, (1 - d2 / d1) / st.dt)


def test_kwt_amplitude_decay_rates():
    _decay_rates(_Oracle)


@pytest.mark.gpu
def test_kwt_amplitude_decay_rates_on_the_device():
    _decay_rates(_Device)


def _trsb(Impl):
    γ = -0.1
    md = T.Model.make((T.Band.make(), T.Band.make(), T.Band.make()), [[0.0, γ, γ], [γ, 0.0, γ], [γ, γ, 0.0]], κ=25.0)
    gr = T.Grid.make(8, 8, 4, dx=0.5)
    mk = T.box_masks(gr)
    st = T.Stepper.make(md, gr, mk)
    s = T.initial_state(md, gr, mk, 0.0)
    s.G[1][...] *= cmath.exp(1j * 1.0)
    s.G[2][...] *= cmath.exp(1j * 2.5)
    Impl(st).step(s, round(200 / st.dt))
    c = ((gr.x1 + gr.x2 + 1) // 2 - 1, (gr.y1 + gr.y2 + 1) // 2 - 1, (gr.z1 + gr.z2 + 1) // 2 - 1)
    psi = [s.G[µ][c] for µ in range(3)]
    a2 = cmath.phase(psi[1] / psi[0])
    a3 = cmath.phase(psi[2] / psi[0])
    assert abs(abs(a2) - 2 * math.pi / 3) < 1e-6 and abs(abs(a3) - 2 * math.pi / 3) < 1e-6
    assert a2 * a3 < 0                     # one chirality, not 0 and π
    assert all(abs(abs(x) ** 2 - (1 + abs(γ))) < 1e-6 for x in psi)


def test_three_frustrated_bands_reach_the_trsb_state():
    _trsb(_Oracle)


@pytest.mark.gpu
def test_three_frustrated_bands_reach_the_trsb_state_on_the_device():
    _trsb(_Device)
