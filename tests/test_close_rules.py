"""The close rules of a ladder point (juliatdgl_b200/protocol.py, as gtdgl/src/protocol.jl:193-209, 466-490) on the
reference's own cases (gtdgl/test/test_protocol.jl:50-58: a slow flow whose last slip fell in the first half is not a
fixed point; the static phase change of a current step is silent) and on constructed series for 'F' and 'V'."""
import math

import numpy as np

from juliatdgl_b200 import protocol as P

TWO_PI = 2 * math.pi


def test_the_reference_cases():
    m, dt_cyc = 500, 0.8
    T1 = [0.0 if k < 150 else -TWO_PI for k in range(1, m + 1)]   # one crossing per line at cycle 150
    Tm1 = np.full((3, 2), -TWO_PI, order="F")
    ok = np.ones((3, 2), dtype=bool, order="F")
    assert P.crossings_now(T1, Tm1, ok, m, dt_cyc) < 0.5
    assert not P.silent_now(T1, Tm1, ok, m, dt_cyc, 0.5)
    T0 = [0.3 * (1 - math.exp(-k / 20)) for k in range(1, m + 1)]   # the static phase change of a current step
    assert P.silent_now(T0, np.full((3, 2), 0.3, order="F"), ok, m, dt_cyc, 0.5)


def test_fixed_point_and_resistive_closes():
    m, dt_cyc = 600, 0.5
    ok = np.ones((2, 2), dtype=bool, order="F")
    kw = dict(dt_cyc=dt_cyc, iter_min=100, it_res_min=200, nwin=50, eps=1e-6, noisy=False)
    quiet = [np.full(m, 0.1)]
    assert P.close_point(m, quiet, [np.full((2, 2), 0.1)], ok, [1e-8], 1e-8, 0.3, **kw) == ("F", None)
    assert P.close_point(m, quiet, [np.full((2, 2), 0.1)], ok, [1e-3], 1e-8, 0.3, **kw) == (None, None)
    # a steady flow of 30 crossings over the point: a plateau and ≥ 10 crossings by the slope
    flow = [np.linspace(0.0, -30 * TWO_PI, m)]
    assert P.close_point(m, flow, [np.full((2, 2), -30 * TWO_PI)], ok, [1e-3], 1e-3, 0.3, **kw) == ("V", 0)
    assert P.close_point(m, flow, [np.full((2, 2), -30 * TWO_PI)], ok, [1e-3], 1e-3, 0.0, **kw) == (None, None)
    # with noise: a silent rung closes after it_res_min cycles
    noisy = dict(kw, noisy=True)
    assert P.close_point(m, quiet, [np.full((2, 2), 0.1)], ok, [0.2], 0.2, 0.3, **noisy) == ("F", None)
    assert P.close_point(150, quiet, [np.full((2, 2), 0.1)], ok, [0.2], 0.2, 0.3, **noisy) == (None, None)


def test_a_sample_gone_normal_closes_N():
    # the largest 'F' so far holds ⟨|Ψ₁|²⟩ = 0.8; a later fixed point at 0.01 < 0.02 × 0.8 is normal
    v, last = P.normal_verdict("F", 0.3, 0.8, 0.0)
    assert (v, last) == ("F", 0.8)
    assert P.normal_verdict("F", 0.9, 0.01, last) == ("N", 0.8)
    assert P.normal_verdict("F", 0.0, 0.01, last) == ("F", 0.8)     # at J = 0 a fixed point stays 'F'
    assert P.normal_verdict("V", 0.9, 0.01, last) == ("V", 0.8)
