"""Thermal noise on the device (noise.cu and the noisy paths of bands.cu) against the oracle.

Both draw the same counter-based normals (Philox4x32-10 on {node, step, stream} under the seed), so the noisy step
is compared like the deterministic one: per step, whole-vector relative, 1e-10 for the exact field solves (the
Box–Muller log/sincos and the rotations round differently in CUDA's and the host's libm, and the noise feeds those
ulps on) and 1e-7 for the PCG paths.  The statistical contract of the reference's own tests
(gtdgl/test/test_physics.jl:475-537) is then checked on the device itself, and the resumability of the streams
(the draws of step q depend on q only, not on how the run was split into calls or contexts).
"""
import dataclasses

import numpy as np
import pytest

import cases
from juliatdgl_b200 import gpu
from oracle import pyoracle
from test_noise_oracle import (T9_CASES, check_decoupled, check_kwt, decoupled, equilibrium_decoupled, equilibrium_kwt,
                               equipartition, normal_box)

pytestmark = pytest.mark.gpu


def tol_for(st):
    return 1e-7 if st.solver == 3 else 1e-10


@pytest.mark.parametrize("kind", list(cases.NOISY))
def test_noisy_step_matches_the_oracle(kind):
    st, s, H, HJ = cases.small(kind, **cases.NOISY[kind])
    s = pyoracle.run(st, s, 5, H, HJ)
    o = pyoracle.OracleStepper(st)
    o.upload(s)
    gs = gpu.GPUStepper(st)
    try:
        gs.upload(s)
        a, b = s.copy(), s.copy()
        for q in range(4):
            o.steps(5, H, HJ)
            gs.steps(5, H, HJ)
            o.download(a)
            gs.download(b)
            w, per = cases.compare_states(b, a)
            assert w <= tol_for(st), (q, per)
        # the noise did something: the same steps without it land elsewhere
        quiet = dataclasses.replace(st, noise_T=None, noise_field=False)
        c = pyoracle.run(quiet, s, 20, H, HJ)
        assert cases.compare_states(c, a)[0] > 1e-6
    finally:
        gs.close()


def test_streams_resume_across_contexts():
    """20 steps in one context equal 10 + 10 in two, the second started with noise_step0 = 10 and the carry."""
    st, s, H, HJ = cases.small("three_bands", **cases.NOISY["three_bands"])
    one = gpu.GPUStepper(st)
    a = s.copy()
    one.upload(a)
    one.steps(10, H, HJ)
    mid = one.download(s.copy())
    carry = one.get_carry()
    one.steps(10, H, HJ)
    one.download(a)
    one.close()
    two = gpu.GPUStepper(dataclasses.replace(st, noise_step0=10))
    b = mid.copy()
    two.upload(b)
    two.set_carry(carry)
    two.steps(10, H, HJ)
    two.download(b)
    two.close()
    assert cases.compare_states(b, a)[0] == 0.0


def test_seed_selects_the_stream():
    st, s, H, HJ = cases.small("euler_substeps", **cases.NOISY["euler_substeps"])
    out = []
    for seed in (7, 7, 8):
        gs = gpu.GPUStepper(dataclasses.replace(st, noise_seed=seed))
        b = s.copy()
        gs.upload(b)
        gs.steps(3, H, HJ)
        out.append(gs.download(b))
        gs.close()
    assert cases.compare_states(out[0], out[1])[0] == 0.0
    assert cases.compare_states(out[0], out[2])[0] > 1e-6


def test_device_equilibrium_of_decoupled_nodes():
    st, s = decoupled(11)
    gs = gpu.GPUStepper(st)
    try:
        check_decoupled(st, *equilibrium_decoupled(gs, st, s))
    finally:
        gs.close()


def test_device_equilibrium_with_kwt():
    st, s = decoupled(5, γk=3.0)
    gs = gpu.GPUStepper(st)
    try:
        check_kwt(st, *equilibrium_kwt(gs, st, s))
    finally:
        gs.close()


@pytest.mark.parametrize("case", list(T9_CASES))
def test_device_field_equipartition(case):
    κ, σvac, buf, teq, tav = T9_CASES[case]
    st, s = normal_box(κ, σvac, buf)
    gs = gpu.GPUStepper(st)
    try:
        r, psi = equipartition(gs, st, s, teq, tav)
    finally:
        gs.close()
    assert r == pytest.approx(1.0, abs=0.01) and psi == 0
