"""The temporal link rotations near 0 and ±π on the reference's manufactured links.

The inputs restate gtdgl/test/rotation_fixture.jl:4-20 (93 link phases: 0, ±π, ±0.02, ±0.4 and the branch points
of the short series ±0.05 and ±asin 0.05, each nudged by ±1e-9 and taken at three moduli 1, 1 ± 2.6e-7).  The
checks are gtdgl/test/test_link_rotations.jl:5-29 on the oracle, and gpu/TDGLGPU/test/test_link_rotations.jl:12-60
on the device: the device formulas against the oracle's within 1e-13 (a different branch of the short series near
its cutoff would differ by ~1e-7, not a few ulps).
"""
import math

import numpy as np
import pytest

from oracle import pyoracle


def fixture():
    """gtdgl/test/rotation_fixture.jl:4-20."""
    angles = [0.0, math.pi, -math.pi, 0.02, -0.02, 0.4, -0.4]
    for t in (0.05, math.asin(0.05), math.pi - 0.05, math.pi - math.asin(0.05)):
        for s in (-1, 1):
            for d in (-1e-9, 0.0, 1e-9):
                angles.append(s * t + d)
    angles = sorted(set(angles))
    scales = (1.0, 1 - 2.6e-7, 1 + 2.6e-7)
    ph = [a for r in scales for a in angles]
    sc = [r for r in scales for a in angles]
    n = len(ph)
    ph.append(ph[-1])
    sc.append(sc[-1])
    V = np.ones((n + 1, 2, 2), dtype=np.complex128, order="F")
    U = np.zeros((n + 1, 2, 2), dtype=np.complex128, order="F")
    om = np.zeros((n + 1, 2, 2), order="F")
    for i in range(n + 1):
        for j in range(2):
            for k in range(2):
                U[i, j, k] = sc[i] * complex(math.cos(-ph[i]), math.sin(-ph[i]))
                om[i, j, k] = (i + 1) / 64 + (j + 1) / 32 - (k + 1) / 16
    q = V * np.conj(U)
    phase = np.arctan2(q.imag, q.real)
    ranges = ((1, n, 1, 2, 1, 2), (1, n + 1, 1, 1, 1, 2), (1, n + 1, 1, 2, 1, 1))
    return dict(V=V, U=U, omega=om, phase=phase, n=n, ranges=ranges, dt=1 / 32)


def cis(x):
    return np.cos(x) + 1j * np.sin(x)


def mask(shape, rng):
    m = np.zeros(shape, dtype=bool)
    i0, i1, j0, j1, k0, k1 = rng
    m[i0 - 1:i1, j0 - 1:j1, k0 - 1:k1] = True
    return m


def all_rng(f):
    return (1, f["n"] + 1, 1, 2, 1, 2)


def test_fixture_has_93_inputs():
    assert fixture()["n"] == 93


def _check_rotations(rot):
    """test_link_rotations.jl:5-28 on one implementation (rot = pyoracle.link_rotations or the device's)."""
    f = fixture()
    V, U, phase = f["V"], f["U"], f["phase"]
    large = np.abs(phase) > 0.1
    for c in (0.25, 0.5, 0.9, 1.0):
        L = rot(1, V, U, all_rng(f), c)
        ref = V * cis(c * phase)
        assert np.max(np.abs(L - ref)) < 4e-7
        assert np.max(np.abs(L - ref)[large]) < 2e-14
        assert np.max(np.abs(np.abs(L) - 1)) < 3e-7
    for n in (2, 5, 9):
        L, R = rot(0, V, U, all_rng(f), n)
        ref = cis(phase / n)
        assert np.array_equal(L, V)
        assert np.max(np.abs(R - ref)) < 4e-8
        assert np.max(np.abs(R - ref)[large]) < 2e-14
    for ax, rng in enumerate(f["ranges"]):
        R = rot(2, V, U, rng, f["dt"], ax=ax, Om=f["omega"])
        m = mask(V.shape, rng)
        om = f["omega"]
        sh = np.zeros_like(om)
        sl = [slice(None)] * 3
        sl[ax] = slice(0, -1)
        src = [slice(None)] * 3
        src[ax] = slice(1, None)
        sh[tuple(sl)] = om[tuple(src)]
        expected = phase + (sh - om) * f["dt"]
        err = np.abs(R - expected)
        assert np.max(err[m]) < 4e-8
        assert np.max(err[m & large]) < 2e-14


def test_oracle_rotations_near_zero_and_pi():
    _check_rotations(pyoracle.link_rotations)


def test_oracle_short_cis():
    """test_link_rotations.jl:29: the series e^{ia} at its cutoff is within 2.605e-7 of cis."""
    assert abs(pyoracle.cis_short(0.05) - complex(math.cos(0.05), math.sin(0.05))) < 2.605e-7


@pytest.mark.gpu
def test_device_rotations_near_zero_and_pi():
    from juliatdgl_b200 import gpu
    _check_rotations(gpu.link_rotations)


@pytest.mark.gpu
def test_device_rotations_match_the_oracle():
    """gpu/TDGLGPU/test/test_link_rotations.jl:12-18: device against CPU within 1e-13, every input and range."""
    from juliatdgl_b200 import gpu
    f = fixture()
    V, U = f["V"], f["U"]
    for c in (0.25, 0.5, 0.9, 1.0):
        a = gpu.link_rotations(1, V, U, all_rng(f), c)
        b = pyoracle.link_rotations(1, V, U, all_rng(f), c)
        assert np.max(np.abs(a - b)) < 1e-13
    for n in (2, 5, 9):
        (La, Ra), (Lb, Rb) = gpu.link_rotations(0, V, U, all_rng(f), n), pyoracle.link_rotations(0, V, U, all_rng(f), n)
        assert np.array_equal(La, Lb) and np.max(np.abs(Ra - Rb)) < 1e-13
    for ax, rng in enumerate(f["ranges"]):
        a = gpu.link_rotations(2, V, U, rng, f["dt"], ax=ax, Om=f["omega"])
        b = pyoracle.link_rotations(2, V, U, rng, f["dt"], ax=ax, Om=f["omega"])
        assert np.max(np.abs(a - b)) < 1e-13
