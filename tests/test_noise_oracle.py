"""The oracle's thermal noise against published answers and the reference's own statistical contract.

The reference draws its Langevin noise from Julia's Xoshiro stream in a fixed loop order (gtdgl/src/noise.jl:28-35);
a parallel device cannot reproduce that sequence, so both the oracle and the CUDA path draw from a counter-based
generator instead — Philox4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy as 1, 2, 3",
SC'11) keyed by the seed, with the counter {node, step (2 words), stream} — and the draws themselves are not
comparable with the reference's.  What is pinned here:

* the generator: the three known-answer vectors published with Philox4x32-10 (zero, all-ones and the digits of π);
* the normals: Box–Muller on two 53-bit uniforms — moments and independence of the pair;
* the physics: the reference's own tests of the noise (gtdgl/test/test_physics.jl:475-537) run on the oracle with
  the same models, grids, steps, lags and tolerances — the exact equilibrium of decoupled nodes (mean and variance
  of |Ψ|² with the Euler–Maruyama bias, the time correlation of the amplitude) without and with KWT (the mobility
  split along and across Ψ, the phase diffusing s times faster).
"""
import ctypes as C
import math

import numpy as np
import pytest

import juliatdgl_b200 as T
from juliatdgl_b200.state import initial_state
from oracle import pyoracle

# (counter, key) -> output, as published with the Philox4x32-10 reference implementation
PHILOX_KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff), (0xffffffff, 0xffffffff),
     (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(ctr, key, want):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    pyoracle.lib().oracle_philox4x32_10(c, k)
    assert tuple(c) == want


def normals(seed, step, stream, node0, n):
    L = pyoracle.lib()
    L.oracle_normals.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_int, C.POINTER(C.c_double)]
    out = np.zeros(2 * n)
    L.oracle_normals(seed, step, stream, node0, n, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out[0::2], out[1::2]


def test_normal_pairs_are_standard_and_independent():
    n = 1 << 20
    a, b = normals(7, 3, 1, 0, n)
    z = np.concatenate([a, b])
    se = 1 / math.sqrt(z.size)
    assert abs(z.mean()) < 5 * se
    assert abs(z.var() - 1) < 5 * math.sqrt(2) * se
    assert abs((z ** 3).mean()) < 5 * math.sqrt(15) * se
    assert abs((z ** 4).mean() - 3) < 5 * math.sqrt(96) * se
    assert abs(np.mean(a * b)) < 5 * se
    # neighbouring counters (node, step, stream, seed) give uncorrelated draws
    for other in (normals(7, 3, 1, 1, n)[0], normals(7, 4, 1, 0, n)[0], normals(7, 3, 2, 0, n)[0],
                  normals(8, 3, 1, 0, n)[0]):
        assert abs(np.mean(a * other)) < 5 * se
    assert np.all(np.isfinite(z)) and np.abs(z).max() < 8.6    # |z| ≤ √(−2 ln 2⁻⁵³)


def decoupled(seed, γk=0.0):
    """One band of m = 10⁸ (the nodes decouple), Γ = 2, T̃ = 0.01 on 10×10×2 cells (test_physics.jl:479-483)."""
    md = T.Model.make((T.Band.make(m=1e8, Γ=2.0, γkwt=γk),), [[0.0]], κ=2.0)
    gr = T.Grid.make(10, 10, 2, dx=0.5)
    mk = T.box_masks(gr)
    st = T.Stepper.make(md, gr, mk, dt_scale=0.02, noise=0.01, noise_seed=seed)
    s = initial_state(md, gr, mk, 0.0)
    return st, s


def interior(s, gr):
    return s.G[0][gr.x1:gr.x2, gr.y1:gr.y2, gr.z1:gr.z2]


def equilibrium_decoupled(stepper, st, s):
    """test_physics.jl:484-496 on `stepper` (the oracle or the device): (mean, var, lag correlation) of |Ψ|²."""
    gr, Γ, Tn = st.grid, 2.0, st.noise_T
    lag = round(Γ / 4 / st.dt)
    stepper.upload(s)
    stepper.steps(round(20 / st.dt), 0.0, 0.0)

    def n():
        stepper.download(s)
        return np.abs(interior(s, gr)).ravel() ** 2

    sm = s2 = c = 0.0
    N = 0
    prev = n()
    for q in range(round(1500 / (lag * st.dt))):
        stepper.steps(lag, 0.0, 0.0)
        x = n()
        sm += x.sum()
        s2 += (x * x).sum()
        c += ((x - 1) * (prev - 1)).sum()
        N += x.size
        prev = x
    mean = sm / N
    var = s2 / N - mean ** 2
    return mean, var, (c / N) / var


def equilibrium_kwt(stepper, st, s):
    """test_physics.jl:508-536: (mean, var of |Ψ|², phase correlation at lagp, amplitude correlation at lagn)."""
    gr, Γ, Tn = st.grid, 2.0, st.noise_T
    sk = math.sqrt(1 + 3.0 ** 2)
    dV = gr.dx * gr.dy * gr.dz
    stepper.upload(s)
    stepper.steps(round(40 / st.dt), 0.0, 0.0)

    def g():
        stepper.download(s)
        return interior(s, gr).copy()

    lagn = round(Γ * sk / 4 / st.dt)
    lagp = round(2 * Γ * dV / (Tn * sk) * 0.5 / st.dt)
    sm = s2 = cp = 0.0
    N = Np = 0
    prev, since, q, nst = g(), 0, 0, round(3000 / st.dt)
    while q < nst:
        d = min(lagn - since % lagn, lagp - since, nst - q)      # to the next sample of either kind
        stepper.steps(d, 0.0, 0.0)
        q += d
        since += d
        if since % lagn == 0 or since == lagp:
            x = g()
        if since % lagn == 0:
            a2 = np.abs(x) ** 2
            sm += a2.sum()
            s2 += (a2 * a2).sum()
            N += a2.size
        if since == lagp:
            cp += (np.real(x * np.conj(prev)) / (np.abs(x) * np.abs(prev))).sum()
            Np += x.size
            prev, since = x, 0
    xs, ys = [], []
    for _ in range(400):
        a = np.abs(g()) ** 2
        stepper.steps(lagn, 0.0, 0.0)
        b = np.abs(g()) ** 2
        xs.append(a.ravel() - 1)
        ys.append(b.ravel() - 1)
    xs, ys = np.concatenate(xs), np.concatenate(ys)
    mean = sm / N
    return mean, s2 / N - mean ** 2, cp / Np, (xs * ys).sum() / (xs * xs).sum()


def check_decoupled(st, mean, var, rho):
    dV = st.grid.dx * st.grid.dy * st.grid.dz
    assert mean == pytest.approx(1.0, abs=0.01)
    assert var == pytest.approx(st.noise_T / dV / (1 - st.dt / 2.0), rel=0.04)
    assert rho == pytest.approx(math.exp(-0.5), abs=0.03)


def check_kwt(st, mean, var, cphase, camp):
    dV = st.grid.dx * st.grid.dy * st.grid.dz
    assert mean == pytest.approx(1.0, abs=0.01)
    assert var == pytest.approx(st.noise_T / dV, rel=0.06)
    assert cphase == pytest.approx(math.exp(-0.5), abs=0.03)
    assert camp == pytest.approx(math.exp(-0.5), abs=0.04)


def test_oracle_equilibrium_of_decoupled_nodes():
    st, s = decoupled(11)
    check_decoupled(st, *equilibrium_decoupled(pyoracle.OracleStepper(st), st, s))


def test_oracle_equilibrium_with_kwt():
    st, s = decoupled(5, γk=3.0)
    assert st.rotframe and st.rkc is not None
    check_kwt(st, *equilibrium_kwt(pyoracle.OracleStepper(st), st, s))
