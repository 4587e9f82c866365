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
  split along and across Ψ, the phase diffusing s times faster), and the equipartition of the field's free modes
  under the link kick (T9, test_physics.jl:697-737; here its stiff case, the device runs all three).
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


def curl_h(phx, phy, phz, gr):
    """curl_h! (gtdgl/src/field.jl:124-137) on the plaquettes it writes, flattened hx, hy, hz (0-based slices)."""
    Nx, Ny, Nz, dx, dy, dz = gr.Nx, gr.Ny, gr.Nz, gr.dx, gr.dy, gr.dz
    hx = ((phz[1:Nx, 2:Ny, 1:Nz - 1] - phz[1:Nx, 1:Ny - 1, 1:Nz - 1]) - phy[1:Nx, 1:Ny - 1, 2:Nz]
          + phy[1:Nx, 1:Ny - 1, 1:Nz - 1]) / (dy * dz)
    hy = ((phx[1:Nx - 1, 1:Ny, 2:Nz] - phx[1:Nx - 1, 1:Ny, 1:Nz - 1]) - phz[2:Nx, 1:Ny, 1:Nz - 1]
          + phz[1:Nx - 1, 1:Ny, 1:Nz - 1]) / (dz * dx)
    hz = ((phy[2:Nx, 1:Ny - 1, 1:Nz] - phy[1:Nx - 1, 1:Ny - 1, 1:Nz]) - phx[1:Nx - 1, 2:Ny, 1:Nz]
          + phx[1:Nx - 1, 1:Ny - 1, 1:Nz]) / (dx * dy)
    return np.concatenate([hx.ravel(), hy.ravel(), hz.ravel()])


def free_plaquettes(s, gr):
    Nx, Ny, Nz = gr.Nx, gr.Ny, gr.Nz
    return np.concatenate([s.hx[1:Nx, 1:Ny - 1, 1:Nz - 1].ravel(), s.hy[1:Nx - 1, 1:Ny, 1:Nz - 1].ravel(),
                           s.hz[1:Nx - 1, 1:Ny - 1, 1:Nz].ravel()])


def normal_box(κ, σvac, buf):
    """test_physics.jl:703-707: a normal box (f = 0 held by hard masks, Ψ = 0), T̃ = 0.02 on Ψ and the field."""
    md = T.Model.make((T.Band.make(m=1.0, Γ=1.0),), [[0.0]], κ=κ)
    gr = T.Grid.make(6, 4, 4, dx=0.5, buf=buf)
    mk = T.box_masks(gr)
    mk.f[...] = 0.0
    st = T.Stepper.make(md, gr, mk, hard=True, noise=0.02, noise_seed=3, noise_field=True, σvac=σvac)
    s = initial_state(md, gr, mk, 0.0)
    s.G[0][...] = 0
    s.F[0][...] = 0
    return st, s


def equipartition_expected(st):
    """Σ_m (T̃/2)/(1 + λ_m dt/2) over the transverse modes, λ_m = (κ²dx²/σn)·eig(D^{-1/2} CᵀC D^{-1/2}), C the curl
    of curl_h! on every evolving link (test_physics.jl:709-721)."""
    gr, md = st.grid, st.model
    Nx, Ny, Nz = gr.Nx, gr.Ny, gr.Nz
    links = [(0, i, j, k) for k in range(1, Nz) for j in range(1, Ny) for i in range(0, Nx)]
    links += [(1, i, j, k) for k in range(1, Nz) for j in range(0, Ny) for i in range(1, Nx)]
    links += [(2, i, j, k) for k in range(0, Nz) for j in range(1, Ny) for i in range(1, Nx)]
    shapes = (gr.xlink, gr.ylink, gr.zlink)
    cols = []
    for ax, i, j, k in links:
        ph = [np.zeros(sh, order="F") for sh in shapes]
        ph[ax][i, j, k] = 1.0
        cols.append(curl_h(*ph, gr))
    Cm = np.array(cols).T
    Dl = np.ones(len(links)) if st.D is None else np.array([st.D[ax][i, j, k] for ax, i, j, k in links])
    Di = np.diag(1 / np.sqrt(Dl))
    ev = np.linalg.eigvalsh(Di @ (Cm.T @ Cm) @ Di)
    ev = ev[ev > 1e-9 * ev.max()]
    return float(np.sum((st.noise_T / 2) / (1 + (md.κ ** 2 * gr.dx ** 2 / md.σn) * ev * (st.dt / 2))))


def equipartition(stepper, st, s, teq, tav):
    """⟨F_A⟩ / expected over tav after teq (F_A = κ²dx³ Σ h² of the free plaquettes, sampled every 10 steps), and
    max|Ψ| at the end."""
    gr, κ = st.grid, st.model.κ
    stepper.upload(s)
    stepper.steps(round(teq / st.dt), 0.0, 0.0)
    acc, n = 0.0, 0
    for _ in range(round(tav / st.dt) // 10):
        stepper.steps(10, 0.0, 0.0)
        stepper.download(s)
        acc += κ ** 2 * gr.dx ** 3 * np.sum(free_plaquettes(s, gr) ** 2)
        n += 1
    return acc / n / equipartition_expected(st), float(np.abs(s.G[0]).max())


# (κ, σvac, buf, teq, tav) of test_physics.jl:732-734: uniform σn; stiff modes (λdt up to 0.87); σ per link (PCG)
T9_CASES = {"uniform": (0.25, None, 1, 500.0, 3000.0), "stiff": (1.0, None, 1, 100.0, 1000.0),
            "sigma_per_link": (0.25, 0.01, 2, 500.0, 3000.0)}


def test_oracle_field_equipartition_stiff():
    κ, σvac, buf, teq, tav = T9_CASES["stiff"]
    st, s = normal_box(κ, σvac, buf)
    r, psi = equipartition(pyoracle.OracleStepper(st), st, s, teq, tav)
    assert r == pytest.approx(1.0, abs=0.01) and psi == 0
