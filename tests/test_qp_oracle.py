"""Normal fluids per band (qp_exchange, gtdgl/src/exchange.jl) on the oracle: the reference's own checks of
gtdgl/test/test_physics.jl:338-433.

* the shares and the exchange conductance of the dirty split: s_σ = 1/(1 + 16·0.59), G = s_σ ν; dt unchanged;
* the δ solve is exact: σn∇²δ − λ0 δ = S on the unknown nodes (mirror ghosts on y, z; δ = 0 on the x faces) to
  1e-11, with |S| > 0.1, on the state of 300 one-fluid steps;
* a fast exchange (ν = 1e6) is the one-fluid step to O(1/ν): 1e-4 after 300 steps;
* in a long strip without Josephson the σ share of the converted current follows the 1D two-fluid law: 0.5664 with
  one fluid, 0.5484 and 0.4567 with ν = 10 and 1;
* N fluids (a matrix of rates): with two bands the two-band model (μ_π − μ_σ = δ to 1e-12, 200 steps to 1e-10); with
  three the gauge Σ s_µμ_µ = 0, each μ_µ solving σn∇²μ − S⁻¹Lμ = S⁻¹C − 𝟙ΣC to 1e-10 with a different conductance
  per pair, a fast exchange equal to one fluid to 1e-4, and the refusals (no detailed balance; a number for three
  bands);
* the Joule heat of the fluids (test_physics.jl:672-693, T8): with the heat model's Joule term a fast exchange heats as
  one fluid (1e-5 of the maximum), ν = 1 heats more (above 1.2 times), and two bands as a matrix heat as the
  two-band model.
"""
import numpy as np
import pytest

import juliatdgl_b200 as T
from juliatdgl_b200.grid import GeomSpec, build_masks
from juliatdgl_b200.model import stiffness
from juliatdgl_b200.state import initial_state
from oracle import pyoracle


def wedge_case():
    md = T.two_band(xi_ratio=4.0, κ=25.0)
    gr = T.Grid.make(24, 12, 4, dx=0.5)
    mk = build_masks(GeomSpec(GEOM_MODE="WEDGE", inj_margin=4), gr)
    return md, gr, mk


def run(st, s, n, H, HJ):
    c = pyoracle.OracleStepper(st)
    c.upload(s)
    assert c.steps(n, H, HJ) == 0
    return c.download(s), c


def conv(s, mk, md, gr, mu, i, j, k, dragν=None):
    """_conv of band µ at the 1-based node (i, j, k) (exchange.jl:303-335), the reference test's form; with the drag
    matrix dragν its share, the links of band µ carrying the other band (exchange.jl:327-332)."""
    P = s.G[mu]
    Q = s.G[1 - mu]
    p = np.conj(P[i - 1, j - 1, k - 1])
    g = [stiffness(md.bands[mu], a) for a in (1, 2, 3)]
    r2 = 1 / gr.dx ** 2

    def im(z):
        return z.imag

    ax = (mk.τx[i - 1, j - 1, k - 1] * im(p * s.Vx[i - 1, j - 1, k - 1] * P[i, j - 1, k - 1]) +
          mk.τx[i - 2, j - 1, k - 1] * im(p * np.conj(s.Vx[i - 2, j - 1, k - 1]) * P[i - 2, j - 1, k - 1]))
    ay = (mk.τy[i - 1, j - 1, k - 1] * im(p * s.Vy[i - 1, j - 1, k - 1] * P[i - 1, j, k - 1]) +
          mk.τy[i - 1, j - 2, k - 1] * im(p * np.conj(s.Vy[i - 1, j - 2, k - 1]) * P[i - 1, j - 2, k - 1]))
    az = (mk.τz[i - 1, j - 1, k - 1] * im(p * s.Vz[i - 1, j - 1, k - 1] * P[i - 1, j - 1, k]) +
          mk.τz[i - 1, j - 1, k - 2] * im(p * np.conj(s.Vz[i - 1, j - 1, k - 2]) * P[i - 1, j - 1, k - 2]))
    c = ((g[0] * ax) * r2 + (g[1] * ay) * r2) + (g[2] * az) * r2
    c = c + md.γ[mu][1 - mu] * im(p * Q[i - 1, j - 1, k - 1])
    if dragν is not None and dragν[mu][1 - mu] != 0:
        qx = (mk.τx[i - 1, j - 1, k - 1] * im(p * s.Vx[i - 1, j - 1, k - 1] * Q[i, j - 1, k - 1]) +
              mk.τx[i - 2, j - 1, k - 1] * im(p * np.conj(s.Vx[i - 2, j - 1, k - 1]) * Q[i - 2, j - 1, k - 1]))
        qy = (mk.τy[i - 1, j - 1, k - 1] * im(p * s.Vy[i - 1, j - 1, k - 1] * Q[i - 1, j, k - 1]) +
              mk.τy[i - 1, j - 2, k - 1] * im(p * np.conj(s.Vy[i - 1, j - 2, k - 1]) * Q[i - 1, j - 2, k - 1]))
        qz = (mk.τz[i - 1, j - 1, k - 1] * im(p * s.Vz[i - 1, j - 1, k - 1] * Q[i - 1, j - 1, k]) +
              mk.τz[i - 1, j - 1, k - 2] * im(p * np.conj(s.Vz[i - 1, j - 1, k - 2]) * Q[i - 1, j - 1, k - 2]))
        c = c + dragν[mu][1 - mu] * ((qx * r2 + qy * r2) + qz * r2)
    return c


@pytest.fixture(scope="module")
def one_fluid_state():
    md, gr, mk = wedge_case()
    H = 0.03
    st0 = T.Stepper.make(md, gr, mk)
    HJ = T.selffield(st0, 0.5)
    s0, _ = run(st0, initial_state(md, gr, mk, H), 300, H, HJ)
    return md, gr, mk, st0, s0, H, HJ


def test_dirty_split_and_conductance():
    md, gr, mk = wedge_case()
    st0 = T.Stepper.make(md, gr, mk)
    st1 = T.Stepper.make(md, gr, mk, qp_exchange=1.0)
    qx = st1.qpx
    assert qx.s[0] == pytest.approx(1 / (1 + 16 * 0.59), rel=1e-12)
    assert qx.G == pytest.approx(qx.s[0] * 1.0, rel=1e-12)
    assert st1.dt == st0.dt


@pytest.mark.parametrize("drag", [None, 0.3])
def test_delta_solves_its_equation(one_fluid_state, drag):
    """σn∇²δ − λ0δ = S on the unknowns, S from the conversions (with the drag: their drag share, exchange.jl:327-332,
    which moves S by more than the tolerance)."""
    md, gr, mk, st0, s0, H, HJ = one_fluid_state
    st1 = T.Stepper.make(md, gr, mk, qp_exchange=1.0, **({} if drag is None else dict(rkl=False, drag=drag)))
    dν = None if drag is None else st1.dragν
    qx = st1.qpx
    c = pyoracle.OracleStepper(st1)
    c.upload(s0)
    δ = c.qp_delta()
    Nx, Ny, Nz, dx = gr.Nx, gr.Ny, gr.Nz, gr.dx
    S = np.zeros_like(δ)
    shift = 0.0
    for k in range(gr.z1, gr.z2 + 2):
        for j in range(gr.y1, gr.y2 + 2):
            for i in range(gr.x1, gr.x2 + 2):
                S[i - 1, j - 1, k - 1] = (conv(s0, mk, md, gr, 1, i, j, k, dν) / qx.s[1] -
                                          conv(s0, mk, md, gr, 0, i, j, k, dν) / qx.s[0])
                if dν is not None:
                    S0 = conv(s0, mk, md, gr, 1, i, j, k) / qx.s[1] - conv(s0, mk, md, gr, 0, i, j, k) / qx.s[0]
                    shift = max(shift, abs(S[i - 1, j - 1, k - 1] - S0))
    res = 0.0
    for k in range(1, Nz + 2):
        for j in range(1, Ny + 2):
            for i in range(2, Nx + 1):
                jm = 2 if j == 1 else j - 1
                jp = Ny if j == Ny + 1 else j + 1
                km = 2 if k == 1 else k - 1
                kp = Nz if k == Nz + 1 else k + 1
                d = lambda a, b, e: δ[a - 1, b - 1, e - 1]
                lap = (d(i + 1, j, k) + d(i - 1, j, k) + d(i, jp, k) + d(i, jm, k) + d(i, j, kp) + d(i, j, km) -
                       6 * d(i, j, k)) / dx ** 2
                res = max(res, abs(qx.σn * lap - qx.λ0 * d(i, j, k) - S[i - 1, j - 1, k - 1]))
    assert np.max(np.abs(S)) > 0.1 and res < 1e-11, res
    assert dν is None or shift > 1e-3, shift


def test_fast_exchange_is_one_fluid(one_fluid_state):
    md, gr, mk, st0, s0, H, HJ = one_fluid_state
    stb = T.Stepper.make(md, gr, mk, qp_exchange=1e6)
    sb, _ = run(stb, initial_state(md, gr, mk, H), 300, H, HJ)
    for mu in range(2):
        assert np.max(np.abs(s0.G[mu] - sb.G[mu])) < 1e-4


def band_currents(s, st):
    """observables.jl:83-99 (one material): each band's x current through the middle plane."""
    gr = st.grid
    i = int(np.floor(gr.Nx / 2 + 0.5))
    out = []
    for mu in range(st.N):
        G = s.G[mu]
        sl = (slice(gr.y1 - 1, gr.y2 + 1), slice(gr.z1 - 1, gr.z2 + 1))
        v = st.w[mu] * np.imag((np.conj(G[i - 1][sl]) * s.Vx[i - 1][sl]) * G[i][sl])
        out.append(np.sum(v.T.ravel()) / gr.dx * gr.dy * gr.dz)
    return out


def test_strip_follows_the_two_fluid_law():
    md = T.two_band(xi_ratio=4.0, κ=25.0, gamma12=0.0, gamma_kwt=10.0)

    def strip(ν):
        g2 = T.Grid.make(80, 4, 2, dx=0.5)
        m2 = build_masks(GeomSpec(GEOM_MODE="SIM"), g2)
        st = T.Stepper.make(md, g2, m2, qp_exchange=ν)
        s = initial_state(md, g2, m2, 0.0)
        HJ2 = T.selffield(st, 0.05)
        s, _ = run(st, s, int(np.floor(300 / st.dt + 0.5)), 0.0, HJ2)
        Ib = band_currents(s, st)
        return Ib[0] / (Ib[0] + Ib[1])

    f_inf, f10, f1 = strip(None), strip(10.0), strip(1.0)
    assert abs(f_inf - 0.5664) <= 0.003 and abs(f10 - 0.5484) <= 0.01 and abs(f1 - 0.4567) <= 0.02, (f_inf, f10, f1)


def test_refusals():
    """A negative rate is refused (exchange.jl:173); the drag goes with the fluids (its share of the conversion)."""
    md, gr, mk = wedge_case()
    st = T.Stepper.make(md, gr, mk, qp_exchange=1.0, rkl=False, drag=0.1)
    assert st.qpx is not None and st.drag is not None
    with pytest.raises(ValueError):
        T.Stepper.make(md, gr, mk, qp_exchange=-1.0)


# ---- N fluids (QPExchangeN, exchange.jl:416-543): gtdgl/test/test_physics.jl:383-433


def conv_n(s, mk, md, gr, mu, i, j, k):
    """_conv with N bands (the Josephson terms with every other band)."""
    P = s.G[mu]
    p = np.conj(P[i - 1, j - 1, k - 1])
    g = [stiffness(md.bands[mu], a) for a in (1, 2, 3)]
    r2 = 1 / gr.dx ** 2
    ax = (mk.τx[i - 1, j - 1, k - 1] * (p * s.Vx[i - 1, j - 1, k - 1] * P[i, j - 1, k - 1]).imag +
          mk.τx[i - 2, j - 1, k - 1] * (p * np.conj(s.Vx[i - 2, j - 1, k - 1]) * P[i - 2, j - 1, k - 1]).imag)
    ay = (mk.τy[i - 1, j - 1, k - 1] * (p * s.Vy[i - 1, j - 1, k - 1] * P[i - 1, j, k - 1]).imag +
          mk.τy[i - 1, j - 2, k - 1] * (p * np.conj(s.Vy[i - 1, j - 2, k - 1]) * P[i - 1, j - 2, k - 1]).imag)
    az = (mk.τz[i - 1, j - 1, k - 1] * (p * s.Vz[i - 1, j - 1, k - 1] * P[i - 1, j - 1, k]).imag +
          mk.τz[i - 1, j - 1, k - 2] * (p * np.conj(s.Vz[i - 1, j - 1, k - 2]) * P[i - 1, j - 1, k - 2]).imag)
    c = ((g[0] * ax) * r2 + (g[1] * ay) * r2) + (g[2] * az) * r2
    for nu in range(md.N):
        if nu != mu:
            c += md.γ[mu][nu] * (p * s.G[nu][i - 1, j - 1, k - 1]).imag
    return c


def three_band_model():
    return T.Model.make((T.Band.make(), T.Band.make(m=2.0, a=0.8), T.Band.make(m=0.5, Γ=1.5, a=0.6)),
                        [[0.0, -0.05, -0.05], [-0.05, 0.0, -0.05], [-0.05, -0.05, 0.0]], κ=25.0)


@pytest.fixture(scope="module")
def three_band_state():
    md, gr, mk = wedge_case()
    m3 = three_band_model()
    st3 = T.Stepper.make(m3, gr, mk)
    H = 0.03
    H3 = T.selffield(st3, 0.3)
    s3, _ = run(st3, initial_state(m3, gr, mk, H), 300, H, H3)
    sh = [stiffness(b) * b.Γ / b.β for b in m3.bands]
    sh = [x / sum(sh) for x in sh]
    χ3 = [sh[µ] * m3.σn * m3.bands[µ].Γ / stiffness(m3.bands[µ]) for µ in range(3)]
    return m3, gr, mk, st3, s3, H, H3, sh, χ3


def rates(χ3, r):
    return [[0.0 if µ == n else r / χ3[µ] for n in range(3)] for µ in range(3)]   # G_µν = r: detailed balance


def test_two_fluids_as_a_matrix_are_the_two_band_model(one_fluid_state):
    md, gr, mk, st0, s0, H, HJ = one_fluid_state
    sa = T.Stepper.make(md, gr, mk, qp_exchange=1.0)
    q2 = sa.qpx
    χ = [q2.s[µ] * md.σn * md.bands[µ].Γ / stiffness(md.bands[µ]) for µ in range(2)]
    sb = T.Stepper.make(md, gr, mk, qp_exchange=[[0.0, 1.0], [χ[0] / χ[1], 0.0]])
    qn = sb.qpx
    assert isinstance(qn, T.QPExchangeN) and np.allclose(qn.s, q2.s, rtol=1e-14)
    ca = pyoracle.OracleStepper(sa)
    ca.upload(s0)
    δ = ca.qp_delta()
    cb = pyoracle.OracleStepper(sb)
    cb.upload(s0)
    μ = cb.qp_mu()
    assert np.max(np.abs((μ[1] - μ[0]) - δ)) < 1e-12 * max(1.0, np.max(np.abs(δ))) and np.max(np.abs(δ)) > 1e-3
    a, _ = run(sa, s0, 200, H, HJ)
    b, _ = run(sb, s0, 200, H, HJ)
    for mu in range(2):
        assert np.max(np.abs(a.G[mu] - b.G[mu])) < 1e-10


def test_three_fluids_keep_the_gauge(three_band_state):
    m3, gr, mk, st3, s3, H, H3, sh, χ3 = three_band_state
    stn = T.Stepper.make(m3, gr, mk, qp_exchange=rates(χ3, 0.5))
    c = pyoracle.OracleStepper(stn)
    c.upload(s3)
    pot = c.qp_mu()
    assert np.max(np.abs(sh[0] * pot[0] + sh[1] * pot[1] + sh[2] * pot[2])) < 1e-12 and np.max(np.abs(pot[2])) > 1e-3


def test_three_fluids_solve_their_equations(three_band_state):
    m3, gr, mk, st3, s3, H, H3, sh, χ3 = three_band_state
    Gp = [[0.0, 0.5, 0.1], [0.5, 0.0, 2.0], [0.1, 2.0, 0.0]]
    stg = T.Stepper.make(m3, gr, mk, qp_exchange=[[0.0 if µ == n else Gp[µ][n] / χ3[µ] for n in range(3)]
                                                  for µ in range(3)])
    c = pyoracle.OracleStepper(stg)
    c.upload(s3)
    M = c.qp_mu()
    Nx, Ny, Nz, dx = gr.Nx, gr.Ny, gr.Nz, gr.dx
    C = [np.zeros_like(M[0]) for _ in range(3)]
    for k in range(gr.z1, gr.z2 + 2):
        for j in range(gr.y1, gr.y2 + 2):
            for i in range(gr.x1, gr.x2 + 2):
                for mu in range(3):
                    C[mu][i - 1, j - 1, k - 1] = conv_n(s3, mk, m3, gr, mu, i, j, k)
    res = 0.0
    for k in range(1, Nz + 2):
        for j in range(1, Ny + 2):
            for i in range(2, Nx + 1):
                jm = 2 if j == 1 else j - 1
                jp = Ny if j == Ny + 1 else j + 1
                km = 2 if k == 1 else k - 1
                kp = Nz if k == Nz + 1 else k + 1
                for mu in range(3):
                    P = M[mu]
                    d = lambda a, b, e: P[a - 1, b - 1, e - 1]
                    lap = (d(i + 1, j, k) + d(i - 1, j, k) + d(i, jp, k) + d(i, jm, k) + d(i, j, kp) + d(i, j, km) -
                           6 * d(i, j, k)) / dx ** 2
                    Lµ = sum(Gp[mu][n] * (P[i - 1, j - 1, k - 1] - M[n][i - 1, j - 1, k - 1]) for n in range(3)) / sh[mu]
                    src = C[mu][i - 1, j - 1, k - 1] / sh[mu] - (C[0][i - 1, j - 1, k - 1] + C[1][i - 1, j - 1, k - 1] +
                                                                 C[2][i - 1, j - 1, k - 1])
                    res = max(res, abs(m3.σn * lap - Lµ - src))
    assert np.max(np.abs(C[2])) > 0.1 and res < 1e-10, res


def test_three_fluids_fast_exchange_is_one_fluid(three_band_state):
    m3, gr, mk, st3, s3, H, H3, sh, χ3 = three_band_state
    sf = T.Stepper.make(m3, gr, mk, qp_exchange=rates(χ3, 1e6))
    x, _ = run(st3, s3, 200, H, H3)
    y, _ = run(sf, s3, 200, H, H3)
    for mu in range(3):
        assert np.max(np.abs(x.G[mu] - y.G[mu])) < 1e-4


def test_three_fluid_refusals():
    md, gr, mk = wedge_case()
    m3 = three_band_model()
    with pytest.raises(ValueError):   # detailed balance violated
        T.Stepper.make(m3, gr, mk, qp_exchange=np.array([[0.0, 1.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 0.0]]) *
                       np.array([1.0, 2.0, 3.0]))
    with pytest.raises(ValueError):   # a number is two bands only
        T.Stepper.make(m3, gr, mk, qp_exchange=0.5)


# ---- the Joule heat of the fluids (qp_joule with the heat model): gtdgl/test/test_physics.jl:672-693


def heated(ν, backend="oracle"):
    """300 steps of the 24×12×4 notched box with the Joule heat (Heat(joule=True, eta=0.05)) and fluids ν; θ."""
    md, gr, mk = wedge_case()
    H = 0.03
    st = T.Stepper.make(md, gr, mk, heat=T.Heat(joule=True, eta=0.05), qp_exchange=ν)
    HJ = T.selffield(st, 0.9)
    from juliatdgl_b200 import abi
    carry = abi.Carry(st)
    if backend == "oracle":
        c = pyoracle.OracleStepper(st)
        c.upload(initial_state(md, gr, mk, H))
        assert c.steps(300, H, HJ) == 0
        c.get_carry(carry)
    else:
        from juliatdgl_b200 import gpu
        c = gpu.GPUStepper(st)
        try:
            c.upload(initial_state(md, gr, mk, H))
            c.steps(300, H, HJ)
            c.get_carry(carry)
        finally:
            c.close()
    return carry.heat_theta.copy(), st


def matrix_of(st):
    md = st.model
    q = st.qpx
    χ = [q.s[µ] * md.σn * md.bands[µ].Γ / stiffness(md.bands[µ]) for µ in range(2)]
    return [[0.0, q.ν], [q.ν * χ[0] / χ[1], 0.0]]


def test_joule_heat_of_the_fluids():
    θ0, _ = heated(None)
    θ6, _ = heated(1e6)
    θ1, st1 = heated(1.0)
    assert np.max(np.abs(θ6 - θ0)) < 1e-5 * np.max(θ0)
    assert np.max(θ1) > 1.2 * np.max(θ0)
    θn, _ = heated(matrix_of(st1))
    assert np.max(np.abs(θn - θ1)) < 1e-9 * np.max(θ1)


def test_two_fluids_with_the_insulating_padding():
    """test_physics.jl:633-642 (T8): with the insulating padding δ lives on the bar of the sample and its contacts
    (its region y1..y2+1, z1..z2+1), the strip's σ share is 0.4427 ± 0.01, and δ is zero in the insulator."""
    md = T.two_band(xi_ratio=4.0, κ=25.0, gamma12=0.0, gamma_kwt=10.0)
    g2 = T.Grid.make(80, 4, 2, dx=0.5)
    k2 = build_masks(GeomSpec(GEOM_MODE="SIM"), g2)
    st = T.Stepper.make(md, g2, k2, qp_exchange=1.0, σvac=0.01)
    q = st.qpx
    assert (g2.Nx - 1, q.nj, q.nk) == (g2.Nx - 1, g2.y2 - g2.y1 + 2, g2.z2 - g2.z1 + 2)
    s, c = run(st, initial_state(md, g2, k2, 0.0), int(np.floor(300 / st.dt + 0.5)), 0.0, T.selffield(st, 0.05))
    Ib = band_currents(s, st)
    assert abs(Ib[0] / (Ib[0] + Ib[1]) - 0.4427) <= 0.01, Ib
    δ = c.qp_delta()
    assert np.all(δ[:, :g2.y1 - 1, :] == 0) and np.all(δ[:, :, g2.z2 + 1:] == 0)


# ---- a sculpted sample: the conjugate-gradient solve of δ (QPSolve): gtdgl/test/test_physics.jl:643-669


def cut_apply(x, cond, σn, lam, h):
    """_qp_apply! (exchange.jl:52-84) on region arrays: y = −(σn∇²_c − λ) x, cut links, mirror ghosts on y and z."""
    n1, n2, n3 = x.shape
    a = σn / h ** 2
    y = np.zeros_like(x)
    for k in range(n3):
        for j in range(n2):
            for i in range(n1):
                if not cond[i, j, k]:
                    y[i, j, k] = (2 * a + 2 * a + 2 * a + lam) * x[i, j, k]
                    continue
                v = x[i, j, k]
                acc = lam * v
                acc += a * (v - ((x[i - 1, j, k] if cond[i - 1, j, k] else v) if i > 0 else 0.0))
                acc += a * (v - ((x[i + 1, j, k] if cond[i + 1, j, k] else v) if i < n1 - 1 else 0.0))
                if n2 > 1:
                    if j == 0:
                        acc += 2 * a * (v - x[i, 1, k]) if cond[i, 1, k] else 0.0
                    elif j == n2 - 1:
                        acc += 2 * a * (v - x[i, n2 - 2, k]) if cond[i, n2 - 2, k] else 0.0
                    else:
                        acc += a * (v - x[i, j - 1, k]) if cond[i, j - 1, k] else 0.0
                        acc += a * (v - x[i, j + 1, k]) if cond[i, j + 1, k] else 0.0
                if n3 > 1:
                    if k == 0:
                        acc += 2 * a * (v - x[i, j, 1]) if cond[i, j, 1] else 0.0
                    elif k == n3 - 1:
                        acc += 2 * a * (v - x[i, j, n3 - 2]) if cond[i, j, n3 - 2] else 0.0
                    else:
                        acc += a * (v - x[i, j, k - 1]) if cond[i, j, k - 1] else 0.0
                        acc += a * (v - x[i, j, k + 1]) if cond[i, j, k + 1] else 0.0
                y[i, j, k] = acc
    return y


def test_sculpted_sample_solves_the_cut_link_equation():
    import dataclasses
    import cases
    st, s, H, HJ = cases.vacuum("vac_plain", qp_exchange=1.0)
    md, gr, mk = st.model, st.grid, st.masks
    s, c = run(st, s, 60, H, HJ)
    q = st.qpx
    δ = c.qp_delta()
    it = c.qp_iters()
    assert 0 < it < q.maxit
    # the source again, cut, and the residual of the cut-link operator on the region
    j0, k0 = q.j0 - 1, q.k0 - 1
    S = np.zeros((gr.Nx - 1, q.nj, q.nk))
    for k in range(gr.z1, gr.z2 + 2):
        for j in range(gr.y1, gr.y2 + 2):
            for i in range(gr.x1, gr.x2 + 2):
                S[i - 2, j - j0 - 1, k - k0 - 1] = (conv(s, mk, md, gr, 1, i, j, k) / q.s[1] -
                                                    conv(s, mk, md, gr, 0, i, j, k) / q.s[0])
    S[~q.cond] = 0
    x = δ[1:gr.Nx, j0:j0 + q.nj, k0:k0 + q.nk]
    y = cut_apply(x, q.cond, q.σn, max(q.λ0, 1e-12 * q.σn), gr.dx)
    assert np.max(np.abs(S)) > 1e-3 and np.max(np.abs(y + S)) < 1e-8 * np.max(np.abs(S))
    assert np.all(x[~q.cond] == 0)
    # nothing cut: the conjugate gradients give the separable solve
    st0 = dataclasses.replace(st, qpx=dataclasses.replace(q, cond=None))
    st1 = dataclasses.replace(st, qpx=dataclasses.replace(q, cond=np.ones_like(q.cond)))
    c0 = pyoracle.OracleStepper(st0)
    c0.upload(s)
    c1 = pyoracle.OracleStepper(st1)
    c1.upload(s)
    d0, d1 = c0.qp_delta(), c1.qp_delta()
    assert np.max(np.abs(d1 - d0)) < 1e-8 * np.max(np.abs(d0))


def test_two_fluids_as_a_matrix_in_a_sculpted_sample_are_the_two_band_model():
    """N fluids in a sculpted sample (exchange.jl:496-506): each mode of S⁻¹L by conjugate gradients over the cut
    links. Two bands as a matrix of rates give μ_π − μ_σ = δ of the two-band solve to the CG tolerance, and the same
    run."""
    import cases
    sa, s, H, HJ = cases.vacuum("vac_qp")
    sb, _, _, _ = cases.vacuum("vac_qpn")
    assert isinstance(sb.qpx, T.QPExchangeN) and sb.qpx.cond is not None
    s = pyoracle.run(sa, s, 10, H, HJ)
    ca = pyoracle.OracleStepper(sa)
    ca.upload(s)
    δ = ca.qp_delta()
    cb = pyoracle.OracleStepper(sb)
    cb.upload(s)
    μ = cb.qp_mu()
    assert np.max(np.abs(δ)) > 1e-4 and cb.qp_iters() > 0
    assert np.max(np.abs((μ[1] - μ[0]) - δ)) < 1e-8 * np.max(np.abs(δ))
    a = pyoracle.run(sa, s, 30, H, HJ)
    b = pyoracle.run(sb, s, 30, H, HJ)
    worst, per = cases.compare_states(b, a)
    assert worst < 1e-8, per
