"""Material per region (gtdgl/src/materials.jl) on the host mirror and the oracle, against the reference's own tests
of it (gtdgl/test/test_materials.jl): two regions of one material are the uniform run to the bit (with noise too);
the lattice continuity through an interface node by node; the proximity decay into a normal metal against the
linearised lattice solution; a strip all of one material is that material's uniform run; the mirror y → −y with
an x slab; the normal state of two conductivities in series; a one-band metal; the link weights ρ = t·m_ref/m_link;
the guards of the constructor.
"""
import math

import numpy as np
import pytest

import cases
import juliatdgl_b200 as T
from juliatdgl_b200.grid import with_materials
from juliatdgl_b200.state import initial_state
from oracle import pyoracle

cm = cases.copy_model


def same(a, b):
    """_same of test_materials.jl:8."""
    return (all(np.array_equal(a.G[µ], b.G[µ]) for µ in range(a.N))
            and all(np.array_equal(getattr(a, q), getattr(b, q)) for q in ("φx", "φy", "φz", "hz")))


def wedge24():
    gr = T.Grid.make(24, 12, 4, dx=0.5)
    mk = T.build_masks(T.GeomSpec(GEOM_MODE="WEDGE", inj_margin=4), gr)
    return gr, mk, with_materials(mk, gr, lambda i, j, k: 2 if i > gr.x1 + 12 else 1)


@pytest.mark.parametrize("model,kw", [
    ("plain", {}), ("kwt", {}), ("k25", dict(rkl=False)),
    ("plain", dict(noise=1e-3, noise_seed=5)), ("kwt", dict(noise=1e-3, noise_seed=5))])
def test_two_regions_of_one_material_are_the_uniform_run(model, kw):
    """test_materials.jl:10-21 and :225-238: the material path with a copy of the material gives the bits."""
    md = {"plain": T.two_band(xi_ratio=4.0, κ=2.0), "kwt": T.two_band(xi_ratio=4.0, κ=2.0, gamma_kwt=10.0),
          "k25": T.two_band(xi_ratio=4.0, κ=25.0)}[model]
    gr, mk, mk2 = wedge24()
    a = T.Stepper.make(md, gr, mk, **kw)
    b = T.Stepper.make(md, gr, mk2, materials=[cm(md)], **kw)
    assert a.rkl == b.rkl and a.dt == b.dt and b.mt is not None
    sa = initial_state(md, gr, mk, 0.03)
    sb = initial_state(md, gr, mk2, 0.03, materials=b.mt.models)
    HJ = T.selffield(a, 0.5)
    n = 50 if (model == "kwt" and kw) else 150
    assert same(pyoracle.run(a, sa, n, 0.03, HJ), pyoracle.run(b, sb, n, 0.03, HJ))


def random_state(md, gr, mk, st, seed=3):
    s = initial_state(md, gr, mk, 0.0, materials=st.mt.models)
    rng = np.random.default_rng(seed)
    G = s.G[0]
    for c in np.ndindex(*G.shape):
        if mk.τψ[c] > 0:
            G[c] *= (0.7 + 0.3 * rng.random()) * np.exp(1j * 2 * rng.standard_normal())
    return s


def continuity_residual(st, mk, s):
    """test_materials.jl:23-38: (Γ_n/dt) Im(Ḡ ΔΨ) = div J/dx² on every interior node after one Euler pass of one
    band (the step's F is that pass; its J is the supercurrent of the same Ψⁿ)."""
    gr = st.grid
    G = s.G[0].copy()
    s1 = pyoracle.run(st, s, 1, 0.0, 0.0)
    F, Jx, Jy, Jz = s1.G[0], s1.Jx, s1.Jy, s1.Jz
    r = 0.0
    for k in range(gr.z1 + 1, gr.z2 + 1):
        for j in range(gr.y1 + 1, gr.y2 + 1):
            for i in range(gr.x1 + 1, gr.x2 + 1):
                c = (i - 1, j - 1, k - 1)
                Γn = st.mt.models[int(mk.mat[c]) - 1].bands[0].Γ
                lhs = (Γn / st.dt) * np.imag(np.conj(G[c]) * (F[c] - G[c]))
                rhs = (((Jx[c] - Jx[i - 2, j - 1, k - 1]) + (Jy[c] - Jy[i - 1, j - 2, k - 1]))
                       + (Jz[c] - Jz[i - 1, j - 1, k - 2])) / gr.dx ** 2
                r = max(r, abs(lhs - rhs))
    return r


@pytest.mark.parametrize("aniso", [False, True])
def test_lattice_continuity_through_an_interface(aniso):
    gr = T.Grid.make(12, 6, 4, dx=0.5)
    mk = with_materials(T.box_masks(gr), gr, lambda i, j, k: 2 if i >= gr.x1 + 6 else 1)
    if aniso:   # test_materials.jl:241-254
        md = T.Model.make((T.Band.make(m_axes=(1.0, 2.0, 0.5)),), [[0.0]], κ=2.0)
        m2 = T.Model.make((T.Band.make(m_axes=(1.5, 0.7, 3.0), a=0.6, Γ=1.3),), [[0.0]], κ=2.0)
    else:
        md = T.Model.make((T.Band.make(),), [[0.0]], κ=2.0)
        m2 = T.Model.make((T.Band.make(m=1.5, a=0.6, Γ=1.3),), [[0.0]], κ=2.0)
    st = T.Stepper.make(md, gr, mk, implicit=False, substeps=(1,), materials=[m2])
    assert continuity_residual(st, mk, random_state(md, gr, mk, st)) < 1e-12


def test_proximity_decay_into_a_normal_metal():
    """test_materials.jl:39-47: |Ψ| decays into S′ (a′ = −0.5, m′ = 2) as the linearised lattice solution."""
    md = T.Model.make((T.Band.make(),), [[0.0]], κ=2.0)
    gr = T.Grid.make(80, 2, 2, dx=0.5)
    i0 = gr.x1 + 40
    mk = with_materials(T.box_masks(gr), gr, lambda i, j, k: 2 if i >= i0 else 1)
    m2 = T.Model.make((T.Band.make(m=2.0, a=-0.5),), [[0.0]], κ=2.0)
    st = T.Stepper.make(md, gr, mk, materials=[m2])
    s = pyoracle.run(st, initial_state(md, gr, mk, 0.0, materials=st.mt.models), round(300 / st.dt), 0.0, 0.0)
    ψ = np.abs(s.G[0][:, 1, 1])
    ld = 0.5 / math.acosh(1 + 0.5 * 0.25 / (2 * 0.5))
    i3, i6 = i0 + round(3 / 0.5), i0 + round(6 / 0.5)
    assert abs((i6 - i3) * 0.5 / math.log(ψ[i3 - 1] / ψ[i6 - 1]) / ld - 1) < 1e-3


def test_a_strip_all_of_one_material_is_its_uniform_run():
    """test_materials.jl:48-56."""
    gr, mk, _ = wedge24()
    md = T.Model.make((T.Band.make(m=1.2, a=0.8), T.Band.make(m=1 / (16 * 0.5), a=0.5)), [[0.0, 1e-3], [1e-3, 0.0]],
                      κ=2.0)
    m2 = T.Model.make((T.Band.make(), T.Band.make(m=1 / (16 * 0.59), a=0.59)), [[0.0, 1e-3], [1e-3, 0.0]], κ=2.0)
    mk2 = with_materials(mk, gr, lambda i, j, k: 2)
    a = T.Stepper.make(md, gr, mk2, materials=[m2])
    b = T.Stepper.make(m2, gr, mk)
    HJ = T.selffield(b, 0.4)
    sa = pyoracle.run(a, initial_state(md, gr, mk2, 0.03, materials=a.mt.models), 500, 0.03, HJ)
    sb = pyoracle.run(b, initial_state(m2, gr, mk, 0.03), 500, 0.03, HJ)
    assert a.dt == b.dt and max(np.abs(sa.G[µ] - sb.G[µ]).max() for µ in range(2)) < 1e-12


def test_mirror_of_the_current_with_an_x_slab():
    """test_materials.jl:57-64: with the SIM geometry, +J is the mirror y → −y of −J."""
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr = T.Grid.make(16, 8, 4, dx=0.5)
    mk = with_materials(T.build_masks(T.GeomSpec(GEOM_MODE="SIM"), gr), gr,
                        lambda i, j, k: 2 if gr.x1 + 6 <= i <= gr.x1 + 10 else 1)
    m2 = T.Model.make((T.Band.make(m=1.5, a=0.7), md.bands[1]), [[0.0, 1e-3], [1e-3, 0.0]], κ=2.0)

    def run(J):
        st = T.Stepper.make(md, gr, mk, materials=[m2])
        s = initial_state(md, gr, mk, 0.05, materials=st.mt.models)
        return pyoracle.run(st, s, round(5 / st.dt), 0.05, T.selffield(st, J))

    p, q = run(0.3), run(-0.3)
    for µ in range(2):
        assert np.max(np.abs(np.abs(p.G[µ]) - np.abs(q.G[µ][:, ::-1, :]))) < 1e-12


def test_normal_state_of_two_conductivities_in_series():
    """test_materials.jl:182-191: Ψ held at 0, the steady E_x in the two halves is in the ratio σ₁/σ₂ = 4."""
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr = T.Grid.make(40, 4, 4, dx=0.5)
    mk = T.build_masks(T.GeomSpec(GEOM_MODE="SIM"), gr)
    mk.f[...] = 0.0
    mk2 = with_materials(mk, gr, lambda i, j, k: 2 if i >= gr.x1 + 20 else 1)
    st = T.Stepper.make(md, gr, mk2, hard=True, materials=[cm(md, σn=0.25)])
    assert st.solver == 3      # σn per region: the PCG path
    s = initial_state(md, gr, mk2, 0.0, materials=st.mt.models)
    HJ = T.selffield(st, 0.1)
    o = pyoracle.OracleStepper(st)
    o.upload(s)
    o.steps(round(150 / st.dt), 0.0, HJ)
    o.download(s)
    θ0 = s.θx.copy()
    o.steps(1, 0.0, HJ)
    o.download(s)

    def E(i):
        return -(s.θx[i - 1, 2, 2] - θ0[i - 1, 2, 2]) / st.dt

    assert E(gr.x2 - 6) / E(gr.x1 + 6) == pytest.approx(4, rel=1e-6)


def test_equal_sigma_keeps_the_separable_solve_and_the_bits():
    """test_materials.jl:192-201."""
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr, mk, mk2 = wedge24()
    a = T.Stepper.make(md, gr, mk)
    b = T.Stepper.make(md, gr, mk2, materials=[cm(md)])
    assert b.solver == 2
    HJ = T.selffield(a, 0.5)
    sa = pyoracle.run(a, initial_state(md, gr, mk, 0.03), 100, 0.03, HJ)
    sb = pyoracle.run(b, initial_state(md, gr, mk2, 0.03, materials=b.mt.models), 100, 0.03, HJ)
    assert same(sa, sb)


def test_one_band_metal():
    """test_materials.jl:208-220: band 2 absent from the metal: Ψπ = 0 there, Ψσ induced, the same stages."""
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr, mk, mk2 = wedge24()
    metal = T.Model.make((T.Band.make(a=-0.5), T.Band.make(m=md.bands[1].m, a=-1.0)), [[0.0, 0.0], [0.0, 0.0]], κ=2.0)
    st = T.Stepper.make(md, gr, mk2, materials=[metal], absent=[[], [2]])
    assert st.rkl == T.Stepper.make(md, gr, mk).rkl
    s = pyoracle.run(st, initial_state(md, gr, mk2, 0.03, materials=st.mt.models), 200, 0.03, T.selffield(st, 0.2))
    inN = (mk2.mat == 2) & (mk.τψ > 0)
    assert np.all(s.G[1][inN] == 0) and np.abs(s.G[0][inN]).max() > 0.1


def test_link_weights():
    """test_materials.jl:87-94 and :128: ρ = t·m_ref/m_link across an interface, m_ref/m inside a slab."""
    gr = T.Grid.make(24, 12, 4, dx=0.5)
    mk = with_materials(T.box_masks(gr), gr, lambda i, j, k: 2 if i > gr.x1 + 10 else 1)
    md = T.Model.make((T.Band.make(),), [[0.0]], κ=2.0)
    m2 = T.Model.make((T.Band.make(m=2.0),), [[0.0]], κ=2.0)
    st = T.Stepper.make(md, gr, mk, materials=[m2], transparency=[[1.0, 0.2], [0.2, 1.0]])
    ρ = st.mt.rho(1, 1, mk.τx)
    i = gr.x1 + 10      # the link from the last node of material 1 to the first of material 2
    assert ρ[i - 1, 4, 2] == pytest.approx(0.2 * 1.0 / ((1.0 + 2.0) / 2))
    assert ρ[i, 4, 2] == 0.5 and ρ[i - 2, 4, 2] == 1.0


def test_guards():
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr, mk, mk2 = wedge24()
    with pytest.raises(ValueError):            # a map of materials needs their models
        T.Stepper.make(md, gr, mk2)
    with pytest.raises(ValueError):            # an absent band has a <= T
        T.Stepper.make(md, gr, mk2, materials=[cm(md)], absent=[[], [2]])
    with pytest.raises(ValueError):            # transparency: symmetric, (0, 1], ones on the diagonal
        T.Stepper.make(md, gr, mk2, materials=[cm(md)], transparency=[[1.0, 0.5], [0.4, 1.0]])
    with pytest.raises(ValueError):            # κ is the sample's
        T.Stepper.make(md, gr, mk2, materials=[T.two_band(xi_ratio=4.0, κ=3.0)])


def test_material_conductivity_is_the_per_link_rule():
    """materials.jl:124-138 link by link (a node outside the block takes the nearest block node's σn; harmonic mean
    where the two differ; the insulating padding keeps σvac) against the vectorised host function."""
    from juliatdgl_b200.scheme import link_conductivity, material_conductivity
    gr = T.Grid.make(10, 6, 4, dx=0.5, buf=2)
    mk = with_materials(T.box_masks(gr), gr, lambda i, j, k: 1 + (i > gr.x1 + 4) + (k > gr.z1 + 2))
    mats = [T.two_band(xi_ratio=4.0, κ=2.0, σn=s) for s in (1.0, 0.5, 2.0)]
    for σvac in (None, 0.01):
        got = material_conductivity(gr, mk, mats, σvac, 1.0)
        base = link_conductivity(gr, σvac, 1.0) if σvac else None
        σ = lambda i, j, k: mats[int(mk.mat[min(max(i, gr.x1), gr.x2 + 1) - 1, min(max(j, gr.y1), gr.y2 + 1) - 1,
                                            min(max(k, gr.z1), gr.z2 + 1) - 1]) - 1].σn
        for ax, o in enumerate(((1, 0, 0), (0, 1, 0), (0, 0, 1))):
            for c in np.ndindex(*got[ax].shape):
                if base is not None and base[ax][c] != 1.0:
                    assert got[ax][c] == base[ax][c]
                    continue
                i, j, k = c[0] + 1, c[1] + 1, c[2] + 1
                a, b = σ(i, j, k), σ(i + o[0], j + o[1], k + o[2])
                assert got[ax][c] == (a if a == b else 2 * a * b / (a + b))


def test_heat_with_two_regions_of_one_material_is_the_uniform_run():
    """test_materials.jl:240: the heat model (D_T 0.25, the Joule term) through the material path with a copy of the
    material gives the uniform run's bits, the temperature field included."""
    from juliatdgl_b200.abi import Carry
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr, mk, mk2 = wedge24()
    heat = T.Heat(D_T=0.25, joule=True)
    a = T.Stepper.make(md, gr, mk, heat=heat)
    b = T.Stepper.make(md, gr, mk2, materials=[cm(md)], heat=heat)
    assert a.dt == b.dt and b.mt is not None and b.heat_DT == (0.25, 0.25)
    out = []
    for st, s in ((a, initial_state(md, gr, mk, 0.03)), (b, initial_state(md, gr, mk2, 0.03, materials=b.mt.models))):
        o = pyoracle.OracleStepper(st)
        o.upload(s)
        assert o.steps(100, 0.03, T.selffield(a, 0.5)) == 0
        o.download(s)
        c = o.get_carry(Carry(st))
        out.append((s, c.heat_theta.copy()))
    assert same(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1]) and out[0][1].max() > 0


def test_heat_DT_per_material_conserves_the_heat_content():
    """test_materials.jl:255-262: D_T per material (0.25 and 1.0, the Jacobi update with harmonic means), no bath and
    no source: the heat content of the block is conserved to 1e-12 over 2000 steps."""
    from juliatdgl_b200.abi import Carry
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    g = T.Grid.make(40, 4, 2, dx=0.5)
    m = T.box_masks(g)
    m.f[...] = 0.0
    m2 = with_materials(m, g, lambda i, j, k: 2 if i > g.x1 + 20 else 1)
    st = T.Stepper.make(md, g, m2, hard=True, heat=T.Heat(D_T=0.25, gamma_bath=0.0, eta=0.0), materials=[cm(md)],
                        heat_DT=[0.25, 1.0])
    s = initial_state(md, g, m2, 0.0, materials=st.mt.models)
    c = Carry(st)
    ii = np.arange(1, g.Nx + 2)[:, None, None]
    c.heat_theta[...] = np.where(ii <= g.x1 + 10, 0.4, 0.1) + 0.0 * c.heat_theta
    blk = (slice(g.x1, g.x2), slice(g.y1, g.y2), slice(g.z1, g.z2))   # 1-based x1+1..x2 as 0-based slices
    S0 = c.heat_theta[blk].sum()
    o = pyoracle.OracleStepper(st)
    o.upload(s)
    o.set_carry(c)
    assert o.steps(2000, 0.0, 0.0) == 0
    o.get_carry(c)
    assert abs(c.heat_theta[blk].sum() / S0 - 1) < 1e-12


# ---- normal fluids per band with materials (exchange.jl:193-290, QPVar): test_materials.jl:192-219


def test_two_fluids_with_a_copy_of_the_material_keep_the_bits():
    """test_materials.jl:193-201 with qp_exchange: the material path with a copy of the material (the first material's
    σn and λ everywhere: the separable solve) gives the uniform run's bits."""
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr, mk, mk2 = wedge24()
    a = T.Stepper.make(md, gr, mk, qp_exchange=1.0)
    b = T.Stepper.make(md, gr, mk2, materials=[cm(md)], qp_exchange=1.0)
    assert b.qpx.var is None and b.solver == 2
    HJ = T.selffield(a, 0.5)
    sa = pyoracle.run(a, initial_state(md, gr, mk, 0.03), 100, 0.03, HJ)
    sb = pyoracle.run(b, initial_state(md, gr, mk2, 0.03, materials=b.mt.models), 100, 0.03, HJ)
    assert same(sa, sb)


def test_two_fluids_with_a_rate_per_material_take_the_variable_solve():
    """test_materials.jl:202-209: another exchange rate in one material goes through the variable-coefficient solve
    (conjugate gradients); a dirty split that changes between materials is refused."""
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr, mk, mk2 = wedge24()
    b = T.Stepper.make(md, gr, mk2, qp_exchange=1.0, materials=[cm(md)], qp_rates=[1.0, 10.0])
    assert b.qpx.var is not None
    c = pyoracle.OracleStepper(b)
    c.upload(initial_state(md, gr, mk2, 0.03))
    assert c.steps(50, 0.03, T.selffield(b, 0.5)) == 0
    s = c.download(initial_state(md, gr, mk2, 0.03))
    assert np.all(np.isfinite(s.G[0])) and c.qp_iters() > 0
    other = T.Model.make((md.bands[0], T.Band.make(m=2 * md.bands[1].m, a=0.59)), [[0.0, 1e-3], [1e-3, 0.0]], κ=2.0)
    with pytest.raises(ValueError):
        T.Stepper.make(md, gr, mk2, qp_exchange=1.0, materials=[other])


def test_two_fluids_in_a_one_band_metal():
    """test_materials.jl:210-219 with qp_exchange: band 2 absent from the metal, one normal fluid there (δ = 0)."""
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr, mk, mk2 = wedge24()
    metal = T.Model.make((T.Band.make(a=-0.5), T.Band.make(m=md.bands[1].m, a=-1.0)), [[0.0, 0.0], [0.0, 0.0]], κ=2.0)
    st = T.Stepper.make(md, gr, mk2, materials=[metal], absent=[[], [2]], qp_exchange=1.0)
    assert st.rkl == T.Stepper.make(md, gr, mk, qp_exchange=1.0).rkl and st.qpx.var is not None
    c = pyoracle.OracleStepper(st)
    s0 = initial_state(md, gr, mk2, 0.03, materials=st.mt.models)
    c.upload(s0)
    assert c.steps(200, 0.03, T.selffield(st, 0.2)) == 0
    s = c.download(s0.copy())
    inN = (mk2.mat == 2) & (mk.τψ > 0)
    assert np.all(s.G[1][inN] == 0) and np.abs(s.G[0][inN]).max() > 0.1
    δ = c.qp_delta()
    inNx = inN.copy()
    inNx[gr.Nx:, :, :] = False   # the nodes of δ's array up to Nx
    assert np.all(δ[inNx] == 0)
