"""Configurations shared by the tests: the release-1.2 golden cases and small cases of every path of the step.

Each builder returns (Stepper, State, H, HJ).  States are taken a few steps off their seed by the oracle where a
case needs nonzero links and currents (as gpu/TDGLGPU/test/compare_cpu.jl:72 does with 5 CPU steps).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

import juliatdgl_b200 as T
from juliatdgl_b200.grid import Masks, with_materials
from juliatdgl_b200.state import State, seeded_state

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN_CASES = ("k2_R13_explicit", "k2_R4_prod", "k25_R4_prod", "k2_R4_drag", "k2_R4_heat")


def golden(name):
    """The release-1.2 regression case (gtdgl/test/test_regression12.jl:9-29)."""
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    par = json.loads(str(d["par"]))
    md = T.two_band(xi_ratio=math.sqrt(1 / (par["m_ratio"] * par["a2n"])), a2n=par["a2n"], gamma12=par["gamma12"],
                    gamma_ratio=par["gamma_ratio"], κ=par["kappa"])
    b1, b2 = md.bands
    md = T.Model.make((b1, T.Band.make(m=par["m_ratio"], Γ=b2.Γ, a=b2.a, β=b2.β)),
                      [[0.0, par["gamma12"]], [par["gamma12"], 0.0]], κ=par["kappa"])
    gr = T.Grid.make(par["Nx_sc"], par["Ny_sc"], par["Nz_sc"], dx=par["dx"], buf=par["buf"])
    mk = Masks(*(np.asfortranarray(d[k]) for k in ("fmask", "taux", "tauy", "tauz", "taupsi")))
    drag = par.get("drag", 0.0)
    terms = par.get("heat", False) or drag != 0   # test_regression12.jl:21-25: one pi substep with terms on
    sub = (1, 1) if (par["pi_substeps_cfg"] == 1 or terms) else (1, 0)
    heat = T.Heat(D_T=par["D_T"], gamma_bath=par["gamma_bath"], eta=par["eta_J"], joule=par["joule"],
                  margin=par["heat_margin"]) if par.get("heat", False) else None
    st = T.Stepper.make(md, gr, mk, implicit=par["implicit"], substeps=sub, dt_scale=par["dt_scale"],
                        extrap=par["extrap"], selffield_bc="slab", rkl=False, drag=drag if drag != 0 else None,
                        heat=heat)
    ini = {k[4:]: d[k] for k in d.files if k.startswith("ini_")}
    fin = {k[4:]: d[k] for k in d.files if k.startswith("fin_")}
    s = State.from_fields(gr, (ini["G1"], ini["G2"]), (ini["thetax"], ini["thetay"], ini["thetaz"]),
                          (ini["phix"], ini["phiy"], ini["phiz"]), (ini["hx"], ini["hy"], ini["hz"]))
    return st, s, par, ini, fin


def config1():
    """The two-band parity case: 12×8×4 cells, h = 0.5ξ, κ = 25, dt = 0.01, KWT (10, 5), Josephson −0.05,
    H = 0.3, Jx = 0.02 (bar self-field), Ψ_b = 1 + 1e-3·(complex Gaussian, seed 0), A = 0."""
    b1 = T.Band.make(m=1.0, Γ=1.0, a=1.0, β=1.0, γkwt=10.0)
    b2 = T.Band.make(g=0.6, Γ=1.5, a=0.8, β=1.0, γkwt=5.0)
    md = T.Model.make((b1, b2), [[0.0, -0.05], [-0.05, 0.0]], κ=25.0)
    gr = T.Grid.make(12, 8, 4, dx=0.5, buf=1)
    mk = T.box_masks(gr)
    st = T.Stepper.make(md, gr, mk, dt=0.01)
    s = seeded_state(md, gr, mk, 0.3, seed=0, amp=1e-3, base=1.0)
    return st, s, 0.3, T.selffield(st, 0.02)


def _mgb2(κ=2.0, γkwt=0.0):
    return T.two_band(xi_ratio=4.0, κ=κ, gamma_kwt=γkwt)


def small(kind: str, grid=(16, 8, 4), **kw):
    """Small cases of each path: (Stepper, State, H, HJ).  J = 0.3, H = 0.03 as compare_cpu.jl.  `grid`: the cells
    of the kinds on the plain 16×8×4 grid (the padded kinds keep theirs); `kw` goes to Stepper.make (e.g.
    noise=T̃, noise_seed, noise_field)."""
    gr = T.Grid.make(*grid, dx=0.5)
    wedge = T.build_masks(T.GeomSpec(GEOM_MODE="WEDGE"), gr)
    H = 0.03
    if kind == "euler_substeps":           # release-1.2 scheme: Euler substeps with extrapolated links, slab
        md = _mgb2()
        st = T.Stepper.make(md, gr, wedge, rkl=False, selffield_bc="slab", **kw)
    elif kind == "rkl_bar":                # RKL1 stages, bar field
        md = _mgb2(γkwt=0.0)
        st = T.Stepper.make(md, gr, wedge, rkl=True, **kw)
    elif kind == "rkc_kwt_rotframe":       # damped RKC with KWT and the rotating frame
        md = _mgb2(γkwt=10.0)
        st = T.Stepper.make(md, gr, wedge, **kw)
    elif kind == "kwt_substeps_rotframe":  # KWT on Euler substeps with the rotating frame
        md = _mgb2(γkwt=10.0)
        st = T.Stepper.make(md, gr, wedge, rkl=False, **kw)
    elif kind == "kwt_euler_rotframe":     # one Euler pass per band with the frame (substeps = 1)
        md = _mgb2(γkwt=3.0)
        st = T.Stepper.make(md, gr, wedge, rkl=False, substeps=(1, 1), dt_scale=0.2, **kw)
    elif kind == "explicit_scale":         # explicit curl-curl with the insulating padding (σ per link)
        gr = T.Grid.make(16, 8, 4, dx=0.5, buf=2)
        mk = T.build_masks(T.GeomSpec(GEOM_MODE="WEDGE"), gr)
        md = _mgb2()
        st = T.Stepper.make(md, gr, mk, implicit=False, σvac=0.1, **kw)
    elif kind in ("pcg", "pcg_fast", "pcg_f32"):   # insulating padding: PCG (plain, fast FP64, fast FP32 preconditioner)
        gr = T.Grid.make(16, 8, 4, dx=0.5, buf=2)
        mk = T.build_masks(T.GeomSpec(GEOM_MODE="WEDGE"), gr)
        md = _mgb2(γkwt=10.0)
        fast = kind != "pcg"
        st = T.Stepper.make(md, gr, mk, σvac=0.01, pcg_fast=fast, pcg_f32=(kind == "pcg_f32"), pcg_tol=1e-10, **kw)
    elif kind == "open":                   # the open boundary, ramps and recomputations
        md = _mgb2()
        st = T.Stepper.make(md, gr, wedge, selffield_bc="open", open_every=0.2, **kw)
    elif kind == "open_pcg":               # open boundary with the insulating padding
        gr = T.Grid.make(16, 8, 4, dx=0.5, buf=2)
        mk = T.build_masks(T.GeomSpec(GEOM_MODE="WEDGE"), gr)
        md = _mgb2(γkwt=10.0)
        st = T.Stepper.make(md, gr, mk, selffield_bc="open", open_every=0.2, σvac=0.01, pcg_tol=1e-10, **kw)
    elif kind == "three_bands":            # three frustrated bands with KWT on one
        bands = (T.Band.make(), T.Band.make(m=2.0, Γ=1.2, a=0.8, γkwt=5.0), T.Band.make(m=0.7, Γ=0.9, a=0.6))
        γ = [[0.0, -0.1, -0.05], [-0.1, 0.0, -0.08], [-0.05, -0.08, 0.0]]
        md = T.Model.make(bands, γ, κ=2.0)
        st = T.Stepper.make(md, gr, wedge, **kw)
    elif kind == "hard":                   # f = 0 nodes held at Ψ = 0
        md = _mgb2()
        st = T.Stepper.make(md, gr, wedge, hard=True, rkl=False, **kw)
    elif kind == "drag_substeps":          # the interband drag on Euler substeps with extrapolated links
        md = _mgb2()
        st = T.Stepper.make(md, gr, wedge, rkl=False, drag=0.3, **kw)
    elif kind == "drag_rkc_kwt":           # the drag on damped RKC stages with KWT and the rotating frame (ν = 0.05:
        md = _mgb2(γkwt=10.0)              # at 0.2 these stages amplify a 1e-16 perturbation to 1e-10 in 20 steps)
        st = T.Stepper.make(md, gr, wedge, drag=0.05, **kw)
    elif kind == "heat_joule":             # the heat model with the Joule term and a contact margin, RKC stages
        md = _mgb2(γkwt=3.0)
        st = T.Stepper.make(md, gr, wedge, heat=T.Heat(eta=0.5, joule=True, margin=2), **kw)
    elif kind == "drag_three":             # three bands, a drag matrix, RKL stages and the bar field
        bands = (T.Band.make(), T.Band.make(m=2.0, Γ=1.2, a=0.8), T.Band.make(m=0.7, Γ=0.9, a=0.6))
        γ = [[0.0, -0.1, -0.05], [-0.1, 0.0, -0.08], [-0.05, -0.08, 0.0]]
        md = T.Model.make(bands, γ, κ=2.0)
        st = T.Stepper.make(md, gr, wedge, rkl="rkl", drag=[[0.0, 0.2, 0.1], [0.2, 0.0, 0.3], [0.1, 0.3, 0.0]], **kw)
    elif kind == "qp_rkc_kwt":             # two normal fluids (exchange.jl) on RKC stages with KWT and the frame
        md = _mgb2(γkwt=10.0)
        st = T.Stepper.make(md, gr, wedge, qp_exchange=1.0, **kw)
    elif kind == "qp_drag":                # two normal fluids with the drag's share of the conversion, substeps
        md = _mgb2()
        st = T.Stepper.make(md, gr, wedge, rkl=False, drag=0.3, qp_exchange=1.0, **kw)
    elif kind == "qp_drag_rkc":            # the same on damped RKC stages with KWT and the frame
        md = _mgb2(γkwt=10.0)
        st = T.Stepper.make(md, gr, wedge, drag=0.05, qp_exchange=1.0, **kw)
    elif kind == "qp_substeps":            # two normal fluids on Euler substeps, a split given, the slab field
        md = _mgb2()
        st = T.Stepper.make(md, gr, wedge, rkl=False, selffield_bc="slab", qp_exchange=0.5, qp_split=(0.3, 0.7),
                            **kw)
    elif kind == "qp_pcg":                 # two normal fluids on the bar of the sample (insulating padding, PCG)
        gr = T.Grid.make(16, 8, 4, dx=0.5, buf=2)
        mk = T.build_masks(T.GeomSpec(GEOM_MODE="WEDGE"), gr)
        md = _mgb2(γkwt=10.0)
        st = T.Stepper.make(md, gr, mk, σvac=0.01, pcg_tol=1e-10, qp_exchange=2.0, **kw)
    elif kind == "qp_matrix2":             # two bands' fluids as a matrix of rates (QPExchangeN), RKL stages
        md = _mgb2()
        b = md.bands
        sh = [T.stiffness(x) * x.Γ / x.β for x in b]
        χ = [sh[µ] / sum(sh) * md.σn * b[µ].Γ / T.stiffness(b[µ]) for µ in range(2)]
        st = T.Stepper.make(md, gr, wedge, rkl=True, qp_exchange=[[0.0, 1.5], [1.5 * χ[0] / χ[1], 0.0]], **kw)
    elif kind == "qp_heat":                # two normal fluids with the heat model's Joule term (qp_joule)
        md = _mgb2(γkwt=3.0)
        st = T.Stepper.make(md, gr, wedge, heat=T.Heat(eta=0.5, joule=True), qp_exchange=1.0, **kw)
    elif kind == "qp_three":               # three fluids, a different conductance per pair, KWT on one band
        bands = (T.Band.make(), T.Band.make(m=2.0, Γ=1.2, a=0.8, γkwt=5.0), T.Band.make(m=0.7, Γ=0.9, a=0.6))
        γ = [[0.0, -0.1, -0.05], [-0.1, 0.0, -0.08], [-0.05, -0.08, 0.0]]
        md = T.Model.make(bands, γ, κ=2.0)
        sh = [T.stiffness(x) * x.Γ / x.β for x in bands]
        χ = [sh[µ] / sum(sh) * md.σn * bands[µ].Γ / T.stiffness(bands[µ]) for µ in range(3)]
        Gp = [[0.0, 0.5, 0.1], [0.5, 0.0, 2.0], [0.1, 2.0, 0.0]]
        st = T.Stepper.make(md, gr, wedge, qp_exchange=[[0.0 if µ == n else Gp[µ][n] / χ[µ] for n in range(3)]
                                                        for µ in range(3)], **kw)
    else:
        raise KeyError(kind)
    s = T.initial_state(st.model, st.grid, st.masks, H)
    return st, s, H, T.selffield(st, 0.3)


SMALL_KINDS = ("euler_substeps", "rkl_bar", "rkc_kwt_rotframe", "kwt_substeps_rotframe", "kwt_euler_rotframe",
               "explicit_scale", "pcg", "pcg_fast", "pcg_f32", "open", "open_pcg", "three_bands", "hard",
               "drag_substeps", "drag_rkc_kwt", "drag_three", "heat_joule", "qp_rkc_kwt", "qp_substeps", "qp_pcg",
               "qp_matrix2", "qp_three", "qp_heat", "qp_drag", "qp_drag_rkc")

# noisy variants of the small cases (kind, Stepper.make arguments): the Cartesian kick (no KWT), SK-ROCK with the
# low-passed frame and the log-polar combination (KWT on RKC stages), the polar kick on KWT substeps and on one Euler
# pass, three bands mixing both, and the field kick with the conductivity per link of the PCG padding
NOISY = {"euler_substeps": dict(noise=1e-3, noise_seed=7),
         "rkc_kwt_rotframe": dict(noise=1e-3, noise_seed=8),
         "kwt_substeps_rotframe": dict(noise=1e-3, noise_seed=9),
         "kwt_euler_rotframe": dict(noise=1e-3, noise_seed=10),
         "three_bands": dict(noise=1e-3, noise_seed=11, noise_field=True),
         "pcg_f32": dict(noise=1e-3, noise_seed=12, noise_field=True),
         "hard": dict(noise=1e-3, noise_seed=13),
         "qp_rkc_kwt": dict(noise=1e-3, noise_seed=14)}


def copy_model(m, σn=None, bands=None):
    """The same material as a separate model (test_materials.jl:7), optionally with another σn or other bands."""
    return T.Model.make(m.bands if bands is None else bands, m.γ, κ=m.κ, σn=m.σn if σn is None else σn, T=m.T)


def material(kind: str, **kw):
    """Small cases of material per region (materials.jl), (Stepper, State, H, HJ): 24×12×4 cells, the WEDGE notch,
    the second material on the slab x > x1 + 12 unless stated."""
    gr = T.Grid.make(24, 12, 4, dx=0.5)
    wedge = T.build_masks(T.GeomSpec(GEOM_MODE="WEDGE", inj_margin=4), gr)
    half = with_materials(wedge, gr, lambda i, j, k: 2 if i > gr.x1 + 12 else 1)
    H, J = 0.03, 0.4
    md = _mgb2()
    if kind == "mat_two":                  # another σ band and a barrier of transparency 0.5
        m2 = T.Model.make((T.Band.make(m=1.5, a=0.7, Γ=1.3), md.bands[1]), md.γ, κ=2.0)
        st = T.Stepper.make(md, gr, half, materials=[m2], transparency=[[1.0, 0.5], [0.5, 1.0]], **kw)
    elif kind == "mat_three_kwt":          # three slabs, KWT in the middle one only (RKC stages, rotating frame)
        three = with_materials(wedge, gr, lambda i, j, k: 1 if i <= gr.x1 + 8 else (2 if i <= gr.x1 + 16 else 3))
        b1, b2 = md.bands
        m2 = T.Model.make((T.Band.make(m=1.2, a=0.9, γkwt=10.0), T.Band.make(m=b2.m, Γ=b2.Γ, a=0.5, γkwt=10.0)),
                          [[0.0, 2e-3], [2e-3, 0.0]], κ=2.0)
        m3 = T.Model.make((T.Band.make(m=0.8, a=0.6, Γ=0.7), b2), md.γ, κ=2.0)
        st = T.Stepper.make(md, gr, three, materials=[m2, m3],
                            transparency=[[1.0, 0.3, 1.0], [0.3, 1.0, 0.6], [1.0, 0.6, 1.0]], **kw)
    elif kind == "mat_absent":             # a one-band metal: band 2 absent from the second material
        metal = T.Model.make((T.Band.make(a=-0.5), T.Band.make(m=md.bands[1].m, a=-1.0)), [[0.0, 0.0], [0.0, 0.0]],
                             κ=2.0)
        st = T.Stepper.make(md, gr, half, materials=[metal], absent=[[], [2]], **kw)
    elif kind == "mat_sigma":              # σn per region: the field solve takes the PCG path without padding
        st = T.Stepper.make(md, gr, half, materials=[copy_model(md, σn=0.25)], pcg_tol=1e-10, **kw)
    elif kind == "mat_aniso":              # anisotropic bands, masses per axis changing across the interface
        a1 = T.Model.make((T.Band.make(m_axes=(1.0, 2.0, 0.5)), T.Band.make(m=0.106, a=0.59)),
                          [[0.0, 1e-3], [1e-3, 0.0]], κ=2.0)
        a2 = T.Model.make((T.Band.make(m_axes=(1.5, 0.7, 3.0), a=0.6, Γ=1.3), T.Band.make(m=0.2, a=0.5)),
                          [[0.0, 1e-3], [1e-3, 0.0]], κ=2.0)
        md = a1
        st = T.Stepper.make(a1, gr, half, materials=[a2], **kw)
    elif kind == "mat_heat":               # the heat model with two materials and the Joule term (one D_T)
        m2 = T.Model.make((T.Band.make(m=1.5, a=0.7, Γ=1.3, γkwt=2.0), md.bands[1]), md.γ, κ=2.0, σn=0.7)
        st = T.Stepper.make(md, gr, half, materials=[m2], heat=T.Heat(eta=0.5, joule=True, margin=2), pcg_tol=1e-10,
                            **kw)
    elif kind == "mat_heat_dt":            # D_T per material: the Jacobi update with harmonic means on the links
        m2 = T.Model.make((T.Band.make(m=1.5, a=0.7, Γ=1.3), md.bands[1]), md.γ, κ=2.0)
        st = T.Stepper.make(md, gr, half, materials=[m2], heat=T.Heat(eta=0.5, joule=True), heat_DT=[0.25, 0.6],
                            **kw)
    else:
        raise KeyError(kind)
    s = T.initial_state(st.model, st.grid, st.masks, H, materials=st.mt.models)
    return st, s, H, T.selffield(st, J)


MATERIAL_KINDS = ("mat_two", "mat_three_kwt", "mat_absent", "mat_sigma", "mat_aniso", "mat_heat", "mat_heat_dt")
# noise with materials: the per-material Cartesian kick, and SK-ROCK with KWT in one material and the field kick
MATERIAL_NOISY = {"mat_two": dict(noise=1e-3, noise_seed=21),
                  "mat_three_kwt": dict(noise=1e-3, noise_seed=22, noise_field=True),
                  "mat_absent": dict(noise=1e-3, noise_seed=23)}


def vacuum(kind: str, **kw):
    """Small sculpted samples (a shape with vacuum, sculpt!, geometry.jl:537-557), (Stepper, State, H, HJ): 16×8×6
    cells with a 2-cell insulating buffer (σvac = 0.01: PCG), a vacuum slot through the bar from the y1 face."""
    from juliatdgl_b200.grid import sculpt
    gr = T.Grid.make(16, 8, 6, dx=0.5, buf=2)
    v = np.zeros(gr.node, dtype=bool)
    v[gr.x1 + 4:gr.x1 + 8, gr.y1:gr.y1 + 3, gr.z1:gr.z2] = True
    mk = sculpt(T.box_masks(gr), gr, v)
    H, J = 0.03, 0.3
    if kind == "vac_plain":
        md = _mgb2()
        st = T.Stepper.make(md, gr, mk, σvac=0.01, pcg_tol=1e-10, **kw)
    elif kind == "vac_kwt":             # KWT with RKC stages and the rotating frame
        md = _mgb2(γkwt=10.0)
        st = T.Stepper.make(md, gr, mk, σvac=0.01, pcg_tol=1e-10, **kw)
    elif kind == "vac_open":            # the open boundary over the section of the sample
        md = _mgb2()
        st = T.Stepper.make(md, gr, mk, σvac=0.01, pcg_tol=1e-10, selffield_bc="open", open_every=0.2, **kw)
    elif kind == "vac_qp":              # two normal fluids: δ by conjugate gradients over the cut links (QPSolve)
        md = _mgb2(γkwt=10.0)
        st = T.Stepper.make(md, gr, mk, σvac=0.01, pcg_tol=1e-10, qp_exchange=1.0, **kw)
    elif kind == "vac_qpn":             # the same two fluids as a matrix of rates: each mode by conjugate gradients
        md = _mgb2(γkwt=10.0)
        st = T.Stepper.make(md, gr, mk, σvac=0.01, pcg_tol=1e-10, qp_exchange=1.0, **kw)
        q = st.qpx
        χ = [q.s[µ] * md.σn * md.bands[µ].Γ / T.stiffness(md.bands[µ]) for µ in range(2)]
        st = T.Stepper.make(md, gr, mk, σvac=0.01, pcg_tol=1e-10, qp_exchange=[[0.0, 1.0], [χ[0] / χ[1], 0.0]], **kw)
    elif kind == "vac_mat":             # two materials around the slot
        md = _mgb2()
        mk = with_materials(mk, gr, lambda i, j, k: 2 if i > gr.x1 + 8 else 1)
        m2 = T.Model.make((T.Band.make(m=1.5, a=0.7, Γ=1.3), md.bands[1]), md.γ, κ=2.0)
        st = T.Stepper.make(md, gr, mk, σvac=0.01, pcg_tol=1e-10, materials=[m2], **kw)
    else:
        raise KeyError(kind)
    s = T.initial_state(st.model, st.grid, st.masks, H, materials=st.mt.models if st.mt is not None else None)
    return st, s, H, T.selffield(st, J)


VACUUM_KINDS = ("vac_plain", "vac_kwt", "vac_open", "vac_mat", "vac_qp", "vac_qpn")


def maxrel(a, b):
    d = np.max(np.abs(a - b))
    m = np.max(np.abs(b))
    return d if m == 0 else d / m


def compare_states(a: State, b: State):
    """Largest relative difference per field group (gpu/TDGLGPU/test/compare_cpu.jl:90-96): Ψ_µ against its own
    size, each vector field (θ, φ, h, J) against the size of the whole vector; returns (worst, {name: value})."""
    out = {}
    for µ in range(a.N):
        out[f"G{µ + 1}"] = maxrel(a.G[µ], b.G[µ])
        out[f"F{µ + 1}"] = maxrel(a.F[µ], b.F[µ])
    for grp in (("θx", "θy", "θz"), ("φx", "φy", "φz"), ("hx", "hy", "hz"), ("Jx", "Jy", "Jz"),
                ("Ux", "Uy", "Uz"), ("Vx", "Vy", "Vz")):
        m = max(np.max(np.abs(getattr(b, q))) for q in grp)
        for q in grp:
            d = np.max(np.abs(getattr(a, q) - getattr(b, q)))
            out[q] = d if m == 0 else d / m
    k = max(out, key=out.get)
    return out[k], out
