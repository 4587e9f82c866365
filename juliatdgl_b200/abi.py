"""ctypes mirror of ``include/tdgl_b200.h`` and the packing of a host ``Stepper`` / ``State`` into it.

This is the Python equivalent of the ``ccall`` shim a Julia host uses (a ``TDGLB200`` module next to the
reference's ``gpu/TDGLGPU``): the Stepper's fields become a ``tdgl_params``, the State's arrays a ``tdgl_state_view``
of host pointers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .model import stiffness
from .scheme import BC_SLAB, SOLVER_PCG, SOLVER_SCALE, QPExchange, Stepper, sep_ranges

ABI_VERSION = 8
MAXB = 8
MAXSTG = 64
MAXMAT = 8

E_OK, E_INVAL, E_NOMEM, E_CUDA, E_NOCONV, E_DIVERGED, E_STATE = 0, -1, -2, -3, -4, -5, -6
ERRNAMES = {E_INVAL: "EINVAL", E_NOMEM: "ENOMEM", E_CUDA: "ECUDA", E_NOCONV: "ENOCONV", E_DIVERGED: "EDIVERGED",
            E_STATE: "ESTATE"}

dptr = C.POINTER(C.c_double)


class Grid_t(C.Structure):
    _fields_ = [("Nx", C.c_int32), ("Ny", C.c_int32), ("Nz", C.c_int32),
                ("x1", C.c_int32), ("x2", C.c_int32), ("y1", C.c_int32), ("y2", C.c_int32),
                ("z1", C.c_int32), ("z2", C.c_int32), ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double)]


class BandCoef_t(C.Structure):
    _fields_ = [("kx", C.c_double), ("ky", C.c_double), ("kz", C.c_double), ("c", C.c_double),
                ("eps", C.c_double), ("beta", C.c_double), ("gamma2", C.c_double), ("cpl", C.c_double * MAXB)]


class Materials_t(C.Structure):
    _fields_ = [("nmat", C.c_int32), ("idx", C.POINTER(C.c_uint8)), ("full", (BandCoef_t * MAXB) * MAXMAT),
                ("stage", (BandCoef_t * MAXB) * MAXMAT), ("ma", ((C.c_double * 3) * MAXB) * MAXMAT),
                ("transparency", (C.c_double * MAXMAT) * MAXMAT), ("absent", (C.c_int32 * MAXB) * MAXMAT),
                ("gamma", (C.c_double * MAXB) * MAXMAT),
                ("a", (C.c_double * MAXB) * MAXMAT), ("gk", (C.c_double * MAXB) * MAXMAT),
                ("sigma_n", C.c_double * MAXMAT), ("heat_DT", C.c_double * MAXMAT)]


class Params_t(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("nbands", C.c_int32), ("grid", Grid_t), ("dt", C.c_double),
                ("nsub", C.c_int32 * MAXB), ("stages", C.c_int32 * MAXB), ("use_rkc", C.c_int32 * MAXB),
                ("rkc_q", C.c_double * MAXB), ("rkc_mu", (C.c_double * MAXSTG) * MAXB),
                ("rkc_nu", (C.c_double * MAXSTG) * MAXB), ("rkc_c", (C.c_double * MAXSTG) * MAXB),
                ("rkc_sk", (C.c_double * 2) * MAXB), ("bc", BandCoef_t * MAXB), ("bcs", BandCoef_t * MAXB),
                ("wa", (C.c_double * MAXB) * 3),
                ("d1", C.c_double), ("sxy", C.c_double), ("sxz", C.c_double), ("syx", C.c_double),
                ("syz", C.c_double), ("szx", C.c_double), ("szy", C.c_double), ("a_imp", C.c_double),
                ("solver", C.c_int32), ("selffield_bc", C.c_int32), ("extrap", C.c_int32), ("rotframe", C.c_int32),
                ("hard", C.c_int32),
                ("f", dptr), ("taux", dptr), ("tauy", dptr), ("tauz", dptr),
                ("Dx", dptr), ("Dy", dptr), ("Dz", dptr),
                ("bar_hy_z", dptr), ("bar_hy_y", dptr), ("bar_hz_z", dptr), ("bar_hz_y", dptr), ("bar_hz_x", dptr),
                ("bar_hy_x", dptr),
                ("pcg_tol", C.c_double), ("pcg_maxit", C.c_int32), ("pcg_fast", C.c_int32), ("pcg_f32", C.c_int32),
                ("pcg_extrap", C.c_int32),
                ("open_every", C.c_int32), ("open_R", C.c_int32), ("kappa2", C.c_double), ("open_fac", C.c_double),
                ("open_green", dptr), ("open_jbar", dptr),
                ("noise_on", C.c_int32), ("noise_field", C.c_int32), ("noise_T", C.c_double),
                ("noise_seed", C.c_uint64), ("noise_gamma", C.c_double * MAXB), ("noise_sigma_n", C.c_double),
                ("noise_step0", C.c_int64), ("materials", C.POINTER(Materials_t)), ("vac", C.POINTER(C.c_uint8)),
                ("drag_on", C.c_int32), ("drag_c", ((C.c_double * 3) * MAXB) * MAXB),
                ("drag_nu", (C.c_double * MAXB) * MAXB),
                ("heat_on", C.c_int32), ("heat_joule", C.c_int32), ("heat_margin", C.c_int32),
                ("heat_DT", C.c_double), ("heat_gamma_bath", C.c_double), ("heat_eta", C.c_double),
                ("heat_cap", C.c_double), ("heat_T", C.c_double), ("heat_sigma_n", C.c_double),
                ("heat_a", C.c_double * MAXB),
                ("heat_Gamma", C.c_double * MAXB), ("heat_gk", C.c_double * MAXB),
                ("qp_on", C.c_int32), ("qp_s", C.c_double * MAXB), ("qp_sigma_n", C.c_double),
                ("qp_lambda0", C.c_double), ("qp_g", (C.c_double * 3) * MAXB),
                ("qp_gamma", (C.c_double * MAXB) * MAXB), ("qp_P", (C.c_double * MAXB) * MAXB),
                ("qp_Pinv", (C.c_double * MAXB) * MAXB), ("qp_lam", C.c_double * MAXB),
                ("qp_Gm", (C.c_double * MAXB) * MAXB), ("qp_j0", C.c_int32), ("qp_nj", C.c_int32), ("qp_k0", C.c_int32), ("qp_nk", C.c_int32),
                ("qp_Vx", dptr), ("qp_Wx", dptr), ("qp_ex", dptr), ("qp_Vy", dptr), ("qp_Wy", dptr),
                ("qp_ey", dptr), ("qp_Vz", dptr), ("qp_Wz", dptr), ("qp_ez", dptr),
                ("qp_cond", C.POINTER(C.c_uint8)), ("qp_tol", C.c_double), ("qp_maxit", C.c_int32),
                ("qp_cx", dptr), ("qp_cy", dptr), ("qp_cz", dptr), ("qp_lamv", dptr), ("qp_d", C.c_double),
                ("qp_mgamma", ((C.c_double * 2) * 2) * MAXMAT)]


class StateView_t(C.Structure):
    _fields_ = [("G", dptr * MAXB), ("F", dptr * MAXB), ("th", dptr * 3), ("ph", dptr * 3), ("U", dptr * 3),
                ("V", dptr * 3), ("J", dptr * 3), ("h", dptr * 3)]


class CarryView_t(C.Structure):
    _fields_ = [("pcg_x", dptr), ("pcg_xprev", dptr), ("pcg_warm", C.c_int32), ("pcg_have2", C.c_int32),
                ("open_count", C.c_int32), ("open_old", dptr * 3), ("open_new", dptr * 3), ("open_theta", dptr * 3),
                ("heat_theta", dptr)]


class Stats_t(C.Structure):
    _fields_ = [("steps", C.c_int64), ("pcg_last_iters", C.c_int32), ("pcg_total_iters", C.c_int64),
                ("open_recomputes", C.c_int32), ("kernel_launches_last_call", C.c_int32),
                ("qp_cg_total_iters", C.c_int64)]


class Meter_t(C.Structure):
    _fields_ = [("vi", C.c_int32), ("vo", C.c_int32), ("nphase", C.c_int32), ("Min", C.POINTER(C.c_uint8)),
                ("Mou", C.POINTER(C.c_uint8)), ("line_ok", C.POINTER(C.c_uint8))]


class Obs_t(C.Structure):
    _fields_ = [("D", dptr * MAXB), ("vsum_in", C.c_double), ("vsum_out", C.c_double), ("ta_sum", C.c_double),
                ("res", C.c_double * MAXB), ("amax", C.c_double), ("diffh", C.c_double), ("Itot", C.c_double),
                ("Isam", C.c_double)]


def _ptr(a: np.ndarray):
    assert a.flags["F_CONTIGUOUS"] or a.ndim <= 1, "arrays must be column-major"
    assert a.dtype in (np.float64, np.complex128)
    return a.ctypes.data_as(dptr)


def pack_params(st: Stepper):
    """tdgl_params of a Stepper, and the arrays that must outlive the call that reads it."""
    gr, md = st.grid, st.model
    N = md.N
    if N > MAXB:
        raise ValueError(f"at most {MAXB} bands")
    keep = []

    def setcoef(dst, b):
        dst.kx, dst.ky, dst.kz, dst.c = b.kx, b.ky, b.kz, b.c
        dst.eps, dst.beta, dst.gamma2 = b.ε, b.β, b.γ2
        for ν in range(N):
            dst.cpl[ν] = b.cpl[ν]

    def arr(a):
        a = np.asfortranarray(np.asarray(a, dtype=np.float64))
        keep.append(a)
        return _ptr(a)

    p = Params_t()
    p.abi_version = ABI_VERSION
    p.nbands = N
    p.grid = Grid_t(gr.Nx, gr.Ny, gr.Nz, gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2, gr.dx, gr.dy, gr.dz)
    p.dt = st.dt
    for µ in range(N):
        p.nsub[µ] = st.nsub[µ]
        p.stages[µ] = st.rkl[µ]
        rc = st.rkc[µ] if st.rkc is not None else None
        if st.rkl[µ] > MAXSTG:
            raise ValueError(f"band {µ + 1}: {st.rkl[µ]} stages, at most {MAXSTG}")
        if rc is not None:
            p.use_rkc[µ] = 1
            p.rkc_q[µ] = rc.q
            for j in range(len(rc.μ)):
                p.rkc_mu[µ][j] = rc.μ[j]
                p.rkc_nu[µ][j] = rc.ν[j]
                p.rkc_c[µ][j] = rc.c[j]
            p.rkc_sk[µ][0], p.rkc_sk[µ][1] = rc.sk
        setcoef(p.bc[µ], st.bc[µ])
        setcoef(p.bcs[µ], st.bcs[µ])
        for ax in range(3):
            p.wa[ax][µ] = st.wa[ax][µ]
    fc = st.fc
    p.d1, p.sxy, p.sxz, p.syx, p.syz, p.szx, p.szy, p.a_imp = fc.d1, fc.sxy, fc.sxz, fc.syx, fc.syz, fc.szx, fc.szy, fc.a
    p.solver = st.solver
    p.selffield_bc = st.selffield_bc
    p.extrap, p.rotframe, p.hard = int(st.extrap), int(st.rotframe), int(st.hard)
    mk = st.masks
    p.f, p.taux, p.tauy, p.tauz = arr(mk.f), arr(mk.τx), arr(mk.τy), arr(mk.τz)
    if st.D is not None:
        p.Dx, p.Dy, p.Dz = arr(st.D[0]), arr(st.D[1]), arr(st.D[2])
    if st.bar is not None:
        b = st.bar
        p.bar_hy_z, p.bar_hy_y, p.bar_hz_z = arr(b.hy_z), arr(b.hy_y), arr(b.hz_z)
        p.bar_hz_y, p.bar_hz_x, p.bar_hy_x = arr(b.hz_y), arr(b.hz_x), arr(b.hy_x)
    if st.pcg is not None:
        p.pcg_tol, p.pcg_maxit = st.pcg.tol, st.pcg.maxit
        p.pcg_fast, p.pcg_f32, p.pcg_extrap = int(st.pcg.fast), int(st.pcg.f32), int(st.pcg.extrap)
    if st.open is not None:
        o = st.open
        p.open_every, p.open_R, p.open_fac = o.every, o.R, o.fac
        p.open_green = arr(o.G)
        p.open_jbar = arr(o.Jbar)
    p.kappa2 = md.κ * md.κ
    if st.noise_T is not None:
        p.noise_on, p.noise_field, p.noise_T, p.noise_seed = 1, int(st.noise_field), st.noise_T, st.noise_seed
        for mu, b in enumerate(md.bands):
            p.noise_gamma[mu] = b.Γ
        p.noise_sigma_n = md.σn
        p.noise_step0 = int(st.noise_step0)
    if st.drag is not None:
        p.drag_on = 1
        for µ in range(N):
            for ν in range(N):
                p.drag_nu[µ][ν] = st.dragν[µ][ν]
                for ax in range(3):
                    p.drag_c[µ][ν][ax] = st.drag[µ][ν][ax]
    if st.heat is not None:
        h = st.heat
        p.heat_on, p.heat_joule, p.heat_margin = 1, int(h.joule), int(h.margin)
        p.heat_DT, p.heat_gamma_bath, p.heat_eta, p.heat_cap, p.heat_T = h.D_T, h.gamma_bath, h.eta, h.cap, md.T
        p.heat_sigma_n = md.σn
        for µ, b in enumerate(md.bands):
            p.heat_a[µ], p.heat_Gamma[µ], p.heat_gk[µ] = b.a, b.Γ, b.γkwt
    if st.qpx is not None:   # exchange.jl: QPExchange (two bands, δ) or QPExchangeN (N fluids)
        q = st.qpx
        two = isinstance(q, QPExchange)
        p.qp_on = 1 if two else 2
        for µ in range(N):
            p.qp_s[µ] = q.s[µ]
        p.qp_sigma_n = q.σn
        p.qp_lambda0 = q.λ0 if two else 0.0
        for µ, b in enumerate(md.bands):
            for ax in range(3):
                p.qp_g[µ][ax] = stiffness(b, ax + 1)
            for ν in range(N):
                p.qp_gamma[µ][ν] = md.γ[µ][ν]
        if two:
            p.qp_Gm[0][1] = q.G
        else:
            for a in range(N):
                p.qp_lam[a] = q.λ[a]
                for c in range(N):
                    p.qp_Gm[a][c] = q.Gm[a, c]
                for c in range(N):
                    p.qp_P[a][c] = q.P[a, c]
                    p.qp_Pinv[a][c] = q.Pinv[a, c]
        p.qp_j0, p.qp_nj, p.qp_k0, p.qp_nk = q.j0, q.nj, q.k0, q.nk
        p.qp_Vx, p.qp_Vy, p.qp_Vz = (arr(a) for a in q.V)
        p.qp_Wx, p.qp_Wy, p.qp_Wz = (arr(a) for a in q.W)
        p.qp_ex, p.qp_ey, p.qp_ez = (arr(a) for a in q.e)
        var = q.var if two else None
        if q.cond is not None or var is not None:   # the conjugate-gradient solve of δ (of each mode)
            typ = np.asfortranarray(var.typ if var is not None else q.cond, dtype=np.uint8)
            keep.append(typ)
            p.qp_cond = typ.ctypes.data_as(C.POINTER(C.c_uint8))
            p.qp_tol, p.qp_maxit = q.tol, q.maxit
            if var is not None:   # QPVar: the variable coefficients
                p.qp_cx, p.qp_cy, p.qp_cz, p.qp_lamv = (arr(a) for a in (var.cx, var.cy, var.cz, var.λ))
                p.qp_d = var.d
        if two and st.mt is not None:   # the Josephson matrix of each material (_conv at its nodes)
            for m, mm in enumerate(st.mt.models):
                for µ in range(2):
                    for ν in range(2):
                        p.qp_mgamma[m][µ][ν] = mm.γ[µ][ν]
    if st.masks.vac is not None:
        vac = np.asfortranarray(st.masks.vac, dtype=np.uint8)
        keep.append(vac)
        p.vac = vac.ctypes.data_as(C.POINTER(C.c_uint8))
    if st.mt is not None:
        mt = st.mt
        M = len(mt.models)
        if M > MAXMAT:
            raise ValueError(f"at most {MAXMAT} materials")
        m = Materials_t()
        m.nmat = M
        idx = np.asfortranarray(mt.idx, dtype=np.uint8)
        keep.append(idx)
        m.idx = idx.ctypes.data_as(C.POINTER(C.c_uint8))
        for a, md_a in enumerate(mt.models):
            for µ in range(N):
                setcoef(m.full[a][µ], mt.full[µ][a])
                setcoef(m.stage[a][µ], mt.stage[µ][a])
                for ax in range(3):
                    m.ma[a][µ][ax] = md_a.bands[µ].ma[ax]
                m.absent[a][µ] = int(mt.absent[a, µ])
                m.gamma[a][µ] = md_a.bands[µ].Γ
                m.a[a][µ] = md_a.bands[µ].a
                m.gk[a][µ] = md_a.bands[µ].γkwt
            for b in range(M):
                m.transparency[a][b] = mt.t[a, b]
            m.sigma_n[a] = md_a.σn
            m.heat_DT[a] = st.heat_DT[a] if st.heat_DT is not None else 0.0
        keep.append(m)
        p.materials = C.pointer(m)
    return p, keep


def state_view(s) -> StateView_t:
    v = StateView_t()
    for µ in range(s.N):
        v.G[µ] = _ptr(s.G[µ])
        v.F[µ] = _ptr(s.F[µ])
    for ax, c in enumerate("xyz"):
        v.th[ax] = _ptr(getattr(s, "θ" + c))
        v.ph[ax] = _ptr(getattr(s, "φ" + c))
        v.U[ax] = _ptr(getattr(s, "U" + c))
        v.V[ax] = _ptr(getattr(s, "V" + c))
        v.J[ax] = _ptr(getattr(s, "J" + c))
        v.h[ax] = _ptr(getattr(s, "h" + c))
    return v


class Carry:
    """Host copy of the carry (PCG warm start, open ramp) of one context."""

    def __init__(self, st: Stepper):
        gr = st.grid
        n = 0
        for r in sep_ranges(gr):
            m = 1
            for a, b in r:
                m *= b - a + 1
            n += m
        self.pcg_x = np.zeros(n)
        self.pcg_xprev = np.zeros(n)
        self.pcg_warm = 0
        self.pcg_have2 = 0
        self.open_count = -1
        self.open_old = [np.zeros(s, order="F") for s in (gr.hx_shape, gr.hy_shape, gr.hz_shape)]
        self.open_new = [np.zeros(s, order="F") for s in (gr.hx_shape, gr.hy_shape, gr.hz_shape)]
        self.open_theta = [np.zeros(s, order="F") for s in (gr.xlink, gr.ylink, gr.zlink)]
        # the temperature field (Stepper.heat.θ, scheme.jl:403: the bath everywhere at the start)
        self.heat_theta = None if st.heat is None else np.full((gr.Nx + 1, gr.Ny + 1, gr.Nz + 1), float(st.model.T), order="F")

    def view(self) -> CarryView_t:
        v = CarryView_t()
        v.pcg_x = _ptr(self.pcg_x)
        v.pcg_xprev = _ptr(self.pcg_xprev)
        v.pcg_warm = self.pcg_warm
        v.pcg_have2 = self.pcg_have2
        v.open_count = self.open_count
        for ax in range(3):
            v.open_old[ax] = _ptr(self.open_old[ax])
            v.open_new[ax] = _ptr(self.open_new[ax])
            v.open_theta[ax] = _ptr(self.open_theta[ax])
        if self.heat_theta is not None:
            v.heat_theta = _ptr(self.heat_theta)
        return v

    def absorb(self, v: CarryView_t):
        self.pcg_warm, self.pcg_have2, self.open_count = v.pcg_warm, v.pcg_have2, v.open_count
