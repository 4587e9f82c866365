"""The Stepper: time step, stage counts and coefficients of the update (host side).

Restates the constructor of ``gtdgl/src/scheme.jl`` (``Stepper`` :250-434) for one material: the stability
bounds (``_psi2_bound`` :38-52, ``_band_bounds`` :107-137), dt (:299-322), the automatic substeps
(:306-311), the RKL1 / damped-RKC1 stage counts (:326-366, ``RKCCoef`` :77-104), ``BandCoef`` (:21-28,
``_bandcoef`` :141-147, ``_divided`` :63-64) and ``FieldCoef`` (:149-153, :374-379); the insulating padding's
link conductivity (``gtdgl/src/implicit.jl:126-140``); the field of the bar current on the outer faces
(``bar_field``, ``gtdgl/src/field.jl:151-180``); and the set-up of the open boundary (``OpenBC``,
``gtdgl/src/openbc.jl:63-136``: the lattice Green table, the ramp interval, the bar current J_bar).

These are host decisions in the reference as well; the kernels receive them through the C-ABI
(``include/tdgl_b200.h``).  Every scalar expression keeps the reference's order of operations, so the
coefficients are the reference's to the bit (pinned by the release-1.2 regression parameters).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np

from .grid import Grid, Masks, conducting_nodes, dl, slab_thickness
from .model import Model, equilibrium, eps_band, isotropic, stiffness

RKC_EPS = 0.5
ROT_MIN2 = 1e-3
ROT_MAXDT = 0.5


# ----------------------------------------------------------------------------------------- coefficients
@dataclass(frozen=True)
class BandCoef:
    """kx, ky, kz, c = dt/Γ, ε, β, the Josephson row cpl and γ̃² (scheme.jl:21-28)."""
    kx: float
    ky: float
    kz: float
    c: float
    ε: float
    β: float
    cpl: Tuple[float, ...]
    γ2: float


def _divided(b: BandCoef, n) -> BandCoef:
    return BandCoef(b.kx / n, b.ky / n, b.kz / n, b.c / n, b.ε, b.β, tuple(x / n for x in b.cpl), b.γ2)


def _bandcoef(md: Model, µ: int, dt, rx, ry, rz, mref) -> BandCoef:
    b = md.bands[µ - 1]
    c = dt / b.Γ
    Γh = dt / c
    return BandCoef(rx / (mref[0] * Γh), ry / (mref[1] * Γh), rz / (mref[2] * Γh), c, eps_band(md, µ), b.β,
                    tuple((dt / Γh) * md.γ[µ - 1][ν] for ν in range(md.N)), b.γkwt * b.γkwt)


@dataclass(frozen=True)
class FieldCoef:
    d1: float
    sxy: float
    sxz: float
    syx: float
    syz: float
    szx: float
    szy: float
    a: float


def _rkc_cheb(s: int, ω0: float):
    """(T_s(ω₀), T_s'(ω₀)) (scheme.jl:82-89)."""
    if s == 0:
        return (1.0, 0.0)
    T0, T1, d0, d1 = 1.0, ω0, 0.0, 1.0
    for _ in range(2, s + 1):
        T0, T1, d0, d1 = T1, 2 * ω0 * T1 - T0, d1, 2 * T1 + 2 * ω0 * d1 - d0
    return T1, d1


@dataclass(frozen=True)
class RKCCoef:
    q: float
    μ: Tuple[float, ...]
    ν: Tuple[float, ...]
    c: Tuple[float, ...]
    sk: Tuple[float, float]

    @staticmethod
    def make(s: int, ε: float = RKC_EPS) -> "RKCCoef":
        """scheme.jl:90-100."""
        ω0 = 1 + ε / (s * s)
        Ts, dTs = _rkc_cheb(s, ω0)
        ω1 = Ts / dTs
        μ = [1.0] * s
        ν = [0.0] * s
        c = [0.0] * s
        for j in range(1, s + 1):
            Tj, dTj = _rkc_cheb(j, ω0)
            c[j - 1] = ω1 * dTj / Tj
            if j >= 2:
                μ[j - 1] = 2 * ω0 * _rkc_cheb(j - 1, ω0)[0] / Tj
                ν[j - 1] = -_rkc_cheb(j - 2, ω0)[0] / Tj
        c[s - 1] = 1.0
        return RKCCoef(ω0 / ω1, tuple(μ), tuple(ν), tuple(c), (s * ω1 / 2, s * ω1 / ω0))


def _rkc_ratio(s: int, ε: float = RKC_EPS) -> float:
    ω0 = 1 + ε / (s * s)
    Ts, dTs = _rkc_cheb(s, ω0)
    return (1 + ω0) / (2 * Ts / dTs)


def _lsum(values):
    """Julia's sum over a tuple / short range: a left fold from the first element."""
    out = None
    for v in values:
        out = v if out is None else out + v
    return out


def _psi2_bound(md: Model):
    """scheme.jl:38-52."""
    b = md.bands
    N = md.N
    p = tuple(math.sqrt(max(eps_band(md, µ + 1), 0.0) / b[µ].β) + 1e-3 for µ in range(N))
    done = False
    for _ in range(10_000):
        q = []
        for µ in range(N):
            c = _lsum(0.0 if ν == µ else abs(md.γ[µ][ν]) * p[ν] for ν in range(N)) / p[µ]
            q.append(0.5 * p[µ] + 0.5 * math.sqrt(max(eps_band(md, µ + 1) + c, 0.0) / b[µ].β))
        q = tuple(q)
        if max(abs(a - bb) for a, bb in zip(q, p)) < 1e-13:
            p = q
            done = True
            break
        p = q
    if not done:
        p = equilibrium(md)
    out = []
    for µ in range(N):
        if p[µ] < 2e-3 and all(ν == µ or md.γ[µ][ν] == 0 for ν in range(N)):
            out.append(max(eps_band(md, µ + 1), 0.0) / b[µ].β)
        else:
            out.append(p[µ] * p[µ])
    return tuple(out)


def _band_bounds(md: Model, gr: Grid, l: float, present=None):
    """(bb0, bbk, λL) of scheme.jl:107-137; `present` (per band) drops the bands a material lacks."""
    bands = md.bands
    N = md.N
    P2 = []
    for p, bd in zip(_psi2_bound(md), bands):
        q = bd.a / bd.β
        P2.append(q if (q > 0 and p <= 1.01 * q) else p)
    hr = []
    for µ in range(N):
        bd = bands[µ]
        if P2[µ] == bd.a / bd.β and bd.β == 1:
            hr.append(2 * (bd.a / bd.β))
        else:
            hr.append(max(3 * bd.β * P2[µ] - eps_band(md, µ + 1), 0.0))
    dif = []
    for bd in bands:
        if isotropic(bd):
            dif.append(8 / (l * bd.m))
        else:
            dif.append(4 * (1 / (bd.ma[0] * (gr.dx * gr.dx)) + 1 / (bd.ma[1] * (gr.dy * gr.dy))
                            + 1 / (bd.ma[2] * (gr.dz * gr.dz))))
    bb0 = tuple(2 * bands[µ].Γ / (dif[µ] + hr[µ]) for µ in range(N))
    bbk = tuple(bb0[µ] / math.sqrt(1 + (bands[µ].γkwt * bands[µ].γkwt) * P2[µ]) if bands[µ].γkwt > 0 else bb0[µ]
                for µ in range(N))
    ns = [bd.a / bd.β if bd.a > 0 else P2[µ] for µ, bd in enumerate(bands)]
    if present is None or all(present):
        λL = _lsum((stiffness(bd) if isotropic(bd) else 1 / min(bd.ma)) * ns[µ] for µ, bd in enumerate(bands))
        return bb0, bbk, λL
    λL = _lsum((stiffness(bd) if isotropic(bd) else 1 / min(bd.ma)) * ns[µ] if present[µ] else 0.0
               for µ, bd in enumerate(bands))
    return (tuple(bb0[µ] if present[µ] else math.inf for µ in range(N)),
            tuple(bbk[µ] if present[µ] else math.inf for µ in range(N)), λL)


# ----------------------------------------------------------------------------------------- padding, bar
def link_conductivity(gr: Grid, σvac: float, σn: float, cond=None):
    """σ_l/σ_n on every link (implicit.jl:126-140): 1 inside the bar y1:y2+1 × z1:z2+1, σvac/σn elsewhere; with
    `cond` (the conducting nodes of a sculpted sample) 1 where both ends conduct."""
    r = σvac / σn
    Nx, Ny, Nz = gr.Nx, gr.Ny, gr.Nz
    if cond is not None:
        c = np.asarray(cond, dtype=bool)
        return (np.asfortranarray(np.where(c[:-1, :, :] & c[1:, :, :], 1.0, r)),
                np.asfortranarray(np.where(c[:, :-1, :] & c[:, 1:, :], 1.0, r)),
                np.asfortranarray(np.where(c[:, :, :-1] & c[:, :, 1:], 1.0, r)))
    j = np.arange(1, Ny + 2)
    k = np.arange(1, Nz + 2)
    iny = (gr.y1 <= j) & (j <= gr.y2 + 1)
    inz = (gr.z1 <= k) & (k <= gr.z2 + 1)
    jj = np.arange(1, Ny + 1)
    kk = np.arange(1, Nz + 1)
    iny_y = (gr.y1 <= jj) & (jj <= gr.y2 + 1) & (gr.y1 <= jj + 1) & (jj + 1 <= gr.y2 + 1)
    inz_z = (gr.z1 <= kk) & (kk <= gr.z2 + 1) & (gr.z1 <= kk + 1) & (kk + 1 <= gr.z2 + 1)
    Dx = np.where(iny[None, :, None] & inz[None, None, :], 1.0, r) * np.ones((Nx, 1, 1))
    Dy = np.where(iny_y[None, :, None] & inz[None, None, :], 1.0, r) * np.ones((Nx + 1, 1, 1))
    Dz = np.where(iny[None, :, None] & inz_z[None, None, :], 1.0, r) * np.ones((Nx + 1, 1, 1))
    return tuple(np.asfortranarray(D) for D in (Dx, Dy, Dz))


# ----------------------------------------------------------------------------------------- materials
def _absent_matrix(absent, M: int, N: int) -> np.ndarray:
    """materials.jl:42-56: None, an M×N bool matrix, or per material the list of its absent (1-based) bands."""
    A = np.zeros((M, N), dtype=bool)
    if absent is not None:
        if isinstance(absent, np.ndarray) and absent.ndim == 2:
            if absent.shape != (M, N):
                raise ValueError(f"absent: a {M}×{N} matrix (materials × bands)")
            A[...] = absent
        else:
            if len(absent) != M:
                raise ValueError(f"absent: one list of bands per material ({M})")
            for m, lst in enumerate(absent):
                for µ in lst:
                    A[m, µ - 1] = True
    if A[0].any():
        raise ValueError("absent: the first material ([material]) has all its bands")
    if any(A[m].all() for m in range(M)):
        raise ValueError("absent: a material keeps at least one band")
    return A


def _check_materials(md: Model, materials, mk: Masks, absent):
    """materials.jl:58-81 (without the heat, drag and exchange options): the models, first the Stepper's."""
    if mk.mat is None:
        raise ValueError('materials: the shape names no material (material = "name" in a region)')
    mats = [md]
    for m in materials:
        if not isinstance(m, Model) or m.N != md.N:
            raise ValueError(f"materials: every material needs {md.N} bands")
        if not (m.κ == md.κ and m.T == md.T):
            raise ValueError("materials: κ and T are those of the sample (the field and the bath); a material gives its "
                             "bands, Josephson matrix and σn")
        if not m.σn > 0:
            raise ValueError("materials: σn must be positive")
        mats.append(m)
    A = _absent_matrix(absent, len(mats), md.N)
    for m in range(1, len(mats)):
        for µ in range(md.N):
            if A[m, µ] and eps_band(mats[m], µ + 1) > 0:
                raise ValueError(f"absent: band {µ + 1} of material {m + 1} has ε = a − T > 0; an absent band has a <= T")
    if int(mk.mat.max()) > len(mats):
        raise ValueError(f"materials: the shape names material {int(mk.mat.max())} of {len(mats)}")
    return mats, A


@dataclass
class MatField:
    """MatField (materials.jl:28-39): the material of each node, the models (the first is the Stepper's), the
    coefficient tables per band [µ][material] (full step and per stage), the transparency of each pair, the absent
    bands (materials × bands)."""
    idx: np.ndarray
    models: Tuple[Model, ...]
    full: Tuple[Tuple[BandCoef, ...], ...]
    stage: Tuple[Tuple[BandCoef, ...], ...]
    t: np.ndarray
    absent: np.ndarray

    @staticmethod
    def make(mats, mk: Masks, gr: Grid, dt, rx, ry, rz, div, transparency=None, absent=None) -> "MatField":
        """materials.jl:83-114: the tables with the first material's masses as m_ref (its links carry the ratio)."""
        M, N = len(mats), mats[0].N
        t = np.ones((M, M)) if transparency is None else np.array(transparency, dtype=np.float64)
        if not (t.shape == (M, M) and np.array_equal(t, t.T) and np.all((0 < t) & (t <= 1))
                and all(t[m, m] == 1 for m in range(M))):
            raise ValueError(f"transparency: a symmetric {M}×{M} matrix in (0, 1] with ones on the diagonal")
        mref = [mats[0].bands[µ].ma for µ in range(N)]
        full = tuple(tuple(_bandcoef(m, µ + 1, dt, rx, ry, rz, mref[µ]) for m in mats) for µ in range(N))
        stage = tuple(full[µ] if div[µ] == 1 else
                      tuple(_divided(_bandcoef(m, µ + 1, dt, rx, ry, rz, mref[µ]), div[µ]) for m in mats)
                      for µ in range(N))
        A = _absent_matrix(None, M, N) if absent is None else absent
        return MatField(np.asfortranarray(mk.mat, dtype=np.uint8), tuple(mats), full, stage, t, A)

    def rho(self, µ: int, ax: int, τ: np.ndarray) -> np.ndarray:
        """The link weights of band µ (1-based) along axis ax (1, 2, 3), τ included (materials.jl:97-110)."""
        idx, mats, t, A = self.idx, self.models, self.t, self.absent
        ρ = np.array(τ, dtype=np.float64, order="F", copy=True)
        m0 = mats[0].bands[µ - 1].ma[ax - 1]
        o = (ax == 1, ax == 2, ax == 3)
        n1, n2, n3 = idx.shape
        for c in np.ndindex(*ρ.shape):
            d = (c[0] + o[0], c[1] + o[1], c[2] + o[2])
            if not (d[0] < n1 and d[1] < n2 and d[2] < n3):
                continue
            a, b = int(idx[c]) - 1, int(idx[d]) - 1
            ma, mb = mats[a].bands[µ - 1].ma[ax - 1], mats[b].bands[µ - 1].ma[ax - 1]
            ml = ma if ma == mb else (ma + mb) / 2
            w = (1.0 if ml == m0 else m0 / ml) * (1.0 if a == b else t[a, b])
            ρ[c] = 0.0 if (A[a, µ - 1] or A[b, µ - 1]) else τ[c] * w
        return ρ


def material_conductivity(gr: Grid, mk: Masks, mats, σvac, σref: float, cond=None):
    """σ_l/σ_ref with σn per region (materials.jl:124-138): the harmonic mean of the two nodes on a conducting
    link, a node outside the block taking the material of the nearest block node; the insulating padding
    (σvac) as link_conductivity.  (Vectorised over the links; the values are the per-link loop's.)"""
    Nx, Ny, Nz = gr.Nx, gr.Ny, gr.Nz
    if σvac is None:
        base = (np.ones((Nx, Ny + 1, Nz + 1), order="F"), np.ones((Nx + 1, Ny, Nz + 1), order="F"),
                np.ones((Nx + 1, Ny + 1, Nz), order="F"))
    else:
        base = tuple(np.array(D, order="F", copy=True) for D in link_conductivity(gr, σvac, σref, cond=cond))
    σs = np.array([m.σn for m in mats])
    # σ of every node (1-based i clamped to x1..x2+1 and so on), over the node box
    ci = np.clip(np.arange(1, Nx + 2), gr.x1, gr.x2 + 1) - 1
    cj = np.clip(np.arange(1, Ny + 2), gr.y1, gr.y2 + 1) - 1
    ck = np.clip(np.arange(1, Nz + 2), gr.z1, gr.z2 + 1) - 1
    sig = σs[mk.mat[np.ix_(ci, cj, ck)].astype(np.int64) - 1]
    for ax, D in enumerate(base):
        n1, n2, n3 = D.shape
        a = sig[:n1, :n2, :n3]
        b = sig[(ax == 0):(ax == 0) + n1, (ax == 1):(ax == 1) + n2, (ax == 2):(ax == 2) + n3]
        with np.errstate(divide="ignore", invalid="ignore"):
            hm = np.where(a == b, a, 2 * a * b / (a + b)) / σref
        cond = D == 1.0                      # insulating links keep σvac
        D[cond] = hm[cond]
    return base


@dataclass
class BarField:
    """The field of the bar current per unit HJ on the outer faces (field.jl:151-180)."""
    hy_z: np.ndarray   # (Ny+1, 2)   hy on the z faces k = 1, Nz
    hy_y: np.ndarray   # (2, Nz)     hy on the y faces j = 1, Ny+1
    hz_z: np.ndarray   # (Ny, 2)     hz on the z faces k = 1, Nz+1
    hz_y: np.ndarray   # (2, Nz+1)   hz on the y faces j = 1, Ny
    hz_x: np.ndarray   # (Ny, Nz+1)  hz on the x faces
    hy_x: np.ndarray   # (Ny+1, Nz)  hy on the x faces


_BAR_CACHE: dict = {}


def _section(gr: Grid, mk: Masks) -> np.ndarray:
    """The section of a sculpted sample at the contact x1 (scheme.jl:54-61): the nodes j in y1:y2+1, k in z1:z2+1
    of plane x1+1 that are not vacuum; the current enters and leaves through it."""
    ys, zs = slice(gr.y1 - 1, gr.y2 + 1), slice(gr.z1 - 1, gr.z2 + 1)
    return ~np.asarray(mk.vac[gr.x1, ys, zs], dtype=bool)


def bar_field(gr: Grid, nq: int = 8, backend: str = "auto", section=None) -> BarField:
    """2D Biot–Savart field of a uniform current density over the bar section (field.jl:151-180), evaluated
    with the reference's 8×8 midpoint quadrature per section cell.  It depends on the y–z section only, so it is
    kept per section (the tables are shared read-only between Steppers).

    ``backend``: "numpy" (vectorised over the quadrature points, here on the host), "device" (the library's
    ``tdgl_bar_field`` kernel), or "auto": the device for sections of 256 cells or more when a GPU is present
    (the sum has sections × 64 × face-points terms: 3.7e9 at 256×128×32)."""
    if section is not None:   # a sculpted sample's section (the conducting nodes of the contact face): on the host
        return _bar_field_host(gr, nq, np.asarray(section, dtype=bool))
    if backend == "auto":
        big = (gr.y2 - gr.y1 + 1) * (gr.z2 - gr.z1 + 1) >= 256
        backend = "device" if big and _device_available() else "numpy"
    key = (gr.Ny, gr.Nz, gr.y1, gr.y2, gr.z1, gr.z2, gr.dy, gr.dz, nq, backend)
    if key not in _BAR_CACHE:
        _BAR_CACHE[key] = _bar_field_device(gr, nq) if backend == "device" else _bar_field_host(gr, nq)
    return _BAR_CACHE[key]


def _bar_field_host(gr: Grid, nq: int, section=None) -> BarField:
    dy, dz = gr.dy, gr.dz
    ya, yb = (gr.y1 - 1) * dy, gr.y2 * dy
    za, zb = (gr.z1 - 1) * dz, gr.z2 * dz
    d = (gr.z2 - gr.z1 + 1) * dz
    c = (-2 / d) / (2 * math.pi)
    ny = nq * (gr.y2 - gr.y1 + 1)
    nz = nq * (gr.z2 - gr.z1 + 1)
    hq = (yb - ya) / ny
    kq = (zb - za) / nz
    yp = ya + (np.arange(1, ny + 1) - 0.5) * hq
    zp = za + (np.arange(1, nz + 1) - 0.5) * kq
    YP = np.broadcast_to(yp[:, None], (ny, nz)).ravel(order="F")
    ZP = np.broadcast_to(zp[None, :], (ny, nz)).ravel(order="F")
    if section is not None:
        # a quadrature point belongs to the node whose dual cell holds it (field.jl:160-161; no ties: the points sit
        # at the sixteenths of a cell)
        jn = np.clip(np.rint(YP / dy).astype(np.int64) + 1, gr.y1, gr.y2 + 1) - gr.y1
        kn = np.clip(np.rint(ZP / dz).astype(np.int64) + 1, gr.z1, gr.z2 + 1) - gr.z1
        keep = section[jn, kn]
        YP, ZP = YP[keep], ZP[keep]

    def h(ys, zs):
        ys = np.asarray(ys, dtype=np.float64).ravel()
        zs = np.asarray(zs, dtype=np.float64).ravel()
        HY = np.empty(ys.size)
        HZ = np.empty(ys.size)
        step = max(1, int(4e6 // max(1, YP.size)))
        for s in range(0, ys.size, step):
            y = ys[s:s + step, None]
            z = zs[s:s + step, None]
            r2 = (y - YP) ** 2 + (z - ZP) ** 2
            HY[s:s + step] = (-(z - ZP) / r2).sum(axis=1)
            HZ[s:s + step] = ((y - YP) / r2).sum(axis=1)
        return c * HY * hq * kq, c * HZ * hq * kq

    Ny, Nz = gr.Ny, gr.Nz
    yc = lambda j: (j - 0.5) * dy
    yn = lambda j: (j - 1) * dy
    zc = lambda k: (k - 0.5) * dz
    zn = lambda k: (k - 1) * dz

    def table(yf, zf, js, ks, comp):
        J, K = np.meshgrid(np.asarray(js, dtype=float), np.asarray(ks, dtype=float), indexing="ij")
        out = h(yf(J), zf(K))[comp]
        return out.reshape(J.shape)

    return BarField(
        hy_z=table(yn, zc, range(1, Ny + 2), (1, Nz), 0),
        hy_y=table(yn, zc, (1, Ny + 1), range(1, Nz + 1), 0),
        hz_z=table(yc, zn, range(1, Ny + 1), (1, Nz + 1), 1),
        hz_y=table(yc, zn, (1, Ny), range(1, Nz + 2), 1),
        hz_x=table(yc, zn, range(1, Ny + 1), range(1, Nz + 2), 1),
        hy_x=table(yn, zc, range(1, Ny + 2), range(1, Nz + 1), 0))


def _device_available() -> bool:
    try:
        from . import gpu
        gpu.lib()
    except Exception:
        return False
    import ctypes
    for name in ("libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so.12"):
        try:
            rt = ctypes.CDLL(name)
        except OSError:
            continue
        n = ctypes.c_int(0)
        return rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
    return False


def _bar_field_device(gr: Grid, nq: int) -> BarField:
    import ctypes as C

    from . import abi, gpu
    L = gpu.lib()
    Ny, Nz = gr.Ny, gr.Nz
    out = [np.zeros((Ny + 1, 2), order="F"), np.zeros((2, Nz), order="F"), np.zeros((Ny, 2), order="F"),
           np.zeros((2, Nz + 1), order="F"), np.zeros((Ny, Nz + 1), order="F"), np.zeros((Ny + 1, Nz), order="F")]
    g = abi.Grid_t(gr.Nx, gr.Ny, gr.Nz, gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2, gr.dx, gr.dy, gr.dz)
    L.tdgl_bar_field.argtypes = [C.POINTER(abi.Grid_t), C.c_int32] + [abi.dptr] * 6
    rc = L.tdgl_bar_field(C.byref(g), int(nq), *[o.ctypes.data_as(abi.dptr) for o in out])
    if rc != 0:
        raise RuntimeError(f"tdgl_bar_field failed ({rc})")
    return BarField(*out)


# ----------------------------------------------------------------------------------------- open boundary
def _gauss_legendre(n: int):
    k = np.arange(1, n)
    β = k / np.sqrt(4.0 * k * k - 1)
    T = np.diag(β, 1) + np.diag(β, -1)
    w, V = np.linalg.eigh(T)
    return w, 2 * V[0, :] ** 2


def lattice_green(R: int) -> np.ndarray:
    """G[0:R,0:R,0:R] of −Δ_h on the unit cubic lattice (openbc.jl:63-87): Gauss–Legendre in t over 6 intervals
    of the product of scaled Bessel functions (trapezoid in θ, openbc.jl:40-53), plus the t > 512 tail."""
    x, w = _gauss_legendre(48)
    edges = (0.0, 0.5, 2.0, 8.0, 32.0, 128.0, 512.0)
    T = edges[-1]
    G = np.zeros((R + 1, R + 1, R + 1))
    n = np.arange(R + 1)
    for p in range(len(edges) - 1):
        a, c = edges[p], edges[p + 1]
        for q in range(len(x)):
            t = (a + c) / 2 + (c - a) / 2 * x[q]
            wt = (c - a) / 2 * w[q]
            xx = 2 * t
            M = 32 + math.ceil(12 * math.sqrt(xx))
            θ = math.pi * np.arange(M + 1) / M
            wq = np.ones(M + 1)
            wq[0] = wq[-1] = 0.5
            e = wq * np.exp(xx * (np.cos(θ) - 1))
            b = (e[None, :] * np.cos(n[:, None] * θ[None, :])).sum(axis=1) / M
            G += wt * b[:, None, None] * b[None, :, None] * b[None, None, :]
    i = n[:, None, None]
    j = n[None, :, None]
    k = n[None, None, :]
    cc = ((4 * i * i - 1) + (4 * j * j - 1) + (4 * k * k - 1)) / 16
    G += (4 * math.pi) ** -1.5 * (2 / math.sqrt(T) - cc * (2 / 3) / T ** 1.5)
    return G


def lgf_far(i, j, k):
    """1/(4πr) with Duffin's first cubic correction (openbc.jl:90-93)."""
    r2 = float(i * i + j * j + k * k)
    r = math.sqrt(r2)
    return (1 + (5 * (i ** 4 + j ** 4 + k ** 4) / (r2 * r2) - 3) / (8 * r2)) / (4 * math.pi * r)


@dataclass
class OpenBCSpec:
    """The host side of ``OpenBC`` (openbc.jl:100-136): the ramp interval, the Green table and J_bar."""
    every: int
    R: int
    G: np.ndarray                 # (R+1)^3 lattice Green table
    fac: float                    # dx³/κ²
    Jbar: np.ndarray              # (Ny+1, Nz+1) κ² curl of the x-face bar field per unit HJ


def open_spec(gr: Grid, κ: float, bar: BarField, every: int, R: int = 8) -> OpenBCSpec:
    if not (gr.dx == gr.dy == gr.dz):
        raise ValueError(":open needs dx = dy = dz")
    Jb = np.zeros((gr.Ny + 1, gr.Nz + 1), order="F")
    κ2 = κ * κ
    for k in range(2, gr.Nz + 1):
        for j in range(2, gr.Ny + 1):
            Jb[j - 1, k - 1] = κ2 * ((bar.hz_x[j - 1, k - 1] - bar.hz_x[j - 2, k - 1]) / gr.dy
                                     - (bar.hy_x[j - 1, k - 1] - bar.hy_x[j - 1, k - 2]) / gr.dz)
    return OpenBCSpec(every, R, lattice_green(R), gr.dx ** 3 / κ2, Jb)


# ----------------------------------------------------------------------------------------- Stepper
SOLVER_EXPLICIT, SOLVER_SCALE, SOLVER_SEP, SOLVER_PCG = 0, 1, 2, 3
BC_SLAB, BC_BAR, BC_OPEN = 0, 1, 2


@dataclass
class PCGSpec:
    tol: float
    maxit: int
    fast: bool
    f32: bool
    extrap: bool


@dataclass(frozen=True)
class Heat:
    """The temperature field's coefficients (terms.jl:17-31), in t_GL and ξ₁: dθ/dt = D_T Δθ + η (dissipation
    [+ σn|E|² with joule]) − γ_bath (θ − T), θ capped at `cap`; cells within `margin` of the injection faces add no
    source; a ladder point whose max θ exceeds `cut` is cut ('T')."""
    D_T: float = 0.25
    gamma_bath: float = 0.2
    eta: float = 0.05
    joule: bool = False
    margin: int = 0
    cap: float = 1.5
    cut: float = 0.45


def lap1d(n: int, h: float, dirichlet: bool):
    """exchange.jl:150-162: the second difference on n nodes with spacing h, Dirichlet (the unknowns between two
    fixed ends) or Neumann (mirror ghosts at both ends); its eigenbasis V (columns), W = V⁻¹ and the eigenvalues."""
    L = np.zeros((n, n))
    h2 = h * h
    for a in range(n):
        L[a, a] = -2 / h2
        if a > 0:
            L[a, a - 1] = 1 / h2
        if a < n - 1:
            L[a, a + 1] = 1 / h2
    if not dirichlet and n > 1:
        L[0, 1] = 2 / h2
        L[n - 1, n - 2] = 2 / h2
    e, V = np.linalg.eig(L)
    V = np.ascontiguousarray(np.real(V))
    return V, np.linalg.inv(V), np.real(e).copy()


@dataclass
class QPVar:
    """The coefficients of the δ equation per unknown and link with materials (exchange.jl:193-228, QPVar): typ 1 free,
    0 cut (vacuum), 2 held at δ = 0 (a one-fluid material); σ_l/h² on the links of the region (cx with the two x ends,
    (Nx) × nj × nk; cy (Nx−1) × (nj−1) × nk; cz (Nx−1) × nj × (nk−1)); λ per unknown; d the diagonal of a decoupled
    unknown, σn(2/dx² + 2/dy² + 2/dz²) + λ0."""
    typ: np.ndarray
    cx: np.ndarray
    cy: np.ndarray
    cz: np.ndarray
    λ: np.ndarray
    d: float


def _qp_var(md, gr, mt, s, split, ν, rates, j0, j1, k0, k1, cond, λ0):
    """exchange.jl:193-228: None when every material has the first one's σn and λ (the separable or sculpted solve)."""
    mats = mt.models
    M = len(mats)
    r = [float(ν)] * M if rates is None else [float(x) for x in rates]
    if not (len(r) == M and r[0] == ν and all(x >= 0 for x in r)):
        raise ValueError(f"qp_exchange per material: {M} rates, the first that of [material] ({ν})")
    one = [r[m] == math.inf or bool(np.any(mt.absent[m, :])) for m in range(M)]
    if one[0]:
        raise ValueError("qp_exchange: the first material has two fluids (a finite rate)")
    if split is None:
        for m in range(1, M):
            if one[m]:
                continue
            bm = mats[m].bands
            wm = tuple(stiffness(bm[µ]) * bm[µ].Γ / bm[µ].β for µ in range(2))
            sm = wm[0] / (wm[0] + wm[1])
            if not abs(sm - s[0]) <= 1e-12:
                raise ValueError(f"qp_exchange with materials: the dirty split of material {m + 1} (s_σ = {sm:.10g}) is "
                                 f"not that of [material] ({s[0]:.10g}); a split that changes by region is not "
                                 "supported: give qp_split, the same for every material")
    λm = [0.0 if one[m] else s[0] * mats[m].σn * mats[m].bands[0].Γ / stiffness(mats[m].bands[0]) * r[m] *
          (1 / s[0] + 1 / s[1]) for m in range(M)]
    if not any(one) and all(mats[m].σn == md.σn and λm[m] == λm[0] for m in range(M)):
        return None
    x1, x2, y1, y2, z1, z2 = gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2
    idx = mt.idx

    def mat(i, j, k):   # 1-based node, clamped to the block; 0-based material
        return int(idx[min(max(i, x1), x2 + 1) - 1, min(max(j, y1), y2 + 1) - 1, min(max(k, z1), z2 + 1) - 1]) - 1

    def conducts(i, j, k):
        return cond is None or bool(cond[i - 1, j - 1, k - 1])

    def hm(a, b):
        return a if a == b else 2 * a * b / (a + b)

    def link(a, b, h):
        if not (conducts(*a) and conducts(*b)):
            return 0.0
        return hm(mats[mat(*a)].σn, mats[mat(*b)].σn) / (h * h)

    n1, nj, nk = gr.Nx - 1, j1 - j0 + 1, k1 - k0 + 1
    jo, ko = j0 - 1, k0 - 1
    typ = np.zeros((n1, nj, nk), dtype=np.uint8, order="F")
    lam = np.zeros((n1, nj, nk), order="F")
    for k in range(1, nk + 1):
        for j in range(1, nj + 1):
            for i in range(1, n1 + 1):
                I, J, K = i + 1, j + jo, k + ko
                typ[i - 1, j - 1, k - 1] = 0 if not conducts(I, J, K) else (2 if one[mat(I, J, K)] else 1)
                lam[i - 1, j - 1, k - 1] = λm[mat(I, J, K)]
    cx = np.zeros((n1 + 1, nj, nk), order="F")
    for k in range(1, nk + 1):
        for j in range(1, nj + 1):
            for i in range(1, n1 + 2):
                cx[i - 1, j - 1, k - 1] = link((i, j + jo, k + ko), (i + 1, j + jo, k + ko), gr.dx)
    cy = np.zeros((n1, max(nj - 1, 0), nk), order="F")
    for k in range(1, nk + 1):
        for j in range(1, nj):
            for i in range(1, n1 + 1):
                cy[i - 1, j - 1, k - 1] = link((i + 1, j + jo, k + ko), (i + 1, j + 1 + jo, k + ko), gr.dy)
    cz = np.zeros((n1, nj, max(nk - 1, 0)), order="F")
    for k in range(1, nk):
        for j in range(1, nj + 1):
            for i in range(1, n1 + 1):
                cz[i - 1, j - 1, k - 1] = link((i + 1, j + jo, k + ko), (i + 1, j + jo, k + 1 + ko), gr.dz)
    dd = md.σn * (2 / (gr.dx * gr.dx) + 2 / (gr.dy * gr.dy) + 2 / (gr.dz * gr.dz)) + λ0
    return QPVar(typ, cx, cy, cz, lam, dd)


@dataclass
class QPExchange:
    """Two normal fluids of a two-band model (exchange.jl:170-191, QPExchange): each band's quasiparticles carry
    their own potential and the bands exchange them at the rate ν; s the shares of σn (by default the dirty ones,
    ∝ g_µΓ_µ/β_µ), G = χ_σ ν, λ0 = G (1/s_σ + 1/s_π).  δ = μ_π − μ_σ lives on the x nodes 2..Nx and on the y, z nodes
    of the region (the whole section, or with the insulating padding the bar of the sample: y1..y2+1, z1..z2+1);
    V, W = V⁻¹ and e are the eigenbases of the three 1D second differences (x Dirichlet, y and z Neumann)."""
    ν: float
    s: Tuple[float, float]
    G: float
    λ0: float
    σn: float
    j0: int
    nj: int
    k0: int
    nk: int
    V: Tuple[np.ndarray, np.ndarray, np.ndarray]
    W: Tuple[np.ndarray, np.ndarray, np.ndarray]
    e: Tuple[np.ndarray, np.ndarray, np.ndarray]
    # a sculpted sample (QPSolve, exchange.jl:34-49): the conducting unknowns of the region ((Nx−1) × nj × nk; None:
    # nothing cut), δ then by conjugate gradients to `tol` in at most `maxit` iterations
    cond: Optional[np.ndarray] = None
    tol: float = 1e-10
    maxit: int = 1000
    var: Optional[QPVar] = None   # materials whose σn, λ or fluids differ (QPVar); None: the first material's

    @staticmethod
    def make(md: Model, gr: Grid, ν: float, split=None, conductor: bool = False, cond=None, mt=None,
             rates=None) -> "QPExchange":
        if md.N != 2:
            raise ValueError(f"qp_exchange: a number is for two bands; with {md.N} bands give the matrix of rates "
                             "(QPExchangeN, not built)")
        if not ν >= 0:
            raise ValueError("qp_exchange: the rate must be >= 0")
        b = md.bands
        w = (tuple(stiffness(b[µ]) * b[µ].Γ / b[µ].β for µ in range(2)) if split is None
             else tuple(float(x) for x in split))
        if len(w) != 2 or not all(x > 0 for x in w):
            raise ValueError("qp_split: two positive shares")
        s = (w[0] / (w[0] + w[1]), w[1] / (w[0] + w[1]))
        χσ = s[0] * md.σn * b[0].Γ / stiffness(b[0])
        G = χσ * float(ν)
        j0, j1 = (gr.y1, gr.y2 + 1) if conductor else (1, gr.Ny + 1)
        k0, k1 = (gr.z1, gr.z2 + 1) if conductor else (1, gr.Nz + 1)
        Vx, Wx, ex = lap1d(gr.Nx - 1, gr.dx, True)
        Vy, Wy, ey = lap1d(j1 - j0 + 1, gr.dy, False)
        Vz, Wz, ez = lap1d(k1 - k0 + 1, gr.dz, False)
        qc = None
        if cond is not None:   # QPSolve: cond[i+1, j, k] for the unknowns i = 1..Nx−1 of the region
            qc = np.asfortranarray(np.asarray(cond, dtype=bool)[1:gr.Nx, j0 - 1:j1, k0 - 1:k1])
        λ0 = G * (1 / s[0] + 1 / s[1])
        var = None if mt is None else _qp_var(md, gr, mt, s, split, float(ν), rates, j0, j1, k0, k1, cond, λ0)
        return QPExchange(float(ν), s, G, λ0, float(md.σn), j0, j1 - j0 + 1, k0, k1 - k0 + 1,
                          (Vx, Vy, Vz), (Wx, Wy, Wz), (ex, ey, ez), qc, var=var)


@dataclass
class QPExchangeN:
    """N normal fluids (exchange.jl:449-476, QPExchangeN; any N ≥ 2): ν the matrix of exchange rates µ → ν (zero
    diagonal, detailed balance χ_µν_µν = χ_νν_νµ with χ = s σn Γ/g), s the shares of σn.  With L the Laplacian of the
    exchange graph and S = diag(s), the potentials solve σn∇²μ − S⁻¹Lμ = S⁻¹C − 𝟙ΣC; in the modes m = Pinv μ of
    S^{-1/2} L S^{-1/2} = QΛQᵀ (P = S^{-1/2}Q, Pinv = QᵀS^{1/2}) they are N Helmholtz problems with λ = max(Λ, 0)."""
    ν: np.ndarray
    s: Tuple[float, ...]
    P: np.ndarray
    Pinv: np.ndarray
    λ: Tuple[float, ...]
    σn: float
    Gm: np.ndarray
    j0: int
    nj: int
    k0: int
    nk: int
    V: Tuple[np.ndarray, np.ndarray, np.ndarray]
    W: Tuple[np.ndarray, np.ndarray, np.ndarray]
    e: Tuple[np.ndarray, np.ndarray, np.ndarray]
    # a sculpted sample (QPSolve): the conducting unknowns of the region, each mode then by conjugate gradients
    cond: Optional[np.ndarray] = None
    tol: float = 1e-10
    maxit: int = 1000

    @staticmethod
    def make(md: Model, gr: Grid, ν, split=None, conductor: bool = False, cond=None) -> "QPExchangeN":
        N = md.N
        νm = np.asarray(ν, dtype=np.float64)
        if νm.shape != (N, N):
            raise ValueError(f"qp_exchange: an {N}×{N} matrix of rates for {N} bands")
        if not (all(νm[µ, µ] == 0 for µ in range(N)) and np.all(νm >= 0)):
            raise ValueError("qp_exchange: rates >= 0 with a zero diagonal")
        b = md.bands
        w = (tuple(stiffness(b[µ]) * b[µ].Γ / b[µ].β for µ in range(N)) if split is None
             else tuple(float(x) for x in split))
        if len(w) != N or not all(x > 0 for x in w):
            raise ValueError(f"qp_split: {N} positive shares")
        sw = sum(w)
        s = tuple(w[µ] / sw for µ in range(N))
        χ = [s[µ] * md.σn * b[µ].Γ / stiffness(b[µ]) for µ in range(N)]
        G = np.array([[χ[µ] * νm[µ, n] for n in range(N)] for µ in range(N)])
        # isapprox(G, Gᵀ; rtol=1e-10, atol=1e-14): Frobenius norms
        if not np.linalg.norm(G - G.T) <= max(1e-14, 1e-10 * max(np.linalg.norm(G), np.linalg.norm(G.T))):
            raise ValueError("qp_exchange: the rates must satisfy detailed balance, χ_µν_µν = χ_νν_νµ "
                             f"(χ = s σn Γ/g: {[float(f'{x:.4g}') for x in χ]})")
        G = (G + G.T) / 2
        L = -G
        for µ in range(N):
            acc = None
            for n in range(N):
                if n != µ:
                    acc = G[µ, n] if acc is None else acc + G[µ, n]
            L[µ, µ] = acc
        rs = np.sqrt(np.array(s))
        lam, Q = np.linalg.eigh(L / np.outer(rs, rs))
        j0, j1 = (gr.y1, gr.y2 + 1) if conductor else (1, gr.Ny + 1)
        k0, k1 = (gr.z1, gr.z2 + 1) if conductor else (1, gr.Nz + 1)
        Vx, Wx, ex = lap1d(gr.Nx - 1, gr.dx, True)
        Vy, Wy, ey = lap1d(j1 - j0 + 1, gr.dy, False)
        Vz, Wz, ez = lap1d(k1 - k0 + 1, gr.dz, False)
        qc = (None if cond is None else
              np.asfortranarray(np.asarray(cond, dtype=bool)[1:gr.Nx, j0 - 1:j1, k0 - 1:k1]))
        return QPExchangeN(νm, s, Q / rs[:, None], Q.T * rs[None, :], tuple(float(max(x, 0.0)) for x in lam),
                           float(md.σn), G, j0, j1 - j0 + 1, k0, k1 - k0 + 1, (Vx, Vy, Vz), (Wx, Wy, Wz),
                           (ex, ey, ez), qc)


@dataclass
class Stepper:
    model: Model
    grid: Grid
    masks: Masks
    dt: float
    nsub: Tuple[int, ...]
    rkl: Tuple[int, ...]
    bc: Tuple[BandCoef, ...]
    bcs: Tuple[BandCoef, ...]
    w: Tuple[float, ...]
    wa: Tuple[Tuple[float, ...], Tuple[float, ...], Tuple[float, ...]]
    fc: FieldCoef
    solver: int
    D: Optional[Tuple[np.ndarray, np.ndarray, np.ndarray]]
    bar: Optional[BarField]
    open: Optional[OpenBCSpec]
    extrap: bool
    rotframe: bool
    hard: bool
    limit: str
    dt_scale: float
    rkl_margin: float
    rkc: Optional[Tuple[Optional[RKCCoef], ...]]
    pcg: Optional[PCGSpec]
    selffield_bc: int
    noise_T: Optional[float] = None
    noise_seed: int = 1
    noise_field: bool = False
    # the step index of the first draw: the draws are a function of (seed, step index, stream, node), so a run resumed
    # at step q with noise_step0 = q continues the noise of the run it resumes
    noise_step0: int = 0
    # material per region (materials.jl); None: one material
    mt: Optional[MatField] = None
    # the interband drag (scheme.jl:188-189, 404-413): per band µ the full-step coefficients (x, y, z) of band ν's
    # lattice Laplacian, and the symmetric matrix ν_µν of the supercurrent; None: no drag
    drag: Optional[tuple] = None
    dragν: Optional[tuple] = None
    heat: Optional["Heat"] = None   # the temperature field's coefficients (terms.jl:17-31); None: no heat model
    heat_DT: Optional[tuple] = None   # with materials: D_T per material (MatField.DT, materials.jl:38)
    qpx: Optional[object] = None   # normal fluids per band (exchange.jl: QPExchange, QPExchangeN); None: one fluid

    @property
    def N(self) -> int:
        return self.model.N

    @staticmethod
    def make(md: Model, gr: Grid, mk: Masks, *, implicit=True, substeps=None, dt_scale=0.5, extrap=True, hard=False,
             σvac=None, pcg_tol=1e-8, selffield_bc="bar", rkl="rkc", open_every=1.0, rotframe=None, rkl_margin=None,
             noise=None, noise_seed=1, noise_field=False, rkc_damping=RKC_EPS, pcg_fast=True, pcg_f32=True,
             pcg_extrap=True, dt=None, bar_backend="auto", bar_tables=None, materials=None, transparency=None,
             absent=None, drag=None, heat=None, heat_DT=None, qp_exchange=None, qp_split=None,
             qp_rates=None) -> "Stepper":
        """scheme.jl:250-434 without heat or normal-fluid exchange; `materials` = the models of materials 2, 3, …
        that `mk.mat` names (materials.jl), `transparency` their barriers, `absent` the bands a material lacks;
        `drag` the interband drag ν (a number for two bands, or the symmetric N×N matrix; scheme.jl:404-413);
        `heat` a Heat (the temperature field, terms.jl; not with vacuum), `heat_DT` its D_T per material;
        `qp_exchange` ν and `qp_split` the normal fluids per band (exchange.jl: a number, two bands, QPExchange; a
        matrix of rates, N bands, QPExchangeN; with materials or in a sculpted sample two bands, `qp_rates` the rate of
        each material; not with the drag).

        ``dt`` overrides the step the bounds give (the stage and substep counts then follow from it with the
        same formulas); the reference always takes the bound."""
        N = md.N
        if substeps is None:
            substeps = tuple(1 if µ == 0 else 0 for µ in range(N))
        selffield_bc = str(selffield_bc).lstrip(":")
        if isinstance(rkl, bool):
            rkc = False
        elif str(rkl).lstrip(":") == "rkc":
            rkc = True
        elif str(rkl).lstrip(":") == "rkl":
            rkc = False
        else:
            raise ValueError(f'rkl must be true, false, "rkl" or "rkc", not {rkl!r}')
        rkl = rkl if isinstance(rkl, bool) else True
        if not (0 < dt_scale <= 1):
            raise ValueError(f"dt_scale must be in (0, 1], not {dt_scale}")
        kwt = any(b.γkwt > 0 for b in md.bands) or (materials is not None and
                                                     any(b.γkwt > 0 for m in materials for b in m.bands))
        rotframe = kwt if rotframe is None else rotframe
        rkl_margin = float(rkl_margin if rkl_margin is not None else (1.1 if kwt else 1.0))
        if rkl_margin < 1:
            raise ValueError("rkl_margin must be >= 1")
        if rotframe and not extrap:
            raise ValueError("rotframe needs extrap = true (it turns copies of the links)")
        if any(s < 0 for s in substeps):
            raise ValueError("substeps must be >= 0")
        if implicit and not (gr.dx == gr.dy == gr.dz):
            raise ValueError("the implicit curl-curl needs dx = dy = dz (separable solve)")
        sculpted = mk.vac is not None
        l = dl(gr)
        bands = md.bands
        if mk.mat is not None and materials is None:
            raise ValueError('the shape names materials (material = "name"): pass materials (the [materials.<name>] '
                             "tables of a run file)")
        mats, abs_m = _check_materials(md, materials, mk, absent) if materials is not None else (None, None)
        bb0, bbk, λL = _band_bounds(md, gr, l)
        bsc_m = math.inf
        if mats is not None:
            # the bound of each band is the smallest over the materials; a band absent from a material adds none
            for q, m in enumerate(mats[1:]):
                pr = tuple(not abs_m[q + 1, µ] for µ in range(N))
                b0, bk, λ = _band_bounds(m, gr, l, present=pr)
                bb0 = tuple(min(x, y) for x, y in zip(bb0, b0))
                bbk = tuple(min(x, y) for x, y in zip(bbk, bk))
                if m.σn == md.σn:
                    λL = max(λL, λ)
                elif λ > 0:
                    bsc_m = min(bsc_m, 2 * m.σn / λ)
        σvar = mats is not None and any(m.σn != md.σn for m in mats)
        bb = bb0 if rkl else bbk
        pad = σvac is not None and float(σvac) != md.σn
        if pad and not (0 < σvac <= md.σn):
            raise ValueError("σvac must be in (0, σn]")
        σf = float(σvac) if pad else (min(m.σn for m in mats) if σvar else md.σn)
        bfield = math.inf if implicit else σf * l / (4 * (md.κ * md.κ))
        bsc0 = 2 * md.σn / λL if λL != 0 else math.inf   # Julia's IEEE division: no condensate, no bound
        bsc = min(bsc0, bsc_m) if σvar else bsc0
        ref = min(bfield, bsc, min(math.inf if substeps[µ] == 0 else bb[µ] * max(substeps[µ], 1) for µ in range(N)))
        nsub = tuple(max(1, math.ceil(dt_scale * ref / bb[µ] - 1e-12)) if substeps[µ] == 0 else substeps[µ]
                     for µ in range(N))
        bbn = tuple(bb[µ] if (nsub[µ] == 1 and substeps[µ] == 1) else bb[µ] * (nsub[µ] / dt_scale) for µ in range(N))
        cands = bbn + (bfield, bsc)
        names = tuple(f"band {µ + 1}" for µ in range(N)) + ("field (explicit curl-curl)", "explicit supercurrent")
        dtc = 0.99 * min(cands)
        if dt_scale != 1:
            dtc *= dt_scale
        # scheme.jl:316-321: the explicit diffusion of the temperature field (the largest D_T of the materials)
        DTmax = 0.0 if heat is None else (heat.D_T if heat_DT is None else max(heat.D_T, max(heat_DT)))
        if heat is not None and DTmax > 0:
            dt_dif = 0.15 * min(gr.dx, gr.dy, gr.dz) ** 2 / DTmax
            if dt_dif < dtc:
                dtc = dt_dif
                cands = cands + (dt_dif,)
                names = names + ("heat diffusion",)
        limit = names[int(np.argmin(cands))]
        if dt is not None:
            dtc = float(dt)
            limit = "given"
        dt = dtc
        rx = dt / (gr.dx * gr.dx)
        ry = dt / (gr.dy * gr.dy)
        rz = dt / (gr.dz * gr.dz)
        bc = tuple(_bandcoef(md, µ + 1, dt, rx, ry, rz, bands[µ].ma) for µ in range(N))

        def haskwt(µ):
            return bands[µ].γkwt > 0 or (materials is not None and any(m.bands[µ].γkwt > 0 for m in materials))

        stg = []
        for µ in range(N):
            if not rkl:
                stg.append(0)
                continue
            r = rkl_margin * dt / (0.99 * bbk[µ])
            if r <= 1 + 1e-12:
                stg.append(0)
                continue
            s = 1
            while s * (s + 1) // 2 < r - 1e-12:
                s += 1
            if rkc:
                q = 2
                while _rkc_ratio(q, float(rkc_damping)) < r - 1e-12:
                    q += 1
                if q < s or (noise is not None and haskwt(µ)):
                    s = -q
            stg.append(s)
        usec = tuple(s < 0 for s in stg)
        skb = tuple(noise is not None and rkc and usec[µ] and haskwt(µ) for µ in range(N))
        stg = tuple(abs(s) for s in stg)
        nsub = tuple(1 if stg[µ] > 0 else nsub[µ] for µ in range(N))
        if noise is not None and any(haskwt(µ) and not skb[µ] and stg[µ] > 0 for µ in range(N)):
            raise ValueError('noise with KWT on RKL stages: the equilibrium comes out biased. Use rkl = "rkc" or '
                             "rkl = false")
        rkcc = tuple(RKCCoef.make(stg[µ], float(rkc_damping)) if usec[µ] else None for µ in range(N)) if rkc else None

        def divisor(µ):
            if stg[µ] > 0:
                if rkcc is not None and rkcc[µ] is not None:
                    return rkcc[µ].q
                return stg[µ] * (stg[µ] + 1) // 2
            return nsub[µ]

        bcs = tuple(_divided(bc[µ], divisor(µ)) if stg[µ] > 0 else (bc[µ] if nsub[µ] == 1 else _divided(bc[µ], nsub[µ]))
                    for µ in range(N))
        w = tuple(stiffness(b) for b in bands)
        wa = tuple(tuple(stiffness(b, i) for b in bands) for i in (1, 2, 3))
        dtσ = dt / md.σn
        ks2 = md.κ * md.κ
        fc = FieldCoef(dtσ, (dtσ * ks2) * (gr.dx / gr.dy), (dtσ * ks2) * (gr.dx / gr.dz),
                       (dtσ * ks2) * (gr.dy / gr.dx), (dtσ * ks2) * (gr.dy / gr.dz),
                       (dtσ * ks2) * (gr.dz / gr.dx), (dtσ * ks2) * (gr.dz / gr.dy),
                       dtσ * ks2 / (gr.dx * gr.dx))
        mt = None if mats is None else MatField.make(
            mats, mk, gr, dt, rx, ry, rz,
            tuple(float(divisor(µ)) if (stg[µ] > 0 or nsub[µ] > 1) else 1.0 for µ in range(N)),
            transparency=transparency, absent=abs_m)
        if sculpted:   # scheme.jl:380-386: the free surface needs the insulating padding and the field of the bar
            if not pad:
                raise ValueError("a sculpted sample (a shape with vacuum) needs the insulating padding: σvac below σn")
            if str(selffield_bc) not in ("bar", "open"):
                raise ValueError("a sculpted sample needs selffield_bc = :bar or :open")
        cond = conducting_nodes(gr, mk) if sculpted else None
        if σvar:
            D = material_conductivity(gr, mk, mats, float(σvac) if pad else None, md.σn, cond=cond)
        else:
            D = link_conductivity(gr, float(σvac), md.σn, cond=cond) if pad else None
        if not implicit:
            solver = SOLVER_SCALE if D is not None else SOLVER_EXPLICIT
            pcg = None
        elif pad or σvar:
            solver = SOLVER_PCG
            pcg = PCGSpec(float(pcg_tol), 500, bool(pcg_fast), bool(pcg_f32), bool(pcg_extrap) and bool(pcg_fast))
        else:
            solver = SOLVER_SEP
            pcg = None
        if selffield_bc not in ("slab", "bar", "open"):
            raise ValueError("selffield_bc must be :slab, :bar or :open")
        section = _section(gr, mk) if sculpted else None
        bar = None
        if selffield_bc in ("bar", "open"):   # bar_tables: the six tables computed elsewhere (a BarField)
            bar = bar_tables if bar_tables is not None else bar_field(gr, backend=bar_backend, section=section)
        ob = open_spec(gr, md.κ, bar, every=max(1, round(open_every / dt))) if selffield_bc == "open" else None
        if noise_field and noise is None:
            raise ValueError("noise_field needs noise = T̃ (the same bath for Ψ and A)")
        hDT = None
        if heat is not None:   # scheme.jl:369-370, 383, 428-429
            if mats is not None:
                hDT = tuple(float(heat.D_T) for _ in mats) if heat_DT is None else tuple(float(x) for x in heat_DT)
                if len(hDT) != len(mats):
                    raise ValueError(f"heat_DT: one D_T per material ({len(mats)})")
            if sculpted:
                raise ValueError("a sculpted sample: not with the heat model yet (its diffusion does not see the free "
                                 "surface)")
            if noise is not None:
                raise ValueError("noise with the heat model: the heat source counts the Langevin kicks as dissipation")
        dragν = dragc = None
        if drag is not None:   # scheme.jl:404-413 (materials.jl:75 and scheme.jl:384 refuse it with materials, vacuum)
            if mats is not None:
                raise ValueError("materials: not with the drag yet")
            if sculpted:
                raise ValueError("a sculpted sample: not with the drag yet (its stencil does not see the free surface)")
            if np.ndim(drag) == 0:
                if N != 2:
                    raise ValueError("drag: a number is for two bands; give the matrix")
                νm = np.array([[0.0, float(drag)], [float(drag), 0.0]])
            else:
                νm = np.asarray(drag, dtype=np.float64)
            if νm.shape != (N, N) or not np.array_equal(νm, νm.T):
                raise ValueError(f"drag must be a symmetric {N}×{N} matrix")
            dragν = tuple(tuple(float(νm[µ, ν]) for ν in range(N)) for µ in range(N))

            def drag_coef(v, Γh):   # terms.jl:41
                return ((v * rx) / Γh, (v * ry) / Γh, (v * rz) / Γh)

            dragc = tuple(tuple(drag_coef(float(νm[µ, ν]), dt / (dt / bands[µ].Γ)) for ν in range(N)) for µ in range(N))
        qpx = None
        if qp_exchange is not None:   # scheme.jl:418-423 (exchange.jl)
            if mats is not None and np.ndim(qp_exchange) != 0:   # materials.jl:76-77
                raise ValueError("materials: qp_exchange with materials is the two-band one (a number); N fluids (a "
                                 "matrix) are not supported per region")
            qcond = conducting_nodes(gr, mk) if sculpted else None   # scheme.jl:419
            qpx = (QPExchange.make(md, gr, float(qp_exchange), qp_split, conductor=pad, cond=qcond, mt=mt,
                                   rates=qp_rates)
                   if np.ndim(qp_exchange) == 0
                   else QPExchangeN.make(md, gr, qp_exchange, qp_split, conductor=pad, cond=qcond))
        return Stepper(md, gr, mk, dt, nsub, stg, bc, bcs, w, wa, fc, solver, D, bar, ob, bool(extrap),
                       bool(rotframe), bool(hard), limit, float(dt_scale), rkl_margin, rkcc, pcg,
                       {"slab": BC_SLAB, "bar": BC_BAR, "open": BC_OPEN}[selffield_bc],
                       None if noise is None else float(noise), int(noise_seed), bool(noise_field), 0, mt, dragc,
                       dragν, heat, hDT, qpx)


def selffield(st: Stepper, J: float) -> float:
    """Self-field on the z faces for an injected current density J (step.jl:38)."""
    return J * slab_thickness(st.grid) / (2 * (st.model.κ * st.model.κ))


def sep_ranges(gr: Grid):
    """The link ranges of the separable / PCG solve (implicit.jl:52), 1-based inclusive (start, stop) per axis."""
    Nx, Ny, Nz = gr.Nx, gr.Ny, gr.Nz
    rx = ((2, Nx - 1), (2, Ny), (2, Nz))
    ry = ((2, Nx), (2, Ny - 1), (2, Nz))
    rz = ((2, Nx), (2, Ny), (2, Nz - 1))
    return rx, ry, rz


def sep_unknowns(gr: Grid) -> int:
    tot = 0
    for r in sep_ranges(gr):
        n = 1
        for a, b in r:
            n *= b - a + 1
        tot += n
    return tot
