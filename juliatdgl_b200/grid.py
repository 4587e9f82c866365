"""The staggered mesh, the masks and the WEDGE / SIM geometry of the catalogue (host side).

Restates ``gtdgl/src/grid.jl`` (``Grid`` :9-27, ``Masks`` :35-45, ``box_masks`` :47-58) and the part of
``gtdgl/src/geometry.jl`` that the ladder configurations use: ``oround`` (:12-13), the wedge rasteriser
(:120-137), ``apply_zmode!`` (:220-236), the WEDGE / WEDGE_BOTH / SIM entries of ``build_defect_list``
(:268-308, with the shifts of :309-318) and ``build_masks`` (:485-511).  ``conducting_nodes``
(:545-560) gives the σn links of the insulating padding.

Arrays are numpy arrays in Fortran (column-major) order with the reference's shapes, so index (i, j, k)
of the reference is ``[i-1, j-1, k-1]`` here and the raw memory is the reference's.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import shapes


def oround(x: float) -> int:
    """round(Int, x, RoundNearestTiesAway) (geometry.jl:12)."""
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


@dataclass(frozen=True)
class Grid:
    """Cells with padding (Nx, Ny, Nz), the block's node range x1..x2+1 etc. (1-based), and the spacings."""
    Nx: int
    Ny: int
    Nz: int
    x1: int
    x2: int
    y1: int
    y2: int
    z1: int
    z2: int
    dx: float
    dy: float
    dz: float

    @staticmethod
    def make(nx, ny, nz, *, dx, dy=None, dz=None, buf=1, bufx=None, bufy=None, bufz=None):
        """grid.jl:20-27: nx×ny×nz sample cells with `buf` padding cells on each face."""
        dy = dx if dy is None else dy
        dz = dx if dz is None else dz
        bufx = buf if bufx is None else bufx
        bufy = buf if bufy is None else bufy
        bufz = buf if bufz is None else bufz
        if min(nx, ny, nz) < 2:
            raise ValueError("Grid: at least 2 cells per axis")
        if min(bufx, bufy, bufz) < 1:
            raise ValueError("Grid: at least one padding cell per face")
        return Grid(nx + 2 * bufx, ny + 2 * bufy, nz + 2 * bufz, bufx + 1, bufx + nx, bufy + 1, bufy + ny,
                    bufz + 1, bufz + nz, float(dx), float(dy), float(dz))

    # array shapes of the state (state.jl:13-22)
    @property
    def node(self):
        return (self.Nx + 1, self.Ny + 1, self.Nz + 1)

    @property
    def xlink(self):
        return (self.Nx, self.Ny + 1, self.Nz + 1)

    @property
    def ylink(self):
        return (self.Nx + 1, self.Ny, self.Nz + 1)

    @property
    def zlink(self):
        return (self.Nx + 1, self.Ny + 1, self.Nz)

    @property
    def hx_shape(self):
        return (self.Nx + 1, self.Ny, self.Nz)

    @property
    def hy_shape(self):
        return (self.Nx, self.Ny + 1, self.Nz)

    @property
    def hz_shape(self):
        return (self.Nx, self.Ny, self.Nz + 1)

    @property
    def sample_cells(self) -> int:
        return (self.x2 - self.x1 + 1) * (self.y2 - self.y1 + 1) * (self.z2 - self.z1 + 1)


def slab_thickness(gr: Grid) -> float:
    """grid.jl:30."""
    return (gr.z2 - gr.z1 + 1) * gr.dz


def dl(gr: Grid) -> float:
    """2/(dx⁻² + dy⁻² + dz⁻²) (grid.jl:33)."""
    return 2.0 / (1 / (gr.dx * gr.dx) + 1 / (gr.dy * gr.dy) + 1 / (gr.dz * gr.dz))


def _zeros(shape):
    return np.zeros(shape, dtype=np.float64, order="F")


@dataclass
class Masks:
    """Condensation f, link masks τx/τy/τz, node mask τψ; vacuum and material maps are not used here."""
    f: np.ndarray
    τx: np.ndarray
    τy: np.ndarray
    τz: np.ndarray
    τψ: np.ndarray
    vac: Optional[np.ndarray] = None
    mat: Optional[np.ndarray] = None


def box_masks(gr: Grid) -> Masks:
    """grid.jl:47-58 (0-based slices of the 1-based ranges)."""
    n = gr.node
    f = np.ones(n, order="F")
    τx, τy, τz, τψ = _zeros(n), _zeros(n), _zeros(n), _zeros(n)
    x1, x2, y1, y2, z1, z2 = gr.x1 - 1, gr.x2 - 1, gr.y1 - 1, gr.y2 - 1, gr.z1 - 1, gr.z2 - 1
    τx[x1:x2 + 1, y1:y2 + 2, z1:z2 + 2] = 1.0
    τy[x1:x2 + 2, y1:y2 + 1, z1:z2 + 2] = 1.0
    τz[x1:x2 + 2, y1:y2 + 2, z1:z2 + 1] = 1.0
    τψ[x1:x2 + 2, y1:y2 + 2, z1:z2 + 2] = 1.0
    return Masks(f, τx, τy, τz, τψ)


@dataclass
class GeomSpec:
    """What sets the shape (geometry.jl:22-40): a catalogue mode (any with the `_REF` mirror) or a shape file
    (CUSTOM, CUSTOM_REF: geom_file; materials: the names of the run file's [materials.<name>] tables, in order), and
    the catalogue parameters, with release 1.2's names and defaults."""
    GEOM_MODE: str = "SIM"
    geom_file: str = ""
    wedge_depth: float = 0.35
    wedge_half: float = 0.20
    wedge_depth2: float = 0.00
    fgrad_flo: float = 1.00
    fgrad_fhi: float = 1.50
    fgrad_nper: int = 2
    fgrad_dir: int = +1
    inj_margin: int = 6
    strict_margin: bool = True
    x_shift: float = 0.0
    y_shift: float = 0.0
    z_mode: str = "through"
    prism_phi: float = math.nan
    current_axis: str = "x"
    verbose: bool = False
    materials: tuple = ()


CATALOGUE = ("SIM", "ESFERA", "ARRAY", "WEDGE", "WEDGE_BOTH", "ESF_CUNA", "FGRAD", "SAWROW", "SPHROW", "SAWSPH",
             "STAGGER", "FUNNEL", "FUNNEL_IN", "TRI_Y1", "TRI_Y1_INV", "RECT_Y1", "HEX", "HEX_STAG")


@dataclass
class _Defect:
    """A catalogue defect (geometry.jl:42-67); fields a type does not use stay None."""
    type: str
    xc: Optional[int] = None
    yc: Optional[int] = None
    zc: Optional[int] = None
    R: Optional[float] = None
    n: Optional[int] = None
    phi: Optional[float] = None
    hx: Optional[int] = None
    hy: Optional[int] = None
    hz: Optional[int] = None
    half: Optional[int] = None
    depth: Optional[int] = None
    f: float = 1.0
    xa: Optional[int] = None
    xb: Optional[int] = None
    ya: Optional[int] = None
    yb: Optional[int] = None
    flo: Optional[float] = None
    fhi: Optional[float] = None
    nper: Optional[int] = None
    dir: Optional[int] = None
    zmode: Optional[str] = None
    zlo: Optional[int] = None
    zhi: Optional[int] = None


def _in_ngon(px, py, cx, cy, R, n, phi) -> bool:
    """A point inside the regular n-gon of circumradius R turned by phi (in_ngon, geometry.jl:76-87): apothem
    a = R cos(π/n), the edge at radius a / cos(mod(θ, 2π/n) − π/n); the 1e-9 keeps the rows that land on an edge."""
    dx, dy = px - cx, py - cy
    r = math.hypot(dx, dy)
    a = R * math.cos(math.pi / n)
    if r <= a + 1e-9:
        return True
    if r > R + 1e-9:
        return False
    th = math.atan2(dy, dx) - phi
    seg = th % (2 * math.pi / n) - math.pi / n   # Python's float % is Julia's mod (sign of the divisor)
    return r <= a / math.cos(seg) + 1e-9


def _paint(fmask, d: _Defect, x1, x2, y1, y2, z1, z2):
    """paint_defect! (geometry.jl:89-155): writes d.f in the region of the defect (1-based loop indices)."""
    zA = z1 if d.zlo is None else max(z1, d.zlo)
    zB = z2 if d.zhi is None else min(z2, d.zhi)
    if zB < zA:
        return
    I = np.arange(x1, x2 + 1)[:, None]
    J = np.arange(y1, y2 + 1)[None, :]
    blk = fmask[x1 - 1:x2, y1 - 1:y2, zA - 1:zB]
    if d.type == "sphere":
        for k in range(zA, zB + 1):
            m = (I - d.xc) ** 2 + (J - d.yc) ** 2 + (k - d.zc) ** 2 <= d.R ** 2
            blk[:, :, k - zA][m] = d.f
    elif d.type == "cylinder":
        m = (I - d.xc) ** 2 + (J - d.yc) ** 2 <= d.R ** 2
        blk[m] = d.f
    elif d.type == "box":
        for k in range(zA, zB + 1):
            if abs(k - d.zc) <= d.hz:
                m = (np.abs(I - d.xc) <= d.hx) & (np.abs(J - d.yc) <= d.hy)
                blk[:, :, k - zA][m] = d.f
    elif d.type == "prism":
        m = np.array([[_in_ngon(i, j, d.xc, d.yc, d.R, d.n, d.phi) for j in range(y1, y2 + 1)]
                      for i in range(x1, x2 + 1)], dtype=bool).reshape(x2 - x1 + 1, y2 - y1 + 1)
        blk[m] = d.f
    elif d.type == "wedge":
        # dir: the notch grows in +y (from face y1) or in −y (from y2); its mirror is exact (yc → y1+y2+1−yc)
        dd = 1 if d.dir is None else d.dir
        for j in range(y1, y2 + 1):
            layer = dd * (j - d.yc)
            if 0 <= layer < d.depth:
                frac = 1 - layer / d.depth
                w_steep = max(1, oround(2 * frac))     # the steep wall
                w_gentle = oround(d.half * frac)       # the gentle ramp
                for i in range(x1, x2 + 1):
                    if -w_steep <= i - d.xc <= w_gentle:
                        blk[i - x1, j - y1, :] = d.f
    elif d.type == "fgrad":
        # a sawtooth in f(y): t over [0, 1] along [ya, yb] (reversed if dir < 0), f from fhi down to flo per tooth
        Ly = max(1, d.yb - d.ya)
        for j in range(max(y1, d.ya), min(y2, d.yb) + 1):
            t = (j - d.ya) / Ly
            if d.dir < 0:
                t = 1 - t
            phase = (t * d.nper) % 1
            fj = d.fhi + (d.flo - d.fhi) * phase
            fmask[max(x1, d.xa) - 1:min(x2, d.xb), j - 1, zA - 1:zB] = fj
    else:
        raise ValueError(f"unknown defect type: {d.type}")


def _linrange(a, b, n):
    """Julia's range(a, b, length=n) for endpoints of integer value: each point the exact rational rounded once."""
    from fractions import Fraction
    fa, fb = Fraction(a), Fraction(b)
    return [float(fa + (fb - fa) * q / (n - 1)) for q in range(n)]


def _phi_cat(cfg: GeomSpec, default: float) -> float:
    return default if math.isnan(cfg.prism_phi) else cfg.prism_phi


def _defects(cfg: GeomSpec, x1, x2, y1, y2, z1, z2):
    """build_defect_list (geometry.jl:300-478): the catalogue (J ∥ x), then the shifts, the `_REF` mirror and the z
    mode."""
    yc = oround((y1 + y2) / 2)
    zc = oround((z1 + z2) / 2)
    xc = oround((x1 + x2) / 2)
    nx_sc, ny_sc = x2 - x1 + 1, y2 - y1 + 1
    D = []
    mode = cfg.GEOM_MODE.upper()
    is_ref = len(mode) > 4 and mode.endswith("_REF")
    if is_ref:
        mode = mode[:-4]
    mg = cfg.inj_margin
    xsafe_lo, xsafe_hi = (x1 + mg, x2 - mg) if cfg.current_axis.lower() == "x" else (x1, x2)
    W = lambda **kw: D.append(_Defect(type="wedge", f=0.0, **kw))
    S = lambda xc_, yc_, zc_, R: D.append(_Defect(type="sphere", xc=xc_, yc=yc_, zc=zc_, R=R, f=0.0))
    P = lambda xc_, yc_, R, n, phi: D.append(_Defect(type="prism", xc=xc_, yc=yc_, zc=zc, R=R, n=n, phi=phi, f=0.0))
    if mode == "SIM":
        pass
    elif mode == "ESFERA":
        S(xc, yc, zc, 6.0)
    elif mode == "ARRAY":
        for s, R in zip((oround(q * nx_sc) + x1 for q in (0.30, 0.50, 0.70)), (4.0, 6.0, 8.0)):
            S(s, yc, zc, R)
    elif mode in ("WEDGE", "WEDGE_BOTH"):
        W(xc=xc, yc=y1, dir=+1, half=oround(cfg.wedge_half * nx_sc), depth=oround(cfg.wedge_depth * ny_sc))
        if mode == "WEDGE_BOTH" and cfg.wedge_depth2 > 0:   # at yc = y2 + 1: the exact node mirror of y1
            W(xc=xc, yc=y2 + 1, dir=-1, half=oround(cfg.wedge_half * nx_sc), depth=oround(cfg.wedge_depth2 * ny_sc))
    elif mode == "ESF_CUNA":
        S(xc, yc, zc, 6.0)
        W(xc=xc + oround(0.18 * nx_sc), yc=y1, dir=+1, half=oround(0.10 * nx_sc), depth=oround(0.22 * ny_sc))
    elif mode == "FGRAD":
        D.append(_Defect(type="fgrad", xa=xsafe_lo, xb=xsafe_hi, ya=y1, yb=y2, flo=cfg.fgrad_flo, fhi=cfg.fgrad_fhi,
                         nper=cfg.fgrad_nper, dir=cfg.fgrad_dir, f=math.nan))
    elif mode in ("SAWROW", "SAWSPH"):
        nteeth = 5
        dep = oround(0.55 * ny_sc)
        xlo, xhi = x1 + mg + 2, x2 - mg - 2
        half = max(3, math.floor((xhi - xlo) / (2 * nteeth)) - 1)
        for s in _linrange(xlo + half, xhi - half, nteeth):
            W(xc=oround(s), yc=y1, dir=+1, half=half, depth=dep)
        if mode == "SAWSPH":
            zc0 = oround((z1 + z2) / 2)
            ysph = y2 - oround(0.25 * ny_sc)
            for s, R in zip((oround(q * (x2 - x1)) + x1 for q in (0.30, 0.50, 0.70)), (3.0, 5.0, 4.0)):
                S(s, ysph, zc0, R)
    elif mode == "SPHROW":
        zc0, yc0 = oround((z1 + z2) / 2), oround((y1 + y2) / 2)
        for s, R in zip((oround(q * (x2 - x1)) + x1 for q in (0.30, 0.50, 0.70)), (3.0, 6.0, 4.0)):
            S(s, yc0, zc0, R)
    elif mode in ("STAGGER", "HEX_STAG"):
        if mode == "HEX_STAG":
            Rhex = max(3.0, min(0.20 * min(float(nx_sc), float(ny_sc)), 0.5 * nx_sc - mg - 2.0))
            P(xc, yc, Rhex, 6, _phi_cat(cfg, 0.0))
        Rtri = 5.0 if mode == "STAGGER" else 4.0
        xs = [oround(v) for v in _linrange(xsafe_lo + Rtri, xsafe_hi - Rtri, 4)]
        dyr = oround(0.22 * ny_sc)
        for s_, xv in enumerate(xs, 1):
            ys = [yc - dyr, yc + dyr] if s_ % 2 == 1 else [yc - 2 * dyr, yc, yc + 2 * dyr]
            for yv in ys:
                if not (y1 + 2 < yv < y2 - 2):
                    continue
                if mode == "HEX_STAG" and not math.hypot(float(xv - xc), float(yv - yc)) > Rhex + Rtri + 1:
                    continue
                P(xv, oround(yv), Rtri, 3, _phi_cat(cfg, 0.0))
    elif mode in ("FUNNEL", "FUNNEL_IN"):
        Rtri, dyrow, per = 6.0, 10, 16
        inset = 4 if mode == "FUNNEL_IN" else 0
        xa, xb = xsafe_lo + Rtri, xsafe_hi - Rtri
        if xb < xa:
            raise ValueError("FUNNEL: the mesh is too short in x to place triangles inside the margin")
        xs = [xa + q * (per / 2) for q in range(int(math.floor((xb - xa) / (per / 2))) + 1)]
        for s, xv in enumerate(xs, 1):
            yrow = yc - dyrow / 2 if s % 2 == 1 else yc + dyrow / 2
            if inset > 0:   # φ = π/2: apex towards +y at yc + R, base at yc − R/2
                ymax = y2 - Rtri - inset
                ymin = y1 + Rtri * math.cos(math.pi / 3) + inset
                yrow = min(max(float(yrow), ymin), ymax)
            P(oround(xv), oround(yrow), Rtri, 3, _phi_cat(cfg, math.pi / 2))
    elif mode == "TRI_Y1":
        Rtri = 6.0
        P(xc, y1 + oround(Rtri * math.cos(math.pi / 3)), Rtri, 3, _phi_cat(cfg, math.pi / 2))
    elif mode == "TRI_Y1_INV":
        Rtri = 6.0
        P(xc, y1 + oround(Rtri), Rtri, 3, _phi_cat(cfg, -math.pi / 2))
    elif mode == "RECT_Y1":
        hx, hy = 5, 2
        D.append(_Defect(type="box", xc=xc, yc=y1 + hy, zc=zc, hx=hx, hy=hy, hz=max(z2 - z1, 8), f=0.0))
    elif mode == "HEX":
        Rhex = max(3.0, min(0.22 * min(float(nx_sc), float(ny_sc)), 0.5 * nx_sc - mg - 2.0))
        P(xc, yc, Rhex, 6, _phi_cat(cfg, 0.0))
    else:
        raise ValueError(f"unknown GEOM_MODE: {cfg.GEOM_MODE} (catalogue: {' | '.join(CATALOGUE)}, any with _REF; "
                         "or CUSTOM / CUSTOM_REF with geom_file)")
    # shifts of the whole array (robustness tests)
    if cfg.x_shift != 0:
        dxs = oround(cfg.x_shift * nx_sc)
        for d in D:
            if d.xc is not None:
                d.xc += dxs
            if d.xa is not None:
                d.xa += dxs
                d.xb += dxs
    if cfg.y_shift != 0:
        dys = oround(cfg.y_shift * ny_sc)
        for d in D:
            if d.yc is not None:
                d.yc += dys
            if d.ya is not None:
                d.ya += dys
                d.yb += dys
    if is_ref:   # the exact mirror along the vortex motion: y → y1 + y2 + 1 − y with J ∥ x (mirror_defects!)
        mirror_y = cfg.current_axis.lower() == "x"
        for d in D:
            if d.type == "wedge" and not mirror_y:
                raise ValueError("mirroring 'wedge' in x is not defined (its wall/ramp asymmetry is along x)")
            if mirror_y:
                if d.yc is not None:
                    d.yc = (y1 + y2 + 1) - d.yc
                if d.phi is not None:
                    d.phi = -d.phi
                if d.type == "fgrad":
                    d.ya, d.yb = (y1 + y2 + 1) - d.yb, (y1 + y2 + 1) - d.ya
                    d.dir = -d.dir
                if d.type == "wedge":
                    d.dir = -d.dir
            else:
                if d.xc is not None:
                    d.xc = (x1 + x2 + 1) - d.xc
                if d.phi is not None:
                    d.phi = math.pi - d.phi
                if d.type == "fgrad":
                    raise ValueError("fgrad is only defined for J ∥ x")
    zc = oround((z1 + z2) / 2)
    for d in D:   # apply_zmode!
        zm = (cfg.z_mode if d.zmode is None else d.zmode).lower()
        if zm == "through":
            d.zlo, d.zhi = z1, z2
        elif zm == "half":
            d.zlo, d.zhi = z1, zc
        elif zm == "buried":
            q = max(1, oround((z2 - z1) / 4))
            d.zlo, d.zhi = z1 + q, z2 - q
        else:
            raise ValueError(f"unknown z_mode: {zm} (use through|half|buried)")
    return D


def build_masks(cfg: GeomSpec, gr: Grid) -> Masks:
    """geometry.jl:485-511: a catalogue mode (CATALOGUE, any with the `_REF` mirror), or a shape file (CUSTOM, CUSTOM_REF:
    shapes.py).  A shape with vacuum gives a sculpted sample (`sculpt`); a shape with materials a material map whose
    ghost planes copy the block."""
    mode = cfg.GEOM_MODE.upper()
    if mode in ("CUSTOM", "CUSTOM_REF"):
        if not cfg.geom_file:
            raise ValueError(f"GEOM_MODE={mode} needs geom_file")
        mk = box_masks(gr)
        elems = shapes.read_shape(cfg.geom_file)
        vac = np.zeros(gr.node, dtype=bool, order="F")
        has_mat = any("material" in e or ("palette" in e and any("material" in q for q in e["palette"].values()))
                      for e in elems)
        mat = np.ones(gr.node, dtype=np.uint8, order="F") if has_mat else None
        shapes.rasterize_shape(mk.f, elems, gr, mirror=mode == "CUSTOM_REF", vac=vac, mat=mat,
                               matnames=cfg.materials)
        if mat is not None:
            ghost_planes(mat, gr)
            mk = Masks(mk.f, mk.τx, mk.τy, mk.τz, mk.τψ, None, mat)
        if vac.any():
            return sculpt(mk, gr, vac)
        return mk
    mk = box_masks(gr)
    for d in _defects(cfg, gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2):
        _paint(mk.f, d, gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2)
    return mk


def ghost_planes(v: np.ndarray, gr: Grid) -> np.ndarray:
    """_ghost_planes! (geometry.jl:529-535): the ghost planes of a node map copy the block plane inside, x then y
    then z."""
    x1, x2, y1, y2, z1, z2 = gr.x1 - 1, gr.x2 - 1, gr.y1 - 1, gr.y2 - 1, gr.z1 - 1, gr.z2 - 1
    v[x1, :, :] = v[x1 + 1, :, :]
    v[x2 + 1, :, :] = v[x2, :, :]
    v[:, y1, :] = v[:, y1 + 1, :]
    v[:, y2 + 1, :] = v[:, y2, :]
    v[:, :, z1] = v[:, :, z1 + 1]
    v[:, :, z2 + 1] = v[:, :, z2]
    return v


def with_materials(mk: Masks, gr: Grid, material) -> Masks:
    """The masks with a material map: `material(i, j, k)` (1-based node) gives the material of each node (1 = the
    Stepper's model), or `material` is that node array itself; the ghost planes then copy the block (as a shape
    region with material = "name" rasterised by build_masks, geometry.jl:485-511)."""
    if isinstance(material, np.ndarray):
        if material.shape != gr.node:
            raise ValueError(f"material map: the node shape {gr.node}")
        mat = np.asfortranarray(material, dtype=np.uint8).copy(order="F")
    else:
        mat = np.ones(gr.node, dtype=np.uint8, order="F")
        for c in np.ndindex(*gr.node):
            mat[c] = material(c[0] + 1, c[1] + 1, c[2] + 1)
    ghost_planes(mat, gr)
    return Masks(mk.f, mk.τx, mk.τy, mk.τz, mk.τψ, mk.vac, mat)


def sculpt(mk: Masks, gr: Grid, vac: np.ndarray) -> Masks:
    """sculpt! (geometry.jl:537-557): the masks of a sample with vacuum.  `vac` marks the vacuum nodes of the block
    (node-shaped bool); its ghost planes take the vacuum of the plane they copy, and on every vacuum node
    τψ = f = 0 and every link that touches it leaves the block (τ = 0: no supercurrent, no neighbour read across it,
    the zero-flux condition of a free surface)."""
    v = np.asfortranarray(np.array(vac, dtype=bool), dtype=bool).copy(order="F")
    if v.shape != gr.node:
        raise ValueError(f"vacuum map: the node shape {gr.node}")
    ghost_planes(v, gr)
    f, tx, ty, tz, tp = (np.array(a, order="F", copy=True) for a in (mk.f, mk.τx, mk.τy, mk.τz, mk.τψ))
    tp[v] = 0.0
    f[v] = 0.0
    tx[v] = 0.0
    ty[v] = 0.0
    tz[v] = 0.0
    tx[:-1][v[1:]] = 0.0       # the link from i−1 into a vacuum node
    ty[:, :-1][v[:, 1:]] = 0.0
    tz[:, :, :-1][v[:, :, 1:]] = 0.0
    x1, x2, y1, y2, z1, z2 = gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2
    if not (tp[x1:x2, y1:y2, z1:z2] > 0).any():
        raise ValueError("the shape leaves no material: everything is vacuum")
    return Masks(f, tx, ty, tz, tp, v, mk.mat)


def conducting_nodes(gr: Grid, mk: Masks) -> np.ndarray:
    """The σn nodes (geometry.jl:545-560): the bar y1:y2+1 × z1:z2+1 along all of x, minus the vacuum of a sculpted
    sample (a node outside x1..x2+1 takes the vacuum of the face node it continues)."""
    c = np.zeros(gr.node, dtype=bool, order="F")
    c[:, gr.y1 - 1:gr.y2 + 1, gr.z1 - 1:gr.z2 + 1] = True
    if mk.vac is not None:
        ii = np.clip(np.arange(1, gr.Nx + 2), gr.x1, gr.x2 + 1) - 1
        vv = mk.vac[ii][:, gr.y1 - 1:gr.y2 + 1, gr.z1 - 1:gr.z2 + 1]
        sub = c[:, gr.y1 - 1:gr.y2 + 1, gr.z1 - 1:gr.z2 + 1]
        sub[vv] = False
    return c
