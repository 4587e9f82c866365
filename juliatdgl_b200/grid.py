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
    """The catalogue keywords of geometry.jl:22-40 that the WEDGE / SIM modes read, and the shape file of the CUSTOM
    modes (geom_file; materials: the names of the run file's [materials.<name>] tables, in order)."""
    GEOM_MODE: str = "SIM"
    geom_file: str = ""
    materials: tuple = ()
    wedge_depth: float = 0.35
    wedge_half: float = 0.20
    wedge_depth2: float = 0.00
    inj_margin: int = 6
    x_shift: float = 0.0
    y_shift: float = 0.0
    z_mode: str = "through"
    current_axis: str = "x"


@dataclass
class _Wedge:
    xc: int
    yc: int
    dir: int
    half: int
    depth: int
    f: float = 0.0
    zlo: int = 0
    zhi: int = 0


def _defects(cfg: GeomSpec, x1, x2, y1, y2, z1, z2):
    mode = cfg.GEOM_MODE.upper()
    if mode.endswith("_REF") and len(mode) > 4:
        raise NotImplementedError("mirrored (_REF) catalogue modes are not part of the ladder configurations")
    xc = oround((x1 + x2) / 2)
    nx_sc, ny_sc = x2 - x1 + 1, y2 - y1 + 1
    D = []
    if mode == "SIM":
        pass
    elif mode in ("WEDGE", "WEDGE_BOTH"):
        D.append(_Wedge(xc=xc, yc=y1, dir=+1, half=oround(cfg.wedge_half * nx_sc), depth=oround(cfg.wedge_depth * ny_sc)))
        if mode == "WEDGE_BOTH" and cfg.wedge_depth2 > 0:
            D.append(_Wedge(xc=xc, yc=y2 + 1, dir=-1, half=oround(cfg.wedge_half * nx_sc),
                            depth=oround(cfg.wedge_depth2 * ny_sc)))
    else:
        raise NotImplementedError(f"GEOM_MODE {cfg.GEOM_MODE}: only SIM, WEDGE and WEDGE_BOTH are built here")
    if cfg.x_shift != 0:
        dxs = oround(cfg.x_shift * nx_sc)
        for d in D:
            d.xc += dxs
    if cfg.y_shift != 0:
        dys = oround(cfg.y_shift * ny_sc)
        for d in D:
            d.yc += dys
    zc = oround((z1 + z2) / 2)
    zm = cfg.z_mode.lower()
    for d in D:
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


def _paint_wedge(fmask, d: _Wedge, x1, x2, y1, y2, z1, z2):
    """geometry.jl:120-137 (1-based loop indices, 0-based array access)."""
    zA = max(z1, d.zlo)
    zB = min(z2, d.zhi)
    for k in range(zA, zB + 1):
        for j in range(y1, y2 + 1):
            layer = d.dir * (j - d.yc)
            if layer >= 0 and layer < d.depth:
                frac = 1 - layer / d.depth
                w_steep = max(1, oround(2 * frac))
                w_gentle = oround(d.half * frac)
                for i in range(x1, x2 + 1):
                    dxr = i - d.xc
                    if -w_steep <= dxr <= w_gentle:
                        fmask[i - 1, j - 1, k - 1] = d.f


def build_masks(cfg: GeomSpec, gr: Grid) -> Masks:
    """geometry.jl:485-511: the catalogue modes SIM / WEDGE / WEDGE_BOTH, and a shape file (CUSTOM, CUSTOM_REF:
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
        _paint_wedge(mk.f, d, gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2)
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
