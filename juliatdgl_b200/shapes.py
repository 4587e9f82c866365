"""Geometry from a shape file (GEOM_MODE = "CUSTOM" | "CUSTOM_REF"), as gtdgl/src/shapes.jl reads and rasterises it.

A shape file (TOML) lists, in order, regions of the sample box whose condensation strength f is overwritten (or that
become vacuum, or take a material).  Positions and sizes are in units of ξσ with the origin at the corner
(x1, y1, z1), so a file rasterises on any mesh; nodes are tested at their physical position X = (i − x1) dx over
the node range x1:x2, y1:y2, z1:z2 (shapes.jl:1-50 for the format).  CUSTOM_REF evaluates the shapes at the
mirrored node j → (y1 + y2 + 1) − j.

Element types: circle, rect, triangle, ngon, polygon, sphere, pixels, voxels; keys x, y (centre), r, w, h, skew,
n, points, rot (degrees about the axis), z ("all" | "bottom" | "top" | "buried" | [z0, z1]), f, outside, vacuum,
material; axis = "x" | "y" draws the figure on the y–z or x–z plane (centre u, v) and extrudes it over `along`.
The first version's keys ([[forma]], tipo = "circulo", z = "todo", …) are read too.
"""
from __future__ import annotations

import math
import tomllib

import numpy as np

Z_WORDS = ("all", "bottom", "top", "buried")
TYPES = ("circle", "rect", "triangle", "ngon", "polygon", "sphere", "pixels", "voxels")
AXES = ("x", "y", "z")
TOL = 1e-9

# the names of the format's first version (shapes.jl:54-62)
_OLD_KEYS = {"tipo": "type", "sesgo": "skew", "puntos": "points", "filas": "rows", "paleta": "palette",
             "capas": "layers"}
_OLD_TYPES = {"circulo": "circle", "triangulo": "triangle", "ngono": "ngon", "poligono": "polygon",
              "esfera": "sphere", "pixeles": "pixels", "voxeles": "voxels"}
_OLD_Z = {"todo": "all", "abajo": "bottom", "arriba": "top", "enterrado": "buried"}


def _normalise_z(z):
    return _OLD_Z.get(z, z) if isinstance(z, str) else z


def _normalise(e: dict) -> dict:
    o = {_OLD_KEYS.get(k, k): v for k, v in e.items()}
    if "type" in o:
        o["type"] = _OLD_TYPES.get(o["type"], o["type"])
    if "z" in o:
        o["z"] = _normalise_z(o["z"])
    if "palette" in o:
        o["palette"] = {ch: {k: (_normalise_z(v) if k == "z" else v) for k, v in q.items()}
                        for ch, q in o["palette"].items()}
    return o


def parse_shape(text: str, name: str = "shape file") -> list:
    """The elements of a shape file's text (read_shape, shapes.jl:79-92)."""
    d = tomllib.loads(text)
    raw = d.get("shape", d.get("forma"))
    if raw is None:
        raise ValueError(f"{name}: no [[shape]] block")
    elems = [_normalise(e) for e in raw]
    for n, e in enumerate(elems, 1):
        if "type" not in e:
            raise ValueError(f"{name}: shape #{n} has no 'type'")
        if e["type"] not in TYPES:
            raise ValueError(f"{name}: shape #{n} has unknown type '{e['type']}'")
    return elems


def read_shape(path: str) -> list:
    """The elements of the shape file at `path`."""
    with open(path, "rb") as fh:
        text = fh.read().decode()
    return parse_shape(text, path)


def _range(spec, L):
    """The extent in ξσ of a z (or along) specification, L the top node plane the painter reaches."""
    if spec is None:
        return -math.inf, math.inf
    if isinstance(spec, str):
        if spec == "all":
            return -math.inf, math.inf
        if spec == "bottom":
            return -math.inf, L / 2
        if spec == "top":
            return L / 2, math.inf
        if spec == "buried":
            return L / 4, 3 * L / 4
        raise ValueError(f"z = '{spec}' is not one of {Z_WORDS} nor [z0, z1]")
    if len(spec) != 2:
        raise ValueError(f"z = {spec}: expected [z0, z1]")
    return float(spec[0]), float(spec[1])


def _local(e, X, Y):
    """(X, Y) in the element's frame: centre at the origin, its rotation undone."""
    dx = X - float(e.get("x", 0.0))
    dy = Y - float(e.get("y", 0.0))
    th = math.radians(float(e.get("rot", 0.0)))
    if th == 0.0:
        return dx, dy
    c, s = math.cos(th), math.sin(th)
    return c * dx + s * dy, -s * dx + c * dy


def _in_polygon(px, py, vx, vy) -> bool:
    """Crossing number; a point on an edge counts as inside."""
    n = len(vx)
    inside = False
    j = n - 1
    for i in range(n):
        xi, yi, xj, yj = vx[i], vy[i], vx[j], vy[j]
        cr = (xj - xi) * (py - yi) - (yj - yi) * (px - xi)
        if (abs(cr) <= TOL * max(1.0, math.hypot(xj - xi, yj - yi)) and
                min(xi, xj) - TOL <= px <= max(xi, xj) + TOL and min(yi, yj) - TOL <= py <= max(yi, yj) + TOL):
            return True
        if (yi > py) != (yj > py):
            xint = xi + (py - yi) * (xj - xi) / (yj - yi)
            if px < xint:
                inside = not inside
        j = i
    return inside


def _inside(e, X, Y, Z, L) -> bool:
    """Is the physical point (X, Y, Z) inside element e (not the pixel or voxel layers)?"""
    t = e["type"]
    if t == "sphere":
        cx, cy, cz, r = float(e["x"]), float(e["y"]), float(e["zc"]), float(e["r"])
        return (X - cx) ** 2 + (Y - cy) ** 2 + (Z - cz) ** 2 <= r ** 2 + TOL
    ax = e.get("axis", "z")
    if ax not in AXES:
        raise ValueError(f"axis = '{ax}' is not one of {AXES}")
    if ax != "z":
        # the figure in its own plane: (u, v, along) = (y, z, x) or (x, z, y), centred at (u, v)
        A, la, U, V = (X, L[0], Y, Z) if ax == "x" else (Y, L[1], X, Z)
        a0, a1 = _range(e.get("along", "all"), la)
        if not (a0 - TOL <= A <= a1 + TOL):
            return False
        q = {k: v for k, v in e.items() if k not in ("x", "y", "z", "u", "v", "axis", "along")}
        q["x"], q["y"] = e.get("u", 0.0), e.get("v", 0.0)
        return _inside(q, U, V, 0.0, L)
    z0, z1 = _range(e.get("z", "all"), L[2])
    if not (z0 - TOL <= Z <= z1 + TOL):
        return False
    if t == "circle":
        cx, cy, r = float(e["x"]), float(e["y"]), float(e["r"])
        return (X - cx) ** 2 + (Y - cy) ** 2 <= r ** 2 + TOL
    if t == "rect":
        u, v = _local(e, X, Y)
        return abs(u) <= float(e["w"]) / 2 + TOL and abs(v) <= float(e["h"]) / 2 + TOL
    if t == "triangle":
        u, v = _local(e, X, Y)
        w, h, s = float(e["w"]), float(e["h"]), float(e.get("skew", 0.0))
        return _in_polygon(u, v, (-w / 2, w / 2, s), (0.0, 0.0, h))
    if t == "ngon":
        u, v = _local(e, X, Y)
        n, r = int(e["n"]), float(e["r"])
        vx = [r * math.cos(2 * math.pi * k / n) for k in range(n)]
        vy = [r * math.sin(2 * math.pi * k / n) for k in range(n)]
        return _in_polygon(u, v, vx, vy)
    if t == "polygon":
        pts = e["points"]
        if len(pts) < 3:
            raise ValueError("polygon with fewer than 3 points")
        u, v = _local(e, X, Y)   # x, y default to 0: the points are absolute unless offset
        return _in_polygon(u, v, [float(p[0]) for p in pts], [float(p[-1]) for p in pts])
    raise ValueError(f"type '{t}' not handled here")


def _rows(t):
    """The rows of a pixel or voxel block: a string (one trailing newline dropped, as Julia's chomp) or a list."""
    if isinstance(t, str):
        return (t[:-1] if t.endswith("\n") else t).split("\n")
    return list(t)


def _pick(pal, ch, what):
    if ch in (".", " "):
        return None
    if ch not in pal:
        raise ValueError(f"{what}: character '{ch}' is not in the palette")
    return pal[ch]


def _pixel(e, X, Y, Z, Lz):
    """The palette entry the pixel layer writes at (X, Y, Z), or None (first row = largest y, first column x = 0)."""
    d = float(e.get("dx", 0.5))
    rows = _rows(e["rows"])
    nr = len(rows)
    c = _round(X / d) + 1
    r = nr - _round(Y / d)
    if not (1 <= r <= nr) or not (1 <= c <= len(rows[r - 1])):
        return None
    q = _pick(e["palette"], rows[r - 1][c - 1], "pixels")
    if q is None:
        return None
    z0, z1 = _range(q.get("z", "all"), Lz)
    return q if z0 - TOL <= Z <= z1 + TOL else None


def _voxel(e, X, Y, Z):
    """The palette entry the voxel layer writes at (X, Y, Z), or None (first block of rows = z = 0)."""
    d = float(e.get("dx", 0.5))
    dz = float(e.get("dz", d))
    layers = e["layers"]
    l = _round(Z / dz) + 1
    if not 1 <= l <= len(layers):
        return None
    rows = _rows(layers[l - 1])
    nr = len(rows)
    r = nr - _round(Y / d)
    c = _round(X / d) + 1
    if not (1 <= r <= nr) or not (1 <= c <= len(rows[r - 1])):
        return None
    return _pick(e["palette"], rows[r - 1][c - 1], "voxels")


def _round(x: float) -> int:
    """Julia's round(Int, x): to nearest, ties to even (as Python's round)."""
    return int(round(x))


def _value(q) -> float:
    """What an element or palette entry writes: its f, or NaN for vacuum (a material region is f = 1 unless given)."""
    if q.get("vacuum", False) is True:
        return math.nan
    return float(q.get("f", 1.0 if "material" in q else 0.0))


def rasterize_shape(fmask: np.ndarray, elems: list, gr, *, mirror: bool = False, vac: np.ndarray | None = None,
                    mat: np.ndarray | None = None, matnames=()) -> np.ndarray:
    """Writes the f of each element, in order, on the nodes x1:x2, y1:y2, z1:z2 of the node arrays (rasterize_shape!,
    shapes.jl:242-285).  A vacuum element marks its nodes in `vac` (f = 0 there); a later element that writes an f
    gives the material back.  An element with material = "name" writes 1 + the index of that name in `matnames` in
    `mat`."""
    x1, x2, y1, y2, z1, z2 = gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2
    dx, dy, dz = gr.dx, gr.dy, gr.dz
    L = ((x2 - x1) * dx, (y2 - y1) * dy, (z2 - z1) * dz)
    names = [str(n) for n in matnames]
    for k in range(z1, z2 + 1):
        Z = (k - z1) * dz
        for j in range(y1, y2 + 1):
            jj = (y1 + y2 + 1) - j if mirror else j
            Y = (jj - y1) * dy
            for i in range(x1, x2 + 1):
                X = (i - x1) * dx
                for e in elems:
                    t = e["type"]
                    if t == "pixels":
                        q = _pixel(e, X, Y, Z, L[2])
                    elif t == "voxels":
                        q = _voxel(e, X, Y, Z)
                    else:
                        q = e if _inside(e, X, Y, Z, L) != (e.get("outside", False) is True) else None
                    if q is None:
                        continue
                    v = _value(q)
                    c = (i - 1, j - 1, k - 1)
                    if "material" in q:
                        if mat is None:
                            raise ValueError(f"material = \"{q['material']}\": no material tables were given")
                        if str(q["material"]) not in names:
                            raise ValueError(f"material = \"{q['material']}\" is not one of the materials "
                                             f"({', '.join(names)})")
                        mat[c] = names.index(str(q["material"])) + 2
                    if math.isnan(v):
                        if vac is None:
                            raise ValueError("vacuum = true needs an insulating padding (sigma_vac)")
                        vac[c] = True
                        fmask[c] = 0.0
                    else:
                        if vac is not None:
                            vac[c] = False
                        fmask[c] = v
    return fmask


def write_voxels(path: str, fmask: np.ndarray, gr, comment: str = "") -> str:
    """The mask on the nodes x1:x2, y1:y2, z1:z2 as a voxel shape file: any 3D pattern, one character per value of
    f other than 1 (write_voxels, shapes.jl:287-325)."""
    chars = "#abcdefghijklmnopqrstuvwxyz0123456789ABCDEFGHIJKLMNOPQRSTUVWXYZ"
    pal = {}
    layers = []
    for k in range(gr.z1, gr.z2 + 1):
        rows = []
        for j in range(gr.y2, gr.y1 - 1, -1):
            row = []
            for i in range(gr.x1, gr.x2 + 1):
                v = float(fmask[i - 1, j - 1, k - 1])
                if v == 1:
                    row.append(".")
                else:
                    if v not in pal:
                        if len(pal) >= len(chars):
                            raise ValueError(f"more than {len(chars)} values of f")
                        pal[v] = chars[len(pal)]
                    row.append(pal[v])
            rows.append("".join(row))
        layers.append("\n".join(rows))
    with open(path, "w") as fh:
        if comment:
            fh.write(f"# {comment}\n")
        fh.write(f'[[shape]]\ntype = "voxels"\ndx = {gr.dx!r}\ndz = {gr.dz!r}\nlayers = [\n')
        for n, c in enumerate(layers):
            fh.write('"""\n' + c + '"""' + ("," if n < len(layers) - 1 else "") + "\n")
        fh.write("]\n\n[shape.palette]\n")
        for v, c in sorted(pal.items(), key=lambda kv: kv[1]):
            fh.write(f'"{c}" = {{ f = {v!r} }}\n')
    return path


def margin_nodes(fmask: np.ndarray, gr, inj_margin: int, current_axis: str = "x") -> int:
    """Nodes with f < 1 closer than `inj_margin` cells to the injection faces (margen_forma, shapes.jl:328-347)."""
    x1, x2, y1, y2, z1, z2 = gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2
    blk = fmask[x1 - 1:x2, y1 - 1:y2, z1 - 1:z2] < 1
    if current_axis.lower() == "x":
        i = np.arange(x1, x2 + 1)
        near = (i < x1 + inj_margin) | (i > x2 - inj_margin)
        return int(blk[near].sum())
    j = np.arange(y1, y2 + 1)
    near = (j < y1 + inj_margin) | (j > y2 - inj_margin)
    return int(blk[:, near].sum())
