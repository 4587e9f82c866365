"""Shape files (GEOM_MODE = "CUSTOM" | "CUSTOM_REF", juliatdgl_b200/shapes.py) against gtdgl's rules for them
(gtdgl/src/shapes.jl) and the expectations of the reference's own test (gtdgl/test/test_geometry.jl:35-70: a disc on
the y–z plane, the disc kept with outside = true, a rectangle on the x–z plane over part of y, and a cable of vacuum
with its free-surface masks), plus: a catalogue mask written as a voxel file rasterises back to the same mask bit for
bit, the mirror mode, each element type, the first version's key names, and material regions."""
import math

import numpy as np
import pytest

import juliatdgl_b200 as T
from juliatdgl_b200 import shapes
from juliatdgl_b200.grid import conducting_nodes
from juliatdgl_b200.scheme import link_conductivity


def forma(tmp_path, txt, mode="CUSTOM", **kw):
    p = tmp_path / f"f{abs(hash(txt))}.toml"
    p.write_text(txt)
    return T.GeomSpec(GEOM_MODE=mode, geom_file=str(p), **kw)


def blk(a, gr):
    return a[gr.x1 - 1:gr.x2, gr.y1 - 1:gr.y2, gr.z1 - 1:gr.z2]


def physical(gr):
    i = np.arange(gr.x1, gr.x2 + 1)[:, None, None]
    j = np.arange(gr.y1, gr.y2 + 1)[None, :, None]
    k = np.arange(gr.z1, gr.z2 + 1)[None, None, :]
    return (i - gr.x1) * gr.dx, (j - gr.y1) * gr.dy, (k - gr.z1) * gr.dz


@pytest.fixture
def gr():
    return T.Grid.make(20, 12, 12, dx=0.5, buf=2)


def test_disc_outside_and_rectangle_on_other_faces(gr, tmp_path):
    X, Y, Z = physical(gr)
    mk = T.build_masks(forma(tmp_path, '[[shape]]\ntype = "circle"\naxis = "x"\nu = 3.0\nv = 2.5\nr = 1.5\nf = 0.3\n'), gr)
    disc = np.broadcast_to((Y - 3.0) ** 2 + (Z - 2.5) ** 2 <= 1.5 ** 2 + 1e-9, (X + Y + Z).shape)
    assert np.array_equal(blk(mk.f, gr), np.where(disc, 0.3, 1.0)) and mk.vac is None
    mk2 = T.build_masks(forma(tmp_path, '[[shape]]\ntype = "circle"\naxis = "x"\nu = 3.0\nv = 2.5\nr = 1.5\nf = 0.3\n'
                                        'outside = true\n'), gr)
    assert np.array_equal(blk(mk2.f, gr), np.where(disc, 1.0, 0.3))
    mk3 = T.build_masks(forma(tmp_path, '[[shape]]\ntype = "rect"\naxis = "y"\nu = 5.0\nv = 3.0\nw = 2.0\nh = 2.0\n'
                                        'along = [0.0, 2.0]\n'), gr)
    want = (np.abs(X - 5.0) <= 1 + 1e-9) & (np.abs(Z - 3.0) <= 1 + 1e-9) & (Y <= 2 + 1e-9)
    assert np.array_equal(blk(mk3.f, gr), np.where(want, 0.0, 1.0))


CABLE = """[[shape]]
type = "circle"
axis = "x"
u = 3.0
v = 3.0
r = 2.75
along = "all"
outside = true
vacuum = true
"""


def test_a_cable_of_vacuum_is_a_sculpted_sample(gr, tmp_path):
    mk = T.build_masks(forma(tmp_path, CABLE), gr)
    v = mk.vac
    x1, x2, y1, y2, z1, z2 = gr.x1 - 1, gr.x2 - 1, gr.y1 - 1, gr.y2 - 1, gr.z1 - 1, gr.z2 - 1
    assert v is not None and v.any() and not v[x1 + 1:x2 + 1, y1 + 1:y2 + 1, z1 + 1:z2 + 1].all()
    assert np.array_equal(v[x1], v[x1 + 1]) and np.array_equal(v[:, y2 + 1], v[:, y2])
    assert np.array_equal(v[:, :, z2 + 1], v[:, :, z2])
    assert (mk.τψ[v] == 0).all() and (mk.f[v] == 0).all()
    for i in range(x1, x2 + 1):
        sl = (i, slice(y1, y2 + 2), slice(z1, z2 + 2))
        touch = v[sl] | v[(i + 1,) + sl[1:]]
        assert (mk.τx[sl][touch] == 0).all() and (mk.τx[sl][~touch] == 1).all()
    c = conducting_nodes(gr, mk)
    assert np.array_equal(c[0], ~v[x1] & c[x1]) and np.array_equal(c[-1], c[x2 + 1])
    box = T.box_masks(gr)
    assert np.array_equal(conducting_nodes(gr, T.build_masks(T.GeomSpec(GEOM_MODE="WEDGE"), gr)),
                          conducting_nodes(gr, box))
    for a, b in zip(link_conductivity(gr, 0.01, 1.0, cond=conducting_nodes(gr, box)), link_conductivity(gr, 0.01, 1.0)):
        assert np.array_equal(a, b)


def test_a_catalogue_mask_written_as_voxels_comes_back_to_the_bit(tmp_path):
    gr = T.Grid.make(40, 24, 6, dx=0.5, buf=1)
    cat = T.build_masks(T.GeomSpec(GEOM_MODE="WEDGE_BOTH", wedge_depth2=0.2), gr)
    p = shapes.write_voxels(str(tmp_path / "w.toml"), cat.f, gr, comment="WEDGE_BOTH 40x24x6")
    back = T.build_masks(T.GeomSpec(GEOM_MODE="CUSTOM", geom_file=p), gr)
    assert np.array_equal(back.f, cat.f)


def test_the_mirror_mode_reflects_y(gr, tmp_path):
    txt = '[[shape]]\ntype = "triangle"\nx = 4.0\ny = 0.0\nw = 3.0\nh = 2.5\nskew = 1.0\nf = 0.2\n'
    a = T.build_masks(forma(tmp_path, txt), gr).f
    b = T.build_masks(forma(tmp_path, txt, mode="CUSTOM_REF"), gr).f
    y1, y2 = gr.y1, gr.y2
    for j in range(y1 + 1, y2 + 1):   # node j is evaluated at node (y1 + y2 + 1) − j: the interior nodes' mirror
        assert np.array_equal(blk(b, gr)[:, j - y1], blk(a, gr)[:, (y1 + y2 + 1 - j) - y1])
    assert not np.array_equal(a, b)


def test_each_element_type(gr, tmp_path):
    X, Y, Z = physical(gr)
    L = ((gr.x2 - gr.x1) * gr.dx, (gr.y2 - gr.y1) * gr.dy, (gr.z2 - gr.z1) * gr.dz)
    full = np.ones_like(X + Y + Z)
    cases = {
        '[[shape]]\ntype = "sphere"\nx = 5.0\ny = 3.0\nzc = 2.0\nr = 1.6\nf = 0.5\n':
            (X - 5) ** 2 + (Y - 3) ** 2 + (Z - 2) ** 2 <= 1.6 ** 2 + 1e-9,
        '[[shape]]\ntype = "rect"\nx = 5.0\ny = 3.0\nw = 4.0\nh = 1.0\nrot = 90.0\nz = "bottom"\nf = 0.5\n':
            (np.abs(Y - 3) <= 2 + 1e-9) & (np.abs(X - 5) <= 0.5 + 1e-9) & (Z <= L[2] / 2 + 1e-9),
        '[[shape]]\ntype = "ngon"\nx = 5.0\ny = 3.0\nn = 4\nr = 2.0\nz = [1.0, 3.0]\nf = 0.5\n':
            (np.abs(X - 5) + np.abs(Y - 3) <= 2 + 1e-9) & (Z >= 1 - 1e-9) & (Z <= 3 + 1e-9),
        '[[shape]]\ntype = "polygon"\npoints = [[1.0, 1.0], [6.0, 1.0], [6.0, 4.0], [1.0, 4.0]]\nf = 0.5\n':
            (X >= 1 - 1e-9) & (X <= 6 + 1e-9) & (Y >= 1 - 1e-9) & (Y <= 4 + 1e-9),
        '[[shape]]\ntype = "triangle"\nx = 5.0\ny = 0.0\nw = 4.0\nh = 2.0\nz = "top"\nf = 0.5\n':
            (Y >= -1e-9) & (np.abs(X - 5) <= 2 * (1 - Y / 2) + 1e-9) & (Z >= L[2] / 2 - 1e-9),
    }
    for txt, inside in cases.items():
        f = blk(T.build_masks(forma(tmp_path, txt), gr).f, gr)
        assert np.array_equal(f, np.where(np.broadcast_to(inside, full.shape), 0.5, 1.0)), txt
    # pixels: 13 rows, the first the largest y; row r (0-based) at y = (12 − r) dx and column c at x = c dx
    rows = ["." * 21] * 13
    rows[10] = "....#" + "." * 16          # x = 2.0, y = 1.0 ξσ: block node offsets (4, 2)
    rows[9] = "....a" + "." * 16           # x = 2.0, y = 1.5 ξσ: (4, 3), in the bottom half of z only
    txt = ('[[shape]]\ntype = "pixels"\ndx = 0.5\nrows = """\n' + "\n".join(rows) + '\n"""\n'
           '[shape.palette]\n"#" = { f = 0.0 }\n"a" = { z = "bottom", f = 0.25 }\n')
    f = blk(T.build_masks(forma(tmp_path, txt), gr).f, gr)
    want = np.ones_like(f)
    want[4, 2, :] = 0.0
    want[4, 3, :] = np.where(np.arange(f.shape[2]) * gr.dz <= L[2] / 2 + 1e-9, 0.25, 1.0)
    assert np.array_equal(f, want)


def test_the_first_versions_key_names(gr, tmp_path):
    new = '[[shape]]\ntype = "circle"\nx = 4.0\ny = 3.0\nr = 2.0\nz = "all"\nf = 0.1\n'
    old = '[[forma]]\ntipo = "circulo"\nx = 4.0\ny = 3.0\nr = 2.0\nz = "todo"\nf = 0.1\n'
    assert np.array_equal(T.build_masks(forma(tmp_path, new), gr).f, T.build_masks(forma(tmp_path, old), gr).f)
    with pytest.raises(ValueError):
        shapes.parse_shape('[[shape]]\ntype = "blob"\n')


def test_material_regions(gr, tmp_path):
    txt = ('[[shape]]\ntype = "rect"\nx = 5.0\ny = 3.0\nw = 2.0\nh = 2.0\nmaterial = "top"\n'
           '[[shape]]\ntype = "circle"\nx = 2.0\ny = 2.0\nr = 1.0\nmaterial = "barrier"\nf = 0.5\n')
    mk = T.build_masks(forma(tmp_path, txt, materials=("barrier", "top")), gr)
    X, Y, Z = physical(gr)
    rect = np.broadcast_to((np.abs(X - 5) <= 1 + 1e-9) & (np.abs(Y - 3) <= 1 + 1e-9), blk(mk.f, gr).shape)
    disc = np.broadcast_to((X - 2) ** 2 + (Y - 2) ** 2 <= 1 + 1e-9, rect.shape)
    want_mat = np.where(disc, 2, np.where(rect, 3, 1))
    assert np.array_equal(blk(mk.mat, gr), want_mat)
    assert np.array_equal(blk(mk.f, gr), np.where(disc, 0.5, 1.0))   # a material region writes f = 1 unless given
    x1 = gr.x1 - 1
    assert np.array_equal(mk.mat[x1], mk.mat[x1 + 1])               # ghost planes copy the block
    with pytest.raises(ValueError):
        T.build_masks(forma(tmp_path, txt, materials=("top",)), gr)


def test_vacuum_needs_the_sculpted_path(gr):
    elems = shapes.parse_shape(CABLE)
    with pytest.raises(ValueError):
        shapes.rasterize_shape(np.ones(gr.node, order="F"), elems, gr)
    assert math.isnan(shapes._value({"vacuum": True}))


def test_the_reference_golden_shape_masks(tmp_path):
    """Every shape-file case of the reference's golden masks (gtdgl/test/golden/masks.jld2, written by release 1.2;
    the fixture holds the masks and the shape files' text, tests/golden/make_fixtures.py): the same mask to the
    bit, as gtdgl/test/test_geometry.jl:7-21 asks of the reference."""
    import json
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "masks_custom.npz"))
    meta = json.loads(str(d["meta"]))
    texts = json.loads(str(d["shape_files"]))
    assert len(meta) == 46
    for name, files in texts.items():
        (tmp_path / name).write_text(files)
    bad = []
    for name, m in sorted(meta.items()):
        g = m["malla"]
        gr = T.Grid.make(g["Nx_sc"], g["Ny_sc"], g["Nz_sc"], dx=g["dx"], buf=g["buf"])
        spec = T.GeomSpec(GEOM_MODE=m["geo"]["GEOM_MODE"], geom_file=str(tmp_path / m["geo"]["geom_file"]))
        if not np.array_equal(T.build_masks(spec, gr).f, d[name]):
            bad.append(name)
    assert bad == []


def test_the_reference_golden_catalogue_masks():
    """Every catalogue case of the reference's golden masks (18 modes and their _REF mirrors on two meshes, the z
    modes, the shifts, the prism angle, the fgrad direction; written by release 1.2): the same mask to the bit."""
    import json
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "masks_catalogue.npz"))
    meta = json.loads(str(d["meta"]))
    assert len(meta) == 82
    bad = []
    for name, m in sorted(meta.items()):
        g = m["malla"]
        gr = T.Grid.make(g["Nx_sc"], g["Ny_sc"], g["Nz_sc"], dx=g["dx"], buf=g["buf"])
        if not np.array_equal(T.build_masks(T.GeomSpec(**m["geo"]), gr).f, d[name]):
            bad.append(name)
    assert bad == []
