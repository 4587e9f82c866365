"""Sculpted samples (a shape with vacuum: sculpt!, gtdgl/src/geometry.jl:537-557) on the host mirror and the oracle:
the masks sculpt! leaves, the conducting nodes and the section of the self-field, the constructor's guards, and the
reference's own test of the free surface (gtdgl/test/test_physics.jl:583-600): with H = 0 and J = 0 the uniform state
stays uniform up to the surface (zero flux) and Ψ = 0 in the vacuum.
"""
import numpy as np
import pytest

import cases
import juliatdgl_b200 as T
from juliatdgl_b200.grid import conducting_nodes, sculpt
from juliatdgl_b200.scheme import bar_field
from oracle import pyoracle


def slot(gr):
    v = np.zeros(gr.node, dtype=bool)
    v[gr.x1 + 4:gr.x1 + 8, gr.y1:gr.y1 + 3, gr.z1:gr.z2] = True
    return v


def test_sculpt_follows_the_reference_rule():
    gr = T.Grid.make(16, 8, 6, dx=0.5, buf=2)
    mk0 = T.box_masks(gr)
    mk = sculpt(mk0, gr, slot(gr))
    v = mk.vac
    # ghost planes copy the plane inside (x, then y, then z)
    assert np.array_equal(v[gr.x1 - 1], v[gr.x1]) and np.array_equal(v[:, gr.y1 - 1], v[:, gr.y1])
    # every vacuum node and every link into it: τ = 0; τψ = f = 0 on the vacuum
    for (i, j, k) in zip(*np.nonzero(v)):
        assert mk.τψ[i, j, k] == 0 and mk.f[i, j, k] == 0 and mk.τx[i, j, k] == 0 and mk.τy[i, j, k] == 0
        assert i == 0 or mk.τx[i - 1, j, k] == 0
        assert j == 0 or mk.τy[i, j - 1, k] == 0
        assert k == 0 or mk.τz[i, j, k - 1] == 0
    assert np.array_equal(mk.τx[~v & (np.roll(v, -1, axis=0) == 0)], mk0.τx[~v & (np.roll(v, -1, axis=0) == 0)])
    c = conducting_nodes(gr, mk)
    assert not c[gr.x1 + 5, gr.y1, gr.z1 + 1] and c[gr.x1 + 5, gr.y1 + 4, gr.z1 + 1] and not c[0, 0, 0]


def test_a_full_section_gives_the_bar_field():
    gr = T.Grid.make(12, 6, 4, dx=0.5, buf=2)
    a = bar_field(gr, backend="numpy")
    b = bar_field(gr, backend="numpy", section=np.ones((gr.y2 - gr.y1 + 2, gr.z2 - gr.z1 + 2), dtype=bool))
    for q in ("hy_z", "hy_y", "hz_z", "hz_y", "hz_x", "hy_x"):
        assert np.array_equal(getattr(a, q), getattr(b, q))


def test_guards():
    gr = T.Grid.make(16, 8, 6, dx=0.5, buf=2)
    mk = sculpt(T.box_masks(gr), gr, slot(gr))
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    with pytest.raises(ValueError):      # the free surface needs the insulating padding
        T.Stepper.make(md, gr, mk)
    with pytest.raises(ValueError):      # and the field of the bar
        T.Stepper.make(md, gr, mk, σvac=0.01, selffield_bc="slab")
    with pytest.raises(ValueError):      # a shape that leaves no material
        sculpt(T.box_masks(gr), gr, np.ones(gr.node, dtype=bool))


def free_surface(run):
    """test_physics.jl:594-600 on a slot: |Ψ|² after 100 steps at H = J = 0 against a node far from the slot."""
    gr = T.Grid.make(16, 8, 6, dx=0.5, buf=2)
    mk = sculpt(T.box_masks(gr), gr, slot(gr))
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    st = T.Stepper.make(md, gr, mk, σvac=0.01)
    s = run(st, T.initial_state(md, gr, mk, 0.0), 100)
    ref = abs(s.G[0][gr.x1 + 11, gr.y1 + 5, gr.z1 + 2]) ** 2
    live = ~mk.vac & (mk.τψ > 0)
    dev = np.max(np.abs(np.abs(s.G[0][live]) ** 2 - ref))
    return dev, max(np.abs(s.G[µ][mk.vac]).max() for µ in range(2))


def test_free_surface_on_the_oracle():
    dev, vac = free_surface(lambda st, s, n: pyoracle.run(st, s, n, 0.0, 0.0))
    assert dev < 1e-13 and vac == 0


@pytest.mark.parametrize("kind", cases.VACUUM_KINDS)
def test_vacuum_cases_step_on_the_oracle(kind):
    st, s, H, HJ = cases.vacuum(kind)
    s1 = pyoracle.run(st, s, 10, H, HJ)
    assert all(np.all(np.isfinite(s1.G[µ])) for µ in range(st.model.N))
    assert max(np.abs(s1.G[µ][st.masks.vac]).max() for µ in range(st.model.N)) == 0
