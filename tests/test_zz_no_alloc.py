"""The separable inverse without device allocation (tdgl_sep_apply_noalloc), against the allocating entry point.

Callers that cannot allocate device memory (a solver inside another framework's memory pool or stream capture, a
process whose device memory is reserved up front, a plugin forbidden to allocate) pass their own input and output
buffers and get (I + aK)^{-1} from the library's fixed scratch.  This file runs last (pytest collects it after the
others), and each test works from a fresh or a reused scratch alike: two calls in a row must both match
tdgl_sep_apply, the context-based entry point, to rounding (the bases are evaluated on the device here and on
the host there, 1e-12 relative).
"""
import ctypes as C

import numpy as np
import pytest

import cases
from juliatdgl_b200 import abi, gpu
from juliatdgl_b200.scheme import sep_ranges, sep_unknowns

pytestmark = pytest.mark.gpu


def _lib():
    L = gpu.lib()
    L.tdgl_sep_apply_noalloc.argtypes = [C.POINTER(abi.Grid_t), C.c_double, C.POINTER(C.c_void_p),
                                         C.POINTER(C.c_void_p), C.c_void_p]
    L.tdgl_sep_apply_noalloc.restype = C.c_int
    return L


def _to_planes(gr, packed):
    """packed ranges (x-fastest per component, x | y | z) → three plane-major node-shaped arrays."""
    n1, n2, n3 = gr.Nx + 1, gr.Ny + 1, gr.Nz + 1
    out, off = [], 0
    for (i0, i1), (j0, j1), (k0, k1) in sep_ranges(gr):
        ni, nj, nk = i1 - i0 + 1, j1 - j0 + 1, k1 - k0 + 1
        blk = packed[off:off + ni * nj * nk].reshape((ni, nj, nk), order="F")
        off += ni * nj * nk
        pm = np.zeros((n2, n3, n1), order="F")
        pm[j0 - 1:j1, k0 - 1:k1, i0 - 1:i1] = blk.transpose(1, 2, 0)
        out.append(pm)
    return out


def _from_planes(gr, pms):
    parts = []
    for pm, ((i0, i1), (j0, j1), (k0, k1)) in zip(pms, sep_ranges(gr)):
        parts.append(pm[j0 - 1:j1, k0 - 1:k1, i0 - 1:i1].transpose(2, 0, 1).ravel(order="F"))
    return np.concatenate(parts)


def _noalloc(st, b_packed, in_place=False):
    import torch
    gr = st.grid
    pms = _to_planes(gr, b_packed)
    dev_b = [torch.from_numpy(np.ascontiguousarray(pm.ravel(order="F"))).cuda() for pm in pms]
    dev_z = dev_b if in_place else [torch.zeros_like(t) for t in dev_b]
    g = abi.Grid_t(gr.Nx, gr.Ny, gr.Nz, gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2, gr.dx, gr.dy, gr.dz)
    bp = (C.c_void_p * 3)(*[t.data_ptr() for t in dev_b])
    zp = (C.c_void_p * 3)(*[t.data_ptr() for t in dev_z])
    rc = _lib().tdgl_sep_apply_noalloc(C.byref(g), st.fc.a, bp, zp, None)
    assert rc == 0, gpu.lib().tdgl_last_error(None).decode()
    torch.cuda.synchronize()
    out = [t.cpu().numpy().reshape((gr.Ny + 1, gr.Nz + 1, gr.Nx + 1), order="F") for t in dev_z]
    return _from_planes(gr, out)


@pytest.mark.parametrize("kind", ["euler_substeps", "three_bands"])
def test_noalloc_matches_context_solve_twice(kind):
    st, s, H, HJ = cases.small(kind)
    assert st.solver == 2                     # a SepSolver case
    gs = gpu.GPUStepper(st)
    rng = np.random.default_rng(11)
    try:
        for _ in range(2):                    # two calls in a row: the scratch keeps the previous call's contents
            b = rng.standard_normal(sep_unknowns(st.grid))
            ref = gs.sep_apply(b, f32=False)
            out = _noalloc(st, b)
            assert np.max(np.abs(out - ref)) <= 1e-12 * np.max(np.abs(ref))
    finally:
        gs.close()


def test_noalloc_rejects_grids_beyond_the_scratch():
    import juliatdgl_b200 as T
    gr = T.Grid.make(512, 256, 64, dx=0.5, buf=16)
    g = abi.Grid_t(gr.Nx, gr.Ny, gr.Nz, gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2, gr.dx, gr.dy, gr.dz)
    nul = (C.c_void_p * 3)(1, 1, 1)          # never dereferenced: the size check comes first
    rc = _lib().tdgl_sep_apply_noalloc(C.byref(g), 0.1, nul, nul, None)
    assert rc == abi.E_INVAL
    assert "scratch" in gpu.lib().tdgl_last_error(None).decode()


def test_noalloc_in_place():
    """z may be b (the header's promise): the solve reads b before it writes z."""
    st, s, H, HJ = cases.small("euler_substeps")
    gs = gpu.GPUStepper(st)
    try:
        b = np.random.default_rng(12).standard_normal(sep_unknowns(st.grid))
        ref = gs.sep_apply(b, f32=False)
        out = _noalloc(st, b, in_place=True)
        assert np.max(np.abs(out - ref)) <= 1e-12 * np.max(np.abs(ref))
    finally:
        gs.close()


def test_noalloc_near_the_scratch_limit():
    """The largest grid the header names as fitting (192×64×16 cells, one padding cell), twice in a row."""
    import juliatdgl_b200 as T
    gr = T.Grid.make(192, 64, 16, dx=0.5, buf=1)
    st = T.Stepper.make(T.two_band(xi_ratio=4.0, κ=2.0), gr, T.box_masks(gr), selffield_bc="slab")
    assert st.solver == 2
    gs = gpu.GPUStepper(st)
    rng = np.random.default_rng(13)
    try:
        for _ in range(2):
            b = rng.standard_normal(sep_unknowns(gr))
            ref = gs.sep_apply(b, f32=False)
            out = _noalloc(st, b)
            assert np.max(np.abs(out - ref)) <= 1e-12 * np.max(np.abs(ref))
    finally:
        gs.close()
