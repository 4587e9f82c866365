"""Parity of the CUDA path (through the C-ABI) with the oracle, on the same seeded inputs.

Tolerances (whole-vector relative, gpu/TDGLGPU/test/compare_cpu.jl:65-109): 1e-11 for every path with an exact
field solve (the stencils keep the reference's operation order; only sin/cos/atan2 and the summation order of the
dense line transforms round differently); the PCG paths are exact to their solve tolerance only, so 1e-7 as the
reference's own CPU-versus-device record for the fast PCG.
"""
import numpy as np
import pytest

import cases
from juliatdgl_b200 import gpu
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def tol_for(st):
    return 1e-7 if st.solver == 3 else 1e-11


def run_both(st, s, n, H, HJ):
    a = pyoracle.run(st, s, n, H, HJ)
    gs = gpu.GPUStepper(st)
    b = s.copy()
    gs.upload(b)
    gs.steps(n, H, HJ)
    gs.download(b)
    gs.close()
    return a, b


@pytest.mark.parametrize("kind", cases.SMALL_KINDS)
def test_small_cases(kind):
    st, s, H, HJ = cases.small(kind)
    s = pyoracle.run(st, s, 5, H, HJ)          # off the seed: links and currents nonzero
    n = 60 if kind.startswith("open") else 20
    a, b = run_both(st, s, n, H, HJ)
    worst, per = cases.compare_states(b, a)
    assert worst <= tol_for(st), per


@pytest.mark.parametrize("name", cases.GOLDEN_CASES)
def test_golden_cases_on_gpu(name):
    st, s, par, ini, fin = cases.golden(name)
    gs = gpu.GPUStepper(st)
    b = s.copy()
    gs.upload(b)
    if st.heat is not None:   # test_regression12.jl:66: the golden's temperature field
        gs.carry.heat_theta[...] = ini["Temp"]
        gs.set_carry()
    gs.steps(par["N1"], par["H"], par["HJ"])
    gs.download(b)
    for k, get in (("G1", lambda x: x.G[0]), ("G2", lambda x: x.G[1]), ("thetax", lambda x: x.θx),
                   ("thetay", lambda x: x.θy), ("thetaz", lambda x: x.θz), ("hx", lambda x: x.hx),
                   ("hy", lambda x: x.hy), ("hz", lambda x: x.hz), ("Vx", lambda x: x.Vx)):
        d = np.max(np.abs(get(b) - fin[k]) / np.maximum(1.0, np.abs(fin[k])))
        assert d <= 1e-10, (k, d)
    if st.heat is not None:
        th = gs.get_carry().heat_theta
        assert np.max(np.abs(th - fin["Temp"]) / np.maximum(1.0, np.abs(fin["Temp"]))) <= 1e-10


def test_config1_per_step():
    """The two-band parity case, step by step for 200 steps against the oracle at 1e-11."""
    st, s, H, HJ = cases.config1()
    o = pyoracle.OracleStepper(st)
    o.upload(s)
    gs = gpu.GPUStepper(st)
    gs.upload(s)
    a = s.copy()
    b = s.copy()
    worst = 0.0
    for q in range(200):
        o.steps(1, H, HJ)
        gs.steps(1, H, HJ)
        if q % 20 == 19:
            o.download(a)
            gs.download(b)
            w, per = cases.compare_states(b, a)
            worst = max(worst, w)
            assert w <= 1e-11, (q, per)


@pytest.mark.parametrize("kind,f32,tol", [("pcg", False, 1e-13), ("pcg_f32", True, 2e-6)])
def test_separable_inverse(kind, f32, tol):
    """(I + aK)^{-1} on random packed ranges: the GPU's y/z transforms with the tridiagonal x solve against the
    oracle's dense three-axis transforms (the reference's algorithm), FP64 and FP32."""
    st, s, H, HJ = cases.small(kind)
    o = pyoracle.OracleStepper(st)
    gs = gpu.GPUStepper(st)
    from juliatdgl_b200.scheme import sep_unknowns
    b = np.random.default_rng(7).standard_normal(sep_unknowns(st.grid))
    ref = o.sep_apply(b, f32=False)
    out = gs.sep_apply(b, f32=f32)
    gs.close()
    assert np.max(np.abs(out - ref)) / np.max(np.abs(ref)) <= tol


@pytest.mark.parametrize("kind", ["pcg", "pcg_fast", "pcg_f32", "open_pcg"])
def test_pcg_iteration_counts_follow_the_oracle(kind):
    """The same solve takes the same iterations: the warm start, the extrapolated guess 2xₙ − xₙ₋₁ and the stopping
    test are the reference's (implicit.jl:376-446); rounding may move a count at the tolerance by one now and then."""
    st, s, H, HJ = cases.small(kind)
    o = pyoracle.OracleStepper(st)
    o.upload(s)
    gs = gpu.GPUStepper(st)
    try:
        gs.upload(s)
        n = 30
        o.steps(n, H, HJ)
        gs.steps(n, H, HJ)
        a, b = o.stats().pcg_total_iters, gs.stats().pcg_total_iters
    finally:
        gs.close()
    assert a > n and abs(a - b) <= max(2, a // 50), (a, b)


@pytest.mark.parametrize("ny,nz,f32,tol", [(220, 60, False, 1e-13), (480, 60, True, 2e-6)])
def test_separable_inverse_on_planes_larger_than_a_block(ny, nz, f32, tol):
    """y-z planes whose input does not fit one block's shared memory (FP64 from about 200 × 60 nodes, FP32 from about
    450 × 60) take the chunked plane transform: the same inverse as the oracle's dense transforms."""
    import juliatdgl_b200 as T
    from juliatdgl_b200.scheme import sep_unknowns
    gr = T.Grid.make(8, ny, nz, dx=0.5, buf=1 if not f32 else 2)
    mk = T.box_masks(gr)
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    st = T.Stepper.make(md, gr, mk, σvac=0.01 if f32 else None, pcg_f32=f32, selffield_bc="slab")
    o = pyoracle.OracleStepper(st)
    gs = gpu.GPUStepper(st)
    try:
        b = np.random.default_rng(3).standard_normal(sep_unknowns(gr))
        ref = o.sep_apply(b, f32=False)
        out = gs.sep_apply(b, f32=f32)
    finally:
        gs.close()
    assert np.max(np.abs(out - ref)) / np.max(np.abs(ref)) <= tol
