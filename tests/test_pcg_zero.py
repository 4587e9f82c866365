"""A zero right-hand side in the PCG field solve, and the solver's carry through a checkpoint.

Restates the reference's shared CPU/device regression gtdgl/test/pcg_zero_fixture.jl:4-82 (driven on the CPU by
gtdgl/test/test_pcg_zero_rhs.jl and on the device by gpu/TDGLGPU/test/test_pcg_zero_rhs.jl): in four solver modes
(plain, fast FP64, fast FP32 preconditioner, fast without the extrapolated guess), a zero source must erase a warm
increment (x = 0, φ = θ on the ranges and θ + (φ − θ)/D on the decoupled links, iterations 0), keep the actual
previous solution for the extrapolation, and survive a checkpoint: a solver given back (x, and xprev when the
extrapolation has two solutions) continues bit for bit like the one that never stopped.  Here the checkpoint is the
carry of the solver (tdgl_get_carry / tdgl_set_carry), and "a solve" uploads the state and the carry, runs the
field solve alone and reads both back, as the reference's device driver does (_pcg_up!, _implicit_curl!,
host_state!, _pcg_down!).
"""
import math

import numpy as np
import pytest

import juliatdgl_b200 as T
from juliatdgl_b200 import abi
from juliatdgl_b200.scheme import sep_ranges

MODES = ((False, False, True), (True, False, True), (True, True, True), (True, True, False))


def setup():
    md = T.two_band(xi_ratio=4.0, κ=2.0)
    gr = T.Grid.make(4, 4, 4, dx=0.5, buf=2)
    mk = T.build_masks(T.GeomSpec(GEOM_MODE="SIM"), gr)
    return md, gr, mk


def new_stepper(md, gr, mk, fast, f32, extrap):
    return T.Stepper.make(md, gr, mk, σvac=0.01, pcg_fast=fast, pcg_f32=f32, pcg_extrap=extrap)


class Solve:
    """One solver (a Stepper's PCG state) on an implementation: the oracle or the device context."""

    def __init__(self, make_ctx, st):
        self.ctx = make_ctx(st)
        self.carry = abi.Carry(st)
        self.iters = None

    def __call__(self, s):
        self.ctx.upload(s)
        self.ctx.set_carry(self.carry)
        rc = self.ctx.field_solve()
        assert rc == 0
        self.ctx.download(s)
        self.ctx.get_carry(self.carry)
        self.iters = self.ctx.stats().pcg_last_iters

    def snap(self):
        c = self.carry
        return (c.pcg_warm, c.pcg_x.copy(), c.pcg_have2, c.pcg_xprev.copy())


def theta(s):
    return (s.θx, s.θy, s.θz)


def phi(s):
    return (s.φx, s.φy, s.φz)


def range_view(a, r):
    return a[r[0][0] - 1:r[0][1], r[1][0] - 1:r[1][1], r[2][0] - 1:r[2][1]]


def source(s, q, ranges):
    """pcg_zero_fixture.jl:27-37: a nonzero background θ, φ = θ + 0.003 off the ranges, and on the ranges
    φ = θ (q = 0) or θ + 0.001 sin(0.17 n + c + q)."""
    for c in range(1, 4):
        t, p = theta(s)[c - 1], phi(s)[c - 1]
        idx = np.arange(1, t.size + 1, dtype=np.float64)
        t[...] = (0.01 * np.sin(0.13 * idx + c)).reshape(t.shape, order="F")
        p[...] = t + 0.003
        b = range_view(p, ranges[c - 1])
        th = range_view(t, ranges[c - 1])
        n = np.arange(1, b.size + 1, dtype=np.float64).reshape(b.shape, order="F")
        b[...] = th + (0.0 if q == 0 else 0.001 * np.sin(0.17 * n + c + q))


def check_zero(solve, s, st, ranges, fast, extrap, cold=False):
    """pcg_zero_fixture.jl:38-55."""
    previous = solve.carry.pcg_x.copy()
    expected = [t + (p - t) / d for p, t, d in zip(phi(s), theta(s), st.D)]
    solve(s)
    assert not np.any(solve.carry.pcg_x)
    assert solve.carry.pcg_warm and solve.iters == 0
    for c in range(3):
        assert np.array_equal(range_view(phi(s)[c], ranges[c]), range_view(theta(s)[c], ranges[c]))
        range_view(expected[c], ranges[c])[...] = range_view(theta(s)[c], ranges[c])
        assert np.array_equal(phi(s)[c], expected[c])      # the decoupled links too
    if fast:
        assert bool(solve.carry.pcg_have2) == ((not cold) and extrap)
        if not cold and extrap:
            assert np.array_equal(solve.carry.pcg_xprev, previous)


def run_fixture(make_ctx):
    md, gr, mk = setup()
    ranges = sep_ranges(gr)
    for fast, f32, extrap in MODES:
        st = new_stepper(md, gr, mk, fast, f32, extrap)
        assert st.solver == T.scheme.SOLVER_PCG
        solve = Solve(make_ctx, st)
        s = T.initial_state(md, gr, mk, 0.0)
        source(s, 0, ranges)
        check_zero(solve, s, st, ranges, fast, extrap, cold=True)
        for q in range(1, 4):
            source(s, q, ranges)
            solve(s)
            assert np.any(solve.carry.pcg_x)
        source(s, 0, ranges)
        check_zero(solve, s, st, ranges, fast, extrap)
        # the checkpoint: x, and xprev when the extrapolation holds two solutions (pcg_zero_fixture.jl:58-67)
        resumed = s.copy()
        restored = Solve(make_ctx, new_stepper(md, gr, mk, fast, f32, extrap))
        restored.carry.pcg_warm = 1
        restored.carry.pcg_x[...] = solve.carry.pcg_x
        if fast and solve.carry.pcg_have2:
            restored.carry.pcg_have2 = 1
            restored.carry.pcg_xprev[...] = solve.carry.pcg_xprev
        for q in (0, 4, 5):
            source(s, q, ranges)
            source(resumed, q, ranges)
            solve(s)
            restored(resumed)
            for a, b in zip(phi(s), phi(resumed)):
                assert np.array_equal(a, b)
            sa, sb = solve.snap(), restored.snap()
            assert sa[0] == sb[0] and np.array_equal(sa[1], sb[1])
            if fast:
                assert sa[2] == sb[2]
                if sa[2]:
                    assert np.array_equal(sa[3], sb[3])
        source(s, 0, ranges)
        check_zero(solve, s, st, ranges, fast, extrap)
        source(s, 0, ranges)
        check_zero(solve, s, st, ranges, fast, extrap)   # the previous solution is now also zero
        solve.carry.pcg_warm = 0                          # _pcg_reset! (implicit.jl:195)
        solve.carry.pcg_have2 = 0
        source(s, 0, ranges)
        check_zero(solve, s, st, ranges, fast, extrap, cold=True)


def test_oracle_pcg_zero_source_and_checkpoint():
    from oracle import pyoracle
    run_fixture(pyoracle.OracleStepper)


@pytest.mark.gpu
def test_device_pcg_zero_source_and_checkpoint():
    from juliatdgl_b200 import gpu
    run_fixture(gpu.GPUStepper)


@pytest.mark.gpu
def test_device_field_solve_matches_the_oracle():
    """The device's field solve on the fixture's sources against the oracle's, per mode: φ within 1e-7 of the whole
    vector (the PCG bar of gpu/TDGLGPU/test/compare_cpu.jl:69) and the same iteration counts within one."""
    from juliatdgl_b200 import gpu
    from oracle import pyoracle
    md, gr, mk = setup()
    ranges = sep_ranges(gr)
    for fast, f32, extrap in MODES:
        st = new_stepper(md, gr, mk, fast, f32, extrap)
        a, b = Solve(gpu.GPUStepper, st), Solve(pyoracle.OracleStepper, st)
        sa, sb = T.initial_state(md, gr, mk, 0.0), T.initial_state(md, gr, mk, 0.0)
        for q in (1, 2, 3, 0, 4):
            source(sa, q, ranges)
            source(sb, q, ranges)
            a(sa)
            b(sb)
            m = max(np.max(np.abs(x)) for x in phi(sb))
            d = max(np.max(np.abs(x - y)) for x, y in zip(phi(sa), phi(sb)))
            assert d <= 1e-7 * m, (fast, f32, extrap, q, d / m)
            assert abs(a.iters - b.iters) <= 1, (a.iters, b.iters)
