"""The reference's golden ladder (gtdgl/test/golden/ladder_k25.jld2, made by golden/make_ladder.jl with release 1.2;
checked by gtdgl/test/test_protocol.jl:4-29): a two-polarity current ladder of the two-band notched box at κ = 25
(24×12×4 cells, WEDGE with inj_margin 4, slab self-field, Euler substeps), J = 0.3 … 1.5, H = 0.03, with short
windows.  Point by point: the currents, verdicts (F/V), cycles, band-1 and band-2 voltages, the static voltage, the
half-window slopes, slip counts, magnetisation, vortex counts, residuals, the final Ψ of both bands, and the
brackets of the critical current.

* On the oracle, through the ladder driver of juliatdgl_b200/ladder.py with the observables computed on the host
  (oracle/observables.py) from the oracle's state: every value within 1e-10 of max(1, |golden|), the reference's
  own bar (test_regression12.jl:51-57), verdicts and cycles exactly.
* On the device, the same driver with the observables measured on the resident state (tdgl_measure): the
  reference's CPU-versus-device bar of gpu/TDGLGPU/test/compare_ladder.jl:45-58 — the same verdicts and cycles,
  voltages within 1e-6 relative or 1e-10 absolute, the final state within 1e-9 — and the brackets exactly.
"""
import math
import os

import numpy as np
import pytest

import juliatdgl_b200 as T
from juliatdgl_b200 import ladder as L
from juliatdgl_b200.grid import GeomSpec, build_masks
from oracle import observables as ob
from oracle import pyoracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ladder_k25.npz")


def golden_case():
    d = np.load(GOLDEN)
    md = T.Model.make((T.Band.make(), T.Band.make(m=float(d["mr"]), Γ=1.0, a=0.59)), [[0.0, 1e-3], [1e-3, 0.0]],
                      κ=25.0)
    gr = T.Grid.make(24, 12, 4, dx=0.5)
    mk = build_masks(GeomSpec(GEOM_MODE="WEDGE", inj_margin=4), gr)
    st = T.Stepper.make(md, gr, mk, selffield_bc="slab", rkl=False)
    pr = L.Protocol(t_min_GL=20.0, t_min_GL_res=60.0, mMax=4000, delta_v=6, v_margin=1.0, f_strict=False)
    return d, st, pr


class OracleLadder:
    """The ladder's backend over the oracle: the state stepped on the CPU, the cycle observables computed on the host
    from it with the restatements of the reference's measurement functions."""

    def __init__(self, st):
        self.st = st
        self.o = pyoracle.OracleStepper(st)
        self.s = None

    def reset(self, s):
        self.s = s.copy()
        self.o.upload(self.s)

    def meter_set(self, vm):
        gr, N = self.st.grid, self.st.N
        self.vm = vm
        self.cooper0 = [ob.block_abs(self.s.G[mu], gr) for mu in range(N)]
        self.hz0 = self.s.hz.copy()

    def cycle(self, n, H, HJ):
        assert self.o.steps(n, H, HJ) == 0
        self.o.download(self.s)

    def measure(self):
        st, gr, vm, s = self.st, self.st.grid, self.vm, self.s
        D, res, amax = [], [], 0.0
        for mu in range(st.N):
            D.append(ob.path_phase(s.G[mu], s.Vx, gr, vm.vi, vm.vo))
            r, a = ob.cooper_residual(s.F[mu], self.cooper0[mu], gr)
            res.append(r)
            self.cooper0[mu] = a
            amax = max(amax, ob.nanmax(ob.block_abs(s.F[mu], gr)))
        diffh = ob.nanmax(np.abs(s.hz - self.hz0))
        self.hz0 = s.hz.copy()
        it, isam = ob.midplane_current(s.hy, s.hz, gr, st.model.κ ** 2)
        return {"D": D, "vsum_in": ob.plane_sum(s.φx, gr, vm.vi, vm.Min),
                "vsum_out": ob.plane_sum(s.φx, gr, vm.vo, vm.Mou),
                "ta_sum": ob.theta_A_sum(s.φx, gr, vm.vi, vm.vo, vm.line_ok), "res": res, "amax": amax,
                "diffh": diffh, "Itot": it, "Isam": isam}

    def download(self, s):
        for name, a in self.s.fields():
            dst = getattr(s, name) if not name[0] in "GF" or not name[1:].isdigit() else \
                (s.G if name[0] == "G" else s.F)[int(name[1:]) - 1]
            dst[...] = a

    def vortices(self, band, kc):
        s = self.s
        return ob.count_vortices(s.F[band], s.Vx, s.Vy, s.hz, self.st.masks.f, self.st.grid, kc)[0]


def check_setup(d, st, pr):
    """test_protocol.jl:10-12: the same step, substeps and fixed-point tolerance as the golden's release."""
    assert st.dt == float(d["dt"]) and st.nsub == (1, int(d["n_pi"]))
    assert L.eps_cycle(pr, st) == float(d["eps_c"])


def close(a, b, tol):
    a, b = np.asarray(a, dtype=np.complex128), np.asarray(b, dtype=np.complex128)
    return a.shape == b.shape and bool(np.all(np.abs(a - b) <= tol * np.maximum(1.0, np.abs(b))))


def compare(lad, g, pol, tol_v, tol_state, rel_v):
    assert np.array_equal(lad.J, g[f"{pol}_J"])
    assert lad.conv == str(g[f"{pol}_conv"]), (lad.conv, str(g[f"{pol}_conv"]))
    assert np.array_equal(lad.m, g[f"{pol}_m"]), (lad.m, g[f"{pol}_m"])
    vals = {"V": lad.V, "V2": lad.Vb[:, 1], "Vst": lad.Vstatic, "Vh": lad.Vh[:, 0], "Vh2": lad.Vh[:, 1],
            "nslip": lad.nslip, "M": lad.M, "r1": lad.res[:, 0], "r2": lad.res[:, 1]}
    for k, v in vals.items():
        ref = g[f"{pol}_{k}"]
        if rel_v:   # compare_ladder.jl: relative 1e-6, or 1e-10 absolute
            ok = np.all((np.abs(v - ref) <= tol_v * np.abs(ref)) | (np.abs(v - ref) <= 1e-10))
        else:
            ok = close(v, ref, tol_v)
        assert ok, (pol, k, v, ref)
    assert np.array_equal(lad.Nv[:, 0], g[f"{pol}_Nv1"]) and np.array_equal(lad.Nv[:, 1], g[f"{pol}_Nv2"])
    for mu, key in ((0, "G1"), (1, "G2")):
        ref = g[f"{pol}_{key}"]
        d = np.max(np.abs(lad.state.G[mu] - ref)) / max(np.max(np.abs(ref)), 1.0)
        assert d <= tol_state, (pol, key, d)


def check_brackets(b, g):
    assert (b["pos"][0], b["pos"][1], b["neg"][0], b["neg"][1]) == \
        (float(g["lo_pos"]), float(g["hi_pos"]), float(g["lo_neg"]), float(g["hi_neg"]))


def test_oracle_reproduces_the_golden_ladder():
    g, st, pr = golden_case()
    check_setup(g, st, pr)
    pos, neg, b = L.run_ladders(OracleLadder, st, [0.30, 0.60, 0.90, 1.20, 1.50], H=0.03, pr=pr)
    compare(pos, g, "pos", 1e-10, 1e-10, rel_v=False)
    compare(neg, g, "neg", 1e-10, 1e-10, rel_v=False)
    check_brackets(b, g)


@pytest.mark.gpu
def test_device_reproduces_the_golden_ladder():
    g, st, pr = golden_case()
    check_setup(g, st, pr)
    runs = []

    def make(st):
        r = L.DeviceLadder(st)
        runs.append(r)
        return r

    try:
        pos, neg, b = L.run_ladders(make, st, [0.30, 0.60, 0.90, 1.20, 1.50], H=0.03, pr=pr)
    finally:
        for r in runs:
            r.close()
    compare(pos, g, "pos", 1e-6, 1e-9, rel_v=True)
    compare(neg, g, "neg", 1e-6, 1e-9, rel_v=True)
    check_brackets(b, g)
