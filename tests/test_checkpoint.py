"""Checkpoint files (juliatdgl_b200/checkpoint.py) on the host: the state, the PCG and open-boundary carry and the
noise index round-trip exactly, under the reference's key names (gtdgl/src/io.jl:131-171,
gtdgl/src/protocol.jl:656-658), and a file with only the reference's keys loads with the derived fields rebuilt as
the reference rebuilds them (state.jl:31-46)."""
import os

import numpy as np

import cases
from juliatdgl_b200 import checkpoint
from juliatdgl_b200.abi import Carry
from juliatdgl_b200.state import LINK_FIELDS, State


def _filled(st, s, seed=1):
    rng = np.random.default_rng(seed)
    s = s.copy()
    for _, a in s.fields():
        a[...] = rng.standard_normal(a.shape) + (1j * rng.standard_normal(a.shape) if np.iscomplexobj(a) else 0)
    c = Carry(st)
    c.pcg_x[:] = rng.standard_normal(c.pcg_x.shape)
    c.pcg_xprev[:] = rng.standard_normal(c.pcg_xprev.shape)
    c.pcg_warm, c.pcg_have2, c.open_count = 1, 1, 7
    for ax in range(3):
        c.open_old[ax][...] = rng.standard_normal(c.open_old[ax].shape)
        c.open_new[ax][...] = rng.standard_normal(c.open_new[ax].shape)
        c.open_theta[ax][...] = rng.standard_normal(c.open_theta[ax].shape)
    return s, c


def test_round_trip_is_exact(tmp_path):
    st, s, H, HJ = cases.small("open_pcg")
    s, c = _filled(st, s)
    p = str(tmp_path / "run.npz")
    checkpoint.save(p, s, c, grid=st.grid, steps=123, noise_step=456, extra={"J": 0.25})
    assert os.listdir(tmp_path) == ["run.npz"]   # written through a temporary file, renamed
    s2, c2, info = checkpoint.load(p, st)
    for (k, a), (_, b) in zip(s.fields(), s2.fields()):
        assert np.array_equal(a, b), k
    assert np.array_equal(c.pcg_x, c2.pcg_x) and np.array_equal(c.pcg_xprev, c2.pcg_xprev)
    assert (c2.pcg_warm, c2.pcg_have2, c2.open_count) == (1, 1, 7)
    for ax in range(3):
        assert np.array_equal(c.open_old[ax], c2.open_old[ax]) and np.array_equal(c.open_new[ax], c2.open_new[ax])
        assert np.array_equal(c.open_theta[ax], c2.open_theta[ax])
    assert info["steps"] == 123 and info["noise_step"] == 456 and float(info["J"]) == 0.25


def test_reference_key_names(tmp_path):
    st, s, H, HJ = cases.small("pcg")
    s, c = _filled(st, s, seed=2)
    c.open_count = -1
    p = str(tmp_path / "run.npz")
    checkpoint.save(p, s, c, grid=st.grid)
    with np.load(p) as w:
        keys = set(w.files)
    assert {"nbands", "G1", "G2", "thetax", "thetay", "thetaz", "thetax_prev", "thetay_prev", "thetaz_prev",
            "hx", "hy", "hz", "pcg_x1", "pcg_x2", "pcg_x3", "pcg_p1", "pcg_p2", "pcg_p3"} <= keys
    with np.load(p) as w:   # the warm start on its link range (implicit.jl:52)
        gr = st.grid
        assert w["pcg_x1"].shape == (gr.Nx - 2, gr.Ny - 1, gr.Nz - 1)


def test_a_file_with_the_reference_keys_only(tmp_path):
    st, s, H, HJ = cases.small("rkl_bar")
    s, _ = _filled(st, s, seed=3)
    p = str(tmp_path / "ref.npz")
    ref = {"nbands": np.array(s.N), "thetax": s.θx, "thetay": s.θy, "thetaz": s.θz, "thetax_prev": s.φx,
           "thetay_prev": s.φy, "thetaz_prev": s.φz, "hx": s.hx, "hy": s.hy, "hz": s.hz}
    ref.update({f"G{µ + 1}": g for µ, g in enumerate(s.G)})
    np.savez(p, **ref)
    s2, c2, info = checkpoint.load(p, st)
    want = State.from_fields(st.grid, s.G, (s.θx, s.θy, s.θz), (s.φx, s.φy, s.φz), (s.hx, s.hy, s.hz))
    for (k, a), (_, b) in zip(want.fields(), s2.fields()):
        assert np.array_equal(a, b), k
    assert c2.pcg_warm == 0 and c2.open_count == -1 and info["noise_step"] is None


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
STATE_KEYS = {"G1": lambda s: s.G[0], "G2": lambda s: s.G[1], "thetax": lambda s: s.θx, "thetay": lambda s: s.θy,
              "thetaz": lambda s: s.θz, "phix": lambda s: s.φx, "hx": lambda s: s.hx, "hz": lambda s: s.hz,
              "Vx": lambda s: s.Vx}


def _close(a, b, tol=1e-10):
    return a.shape == b.shape and float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b)))) <= tol


def test_a_reference_jld2_file_continues_on_the_oracle():
    """A file gtdgl wrote (tests/golden/k2_R4_heat.jld2, the heat regression case of test_regression12.jl, kept as
    the reference wrote it): its `ini` group read by checkpoint.load through the package's JLD2 reader, the
    temperature field `Temp` into the carry, 40 steps on the oracle, and the file's own `fin` group reached at 1e-10
    (test_regression12.jl:58-78), temperature included."""
    from juliatdgl_b200 import jld2
    from oracle import pyoracle
    st, _, par, _, _ = cases.golden("k2_R4_heat")
    path = os.path.join(GOLDEN, "k2_R4_heat.jld2")
    s, carry, info = checkpoint.load(path, st, group="ini", prev="phix")
    assert st.heat is not None and float(np.max(carry.heat_theta)) > 0
    o = pyoracle.OracleStepper(st)
    o.upload(s)
    o.set_carry(carry)
    assert o.steps(par["N1"], par["H"], par["HJ"]) == 0
    o.download(s)
    o.get_carry(carry)
    fin = jld2.load(path)["fin"]
    for k, get in STATE_KEYS.items():
        assert _close(get(s), np.asarray(fin[k])), k
    assert _close(carry.heat_theta, np.asarray(fin["Temp"])) and carry.heat_theta.max() > 1e-4
