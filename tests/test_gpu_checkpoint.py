"""A run checkpointed to a file and resumed in a new context continues to the bit: the PCG warm start (and pcg_fast's
extrapolation), the open boundary's ramp and the noise stream all resume (as gpu/TDGLGPU/test/test_resume.jl asks of
the reference's accelerator, here exactly), and a file the reference wrote resumes on the device."""
import numpy as np
import pytest

import cases
from juliatdgl_b200 import checkpoint, gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,kw", [("pcg_fast", {}), ("open", {}), ("open_pcg", {}),
                                     ("three_bands", cases.NOISY["three_bands"])])
def test_checkpoint_and_resume_continues_to_the_bit(kind, kw, tmp_path):
    st, s, H, HJ = cases.small(kind, **kw)
    one = gpu.GPUStepper(st)
    a = s.copy()
    one.upload(a)
    one.steps(20, H, HJ)
    one.download(a)
    one.close()
    first = gpu.GPUStepper(st)
    first.upload(s.copy())
    first.steps(10, H, HJ)
    p = str(tmp_path / "run.npz")
    checkpoint.save_run(p, first, st, s)
    first.close()
    second, st2, info = checkpoint.resume(p, st)
    try:
        assert info["steps"] == 10
        second.steps(10, H, HJ)
        b = second.download(s.copy())
    finally:
        second.close()
    assert cases.compare_states(b, a)[0] == 0.0


def test_a_reference_jld2_file_resumes_on_the_device():
    """The reference-written tests/golden/k2_R4_heat.jld2: its `ini` group resumed in a device context by
    checkpoint.resume (state, temperature field), 40 steps, the file's `fin` group at 1e-10 (test_regression12.jl)."""
    import os
    from juliatdgl_b200 import jld2
    st, _, par, _, _ = cases.golden("k2_R4_heat")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "k2_R4_heat.jld2")
    gs, st, info = checkpoint.resume(path, st, group="ini", prev="phix")
    try:
        s, _, _ = checkpoint.load(path, st, group="ini", prev="phix")
        gs.steps(par["N1"], par["H"], par["HJ"])
        gs.download(s)
        th = gs.get_carry().heat_theta
    finally:
        gs.close()
    fin = jld2.load(path)["fin"]
    for k, get in (("G1", lambda x: x.G[0]), ("G2", lambda x: x.G[1]), ("thetax", lambda x: x.θx),
                   ("hz", lambda x: x.hz), ("Vx", lambda x: x.Vx)):
        ref = np.asarray(fin[k])
        assert np.max(np.abs(get(s) - ref) / np.maximum(1.0, np.abs(ref))) <= 1e-10, k
    ref = np.asarray(fin["Temp"])
    assert np.max(np.abs(th - ref) / np.maximum(1.0, np.abs(ref))) <= 1e-10
