"""A run checkpointed to a file and resumed in a new context continues to the bit: the PCG warm start (and pcg_fast's
extrapolation), the open boundary's ramp and the noise stream all resume (as gpu/TDGLGPU/test/test_resume.jl asks of
the reference's accelerator, here exactly)."""
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
