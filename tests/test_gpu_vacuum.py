"""Sculpted samples on the device (the vacuum variant of the band stage, the vacuum ghosts, the noise skipping the
vacuum) against the oracle through the C-ABI, at the PCG's 1e-7 (the padding makes the field solve a PCG), and the
reference's free-surface test (gtdgl/test/test_physics.jl:583-600) on the device.
"""
import pytest

import cases
from juliatdgl_b200 import gpu
from oracle import pyoracle
from test_vacuum_oracle import free_surface

pytestmark = pytest.mark.gpu


def gpu_run(st, s, n, H, HJ):
    gs = gpu.GPUStepper(st)
    try:
        b = s.copy()
        gs.upload(b)
        gs.steps(n, H, HJ)
        return gs.download(b)
    finally:
        gs.close()


@pytest.mark.parametrize("kind,kw", [(k, {}) for k in cases.VACUUM_KINDS] +
                         [("vac_kwt", dict(noise=1e-3, noise_seed=31, noise_field=True))],
                         ids=list(cases.VACUUM_KINDS) + ["vac_kwt_noise"])
def test_vacuum_cases(kind, kw):
    st, s, H, HJ = cases.vacuum(kind, **kw)
    s = pyoracle.run(st, s, 5, H, HJ)
    n = 40 if kind == "vac_open" else 20
    a = pyoracle.run(st, s, n, H, HJ)
    b = gpu_run(st, s, n, H, HJ)
    worst, per = cases.compare_states(b, a)
    assert worst <= 1e-7, per
    assert max(abs(b.G[µ][st.masks.vac]).max() for µ in range(st.model.N)) == 0


def test_free_surface_on_the_device():
    dev, vac = free_surface(lambda st, s, n: gpu_run(st, s, n, 0.0, 0.0))
    assert dev < 1e-13 and vac == 0
