"""The oracle against the reference's own golden data (CPU).

Pins the C++ restatement of the step (oracle/oracle.cpp) to the release-1.2 regression states of
gtdgl/test/test_regression12.jl (40 steps from a warm state, every field to 1e-10 of max(1, |x|)), and the host
Stepper mirror to the step, substep count and self-field the reference derived for those cases.
"""
import numpy as np
import pytest

import cases
import juliatdgl_b200 as T
from juliatdgl_b200 import abi
from oracle import pyoracle

FIELDS = {"G1": lambda s: s.G[0], "G2": lambda s: s.G[1], "thetax": lambda s: s.θx, "thetay": lambda s: s.θy,
          "thetaz": lambda s: s.θz, "phix": lambda s: s.φx, "phiy": lambda s: s.φy, "phiz": lambda s: s.φz,
          "Vx": lambda s: s.Vx, "Vy": lambda s: s.Vy, "Vz": lambda s: s.Vz, "hx": lambda s: s.hx, "hy": lambda s: s.hy,
          "hz": lambda s: s.hz}


def same(a, b, tol=1e-10):
    """gtdgl/test/test_regression12.jl:46-52: every entry to tol of max(1, |entry|)."""
    return a.shape == b.shape and float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b)))) <= tol


@pytest.mark.parametrize("name", cases.GOLDEN_CASES)
def test_stepper_matches_reference_parameters(name):
    st, s, par, ini, fin = cases.golden(name)
    assert st.dt == par["dt"]                       # test_regression12.jl:60, to the bit
    assert st.nsub == (1, par["n_pi"])
    assert T.selffield(st, par["J"]) == par["HJ"]
    assert same(s.Vx, ini["Vx"]) and same(s.Ux, ini["Ux"]) and same(s.Uz, ini["Uz"])


@pytest.mark.parametrize("name", cases.GOLDEN_CASES)
def test_oracle_reproduces_golden(name):
    """test_regression12.jl:58-78; the heat case starts its temperature field from the golden's (:66) and ends on
    the golden's (:78)."""
    st, s, par, ini, fin = cases.golden(name)
    o = pyoracle.OracleStepper(st)
    s2 = s.copy()
    o.upload(s2)
    carry = abi.Carry(st)
    if st.heat is not None:
        carry.heat_theta[...] = ini["Temp"]
        o.set_carry(carry)
    assert o.steps(par["N1"], par["H"], par["HJ"]) == 0
    o.download(s2)
    for k, get in FIELDS.items():
        assert same(get(s2), fin[k]), k
    if st.heat is not None:
        o.get_carry(carry)
        assert same(carry.heat_theta, fin["Temp"]) and carry.heat_theta.max() > 1e-4
