"""The oracle's OpenMP loops are element-wise (no reductions across threads), so its result must not depend on the
thread count: the same case run with 1 and with 3 threads gives bit-identical states."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))

SCRIPT = r"""
import sys
sys.path[:0] = [{root!r}, {here!r}]
import numpy as np
import cases
from oracle import pyoracle
st, s, H, HJ = cases.small({kind!r})
out = pyoracle.run(st, s, 6, H, HJ)
np.savez({path!r}, **{{k: np.asarray(v) for k, v in out.fields()}})
"""


@pytest.mark.parametrize("kind", ["open_pcg", "rkc_kwt_rotframe"])
def test_oracle_is_independent_of_the_thread_count(kind, tmp_path):
    res = []
    for threads in (1, 3):
        path = str(tmp_path / f"{kind}_{threads}.npz")
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        code = SCRIPT.format(root=ROOT, here=HERE, kind=kind, path=path)
        subprocess.run([sys.executable, "-c", code], env=env, check=True, timeout=600)
        res.append(np.load(path))
    a, b = res
    assert set(a.files) == set(b.files) and a.files
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k
