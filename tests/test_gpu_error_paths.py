"""Error paths of the step, through the C ABI.

* A non-finite particle position is reported as MPM_ERR_NONFINITE (the
  reference has no such check; its nearest counterpart is the
  particle-outside-the-mesh error of mpm_scheme.tcc:250-256).
* A bounded device wait that runs out is reported as MPM_ERR_TIMEOUT and
  stores nothing.  The staged G2P's test hook (MPM_B200_TEST_WAIT_TIMEOUT)
  makes its first copy wait run out after the copies have landed; the block
  drains its other copies and returns.  No GPU fault is involved, and the
  context stays usable: a new solver in the same process steps normally.
"""
import os

import numpy as np
import pytest

from mpm_b200 import MPMError
from mpm_b200 import problems as P

pytestmark = pytest.mark.gpu

NONFINITE, TIMEOUT = -4, -5


def _column(scheme="usl"):
    return P.column_3d(shape=(12, 8, 10), block=(6, 4, 6), dt=1e-5, c=2000., psi=5., scheme=scheme)


@pytest.mark.parametrize("precision,scheme", [("fp64", "usl"), ("fp64", "usf"), ("mixed", "usl")])
def test_nan_velocity_is_reported_as_nonfinite(precision, scheme):
    s = P.build_solver(_column(scheme), precision=precision)
    st = s.read()
    st["v"][7] = np.nan
    s.load(st)
    with pytest.raises(MPMError) as e:
        s.step(1)
    assert e.value.code == NONFINITE
    assert "non-finite" in str(e.value)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_wait_timeout_is_reported_and_stores_nothing(precision):
    prob = _column("usl")
    os.environ["MPM_B200_TEST_WAIT_TIMEOUT"] = "1"
    try:
        s = P.build_solver(prob, precision=precision)
    finally:
        del os.environ["MPM_B200_TEST_WAIT_TIMEOUT"]
    before = s.read()
    with pytest.raises(MPMError) as e:
        s.step(1)
    assert e.value.code == TIMEOUT
    after = s.read()
    for f in ("x", "u", "v", "stress", "strain", "F", "volume", "cell", "svars"):
        assert np.array_equal(before[f], after[f]), f
    s.close()
    # the context is intact: a solver without the hook steps as usual
    ok = P.build_solver(prob, precision=precision)
    ok.step(3)
    assert np.isfinite(ok.read()["x"]).all()
