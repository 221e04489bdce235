"""The oracle's ASFLIP / APIC / TPIC velocity updates (particle.tcc:630-721,
994-1139, 1663-1730) on properties the reference's mapping preserves: a
rigid translation stays a rigid translation with a zero mapping matrix, and
the first TPIC step (zero mapping matrix) equals the PIC step."""
import numpy as np
import pytest

from mpm_b200 import problems as P
from oracle.oracle import build_oracle


def _free_block(velocity_update):
    prob = P.column_2d(shape=(16, 12), block=(4, 4), nsteps=10, material="LinearElastic",
                       velocity_update=velocity_update)
    prob.velocity_constraints = None
    prob.analysis["gravity"] = (0.0, 0.0)
    pts, mid = prob.particles[0]
    prob.particles = [(pts + np.array([0.05, 0.04]), mid)]
    return prob


@pytest.mark.parametrize("vu", ["apic", "tpic", "asflip"])
def test_rigid_translation_is_kept(vu):
    prob = _free_block(vu)
    o = build_oracle(prob)
    st = o.get()
    st["v"] = np.tile([0.3, -0.2], (len(st["x"]), 1))
    o.set(st)
    x0 = o.get()["x"].copy()
    o.step(10)
    st = o.get()
    assert np.allclose(st["v"], [0.3, -0.2], rtol=0, atol=1e-12)
    assert np.allclose(st["x"] - x0, np.array([0.3, -0.2]) * 10 * prob.analysis["dt"], rtol=0, atol=1e-12)
    assert np.max(np.abs(st["mapping"])) < 1e-12
    assert np.max(np.abs(st["stress"])) < 1e-6


def test_first_tpic_step_is_the_pic_step():
    a = build_oracle(P.column_2d(shape=(16, 12), block=(6, 8), velocity_update="tpic"))
    b = build_oracle(P.column_2d(shape=(16, 12), block=(6, 8), velocity_update="pic"))
    a.step(1)
    b.step(1)
    sa, sb = a.get(), b.get()
    for k in ("x", "v", "stress"):
        assert np.array_equal(sa[k], sb[k]), k
    assert np.max(np.abs(sa["mapping"])) > 0.0
