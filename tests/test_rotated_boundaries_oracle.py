"""General (rotated) boundaries in the oracle (node.tcc:370-483, 510-657 with
generic_boundary_constraints_): zero Euler angles change nothing, and a frame
turned by 90 degrees makes a constraint on local direction 0 act on the global
direction 1."""
import numpy as np
import pytest

from mpm_b200 import problems as P
from oracle.oracle import build_oracle


def floor_nodes(prob):
    axis = prob.dim - 1
    return np.nonzero(np.abs(prob.coords[:, axis] - prob.coords[:, axis].min()) < 1e-12)[0]


@pytest.mark.parametrize("dim", [2, 3])
def test_zero_angles_change_nothing(dim):
    def make():
        if dim == 2:
            return P.column_2d(shape=(16, 12), block=(6, 8), scheme="usl")
        return P.column_3d(shape=(8, 6, 8), block=(4, 4, 4), scheme="usl", dt=1e-5, c=2000., psi=5.)
    a, b = make(), make()
    nid = floor_nodes(b)
    b.nodal_euler_angles = (nid, np.zeros((len(nid), dim)))
    oa, ob = build_oracle(a), build_oracle(b)
    oa.step(50)
    ob.step(50)
    sa, sb = oa.get(), ob.get()
    for k in ("x", "v", "stress"):
        assert np.array_equal(sa[k], sb[k]), k


def test_quarter_turn_swaps_the_constrained_direction():
    """Floor nodes in a frame turned by 90 degrees: local direction 0 is global
    y and local 1 is global x, so swapping the directions of their constraints
    reproduces the Cartesian run (to the rounding of cos(pi / 2))."""
    a = P.column_2d(shape=(16, 12), block=(6, 8), scheme="usl")
    b = P.column_2d(shape=(16, 12), block=(6, 8), scheme="usl")
    nid, dirs, vals = b.velocity_constraints
    fn = floor_nodes(b)
    on_floor = np.isin(nid, fn)
    b.velocity_constraints = (nid, np.where(on_floor, 1 - dirs, dirs), vals)
    b.nodal_euler_angles = (fn, np.tile([np.pi / 2, 0.0], (len(fn), 1)))
    oa, ob = build_oracle(a), build_oracle(b)
    oa.step(100)
    ob.step(100)
    sa, sb = oa.get(), ob.get()
    assert np.array_equal(sa["cell"], sb["cell"])
    for k in ("x", "v", "stress"):
        scale = np.max(np.abs(sa[k]))
        assert np.max(np.abs(sa[k] - sb[k])) <= 1e-10 * scale, k
