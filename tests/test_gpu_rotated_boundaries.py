"""General (rotated) boundaries on the CUDA path against the oracle: the
velocity, acceleration and friction constraints of nodes with Euler angles
act on the components of the nodes' rotated frames (node.tcc:370-483,
510-657).  FP64 bar of test_gpu_parity."""
import numpy as np
import pytest

from mpm_b200 import problems as P
from tests.parity import assert_parity, field_errors
from tests.test_gpu_parity import _run_both, small_column_2d, small_column_3d
from tests.test_rotated_boundaries_oracle import floor_nodes

pytestmark = pytest.mark.gpu


def tilted_floor_2d(scheme):
    prob = small_column_2d(scheme=scheme)
    fn = floor_nodes(prob)
    prob.nodal_euler_angles = (fn, np.tile([np.pi / 6, 0.05], (len(fn), 1)))
    return prob


def tilted_friction_floor_3d(scheme):
    prob = small_column_3d(scheme=scheme, dt=1e-5, c=2000., psi=5.)
    fn = floor_nodes(prob)
    prob.nodal_euler_angles = (fn, np.tile([0.3, 0.1, 0.2], (len(fn), 1)))
    return prob


@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_2d_tilted_slip_floor(scheme):
    for s, g, o in _run_both(tilted_floor_2d(scheme), [1, 10, 100]):
        assert_parity(g, o, label=f"2D rotated floor {scheme} step {s}")


@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_3d_tilted_friction_floor(scheme):
    for s, g, o in _run_both(tilted_friction_floor_3d(scheme), [1, 10, 50]):
        assert_parity(g, o, label=f"3D rotated friction floor {scheme} step {s}")


def test_mixed_precision_with_rotated_boundaries():
    out = {}
    for prec in ("fp64", "mixed"):
        sol = P.build_solver(tilted_friction_floor_3d("usl"), precision=prec)
        sol.step(50)
        out[prec] = sol.read()
    assert np.array_equal(out["mixed"]["cell"], out["fp64"]["cell"])
    errs = field_errors(out["mixed"], out["fp64"], ("u", "v", "stress", "strain"))
    assert all(v <= 1e-5 for v in errs.values()), errs


def test_rotation_changes_the_run():
    a = P.build_solver(small_column_2d(scheme="usl"))
    b = P.build_solver(tilted_floor_2d("usl"))
    a.step(50)
    b.step(50)
    assert np.max(np.abs(a.read()["x"] - b.read()["x"])) > 1e-9
