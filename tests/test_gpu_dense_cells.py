"""Dense cells against the oracle: 25 particles per quad4 cell and 27 per hex8
cell.  A P2G tile then holds more particles than its threads, so it stages
them in several chunks, and every cell's particle segment is longer than the
16 entries the parallel rank sort covers, so each is sorted by one thread.
FP64 bar of test_gpu_parity; mixed precision against FP64."""
import numpy as np
import pytest

from mpm_b200 import problems as P
from tests.parity import assert_parity, field_errors
from tests.test_gpu_parity import _run_both

pytestmark = pytest.mark.gpu


def dense_2d(scheme):
    prob = P.column_2d(shape=(16, 12), block=(6, 8), nsteps=50, scheme=scheme)
    pts = P.quarter_point_particles(2, [(0, 6), (0, 8)], prob.dx, ppc_dir=5, seed=P.SEED_BASE + 7)
    prob.particles = [(pts, 0)]
    return prob


def dense_3d(scheme):
    prob = P.column_3d(shape=(8, 6, 8), block=(4, 4, 4), scheme=scheme, dt=1e-5, c=2000., psi=5.)
    pts = P.quarter_point_particles(3, [(0, 4), (0, 4), (0, 4)], prob.dx, ppc_dir=3,
                                    seed=P.SEED_BASE + 8)
    prob.particles = [(pts, 0)]
    prob.initial_stress = P.geostatic_stress(pts, 3, 1800., 0.3, 4 * prob.dx)
    return prob


@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_2d_dense_cells(scheme):
    for s, g, o in _run_both(dense_2d(scheme), [1, 10, 50]):
        assert_parity(g, o, label=f"2D dense {scheme} step {s}")


@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_3d_dense_cells(scheme):
    for s, g, o in _run_both(dense_3d(scheme), [1, 10, 30]):
        assert_parity(g, o, label=f"3D dense {scheme} step {s}")


def test_dense_cells_mixed_precision():
    out = {}
    for prec in ("fp64", "mixed"):
        sol = P.build_solver(dense_3d("usl"), precision=prec)
        sol.step(30)
        out[prec] = sol.read()
    assert np.array_equal(out["mixed"]["cell"], out["fp64"]["cell"])
    errs = field_errors(out["mixed"], out["fp64"], ("u", "v", "stress", "strain"))
    assert all(v <= 1e-5 for v in errs.values()), errs
