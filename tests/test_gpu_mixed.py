"""Mixed-precision path (MPM_PRECISION_MIXED) against the FP64 path.

The mixed path has no counterpart in the reference.  Its error is reported per
field as max |mixed - fp64| / max |fp64| after a run.  Some problems amplify
any perturbation: the cohesionless MohrCoulomb column (c = 0, psi = 0) turns a
1e-8 change of the initial stress into a 1e-3 change of the stress field after
a few hundred steps.  There the bar is the problem's own conditioning: the FP64
path started from the FP32-rounded initial state (the "floor") differs from the
FP64 path by as much as the mixed path does.
"""
import numpy as np
import pytest

from mpm_b200 import problems as P
from tests.parity import field_errors

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "stress", "strain", "F", "volume", "density")


def _errors(a, b):
    a = dict(a)
    b = dict(b)
    a["F"] = a["F"] - np.eye(3).reshape(1, 9)  # compare F - I: F is I + O(1e-4)
    b["F"] = b["F"] - np.eye(3).reshape(1, 9)
    return field_errors(a, b, FIELDS)


def _run(prob, steps, precision, floor=False):
    s = P.build_solver(prob, precision=precision)
    if floor:
        st = s.read()
        for k in ("stress", "v", "volume", "density", "mass"):
            st[k] = st[k].astype(np.float32).astype(np.float64)
        s.load(st)
    s.step(steps)
    return s.read()


def test_linear_elastic_2d_within_1e5_of_fp64():
    """2D LinearElastic column, USF, 2,000 steps: every field within 1e-5."""
    prob = P.column_2d()
    m, f = _run(prob, 2000, "mixed"), _run(prob, 2000, "fp64")
    assert np.array_equal(m["cell"], f["cell"])
    errs = _errors(m, f)
    assert all(v <= 1e-5 for v in errs.values()), errs


@pytest.mark.parametrize("scheme", ["usf", "usl", "musl"])
def test_mohr_coulomb_3d_short_horizon_within_1e5(scheme):
    prob = P.column_3d(shape=(20, 10, 10), block=(10, 10, 10), scheme=scheme)
    m, f = _run(prob, 50, "mixed"), _run(prob, 50, "fp64")
    assert np.array_equal(m["cell"], f["cell"])
    errs = _errors(m, f)
    assert all(v <= 1e-5 for v in errs.values()), errs
    pd = np.max(np.abs(m["svars"][:, 8] - f["svars"][:, 8])) / np.max(f["svars"][:, 8])
    assert pd <= 1e-3


def test_cohesionless_column_error_is_the_problems_conditioning():
    """c = 0 column, USL, 300 steps: the mixed error is no larger than twice
    the spread between FP64 runs whose initial states differ by FP32 rounding."""
    prob = P.column_3d(shape=(20, 10, 10), block=(10, 10, 10))
    f = _run(prob, 300, "fp64")
    m = _run(prob, 300, "mixed")
    fl = _run(prob, 300, "fp64", floor=True)
    em, ef = _errors(m, f), _errors(fl, f)
    for k in ("u", "v", "stress", "strain"):
        assert em[k] <= 2 * ef[k] + 1e-5, (k, em[k], ef[k])


def test_cohesive_column_long_horizon():
    """c = 2 kPa, psi = 5 deg column, USL, 500 steps: a well-conditioned
    problem, where the FP32 rounding of the stored state accumulates to a few
    1e-5 of each field."""
    prob = P.column_3d(shape=(20, 10, 10), block=(10, 10, 10), c=2000., psi=5.)
    m, f = _run(prob, 500, "mixed"), _run(prob, 500, "fp64")
    errs = _errors(m, f)
    assert all(v <= 2e-4 for v in errs.values()), errs


def test_rigid_translation_keeps_cells_and_positions():
    """A stress-free block moving across cell faces: cells identical to the FP64
    path; displacements (FP64 sums of FP32 nodal velocity times dt) within 1e-6."""
    prob = P.column_3d(shape=(12, 10, 10), block=(4, 4, 4), material="LinearElastic", E=5e5,
                       scheme="usl", dt=2e-4, geostatic=False)
    prob.analysis["gravity"] = (0.0, 0.0, 0.0)
    pts, mid = prob.particles[0]
    prob.particles = [(pts + np.array([0.03, 0.03, 0.04]), mid)]
    out = {}
    for prec in ("fp64", "mixed"):
        s = P.build_solver(prob, precision=prec)
        st = s.read()
        st["v"] = np.tile([2.0, -1.5, 1.0], (len(st["x"]), 1))
        s.load(st)
        c0 = st["cell"].copy()
        s.step(40)
        out[prec] = s.read()
    assert np.array_equal(out["mixed"]["cell"], out["fp64"]["cell"])
    assert np.count_nonzero(out["fp64"]["cell"] != c0) > len(c0) // 2
    x, y = out["mixed"]["u"], out["fp64"]["u"]
    assert np.max(np.abs(x - y)) / np.max(np.abs(y)) <= 1e-6


def test_mixed_runs_are_bitwise_deterministic():
    prob = P.column_3d(shape=(20, 10, 10), block=(10, 10, 10))
    a, b = _run(prob, 100, "mixed"), _run(prob, 100, "mixed")
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_read_load_round_trip():
    """read -> load into a new mixed solver -> read gives the same state (F, V
    and rho pass through their deviation forms)."""
    prob = P.column_3d(shape=(12, 6, 8), block=(6, 6, 8))
    a = P.build_solver(prob, precision="mixed")
    a.step(30)
    A = a.read()
    b = P.build_solver(prob, precision="mixed")
    b.load(A)
    B = b.read()
    for k in A:
        np.testing.assert_allclose(B[k], A[k], rtol=1e-6, atol=0, err_msg=k)


def test_footing_on_slope_mixed():
    """Two materials and a footing constraint, USL, 200 steps: the footing
    yields the slope under it; the FP32 elastic predictor and stored stress put
    the stress field within a few 1e-4 of the FP64 path, the kinematic fields
    within a few 1e-5."""
    prob = P.footing_slope(shape=(40, 10, 20), foundation=4, slope_height=8, slope_top=6,
                           footing=(1, 5), dt=1e-5)
    m, f = _run(prob, 200, "mixed"), _run(prob, 200, "fp64")
    assert np.array_equal(m["cell"], f["cell"])
    errs = _errors(m, f)
    assert all(v <= 3e-4 for v in errs.values()), errs
    assert errs["u"] <= 1e-5 and errs["v"] <= 5e-5, errs


def test_musl_2d_linear_elastic_within_1e5_of_fp64():
    """MUSL (mpm_scheme_musl.tcc:20-35) in mixed precision: the 2D LinearElastic
    column over 1,000 steps, every field within 1e-5 of the FP64 MUSL run."""
    prob = P.column_2d(scheme="musl")
    m, f = _run(prob, 1000, "mixed"), _run(prob, 1000, "fp64")
    assert np.array_equal(m["cell"], f["cell"])
    errs = _errors(m, f)
    assert all(v <= 1e-5 for v in errs.values()), errs


def _mapping_error(m, f):
    return float(np.max(np.abs(m["mapping"] - f["mapping"])) / np.max(np.abs(f["mapping"])))


@pytest.mark.parametrize("vu", ["asflip", "tpic", "apic"])
@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_mapping_matrix_updates_2d_within_1e5_of_fp64(vu, scheme):
    """ASFLIP / TPIC / APIC (particle.tcc:1071-1139, 1663-1730) in mixed
    precision: the 2D LinearElastic column over 1,000 steps, every field within
    1e-5 of the FP64 run of the same update, the mapping matrix within 1e-4
    (it is a difference of nodal velocities, formed from FP32 values)."""
    prob = P.column_2d(scheme=scheme, velocity_update=vu)
    m, f = _run(prob, 1000, "mixed"), _run(prob, 1000, "fp64")
    assert np.array_equal(m["cell"], f["cell"])
    errs = _errors(m, f)
    assert all(v <= 1e-5 for v in errs.values()), (vu, scheme, errs)
    assert _mapping_error(m, f) <= 1e-4, (vu, scheme, _mapping_error(m, f))


@pytest.mark.parametrize("vu", ["asflip", "tpic", "apic"])
def test_mapping_matrix_updates_3d_mohr_coulomb_short_horizon(vu):
    """The cohesive column (c = 2 kPa, psi = 5 deg) over 50 USL steps: every
    field within 1e-5.  In the cohesionless column APIC and TPIC bring the
    top corner's points to the apex (tension state) within 50 steps; those
    few points' stresses are then within 7e-4 of FP64, every other point's
    within 7e-7, which is the apex return's conditioning."""
    prob = P.column_3d(shape=(20, 10, 10), block=(10, 10, 10), scheme="usl", velocity_update=vu,
                       c=2000., psi=5.)
    m, f = _run(prob, 50, "mixed"), _run(prob, 50, "fp64")
    assert np.array_equal(m["cell"], f["cell"])
    errs = _errors(m, f)
    assert all(v <= 1e-5 for v in errs.values()), (vu, errs)
    assert _mapping_error(m, f) <= 1e-4, (vu, _mapping_error(m, f))
