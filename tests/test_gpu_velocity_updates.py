"""ASFLIP / APIC / TPIC velocity updates (particle.tcc:630-721, 994-1139,
1663-1730) on the CUDA path against the oracle: the affine or Taylor
mass-momentum mapping in P2G, the mapping matrix and the position update in
G2P, the ASFLIP beta (velocity-constrained nodes, compressive deformation
gradient increment).  FP64 bar of test_gpu_parity: cell ids bit-exact, every
field and the mapping matrix within FP64_RTOL."""
import numpy as np
import pytest

from mpm_b200 import problems as P
from mpm_b200.solver import MPMError
from tests.parity import FP64_RTOL, assert_parity, field_errors
from tests.test_gpu_general_mesh import distort_interior
from tests.test_gpu_parity import _run_both, small_column_2d, small_column_3d

pytestmark = pytest.mark.gpu

UPDATES = ["asflip", "tpic", "apic"]


def _assert_mapping(g, o, label):
    errs = field_errors(g, o, ("mapping",))
    assert errs["mapping"] <= FP64_RTOL, f"{label}: mapping matrix {errs}"


@pytest.mark.parametrize("vu", UPDATES)
@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_2d_linear_elastic_column(vu, scheme):
    prob = small_column_2d(scheme=scheme, velocity_update=vu)
    for s, g, o in _run_both(prob, [1, 10, 100]):
        label = f"2D LE {vu} {scheme} step {s}"
        assert_parity(g, o, label=label)
        _assert_mapping(g, o, label)


@pytest.mark.parametrize("vu", UPDATES)
def test_3d_mohr_coulomb_column_usl(vu):
    prob = small_column_3d(scheme="usl", dt=1e-5, c=2000., psi=5., velocity_update=vu)
    for s, g, o in _run_both(prob, [1, 10, 50]):
        label = f"3D MC {vu} USL step {s}"
        assert_parity(g, o, label=label)
        _assert_mapping(g, o, label)


@pytest.mark.parametrize("vu", ["asflip", "apic"])
def test_distorted_mesh(vu):
    prob = distort_interior(small_column_2d(scheme="usl", velocity_update=vu))
    for s, g, o in _run_both(prob, [1, 20]):
        label = f"2D distorted {vu} step {s}"
        assert_parity(g, o, label=label)
        _assert_mapping(g, o, label)


def test_mapping_matrix_load_and_read():
    s = P.build_solver(small_column_3d(scheme="usl", velocity_update="apic"))
    st = s.read()
    assert np.all(st["mapping"] == 0.0)
    rng = np.random.default_rng(5)
    b = rng.normal(0.0, 1e-3, st["mapping"].shape)
    st["mapping"] = b
    s.load(st)
    assert np.array_equal(s.read()["mapping"], b)


@pytest.mark.parametrize("over", [dict(scheme="musl"), dict(scheme="musl", precision="mixed")])
def test_unsupported_combinations_are_refused(over):
    prob = small_column_2d(velocity_update="apic")
    with pytest.raises(MPMError):
        P.build_solver(prob, **over)
