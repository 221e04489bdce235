"""Sensitivities (forward-mode derivatives of the FP64 USL step) through the C ABI.

The values a tangent run computes must be the FP64 step's, bit for bit (same
operations, the derivatives ride alongside); the gradient of a calibration loss
must match central finite differences of the FP64 path (relative step 1e-6)
within 1e-4 relative.
"""
import numpy as np
import pytest

from mpm_b200 import problems as P
from mpm_b200.sensitivity import run_with_sensitivities

pytestmark = pytest.mark.gpu

PARAMS = [(0, "youngs_modulus"), (0, "friction")]


def _prob(theta):
    E, phi = theta
    return P.calibration_column(phi=phi, E=E, shape=(16, 8, 12), block=(8, 6, 8), dx=0.01,
                                dt=5e-6, c=200.0, tension_cutoff=0.0)


def _build(theta):
    return P.build_solver(_prob(theta), precision="fp64")


def test_tangent_run_values_equal_the_fp64_run():
    theta = (1e7, 30.0)
    a = _build(theta)
    a.set_sensitivities(PARAMS)
    a.step(40)
    b = _build(theta)
    b.step(40)
    A, B = a.read(), b.read()
    for k in ("x", "u", "v", "stress", "strain", "F", "volume", "density", "svars", "cell"):
        assert np.array_equal(A[k], B[k]), k


def _prob_tc(theta):
    """Column with cohesion 500 Pa and a 10 kPa tension cutoff: shear returns
    during the run, a loss that is smooth in (E, phi)."""
    E, phi = theta
    return P.calibration_column(phi=phi, E=E, shape=(16, 8, 12), block=(8, 6, 8), dx=0.01,
                                dt=1e-5, c=500.0, tension_cutoff=1e4)


@pytest.mark.parametrize("mesh", ["renumbered", "distorted"])
def test_tangent_values_on_a_general_mesh_equal_the_fp64_run(mesh):
    """The tangent step's general-mesh kernels (nodal coordinates, J^-1 at every
    point, 64-thread P2G tiles): values bit for bit those of the FP64 step."""
    from tests.test_gpu_general_mesh import distort_interior, renumber_nodes
    make = renumber_nodes if mesh == "renumbered" else distort_interior
    theta = (1e7, 30.0)
    a = P.build_solver(make(_prob(theta)), precision="fp64")
    a.set_sensitivities(PARAMS)
    a.step(40)
    b = P.build_solver(make(_prob(theta)), precision="fp64")
    b.step(40)
    A, B = a.read(), b.read()
    for k in ("x", "u", "v", "stress", "strain", "F", "volume", "density", "svars", "cell"):
        assert np.array_equal(A[k], B[k]), k
    J = a.read_sensitivities("x")
    assert np.all(np.isfinite(J)) and np.max(np.abs(J)) > 0


def test_gradient_of_a_calibration_loss_matches_central_differences():
    """Loss = sum |x_final - x_target|^2 with the target run at (8e6, 32 deg),
    gradient at (1e7, 30 deg) after 150 steps: within 1e-4 of central
    differences with relative step 1e-6."""
    steps = 150
    build = lambda th: P.build_solver(_prob_tc(th), precision="fp64")

    def loss(theta):
        s = build(theta)
        s.step(steps)
        v = np.sum((s.read()["x"] - target) ** 2)
        s.close()
        return v

    s = build((8e6, 32.0))
    s.step(steps)
    target = s.read()["x"]
    theta = np.array([1e7, 30.0])
    x, J = run_with_sensitivities(build, theta, PARAMS, steps)
    grad = 2.0 * np.einsum("pd,kpd->k", x - target, J)
    assert grad[1] != 0.0  # the friction angle acts through plastic returns
    for k in range(2):
        h = 1e-6 * theta[k]
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (loss(tp) - loss(tm)) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-4 * abs(fd), (k, grad[k], fd)


def test_autograd_function_contracts_the_terminal_jacobian():
    torch = pytest.importorskip("torch")
    from mpm_b200.sensitivity import TerminalPositions
    theta = torch.tensor([1e7, 30.0], dtype=torch.float64, requires_grad=True)
    x = TerminalPositions.apply(theta, _build, PARAMS, 30)
    w = torch.linspace(0.0, 1.0, x.numel(), dtype=torch.float64).reshape(x.shape)
    (x * w).sum().backward()
    _, J = run_with_sensitivities(_build, theta.detach().numpy(), PARAMS, 30)
    ref = np.einsum("pd,kpd->k", w.numpy(), J)
    assert np.allclose(theta.grad.numpy(), ref, rtol=1e-12, atol=0)


def test_sensitivities_need_fp64_usl():
    from mpm_b200._native import MPMError
    s = P.build_solver(_prob((1e7, 30.0)), precision="mixed")
    with pytest.raises(MPMError, match="FP64"):
        s.set_sensitivities(PARAMS)
