"""The reverse-mode adjoint of the FP64 USL step, through the C ABI.

Its gradient is checked three ways:
* against the forward-mode tangent (the same derivative of the same discrete
  step, computed the other way round): within 1e-8 relative, on columns with
  shear, tensile and apex returns, over several checkpoint segments;
* against central differences of the CPU oracle's loss (relative step 1e-6)
  on a smooth case, an FP64 reference gradient independent of the GPU code;
* against central differences of the GPU's loss on the same smooth case, and,
  for the initial state (positions, velocities, stresses), on a LinearElastic
  column.
The loss is L = sum |x_final - x_target|^2 (x_target from a run at E = 8e6 Pa,
phi = 32 deg), the parameters Young's modulus and the friction angle.
"""
import numpy as np
import pytest

from mpm_b200 import problems as P
from mpm_b200.sensitivity import run_with_sensitivities

pytestmark = pytest.mark.gpu

PARAMS = [(0, "youngs_modulus"), (0, "friction")]
THETA = np.array([1e7, 30.0])


def _column(theta, c=500.0, tc=1e4, dt=1e-5, shape=(16, 8, 12), block=(8, 6, 8), vu="flip"):
    E, phi = theta
    p = P.calibration_column(phi=phi, E=E, shape=shape, block=block, dx=0.01, dt=dt, c=c,
                             tension_cutoff=tc)
    p.analysis["velocity_update"] = vu
    return p


def _target(make, steps):
    s = P.build_solver(make((8e6, 32.0)), precision="fp64")
    s.step(steps)
    x = s.read()["x"]
    s.close()
    return x


def _tangent_grad(make, steps, target):
    build = lambda th: P.build_solver(make(th), precision="fp64")
    x, J = run_with_sensitivities(build, THETA, PARAMS, steps)
    return 2.0 * np.einsum("pd,kpd->k", x - target, J)


def _adjoint_grad(make, steps, target, every):
    s = P.build_solver(make(THETA), precision="fp64")
    loss, g = s.adjoint_run(steps, PARAMS, target, checkpoint_every=every)
    s.close()
    return loss, g


@pytest.mark.parametrize("case", ["smooth", "tensile_apex", "pic"])
def test_adjoint_gradient_equals_the_tangent_gradient(case):
    if case == "smooth":  # c = 500 Pa, 10 kPa tension cutoff: shear returns
        make, steps, every = (lambda th: _column(th)), 150, 40
    elif case == "tensile_apex":  # c = 200 Pa, no tension cutoff: tensile and apex returns
        make, steps, every = (lambda th: _column(th, c=200.0, tc=0.0, dt=5e-6)), 60, 7
    else:  # PIC damps the motion so that no point yields: dL/dphi is exactly 0
        make, steps, every = (lambda th: _column(th, vu="pic")), 150, 60
    target = _target(make, steps)
    gt = _tangent_grad(make, steps, target)
    _, ga = _adjoint_grad(make, steps, target, every)
    assert gt[0] != 0.0 and (case == "pic" or gt[1] != 0.0)
    for k in range(2):
        assert abs(ga[k] - gt[k]) <= 1e-8 * abs(gt[k]), (case, k, ga[k], gt[k])


def test_adjoint_matches_central_differences_of_the_oracle():
    """An FP64 reference gradient from the CPU oracle: central differences of
    the oracle's own loss with relative step 1e-6, within 1e-4 (the bound the
    central differences of a smooth case meet; over 150 steps the shear
    returns give the friction angle a gradient far above the loss's rounding)."""
    from oracle.oracle import build_oracle
    steps = 150

    def oracle_x(theta):
        o = build_oracle(_column(theta))
        o.step(steps)
        return o.get()["x"]

    target = oracle_x((8e6, 32.0))
    _, ga = _adjoint_grad(lambda th: _column(th), steps, target, 30)
    for k in range(2):
        h = 1e-6 * THETA[k]
        tp, tm = THETA.copy(), THETA.copy()
        tp[k] += h
        tm[k] -= h
        fd = (np.sum((oracle_x(tp) - target) ** 2) - np.sum((oracle_x(tm) - target) ** 2)) / (2 * h)
        assert abs(ga[k] - fd) <= 1e-4 * abs(fd), (k, ga[k], fd)


def test_adjoint_matches_central_differences_of_the_gpu_loss():
    steps = 150
    make = lambda th: _column(th)
    target = _target(make, steps)

    def loss(theta):
        s = P.build_solver(make(theta), precision="fp64")
        s.step(steps)
        v = np.sum((s.read()["x"] - target) ** 2)
        s.close()
        return v

    L, ga = _adjoint_grad(make, steps, target, 50)
    assert abs(L - loss(THETA)) <= 1e-12 * L
    for k in range(2):
        h = 1e-6 * THETA[k]
        tp, tm = THETA.copy(), THETA.copy()
        tp[k] += h
        tm[k] -= h
        fd = (loss(tp) - loss(tm)) / (2 * h)
        assert abs(ga[k] - fd) <= 1e-4 * abs(fd), (k, ga[k], fd)


def test_initial_state_gradient_matches_central_differences():
    """dL/dx0, dL/dv0 and dL/dstress0 of a LinearElastic 3D column in a slip
    box, for a few particles and components.  The step snaps entries below
    1e-15 to zero and a frictional floor switches between stick and slip: at
    such kinks the derivative is that of the branch taken, which central
    differences straddle.  So the column starts from random velocities (no
    nodal velocity or strain rate exactly zero) and has no frictional floor."""
    steps = 60
    prob = P.column_3d(shape=(12, 8, 10), block=(6, 4, 6), material="LinearElastic", E=1e6,
                       scheme="usl", dt=1e-5)
    prob.friction_constraints = None
    s = P.build_solver(prob)
    st0 = s.read()
    st0["v"] = np.random.default_rng(11).normal(0.0, 1e-2, st0["v"].shape)
    s.load(st0)
    st0 = s.read()
    s.step(steps)
    rng = np.random.default_rng(5)
    target = s.read()["x"] + rng.normal(0, 1e-3, st0["x"].shape)
    s.close()

    def loss(state):
        q = P.build_solver(prob)
        q.load(state)
        q.step(steps)
        v = np.sum((q.read()["x"] - target) ** 2)
        q.close()
        return v

    a = P.build_solver(prob)
    a.load(st0)
    a.adjoint_record(steps, [], checkpoint_every=17)
    r = a.adjoint_reverse(dL_dx=2.0 * (a.read()["x"] - target))
    steps_h = {"x": 1e-7, "v": 1e-5, "stress": 1.0}
    key = {"x": "x0", "v": "v0", "stress": "stress0"}
    picks = [(f, p, c) for f in steps_h for p, c in ((3, 0), (100, 2), (777, 1))]
    for f, p, c in picks:
        h = steps_h[f]
        sp = {k: np.array(v, copy=True) for k, v in st0.items()}
        sm = {k: np.array(v, copy=True) for k, v in st0.items()}
        sp[f][p, c] += h
        sm[f][p, c] -= h
        fd = (loss(sp) - loss(sm)) / (2 * h)
        g = r[key[f]][p, c]
        assert abs(g - fd) <= 1e-4 * max(abs(fd), 1e-12), (f, p, c, g, fd)


def test_reverse_restores_the_end_state_and_repeats_bitwise():
    make = lambda th: _column(th)
    a = P.build_solver(make(THETA), precision="fp64")
    a.adjoint_record(50, PARAMS, checkpoint_every=20)
    end = a.read()
    b = P.build_solver(make(THETA), precision="fp64")
    b.step(50)
    ref = b.read()
    for k in ("x", "v", "stress", "cell", "svars"):
        assert np.array_equal(end[k], ref[k]), k
    w = np.linspace(-1.0, 1.0, end["x"].size).reshape(end["x"].shape)
    r1 = a.adjoint_reverse(dL_dx=w)
    after = a.read()
    for k in ("x", "v", "stress", "cell", "svars"):
        assert np.array_equal(after[k], ref[k]), k
    r2 = a.adjoint_reverse(dL_dx=w)
    for k in ("params", "x0", "v0", "stress0"):
        assert np.array_equal(r1[k], r2[k]), k


def test_checkpoint_spacing_does_not_change_the_gradient():
    """Every spacing -- each step kept (no recompute), the library's choice,
    uneven segments, one segment -- gives the same gradient bit for bit: the
    recomputed steps are the forward steps' own arithmetic."""
    make = lambda th: _column(th)
    w = None
    out = {}
    for every in (1, 0, 7, 45):
        s = P.build_solver(make(THETA), precision="fp64")
        s.adjoint_record(45, PARAMS, checkpoint_every=every)
        if w is None:
            x = s.read()["x"]
            w = np.cos(np.arange(x.size)).reshape(x.shape)
        out[every] = s.adjoint_reverse(dL_dx=w)
        s.close()
    for every, r in out.items():
        for k in ("params", "x0", "v0", "stress0"):
            assert np.array_equal(r[k], out[1][k]), (every, k)


def test_recording_again_reuses_the_tape_and_repeats_bitwise():
    """A calibration loop records the same run shape many times: the tape's
    buffers are kept, and a second record of the same start state gives the
    same gradient bit for bit (also after a record of another shape)."""
    s = P.build_solver(_column(THETA), precision="fp64")
    st0 = s.read()
    w = None
    out = []
    for steps, every in ((30, 1), (12, 5), (30, 1)):
        s.load(st0)
        s.set_current_step(0)
        s.adjoint_record(steps, PARAMS, checkpoint_every=every)
        if w is None:
            x = s.read()["x"]
            w = np.sin(np.arange(x.size)).reshape(x.shape)
        out.append(s.adjoint_reverse(dL_dx=w))
    for k in ("params", "x0", "v0", "stress0"):
        assert np.array_equal(out[0][k], out[2][k]), k
    assert not np.array_equal(out[0]["params"], out[1]["params"])


def test_autograd_function_runs_the_reverse_sweep():
    torch = pytest.importorskip("torch")
    from mpm_b200.sensitivity import AdjointPositions
    build = lambda th: P.build_solver(_column(th), precision="fp64")
    theta = torch.tensor(THETA, dtype=torch.float64, requires_grad=True)
    x = AdjointPositions.apply(theta, build, PARAMS, 40, 15)
    w = torch.linspace(0.0, 1.0, x.numel(), dtype=torch.float64).reshape(x.shape)
    (x * w).sum().backward()
    _, J = run_with_sensitivities(build, THETA, PARAMS, 40)
    ref = np.einsum("pd,kpd->k", w.numpy(), J)
    assert np.allclose(theta.grad.numpy(), ref, rtol=1e-8, atol=0)


def test_adjoint_refuses_paths_it_does_not_differentiate():
    from mpm_b200._native import MPMError
    s = P.build_solver(_column(THETA), precision="mixed")
    with pytest.raises(MPMError, match="FP64"):
        s.adjoint_record(10, PARAMS)
    p = _column(THETA)
    p.analysis["scheme"] = "usf"
    s = P.build_solver(p)
    with pytest.raises(MPMError, match="USL"):
        s.adjoint_record(10, PARAMS)
