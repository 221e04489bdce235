"""Persistent steps (mpm_gpu_set_persistent) against the per-pass launches.

The persistent kernel runs whole mixed USL steps in one cooperative launch,
each pass the body of the corresponding one-pass kernel, so every field must
equal the CUDA-graph path's bit for bit: over launches of uneven length, with
plastic returns, with particles that leave the mesh and are removed by the
exhaustive locate, with a gravity ramp (the ramp is evaluated on the device
per step), and on a packed ensemble.  Configurations it does not run are
refused.
"""
import numpy as np
import pytest

from mpm_b200 import MPMError
from mpm_b200 import ensemble as E
from mpm_b200 import problems as P
from tests.test_gpu_parity import _leaving_block

pytestmark = pytest.mark.gpu

FIELDS = ("x", "u", "v", "stress", "strain", "F", "volume", "density", "cell", "svars")
UNSUPPORTED = -7


def _both(prob, steps, per_launch, prepare=None, **kw):
    out = []
    for persistent in (0, per_launch):
        s = P.build_solver(prob, precision="mixed", **kw)
        if prepare:
            prepare(s)
        s.set_persistent(persistent)
        for n in steps:
            s.step(n)
        out.append(s.read())
        s.close()
    return out


def _assert_same(a, b, label):
    for k in FIELDS:
        assert np.array_equal(a[k], b[k], equal_nan=True), (label, k)


@pytest.mark.parametrize("vu", ["flip", "pic"])
def test_3d_mohr_coulomb_column_bitwise(vu):
    """Cohesionless column: shear, tension and apex returns within 60 steps."""
    prob = P.column_3d(shape=(20, 10, 10), block=(10, 10, 10), scheme="usl", velocity_update=vu)
    g, p = _both(prob, [1, 13, 46], 7)
    _assert_same(g, p, f"3D MC {vu}")
    assert np.any(p["svars"][:, 0] != 0)  # some points returned plastically


def test_2d_linear_elastic_column_with_gravity_ramp_bitwise():
    prob = P.column_2d(scheme="usl")
    prob.analysis["gravity_ramping_time"] = 2e-4  # 20 steps
    g, p = _both(prob, [25, 75], 16)
    _assert_same(g, p, "2D LE ramp")


def test_particles_leaving_the_mesh_bitwise():
    prob, vel = _leaving_block()
    prob.analysis["scheme"] = "usl"

    def push(s):
        st = s.read()
        st["v"] = np.tile(vel, (len(st["x"]), 1))
        s.load(st)

    g, p = _both(prob, [3, 4], 3, prepare=push, locate_particles=False)
    assert np.any(p["cell"] < 0) and np.any(p["cell"] >= 0)
    _assert_same(g, p, "leaving block")


def test_packed_ensemble_bitwise():
    runs = [E.SlopeRun(height=6, width=6, phi=30.0, cohesion=2000.0, margin=6, seed=11),
            E.SlopeRun(height=4, width=5, phi=25.0, cohesion=0.0, margin=6, seed=12),
            E.SlopeRun(height=9, width=4, phi=38.0, cohesion=1500.0, margin=6, seed=13)]
    prob, _ = E.ensemble_problem(runs, nsteps=100)
    g, p = _both(prob, [50, 50], 20)
    _assert_same(g, p, "ensemble")


def test_full_launches_replay_a_captured_graph():
    """After the first launch of a call, launches of steps_per_launch steps
    replay one captured CUDA graph (barrier reset + cooperative launch) whose
    kernel reads the step from device memory: bitwise the per-pass result."""
    prob = P.column_3d(shape=(20, 10, 10), block=(10, 10, 10), scheme="usl")
    prob.analysis["gravity_ramping_time"] = 3e-5  # the ramp spans the first 15 steps
    g, p = _both(prob, [20, 20], 4)
    _assert_same(g, p, "graph-replayed persistent launches")
    s = P.build_solver(prob, precision="mixed")
    s.set_persistent(4)
    s.step(12)
    assert s.persistent() == (4, True)


@pytest.mark.parametrize("over", [dict(precision="fp64"), dict(scheme="usf"), dict(scheme="musl"),
                                  dict(velocity_update="apic")])
def test_other_configurations_are_refused(over):
    over = dict(over)
    prec = over.pop("precision", "mixed")
    s = P.build_solver(P.column_2d(scheme="usl"), precision=prec, **over)
    with pytest.raises(MPMError) as e:
        s.set_persistent(10)
    assert e.value.code == UNSUPPORTED
    s.set_persistent(0)  # the default stays available
    s.step(2)
