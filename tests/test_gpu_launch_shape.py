"""Launch shape of the steps and its autotuner (no counterpart in the
reference, whose steps are host loops).

The launch shape -- threads of a P2G cell tile, threads of a node-kernel
block, blocks per SM of the plastic-return kernel -- changes no result: the
per-(cell, slot) sums run over each cell's particles in particle-id order and
the node gathers over cells in ascending id whatever the tile, and every
plastic return is independent of the others.  So every shape gives the same
run bit for bit, and the autotuner, which times the candidates on the
solver's own state and restores it, leaves the run exactly as it was.
"""
import numpy as np
import pytest

from mpm_b200 import problems as P
from mpm_b200._native import MPMError

pytestmark = pytest.mark.gpu

FIELDS = ("x", "u", "v", "stress", "strain", "F", "volume", "density", "svars", "cell")


def _column(**kw):
    base = dict(shape=(16, 10, 12), block=(8, 6, 8), dt=1e-5)
    base.update(kw)
    return P.column_3d(**base)


def _assert_same(a, b, label):
    for k in FIELDS:
        if k in a:
            assert np.array_equal(a[k], b[k], equal_nan=True), (label, k)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("scheme", ["usl", "usf"])
def test_every_launch_shape_gives_the_same_run(precision, scheme):
    prob = _column(scheme=scheme)
    runs = {}
    for shape in [(0, 0, 0), (128, 128, 4), (256, 256, 16), (128, 256, 8)]:
        s = P.build_solver(prob, precision=precision)
        s.set_launch_shape(*shape)
        s.step(120)  # the c = 0 column: most points return plastically by then
        runs[shape] = s.read()
        s.close()
    ref = runs[(0, 0, 0)]
    assert np.any(ref["svars"][:, 0] != 0), "no plastic point"
    for shape, r in runs.items():
        _assert_same(r, ref, shape)


def test_autotune_restores_the_state_and_the_run():
    prob = _column()
    a = P.build_solver(prob)
    a.step(30)
    ref = a.read()
    a.close()
    b = P.build_solver(prob)
    b.step(10)
    before = b.read()
    report = b.autotune(steps=3)
    _assert_same(b.read(), before, "after autotune")
    chosen = report["chosen"]
    assert b.launch_shape() == (chosen["p2g_tile"], chosen["node_threads"],
                                chosen["return_blocks_per_sm"])
    assert set(report["trials"]) == {"p2g_tile", "node_threads", "return_blocks_per_sm"}
    assert all(v > 0 for t in report["trials"].values() for v in t.values())
    b.step(20)
    _assert_same(b.read(), ref, "run after autotune")


def test_general_mesh_keeps_its_tile():
    from tests.test_gpu_general_mesh import distort_interior
    prob = distort_interior(P.column_2d(shape=(12, 8), block=(4, 6)))
    s = P.build_solver(prob)
    assert s.launch_shape() == (128, 256, 8)
    report = s.autotune(steps=3)
    assert list(report["trials"]["p2g_tile"]) == ["128"]


def test_invalid_launch_shapes_are_refused():
    s = P.build_solver(_column())
    for shape in [(64, 0, 0), (0, 512, 0), (0, 0, 3)]:
        with pytest.raises(MPMError, match="must be"):
            s.set_launch_shape(*shape)
    with pytest.raises(MPMError, match="at least 3"):
        s.autotune(steps=1)
    assert s.launch_shape() == (256, 256, 8)
