"""The oracle's isoparametric local coordinates (cell.tcc:617-826): on a
distorted mesh every particle's xi maps back to its position through the
cell's bilinear / trilinear map, and on a grid the isoparametric xi equals
the Cartesian one to rounding."""
import numpy as np
import pytest

from mpm_b200 import problems as P
from oracle import oracle as O
from oracle.oracle import build_oracle
from tests.test_gpu_general_mesh import distort_interior


def _mapped_back(prob, st):
    """max |sum_i N_i(xi) X_i - x| over the particles."""
    dim = prob.dim
    err = 0.0
    for x, xi, c in zip(st["x"], st["xi"], st["cell"]):
        X = prob.coords[prob.cells[c]]
        N, _, _ = O.element_dn_dx(dim, xi[:dim], X)
        err = max(err, float(np.max(np.abs(N @ X - x[:dim]))))
    return err


@pytest.mark.parametrize("dim", [2, 3])
def test_isoparametric_xi_maps_back_on_a_distorted_mesh(dim):
    base = P.column_2d(shape=(12, 8), block=(6, 6)) if dim == 2 else \
        P.column_3d(shape=(6, 4, 5), block=(3, 3, 3))
    prob = distort_interior(base, frac=0.2)
    prob.analysis["isoparametric"] = True
    o = build_oracle(prob)
    st = o.get()
    assert np.all(st["cell"] >= 0)
    assert _mapped_back(prob, st) < 1e-12 * prob.dx


def test_isoparametric_equals_cartesian_on_a_grid():
    a = P.column_2d(shape=(12, 8), block=(6, 6))
    b = P.column_2d(shape=(12, 8), block=(6, 6))
    b.analysis["isoparametric"] = True
    sa, sb = build_oracle(a).get(), build_oracle(b).get()
    assert np.array_equal(sa["cell"], sb["cell"])
    assert np.max(np.abs(sa["xi"] - sb["xi"])) < 1e-14
