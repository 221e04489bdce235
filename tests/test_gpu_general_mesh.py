"""General meshes (not a tensor-product grid) against the CPU oracle.

On a general mesh the particle kernels read each cell's node ids and nodal
coordinates from the connectivity tables and evaluate J^-1 at every point
(quadrilateral_element.tcc:295-309, hexahedron_element.tcc:307-321), and the
locate step searches the cell-neighbour lists instead of the grid axes.  Two
kinds of meshes take that path here:

* renumbered: a column mesh with its node ids permuted, the geometry
  unchanged (the grid detection needs x-fastest node ids);
* distorted: interior nodes of a column mesh displaced by up to 15% of the
  cell size, so the cells are general quadrilaterals / hexahedra.

FP64 bar as in test_gpu_parity: cell ids bit-exact, fields within FP64_RTOL.
"""
import numpy as np
import pytest

from mpm_b200 import problems as P
from tests.parity import assert_parity, field_errors, mc_state_errors
from tests.test_gpu_parity import _run_both, small_column_2d, small_column_3d

pytestmark = pytest.mark.gpu


def renumber_nodes(prob, seed=11):
    """The same mesh with node ids permuted (constraints follow the nodes)."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(prob.nnodes)  # old id -> new id
    coords = np.empty_like(prob.coords)
    coords[perm] = prob.coords
    prob.coords = coords
    prob.cells = perm[prob.cells]
    if prob.velocity_constraints is not None:
        nid, d, v = prob.velocity_constraints
        prob.velocity_constraints = (perm[nid], d, v)
    if prob.friction_constraints is not None:
        nid, d, sgn, mu = prob.friction_constraints
        prob.friction_constraints = (perm[nid], d, sgn, mu)
    return prob


def distort_interior(prob, frac=0.15, seed=12):
    """Interior nodes moved by up to frac * dx per axis; nodes on the bounding
    box stay, so the wall constraints keep their meaning."""
    rng = np.random.default_rng(seed)
    c = prob.coords
    lo, hi = c.min(axis=0), c.max(axis=0)
    interior = np.all((c > lo + 1e-12) & (c < hi - 1e-12), axis=1)
    shift = rng.uniform(-frac, frac, c.shape) * prob.dx
    prob.coords = c + shift * interior[:, None]
    return prob


@pytest.mark.parametrize("mesh", ["renumbered", "distorted"])
@pytest.mark.parametrize("scheme", ["usf", "usl", "musl"])
def test_2d_linear_elastic_column(mesh, scheme):
    prob = small_column_2d(scheme=scheme)
    prob = renumber_nodes(prob) if mesh == "renumbered" else distort_interior(prob)
    for s, g, o in _run_both(prob, [1, 10, 100]):
        assert_parity(g, o, label=f"2D LE {mesh} {scheme} step {s}")


@pytest.mark.parametrize("mesh", ["renumbered", "distorted"])
@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_3d_mohr_coulomb_column_with_friction(mesh, scheme):
    prob = small_column_3d(scheme=scheme, dt=1e-5, c=2000., psi=5.)
    prob = renumber_nodes(prob) if mesh == "renumbered" else distort_interior(prob)
    for s, g, o in _run_both(prob, [1, 10, 50]):
        assert_parity(g, o, label=f"3D MC {mesh} {scheme} step {s}")
        errs = mc_state_errors(g, o)
        assert np.array_equal(g["svars"][:, 0], o["svars"][:, 0]), "yield states differ"
        assert errs["pdstrain"] < 1e-9 and errs["epsilon"] < 1e-9, errs


def test_renumbered_mesh_matches_the_grid_run():
    """Same geometry through both kernel paths: the per-axis J^-1 of a box
    cell and the general J^-1 differ by rounding only."""
    grid = P.build_solver(small_column_3d(scheme="usl", dt=1e-5, c=2000., psi=5.))
    gen = P.build_solver(renumber_nodes(small_column_3d(scheme="usl", dt=1e-5, c=2000., psi=5.)))
    grid.step(50)
    gen.step(50)
    a, b = grid.read(), gen.read()
    assert np.array_equal(a["cell"], b["cell"])
    errs = field_errors(b, a, ("x", "u", "v", "stress", "strain"))
    assert all(v < 1e-10 for v in errs.values()), errs


@pytest.mark.parametrize("mesh", ["renumbered", "distorted"])
def test_mixed_precision_on_general_mesh(mesh):
    """The mixed-precision kernels' general-mesh path against FP64 over 50
    steps: within 1e-5 plus twice the spread of FP64 runs whose initial states
    differ by FP32 rounding (the bar of the cohesionless column in
    test_gpu_mixed).  Most points of these columns return on the tension
    branch; near the floor those returns turn the FP32 rounding of the initial
    state alone into a 3e-6 velocity difference on the renumbered mesh, and
    the mixed path's largest errors (1e-5) sit on the same points."""
    from tests.test_gpu_mixed import _run

    def make():
        prob = small_column_3d(scheme="usl", dt=1e-5, c=2000., psi=5.)
        return renumber_nodes(prob) if mesh == "renumbered" else distort_interior(prob)

    f, m, fl = _run(make(), 50, "fp64"), _run(make(), 50, "mixed"), _run(make(), 50, "fp64", floor=True)
    assert np.array_equal(m["cell"], f["cell"])
    fields = ("u", "v", "stress", "strain")
    em, ef = field_errors(m, f, fields), field_errors(fl, f, fields)
    for k in fields:
        assert em[k] <= 2 * ef[k] + 1e-5, (k, em[k], ef[k])


@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_isoparametric_2d_distorted_column(scheme):
    """Isoparametric local coordinates (cell.tcc:617-826) on a distorted mesh:
    the locate step and every kernel's local coordinates take the inverse of
    the bilinear map."""
    prob = distort_interior(small_column_2d(scheme=scheme), frac=0.2)
    prob.analysis["isoparametric"] = True
    for s, g, o in _run_both(prob, [1, 10, 100]):
        assert_parity(g, o, label=f"2D LE isoparametric {scheme} step {s}")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_isoparametric_3d_distorted_mohr_coulomb(precision):
    prob = distort_interior(small_column_3d(scheme="usl", dt=1e-5, c=2000., psi=5.), frac=0.2)
    prob.analysis["isoparametric"] = True
    if precision == "fp64":
        for s, g, o in _run_both(prob, [1, 10, 50]):
            assert_parity(g, o, label=f"3D MC isoparametric step {s}")
        return
    out = {}
    for prec in ("fp64", "mixed"):
        sol = P.build_solver(prob, precision=prec)
        sol.step(50)
        out[prec] = sol.read()
    assert np.array_equal(out["mixed"]["cell"], out["fp64"]["cell"])
    errs = field_errors(out["mixed"], out["fp64"], ("u", "v", "stress", "strain"))
    assert all(v <= 1e-5 for v in errs.values()), errs


def test_isoparametric_differs_from_cartesian_on_a_distorted_mesh():
    """The two local-coordinate maps give different positions on a distorted
    mesh (the flag is not ignored)."""
    runs = {}
    for iso in (False, True):
        prob = distort_interior(small_column_2d(scheme="usl"), frac=0.2)
        prob.analysis["isoparametric"] = iso
        sol = P.build_solver(prob)
        sol.step(20)
        runs[iso] = sol.read()
    assert np.max(np.abs(runs[True]["x"] - runs[False]["x"])) > 1e-9
