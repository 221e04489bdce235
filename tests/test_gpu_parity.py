"""CUDA path (libmpm_b200.so through its C ABI) against the CPU oracle.

FP64 bar: cell ids bit-exact; every floating-point field within
FP64_RTOL = 1e-10 of the oracle, relative to the field's largest magnitude.
"""
import numpy as np
import pytest

from mpm_b200 import problems as P
from mpm_b200.solver import material_stress_batch
from oracle import oracle as O
from oracle.oracle import build_oracle
from tests.conftest import catch_approx
from tests.parity import FP64_RTOL, assert_parity, mc_state_errors

pytestmark = pytest.mark.gpu


def _run_both(prob, steps, **over):
    g = P.build_solver(prob, **over)
    o = build_oracle(prob, **over)
    g0, o0 = g.read(), o.get()
    assert_parity(g0, o0, label="initial state")
    done = 0
    out = []
    for s in steps:
        g.step(s - done)
        o.step(s - done)
        done = s
        out.append((s, g.read(), o.get()))
    return out


def small_column_2d(**kw):
    base = dict(shape=(24, 16), block=(6, 10), nsteps=100)
    base.update(kw)
    return P.column_2d(**base)


def small_column_3d(**kw):
    base = dict(shape=(12, 8, 10), block=(6, 4, 6), nsteps=100)
    base.update(kw)
    return P.column_3d(**base)


# ---------------------------------------------------------------- materials
def test_material_kernel_matches_reference_kats(kats):
    """The device constitutive update reproduces the reference's own KATs."""
    for r in kats["mohr_coulomb_stress"]:
        props = r["material"]
        st = O.mc_initial_state(O.material_params("MohrCoulomb", props))
        for k, v in r["state"].items():
            st[O.MC_STATE.index(k)] = v
        dens = props["density"] / (1.0 + r["dvolumetric_strain"])
        out, st2 = material_stress_batch(r["dim"], f"MohrCoulomb{r['dim']}D", props,
                                         [r["stress"]], [r["dstrain"]], dens, [st])
        for i in range(6):
            assert catch_approx(out[0, i], r["expected_stress"][i], r["epsilon"]), r["source"]
        if r["expected_pdstrain"] is not None:
            assert catch_approx(st2[0, 8], r["expected_pdstrain"], r["epsilon"]), r["source"]
    for r in kats["linear_elastic_stress"]:
        out, _ = material_stress_batch(r["dim"], f"LinearElastic{r['dim']}D", r["material"],
                                       [r["stress"]], [r["dstrain"]], r["material"]["density"])
        for i in range(6):
            assert catch_approx(out[0, i], r["expected_stress"][i], r["epsilon"]), r["source"]


@pytest.mark.parametrize("dim", [2, 3])
def test_mohr_coulomb_kernel_branch_coverage(dim):
    """Random stress states covering elastic, shear, tensile, apex and
    separated returns: device vs oracle within FP64_RTOL."""
    rng = np.random.default_rng(7 + dim)
    n = 4000
    props = P.mohr_coulomb(1e7, 0.3, 1800., 30., 2000., 5., tension_cutoff=500.)
    props["packing_fraction"] = 0.6
    props["packing_fraction_minimum"] = 0.4
    params = O.material_params("MohrCoulomb", props)
    stress = rng.normal(-3000., 4000., (n, 6))
    dstrain = rng.normal(0., 4e-4, (n, 6))
    if dim == 2:
        stress[:, 4:] = 0.
        dstrain[:, [2, 4, 5]] = 0.
    stress[: n // 8] = -0.5  # near the apex / zero stress
    density = np.full(n, 1800.)
    density[-n // 10:] = 500.  # separated state (below 0.4 * 1800 / 0.6)
    st0 = np.tile(O.mc_initial_state(params), (n, 1))
    out, st = material_stress_batch(dim, f"MohrCoulomb{dim}D", props, stress, dstrain, density, st0)
    ref = np.zeros((n, 6))
    refst = np.zeros((n, 9))
    for i in range(n):
        ref[i], refst[i] = O.material_stress(dim, "MohrCoulomb", props, stress[i], dstrain[i],
                                             density[i], st0[i])
    kinds = set(np.round(refst[:, 0]).astype(int))
    assert {0, 1, 2, 3} <= kinds, kinds
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(out - ref)) / scale < FP64_RTOL
    assert np.array_equal(np.round(st[:, 0]), np.round(refst[:, 0]))
    for k in range(1, 9):
        sc = max(np.max(np.abs(refst[:, k])), 1e-300)
        assert np.max(np.abs(st[:, k] - refst[:, k])) / sc < 1e-9, k


# -------------------------------------------------------------- whole steps
@pytest.mark.parametrize("scheme", ["usf", "usl"])
@pytest.mark.parametrize("vupd", ["flip", "pic"])
def test_2d_linear_elastic_column(scheme, vupd):
    prob = small_column_2d(scheme=scheme, velocity_update=vupd)
    for s, g, o in _run_both(prob, [1, 10, 100]):
        assert_parity(g, o, label=f"2D LE {scheme} {vupd} step {s}")


@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_3d_mohr_coulomb_column_with_friction(scheme):
    """Cohesive MohrCoulomb (c = 2 kPa, psi = 5) over 50 steps: the points stay
    off the yield-surface apex, where the return map is well conditioned."""
    prob = small_column_3d(scheme=scheme, dt=1e-5, c=2000., psi=5.)
    for s, g, o in _run_both(prob, [1, 10, 50]):
        assert_parity(g, o, label=f"3D MC {scheme} step {s}")
        errs = mc_state_errors(g, o)
        assert np.array_equal(g["svars"][:, 0], o["svars"][:, 0]), "yield states differ"
        assert errs["pdstrain"] < 1e-9 and errs["epsilon"] < 1e-9, errs


@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_3d_cohesionless_mohr_coulomb_short_horizon(scheme):
    """The benchmark material (c = 0, psi = 0).  Near the free surface its
    points sit at the apex of the yield surface where the reference return map
    divides by a vanishing plastic gradient, so ulp-level differences grow
    quickly; parity is asserted over a short horizon."""
    prob = small_column_3d(scheme=scheme, dt=1e-5)
    for s, g, o in _run_both(prob, [1, 5]):
        assert_parity(g, o, label=f"3D MC c=0 {scheme} step {s}")


def test_2d_mohr_coulomb_usf():
    prob = small_column_2d(material="MohrCoulomb", E=1e6)
    for s, g, o in _run_both(prob, [1, 20, 60]):
        assert_parity(g, o, label=f"2D MC step {s}")


def _translating_block(dim, velocity, constrained=True):
    """A stress-free LinearElastic block in uniform motion without gravity:
    every particle translates rigidly, crossing cells."""
    if dim == 2:
        prob = P.column_2d(shape=(24, 16), block=(6, 6), E=5e5, scheme="usl", dt=2e-4)
        prob.analysis["gravity"] = (0.0, 0.0)
        shift = np.array([0.06, 0.05])
    else:
        prob = P.column_3d(shape=(12, 10, 10), block=(4, 4, 4), material="LinearElastic",
                           E=5e5, scheme="usl", dt=2e-4, geostatic=False)
        prob.analysis["gravity"] = (0.0, 0.0, 0.0)
        shift = np.array([0.03, 0.03, 0.04])
    pts, mid = prob.particles[0]
    prob.particles = [(pts + shift, mid)]
    if not constrained:
        prob.velocity_constraints = None
        prob.friction_constraints = None
    return prob, np.asarray(velocity, dtype=float)


@pytest.mark.parametrize("dim", [2, 3])
def test_cell_crossing_is_bit_exact(dim):
    """A block moving diagonally crosses many cell faces: cell ids stay
    bit-exact with the oracle through every crossing."""
    prob, vel = _translating_block(dim, [3.0, 1.5] if dim == 2 else [2.0, -1.5, 1.0])
    g = P.build_solver(prob)
    o = build_oracle(prob)
    st = o.get()
    st["v"] = np.tile(vel, (len(st["x"]), 1))
    g.load(dict(st))
    o.set(dict(st))
    c0 = g.read()["cell"]
    for _ in range(8):
        g.step(5)
        o.step(5)
        gg, oo = g.read(), o.get()
        # rigid motion: stress and strain are round-off noise (|sigma| ~ 1e-9 Pa
        # for E = 5e5 Pa), compared in absolute terms
        assert_parity(gg, oo, fields=("x", "u", "v", "F", "volume", "density", "mass"),
                      label="crossing")
        for f, tol in (("stress", 1e-6), ("strain", 1e-12)):
            assert np.abs(gg[f]).max() < tol and np.abs(oo[f]).max() < tol, f
    assert np.count_nonzero(gg["cell"] != c0) > len(c0) // 2


def _leaving_block():
    prob, vel = _translating_block(2, [0.0, -6.0], constrained=False)
    prob.analysis["dt"] = 1e-3
    pts, mid = prob.particles[0]
    prob.particles = [(pts - np.array([0.0, 0.045]), mid)]  # bottom rows near y = 0
    return prob, vel


def test_particles_leaving_the_mesh_are_removed_when_locate_is_off():
    prob, vel = _leaving_block()
    g = P.build_solver(prob, locate_particles=False)
    o = build_oracle(prob, locate_particles=False)
    st = o.get()
    st["v"] = np.tile(vel, (len(st["x"]), 1))
    g.load(dict(st))
    o.set(dict(st))
    g.step(2)
    o.step(2)
    gg, oo = g.read(), o.get()
    keep = gg["cell"] >= 0
    assert np.count_nonzero(~keep) > 0
    assert np.count_nonzero(keep) == len(oo["x"])
    for f in ("x", "v"):
        assert np.allclose(gg[f][keep], oo[f], rtol=0, atol=1e-12 * max(1.0, np.abs(oo[f]).max()))
    # rigid motion: stresses are round-off noise on both sides
    assert np.abs(gg["stress"][keep]).max() < 1e-6 and np.abs(oo["stress"]).max() < 1e-6


def test_particle_leaving_the_mesh_is_an_error_when_locate_is_on():
    from mpm_b200 import MPMError
    prob, vel = _leaving_block()
    g = P.build_solver(prob)
    st = g.read()
    st["v"] = np.tile(vel, (len(st["x"]), 1))
    g.load(st)
    with pytest.raises(MPMError) as e:
        g.step(2)
    assert e.value.code == -3


def test_3d_linear_elastic_usf_with_gravity_ramp_and_damping():
    prob = small_column_3d(material="LinearElastic", scheme="usf", dt=1e-5)
    for s, g, o in _run_both(prob, [1, 25], gravity_ramping_time=1e-4, damping_factor=0.05):
        assert_parity(g, o, label=f"3D LE ramp+damping step {s}")


def test_particle_velocity_constraint():
    prob = small_column_3d(material="LinearElastic", scheme="usl", dt=1e-5)
    top = np.argsort(prob.particles[0][0][:, 2])[-20:]
    prob.particle_velocity_constraints = [(top, 2, -0.05), (top[:5], 0, 0.01)]
    for s, g, o in _run_both(prob, [1, 30]):
        assert_parity(g, o, label=f"pvc step {s}")


@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_runs_are_bitwise_deterministic(scheme):
    """Two runs of the ill-conditioned cohesionless column give identical
    bits: the nodal sums have a fixed order."""
    prob = small_column_3d(scheme=scheme, dt=1e-5)
    a = P.build_solver(prob)
    b = P.build_solver(prob)
    a.step(30)
    b.step(30)
    ra, rb = a.read(), b.read()
    for f in ("cell", "x", "v", "stress", "svars"):
        assert np.array_equal(ra[f], rb[f]), f


def small_footing(**kw):
    base = dict(shape=(40, 10, 20), foundation=4, slope_height=8, slope_top=6, footing=(1, 5),
                dt=1e-5)
    base.update(kw)
    return P.footing_slope(**base)


@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_footing_on_slope_two_materials(scheme):
    """LinearElastic foundation + MohrCoulomb slope (c = 2 kPa) with a footing
    driven by a particle velocity constraint: two material slots, the
    constraint set, friction floor, 40 steps."""
    prob = small_footing(scheme=scheme)
    for s, g, o in _run_both(prob, [10, 40]):
        assert_parity(g, o, label=f"footing step {s}")
    fp = prob.particle_velocity_constraints[0][0]
    assert np.allclose(g["v"][fp, 2], -0.05)


@pytest.mark.parametrize("vupd", ["flip", "pic"])
def test_2d_linear_elastic_column_musl(vupd):
    """MUSL (mpm_scheme_musl.tcc): a second mapping of mass and momentum with
    the updated particle velocities before the stress update."""
    prob = small_column_2d(scheme="musl", velocity_update=vupd)
    for s, g, o in _run_both(prob, [1, 30, 100]):
        assert_parity(g, o, label=f"2D MUSL {vupd} step {s}")


def test_3d_mohr_coulomb_column_musl():
    prob = small_column_3d(scheme="musl", c=2000., psi=5.)
    for s, g, o in _run_both(prob, [1, 20, 50]):
        assert_parity(g, o, label=f"3D MUSL step {s}")
