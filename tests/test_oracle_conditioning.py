"""The benchmark material (MohrCoulomb, c = 0, psi = 0) in the oracle alone.

1. At zero stress the reference's plastic corrector divides zero by zero
   (mohr_coulomb.tcc:139-191 yield state at the apex; :290-313 the flow-rule
   gradient, whose deviatoric and volumetric parts vanish there for psi = 0;
   :453-455 the plastic multiplier's denominator df/dsigma . De . dp/dsigma),
   so a tensile or shear increment from zero stress gives NaN.  A column
   started from zero stress, as the benchmark text reads, turns NaN on its
   first step; started from a K0 geostatic stress it does not.  This is why
   the generated inputs start MohrCoulomb columns from K0.
2. The c = 0 column is ill-conditioned: one ulp in the initial stress grows to
   visible differences within tens of steps (yield-branch decisions near the
   apex flip), while a cohesive column stays at rounding level.  The CUDA
   path's long-horizon divergence from the oracle is judged against this.
"""
import numpy as np

from mpm_b200 import problems as P
from oracle import oracle as O
from oracle.oracle import build_oracle
from tests.divergence import oracle_floor

CHECK = [10, 30, 60]


def _column(**kw):
    base = dict(shape=(12, 8, 10), block=(6, 4, 6), dt=1e-5)
    base.update(kw)
    return P.column_3d(**base)


def test_apex_return_from_zero_stress_is_nan():
    props = P.mohr_coulomb(1e7, 0.3, 1800., 30., 0., 0.)
    st0 = O.mc_initial_state(O.material_params("MohrCoulomb", props))
    assert st0[4] == 1e-15  # tension cutoff floored at the apex (mohr_coulomb.tcc:97-100)
    zero = np.zeros(6)
    # extension: tensile return (yield state 1 or 2), 0 / 0
    out, st = O.material_stress(3, "MohrCoulomb", props, zero, np.array([1e-6, 0, 0, 0, 0, 0]),
                                1800., st0)
    assert np.all(np.isnan(out)) and st[0] != 0
    # pure shear: shear return, 0 / 0
    out, st = O.material_stress(3, "MohrCoulomb", props, zero, np.array([0, 0, 0, 1e-6, 0, 0]),
                                1800., st0)
    assert np.all(np.isnan(out)) and st[0] != 0
    # isotropic compression stays elastic and finite
    out, st = O.material_stress(3, "MohrCoulomb", props, zero, np.full(6, -1e-6) * [1, 1, 1, 0, 0, 0],
                                1800., st0)
    assert np.all(np.isfinite(out)) and st[0] == 0


def test_cohesionless_column_from_zero_stress_turns_nan_in_one_step():
    o = build_oracle(_column(geostatic=False))
    o.step(1)
    bad = ~np.isfinite(o.get()["stress"]).all(axis=1)
    assert bad.sum() > o.nparticles // 2, bad.sum()
    o = build_oracle(_column())
    o.step(1)
    assert np.isfinite(o.get()["stress"]).all()


def test_cohesionless_column_is_ill_conditioned():
    """One ulp of initial stress: the c = 0 column drifts beyond 1e-6 in stress
    within 60 steps; the c = 2 kPa, psi = 5 column stays below 1e-10."""
    c0 = oracle_floor(_column(), CHECK)
    assert c0[0]["errors"]["stress"] < 1e-12
    assert c0[-1]["errors"]["stress"] > 1e-6, c0[-1]
    assert all(r["cells_equal"] for r in c0)
    cc = oracle_floor(_column(c=2000., psi=5.), CHECK)
    assert all(max(r["errors"].values()) < 1e-10 for r in cc), cc
