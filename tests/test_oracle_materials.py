"""Pin the oracle's constitutive models to the reference's own known answers.

The vectors in tests/golden/reference_kats.json are extracted from
tests/materials/mohr_coulomb_test.cc and tests/materials/linear_elastic_test.cc
of the reference by tests/golden/make_reference_kats.py; every record keeps the
reference file:line.  The comparison is the reference's own Catch v1.12
``Approx(x).epsilon(e)`` rule.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import catch_approx


def _mc_state(props, overrides):
    st = O.mc_initial_state(O.material_params("MohrCoulomb", props))
    for k, v in overrides.items():
        st[O.MC_STATE.index(k)] = v
    return st


def _trial(props, stress, dstrain):
    E, nu = props["youngs_modulus"], props["poisson_ratio"]
    K = E / (3 * (1 - 2 * nu))
    G = E / (2 * (1 + nu))
    a1, a2 = K + 4.0 / 3.0 * G, K - 2.0 / 3.0 * G
    De = np.zeros((6, 6))
    De[:3, :3] = a2
    for i in range(3):
        De[i, i] = a1
    De[3, 3] = De[4, 4] = De[5, 5] = G
    return np.asarray(stress) + De @ np.asarray(dstrain)


def test_kat_counts(kats):
    assert len(kats["mohr_coulomb_stress"]) == 22
    assert len(kats["mohr_coulomb_diagnostics"]) >= 40
    assert len(kats["linear_elastic_stress"]) == 4


def test_mohr_coulomb_compute_stress(kats):
    """mohr_coulomb.tcc:348-513 against every compute_stress KAT."""
    for r in kats["mohr_coulomb_stress"]:
        props = r["material"]
        st = _mc_state(props, r["state"])
        density = props["density"] / (1.0 + r["dvolumetric_strain"])
        out, st2 = O.material_stress(r["dim"], "MohrCoulomb", props, r["stress"], r["dstrain"],
                                     density, st)
        for i in range(6):
            assert catch_approx(out[i], r["expected_stress"][i], r["epsilon"]), (r["source"], i)
        if r["expected_pdstrain"] is not None:
            assert catch_approx(st2[8], r["expected_pdstrain"], r["epsilon"]), r["source"]


def test_mohr_coulomb_invariants_yield_and_gradients(kats):
    """mohr_coulomb.tcc:124-344 (invariants, yield state, dF/dsigma, dP/dsigma)."""
    n = 0
    for r in kats["mohr_coulomb_diagnostics"]:
        props = r["material"]
        st = _mc_state(props, r["state"])
        sig = r["stress"] if r["at"] == "stress" else _trial(props, r["stress"], r["dstrain"])
        dg = O.mc_diagnostics(r["dim"], props, sig, st)
        for name, (val, tol, line) in r["checks"].items():
            if name.startswith("df_dsigma"):
                got = dg["df_dsigma"][int(name[-1])]
            elif name.startswith("dp_dsigma"):
                got = dg["dp_dsigma"][int(name[-1])]
            else:
                got = dg[name]
            assert catch_approx(got, val, tol), (r["source"], name, line, got, val)
            n += 1
    assert n > 400


def test_linear_elastic_compute_stress(kats):
    """linear_elastic.tcc:73-94 against the reference's stress KATs."""
    for r in kats["linear_elastic_stress"]:
        out, _ = O.material_stress(r["dim"], "LinearElastic", r["material"], r["stress"],
                                   r["dstrain"], r["material"]["density"])
        for i in range(6):
            assert catch_approx(out[i], r["expected_stress"][i], r["epsilon"]), (r["source"], i)


def test_oracle_plants_a_mistake_and_the_kat_catches_it(kats):
    """A wrong elastic modulus must fail the LinearElastic KAT (checks the checker)."""
    r = kats["linear_elastic_stress"][0]
    props = dict(r["material"])
    props["youngs_modulus"] *= 1.0 + 1e-5
    out, _ = O.material_stress(r["dim"], "LinearElastic", props, r["stress"], r["dstrain"],
                               props["density"])
    assert not all(catch_approx(out[i], r["expected_stress"][i], r["epsilon"]) for i in range(6))


@pytest.mark.parametrize("dim", [2, 3])
def test_mohr_coulomb_initial_state(dim):
    """mohr_coulomb.tcc:85-111: cohesion 0 gives a tension cutoff of 1e-15."""
    props = dict(density=1800., youngs_modulus=1e7, poisson_ratio=0.3, softening=False,
                 friction=30., dilation=0., cohesion=0., residual_friction=30.,
                 residual_dilation=0., residual_cohesion=0., peak_pdstrain=0.,
                 residual_pdstrain=0., tension_cutoff=0.)
    st = O.mc_initial_state(O.material_params("MohrCoulomb", props))
    assert st[4] == 1e-15
    assert st[1] == 30. * np.pi / 180.
