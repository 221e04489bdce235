"""Batched ensemble of independent 2D slopes in one solver (through the C ABI).

Each run of the ensemble must evolve as it does alone in its own grid: the
packing shares no node between runs, so the only differences are the
rounding of positions offset by the run's origin in the common grid.
"""
import numpy as np
import pytest

from mpm_b200 import ensemble as E
from mpm_b200 import problems as P
from oracle.oracle import build_oracle
from tests.parity import assert_parity, field_errors

pytestmark = pytest.mark.gpu


def _small_runs():
    return [E.SlopeRun(height=6, width=6, phi=30.0, cohesion=2000.0, margin=6, seed=11),
            E.SlopeRun(height=4, width=5, phi=25.0, cohesion=3000.0, margin=6, seed=12),
            E.SlopeRun(height=8, width=4, phi=38.0, cohesion=1500.0, margin=6, seed=13)]


def test_each_run_evolves_as_it_does_alone():
    runs = _small_runs()
    ens = E.Ensemble(runs, precision="fp64")
    ens.step(40)
    together = ens.run_states()
    for r, run in enumerate(runs):
        alone = P.build_solver(E.standalone_problem(run), precision="fp64")
        alone.step(40)
        st = alone.read()
        errs = field_errors(together[r], st, ("x", "u", "v", "stress", "strain", "volume"))
        assert all(v <= 1e-9 for v in errs.values()), (r, errs)


def test_ensemble_matches_the_oracle():
    prob, _ = E.ensemble_problem(_small_runs())
    g = P.build_solver(prob, precision="fp64")
    o = build_oracle(prob)
    g.step(20)
    o.step(20)
    assert_parity(g.read(), o.get(), label="ensemble")


def test_mixed_ensemble_runout_matches_fp64():
    runs = E.random_runs(12, n_min=300, n_max=1500, seed=5)
    out = {}
    for prec in ("fp64", "mixed"):
        ens = E.Ensemble(runs, precision=prec)
        ens.step(300)
        out[prec] = ens.runout()
    assert np.all(np.isfinite(out["fp64"]))
    assert np.max(np.abs(out["mixed"] - out["fp64"]) / out["fp64"]) <= 1e-6


def test_graph_replayed_steps_equal_eager_steps():
    """Steps replayed from the captured CUDA graph give the bitwise state of
    eagerly launched steps (profiling forces eager launches)."""
    prob, _ = E.ensemble_problem(_small_runs())
    a = P.build_solver(prob, precision="mixed")
    b = P.build_solver(prob, precision="mixed")
    a.step(30)
    b.set_profiling(True)
    b.step(30)
    A, B = a.read(), b.read()
    for k in A:
        assert np.array_equal(A[k], B[k]), k
