"""Long-horizon and full-size parity of the FP64 path against the oracle.

* The 2D LinearElastic USF column (100x50 quad4 cells of 0.01 m, 3,200
  particles, dt 1e-5) for its full 10,000 steps against the one-thread
  oracle: cells bit-exact, every field within FP64_RTOL at steps 1, 10, 100,
  1000 and 10000 (mpm_explicit.tcc:112-190, mpm_scheme_usf.tcc:9-12).
* The benchmark's cohesionless MohrCoulomb column (c = 0, psi = 0, K0 start)
  for 60 steps, every step: within FP64_RTOL for the first ten steps and
  while the problem's own floor (the oracle against itself with one ulp of
  input perturbation) stays at rounding level, and never further from the
  oracle than ten times that floor afterwards.
* The 3D column of the benchmark as written (200x100x50 hex8 mesh, the
  1.0x0.5x0.5 m block: 2,000,000 particles, USL, friction floor) for 1 and 10
  steps against the OpenMP oracle.
"""
import os

import numpy as np
import pytest

from mpm_b200 import problems as P
from tests.divergence import CURVE_FIELDS, envelope, gpu_vs_oracle, oracle_floor, running_max
from tests.parity import FP64_RTOL

pytestmark = pytest.mark.gpu


def _fmt(curve):
    return "\n".join(f"{r['step']:>6} " + " ".join(f"{f}={r['errors'][f]:.1e}" for f in CURVE_FIELDS)
                     for r in curve)


def test_config_a_full_10000_steps():
    prob = P.config_a()
    assert prob.nparticles == 3200 and prob.ncells == 5000
    curve = gpu_vs_oracle(prob, [1, 10, 100, 1000, 10000])
    for r in curve:
        assert r["cells_equal"], f"cells differ at step {r['step']}"
        bad = {f: e for f, e in r["errors"].items() if not e <= FP64_RTOL}
        assert not bad, f"step {r['step']}: {bad}\n{_fmt(curve)}"


def _cohesionless(scheme):
    return P.column_3d(shape=(12, 8, 10), block=(6, 4, 6), dt=1e-5, scheme=scheme)


@pytest.mark.parametrize("scheme", ["usl", "usf"])
def test_cohesionless_column_divergence_stays_within_its_conditioning(scheme):
    prob = _cohesionless(scheme)
    steps = list(range(1, 61))
    gpu = gpu_vs_oracle(prob, steps)
    floor = envelope([oracle_floor(prob, steps, field=f, direction=d)
                      for f in ("stress", "x") for d in (1, -1)])
    assert all(r["cells_equal"] for r in gpu), [r["step"] for r in gpu if not r["cells_equal"]]
    # the first ten steps, and every step at which all perturbed runs are
    # still at rounding level, within the FP64 parity tolerance
    quiet = [g for g, f in zip(gpu, floor) if max(f["errors"].values()) < 1e-12]
    for r in gpu[:10] + quiet:
        assert max(r["errors"].values()) <= FP64_RTOL, f"step {r['step']}\n{_fmt(gpu)}"
    # over the window, no field drifts further than ten times the floor
    gmax, fmax = running_max(gpu)[-1]["errors"], running_max(floor)[-1]["errors"]
    for f in CURVE_FIELDS:
        assert gmax[f] <= 10.0 * fmax[f] + FP64_RTOL, (
            f"{f}: {gmax[f]:.2e} vs floor {fmax[f]:.2e}\nGPU\n{_fmt(gpu)}\nfloor\n{_fmt(floor)}")


def test_benchmark_column_as_written_2m_particles():
    prob = P.config_b(block=(100, 50, 50))
    assert prob.nparticles == 2_000_000
    threads = os.cpu_count() or 1
    gpu = gpu_vs_oracle(prob, [1, 10], nthreads=threads)
    floor = oracle_floor(prob, [1, 10], nthreads=threads)
    for g, f in zip(gpu, floor):
        assert g["cells_equal"], f"cells differ at step {g['step']}"
        for k in CURVE_FIELDS:
            bound = max(FP64_RTOL, 10.0 * f["errors"][k])
            assert g["errors"][k] <= bound, (g["step"], k, g["errors"][k], f["errors"][k])
    assert max(gpu[0]["errors"].values()) <= FP64_RTOL, gpu[0]
