"""The C++ host driver (mpm_b200/_lib/mpm_gpu_run) reads the reference's input
format: mpm.json, mesh and particle files, particle stresses, velocity and
friction constraints, particle sets with particle velocity constraints.  On
the CPU it is checked in --parse-only mode; the GPU test runs it and compares
its output records with the Python API's run of the same problem."""
import os
import subprocess

import numpy as np
import pytest

from mpm_b200 import build as B
from mpm_b200 import pod
from mpm_b200 import problems as P


def _footing():
    return P.footing_slope(shape=(40, 10, 20), foundation=4, slope_height=8, slope_top=6,
                           footing=(1, 5), dt=1e-5)


def _run_driver(d, *args):
    return subprocess.run([B.RUNNER, "-f", d, *args], capture_output=True, text=True, timeout=600)


def test_driver_parses_the_reference_input(tmp_path):
    prob = _footing()
    P.write_reference_input(prob, str(tmp_path), nsteps=7)
    r = _run_driver(str(tmp_path), "--parse-only")
    assert r.returncode == 0, r.stderr
    out = r.stdout
    for key, val in (("dim", 3), ("nodes", prob.nnodes), ("cells", prob.ncells),
                     ("particles", prob.nparticles), ("materials", 2), ("nsteps", 7),
                     ("particle_velocity_constraints", 1)):
        assert f"{key} {val} " in out + " ", (key, out)
    assert "scheme usl" in out and "stresses yes" in out


def test_driver_rejects_a_missing_file(tmp_path):
    prob = _footing()
    P.write_reference_input(prob, str(tmp_path), nsteps=7)
    os.remove(os.path.join(str(tmp_path), "mesh.txt"))
    r = _run_driver(str(tmp_path), "--parse-only")
    assert r.returncode != 0 and "mesh.txt" in r.stderr


@pytest.mark.gpu
def test_driver_run_equals_the_python_api_run(tmp_path):
    prob = _footing()
    steps = 25
    P.write_reference_input(prob, str(tmp_path), nsteps=steps)
    r = _run_driver(str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert "Explicit solver duration" in r.stdout
    path = os.path.join(str(tmp_path), "results", f"particles-{prob.name}-{steps}.pod")
    raw = open(path, "rb").read()
    assert raw[:8] == b"MPMPOD01"
    n = int(np.frombuffer(raw[8:16], dtype=np.int64)[0])
    rec = np.frombuffer(raw[16:], dtype=pod.POD_DTYPE, count=n)
    s = P.build_solver(prob)
    s.step(steps)
    ref = s.write_pod()
    assert n == len(ref) == prob.nparticles
    for name in pod.NAMES:
        assert np.array_equal(rec[name], ref[name]), name
