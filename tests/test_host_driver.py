"""The C++ host driver (mpm_b200/_lib/mpm_gpu_run) reads the reference's input
format: mpm.json, mesh and particle files, particle stresses, velocity and
friction constraints, particle sets with particle velocity constraints.  On
the CPU it is checked in --parse-only mode; the GPU tests run it, compare the
particle HDF5 tables it writes (results/<uuid>/particles<step>.h5, as
MPMBase::write_outputs names them) with the Python API's run of the same
problem, and resume a run from one of them."""
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


def _table(d, prob, step):
    from mpm_b200 import h5
    return h5.read_table(os.path.join(d, "results", prob.name, f"particles{step:02d}.h5"))


@pytest.mark.gpu
def test_driver_run_equals_the_python_api_run(tmp_path):
    prob = _footing()
    steps = 25
    P.write_reference_input(prob, str(tmp_path), nsteps=steps, output_steps=10)
    r = _run_driver(str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert "Explicit solver duration" in r.stdout
    s = P.build_solver(prob)
    for step in (0, 10, 20):  # the start and every 10 steps; 25 is not a multiple
        if step:
            s.step(10)
        rec, ref = _table(str(tmp_path), prob, step), s.write_pod()
        assert len(rec) == len(ref) == prob.nparticles
        for name in pod.NAMES:
            assert np.array_equal(rec[name].astype(ref[name].dtype), ref[name]), (step, name)
    assert not os.path.exists(os.path.join(str(tmp_path), "results", prob.name, "particles25.h5"))


@pytest.mark.gpu
def test_driver_resumes_from_its_checkpoint(tmp_path):
    """analysis.resume (mpm_base.tcc:509-551): a run of 30 steps, and a run that
    resumes from the step-10 file, write the same step-30 table."""
    import json
    prob = _footing()
    d = str(tmp_path)
    P.write_reference_input(prob, d, nsteps=30, output_steps=10)
    r = _run_driver(d)
    assert r.returncode == 0, r.stderr
    full = _table(d, prob, 30)
    cfg = os.path.join(d, "mpm.json")
    js = json.load(open(cfg))
    js["analysis"]["resume"] = {"resume": True, "uuid": prob.name, "step": 10}
    js["analysis"]["uuid"] = "resumed"
    json.dump(js, open(cfg, "w"))
    os.remove(os.path.join(d, "results", prob.name, "particles30.h5"))
    r = _run_driver(d)
    assert r.returncode == 0, r.stderr
    assert "Checkpoint resume at step 10" in r.stdout
    again = _table(d, prob, 30)
    for name in pod.NAMES:
        assert np.array_equal(again[name], full[name]), name
