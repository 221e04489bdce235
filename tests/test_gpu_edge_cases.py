"""Edge cases of the particle set: no particles at all, and every particle gone.

The reference removes particles that leave the mesh when locating is off
(mesh.tcc:1099-1151, locate_particles_mesh) and keeps stepping with whatever
remains, down to an empty set; a state can also be replaced by one without
particles (read_particles_hdf5 of an empty table).  Both must step and read back
without error, on the FP64 and the mixed path.
"""
import numpy as np
import pytest

from mpm_b200 import problems as P
from tests.test_gpu_parity import _leaving_block, small_column_3d

pytestmark = pytest.mark.gpu

FIELDS = ("x", "u", "v", "stress", "strain", "F", "volume", "mass", "density", "cell",
          "material", "svars")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_particle_leaves_the_mesh(precision):
    prob, vel = _leaving_block()
    s = P.build_solver(prob, precision=precision, locate_particles=False)
    st = s.read()
    st["v"] = np.tile(vel, (len(st["x"]), 1))
    s.load(st)
    for _ in range(40):
        s.step(5)
        if np.all(s.read()["cell"] < 0):
            break
    gone = s.read()
    assert np.all(gone["cell"] < 0), "some particles never left the mesh"
    assert s.nparticles == len(st["x"])  # removed rows stay, marked by cell -1
    # nothing moves a removed particle, and further steps are not an error
    s.step(10)
    after = s.read()
    for k in FIELDS:
        assert np.array_equal(after[k], gone[k]), k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_state_without_particles(precision):
    s = P.build_solver(small_column_3d(scheme="usl", dt=1e-5, c=2000., psi=5.), precision=precision)
    s.step(2)
    empty = {k: v[:0] for k, v in s.read().items()}
    s.load(empty)
    assert s.nparticles == 0
    s.step(3)
    out = s.read()
    for k in FIELDS:
        assert len(out[k]) == 0, k
    # a full state loaded after the empty one steps as in a solver that never
    # held the empty state
    make = lambda: P.build_solver(small_column_3d(scheme="usl", dt=1e-5, c=2000., psi=5.),
                                  precision=precision)
    src = make()
    src.step(2)
    st = src.read()
    fresh = make()
    for solver in (s, fresh):
        solver.load(st)
        solver.step(1)
    a, b = s.read(), fresh.read()
    for k in FIELDS:
        assert np.array_equal(a[k], b[k]), k
