"""PODParticle records (particle output and checkpoint resume) through the C ABI.

mpm_gpu_write_pod packs Particle::pod (particle.tcc:180-306) on the device into
the caller's record layout; mpm_gpu_load_pod is the checkpoint resume of
MPMBase::checkpoint_resume / Mesh::read_particles_hdf5.  The records must hold
exactly the state the solver reads back, and a run resumed from them must
continue as the uninterrupted run does.
"""
import numpy as np
import pytest

from mpm_b200 import pod
from mpm_b200 import problems as P
from mpm_b200._native import MPMError

pytestmark = pytest.mark.gpu


def _vec(rec, name, dim):
    return np.stack([rec[f"{name}_{c}"] for c in "xyz"[:dim]], axis=1)


def _check_records(rec, st, dim, nsize):
    n = len(st["x"])
    assert len(rec) == n
    assert np.array_equal(rec["id"], np.arange(n, dtype=np.uint64))
    assert np.array_equal(_vec(rec, "coord", dim), st["x"][:, :dim])
    assert np.array_equal(_vec(rec, "displacement", dim), st["u"][:, :dim])
    assert np.array_equal(_vec(rec, "velocity", dim), st["v"][:, :dim])
    if dim == 2:
        for c in "z":
            assert not np.any(rec[f"coord_{c}"]) and not np.any(rec[f"velocity_{c}"])
    assert np.array_equal(_vec(rec, "nsize", dim), np.full((n, dim), nsize))
    assert not np.any(_vec(rec, "acceleration", 3))
    stress = np.stack([rec[k] for k in ("stress_xx", "stress_yy", "stress_zz", "tau_xy", "tau_yz",
                                        "tau_xz")], axis=1)
    strain = np.stack([rec[k] for k in ("strain_xx", "strain_yy", "strain_zz", "gamma_xy",
                                        "gamma_yz", "gamma_xz")], axis=1)
    F = np.stack([rec[f"defgrad_{i}{j}"] for i in range(3) for j in range(3)], axis=1)
    assert np.array_equal(stress, st["stress"])
    assert np.array_equal(strain, st["strain"])
    assert np.array_equal(F, st["F"])
    for k in ("mass", "volume"):
        assert np.array_equal(rec[k], st[k])
    assert not np.any(rec["pressure"])
    assert not np.any(rec["initialise_mapping_matrix"])
    assert not np.any(np.stack([rec[f"mapping_matrix_{i}{j}"] for i in range(3) for j in range(3)]))
    assert np.all(rec["status"])
    assert np.array_equal(rec["cell_id"], st["cell"].astype(np.uint64))
    assert np.array_equal(rec["material_id"], st["material"].astype(np.uint32))
    sv = np.stack([rec[f"svars_{k}"] for k in range(20)], axis=1)
    return sv


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_records_hold_the_particle_state_3d_mohr_coulomb(precision):
    prob = P.column_3d(shape=(12, 6, 8), block=(6, 6, 8))
    s = P.build_solver(prob, precision=precision)
    s.step(20)
    rec = s.write_pod()
    st = s.read()
    sv = _check_records(rec, st, 3, 2.0 / 8 ** (1 / 3))
    assert np.all(rec["nstate_vars"] == 9)
    assert np.array_equal(sv[:, :9], st["svars"])
    assert not np.any(sv[:, 9:])


def test_records_hold_the_particle_state_2d_linear_elastic():
    prob = P.column_2d(shape=(20, 20), block=(8, 10))
    s = P.build_solver(prob)
    s.step(30)
    rec = s.write_pod()
    sv = _check_records(rec, s.read(), 2, 2.0 / 4 ** 0.5)
    assert np.all(rec["nstate_vars"] == 0)
    assert not np.any(sv)


def test_records_follow_the_callers_layout():
    """A layout with a leading 8-byte slot (as a C++ struct with a vtable
    pointer has) and different field order in memory; bytes outside the fields
    are left as they were."""
    prob = P.column_3d(shape=(8, 4, 4), block=(4, 4, 4))
    s = P.build_solver(prob)
    s.step(5)
    names = pod.NAMES
    # reversed order of the doubles, an 8-byte hole in front, natural alignment
    fields = [("hole", np.uint64)] + [(n, pod.POD_DTYPE.fields[n][0]) for n in reversed(names)]
    dt = np.dtype(fields, align=True)
    out = np.zeros(s.nparticles, dtype=dt)
    out["hole"] = 0xDEADBEEFCAFEF00D
    size, offs, sizes = pod.layout(dt)
    import ctypes as C
    n = C.c_int64()
    psz = C.POINTER(C.c_size_t)
    rc = s.L.mpm_gpu_write_pod(s.h, out.ctypes.data_as(C.c_void_p), len(out), C.byref(n), size,
                               offs.ctypes.data_as(psz), sizes.ctypes.data_as(psz), 74)
    assert rc == 0 and n.value == len(out)
    assert np.all(out["hole"] == 0xDEADBEEFCAFEF00D)
    ref = s.write_pod()
    for k in names:
        assert np.array_equal(out[k], ref[k]), k


def test_layout_errors_are_reported():
    prob = P.column_3d(shape=(8, 4, 4), block=(4, 4, 4))
    s = P.build_solver(prob)
    size, offs, sizes = pod.layout()
    import ctypes as C
    psz = C.POINTER(C.c_size_t)
    buf = np.zeros(s.nparticles, dtype=pod.POD_DTYPE)
    n = C.c_int64()
    bad = offs.copy()
    bad[1] += 4  # a double at a 4-byte offset
    rc = s.L.mpm_gpu_write_pod(s.h, buf.ctypes.data_as(C.c_void_p), len(buf), C.byref(n), size,
                               bad.ctypes.data_as(psz), sizes.ctypes.data_as(psz), 74)
    assert rc == -1 and b"misaligned" in s.L.mpm_gpu_last_error(s.h)
    rc = s.L.mpm_gpu_write_pod(s.h, buf.ctypes.data_as(C.c_void_p), 3, C.byref(n), size,
                               offs.ctypes.data_as(psz), sizes.ctypes.data_as(psz), 74)
    assert rc == -1 and n.value == s.nparticles
    rc = s.L.mpm_gpu_write_pod(s.h, buf.ctypes.data_as(C.c_void_p), len(buf), C.byref(n), size,
                               offs.ctypes.data_as(psz), sizes.ctypes.data_as(psz), 73)
    assert rc == -1


@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_resume_continues_the_run(scheme):
    """Checkpoint at step 15, resume in a new solver, run to step 30: the same
    state as the uninterrupted run.  Density is recomputed as mass / volume on
    resume (particle.tcc:46-47), so it may differ in the last bits; it enters
    the MohrCoulomb update only through the separated-state test."""
    prob = P.column_3d(shape=(12, 6, 8), block=(6, 6, 8), scheme=scheme)
    a = P.build_solver(prob)
    a.step(15)
    rec = a.write_pod()
    a.step(15)
    A = a.read()
    b = P.build_solver(prob, with_particles=False)
    b.load_pod(rec)
    b.set_current_step(15)
    b.step(15)
    B = b.read()
    assert b.current_step == 30
    for k in ("x", "u", "v", "stress", "strain", "F", "volume", "mass", "svars", "cell",
              "material"):
        assert np.array_equal(A[k], B[k]), k
    assert np.max(np.abs(A["density"] - B["density"]) / A["density"]) < 1e-14
    assert np.array_equal(b.write_pod()["nsize_x"], rec["nsize_x"])


def test_resume_rejects_particles_outside_the_mesh():
    prob = P.column_3d(shape=(8, 4, 4), block=(4, 4, 4))
    a = P.build_solver(prob)
    rec = a.write_pod()
    rec["coord_x"][5] = 100.0
    b = P.build_solver(prob, with_particles=False)
    with pytest.raises(MPMError, match="outside the mesh"):
        b.load_pod(rec)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_hdf5_table_holds_the_records(tmp_path, precision):
    """Mesh::write_particles_hdf5's table: the records write_pod gives."""
    from mpm_b200 import h5
    prob = P.column_3d(shape=(12, 6, 8), block=(6, 6, 8), scheme="usl")
    a = P.build_solver(prob, precision=precision)
    a.step(7)
    path = tmp_path / "particles07.h5"
    a.write_hdf5(path)
    rec = h5.read_table(path)
    ref = a.write_pod()
    assert len(rec) == len(ref) == prob.nparticles
    for name in ref.dtype.names:
        assert np.array_equal(rec[name].astype(ref[name].dtype), ref[name]), name


def test_hdf5_checkpoint_resumes_the_run(tmp_path):
    """The HDF5 particle table as the checkpoint (Mesh::read_particles_hdf5,
    MPMBase::checkpoint_resume): written at step 15, resumed in a new solver,
    the run reaches step 30 as the uninterrupted one (density to 1e-14,
    recomputed as mass / volume)."""
    prob = P.column_3d(shape=(12, 6, 8), block=(6, 6, 8), scheme="usl")
    precision = "fp64"
    a = P.build_solver(prob, precision=precision)
    a.step(15)
    path = tmp_path / "particles15.h5"
    a.write_hdf5(path)
    a.step(15)
    A = a.read()
    b = P.build_solver(prob, precision=precision, with_particles=False)
    b.load_hdf5(path)
    b.set_current_step(15)
    b.step(15)
    B = b.read()
    for k in ("x", "u", "v", "stress", "strain", "F", "volume", "mass", "svars", "cell",
              "material"):
        assert np.array_equal(A[k], B[k]), k
    assert np.max(np.abs(A["density"] - B["density"]) / A["density"]) < 1e-14
