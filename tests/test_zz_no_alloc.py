"""The no-allocation constitutive update against the allocating one.

mpm_gpu_material_stress_batch_noalloc serves callers that cannot allocate device
memory (a plugin inside another program's memory arena, a real-time loop with a
fixed memory budget).  It stages the points in a fixed array of the library's
device image instead of allocating.  Here it is called twice in a row through
the C ABI and each result is compared with mpm_gpu_material_stress_batch on the
same input, within the FP64 parity tolerance of the other GPU tests; the first
call is also compared with the CPU oracle's material update, so a fault of the
shared kernel would not pass unseen.  The second call is smaller than the
first, so a result that depended on what the first call left in the shared
array would show up.  This file is collected last on purpose.
"""
import ctypes as C
import json

import numpy as np
import pytest

from mpm_b200 import _native
from mpm_b200 import problems as P
from mpm_b200.solver import material_stress_batch
from tests.parity import FP64_RTOL

pytestmark = pytest.mark.gpu

MAX_POINTS = 32768


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _noalloc(dim, mtype, props, stress, dstrain, density, state):
    L = _native.lib()
    n = stress.shape[0]
    stress = np.ascontiguousarray(stress, dtype=np.float64)
    dstrain = np.ascontiguousarray(dstrain, dtype=np.float64)
    density = np.ascontiguousarray(density, dtype=np.float64)
    st = np.array(state, dtype=np.float64).reshape(n, 9)
    out = np.zeros((n, 6))
    err = C.create_string_buffer(256)
    rc = L.mpm_gpu_material_stress_batch_noalloc(0, dim, mtype.encode(),
                                                 json.dumps(props).encode(), n, _dp(stress),
                                                 _dp(dstrain), _dp(density), _dp(st), _dp(out),
                                                 err, len(err))
    return rc, out, st, err.value.decode()


def _inputs(rng, n, dim):
    stress = rng.normal(-3000., 4000., (n, 6))
    dstrain = rng.normal(0., 4e-4, (n, 6))
    if dim == 2:
        stress[:, 4:] = 0.
        dstrain[:, [2, 4, 5]] = 0.
    return stress, dstrain, np.full(n, 1800.)


def _check(ref, got):
    scale = max(np.max(np.abs(ref)), 1e-300)
    assert np.max(np.abs(got - ref)) / scale <= FP64_RTOL


def test_no_alloc_matches_the_allocating_entry_point_on_two_calls():
    rng = np.random.default_rng(2026)
    # first call: 3D MohrCoulomb, a large batch (elastic, shear, tensile returns)
    mc = P.mohr_coulomb(1e7, 0.3, 1800., 30., 2000., 5., tension_cutoff=500.)
    from oracle import oracle as O
    st0 = np.tile(O.mc_initial_state(O.material_params("MohrCoulomb", mc)), (20000, 1))
    s1, d1, r1 = _inputs(rng, 20000, 3)
    ref1, ref_st1 = material_stress_batch(3, "MohrCoulomb3D", mc, s1, d1, r1, st0)
    rc, out1, st1, msg = _noalloc(3, "MohrCoulomb3D", mc, s1, d1, r1, st0)
    assert rc == 0, msg
    _check(ref1, out1)
    _check(ref_st1, st1)
    # the oracle's material update on a sample of the same points
    idx = np.arange(0, 20000, 40)
    ora = np.array([O.material_stress(3, "MohrCoulomb", mc, s1[i], d1[i], r1[i], st0[i])[0]
                    for i in idx])
    _check(ora, out1[idx])
    # second call: 2D LinearElastic, fewer points than the first call left behind
    le = P.linear_elastic(1e6, 0.3, 1800.)
    s2, d2, r2 = _inputs(rng, 777, 2)
    zeros = np.zeros((777, 9))
    ref2, _ = material_stress_batch(2, "LinearElastic2D", le, s2, d2, r2, zeros)
    rc, out2, st2, msg = _noalloc(2, "LinearElastic2D", le, s2, d2, r2, zeros)
    assert rc == 0, msg
    _check(ref2, out2)
    assert np.array_equal(st2, zeros)


def test_no_alloc_rejects_batches_above_its_maximum():
    le = P.linear_elastic(1e6, 0.3, 1800.)
    n = MAX_POINTS + 1
    z6 = np.zeros((n, 6))
    rc, _, _, msg = _noalloc(3, "LinearElastic3D", le, z6, z6, np.ones(n), np.zeros((n, 9)))
    assert rc == -1
    assert "maximum" in msg and str(MAX_POINTS) in msg
