"""Loading and reading a particle state (mpm_gpu_load_particles,
mpm_gpu_read_particles).

A load that gives every field converts the caller's rows on the device; a load
that leaves fields out fills them on the host (zero displacement, the
material's density, mass = volume x density, the MohrCoulomb initial state).
Both must write the same device state, and read-back must return the loaded
values: bitwise in FP64, and in the mixed path the FP32 rounding of each field
(x, u and pdstrain stay FP64).
"""
import numpy as np
import pytest

from mpm_b200 import problems as P
from tests.test_gpu_parity import small_column_2d, small_column_3d

pytestmark = pytest.mark.gpu

FIELDS = ("x", "u", "v", "stress", "strain", "F", "volume", "mass", "density", "cell",
          "material", "svars")


def _stepped(dim, precision):
    prob = small_column_2d(scheme="usl") if dim == 2 else \
        small_column_3d(scheme="usl", dt=1e-5, c=2000., psi=5.)
    s = P.build_solver(prob, precision=precision)
    s.step(20)
    return s


def _same(a, b, label):
    for k in FIELDS:
        assert np.array_equal(a[k], b[k]), f"{label}: {k} differs"


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("dim", [2, 3])
def test_full_and_partial_loads_write_the_same_state(dim, precision):
    s = _stepped(dim, precision)
    st = s.read()
    st["u"] = np.zeros_like(st["u"])  # the value a partial load gives
    s.load(st)
    full = s.read()
    s.load({k: v for k, v in st.items() if k != "u"})
    partial = s.read()
    _same(full, partial, f"{dim}D {precision}")
    # and the two loads step alike
    s.load(st)
    s.step(5)
    a = s.read()
    s.load({k: v for k, v in st.items() if k != "u"})
    s.step(5)
    _same(a, s.read(), f"{dim}D {precision} after 5 steps")


@pytest.mark.parametrize("dim", [2, 3])
def test_fp64_read_returns_the_loaded_state(dim):
    s = _stepped(dim, "fp64")
    st = s.read()
    rng = np.random.default_rng(5)
    st["v"] = st["v"] + rng.standard_normal(st["v"].shape)
    s.load(st)
    _same(s.read(), st, f"{dim}D round trip")


@pytest.mark.parametrize("dim", [2, 3])
def test_mixed_read_returns_the_fp32_rounding(dim):
    s = _stepped(dim, "mixed")
    st = s.read()
    rng = np.random.default_rng(6)
    st["v"] = st["v"] + rng.standard_normal(st["v"].shape)
    s.load(st)
    back = s.read()
    for k in ("x", "u", "cell", "material"):
        assert np.array_equal(back[k], st[k]), k
    for k in ("v", "stress", "strain", "volume", "mass", "density"):
        assert np.array_equal(back[k], st[k].astype(np.float32).astype(np.float64)), k
    F = st["F"].copy()
    eye = np.eye(3).ravel() if dim == 3 else np.array([1, 0, 0, 0, 1, 0, 0, 0, 0.])
    h = (F - eye).astype(np.float32).astype(np.float64) + eye
    if dim == 2:
        h[:, 8] = 1.
    assert np.array_equal(back["F"], h)
    if dim == 3:  # MohrCoulomb: the state in FP32, pdstrain in FP64
        sv = st["svars"].astype(np.float32).astype(np.float64)
        sv[:, 8] = st["svars"][:, 8]
        assert np.array_equal(back["svars"], sv)


def test_read_of_a_subset_of_fields():
    """Arrays left out of the read are not written; the others are as in a full read."""
    from mpm_b200 import _native
    import ctypes as C
    s = _stepped(3, "fp64")
    full = s.read()
    n = s.nparticles
    stress = np.full((n, 6), np.nan)
    mass = np.full(n, np.nan)
    Pt = _native.Particles()
    Pt.stress = stress.ctypes.data_as(C.POINTER(C.c_double))
    Pt.mass = mass.ctypes.data_as(C.POINTER(C.c_double))
    assert s.L.mpm_gpu_read_particles(s.h, C.byref(Pt)) == 0
    assert np.array_equal(stress, full["stress"])
    assert np.array_equal(mass, full["mass"])


def test_2d_load_rejects_out_of_plane_components():
    s = _stepped(2, "fp64")
    st = s.read()
    st["stress"][3, 4] = 1.0
    with pytest.raises(RuntimeError, match="zero yz and xz"):
        s.load(st)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_state_larger_than_one_copy_chunk(precision):
    """512,000 particles: the staged rows (42 doubles a particle) span three
    64 MiB chunks of the pinned copy pipeline in each direction."""
    prob = P.column_3d(shape=(80, 80, 40), block=(40, 40, 40))
    s = P.build_solver(prob, precision=precision)
    s.step(2)
    st = s.read()
    assert len(st["x"]) * 42 * 8 > 2 * (64 << 20)
    s.load(st)
    back = s.read()
    for k in ("x", "u", "v", "stress", "strain", "mass", "cell", "material", "svars"):
        assert np.array_equal(back[k], st[k]), k
    for k in ("volume", "density"):  # mixed: read as V0 (1 + P), loaded in FP32
        want = st[k] if precision == "fp64" else st[k].astype(np.float32).astype(np.float64)
        assert np.array_equal(back[k], want), k
    if precision == "fp64":
        assert np.array_equal(back["F"], st["F"])
    # a subset read: the arrays' offsets in the staged rows shift
    from mpm_b200 import _native
    import ctypes as C
    n = s.nparticles
    svars = np.full((n, 9), np.nan)
    density = np.full(n, np.nan)
    Pt = _native.Particles()
    Pt.svars = svars.ctypes.data_as(C.POINTER(C.c_double))
    Pt.density = density.ctypes.data_as(C.POINTER(C.c_double))
    assert s.L.mpm_gpu_read_particles(s.h, C.byref(Pt)) == 0
    assert np.array_equal(svars, back["svars"]) and np.array_equal(density, back["density"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_page_locked_arrays_load_and_read_as_pageable_ones(precision):
    """Arrays in page-locked memory (pinned_empty) are copied by DMA directly,
    pageable ones through the staging pipeline: the same state either way,
    and a read into page-locked arrays equals the plain read."""
    from mpm_b200 import pinned_empty
    prob = P.column_3d(shape=(80, 80, 40), block=(40, 40, 40))
    s = P.build_solver(prob, precision=precision)
    s.step(3)
    ref = s.read()
    pin = s.state_buffers(pinned=True)
    got = s.read(out=pin)
    for k in ref:
        assert np.array_equal(got[k], ref[k]), k
    s.load(ref)  # the step-3 state from pageable arrays ...
    s.step(2)
    after_pageable = s.read()
    s.load(pin)  # ... and from page-locked ones
    s.step(2)
    after_pinned = s.read(out=s.state_buffers(pinned=True))
    for k in after_pageable:
        assert np.array_equal(after_pinned[k], after_pageable[k]), k
    a = pinned_empty((5, 3))
    assert a.shape == (5, 3) and a.dtype == np.float64
