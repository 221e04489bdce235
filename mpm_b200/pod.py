"""PODParticle records: the reference's particle output / checkpoint row.

Field names, order and types follow pod_particle.h:12-62 and the field table
of pod_particle.cc (74 fields).  ``POD_DTYPE`` lays them out as a C compiler
lays out the struct's data members (natural alignment); the C ABI takes any
layout through per-field offsets, so a C++ caller passes the reference's own
``pod::particle::dst_offset`` / ``dst_sizes`` instead.
"""
import numpy as np

_VEC = lambda p: [f"{p}_x", f"{p}_y", f"{p}_z"]  # noqa: E731

FIELDS = (
    [("id", np.uint64), ("mass", np.float64), ("volume", np.float64), ("pressure", np.float64)]
    + [(n, np.float64) for n in _VEC("coord") + _VEC("displacement") + _VEC("nsize")
       + _VEC("velocity") + _VEC("acceleration")]
    + [(n, np.float64) for n in ("stress_xx", "stress_yy", "stress_zz", "tau_xy", "tau_yz",
                                 "tau_xz", "strain_xx", "strain_yy", "strain_zz", "gamma_xy",
                                 "gamma_yz", "gamma_xz")]
    + [(f"defgrad_{i}{j}", np.float64) for i in range(3) for j in range(3)]
    + [("initialise_mapping_matrix", np.bool_)]
    + [(f"mapping_matrix_{i}{j}", np.float64) for i in range(3) for j in range(3)]
    + [("status", np.bool_), ("cell_id", np.uint64), ("material_id", np.uint32),
       ("nstate_vars", np.uint32)]
    + [(f"svars_{k}", np.float64) for k in range(20)]
)
assert len(FIELDS) == 74

POD_DTYPE = np.dtype(FIELDS, align=True)
NAMES = [n for n, _ in FIELDS]


def layout(dtype=POD_DTYPE):
    """(record_size, offsets, sizes) of a structured dtype with the 74 fields."""
    offs = np.array([dtype.fields[n][1] for n in NAMES], dtype=np.uintp)
    sizes = np.array([dtype.fields[n][0].itemsize for n in NAMES], dtype=np.uintp)
    return dtype.itemsize, offs, sizes
