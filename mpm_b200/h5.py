"""The reference's HDF5 particle table as numpy records.

``REFERENCE_POD_DTYPE`` is PODParticle as the reference's compiler lays it out
(pod_particle.h:12-62: a vtable pointer first, then the data members at
natural alignment, 592 bytes), with the HDF5 field types of pod_particle.cc:
id and cell_id signed 64-bit, the two flags unsigned 8-bit, material_id and
nstate_vars unsigned 32-bit, the rest IEEE doubles.  ``write_table`` /
``read_table`` go through the library's own HDF5 encoder and decoder
(libmpm_b200.so: mpm_h5_write_table / mpm_h5_read_table).
"""
import ctypes as C

import numpy as np

from . import _native
from .pod import NAMES

F64, I64, U64, I32, U32, U8 = 0, 1, 2, 3, 4, 5
_NP = {F64: np.float64, I64: np.int64, U64: np.uint64, I32: np.int32, U32: np.uint32, U8: np.uint8}


def _reference_fields():
    out, off = [], 8  # the vtable pointer
    for n in NAMES:
        if n in ("id", "cell_id"):
            t = I64
        elif n in ("initialise_mapping_matrix", "status"):
            t = U8
        elif n in ("material_id", "nstate_vars"):
            t = U32
        else:
            t = F64
        size = np.dtype(_NP[t]).itemsize
        off = (off + size - 1) // size * size
        out.append((n, t, off))
        off += size
    return out


REFERENCE_FIELDS = _reference_fields()
REFERENCE_POD_DTYPE = np.dtype({"names": [n for n, _, _ in REFERENCE_FIELDS],
                                "formats": [_NP[t] for _, t, _ in REFERENCE_FIELDS],
                                "offsets": [o for _, _, o in REFERENCE_FIELDS],
                                "itemsize": 592})


def _field_args(dtype):
    names = [n for n in dtype.names]
    cn = (C.c_char_p * len(names))(*[n.encode() for n in names])
    offs = np.array([dtype.fields[n][1] for n in names], dtype=np.uintp)
    code = {np.dtype(v): k for k, v in _NP.items()}
    types = np.array([code[np.dtype(dtype.fields[n][0])] for n in names], dtype=np.int32)
    return names, cn, offs, types


def write_table(path, records, title="Table Title", chunk_records=10000):
    """Write a structured array as an HDF5 table (H5TBmake_table's structure)."""
    records = np.ascontiguousarray(records)
    names, cn, offs, types = _field_args(records.dtype)
    rc = _native.lib().mpm_h5_write_table(
        str(path).encode(), title.encode(), len(records), records.dtype.itemsize, len(names), cn,
        offs.ctypes.data_as(C.POINTER(C.c_size_t)), types.ctypes.data_as(C.POINTER(C.c_int32)),
        records.ctypes.data_as(C.c_void_p), chunk_records)
    if rc != 0:
        raise _native.MPMError(rc, f"cannot write {path}")


def read_table(path, dtype=REFERENCE_POD_DTYPE):
    """Read the table's fields named in ``dtype`` into a structured array."""
    names, cn, offs, types = _field_args(dtype)
    L = _native.lib()
    n = C.c_int64()
    err = C.create_string_buffer(256)
    args = (len(names), cn, offs.ctypes.data_as(C.POINTER(C.c_size_t)),
            types.ctypes.data_as(C.POINTER(C.c_int32)))
    rc = L.mpm_h5_read_table(str(path).encode(), C.byref(n), dtype.itemsize, *args, None, 0, err,
                             256)
    if rc != 0:
        raise _native.MPMError(rc, err.value.decode())
    out = np.zeros(n.value, dtype=dtype)
    rc = L.mpm_h5_read_table(str(path).encode(), C.byref(n), dtype.itemsize, *args,
                             out.ctypes.data_as(C.c_void_p), len(out), err, 256)
    if rc != 0:
        raise _native.MPMError(rc, err.value.decode())
    return out
