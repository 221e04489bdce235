"""The HDF5 particle table (Mesh::write_particles_hdf5, mesh.tcc:1573-1613;
Mesh::read_particles_hdf5, mesh.tcc:1663-1720), encoded and decoded by the
library without the HDF5 library.  Checked on the CPU: records round-trip
through the library's writer and reader; an independent reading of the file
structure (tests/h5_structure.py) finds H5TBmake_table's layout -- dataset
"table", the 74 PODParticle fields with the names, offsets and types of
pod_particle.cc in a 592-byte compound, chunks of 10000 records in a version 1
B-tree, attributes CLASS, VERSION, TITLE, FIELD_<i>_NAME -- and the same
records."""
import numpy as np
import pytest

from mpm_b200 import h5
from mpm_b200._native import MPMError
from mpm_b200.pod import NAMES
from tests import h5_structure


def _records(n, seed=3):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, dtype=h5.REFERENCE_POD_DTYPE)
    for name, t, _ in h5.REFERENCE_FIELDS:
        if t == h5.F64:
            r[name] = rng.normal(0, 1e3, n)
        elif t == h5.U8:
            r[name] = rng.integers(0, 2, n)
        else:
            r[name] = rng.integers(0, 2 ** 31, n)
    r["id"] = np.arange(n)
    return r


@pytest.mark.parametrize("n", [0, 1, 9999, 10000, 25001, 700001])
def test_records_round_trip(tmp_path, n):
    rec = _records(n)
    path = tmp_path / "particles.h5"
    h5.write_table(path, rec)
    back = h5.read_table(path)
    assert len(back) == n
    for name in NAMES:
        assert np.array_equal(back[name], rec[name]), name


def test_file_structure_is_h5tb_make_table(tmp_path):
    rec = _records(25001)
    path = tmp_path / "particles.h5"
    h5.write_table(path, rec)
    info = h5_structure.read(path)
    assert info["nrecords"] == 25001 and info["record_size"] == 592
    assert info["chunk_records"] == 10000
    kinds = {h5.F64: "f64", h5.I64: "i64", h5.U8: "u8", h5.U32: "u32"}
    assert info["fields"] == [(n, o, kinds[t]) for n, t, o in h5.REFERENCE_FIELDS]
    a = info["attributes"]
    assert a["CLASS"] == "TABLE" and a["VERSION"] == "3.0" and a["TITLE"] == "Table Title"
    for i, n in enumerate(NAMES):
        assert a[f"FIELD_{i}_NAME"] == n
    raw = h5_structure.records(info, h5.REFERENCE_POD_DTYPE)
    for name in NAMES:
        assert np.array_equal(raw[name], rec[name]), name


def test_multilevel_chunk_index(tmp_path):
    """More than 64 chunks: the chunk B-tree gets an internal level."""
    rec = _records(130 * 100 + 7)
    path = tmp_path / "t.h5"
    h5.write_table(path, rec, chunk_records=100)
    info = h5_structure.read(path)
    assert info["nrecords"] == len(rec)
    raw = h5_structure.records(info, h5.REFERENCE_POD_DTYPE)
    assert np.array_equal(raw["mass"], rec["mass"])
    assert np.array_equal(h5.read_table(path)["svars_19"], rec["svars_19"])


def test_reader_reports_what_it_cannot_read(tmp_path):
    bad = tmp_path / "not.h5"
    bad.write_bytes(b"not an hdf5 file at all" * 10)
    with pytest.raises(MPMError, match="not an HDF5 file"):
        h5.read_table(bad)
    path = tmp_path / "t.h5"
    small = np.zeros(3, dtype=[("id", np.int64), ("mass", np.float64)])
    h5.write_table(path, small)
    with pytest.raises(MPMError, match="no field volume"):
        h5.read_table(path)
