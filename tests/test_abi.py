"""The C-ABI libraries load and export every symbol their headers declare
(no compute calls: this runs on hosts without a GPU)."""
import ctypes
import os
import re

from tests.conftest import ROOT


def _declared(header, prefix):
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(" + prefix + r"\w+)\s*\(", text)))


def test_product_library_exports_header_symbols():
    from mpm_b200 import _native
    assert os.path.exists(_native.LIB_PATH), "libmpm_b200.so not built"
    lib = ctypes.CDLL(_native.LIB_PATH)
    names = _declared(os.path.join(ROOT, "include", "mpm_gpu.h"), "mpm_(?:gpu|h5)_")
    assert len(names) >= 19
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(names) == set(_native.SIGNATURES), set(names) ^ set(_native.SIGNATURES)


def test_version_string_without_gpu():
    from mpm_b200 import _native
    v = _native.lib().mpm_gpu_version().decode()
    assert "sm_100a" in v


def test_create_rejects_bad_config_without_touching_the_device():
    from mpm_b200 import _native
    L = _native.lib()
    cfg = _native.Config()
    cfg.dim = 4
    h = ctypes.c_void_p()
    assert L.mpm_gpu_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    cfg.dim = 3
    cfg.precision = 7
    cfg.dt = 1e-3
    assert L.mpm_gpu_create(ctypes.byref(cfg), ctypes.byref(h)) == -7


def test_oracle_library_exports_header_symbols():
    from oracle import oracle as O
    lib = O.lib()
    names = _declared(os.path.join(ROOT, "oracle", "mpm_oracle.h"), "mpmo_")
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_product_does_not_reference_the_oracle():
    """The product package never imports, links or loads the oracle."""
    pkg = os.path.join(ROOT, "mpm_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".hpp", ".cpp")):
                text = open(os.path.join(dirpath, f)).read()
                assert "mpm_oracle" not in text and "import oracle" not in text \
                    and "from oracle" not in text, f


def test_pod_record_table_matches_the_reference_field_list():
    """74 fields in PODParticle order with the sizes of pod_particle.cc."""
    from mpm_b200 import pod
    assert len(pod.NAMES) == 74
    assert pod.NAMES[:4] == ["id", "mass", "volume", "pressure"]
    assert pod.NAMES[40] == "initialise_mapping_matrix" and pod.NAMES[50] == "status"
    assert pod.NAMES[51:54] == ["cell_id", "material_id", "nstate_vars"]
    assert pod.NAMES[54] == "svars_0" and pod.NAMES[73] == "svars_19"
    size, offs, sizes = pod.layout()
    expect = [1 if i in (40, 50) else 4 if i in (52, 53) else 8 for i in range(74)]
    assert list(sizes) == expect
    assert all(o % s == 0 for o, s in zip(offs, sizes)) and size % 8 == 0
