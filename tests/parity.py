"""Shared helpers of the parity tests: run one problem through the CUDA path
(libmpm_b200.so via its C ABI) and through the CPU oracle, compare fields."""
import numpy as np

FLOAT_FIELDS = ("x", "u", "v", "stress", "strain", "F", "volume", "density", "mass")
# Relative tolerance for the FP64 path: max |gpu - oracle| over a field,
# divided by max |oracle| over that field.
FP64_RTOL = 1e-10


def field_errors(g, o, fields=FLOAT_FIELDS, mask=None):
    errs = {}
    for f in fields:
        a = np.asarray(g[f], dtype=np.float64)
        b = np.asarray(o[f], dtype=np.float64)
        if mask is not None:
            a, b = a[mask], b[mask]
        scale = max(np.max(np.abs(b)) if b.size else 0.0, 1e-300)
        errs[f] = float(np.max(np.abs(a - b)) / scale) if b.size else 0.0
    return errs


def mc_state_errors(g, o):
    """Per-variable relative errors of the MohrCoulomb state (phi..pdstrain)."""
    out = {}
    names = ["yield_state", "phi", "psi", "cohesion", "tension_cutoff", "epsilon", "rho",
             "theta", "pdstrain"]
    for k, n in enumerate(names):
        a, b = g["svars"][:, k], o["svars"][:, k]
        scale = max(np.max(np.abs(b)), 1e-300)
        out[n] = float(np.max(np.abs(a - b)) / scale)
    return out


def assert_parity(g, o, rtol=FP64_RTOL, fields=FLOAT_FIELDS, check_cells=True, label=""):
    if check_cells:
        assert np.array_equal(np.asarray(g["cell"]), np.asarray(o["cell"])), \
            f"{label}: cell ids differ at {np.nonzero(np.asarray(g['cell']) != np.asarray(o['cell']))[0][:10]}"
    errs = field_errors(g, o, fields)
    bad = {k: v for k, v in errs.items() if not v <= rtol}
    assert not bad, f"{label}: fields beyond {rtol}: {bad}"
    return errs
