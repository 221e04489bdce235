"""Per-step divergence curves: the CUDA path against the oracle, and the
oracle against itself with its input perturbed by one ulp (the problem's own
conditioning, the "floor").

A field's error at a step is max |a - b| over the particles divided by
max |b| (``tests.parity.field_errors``).  The floor answers "how far apart do
two runs of the reference arithmetic drift when their inputs differ by one
rounding": the CUDA path differs from the oracle by one rounding in the
order of its nodal sums and in its libm, so its divergence is judged against
that floor, not against zero.
"""
import numpy as np

from tests.parity import FLOAT_FIELDS, field_errors

CURVE_FIELDS = ("x", "u", "v", "stress", "strain", "F", "volume", "density")


def _record(curve, step, a, b):
    e = field_errors(a, b, CURVE_FIELDS)
    curve.append({"step": step, "cells_equal": bool(np.array_equal(a["cell"], b["cell"])),
                  "errors": e})


def gpu_vs_oracle(prob, checkpoints, nthreads=1, **over):
    """Run the problem through the C ABI and the oracle, comparing at each
    checkpoint (ascending step counts)."""
    from mpm_b200 import problems as P
    from oracle.oracle import build_oracle
    g = P.build_solver(prob, **over)
    o = build_oracle(prob, nthreads=nthreads, **over)
    curve, done = [], 0
    for s in checkpoints:
        g.step(s - done)
        o.step(s - done)
        done = s
        _record(curve, s, g.read(), o.get())
    g.close()
    return curve


def perturb_one_ulp(state, field, direction):
    """The field moved by one ulp towards +inf (direction > 0) or -inf; exact
    zeros stay zero (they are structural: 2D components, shear of a K0 state)."""
    a = np.asarray(state[field], dtype=np.float64)
    b = np.nextafter(a, np.inf if direction > 0 else -np.inf)
    return np.where(a == 0.0, 0.0, b)


def oracle_floor(prob, checkpoints, field="stress", direction=1, nthreads=1, **over):
    """Oracle against the oracle started from ``field`` perturbed by one ulp."""
    from oracle.oracle import build_oracle
    a = build_oracle(prob, nthreads=nthreads, **over)
    b = build_oracle(prob, nthreads=nthreads, **over)
    b.set({field: perturb_one_ulp(b.get(), field, direction)})
    curve, done = [], 0
    for s in checkpoints:
        a.step(s - done)
        b.step(s - done)
        done = s
        _record(curve, s, a.get(), b.get())
    return curve


def envelope(curves):
    """Pointwise maximum, per step and field, of several curves with the same
    checkpoints."""
    out = []
    for rows in zip(*curves):
        e = {f: max(r["errors"][f] for r in rows) for f in CURVE_FIELDS}
        out.append({"step": rows[0]["step"], "errors": e,
                    "cells_equal": all(r["cells_equal"] for r in rows)})
    return out


def running_max(curve):
    """Per field, the largest error seen up to each checkpoint."""
    out, best = [], {f: 0.0 for f in CURVE_FIELDS}
    for r in curve:
        best = {f: max(best[f], r["errors"][f]) for f in CURVE_FIELDS}
        out.append({"step": r["step"], "errors": dict(best)})
    return out


__all__ = ["gpu_vs_oracle", "oracle_floor", "envelope", "running_max", "perturb_one_ulp",
           "CURVE_FIELDS", "FLOAT_FIELDS"]
