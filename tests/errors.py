"""Error metric used by every parity test.

Relative error per entry; entries whose reference magnitude is below
floor * max|ref| are measured by absolute error normalised to max|ref|
(floor = 1e-6, stated in every report)."""
import numpy as np

FLOOR = 1e-6


def rel_errors(a, ref, floor=FLOOR):
    a = np.asarray(a, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    scale = np.abs(ref).max()
    if scale == 0:
        return np.abs(a).ravel()
    big = np.abs(ref) >= floor * scale
    denom = np.where(big, np.abs(ref), scale)
    return (np.abs(a - ref) / denom).ravel()


def max_rel(a, ref, floor=FLOOR):
    return float(rel_errors(a, ref, floor).max())


def median_rel(a, ref, floor=FLOOR):
    return float(np.median(rel_errors(a, ref, floor)))
