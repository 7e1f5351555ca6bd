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


def per_channel(counts, ref, floor=FLOOR):
    """Relative errors of counts [n_ch][n_bins] per channel, with the floor taken
    over the whole array: (max over bins, median over bins), one entry per channel."""
    n_ch = np.asarray(ref).shape[0]
    e = rel_errors(counts, ref, floor).reshape(n_ch, -1)
    return e.max(axis=1), np.median(e, axis=1)


def per_channel_summary(counts, ref, floor=FLOOR):
    """Distribution over channels of the per-channel max and median relative error."""
    mx, md = per_channel(counts, ref, floor)
    return {"channels": int(mx.size), "max_of_channel_max": float(mx.max()),
            "median_of_channel_max": float(np.median(mx)), "max_of_channel_median": float(md.max()),
            "median_of_channel_median": float(np.median(md))}
