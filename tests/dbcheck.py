"""The mel-dB parity bar, shared by the GPU tests.

The bar is 1e-3 dB against the FP64 oracle.  A float32 FFT's rounding is
absolute -- a fraction of the frame's largest bins -- so a band's dB error
grows with its distance below the frame's (and so the clip's) maximum: about
4.3 * 2 * 2^-24 * 10^(d / 20) dB at d dB down for a one-bin band.  The
reference's own float32 path (``oracle/refcpu.c``, the C port of its CPU
algorithm: radix-2 FFT, dense mel GEMM) shows exactly this, up to ~2e-3 dB for
values 60-80 dB below the clip maximum that the top_db floor keeps, on small
n_fft with few bins per band.

``check_db`` therefore asserts, value by value within distance bins of the
clip maximum:
- within 60 dB of the maximum: |err| < 1e-3 dB;
- 60-70 dB and 70-80 dB below it: the largest |err| in the bin is at most
  max(1e-3 dB, FACTOR x the largest |err| of the reference's float32 path in
  the same bin of the same clip), i.e. the GPU rounds no worse than the
  reference does there, up to FACTOR.
"""

import numpy as np

DB_TOL = 1e-3
FACTOR = 2.0
BINS = ((60.0, 70.0), (70.0, np.inf))


def check_db(got_db, exp_db, ref_db, what=None, tol=DB_TOL, factor=FACTOR):
    """Assert the bar for one clip's floored mel-dB (got: GPU, exp: FP64
    oracle, ref: the reference's float32 path); returns the per-bin errors."""
    got_db, exp_db, ref_db = (np.asarray(a, np.float64) for a in (got_db, exp_db, ref_db))
    assert got_db.shape == exp_db.shape == ref_db.shape, (got_db.shape, exp_db.shape, ref_db.shape)
    if exp_db.size == 0:
        return {}
    err, err_ref = np.abs(got_db - exp_db), np.abs(ref_db - exp_db)
    dist = exp_db.max() - exp_db
    near = dist <= 60.0
    out = {"near": float(err[near].max())}
    assert out["near"] < tol, (what, out)
    for lo, hi in BINS:
        sel = (dist > lo) & (dist <= hi)
        if not sel.any():
            continue
        g, r = float(err[sel].max()), float(err_ref[sel].max())
        out[f"{lo:.0f}-{hi:.0f}"] = (g, r)
        assert g <= max(tol, factor * r), (what, lo, hi, g, r)
    return out
