"""The statistical acceptance rule of the colour-ordered parity tests (test helper).

z = (mean_a - mean_b) / sqrt(se_a^2 + se_b^2) over independent seeds, per
quantity; every |z| <= 4 and at least 95 % of them <= 3.  Many quantities are
compared at once (up to 128), so a strict "all within 3 standard errors"
fails by chance in a sizeable share of runs (0.35 expected exceedances at 128
quantities); the 3-sigma bound applies to the bulk and a 4-sigma bound to every
quantity.  Quantities whose spread is zero on both sides must agree exactly."""
import numpy as np


def z_ok(a, b, label):
    """a, b: [seeds][k] per-seed means of k quantities."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    se = np.sqrt(a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b))
    d = a.mean(0) - b.mean(0)
    fixed = se == 0
    assert np.all(np.abs(d[fixed]) <= 1e-6 * np.maximum(1.0, np.abs(b.mean(0)[fixed]))), label
    z = np.abs(d[~fixed]) / se[~fixed]
    assert z.size == 0 or (z.max() <= 4.0 and np.mean(z <= 3.0) >= 0.95), (label, np.round(z, 2))
    return z
