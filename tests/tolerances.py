"""Error metrics and tolerances of the parity tests.

chi2 = sum_pix (r^2 - d^2) ierr^2 can be small or near zero while its terms are
large (a faint source in noise), so its error is stated relative to
``chi2_scale`` = max(|chi2|, sum_pix (r^2 + d^2) ierr^2), the magnitude the
rounding errors of any implementation scale with.  Gradients are compared per
parameter column (flux, ra, dec, q, pa, sersic, rhalf): normwise over bands and
sources, since components of one column share units while columns differ by
many orders of magnitude (d/dra is per degree).

Tolerances (the contract of this path):
* vs the reference CPU kernel (FP32): chi2 1e-5, gradient 1e-4;
* vs the FP64 oracle, tiled path:     chi2 1e-6, gradient 1e-5;
* vs the FP64 oracle, plain path:     chi2 1e-5, gradient 1e-4 (FP32 like the reference).
"""

import numpy as np

CHI2_REF = 1e-5
GRAD_REF = 1e-4
CHI2_F64 = 1e-6
GRAD_F64 = 1e-5


def chi2_scale(chi2, data, ierr, residual):
    d = np.asarray(data, np.float64) * ierr
    r = np.asarray(residual, np.float64) * ierr
    return max(float(np.max(np.abs(chi2))), float(np.sum(d * d + r * r)))


def chi2_err(chi2, chi2_ref, scale):
    return float(np.max(np.abs(np.asarray(chi2, np.float64) - chi2_ref)) / scale)


def grad_err(g, gref):
    """max over parameter columns of ||g - gref|| / ||gref||."""
    g = np.asarray(g, np.float64)
    gref = np.asarray(gref, np.float64)
    out = 0.0
    for k in range(gref.shape[-1]):
        den = np.linalg.norm(gref[..., k])
        num = np.linalg.norm(g[..., k] - gref[..., k])
        if den == 0:
            out = max(out, 0.0 if num == 0 else np.inf)
        else:
            out = max(out, num / den)
    return float(out)


def grad_err_columns(g, gref):
    g = np.asarray(g, np.float64)
    gref = np.asarray(gref, np.float64)
    return [float(np.linalg.norm(g[..., k] - gref[..., k]) / max(np.linalg.norm(gref[..., k]), 1e-300))
            for k in range(gref.shape[-1])]
