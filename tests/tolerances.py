"""Error metrics and tolerances of the parity tests.

chi2 is compared RAW, relative to |chi2| itself, band by band:
``chi2_raw_err`` = max_b |chi2[b] - ref[b]| / max(|ref[b]|, RAW_FLOOR * scale[b]),
where scale[b] = sum over the band's pixels of (r^2 + d^2) ierr^2 is the
magnitude every implementation's rounding errors scale with.  chi2 =
sum (r^2 - d^2) ierr^2 can cancel to a small number (a faint source in
noise): only where |chi2[b]| has cancelled by more than 1/RAW_FLOOR = 100
against its own terms is the error measured against the floor instead (there
a tolerance t asks for |dchi2| <= t * 1e-2 * scale).  The floor is set by the
arithmetic of the pixel loops: each (pixel, Gaussian) pair is evaluated in
FP32, whose rounding of the exponent and of 2^x (a few 1e-7 of the pair's
value) leaves an absolute chi2 error of up to about 1e-8 of the scale (6e-9 is
the largest measured, on bright scenes away from their mode), so a raw bound
of 1e-6 holds wherever chi2 keeps at least 1e-2 of its terms.

The reference kernel is FP32 throughout.  Its own chi2 error against FP64,
stated in the same raw metric, can exceed 1e-5 on patches whose chi2 has
cancelled: the comparison against it therefore checks that the GPU's distance
from the reference is the reference's own error (``ref_gap_explained``), plus
the scaled metric below.

``chi2_err`` (the secondary, scaled metric) states the error relative to
``chi2_scale`` = max(|chi2|, sum_pix (r^2 + d^2) ierr^2) of the whole patch.

Gradients are compared per parameter column (flux, ra, dec, q, pa, sersic,
rhalf): normwise over bands and sources, since components of one column share
units while columns differ by many orders of magnitude (d/dra is per degree).

Tolerances (the contract of this path):
* vs the FP64 oracle, tiled path:     raw chi2 1e-6, gradient 1e-5;
* vs the FP64 oracle, plain path:     raw chi2 1e-5, gradient 1e-4 (FP32 like the reference);
* vs the reference CPU kernel (FP32): gap within the reference's own error
  + 1e-6 |chi2|; scaled chi2 1e-5; gradient 1e-4.
"""

import numpy as np

CHI2_REF = 1e-5
GRAD_REF = 1e-4
CHI2_F64 = 1e-6
GRAD_F64 = 1e-5
RAW_FLOOR = 1e-2


def chi2_scale(chi2, data, ierr, residual):
    d = np.asarray(data, np.float64) * ierr
    r = np.asarray(residual, np.float64) * ierr
    return max(float(np.max(np.abs(chi2))), float(np.sum(d * d + r * r)))


def band_scales(p, residual):
    """sum over each band's pixels of (r^2 + d^2) ierr^2, for every band of patch p."""
    out = np.zeros(p.n_bands)
    for b in range(p.n_bands):
        e0, ne = int(p.band_start[b]), int(p.band_N[b])
        if ne == 0:
            continue
        s0 = int(p.exposure_start[e0])
        s1 = int(p.exposure_start[e0 + ne - 1] + p.exposure_N[e0 + ne - 1])
        d = p.data[s0:s1].astype(np.float64) * p.ierr[s0:s1]
        r = np.asarray(residual[s0:s1], np.float64) * p.ierr[s0:s1]
        out[b] = float(np.sum(d * d + r * r))
    return out


def chi2_err(chi2, chi2_ref, scale):
    return float(np.max(np.abs(np.asarray(chi2, np.float64) - chi2_ref)) / scale)


def chi2_raw_errs(chi2, chi2_ref, scales):
    """Per band |chi2 - ref| / max(|ref|, RAW_FLOOR * scale)."""
    c = np.asarray(chi2, np.float64)
    r = np.asarray(chi2_ref, np.float64)
    den = np.maximum(np.abs(r), RAW_FLOOR * np.asarray(scales, np.float64))
    den = np.where(den > 0, den, 1.0)
    return np.abs(c - r) / den


def chi2_raw_err(chi2, chi2_ref, scales):
    e = chi2_raw_errs(chi2, chi2_ref, scales)
    return float(np.max(e)) if e.size else 0.0


def ref_gap_explained(chi2, chi2_ref, chi2_f64, tol=CHI2_F64, scales=0.0):
    """Whether |chi2 - ref| <= |ref - f64| + tol max(|f64|, RAW_FLOOR scale)
    in every band: the GPU result's distance from the FP32 reference kernel
    is the reference's own rounding error, up to the GPU's own tolerance in
    the raw metric (``scales``: per-band sum (r^2 + d^2) ierr^2, for bands
    whose chi2 has cancelled)."""
    c = np.asarray(chi2, np.float64)
    r = np.asarray(chi2_ref, np.float64)
    f = np.asarray(chi2_f64, np.float64)
    den = np.maximum(np.abs(f), RAW_FLOOR * np.asarray(scales, np.float64))
    return bool(np.all(np.abs(c - r) <= np.abs(r - f) + tol * den + 1e-300))


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
