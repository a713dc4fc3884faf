"""Linear flux solve conditional on source shapes.

The reference (forcepho/fitting.py:572-620) builds the design matrix on the
host (one full kernel evaluation per source) and solves the weighted normal
equations per band with numpy.  Here ``optimize_fluxes`` forms the normal
equations on the device in FP64 from one batched forward-only render of all
sources (``forcepho_b200.render.normal_equations``) and solves the small
(n_source x n_source) systems on the host; ``return_all=True`` also returns the
host design matrices, as the reference does.
"""

import numpy as np

__all__ = ["optimize_one_band", "optimize_fluxes"]


def optimize_one_band(X, w, y, fixedX=0):
    """Weighted linear least squares of one band (forcepho/fitting.py:572-587).

    X : (n_source, n_pix) flux-normalised source models; w : (n_pix,) inverse
    errors; y : (n_pix,) data.  Returns (flux (n_source, 1), precision matrix
    (n_source, n_source) = X_w X_wᵀ)."""
    Xp = np.asarray(X, dtype=np.float64) * w
    yp = (np.asarray(y, dtype=np.float64) - fixedX) * w
    ATA = np.dot(Xp, Xp.T)
    Xyp = np.dot(Xp, yp[:, None])
    flux = np.linalg.solve(ATA, Xyp)
    return flux, ATA


def optimize_fluxes(patcher, active, return_all=False):
    """Maximum-likelihood fluxes of the ``active`` catalog's sources in every
    band, conditional on their shapes, and the flux precision matrices
    (forcepho/fitting.py:590-620).  Run ``patcher.subtract_fixed`` first when
    fixed sources are to be removed from the data.

    Returns (fluxes, precisions): lists over bands of (n_source,) and
    (n_source, n_source) arrays; with ``return_all`` also the design matrices,
    data and weights per band.  A singular band returns, as the reference does,
    (band index, the LinAlgError, Xes, ys, ws)."""
    from numpy.linalg import LinAlgError
    if return_all:
        Xes, ys = patcher.design_matrix(active)
        ws = patcher.split_band("ierr")
        fluxes, precisions = [], []
        for i, (w, X, y) in enumerate(zip(ws, Xes, ys)):
            try:
                flux, precision = optimize_one_band(X, w, y)
            except LinAlgError as e:
                return i, e, Xes, ys, ws
            fluxes.append(np.atleast_1d(np.squeeze(flux)))
            precisions.append(precision)
        return fluxes, precisions, Xes, ys, ws

    from .render import normal_equations
    fluxes, precisions = [], []
    for i, (ATA, Xy) in enumerate(normal_equations(patcher, active)):
        try:
            flux = np.linalg.solve(ATA, Xy[:, None])
        except LinAlgError as e:
            Xes, ys = patcher.design_matrix(active)
            return i, e, Xes, ys, patcher.split_band("ierr")
        fluxes.append(np.atleast_1d(np.squeeze(flux)))
        precisions.append(ATA)
    return fluxes, precisions
