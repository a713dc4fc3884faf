"""The adjoint's moment algebra on the CPU.

The tile kernel never forms the reference's per-pixel partials
(forcepho/src/common_kernel.cc:95-143).  It sums moments of K = -2 w exp(-E/2)
and KH = K * H (H the pixel-integral factor) against 1, dx, dy, dx^2, dx dy,
dy^2 over a tile's pixels, and derives the six image-space partials from
them.  Here, in FP64:

* those moments reproduce the oracle's per-pixel gradient, through each
  Gaussian's Jacobian and per-source sums, to rounding;
* the same sums taken as a GEMM over raw monomials about an integer tile
  origin give the same result after an FP64 shift to each Gaussian's centre.
  This is the form a tensor-core adjoint would use: K and KH split into
  TF32 hi + lo parts (monomials of integer pixel offsets are exact in TF32),
  exact products, FP32 accumulation flushed to FP64 every 64 pixels.  Its
  error against the FP64 oracle stays below 5e-6 per gradient column, the
  tiled kernel's own level; a single TF32 pass does not.
"""

import numpy as np
import pytest

from oracle import oracle as O


def _tf32(x):
    """Round float32 to TF32 (10 explicit mantissa bits), nearest even."""
    a = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    a = (a + 0xFFF + ((a >> 13) & 1)) & ~np.uint64(0x1FFF)
    return a.astype(np.uint32).view(np.float32)


def _gemm(A, B, flush=64):
    """sum_p A[g, p] B[p, j]: exact products, FP32 accumulation over 8-wide
    steps, flushed to FP64 every ``flush`` pixels."""
    out = np.zeros((A.shape[0], B.shape[1]))
    for c0 in range(0, A.shape[1], flush):
        acc = np.zeros(out.shape, np.float32)
        for k0 in range(c0, min(A.shape[1], c0 + flush), 8):
            acc = (acc + (A[:, k0:k0 + 8].astype(np.float64) @ B[k0:k0 + 8].astype(np.float64))
                   .astype(np.float32)).astype(np.float32)
        out += acc
    return out


def _gradients(mode):
    from forcepho_b200 import synthetic as S
    p = S.config_multiband(seed=2, render=lambda pp, pr: O.render(pp, pr, precision="f64"), n_sources=4,
                           n_bands=2, exp_per_band=1, size=40, n_psf=4)
    prop = p.scene.get_proposal().copy()
    prop["q"] = np.clip(prop["q"] * 0.97, 0.2, 0.99)
    _, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
    ns = int(p.n_sources)
    out = np.zeros((p.n_bands, ns, 7))
    for e in range(p.n_exp):
        b = int(p.band_of_exp[e])
        G = O.image_gaussians(p, prop, b, e)
        amp, xc, yc, fxx, fyy, fxy = (G[:, i] for i in range(6))
        J = G[:, 6:21]
        s0, n = int(p.exposure_start[e]), int(p.exposure_N[e])
        x = p.xpix[s0:s0 + n].astype(np.float64)
        y = p.ypix[s0:s0 + n].astype(np.float64)
        w = r64[s0:s0 + n] * p.ierr[s0:s0 + n].astype(np.float64) ** 2
        tile = (np.floor((x - x.min()) / 32) * 1000 + np.floor((y - y.min()) / 32))[w != 0]
        x, y, w = x[w != 0], y[w != 0], w[w != 0]
        for t in np.unique(tile):
            X, Y, W = x[tile == t], y[tile == t], w[tile == t]
            dx, dy = X[None] - xc[:, None], Y[None] - yc[:, None]
            vx, vy = fxx[:, None] * dx + fxy[:, None] * dy, fyy[:, None] * dy + fxy[:, None] * dx
            ea = dx * vx + dy * vy
            K = -2 * W[None] * np.where(ea > 36.0, 0.0, np.exp(-0.5 * ea))
            KH = K * (1 + (vx * vx + vy * vy - fxx[:, None] - fyy[:, None]) / 24)
            if mode == "exact":
                def mom(M):
                    return [M.sum(1), (M * dx).sum(1), (M * dy).sum(1), (M * dx * dx).sum(1),
                            (M * dx * dy).sum(1), (M * dy * dy).sum(1)]
                mK, mH = mom(K), mom(KH)
            else:
                ox, oy = np.round(X.mean()), np.round(Y.mean())
                u, v = X - ox, Y - oy
                Psi = np.stack([np.ones_like(u), u, v, u * u, u * v, v * v], 1).astype(np.float32)
                assert np.array_equal(_tf32(Psi), Psi)          # exact in TF32

                def tc(A):
                    A = A.astype(np.float32)
                    hi = _tf32(A)
                    r = _gemm(hi, Psi)
                    if mode == "2xtf32":
                        r = r + _gemm(_tf32(A - hi), Psi)
                    s, su, sv, suu, suv, svv = r.T
                    ax, ay = xc - ox, yc - oy
                    return [s, su - ax * s, sv - ay * s, suu - 2 * ax * su + ax * ax * s,
                            suv - ay * su - ax * sv + ax * ay * s, svv - 2 * ay * sv + ay * ay * s]
                mK, mH = tc(K), tc(KH)
            S0, Sx, Sy, Sxx, Sxy, Syy = mK
            H0, Hx, Hy, Hxx, Hxy, Hyy = mH
            Svx, Svy = fxx * Sx + fxy * Sy, fyy * Sy + fxy * Sx
            d_x = amp * ((fxx * Hx + fxy * Hy) - (fxx * Svx + fxy * Svy) / 12)
            d_y = amp * ((fyy * Hy + fxy * Hx) - (fyy * Svy + fxy * Svx) / 12)
            d_fx = amp * (-0.5 * Hxx - (S0 - 2 * (fxx * Sxx + fxy * Sxy)) / 24)
            d_fy = amp * (-0.5 * Hyy - (S0 - 2 * (fyy * Syy + fxy * Sxy)) / 24)
            d_fxy = amp * (-Hxy + (fxy * (Sxx + Syy) + (fxx + fyy) * Sxy) / 12)
            g7 = np.stack([J[:, 0] * H0, J[:, 1] * d_x + J[:, 2] * d_y, J[:, 3] * d_x + J[:, 4] * d_y,
                           J[:, 5] * H0 + d_fx * J[:, 6] + d_fxy * J[:, 8] + d_fy * J[:, 7],
                           J[:, 9] * H0 + d_fx * J[:, 10] + d_fxy * J[:, 12] + d_fy * J[:, 11],
                           J[:, 13] * H0, J[:, 14] * H0], 1)
            np.add.at(out[b], np.arange(len(amp)) // int(p.n_psf_per_source[b]), g7)
    return out, g64


def _colerr(g, ref):
    return max(np.linalg.norm(g[..., k] - ref[..., k]) / np.linalg.norm(ref[..., k]) for k in range(7))


def test_moments_reproduce_the_per_pixel_partials():
    g, g64 = _gradients("exact")
    assert _colerr(g, g64) < 1e-12


@pytest.mark.parametrize("mode,bound", [("2xtf32", 5e-6), ("1xtf32", None)])
def test_moments_as_a_tf32_gemm(mode, bound):
    g, g64 = _gradients(mode)
    err = _colerr(g, g64)
    if bound is not None:
        assert err < bound, err
    else:
        assert err > 1e-5, err        # one TF32 pass misses the tolerance
