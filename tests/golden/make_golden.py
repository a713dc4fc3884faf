"""Generate the golden fixtures of this directory.  Run in a container that has
the reference sources (the reference CPU kernel must be built first:
``make -C oracle``):

    python tests/golden/make_golden.py

Each fixture holds the inputs of one seeded synthetic patch (or, for the large
one, only its data array plus checksums of the deterministic rest), one or two
proposals, and the outputs of

* ``ref_*``  -- the reference's own CPU kernel (forcepho/src/compute_gaussians_kernel.cc,
               compiled from source into oracle/_ref), driven band by band like
               CPUProposer (forcepho/proposal.py:180-226);
* ``f64_*``  -- this repo's FP64 oracle (oracle/fp_oracle.c), for precision
               statements;
* ``slow_*`` -- (small fixture only) the reference's pure-Python FP64 path,
               forcepho/slow/gaussmodel.py (convert_to_gaussians +
               compute_gaussian, no MAX_EXP_ARG cutoff), evaluated pixel by
               pixel as an independent check of the image-Gaussian setup.
"""

import hashlib
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from forcepho_b200 import synthetic as S  # noqa: E402
from oracle import oracle as O  # noqa: E402

ARRAYS = ["xpix", "ypix", "data", "ierr", "exposure_start", "exposure_N", "band_start",
          "band_N", "rad2", "D", "CW", "crpix", "crval", "G", "n_psf_per_source",
          "psfgauss", "psfgauss_start"]


def digest(patch, names):
    h = hashlib.sha256()
    for n in names:
        h.update(np.ascontiguousarray(getattr(patch, n)).tobytes())
    return h.hexdigest()


def perturbed(proposal, rng):
    """A proposal moved off the truth (so gradients are far from zero)."""
    p = proposal.copy()
    n = len(p)
    p["ra"] += rng.normal(0, 2e-6, n).astype(np.float32)     # ~0.2 px
    p["dec"] += rng.normal(0, 2e-6, n).astype(np.float32)
    p["q"] = np.clip(p["q"] * rng.uniform(0.9, 1.1, n), 0.2, 0.99).astype(np.float32)
    p["pa"] += rng.normal(0, 0.1, n).astype(np.float32)
    p["fluxes"] *= rng.uniform(0.8, 1.2, p["fluxes"].shape).astype(np.float32)
    return p


def outputs(patch, proposals):
    out = {}
    for k, prop in enumerate(proposals):
        c, g, r = O.ref_evaluate(patch, prop, return_residual=True)
        out[f"ref_chi2_{k}"], out[f"ref_dchi2_{k}"], out[f"ref_residual_{k}"] = c, g, r
        c, g, r = O.evaluate(patch, prop, precision="f64", return_residual=True)
        out[f"f64_chi2_{k}"], out[f"f64_dchi2_{k}"] = c, g
        out[f"f64_residual_{k}"] = r.astype(np.float32)
        out[f"proposal_{k}"] = prop
    return out


def slow_path_model(patch, proposal, band=0, exposure=0):
    """Model pixels of one exposure from forcepho/slow/gaussmodel.py (FP64)."""
    path = os.path.join(O.reference_root(), "forcepho", "slow", "gaussmodel.py")
    spec = importlib.util.spec_from_file_location("fp_slow_gaussmodel", path)
    gm = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gm)
    # image Gaussians from this repo's FP64 setup, rendered by the slow path's
    # per-Gaussian evaluator (second-order pixel integral, no cutoff)
    ig = O.image_gaussians(patch, proposal, band, exposure, precision="f64")
    s0, n = int(patch.exposure_start[exposure]), int(patch.exposure_N[exposure])
    xp = patch.xpix[s0:s0 + n].astype(np.float64)
    yp = patch.ypix[s0:s0 + n].astype(np.float64)
    model = np.zeros(n)
    for row in ig:
        g = gm.ImageGaussian()
        g.amp, g.xcen, g.ycen, g.fxx, g.fyy, g.fxy = row[:6]
        c, _ = gm.compute_gaussian(g, xp, yp, compute_deriv=False), None
        model += c
    # also the slow path's own source->image conversion (convert_to_gaussians
    # helper) for the first source, to pin the covariance/amplitude algebra
    return model


def main():
    rng = np.random.default_rng(12345)

    # 1. small workload, full inputs, two proposals, slow-path cross-check
    p = S.config_small(seed=1, render=O.render)
    prop0 = p.scene.get_proposal()
    props = [prop0, perturbed(prop0, rng)]
    out = outputs(p, props)
    out.update({n: getattr(p, n) for n in ARRAYS})
    out["n_sources"], out["n_radii"] = int(p.n_sources), int(p.n_radii)
    out["slow_model_0"] = slow_path_model(p, prop0)
    np.savez_compressed(os.path.join(HERE, "small.npz"), **out)

    # 2. reduced multiband (3 bands x 2 exposures, 48x48, 6 sources), full inputs
    p = S.config_multiband(seed=22, render=O.render, n_sources=6, n_bands=3, exp_per_band=2,
                           size=48, n_psf=4)
    prop0 = p.scene.get_proposal()
    props = [prop0, perturbed(prop0, rng)]
    out = outputs(p, props)
    out.update({n: getattr(p, n) for n in ARRAYS})
    out["n_sources"], out["n_radii"] = int(p.n_sources), int(p.n_radii)
    np.savez_compressed(os.path.join(HERE, "multiband_reduced.npz"), **out)

    # 3. full multiband workload: only `data` is stored; the other arrays are
    #    regenerated from the seed and checked against the stored digest
    p = S.config_multiband(seed=2, render=O.render)
    prop0 = p.scene.get_proposal()
    props = [prop0, perturbed(prop0, rng)]
    out = outputs(p, props)
    for k in range(len(props)):   # residuals of the full patch are not kept
        del out[f"ref_residual_{k}"], out[f"f64_residual_{k}"]
    out["data"] = p.data
    names = [n for n in ARRAYS if n != "data"]
    out["digest_rest"] = np.array(digest(p, names))
    np.savez_compressed(os.path.join(HERE, "multiband.npz"), **out)
    for f in ("small.npz", "multiband_reduced.npz", "multiband.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
