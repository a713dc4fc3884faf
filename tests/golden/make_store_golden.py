"""Generate ``fits_store.npz``: the reference's own test image set packed into
a patch by ``forcepho_b200.stores.FITSPatch``, with FP64-oracle and reference
CPU kernel outputs.  Run where the reference sources exist (the reference CPU
kernel built first: ``make -C oracle``):

    python tests/golden/make_store_golden.py

Inputs (read-only, from the reference's tests/data): the 100x100 science image
with its uncertainty extension, TAN WCS header and source-catalog table
(test_image/sersic1.0_rhalf0.150_snr050_noise1_data.fits), and the PSF store
(test_image/..._psf.h5).  The patch is the pixels with a corner within 5 half-
light radii of the catalog source (a CircularRegion, as a superscene checkout
with roi = 5 rhalf makes it, tests/cswap_test.py:33-46) and the catalog as its
scene.  The fixture keeps the packed arrays, the packing's region and
reference coordinate, and at the catalog proposal and a perturbed one the
FP64 oracle's chi2 / gradient / residual and the reference kernel's chi2 /
gradient, so the GPU tests need no reference files.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from forcepho_b200.stores import fits as F  # noqa: E402
from forcepho_b200.stores.patch import FITSPatch  # noqa: E402
from forcepho_b200.stores.region import CircularRegion  # noqa: E402
from oracle import oracle as O  # noqa: E402

ARRAYS = ["xpix", "ypix", "data", "ierr", "exposure_start", "exposure_N", "band_start",
          "band_N", "rad2", "D", "CW", "crpix", "crval", "G", "n_psf_per_source",
          "psfgauss", "psfgauss_start"]


def image_set():
    base = os.path.join(O.reference_root(), "tests", "data", "test_image")
    return (os.path.join(base, "sersic1.0_rhalf0.150_snr050_noise1_data.fits"),
            os.path.join(base, "sersic1.0_rhalf0.150_snr050_noise1_psf.h5"))


def pack(image, psf):
    hd = F.read_fits(image)
    cat = hd[-1].data
    bands = str(hd[-1].header["FILTERS"]).split(",")
    p = FITSPatch(fitsfiles=[image], psfstore=psf)
    region = CircularRegion(cat["ra"][0], cat["dec"][0], 5 * cat["rhalf"][0] / 3600.0)
    p.build_patch(region, cat, allbands=bands)
    return p, region, cat


def main():
    image, psf = image_set()
    p, region, cat = pack(image, psf)
    out = {n: getattr(p, n) for n in ARRAYS}
    out["n_sources"] = int(p.n_sources)
    out["n_radii"] = int(p.n_radii)
    out["reference_coordinates"] = p.patch_reference_coordinates
    out["region"] = np.array([region.ra, region.dec, region.radius])
    prop0 = p.scene.get_proposal().copy()
    prop1 = prop0.copy()
    prop1["q"] *= 0.9
    prop1["rh"] *= 1.1
    prop1["fluxes"] *= 1.05
    for k, prop in enumerate((prop0, prop1)):
        c, g, r = O.evaluate(p, prop, precision="f64", return_residual=True)
        out["proposal_%d" % k] = prop
        out["f64_chi2_%d" % k], out["f64_dchi2_%d" % k], out["f64_residual_%d" % k] = c, g, r.astype(np.float32)
        cr, gr, _ = O.ref_evaluate(p, prop)
        out["ref_chi2_%d" % k], out["ref_dchi2_%d" % k] = cr, gr
    path = os.path.join(HERE, "fits_store.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, "npix", p.npix)


if __name__ == "__main__":
    main()
