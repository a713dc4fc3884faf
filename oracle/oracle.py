"""Python access to the CPU checkers.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product path never does.

Two checkers:

* ``evaluate(..., precision="f32"|"f64")`` -- this repo's C restatement
  (``fp_oracle.c``) of the reference CPU kernel, FP32 like the reference or
  entirely FP64;
* ``ref_evaluate(...)`` -- the reference's own CPU kernel
  (forcepho/src/compute_gaussians_kernel.cc), compiled from its source into
  ``oracle/_ref`` by ``oracle/Makefile``, driven the way the reference's
  ``CPUProposer.evaluate_proposal`` drives it (forcepho/proposal.py:180-226):
  one ``EvaluateProposal(band, patch_ptr, proposal_ptr)`` call per band on a
  Patch struct of host pointers (forcepho/patches/device_patch.py:446-516).
"""

import ctypes
import glob
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "lib", "libfp_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

import sys  # noqa: E402
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
from forcepho_b200.kernel_limits import MAXSOURCES, NPARAMS  # noqa: E402
from forcepho_b200.structs import patch_struct_dtype, source_struct_dtype  # noqa: E402

_lib = None
_ref = None


def reference_root():
    """Where the reference's sources lie: $FORCEPHO_REF_ROOT, else the default
    REF_ROOT of oracle/Makefile (the one place that names it)."""
    env = os.environ.get("FORCEPHO_REF_ROOT")
    if env:
        return env
    import re
    with open(os.path.join(HERE, "Makefile")) as f:
        m = re.search(r"^REF_ROOT\s*\?=\s*(\S+)", f.read(), re.M)
    return m.group(1) if m else ""


def build(force=False):
    """Compile the oracle (and the reference kernel when its sources exist)."""
    import subprocess
    targets = ["oracle"]
    root = reference_root()
    if root and os.path.isdir(os.path.join(root, "forcepho", "src")):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE] + (["-B"] if force else []) + targets + ["REF_ROOT=" + root],
                   check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, i, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p
        L.fpo_evaluate_band_f32.argtypes = [vp, vp, i, dp, dp, i]
        L.fpo_evaluate_band_f64.argtypes = [vp, vp, i, dp, dp, dp, i]
        L.fpo_image_gaussians.argtypes = [vp, vp, i, i, i, dp]
        L.fpo_count_pairs.argtypes = [vp, vp, i, ctypes.POINTER(ctypes.c_longlong),
                                      ctypes.POINTER(ctypes.c_longlong)]
        for f in (L.fpo_evaluate_band_f32, L.fpo_evaluate_band_f64, L.fpo_image_gaussians,
                  L.fpo_count_pairs):
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def ref_available():
    return bool(glob.glob(os.path.join(REF_DIR, "compute_gaussians_kernel*.so")))


def ref_module():
    """The reference CPU kernel module compiled into oracle/_ref."""
    global _ref
    if _ref is None:
        cands = glob.glob(os.path.join(REF_DIR, "compute_gaussians_kernel*.so"))
        if not cands:
            raise RuntimeError("reference CPU kernel not built (make -C oracle ref)")
        spec = importlib.util.spec_from_file_location("compute_gaussians_kernel", cands[0])
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _ref = mod
    return _ref


class HostStruct:
    """A Patch struct of host pointers to (contiguous copies of) a patch's arrays."""

    NAMES = ["data", "ierr", "xpix", "ypix", "exposure_start", "exposure_N", "band_start",
             "band_N", "rad2", "D", "crpix", "crval", "CW", "G", "n_psf_per_source",
             "psfgauss", "psfgauss_start"]

    def __init__(self, patch, residual=None):
        self.keep = {}
        s = np.zeros(1, dtype=patch_struct_dtype)
        for n in self.NAMES:
            a = np.ascontiguousarray(getattr(patch, n))
            self.keep[n] = a
            s[n] = a.ctypes.data
        if residual is not None:
            self.keep["residual"] = residual
            s["residual"] = residual.ctypes.data
        s["n_sources"] = int(patch.n_sources)
        s["n_radii"] = int(patch.n_radii)
        self.struct = s
        self.ptr = s.ctypes.data


def _proposal(proposal):
    p = np.ascontiguousarray(proposal, dtype=source_struct_dtype)
    return p, p.ctypes.data


def evaluate(patch, proposal, precision="f32", return_residual=False, nthreads=None, bands=None):
    """chi2[n_bands] (f64), dchi2[n_bands, n_sources, 7], residual or None.

    ``precision="f32"`` restates the reference arithmetic (dchi2 f32);
    ``"f64"`` computes everything in FP64 (dchi2 f64, residual f64).
    ``bands``: evaluate only these bands (the others are left zero)."""
    L = lib()
    nb, ns = patch.n_bands, int(patch.n_sources)
    todo = range(nb) if bands is None else list(bands)
    if nthreads is None:
        nthreads = min(os.cpu_count() or 1, 32)
    prop, pptr = _proposal(proposal)
    chi2 = np.zeros(nb, dtype=np.float64)
    if precision == "f32":
        res = np.zeros(patch.npix, dtype=np.float32) if return_residual else None
        hs = HostStruct(patch, residual=res)
        grads = np.zeros((nb, MAXSOURCES * NPARAMS), dtype=np.float32)
        for b in todo:
            c = ctypes.c_double()
            rc = L.fpo_evaluate_band_f32(hs.ptr, pptr, b, ctypes.addressof(c),
                                         grads[b].ctypes.data, nthreads)
            if rc:
                raise RuntimeError("oracle f32 failed (%d)" % rc)
            chi2[b] = c.value
    elif precision == "f64":
        hs = HostStruct(patch)
        res = np.zeros(patch.npix, dtype=np.float64) if return_residual else None
        grads = np.zeros((nb, MAXSOURCES * NPARAMS), dtype=np.float64)
        for b in todo:
            c = ctypes.c_double()
            rc = L.fpo_evaluate_band_f64(hs.ptr, pptr, b, ctypes.addressof(c),
                                         grads[b].ctypes.data,
                                         res.ctypes.data if res is not None else None, nthreads)
            if rc:
                raise RuntimeError("oracle f64 failed (%d)" % rc)
            chi2[b] = c.value
    else:
        raise ValueError(precision)
    dchi2 = grads.reshape(nb, MAXSOURCES, NPARAMS)[:, :ns].copy()
    return chi2, dchi2, res


def ref_evaluate(patch, proposal, return_residual=False, bands=None):
    """The reference CPU kernel, one pybind call per band (CPUProposer's loop);
    ``bands``: only these bands (the others are left zero)."""
    mod = ref_module()
    nb, ns = patch.n_bands, int(patch.n_sources)
    res = np.zeros(patch.npix, dtype=np.float32) if return_residual else None
    hs = HostStruct(patch, residual=res)
    prop, pptr = _proposal(proposal)
    chi2 = np.zeros(nb, dtype=np.float64)
    dchi2 = np.zeros((nb, ns, NPARAMS), dtype=np.float32)
    for b in (range(nb) if bands is None else bands):
        r = mod.EvaluateProposal(b, hs.ptr, pptr)
        chi2[b] = r.chi2
        dchi2[b] = np.asarray(r.dchi2_dp).reshape(MAXSOURCES, NPARAMS)[:ns]
    return chi2, dchi2, res


def render(patch, proposal, precision="f64"):
    """Model counts of every pixel (f32) = -(residual of an all-zero data array)."""
    saved = patch.data
    patch.data = np.zeros_like(saved)
    try:
        _, _, res = evaluate(patch, proposal, precision=precision, return_residual=True)
    finally:
        patch.data = saved
    return (-res).astype(np.float32)


def image_gaussians(patch, proposal, band, exposure, precision="f64"):
    """[n_gauss, 21] image Gaussians (amp, xcen, ycen, fxx, fyy, fxy, 15 Jacobian terms)."""
    ng = int(patch.n_sources) * int(patch.n_psf_per_source[band])
    out = np.zeros((ng, 21), dtype=np.float64)
    hs = HostStruct(patch)
    prop, pptr = _proposal(proposal)
    rc = lib().fpo_image_gaussians(hs.ptr, pptr, band, exposure, int(precision == "f64"),
                                   out.ctypes.data)
    if rc:
        raise RuntimeError("oracle image_gaussians failed")
    return out


def count_pairs(patch, proposal):
    """(all pairs, pairs within the MAX_EXP_ARG cutoff) summed over bands."""
    hs = HostStruct(patch)
    prop, pptr = _proposal(proposal)
    tot = act = 0
    for b in range(patch.n_bands):
        a, c = ctypes.c_longlong(), ctypes.c_longlong()
        lib().fpo_count_pairs(hs.ptr, pptr, b, ctypes.byref(a), ctypes.byref(c))
        tot += a.value
        act += c.value
    return tot, act
