import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running (large workloads)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name), allow_pickle=False) as d:
        return {k: d[k] for k in d.files}


def patch_from_golden(g, cls=None):
    """Rebuild a patch object from a golden fixture holding full inputs."""
    from forcepho_b200.synthetic import SyntheticPatch
    cls = cls or SyntheticPatch
    p = cls()
    for n in ["xpix", "ypix", "data", "ierr", "exposure_start", "exposure_N", "band_start", "band_N",
              "rad2", "D", "CW", "crpix", "crval", "G", "n_psf_per_source", "psfgauss", "psfgauss_start"]:
        setattr(p, n, np.array(g[n]))
    p.n_sources = int(g["n_sources"])
    p.n_radii = int(g["n_radii"])
    return p


@pytest.fixture(scope="session")
def golden_small():
    return load_golden("small.npz")


@pytest.fixture(scope="session")
def golden_reduced():
    return load_golden("multiband_reduced.npz")


@pytest.fixture(scope="session")
def golden_multiband():
    """The full multiband workload: regenerate the deterministic arrays from the
    seed, put back the stored data array, and check the digest."""
    import hashlib
    from forcepho_b200 import synthetic as S
    g = load_golden("multiband.npz")
    p = S.config_multiband(seed=2)
    p.data = np.array(g["data"])
    h = hashlib.sha256()
    for n in ["xpix", "ypix", "ierr", "exposure_start", "exposure_N", "band_start", "band_N", "rad2", "D",
              "CW", "crpix", "crval", "G", "n_psf_per_source", "psfgauss", "psfgauss_start"]:
        h.update(np.ascontiguousarray(getattr(p, n)).tobytes())
    assert h.hexdigest() == str(g["digest_rest"]), "regenerated multiband inputs differ from the fixture"
    return p, g
