"""Device consumers of the kernel (forcepho/patches/device_patch.py:113-254,
forcepho/fitting.py:572-620): model renders, fixed-source subtraction, the
flux design matrix and the linear flux solve, checked against the FP64
oracle's renders of the same scenes."""

import copy

import numpy as np
import pytest

from oracle import oracle as O
from tolerances import CHI2_F64, GRAD_F64, band_scales, chi2_err, chi2_raw_err, chi2_scale, grad_err

pytestmark = pytest.mark.gpu


def _oracle_render(patch, scene):
    """f64 model of a scene over the patch's pixels, from a host copy packed for it."""
    q = copy.copy(patch)
    q.pack_meta(scene)
    return O.render(q, scene.get_proposal(), precision="f64").astype(np.float64)


def _patch(seed=31, n_sources=8):
    from forcepho_b200 import synthetic as S

    def render(p, prop):
        return O.render(p, prop, precision="f64")
    return S.config_multiband(seed=seed, render=render, n_sources=n_sources, n_bands=3, exp_per_band=2, size=48)


def test_render_matches_oracle():
    p = _patch()
    p.send_to_device()
    cat = p.catalog()
    imgs = p.render(cat)
    assert [len(x) for x in imgs] == list(p.exposure_N)
    got = np.concatenate(imgs).astype(np.float64)
    want = _oracle_render(p, p.scene)
    scale = float(np.max(np.abs(want)))
    assert np.max(np.abs(got - want)) <= 1e-6 * scale
    # the patch's own data and metadata are untouched
    assert p.retrieve_array("data").tobytes() == p.data.tobytes()


def test_design_matrix_matches_oracle():
    from forcepho_b200.sources import Scene
    p = _patch()
    p.send_to_device()
    cat = p.catalog()
    active = cat[:5]
    Xes, ys = p.design_matrix(active)
    assert len(Xes) == p.n_bands and [X.shape for X in Xes] == [(5, n) for n in p.band_N_pix]
    np.testing.assert_array_equal(np.concatenate(ys), p.data)
    scene = p.set_scene(active)
    bounds = np.concatenate([[0], np.cumsum(p.band_N_pix)])
    for i, g in enumerate(scene.sources):
        m = _oracle_render(p, Scene([g]))
        for b in range(p.n_bands):
            want = m[bounds[b]:bounds[b + 1]] / active[i][p.bandlist[b]]
            scale = float(np.max(np.abs(want)))
            assert np.max(np.abs(Xes[b][i] - want)) <= 1e-6 * scale, (i, b)


def test_subtract_fixed_matches_sequential_blocks():
    p = _patch(seed=32)
    cat = p.catalog()
    active, fixed = cat[:3], cat[3:]
    data0 = p.data.copy()
    proposer, scene = p.subtract_fixed(fixed, active=active, maxactive=2)
    assert len(scene.sources) == 3 and p.n_sources == 3
    # the reference's semantics: blocks of maxactive subtracted in turn, in FP32
    want = data0.copy()
    for blk in np.array_split(fixed, np.arange(2, len(fixed), 2)):
        m = _oracle_render(p, p.set_scene(blk))
        want = (want.astype(np.float64) - m).astype(np.float32)
    got = p.retrieve_array("data")
    scale = float(np.max(np.abs(data0)))
    assert np.max(np.abs(got.astype(np.float64) - want)) <= 1e-6 * scale
    # proposals of the active scene now see the subtracted data
    chi2, dchi2, res = proposer.evaluate_proposal(scene.get_proposal(), patch=p, unpack=False)
    q = copy.copy(p)
    q.data = got
    c64, g64, r64 = O.evaluate(q, scene.get_proposal(), precision="f64", return_residual=True)
    sc = chi2_scale(chi2, q.data, q.ierr, r64)
    assert chi2_err(chi2, c64, sc) < CHI2_F64
    assert chi2_raw_err(chi2, c64, band_scales(q, r64)) < CHI2_F64
    assert grad_err(dchi2, g64) < GRAD_F64


def test_optimize_fluxes_recovers_noiseless_fluxes():
    from forcepho_b200.fitting import optimize_fluxes
    p = _patch(seed=33, n_sources=5)
    cat = p.catalog()
    model = _oracle_render(p, p.scene)
    live = p.ierr > 0
    p.data = np.where(live, model, 0.0).astype(np.float32)
    p.send_to_device()
    fluxes, precisions = optimize_fluxes(p, cat)
    for b, name in enumerate(p.bandlist):
        np.testing.assert_allclose(fluxes[b], cat[name], rtol=1e-4)
        assert precisions[b].shape == (5, 5)
        assert np.all(np.linalg.eigvalsh(precisions[b]) > 0)
    # the host design-matrix path gives the same answer
    f2, p2, Xes, ys, ws = optimize_fluxes(p, cat, return_all=True)
    for b in range(p.n_bands):
        np.testing.assert_allclose(f2[b], fluxes[b], rtol=1e-6)
        np.testing.assert_allclose(p2[b], precisions[b], rtol=1e-6)
