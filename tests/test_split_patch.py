"""One patch split over ranks by exposure (forcepho_b200.distributed), on CPU.

The FP64 oracle stands in for the kernels: the results of the sub-patches of
any partition of a patch's exposures add up to the whole patch's, a band left
without exposures evaluates to zero, and ``SplitPatchProposer`` over two gloo
ranks gives both ranks the whole patch's chi2 and gradients."""

import os
import socket

import numpy as np
import pytest

from oracle import oracle as O
from forcepho_b200 import distributed as D
from forcepho_b200 import synthetic as S


def _patch(seed=5):
    rng = np.random.default_rng(seed)
    p = S.make_patch(rng, n_sources=3, exp_per_band=[2, 1, 3], exp_pix=[(40, 32), (36, 36), (48, 30), (40, 40),
                                                                          (32, 32), (44, 28)], n_psf=3,
                     source_params=S._broad_source)
    truth = p.scene.get_proposal()
    S.add_noise(p, rng, rng.uniform(0.5, 2.0, p.n_exp), O.render(p, truth))
    prop = truth.copy()
    prop["ra"] += 2e-6
    prop["q"] = np.clip(prop["q"] * 0.96, 0.2, 0.99)
    return p, prop


def _scale(p, prop):
    c, g, r = O.evaluate(p, prop, precision="f64", return_residual=True)
    d = p.data.astype(np.float64) * p.ierr
    rr = r.astype(np.float64) * p.ierr
    return c, g, float(np.sum(d * d + rr * rr))


@pytest.mark.parametrize("world", [2, 3, 6])
def test_partition_sums_to_the_whole_patch(world):
    p, prop = _patch()
    c_all, g_all, scale = _scale(p, prop)
    w = D.exposure_weights(p)
    assert int(w.sum()) == p.n_pairs()
    parts = D.balance(w, world)
    assert sorted(sum(parts, [])) == list(range(p.n_exp))
    # largest first onto the least-loaded rank: no rank above the mean plus the largest exposure
    assert max(sum(w[i] for i in part) for part in parts) <= w.sum() / world + w.max()
    c_sum = np.zeros_like(c_all)
    g_sum = np.zeros_like(g_all, dtype=np.float64)
    for ex in parts:
        if not ex:
            continue
        sub = D.exposure_subpatch(p, ex)
        assert sub.validate()
        assert sub.n_bands == p.n_bands and int(sub.n_sources) == int(p.n_sources)
        c, g, _ = O.evaluate(sub, prop, precision="f64")
        c_sum += c
        g_sum += g
    assert np.max(np.abs(c_sum - c_all)) <= 1e-12 * scale
    for k in range(7):
        den = np.linalg.norm(g_all[..., k])
        assert np.linalg.norm(g_sum[..., k] - g_all[..., k]) <= 1e-12 * max(den, 1e-300)


def test_subpatch_arrays_and_empty_band():
    p, prop = _patch()
    whole = D.exposure_subpatch(p, range(p.n_exp))
    for name in ("xpix", "ypix", "data", "ierr", "exposure_start", "exposure_N", "band_start", "band_N", "D", "CW",
                 "crpix", "crval", "G", "psfgauss", "psfgauss_start"):
        np.testing.assert_array_equal(getattr(whole, name), getattr(p, name), err_msg=name)
    # exposure 2 is band 1's only exposure: without it band 1 is empty
    sub = D.exposure_subpatch(p, [0, 1, 3, 4, 5])
    assert list(sub.band_N) == [2, 0, 3] and list(sub.band_start) == [0, 2, 2]
    c, g, _ = O.evaluate(sub, prop, precision="f64")
    assert c[1] == 0.0 and np.all(g[1] == 0.0)
    assert np.all(c[[0, 2]] != 0.0)
    # the source copy is untouched and owns no device state
    assert "device_ptrs" not in sub.__dict__ and p.n_exp == 6
    with pytest.raises(ValueError):
        D.exposure_subpatch(p, [6])


class _OracleProposer:
    def evaluate_proposal(self, proposal, patch=None):
        c, g, _ = O.evaluate(patch, proposal, precision="f64")
        return c, g.astype(np.float32)


def _worker(rank, world, port, outdir):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        p, prop = _patch()
        sp = D.SplitPatchProposer(p, rank, world, proposer=_OracleProposer(), send=False)
        c, g = sp.evaluate_proposal(prop)
        np.save(os.path.join(outdir, "c%d.npy" % rank), c)
        np.save(os.path.join(outdir, "g%d.npy" % rank), g)
        np.save(os.path.join(outdir, "ex%d.npy" % rank), np.array(sp.exposures, dtype=np.int64))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_gloo_ranks_share_one_patch(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    p, prop = _patch()
    c_all, g_all, scale = _scale(p, prop)
    e0, e1 = np.load(tmp_path / "ex0.npy"), np.load(tmp_path / "ex1.npy")
    assert len(e0) and len(e1) and sorted(np.concatenate([e0, e1]).tolist()) == list(range(p.n_exp))
    for r in (0, 1):
        c, g = np.load(tmp_path / ("c%d.npy" % r)), np.load(tmp_path / ("g%d.npy" % r))
        assert c.dtype == np.float64 and g.dtype == np.float32 and g.shape == (p.n_bands, int(p.n_sources), 7)
        assert np.max(np.abs(c - c_all)) <= 1e-12 * scale
        for k in range(7):
            # the ranks' FP32 gradients summed in FP64 and rounded once
            assert np.linalg.norm(g[..., k] - g_all[..., k]) <= 1e-6 * np.linalg.norm(g_all[..., k])
    np.testing.assert_array_equal(np.load(tmp_path / "c0.npy"), np.load(tmp_path / "c1.npy"))


def test_store_patch_subpatch_repacks_its_own_metadata(tmp_path):
    """A sub-patch of a FITS-backed patch keeps its exposures' WCS, headers
    and band names, so repacking the scene's metadata on it gives the rows
    of the whole patch's metadata for those exposures; the partition sums
    hold as for synthetic patches."""
    from test_stores import _PSF, make_image_set
    from forcepho_b200.stores.patch import FITSPatch
    from forcepho_b200.stores.region import CircularRegion
    paths = make_image_set(tmp_path, seed=9, n_exp=(2, 2))
    p = FITSPatch(fitsfiles=paths)
    p.psfstore = _PSF()
    cat = np.zeros(2, dtype=[(c, np.float64) for c in ("ra", "dec", "q", "pa", "sersic", "rhalf", "B0", "B1")])
    cat["ra"] = [53.1, 53.1 + 5e-5]
    cat["dec"] = [-27.8, -27.8 - 3e-5]
    cat["q"], cat["pa"], cat["sersic"], cat["rhalf"] = [0.8, 0.6], [0.3, -0.5], [2.0, 1.5], [0.1, 0.2]
    cat["B0"], cat["B1"] = [10.0, 5.0], [7.0, 3.0]
    p.build_patch(CircularRegion(53.1, -27.8, 0.6 / 3600.0), cat, allbands=["B0", "B1"])
    prop = p.scene.get_proposal()
    c_all, g_all, _ = O.evaluate(p, prop, precision="f64")
    sub = D.exposure_subpatch(p, [1, 2])
    assert list(sub.band_N) == [1, 1] and list(sub.n_exp_per_band) == [1, 1]
    assert sub.bands == [p.bands[1], p.bands[2]] and sub.wcses == [p.wcses[1], p.wcses[2]]
    meta = sub.meta_for(sub.scene)
    for name in ("D", "CW", "crpix", "crval"):
        np.testing.assert_allclose(meta[name], getattr(p, name)[[1, 2]], rtol=0, atol=0, err_msg=name)
    np.testing.assert_array_equal(meta["psfgauss"], sub.psfgauss)
    rest = D.exposure_subpatch(p, [0, 3])
    c = O.evaluate(sub, prop, precision="f64")[0] + O.evaluate(rest, prop, precision="f64")[0]
    assert np.allclose(c, c_all, rtol=1e-12, atol=0)


def test_more_ranks_than_exposures():
    """With 7 ranks for 6 exposures one rank holds nothing: it evaluates
    nothing and contributes zeros, and the parts still add up."""
    p, prop = _patch()
    c_all, g_all, scale = _scale(p, prop)
    parts = [D.SplitPatchProposer(p, r, 7, proposer=_OracleProposer(), send=False) for r in range(7)]
    assert sum(1 for sp in parts if sp.patch is None) == 1
    total = sum(sp.evaluate_local(prop) for sp in parts)
    empty = [sp for sp in parts if sp.patch is None][0]
    assert not np.any(empty.evaluate_local(prop))
    c, g = parts[0].unpack(total)
    assert np.max(np.abs(c - c_all)) <= 1e-12 * scale
    for k in range(7):
        assert np.linalg.norm(g[..., k] - g_all[..., k]) <= 1e-6 * np.linalg.norm(g_all[..., k])
