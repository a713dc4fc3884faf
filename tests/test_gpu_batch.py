"""The batched public call, ``BatchedProposer.evaluate_proposals``: parity of
every patch of a mixed batch with the FP64 oracle and with the one-patch
``B200Proposer`` (the same tiles, so the same sums), the staging of proposals
of changing length, results that stay valid after later calls, the
asynchronous calls without a host synchronisation, re-planning after a patch
is sent again, the pair census, and a plan over shuffled pixels without
coordinates."""

import numpy as np
import pytest

from oracle import oracle as O
from tolerances import CHI2_F64, GRAD_F64, band_scales, chi2_err, chi2_raw_err, chi2_scale, grad_err

pytestmark = pytest.mark.gpu


def _patches():
    from forcepho_b200 import synthetic as S
    shapes = [(3, 2, 1, 40), (7, 1, 2, 56), (2, 4, 1, 32), (12, 3, 2, 64), (5, 2, 1, 48)]
    out = []
    for i, (ns, nb, epb, size) in enumerate(shapes):
        p = S.config_multiband(seed=300 + i, n_sources=ns, n_bands=nb, exp_per_band=epb, size=size)
        p.return_residual = False
        p.send_to_device()
        out.append(p)
    return out


def _perturbed(patches, seed):
    rng = np.random.default_rng(seed)
    out = []
    for p in patches:
        q = p.scene.get_proposal().copy()
        q["ra"] += rng.normal(0, 2e-6, len(q)).astype(np.float32)
        q["q"] = np.clip(q["q"] * rng.uniform(0.95, 1.05, len(q)), 0.2, 0.99).astype(np.float32)
        out.append(q)
    return out


@pytest.fixture(scope="module")
def batch():
    return _patches()


def test_batch_matches_oracle_and_single_patch(batch):
    from forcepho_b200.batch import BatchedProposer
    from forcepho_b200.proposal import B200Proposer
    props = _perturbed(batch, 1)
    bp = BatchedProposer(batch, tile_pixels=1024)
    res = bp.evaluate_proposals(props)
    single = B200Proposer(tile_pixels=1024)
    for p, prop, (chi2, dchi2) in zip(batch, props, res):
        assert chi2.shape == (p.n_bands,)
        assert dchi2.shape == (p.n_bands, int(p.n_sources), 7)
        c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
        scale = chi2_scale(chi2, p.data, p.ierr, r64)
        assert chi2_err(chi2, c64, scale) < CHI2_F64
        assert chi2_raw_err(chi2, c64, band_scales(p, r64)) < CHI2_F64
        assert grad_err(dchi2, g64) < GRAD_F64
        c1, g1 = single.evaluate_proposal(prop, patch=p)
        np.testing.assert_array_equal(chi2, c1)
        np.testing.assert_array_equal(dchi2, g1)


def test_repeated_calls_and_result_lifetime(batch):
    from forcepho_b200.batch import BatchedProposer
    a, b = _perturbed(batch, 2), _perturbed(batch, 3)
    bp = BatchedProposer(batch, tile_pixels=1024)
    ra = bp.evaluate_proposals(a)
    kept = [(c.copy(), g.copy()) for c, g in ra]
    rb = bp.evaluate_proposals(b)
    for (c, g), (c0, g0) in zip(ra, kept):          # earlier results are not overwritten
        np.testing.assert_array_equal(c, c0)
        np.testing.assert_array_equal(g, g0)
    fresh = BatchedProposer(batch, tile_pixels=1024).evaluate_proposals(b)
    for (c, g), (c2, g2) in zip(rb, fresh):
        np.testing.assert_array_equal(c, c2)
        np.testing.assert_array_equal(g, g2)


def test_staging_zeroes_the_slots_of_a_shorter_proposal(batch):
    from forcepho_b200.batch import BatchedProposer
    from forcepho_b200.structs import source_struct_dtype
    props = _perturbed(batch, 4)
    bp = BatchedProposer(batch, tile_pixels=1024)
    bp.set_proposals_async(props)
    i = 3                                              # the 12-source patch
    bp.set_proposals_async(props[:i] + [props[i][:5]] + props[i + 1:])
    slots = bp._pin_prop.numpy().view(source_struct_dtype).reshape(len(batch), -1)
    np.testing.assert_array_equal(slots[i, :5], props[i][:5])
    assert not slots[i, 5:].view(np.uint8).any()
    bp.set_proposals_async(props[:2])                  # patches past the list: no sources
    assert not slots[2:].view(np.uint8).any()
    with pytest.raises(ValueError):
        bp.set_proposals_async(props + props[:1])
    # and back to full proposals: results equal a fresh proposer's
    res = bp.evaluate_proposals(props)
    want = BatchedProposer(batch, tile_pixels=1024).evaluate_proposals(props)
    for (c, g), (c2, g2) in zip(res, want):
        np.testing.assert_array_equal(c, c2)
        np.testing.assert_array_equal(g, g2)


def test_async_calls_without_host_sync(batch):
    """set_proposals_async / run / fetch_async / results with no synchronisation
    by the caller: restaging waits only for the previous copy out of the
    staging buffer, and results() waits for its own fetch."""
    from forcepho_b200.batch import BatchedProposer
    a, b = _perturbed(batch, 6), _perturbed(batch, 7)
    ref = BatchedProposer(batch, tile_pixels=1024)
    want_a, want_b = ref.evaluate_proposals(a), ref.evaluate_proposals(b)
    bp = BatchedProposer(batch, tile_pixels=1024)
    bp.set_proposals_async(a)
    bp.run()
    bp.fetch_async()
    bp.set_proposals_async(b)
    got_a = bp.results()
    bp.run()
    bp.fetch_async()
    got_b = bp.results()
    for got, want in ((got_a, want_a), (got_b, want_b)):
        for (c, g), (c2, g2) in zip(got, want):
            np.testing.assert_array_equal(c, c2)
            np.testing.assert_array_equal(g, g2)


def test_patch_sent_again_gets_a_new_plan():
    """A proposer kept across uploads of one patch object re-plans for the new
    pixels (here the same shapes, coordinates shifted by 7 px, which the
    allocator may place at the old addresses); plans and batched proposers
    made before the upload refuse to run."""
    from forcepho_b200 import synthetic as S
    from forcepho_b200.batch import BatchedProposer
    from forcepho_b200.proposal import B200Proposer
    p = S.config_multiband(seed=310, n_sources=3, n_bands=2, exp_per_band=1, size=40)
    p.return_residual = False
    p.send_to_device()
    prop = p.scene.get_proposal()
    pr = B200Proposer()
    pr.evaluate_proposal(prop, patch=p)
    old_plan = pr._plan
    bp = BatchedProposer([p], tile_pixels=1024)
    p.xpix = (p.xpix + 7).astype(p.xpix.dtype)
    p.send_to_device()
    c, g = pr.evaluate_proposal(prop, patch=p)
    c2, g2 = B200Proposer().evaluate_proposal(prop, patch=p)
    np.testing.assert_array_equal(c, c2)
    np.testing.assert_array_equal(g, g2)
    with pytest.raises(RuntimeError):
        old_plan.evaluate()
    with pytest.raises(RuntimeError):
        bp.evaluate_proposals([prop])


def test_census_no_within_cutoff_pair_culled(batch):
    from forcepho_b200.batch import BatchedProposer
    bp = BatchedProposer(batch, tile_pixels=1024)
    bp.set_proposals_async(_perturbed(batch, 5))
    kept, active, dropped = bp.count_pairs()
    assert dropped == 0
    assert kept >= active > 0


def test_shuffled_pixels_and_plan_without_coordinates():
    """Pixels shuffled within their exposures and a plan without coordinates:
    tiles are runs of the shuffled order with wide bounding boxes (little is
    culled); results still match the oracle."""
    import torch
    from forcepho_b200 import synthetic as S
    from forcepho_b200.device import Plan, pack_proposals, response_view

    def render(p, prop):
        return O.render(p, prop, precision="f64")
    p = S.config_multiband(seed=60, render=render, n_sources=4, n_bands=2, exp_per_band=1, size=40)
    rng = np.random.default_rng(1)
    for e in range(p.n_exp):
        s0, n = int(p.exposure_start[e]), int(p.exposure_N[e])
        o = s0 + rng.permutation(n)
        for name in ("xpix", "ypix", "data", "ierr"):
            getattr(p, name)[s0:s0 + n] = getattr(p, name)[o]
    p.return_residual = False
    p.send_to_device()
    prop = p.scene.get_proposal().copy()
    prop["q"] *= 0.97
    plan = Plan([p], tile_pixels=1024, compact_tiles=False)
    plan.proposals.copy_(torch.from_numpy(pack_proposals([prop], 1).view(np.uint8).reshape(-1)))
    plan.evaluate(plan.launch(ctas_per_sm=4))
    chi2 = plan.chi2.cpu().numpy()[0, :p.n_bands]
    dchi2 = response_view(plan.response.cpu().numpy()[0], p.n_bands, int(p.n_sources))
    c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
    sc = chi2_scale(chi2, p.data, p.ierr, r64)
    assert chi2_err(chi2, c64, sc) < CHI2_F64
    assert chi2_raw_err(chi2, c64, band_scales(p, r64)) < CHI2_F64
    assert grad_err(dchi2, g64) < GRAD_F64


def test_mixed_tile_classes_in_one_launch(batch):
    """A plan whose exposures take tiles of 256, 512 and 1024 pixels by size
    class runs in one persistent launch: every patch matches the FP64 oracle,
    the census drops no within-cutoff pair, and the per-class autotuner returns
    a valid class list."""
    from forcepho_b200.batch import BatchedProposer
    from forcepho_b200.autotune import Autotuner
    props = _perturbed(batch, 5)
    classes = [(1600, 256), (3000, 512), (2 ** 31 - 1, 1024)]
    bp = BatchedProposer(batch, tile_classes=classes)
    tps = set(int(t) for t in bp.plan.h_tiles["tile_pixels"])
    assert tps == {256, 512, 1024}, tps
    assert bp.launch.tile_pixels == 1024
    res = bp.evaluate_proposals(props)
    for p, prop, (chi2, dchi2) in zip(batch, props, res):
        c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
        assert chi2_raw_err(chi2, c64, band_scales(p, r64)) < CHI2_F64
        assert grad_err(dchi2, g64) < GRAD_F64
    assert bp.count_pairs()[2] == 0
    tuned = BatchedProposer(batch, autotune="classes", tuner=Autotuner(reps=1))
    assert len(tuned.tile_classes) == 3
    assert all(tp in (256, 512, 1024) for _, tp in tuned.tile_classes)
    res2 = tuned.evaluate_proposals(props)
    # tile sizes change the tile origins, hence each pair's FP32 rounding: the
    # two plans agree to twice the tolerance each has against FP64
    for (c1, _), (c2, _), p, prop in zip(res, res2, batch, props):
        r64 = O.evaluate(p, prop, precision="f64", return_residual=True)[2]
        assert chi2_raw_err(c2, c1, band_scales(p, r64)) < 2 * CHI2_F64


def test_swapped_data_is_repacked_before_the_next_replay():
    """The plan's pixel records are a copy of the device data: after
    swap_on_device the next graph replay of a proposer sees the new data."""
    from forcepho_b200 import synthetic as S
    from forcepho_b200.proposal import B200Proposer
    p = S.config_multiband(seed=41, n_sources=3, n_bands=2, exp_per_band=1, size=40)
    p.return_residual = True
    p.send_to_device()
    prop = _perturbed([p], 2)[0]
    pr = B200Proposer()
    chi2a, _, res = pr.evaluate_proposal(prop, patch=p, unpack=False)
    p.swap_on_device()                          # device data <- this residual
    chi2b, dchi2b, _ = pr.evaluate_proposal(prop, patch=p, unpack=False)
    q = S.config_multiband(seed=41, n_sources=3, n_bands=2, exp_per_band=1, size=40)
    q.data = res.astype(np.float32)
    c64, g64, r64 = O.evaluate(q, prop, precision="f64", return_residual=True)
    assert not np.allclose(chi2a, chi2b)
    assert chi2_raw_err(chi2b, c64, band_scales(q, r64)) < CHI2_F64
    assert grad_err(dchi2b, g64) < GRAD_F64
