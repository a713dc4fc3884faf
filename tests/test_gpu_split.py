"""One patch split by exposure, on the GPU: the sub-patches' tiled results add
up to the whole patch's (every exposure keeps its own tiles, so only the
order of the FP64 band sums and the FP32 rounding of each part's gradients
change), and both agree with the FP64 oracle at the parity tolerances.  The
ranks are evaluated one after another in this process: nothing waits on
another rank."""

import numpy as np
import pytest

from oracle import oracle as O
from tolerances import CHI2_F64, GRAD_F64, band_scales, chi2_raw_err, grad_err

pytestmark = pytest.mark.gpu


def _patch(seed):
    from forcepho_b200 import synthetic as S
    p = S.config_multiband(seed=seed)
    p.return_residual = False
    prop = p.scene.get_proposal()
    prop["q"] = np.clip(prop["q"] * 0.97, 0.2, 0.99)
    prop["dec"] -= 3e-6
    return p, prop


@pytest.mark.parametrize("world", [2, 3, 4])
def test_split_patch_adds_up_to_the_whole(world):
    from forcepho_b200 import distributed as D
    from forcepho_b200.proposal import B200Proposer
    p, prop = _patch(21)
    p.send_to_device()
    c_all, g_all = B200Proposer().evaluate_proposal(prop, patch=p)
    c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
    sc = band_scales(p, r64)
    # the all-reduce of the ranks' parts, done here as a plain FP64 sum
    total, seen = None, []
    for rank in range(world):
        sp = D.SplitPatchProposer(p, rank, world)
        seen += sp.exposures
        part = sp.evaluate_local(prop)
        total = part if total is None else total + part
    assert sorted(seen) == list(range(p.n_exp))
    c_sum, g_sum = sp.unpack(total)
    assert chi2_raw_err(c_sum, c_all, sc) < 1e-12
    assert grad_err(g_sum, g_all) < 1e-6
    assert chi2_raw_err(c_sum, c64, sc) < CHI2_F64
    assert grad_err(g_sum, g64) < GRAD_F64


def test_one_rank_split_is_the_whole_patch():
    from forcepho_b200 import distributed as D
    from forcepho_b200.proposal import B200Proposer
    p, prop = _patch(22)
    p.send_to_device()
    c_all, g_all = B200Proposer().evaluate_proposal(prop, patch=p)
    c, g = D.SplitPatchProposer(p, 0, 1).evaluate_proposal(prop)
    np.testing.assert_array_equal(c, c_all)
    np.testing.assert_array_equal(g, g_all)
