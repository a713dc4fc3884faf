"""NUTS over device patches (forcepho_b200/nuts.py with the device posterior):
patches sampled together give exactly the chains they give alone (each
patch's likelihood, gradient and random stream are independent of the
batch), and the draws stay finite and inside the bounds without divergences.
Statistical correctness of the sampler is tested on Gaussian targets on the
CPU (test_nuts.py)."""

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _patches():
    from forcepho_b200 import synthetic as S

    def render(p, prop):
        return O.render(p, prop, precision="f64")
    out, theta0 = [], []
    for i, (ns, nb) in enumerate([(2, 2), (1, 3)]):
        p = S.config_multiband(seed=40 + i, render=render, n_sources=ns, n_bands=nb, exp_per_band=1, size=40)
        p.return_residual = False
        p.send_to_device()
        out.append(p)
        theta0.append(p.scene.get_all_source_params().copy())
    return out, theta0


def test_nuts_batch_matches_single_patches_and_stays_in_bounds():
    from forcepho_b200.hmc import default_bounds
    from forcepho_b200.nuts import run_nuts
    patches, theta0 = _patches()
    kw = dict(n_draws=6, warmup=(6,), max_treedepth=5, random_seed=11)
    chains, nuts, stats = run_nuts(patches, theta0, **kw)
    assert nuts.n_evals > 12
    for i, (p, th) in enumerate(zip(patches, theta0)):
        alone, _, st1 = run_nuts([p], [th], streams=[i], **kw)
        np.testing.assert_array_equal(chains[i], alone[0])
        lo, hi = default_bounds(p, th)
        for c in (chains[i], alone[0]):
            assert np.all(np.isfinite(c))
            assert np.all(c >= lo) and np.all(c <= hi)
    # a healthy sampler: no divergences, finite lnp, trajectories mostly accepted
    assert not np.any([s["diverging"] for s in stats])
    assert np.all(np.isfinite([s["lnp"] for s in stats]))
    assert np.mean([s["mean_tree_accept"] for s in stats]) > 0.3
    assert all(np.all(s["step_size"] > 0) for s in stats)
