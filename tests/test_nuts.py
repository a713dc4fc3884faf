"""The lockstep multinomial NUTS (forcepho_b200/nuts.py) on the CPU.

* A plain recursive single-chain NUTS, written here in the shape of the
  published algorithm (doubling with a recursive subtree build, progressive
  sampling, the additional U-turn checks), with the same random-draw order,
  must reproduce the lockstep sampler's chains bit for bit;
* batched chains equal the same chains run one patch at a time;
* on Gaussian targets the draws have the right mean and covariance and the
  adapted step size reaches the target acceptance.
"""

import numpy as np
import pytest

from forcepho_b200.nuts import BatchedNUTS, DiagAdapt, DualAverage, _Segments


def gaussian_targets(dims, seed=0):
    """Independent Gaussians N(mu_i, C_i); returns (logp_grad over the flat vector, mus, covs)."""
    rng = np.random.default_rng(seed)
    mus, precs, covs = [], [], []
    for d in dims:
        A = rng.normal(size=(d, d))
        C = A @ A.T / d + np.diag(rng.uniform(0.2, 2.0, d))
        mus.append(rng.normal(size=d))
        covs.append(C)
        precs.append(np.linalg.inv(C))
    seg = _Segments(dims)

    def f(z):
        lnp = np.zeros(len(dims))
        g = np.zeros_like(z)
        for i, sl in enumerate(seg.slices):
            r = z[sl] - mus[i]
            g[sl] = -precs[i] @ r
            lnp[i] = -0.5 * r @ precs[i] @ r
        return lnp, g
    return f, mus, covs


# --- a plain recursive NUTS for one chain (the test's restatement) ---------
class RecursiveNUTS:
    def __init__(self, f1, dim, seed, index, max_treedepth=10, emax=1000.0, weight=10.0):
        self.f1 = f1                     # z -> (lnp scalar, grad)
        self.rng = np.random.default_rng([seed, index])
        seg = _Segments([dim])
        self.pot = DiagAdapt(seg, np.zeros(dim), np.ones(dim), weight)
        self.step = DualAverage(np.array([0.25 / dim ** 0.25]))
        self.max_treedepth, self.emax = max_treedepth, emax

    def dot(self, a, b):
        return float(np.add.reduceat(a * b, [0])[0])

    def v(self, p):
        return self.pot.velocity(p)

    def energy(self, lnp, p):
        return -lnp + 0.5 * self.dot(p, self.v(p))

    def turn(self, psum, a, b):
        return self.dot(psum, self.v(a)) <= 0 or self.dot(psum, self.v(b)) <= 0

    def logbern(self, x):
        return np.log(self.rng.random()) < x

    def leaf(self, edge, eps):
        z, p, g = edge
        p_half = p + 0.5 * eps * g
        z1 = z + eps * self.v(p_half)
        lnp1, g1 = self.f1(z1)
        p1 = p_half + 0.5 * eps * g1
        return z1, p1, g1, lnp1

    def build(self, edge, depth, eps):
        """Returns (subtree dict, frontier edge, diverging, turning)."""
        if depth == 0:
            z1, p1, g1, lnp1 = self.leaf(edge, eps)
            H1 = self.energy(lnp1, p1)
            dE = H1 - self.H0
            if np.isnan(dE):
                dE = np.inf
            self.n_leaves += 1
            if abs(dE) > self.emax:
                return None, edge, True, False
            self.acc += min(1.0, np.exp(min(-dE, 0.0)))
            t = dict(lp=p1, rp=p1, psum=p1.copy(), z=z1, g=g1, lnp=lnp1, H=H1, lw=-dE)
            return t, (z1, p1, g1), False, False
        t1, e1, div, turn = self.build(edge, depth - 1, eps)
        if div or turn:
            return t1, e1, div, turn
        t2, e2, div, turn = self.build(e1, depth - 1, eps)
        if div or turn:
            return t2, e2, div, turn
        psum = t1["psum"] + t2["psum"]
        turn = self.turn(psum, t1["lp"], t2["rp"])
        if depth - 1 > 0:
            turn = turn or self.turn(t1["psum"] + t2["lp"], t1["lp"], t2["lp"])
            turn = turn or self.turn(t1["rp"] + t2["psum"], t1["rp"], t2["rp"])
        lw = np.logaddexp(t1["lw"], t2["lw"])
        pick = t2 if self.logbern(t2["lw"] - lw) else t1
        t = dict(lp=t1["lp"], rp=t2["rp"], psum=psum, z=pick["z"], g=pick["g"], lnp=pick["lnp"], H=pick["H"], lw=lw)
        return t, e2, False, turn

    def iterate(self, z, lnp, g, tune):
        eps = float(self.step.current(tune)[0])
        p0 = self.pot.random([self.rng], np.array([True]))
        self.H0 = self.energy(lnp, p0)
        self.acc, self.n_leaves = 0.0, 0
        left = right = (z, p0, g)
        psum = p0.copy()
        prop = (z, g, lnp)
        log_w = 0.0
        for _ in range(self.max_treedepth):
            fwd = self.rng.random() > 0.5
            edge = right if fwd else left
            sub, front, div, turn = self.build(edge, _, eps if fwd else -eps)
            if div or turn:
                break
            if self.logbern(sub["lw"] - log_w):
                prop = (sub["z"], sub["g"], sub["lnp"])
            log_w = np.logaddexp(log_w, sub["lw"])
            if fwd:
                lm_b, lm_e, rm_b, rm_e, lm_ps, rm_ps = left[1], right[1], sub["lp"], sub["rp"], psum, sub["psum"]
                right = front
            else:
                lm_b, lm_e, rm_b, rm_e, lm_ps, rm_ps = sub["rp"], sub["lp"], left[1], right[1], sub["psum"], psum
                left = front
            psum = psum + sub["psum"]
            t0 = self.turn(psum, left[1], right[1])
            t1 = self.turn(lm_ps + rm_b, lm_b, rm_b)
            t2 = self.turn(lm_e + rm_ps, lm_e, rm_e)
            if t0 or t1 or t2:
                break
        return prop, self.acc / max(self.n_leaves, 1)

    def sample(self, z0, draws, tune):
        z = np.array(z0, dtype=np.float64)
        lnp, g = self.f1(z)
        out = []
        for it in range(tune + draws):
            is_tune = it < tune
            (z, g, lnp), acc = self.iterate(z, lnp, g, is_tune)
            self.step.update(np.array([acc]), is_tune)
            self.pot.update(z, is_tune)
            if not is_tune:
                out.append(z.copy())
        return np.array(out)


def _one(f, dims, i):
    seg = _Segments(dims)
    sl = seg.slices[i]

    def f1(zi):
        z = np.zeros(seg.P)
        z[sl] = zi
        lnp, g = f(z)
        return float(lnp[i]), g[sl].copy()
    return f1


def test_lockstep_equals_recursive_restatement():
    dims = [3, 1, 5, 2]
    f, mus, covs = gaussian_targets(dims, seed=1)
    z0 = np.concatenate([m + 1.0 for m in mus])
    nuts = BatchedNUTS(f, dims, seed=7, max_treedepth=6)
    trace, stats = nuts.sample(z0, draws=25, tune=15)
    seg = _Segments(dims)
    for i, sl in enumerate(seg.slices):
        ref = RecursiveNUTS(_one(f, dims, i), dims[i], seed=7, index=i, max_treedepth=6)
        want = ref.sample(z0[sl], draws=25, tune=15)
        np.testing.assert_array_equal(trace[:, sl], want)


def test_batched_equals_one_patch_at_a_time():
    dims = [4, 2, 6]
    f, mus, covs = gaussian_targets(dims, seed=2)
    z0 = np.concatenate([m - 0.5 for m in mus])
    both = BatchedNUTS(f, dims, seed=3, potential="full")
    tb, sb = both.sample(z0, draws=20, tune=20)
    seg = _Segments(dims)
    for i, sl in enumerate(seg.slices):
        fi = _one(f, dims, i)

        def g1(z, fi=fi):
            lnp, g = fi(z)
            return np.array([lnp]), g
        one = BatchedNUTS(g1, [dims[i]], seed=3, potential="full", streams=[i])
        t1, s1 = one.sample(z0[sl], draws=20, tune=20)
        np.testing.assert_array_equal(tb[:, sl], t1)
        np.testing.assert_array_equal([s["depth"][i] for s in sb], [s["depth"][0] for s in s1])


@pytest.mark.parametrize("potential", ["diag", "full"])
def test_gaussian_moments_and_acceptance(potential):
    dims = [3, 2]
    f, mus, covs = gaussian_targets(dims, seed=4)
    z0 = np.concatenate(mus)
    nuts = BatchedNUTS(f, dims, seed=11, potential=potential)
    trace, stats = nuts.sample(z0, draws=1500, tune=500)
    seg = _Segments(dims)
    for i, sl in enumerate(seg.slices):
        x = trace[:, sl]
        sd = np.sqrt(np.diag(covs[i]))
        # NUTS draws are close to independent here; allow a generous error for autocorrelation
        assert np.all(np.abs(x.mean(axis=0) - mus[i]) < 6 * sd / np.sqrt(len(x)) + 0.05 * sd)
        np.testing.assert_allclose(np.cov(x.T).reshape(covs[i].shape), covs[i], rtol=0.25, atol=0.1 * sd.max() ** 2)
    acc = np.mean([s["mean_tree_accept"] for s in stats], axis=0)
    assert np.all(np.abs(acc - 0.8) < 0.12), acc
    assert not np.any([s["diverging"] for s in stats])


def test_divergences_are_flagged_and_rejected():
    # a hard wall: lnp = -inf past |z| > 1 for one patch, a plain Gaussian for the other
    def f(z):
        lnp = np.array([-0.5 * z[0] ** 2, -0.5 * z[1] ** 2])
        if abs(z[0]) > 1.0:
            lnp[0] = -np.inf
        return lnp, -z.copy()
    nuts = BatchedNUTS(f, [1, 1], seed=5)
    nuts.step.log_step[:] = np.log(2.0)          # large steps run into the wall
    z = np.array([0.9, 0.0])
    lnp, g = f(z)
    seen = False
    for _ in range(30):
        z, lnp, g, st = nuts.iterate(z, lnp, g, tune=False)
        seen |= bool(st["diverging"][0])
        assert abs(z[0]) <= 1.0 and np.isfinite(lnp).all()
    assert seen
