"""No-U-Turn sampling of many patches in lockstep.

The reference samples one patch at a time with littlemcmc's NUTS
(forcepho/fitting.py:254-411: ``run_lmc`` with ``get_pot``).  littlemcmc is a
third-party package (littlemcmc == 0.2.0, pinned by the reference's requirements.txt; a standalone copy of PyMC3's NUTS) that is
not installed here; this module restates its published algorithm:

* multinomial NUTS (Betancourt 2017): trajectories grow by doubling in a
  random direction; every leaf is weighted by exp(-dE), proposals are drawn
  by progressive sampling (uniform within a subtree, biased towards the new
  subtree when extending); a subtree stops on a U-turn
  (p_sum . M^-1 p <= 0 at either end) with the additional checks across the
  two halves of each merge, or on a divergence (|dE| > 1000);
* step size: dual averaging (Hoffman & Gelman 2014) towards a target mean
  acceptance of 0.8 during tuning, the averaged step afterwards;
* mass matrix: ``QuadPotentialDiagAdapt`` (a running weighted variance of the
  samples, restarted every ``adaptation_window`` draws from a background
  estimate) or ``QuadPotentialFullAdapt`` (the same for the covariance, with a
  growing window), seeded with ``weight`` virtual samples of the initial
  covariance, as ``get_pot`` sets them up.

The B200 form: all patches advance together, one leapfrog step of every
still-building patch per batched likelihood evaluation (the caller's
``logp_grad(z) -> (lnp[n], grad[P])``, e.g. ``DevicePosterior`` on the GPU);
patches whose tree has stopped are masked out until the slowest finishes.
Positions of all patches are one flat vector (patch i owns ``sizes[i]``
consecutive entries).  Every patch draws from its own random stream, so a
patch's chain does not depend on which other patches share the batch.
"""

import numpy as np

__all__ = ["BatchedNUTS", "DiagAdapt", "FullAdapt", "DualAverage", "DevicePosterior", "run_nuts"]


class _Segments:
    """Per-patch reductions and broadcasts over the flat parameter vector."""

    def __init__(self, sizes):
        self.sizes = np.asarray(sizes, dtype=np.int64)
        if np.any(self.sizes <= 0):
            raise ValueError("every patch needs at least one parameter")
        self.n = len(self.sizes)
        self.starts = np.concatenate([[0], np.cumsum(self.sizes)[:-1]])
        self.P = int(self.sizes.sum())
        self.seg = np.repeat(np.arange(self.n), self.sizes)
        self.slices = [slice(int(a), int(a + b)) for a, b in zip(self.starts, self.sizes)]

    def dot(self, a, b):
        return np.add.reduceat(a * b, self.starts)

    def expand(self, x):
        return np.asarray(x)[self.seg]


class DiagAdapt:
    """Diagonal inverse mass matrix adapted from the running sample variance
    (the published ``QuadPotentialDiagAdapt``), for every patch at once."""

    def __init__(self, segs, init_mean, init_var, weight=10.0, adaptation_window=101):
        self.s = segs
        self.var = np.array(init_var, dtype=np.float64)
        self.fg = _WeightedVariance(segs, init_mean, init_var, weight)
        self.bg = _WeightedVariance(segs)
        self.window = int(adaptation_window)
        self.n_samples = 0

    def velocity(self, p):
        return self.var * p

    def random(self, rngs, mask):
        """Momenta ~ N(0, M) for the patches in ``mask`` (zeros elsewhere)."""
        p = np.zeros(self.s.P)
        for i in np.flatnonzero(mask):
            sl = self.s.slices[i]
            p[sl] = rngs[i].standard_normal(sl.stop - sl.start) / np.sqrt(self.var[sl])
        return p

    def update(self, z, tune):
        if not tune:
            return
        self.fg.add(z)
        self.bg.add(z)
        self.var = self.fg.variance()
        if self.n_samples > 0 and self.n_samples % self.window == 0:
            self.fg, self.bg = self.bg, _WeightedVariance(self.s)
        self.n_samples += 1


class _WeightedVariance:
    def __init__(self, segs, mean=None, var=None, weight=0.0):
        self.w = float(weight)
        self.mean = np.zeros(segs.P) if mean is None else np.array(mean, dtype=np.float64)
        self.raw = np.zeros(segs.P) if var is None else np.array(var, dtype=np.float64) * self.w

    def add(self, x):
        self.w += 1.0
        d_old = x - self.mean
        self.mean += d_old / self.w
        self.raw += d_old * (x - self.mean)

    def variance(self):
        if self.w == 0:
            raise ValueError("no samples")
        return self.raw / self.w


class FullAdapt:
    """Dense inverse mass matrix per patch from the running sample covariance
    (the published ``QuadPotentialFullAdapt``: Cholesky refreshed every
    ``update_window`` draws, windows growing by ``window_multiplier``)."""

    def __init__(self, segs, init_mean, init_cov, weight=10.0, adaptation_window=101,
                 window_multiplier=2.0, update_window=1):
        self.s = segs
        self.cov = [np.array(c, dtype=np.float64) for c in init_cov]
        self.chol = [np.linalg.cholesky(c) for c in self.cov]
        self.fg = [_WeightedCovariance(m, c, weight) for m, c in
                   zip([np.asarray(init_mean)[sl] for sl in segs.slices], self.cov)]
        self.bg = [_WeightedCovariance(np.zeros(len(c))) for c in self.cov]
        self.window = int(adaptation_window)
        self.mult = float(window_multiplier)
        self.update_window = int(update_window)
        self.previous = 0
        self.n_samples = 0

    def velocity(self, p):
        v = np.empty_like(p)
        for i, sl in enumerate(self.s.slices):
            v[sl] = self.cov[i] @ p[sl]
        return v

    def random(self, rngs, mask):
        p = np.zeros(self.s.P)
        for i in np.flatnonzero(mask):
            sl = self.s.slices[i]
            xi = rngs[i].standard_normal(sl.stop - sl.start)
            p[sl] = np.linalg.solve(self.chol[i].T, xi)      # p ~ N(0, cov^-1)
        return p

    def update(self, z, tune):
        if not tune:
            return
        delta = self.n_samples - self.previous
        for i, sl in enumerate(self.s.slices):
            self.fg[i].add(z[sl])
            self.bg[i].add(z[sl])
        if (delta + 1) % self.update_window == 0:
            for i in range(self.s.n):
                c = self.fg[i].covariance()
                try:
                    chol = np.linalg.cholesky(c)
                except np.linalg.LinAlgError:
                    continue                                   # keep the previous matrix
                self.cov[i], self.chol[i] = c, chol
        if delta >= self.window:
            self.fg = self.bg
            self.bg = [_WeightedCovariance(np.zeros(len(c))) for c in self.cov]
            self.previous = self.n_samples
            self.window = int(self.window * self.mult)
        self.n_samples += 1


class _WeightedCovariance:
    def __init__(self, mean, cov=None, weight=0.0):
        self.w = float(weight)
        self.mean = np.array(mean, dtype=np.float64)
        n = len(self.mean)
        self.raw = np.zeros((n, n)) if cov is None else np.array(cov, dtype=np.float64) * self.w

    def add(self, x):
        self.w += 1.0
        d_old = x - self.mean
        self.mean += d_old / self.w
        self.raw += np.outer(d_old, x - self.mean)

    def covariance(self):
        if self.w == 0:
            raise ValueError("no samples")
        return self.raw / self.w


class DualAverage:
    """Per-patch step sizes by dual averaging (Hoffman & Gelman 2014, alg. 5)."""

    def __init__(self, step0, target=0.8, gamma=0.05, k=0.75, t0=10.0):
        step0 = np.asarray(step0, dtype=np.float64)
        self.log_step = np.log(step0)
        self.log_bar = np.log(step0)
        self.hbar = np.zeros_like(step0)
        self.mu = np.log(10.0 * step0)
        self.count = 1
        self.target, self.gamma, self.k, self.t0 = target, gamma, k, t0

    def current(self, tune):
        return np.exp(self.log_step if tune else self.log_bar)

    def update(self, accept_stat, tune):
        if not tune:
            return
        w = 1.0 / (self.count + self.t0)
        self.hbar = (1 - w) * self.hbar + w * (self.target - accept_stat)
        self.log_step = self.mu - self.hbar * np.sqrt(self.count) / self.gamma
        mk = self.count ** -self.k
        self.log_bar = mk * self.log_step + (1 - mk) * self.log_bar
        self.count += 1


def _logbern(rng, log_p):
    if np.isnan(log_p):
        raise FloatingPointError("log_p can't be nan")
    return np.log(rng.random()) < log_p


class BatchedNUTS:
    """NUTS for ``n`` independent targets evaluated together.

    Parameters
    ----------
    logp_grad : callable(z[P]) -> (lnp[n], dlnp/dz[P]); called once per
        leapfrog step with every patch's position (patches not stepping keep
        their previous position)
    sizes : parameters per patch
    potential : "diag" or "full"; init_cov per patch (array (n_i,) for diag,
        (n_i, n_i) for full) or None for the identity; ``weight`` virtual
        samples seed the adaptation, as ``get_pot`` does
    max_treedepth, target_accept, step_scale (initial step = step_scale /
        n_i^(1/4)), max_energy_change: as littlemcmc's NUTS defaults
    seed, streams : patch i draws from ``np.random.default_rng([seed, streams[i]])``
        (default streams[i] = i)
    """

    def __init__(self, logp_grad, sizes, potential="diag", init_mean=None, init_cov=None, weight=10.0,
                 max_treedepth=10, target_accept=0.8, step_scale=0.25, max_energy_change=1000.0, seed=0,
                 streams=None):
        self.f = logp_grad
        self.s = _Segments(sizes)
        self.max_treedepth = int(max_treedepth)
        self.emax = float(max_energy_change)
        streams = range(self.s.n) if streams is None else streams
        if len(streams) != self.s.n:
            raise ValueError("one random stream per patch")
        self.rngs = [np.random.default_rng([int(seed), int(k)]) for k in streams]
        mean = np.zeros(self.s.P) if init_mean is None else np.asarray(init_mean, dtype=np.float64)
        if potential == "diag":
            var = np.ones(self.s.P)
            if init_cov is not None:
                for sl, c in zip(self.s.slices, init_cov):
                    c = np.asarray(c, dtype=np.float64)
                    var[sl] = np.diag(c) if c.ndim == 2 else c
            self.pot = DiagAdapt(self.s, mean, var, weight)
        elif potential == "full":
            covs = [np.eye(n) for n in self.s.sizes] if init_cov is None else \
                [np.asarray(c, dtype=np.float64) for c in init_cov]
            self.pot = FullAdapt(self.s, mean, covs, weight)
        else:
            raise ValueError("potential must be 'diag' or 'full'")
        self.step = DualAverage(step_scale / self.s.sizes.astype(np.float64) ** 0.25, target=target_accept)
        self.n_evals = 0

    # ---------------------------------------------------------------------
    def _eval(self, z):
        lnp, g = self.f(z)
        self.n_evals += 1
        return np.asarray(lnp, dtype=np.float64), np.asarray(g, dtype=np.float64)

    def _energy(self, lnp, p):
        return -lnp + 0.5 * self.s.dot(p, self.pot.velocity(p))

    def _uturn(self, psum, pa, pb):
        """p_sum . v(a) <= 0 or p_sum . v(b) <= 0, per patch."""
        return (self.s.dot(psum, self.pot.velocity(pa)) <= 0) | (self.s.dot(psum, self.pot.velocity(pb)) <= 0)

    def iterate(self, z, lnp, grad, tune):
        """One NUTS transition of every patch from (z, lnp, grad).
        Returns the new (z, lnp, grad) and a dict of per-patch statistics."""
        s, n = self.s, self.s.n
        X = s.expand
        eps = self.step.current(tune)
        everyone = np.ones(n, dtype=bool)
        p0 = self.pot.random(self.rngs, everyone)
        H0 = self._energy(lnp, p0)
        # the whole tree: left/right edges (position, momentum, gradient), p_sum,
        # proposal and log total weight
        L = [z.copy(), p0.copy(), grad.copy()]
        R = [z.copy(), p0.copy(), grad.copy()]
        psum = p0.copy()
        prop_z, prop_g, prop_lnp = z.copy(), grad.copy(), lnp.copy()
        log_w = np.zeros(n)
        active = everyone.copy()
        diverging = np.zeros(n, dtype=bool)
        turning = np.zeros(n, dtype=bool)
        depth = np.zeros(n, dtype=np.int64)
        acc_sum = np.zeros(n)
        n_leaves = np.zeros(n, dtype=np.int64)
        prop_energy = H0.copy()

        for d in range(self.max_treedepth):
            if not active.any():
                break
            direction = np.zeros(n)
            for i in np.flatnonzero(active):
                direction[i] = 1.0 if self.rngs[i].random() > 0.5 else -1.0
            fwd = direction > 0
            FX = X(fwd)
            # frontier: the edge the new subtree grows from
            Ez = np.where(FX, R[0], L[0])
            Ep = np.where(FX, R[1], L[1])
            Eg = np.where(FX, R[2], L[2])
            Elnp = np.zeros(n)
            step = X(eps * direction)
            # subtree slots, one per level: start/far-side momentum, p_sum,
            # proposal (z, grad, lnp, energy) and log weight
            slot = [None] * (d + 1)
            ok = active.copy()                  # still building this subtree
            cur = None
            for k in range(2 ** d):
                live = ok.copy()
                if not live.any():
                    break
                LX = X(live)
                p_half = Ep + 0.5 * step * Eg
                z1 = np.where(LX, Ez + step * self.pot.velocity(p_half), Ez)
                lnp1, g1 = self._eval(z1)
                p1 = p_half + 0.5 * step * g1
                H1 = self._energy(lnp1, p1)
                dE = H1 - H0
                dE = np.where(np.isnan(dE), np.inf, dE)
                div = live & (np.abs(dE) > self.emax)
                acc = np.where(div, 0.0, np.minimum(1.0, np.exp(np.minimum(-dE, 0.0))))
                acc_sum += np.where(live, acc, 0.0)
                n_leaves += live
                diverging |= div
                ok &= ~div
                good = live & ~div
                GX = X(good)
                Ez, Ep, Eg = np.where(GX, z1, Ez), np.where(GX, p1, Ep), np.where(GX, g1, Eg)
                Elnp = np.where(good, lnp1, Elnp)
                leaf = dict(lp=p1, rp=p1, psum=p1, z=z1, g=g1, lnp=lnp1, H=H1, lw=-dE)
                cur = _select(good, GX, leaf, cur)
                # binary-counter merges: bit l of k set -> slot[l] is the left sibling
                level, kk = 0, k
                while kk & 1:
                    cur = self._merge(slot[level], cur, level, ok)
                    kk >>= 1
                    level += 1
                slot[level] = cur
            # extend the whole tree with the completed subtree
            comp = ok & active
            sub = slot[d]
            depth = np.where(active, d + 1, depth)
            if comp.any():
                CX = X(comp)
                for i in np.flatnonzero(comp):
                    if _logbern(self.rngs[i], sub["lw"][i] - log_w[i]):
                        sl = s.slices[i]
                        prop_z[sl], prop_g[sl] = sub["z"][sl], sub["g"][sl]
                        prop_lnp[i], prop_energy[i] = sub["lnp"][i], sub["H"][i]
                log_w = np.where(comp, np.logaddexp(log_w, sub["lw"]), log_w)
                # leftmost/rightmost halves before the update (the new subtree's
                # start side touches the old tree)
                lm_begin = np.where(FX, L[1], sub["rp"])
                lm_end = np.where(FX, R[1], sub["lp"])
                rm_begin = np.where(FX, sub["lp"], L[1])
                rm_end = np.where(FX, sub["rp"], R[1])
                lm_psum = np.where(FX, psum, sub["psum"])
                rm_psum = np.where(FX, sub["psum"], psum)
                new_psum = psum + sub["psum"]
                psum = np.where(CX, new_psum, psum)
                upd_r, upd_l = X(comp & fwd), X(comp & ~fwd)
                R = [np.where(upd_r, Ez, R[0]), np.where(upd_r, Ep, R[1]), np.where(upd_r, Eg, R[2])]
                L = [np.where(upd_l, Ez, L[0]), np.where(upd_l, Ep, L[1]), np.where(upd_l, Eg, L[2])]
                t0 = self._uturn(psum, L[1], R[1])
                ps1 = lm_psum + rm_begin
                t1 = self._uturn(ps1, lm_begin, rm_begin)
                ps2 = lm_end + rm_psum
                t2 = self._uturn(ps2, lm_end, rm_end)
                turn_top = comp & (t0 | t1 | t2)
                turning |= turn_top
            else:
                turn_top = np.zeros(n, dtype=bool)
            turning |= active & ~ok & ~diverging
            active = comp & ~turn_top

        stats = dict(depth=depth, n_steps=n_leaves, mean_tree_accept=acc_sum / np.maximum(n_leaves, 1),
                     diverging=diverging, turning=turning, energy_error=prop_energy - H0,
                     energy=prop_energy, step_size=eps.copy(), lnp=prop_lnp.copy(),
                     max_depth_reached=active)
        return prop_z, prop_lnp, prop_g, stats

    def _merge(self, t1, t2, level, ok):
        """Merge adjacent subtrees t1 (start side) and t2 for the patches in
        ``ok``; patches whose merged tree makes a U-turn leave ``ok``."""
        s = self.s
        X = s.expand
        psum = t1["psum"] + t2["psum"]
        turn = self._uturn(psum, t1["lp"], t2["rp"])
        if level > 0:
            ps1 = t1["psum"] + t2["lp"]
            turn |= self._uturn(ps1, t1["lp"], t2["lp"])
            ps2 = t1["rp"] + t2["psum"]
            turn |= self._uturn(ps2, t1["rp"], t2["rp"])
        lw = np.logaddexp(t1["lw"], t2["lw"])
        take2 = np.zeros(s.n, dtype=bool)
        for i in np.flatnonzero(ok):
            take2[i] = _logbern(self.rngs[i], t2["lw"][i] - lw[i])
        T2 = X(take2)
        merged = dict(lp=t1["lp"], rp=t2["rp"], psum=psum,
                      z=np.where(T2, t2["z"], t1["z"]), g=np.where(T2, t2["g"], t1["g"]),
                      lnp=np.where(take2, t2["lnp"], t1["lnp"]), H=np.where(take2, t2["H"], t1["H"]), lw=lw)
        ok &= ~turn
        return merged

    # ---------------------------------------------------------------------
    def sample(self, z0, draws, tune=0, discard_tuned_samples=True):
        """Run ``tune`` adapting and ``draws`` fixed transitions from z0.
        Returns (trace [n_kept, P], list of per-transition stats dicts)."""
        z = np.array(z0, dtype=np.float64)
        lnp, g = self._eval(z)
        trace, stats = [], []
        for it in range(tune + draws):
            is_tune = it < tune
            z, lnp, g, st = self.iterate(z, lnp, g, is_tune)
            self.step.update(st["mean_tree_accept"], is_tune)
            self.pot.update(z, is_tune)
            st["tune"] = is_tune
            if not (is_tune and discard_tuned_samples):
                trace.append(z.copy())
                stats.append(st)
        self.state = (z, lnp, g)            # where a further call to iterate() continues
        return np.array(trace).reshape(-1, self.s.P), stats


def _select(mask, maskX, new, old):
    """Per patch, ``new`` where mask else ``old`` (old may be None)."""
    if old is None:
        return {k: v.copy() for k, v in new.items()}
    out = {}
    for k, v in new.items():
        m = maskX if v.shape == maskX.shape else mask
        out[k] = np.where(m, v, old[k])
    return out


class DevicePosterior:
    """``logp_grad`` of many device patches for ``BatchedNUTS``: lnp and its
    gradient in the unconstrained parameters z (sigmoid transform of each
    parameter to its bounds, log-Jacobian included), one batched device pass
    (``DeviceHMC.gradient``: device splines and proposals, the tile kernel,
    the per-patch lnp/gradient assembly)."""

    def __init__(self, hmc):
        import torch
        self.hmc = hmc
        self._torch = torch
        self.sizes = [sl.stop - sl.start for sl in hmc.slices]

    def __call__(self, z):
        t = self._torch
        self.hmc.z.copy_(t.from_numpy(np.ascontiguousarray(z, dtype=np.float64)))
        self.hmc.gradient()
        return self.hmc.lnp.cpu().numpy().copy(), self.hmc.grad.cpu().numpy().copy()

    def start(self):
        return self.hmc.z.cpu().numpy().copy()


def run_nuts(patches, theta0, n_draws, warmup=(10,), full=False, weight=10, z_cov=None, max_treedepth=10,
             discard_tuned_samples=True, random_seed=0xDEADBEEF, bounds=None, init_mass="identity",
             streams=None):
    """NUTS on many device patches at once, the batched counterpart of the
    reference's ``run_lmc`` (forcepho/fitting.py:254-341) with ``get_pot``.

    Parameters
    ----------
    patches, theta0, bounds : as ``forcepho_b200.hmc.DeviceHMC`` (device
        patches, starting scene parameters per patch, sampling bounds)
    n_draws : draws kept after ``warmup[0]`` adapting transitions
    full : dense (True) or diagonal mass-matrix adaptation; ``weight``
        virtual samples of the initial covariance
    z_cov : per patch initial covariance in the unconstrained space (or None)
    init_mass : without ``z_cov``, "identity" (the reference's default) or
        "curvature" (the inverse Hessian diagonal at the start)
    random_seed, streams : patch i draws from the random stream
        [random_seed, streams[i]] (default streams[i] = i)

    Returns (chains, sampler, stats): per patch an array (n_kept, n_params)
    of constrained parameters, the ``BatchedNUTS`` and its per-transition
    statistics."""
    from .hmc import DeviceHMC
    hmc = DeviceHMC(patches, theta0, bounds=bounds, n_steps=1, max_traj=1)
    post = DevicePosterior(hmc)
    z0 = post.start()
    cov = z_cov
    if cov is None and init_mass == "curvature":
        var = hmc.estimate_inv_mass().cpu().numpy()
        cov = [np.diag(var[sl]) if full else var[sl] for sl in hmc.slices]
    nuts = BatchedNUTS(post, post.sizes, potential="full" if full else "diag", init_mean=z0, init_cov=cov,
                       weight=weight, max_treedepth=max_treedepth, seed=random_seed, streams=streams)
    trace, stats = nuts.sample(z0, n_draws, tune=int(warmup[0]), discard_tuned_samples=discard_tuned_samples)
    lo, hi = hmc.lower.cpu().numpy(), hmc.upper.cpu().numpy()
    q = lo + (hi - lo) / (1.0 + np.exp(-trace))
    chains = [q[:, sl].copy() for sl in hmc.slices]
    return chains, nuts, stats
