"""Device-resident HMC over many patches.

The reference samples one patch at a time on the host: littlemcmc's NUTS calls
``model.lnprob_and_grad(z)`` (forcepho/fitting.py:254-341), which transforms the
parameters, evaluates the spline amplitudes and packs the proposal on the host,
copies it to the device, runs the kernel and copies chi2 and the gradient back
(forcepho/model.py:302-368).  ``DeviceHMC`` keeps positions, momenta and
gradients of all patches on the device; one trajectory (``n_steps`` leapfrog
steps, a gradient evaluation of every patch per step) is a single CUDA-graph
replay of: transform + proposal (device splines) -> Gaussian setup -> tile
kernel -> reduction -> lnp/gradient -> kick/drift, ending in a per-patch
Metropolis test.

Fixed-length HMC with a diagonal mass matrix stands in for NUTS.  The mass
matrix is estimated from the curvature of lnp at the start (Hutchinson probes
of the Hessian diagonal with the analytic gradient) and, optionally, from the
variance of the warm-up draws.  The step size of each patch is adapted during
warm-up trajectories by dual averaging (Hoffman & Gelman 2014, algorithm 5,
as in Stan and in littlemcmc's NUTS) towards a target acceptance
probability; after warm-up each patch keeps its averaged step size.  The
adaptation runs as device tensor operations between graph replays, with no
host synchronisation.
"""

import ctypes

import numpy as np
import torch

from . import _native as N
from .device import Plan, to_device_bytes
from .kernel_limits import NPARAMS
from .splines import default_splines

__all__ = ["DeviceHMC", "default_bounds", "spline_table"]


def spline_table(device, splines=None):
    """Device copies of the spline knots/coefficients and the C struct naming them."""
    sp = splines or default_splines()
    tx, ty, c, kx, ky = sp.tck()
    keep = [torch.tensor(np.asarray(tx, np.float64), device=device),
            torch.tensor(np.asarray(ty, np.float64), device=device),
            torch.tensor(np.ascontiguousarray(c, np.float64), device=device)]
    tab = N.SplineTable(int(c.shape[0]), len(tx), len(ty), int(kx), int(ky), 0,
                        keep[0].data_ptr(), keep[1].data_ptr(), keep[2].data_ptr())
    tab._keep = keep
    return tab


def source_cos_dec(patch, n_sources):
    """cos(dec) at each source, from the patch's own astrometry of its first
    exposure: CW (pixels per degree) = 3600 D (pixels per arcsec) diag(cos dec, 1)."""
    D = np.asarray(patch.D, np.float64)[0, :n_sources]
    CW = np.asarray(patch.CW, np.float64)[0, :n_sources]
    c = np.linalg.solve(D, CW)[:, 0, 0] / 3600.0
    return np.where(np.isfinite(c) & (c > 0), c, 1.0)


def default_bounds(patch, theta0):
    """Sampling bounds around a starting point, per parameter of ``theta0``
    (one patch): flux in (0, 3 f0 + 1], positions within 0.3 arcsec (in RA
    degrees scaled by 1 / cos dec at each source), q in [0.2, 1], pa in
    [-2, 2] rad, sersic in the spline table's range, rhalf in [0.03, 0.6]
    arcsec."""
    nb = patch.n_bands
    nper = nb + NPARAMS - 1
    th = np.asarray(theta0, np.float64).reshape(-1, nper)
    lo, hi = np.zeros_like(th), np.zeros_like(th)
    lo[:, :nb] = 0.0
    hi[:, :nb] = 3.0 * np.abs(th[:, :nb]) + 1.0
    cosd = source_cos_dec(patch, len(th))
    dpos = 0.3 / 3600.0
    lo[:, nb], hi[:, nb] = th[:, nb] - dpos / cosd, th[:, nb] + dpos / cosd
    lo[:, nb + 1], hi[:, nb + 1] = th[:, nb + 1] - dpos, th[:, nb + 1] + dpos
    lo[:, nb + 2], hi[:, nb + 2] = 0.2, 1.0
    lo[:, nb + 3], hi[:, nb + 3] = -2.0, 2.0
    lo[:, nb + 4], hi[:, nb + 4] = 0.81, 6.19
    lo[:, nb + 5], hi[:, nb + 5] = 0.03, 0.6
    return lo.reshape(-1), hi.reshape(-1)


class DeviceHMC:
    """HMC of every patch of a list of device patches, all state on the device.

    Parameters
    ----------
    patches : device patches (``send_to_device``-ed, ``return_residual`` False)
    theta0 : list of starting scene-parameter vectors, one per patch
    bounds : list of (lower, upper) per patch, or None for ``default_bounds``
    n_steps : leapfrog steps per trajectory
    max_traj : trajectories the pre-drawn random numbers cover
    """

    def __init__(self, patches, theta0, bounds=None, n_steps=16, max_traj=256, seed=0, tile_pixels=1024,
                 ctas_per_sm=3, step_size=0.1):
        self.L = N.load()
        self.patches = list(patches)
        self.n = len(self.patches)
        self.n_steps = int(n_steps)
        self.max_traj = int(max_traj)
        self.plan = Plan(self.patches, tile_pixels=tile_pixels)
        self.launch = self.plan.launch(ctas_per_sm=ctas_per_sm)
        dev = self.plan.device
        self.device = dev
        # parameter layout
        hp = np.zeros(self.n, dtype=N.hmc_patch_dtype)
        off = 0
        self.slices = []
        for i, p in enumerate(self.patches):
            npar = int(p.n_sources) * (p.n_bands + NPARAMS - 1)
            hp[i] = (off, int(p.n_sources), p.n_bands)
            self.slices.append(slice(off, off + npar))
            off += npar
        self.n_params = off
        self.d_hp = to_device_bytes(hp, dev)
        lo = np.zeros(off)
        hi = np.zeros(off)
        z0 = np.zeros(off)
        for i, p in enumerate(self.patches):
            th = np.asarray(theta0[i], np.float64)
            l, h = bounds[i] if bounds is not None else default_bounds(p, th)
            lo[self.slices[i]], hi[self.slices[i]] = l, h
            y = np.clip((th - l) / (h - l), 1e-6, 1 - 1e-6)
            z0[self.slices[i]] = np.log(y) - np.log1p(-y)
        f64 = dict(dtype=torch.float64, device=dev)
        self.lower = torch.tensor(lo, **f64)
        self.upper = torch.tensor(hi, **f64)
        self.z = torch.tensor(z0, **f64)
        self.p = torch.zeros(off, **f64)
        self.grad = torch.zeros(off, **f64)
        self.z0 = torch.zeros(off, **f64)
        self.grad0 = torch.zeros(off, **f64)
        self.theta = torch.zeros(off, **f64)
        self.jac = torch.zeros(off, **f64)
        self.inv_mass = torch.ones(off, **f64)
        self.eps = torch.full((self.n,), float(step_size), **f64)
        self.lnp = torch.zeros(self.n, **f64)
        self.lnp0 = torch.zeros(self.n, **f64)
        self.h0 = torch.zeros(self.n, **f64)
        self.energy_error = torch.zeros(self.n, **f64)
        self.accepted = torch.zeros(self.n, dtype=torch.int32, device=dev)
        self.traj = torch.zeros(1, dtype=torch.int64, device=dev)
        g = torch.Generator(device=dev)
        g.manual_seed(int(seed))
        self.normals = torch.randn((self.max_traj, off), generator=g, **f64)
        self.uniforms = torch.rand((self.max_traj, self.n), generator=g, **f64).clamp_(min=1e-300)
        self.tab = spline_table(dev)
        self.state = N.HMCState(off, self.z.data_ptr(), self.p.data_ptr(), self.grad.data_ptr(),
                                self.z0.data_ptr(), self.grad0.data_ptr(), self.inv_mass.data_ptr(),
                                self.eps.data_ptr(), self.lnp.data_ptr(), self.lnp0.data_ptr(),
                                self.h0.data_ptr(), self.energy_error.data_ptr(), self.accepted.data_ptr(),
                                self.normals.data_ptr(), self.uniforms.data_ptr(), self.traj.data_ptr(),
                                self.max_traj)
        self.graph = None
        self.n_evals = 0

    # --- launch sequences (all asynchronous on the current stream) ---
    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def gradient(self):
        """Queue: transform + proposals, likelihood, lnp and dlnp/dz at self.z."""
        s = self._stream()
        N.check(self.L.fp_hmc_prepare(self.d_hp.data_ptr(), self.n, self.z.data_ptr(), self.lower.data_ptr(),
                                      self.upper.data_ptr(), ctypes.byref(self.tab), self.plan.proposals.data_ptr(),
                                      self.theta.data_ptr(), self.jac.data_ptr(), s), "fp_hmc_prepare")
        self.plan.evaluate(self.launch)
        N.check(self.L.fp_hmc_lnprob(self.d_hp.data_ptr(), self.n, self.z.data_ptr(), self.jac.data_ptr(),
                                     self.plan.chi2.data_ptr(), self.plan.response.data_ptr(), 1, 1,
                                     self.lnp.data_ptr(), self.grad.data_ptr(), s), "fp_hmc_lnprob")

    def _leapfrog(self, stage):
        N.check(self.L.fp_hmc_leapfrog(self.d_hp.data_ptr(), self.n, ctypes.byref(self.state), stage,
                                       self._stream()), "fp_hmc_leapfrog")

    def _trajectory(self):
        self._leapfrog(N.HMC_BEGIN)
        for i in range(self.n_steps):
            self.gradient()
            if i < self.n_steps - 1:
                self._leapfrog(N.HMC_STEP)
        self._leapfrog(N.HMC_END)

    def capture(self):
        self.gradient()           # eager: kernel attributes, and lnp/grad at the start
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        saved = self.traj.clone()
        with torch.cuda.graph(g):
            self._trajectory()
        torch.cuda.synchronize()
        # capture does not execute; nothing to undo, but keep the counter explicit
        self.traj.copy_(saved)
        self.graph = g
        return g

    def run(self, n_traj, adapt=False, target=0.8, record=None):
        """Run n_traj trajectories (graph replays).

        adapt : dual-averaging step-size adaptation of every patch towards a
            mean acceptance probability ``target`` after each trajectory; the
            averaged step size is installed by ``end_adaptation``.
        record : optional {trajectory index within this call: device tensor}
            that receives a copy of the positions z after that trajectory
            (a device copy, no host synchronisation)."""
        self.plan.check_current()
        if self.graph is None:
            self.capture()
        if int(self.traj.item()) + n_traj > self.max_traj:
            raise ValueError("not enough pre-drawn random numbers (max_traj=%d)" % self.max_traj)
        if adapt and getattr(self, "_da", None) is None:
            self.start_adaptation(target)
        for t in range(n_traj):
            self.graph.replay()
            self.n_evals += self.n_steps
            if adapt:
                self._adapt_step()
            if record is not None and t in record:
                record[t].copy_(self.z)
        return self

    # --- dual averaging of the step sizes (device tensors) ---
    def start_adaptation(self, target=0.8, gamma=0.05, kappa=0.75, t0=10.0):
        """Start (or restart) the dual averaging of every patch's step size from
        the current step sizes (Hoffman & Gelman 2014, algorithm 5)."""
        f64 = dict(dtype=torch.float64, device=self.device)
        self._da = {"mu": torch.log(10.0 * self.eps), "hbar": torch.zeros(self.n, **f64),
                    "log_bar": torch.zeros(self.n, **f64), "m": 0, "target": float(target),
                    "gamma": gamma, "kappa": kappa, "t0": t0}

    def _adapt_step(self):
        d = self._da
        d["m"] += 1
        m = float(d["m"])
        # acceptance probability of the trajectory just run: min(1, exp(H0 - H1))
        ee = torch.nan_to_num(self.energy_error, nan=-1e30, posinf=-1e30, neginf=-1e30)
        alpha = torch.exp(torch.clamp(ee, max=0.0))
        eta = 1.0 / (m + d["t0"])
        d["hbar"].mul_(1.0 - eta).add_(eta * (d["target"] - alpha))
        log_eps = d["mu"] - (m ** 0.5 / d["gamma"]) * d["hbar"]
        w = m ** (-d["kappa"])
        d["log_bar"].mul_(1.0 - w).add_(w * log_eps)
        self.eps.copy_(torch.exp(log_eps))

    def end_adaptation(self):
        """Install each patch's averaged step size and stop adapting."""
        if getattr(self, "_da", None) is not None and self._da["m"] > 0:
            self.eps.copy_(torch.exp(self._da["log_bar"]))
        self._da = None

    def adapt_mass_from(self, draws, reg=5.0):
        """Diagonal inverse mass matrix from warm-up draws of z (device tensor
        [n_draws, n_params]): the sample variance, shrunk towards 1e-3 as Stan
        does ((n / (n + 5)) var + 1e-3 (5 / (n + 5)))."""
        n = draws.shape[0]
        if n < 2:
            return self.inv_mass
        var = draws.var(dim=0, unbiased=True)
        self.inv_mass.copy_((n / (n + reg)) * var + 1e-3 * (reg / (n + reg)))
        return self.inv_mass

    def estimate_inv_mass(self, n_probe=8, h=1e-3, floor=1e-8, seed=1):
        """inv_mass = 1 / diag(-d2 lnp / dz2), the Hessian diagonal estimated with
        Rademacher probes v: E[(grad(z + h v) - grad(z)) * v] / h."""
        g = torch.Generator(device=self.device)
        g.manual_seed(seed)
        z = self.z.clone()
        self.gradient()
        g0 = self.grad.clone()
        acc = torch.zeros_like(z)
        for _ in range(n_probe):
            v = torch.randint(0, 2, z.shape, generator=g, device=self.device).to(torch.float64) * 2 - 1
            self.z.copy_(z + h * v)
            self.gradient()
            acc += (self.grad - g0) * v / h
        self.z.copy_(z)
        self.gradient()
        curv = -acc / n_probe
        pos = curv[curv > 0]
        rel = float(pos.median()) * 1e-2 if pos.numel() else 1.0
        curv = torch.clamp(curv, min=max(floor, rel))
        self.inv_mass.copy_(1.0 / curv)
        torch.cuda.synchronize()
        return self.inv_mass

    def positions(self):
        """Per patch the current constrained parameters (host arrays)."""
        s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        N.check(self.L.fp_hmc_prepare(self.d_hp.data_ptr(), self.n, self.z.data_ptr(), self.lower.data_ptr(),
                                      self.upper.data_ptr(), ctypes.byref(self.tab), self.plan.proposals.data_ptr(),
                                      self.theta.data_ptr(), self.jac.data_ptr(), s), "fp_hmc_prepare")
        th = self.theta.cpu().numpy()
        return [th[sl].copy() for sl in self.slices]

    def proposals(self):
        """Host copies of the current device proposal records [n_patches][MAXSOURCES]."""
        from .structs import source_struct_dtype
        raw = self.plan.proposals.cpu().numpy()
        return raw.view(source_struct_dtype).reshape(self.n, -1)
