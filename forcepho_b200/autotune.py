"""Launch-parameter selection for the tiled kernels.

The tile kernel has two free parameters: the pixel-tile size (256, 512 or
1024 pixels: 1, 2 or 4 pixels per thread in the forward pass) and the number
of persistent CTAs per SM.  Small tiles give tighter culling boxes and more
work items for a small patch; large tiles amortise the per-tile work (culling
scan, Gaussian staging, epilogue) and the pixel-loop parameter loads.

``default_tile_pixels`` is the static rule used before any measurement;
``Autotuner`` times the candidates on the device for a patch-size class and
remembers the winner (key: size class of the plan).
"""

import time

import numpy as np
import torch

TILE_CHOICES = (256, 512, 1024)
CTA_CHOICES = (3, 4)


def size_class(n_pairs, n_tiles_at_1024):
    """Coarse class of a workload: (log2 of pairs, log2 of 1024-px tiles)."""
    return (int(np.log2(max(n_pairs, 1))), int(np.log2(max(n_tiles_at_1024, 1))))


def default_tile_pixels(patch, n_sm=148):
    """Largest tile size that still gives every SM at least a few tiles."""
    npix = int(np.sum(patch.exposure_N))
    for tp in (1024, 512):
        if npix / tp >= 4 * n_sm:
            return tp
    return 256


class Autotuner:
    """Times (tile_pixels, ctas_per_sm) candidates for a set of patches.

    ``make_plan(tile_pixels)`` must return a ``device.Plan`` of the workload;
    its ``proposals`` buffer must already hold a representative proposal."""

    def __init__(self, tiles=TILE_CHOICES, ctas=CTA_CHOICES, reps=3):
        self.tiles, self.ctas, self.reps = tiles, ctas, reps
        self.cache = {}
        self.log = []

    def tune(self, key, make_plan, stream=None):
        if key in self.cache:
            return self.cache[key]
        stream = stream or torch.cuda.current_stream()
        best = None
        for tp in self.tiles:
            plan = make_plan(tp)
            for cps in self.ctas:
                lp = plan.launch(ctas_per_sm=cps)
                plan.evaluate(lp, stream=stream)          # warm-up
                stream.synchronize()
                t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                t0.record(stream)
                for _ in range(self.reps):
                    plan.evaluate(lp, stream=stream)
                t1.record(stream)
                t1.synchronize()
                ms = t0.elapsed_time(t1) / self.reps
                self.log.append((key, tp, cps, ms))
                if best is None or ms < best[2]:
                    best = (tp, cps, ms)
            del plan
        self.cache[key] = best
        return best

    def __repr__(self):
        return "Autotuner(%d entries)" % len(self.cache)


def wall_ms(fn, reps=3):
    t = time.perf_counter()
    for _ in range(reps):
        fn()
    return 1e3 * (time.perf_counter() - t) / reps
