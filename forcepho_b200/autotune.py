"""Launch-parameter selection for the tiled kernels.

The tile kernel has two free parameters: the pixel-tile size (256, 512 or
1024 pixels: 1, 2 or 4 pixels per thread in the forward pass) and the number
of persistent CTAs per SM.  Small tiles give tighter culling boxes and more
work items for a small patch; large tiles amortise the per-tile work (culling
scan, Gaussian staging, epilogue) and the pixel-loop parameter loads.  The
tile size can differ by exposure size within one plan (tile classes), all
tiles still running in one persistent launch.

``default_tile_pixels`` is the static rule used before any measurement;
``Autotuner`` times the candidates on the device for a workload-size class and
remembers the winner (key: size class of the plan): one tile size for the
plan (``tune``), or one per exposure-size class (``tune_classes``, coordinate
descent over the classes, then the CTA count).
"""

import time

import numpy as np
import torch

TILE_CHOICES = (256, 512, 1024)
CTA_CHOICES = (3, 4)
# exposure-size classes (upper bounds in pixels; the last takes the rest)
CLASS_BOUNDS = (8192, 32768, 2 ** 31 - 1)


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

    def _time(self, plan, cps, stream):
        lp = plan.launch(ctas_per_sm=cps)
        plan.evaluate(lp, stream=stream)          # warm-up
        stream.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(self.reps):
            plan.evaluate(lp, stream=stream)
        t1.record(stream)
        t1.synchronize()
        return t0.elapsed_time(t1) / self.reps

    def tune_classes(self, key, make_plan, bounds=CLASS_BOUNDS, start=1024, ctas=4, stream=None):
        """Per exposure-size class tile sizes by coordinate descent: from every
        class at ``start``, each class in turn tries every tile size with the
        others fixed and keeps the fastest; then the CTA counts.
        ``make_plan(classes)`` must return a ``device.Plan`` of the workload
        for ``classes`` = [(bound, tile_pixels), ...] with a representative
        proposal loaded.  Returns (classes, ctas_per_sm, ms)."""
        ckey = ("classes",) + tuple(key) if isinstance(key, tuple) else ("classes", key)
        if ckey in self.cache:
            return self.cache[ckey]
        stream = stream or torch.cuda.current_stream()
        tiles = [start] * len(bounds)
        timed = {}

        def run(tl, cps):
            k = (tuple(tl), cps)
            if k not in timed:
                plan = make_plan(list(zip(bounds, tl)))
                timed[k] = self._time(plan, cps, stream)
                self.log.append((ckey, tuple(tl), cps, timed[k]))
                del plan
            return timed[k]

        best = run(tiles, ctas)
        for c in range(len(bounds)):
            for tp in self.tiles:
                cand = list(tiles)
                cand[c] = tp
                ms = run(cand, ctas)
                if ms < best:
                    best, tiles = ms, cand
        best_cps = ctas
        for cps in self.ctas:
            ms = run(tiles, cps)
            if ms < best:
                best, best_cps = ms, cps
        out = (list(zip(bounds, tiles)), best_cps, best)
        self.cache[ckey] = out
        return out

    def __repr__(self):
        return "Autotuner(%d entries)" % len(self.cache)


def wall_ms(fn, reps=3):
    t = time.perf_counter()
    for _ in range(reps):
        fn()
    return 1e3 * (time.perf_counter() - t) / reps
