"""Benchmark of forcepho's likelihood hot path (EvaluateProposal) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|limits|multiband|small] [--patches 512]

Workload (default ``batched``): 512 seeded synthetic patches with uneven
sources (1-30), bands (1-8), exposures per band (1-4) and pixels per exposure
(32^2-256^2), 4-Gaussian PSFs x 9 Sersic radii; data = model + noise.  A
*step* evaluates chi2 and its gradient for one proposal on every patch.

Our arm prints one JSON line: ``value`` = pixel-Gaussian evaluations/s of the
batched persistent kernels (CUDA graph replay, inputs resident in HBM, timed
with CUDA events); ``e2e`` = the same through ``BatchedProposer.evaluate_proposals``
with host proposals in and chi2/gradients out every step; ``plain`` = the
one-launch-per-patch port-equivalent kernel on the same patches;
``roofline`` = the tile kernel's FP32 work against the FP32 peak measured in
this run; ``cpu_baseline`` = the reference CPU kernel on a bounded sample;
``precision`` = errors against the FP64 oracle and the reference kernel on a
sample of patches, and of every patch of the batch against the device FP64
evaluation.

``--impl reference`` times the reference's own CPU kernel
(forcepho/src/compute_gaussians_kernel.cc built from source in oracle/_ref)
on the host cores, on the same workload, and prints its line.
Multi-GPU (torchrun): each rank evaluates its own batch (weak scaling); the
only collectives are a barrier and the max of the timings.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("lnlike+grad evals/s and pixel-Gaussian evals/s (batched vs plain, 1 B200, chi2 relerr<=1e-6)")
UNIT = "pixel-Gaussian evals/s"
FLOPS_PER_PAIR = 84      # FP32 flops (FMA = 2) of one forward + adjoint pair evaluation
EX2_PER_PAIR = 2
# raw chi2 errors of a band are measured against max(|chi2|, RAW_FLOOR * the
# band's sum (r^2 + d^2) ierr^2), as the parity tests measure them
RAW_FLOOR = 1e-2
PARAM_NAMES = ["flux", "ra", "dec", "q", "pa", "sersic", "rhalf"]


# DRAM bytes (read + write) of one tile_kernel launch, measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum, one pass, the first timed
# launch of "bench.py --steps 2 --warmup 3 --no-cpu --no-autotune --tile-pixels
# 1024 --plain-steps 1", NVTX range bench_timed): 4.306 GB read + 0.212 GB
# written.  Keyed by (workload, patches, tile pixels) of a one-size plan;
# other configurations report null.
TILE_TRAFFIC = {("batched", 512, 1024): 4.305974272e9 + 212.12416e6}


def hbm_fraction(traffic_bytes, algorithmic_gbs, kernel_ms):
    """DRAM bandwidth of the tile kernel against the measured HBM copy bandwidth
    (MEASURED_PEAKS.json, else the 6650 GB/s fallback): from the ncu traffic of a
    launch when known, and from the algorithmic pixel stream."""
    peak, src = 6650.0, "fallback 6650 GB/s (no MEASURED_PEAKS.json)"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, src = float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, ValueError, KeyError):
        pass
    traffic_gbs = None if traffic_bytes is None else traffic_bytes / (kernel_ms * 1e-3) / 1e9
    return {"peak_gbs": peak, "peak_source": src, "traffic_gbs": traffic_gbs,
            "traffic_frac": None if traffic_gbs is None else traffic_gbs / peak,
            "algorithmic_gbs": algorithmic_gbs, "algorithmic_frac": algorithmic_gbs / peak}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "limits", "multiband", "small", "hmc", "nuts", "single", "precision",
                             "autograd"])
    ap.add_argument("--nuts-depth", type=int, default=6, help="max tree depth (nuts workload)")
    ap.add_argument("--hmc-steps", type=int, default=16, help="leapfrog steps per trajectory (hmc workload)")
    ap.add_argument("--patches", type=int, default=512)
    ap.add_argument("--plain-steps", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--tile-pixels", type=int, default=0)
    ap.add_argument("--tile-classes", action="store_true", help="autotune a tile size per exposure-size class")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ----------------------------------------------------------------------------
# workload
# ----------------------------------------------------------------------------
def workload_shapes(args, rank):
    """Patch shape draws of the workload (cheap, no pixels)."""
    from forcepho_b200 import synthetic as S
    if args.workload == "batched":
        return [("batched", sh) for sh in S.batched_shapes(seed=4 + 1000 * rank, n_patches=args.patches)]
    return [(args.workload, {"seed": 1 + 1000 * rank})]


def make_patches(args, rank, render_on_gpu=True):
    """The workload's patches; data rendered by the GPU kernel (model + noise)."""
    from forcepho_b200 import synthetic as S
    patches = []
    for kind, sh in workload_shapes(args, rank):
        if kind == "batched":
            rng = np.random.default_rng(sh["seed"])
            p = S.make_patch(rng, n_sources=sh["n_sources"], exp_per_band=sh["exp_per_band"],
                             exp_pix=sh["exp_pix"], n_psf=4, source_params=S._broad_source, raster_width=256)
            p._rng = rng
        else:
            p = S.CONFIGS[kind](seed=sh["seed"])
            p._rng = np.random.default_rng(sh["seed"] + 17)
        patches.append(p)
    sigmas = [p._rng.uniform(0.5, 2.0, p.n_exp) for p in patches]
    models = None
    if render_on_gpu:
        from forcepho_b200.batch import render_models
        models = render_models(patches)
    for i, p in enumerate(patches):
        S.add_noise(p, p._rng, sigmas[i], None if models is None else models[i])
    return patches


def perturbed_proposals(patches, seed=99):
    """Proposals off the truth (non-trivial gradients), fixed per run."""
    rng = np.random.default_rng(seed)
    out = []
    for p in patches:
        q = p.scene.get_proposal().copy()
        n = len(q)
        q["ra"] += rng.normal(0, 2e-6, n).astype(np.float32)
        q["dec"] += rng.normal(0, 2e-6, n).astype(np.float32)
        q["q"] = np.clip(q["q"] * rng.uniform(0.95, 1.05, n), 0.2, 0.99).astype(np.float32)
        out.append(q)
    return out


# ----------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------
# CPU: the reference CPU kernel on a bounded sample
# ----------------------------------------------------------------------------
def _cpu_worker_init(root):
    sys.path.insert(0, root)


def _cpu_item(task):
    """Evaluate one (patch, band) with the reference CPU kernel (or the oracle
    port when the reference was not built); returns (pairs, seconds)."""
    from forcepho_b200 import synthetic as S
    from oracle import oracle as O
    kind, sh, band, use_ref = task
    if kind == "batched":
        rng = np.random.default_rng(sh["seed"])
        p = S.make_patch(rng, n_sources=sh["n_sources"], exp_per_band=sh["exp_per_band"], exp_pix=sh["exp_pix"],
                         n_psf=4, source_params=S._broad_source, raster_width=256)
        S.add_noise(p, rng, rng.uniform(0.5, 2.0, p.n_exp))
    else:
        p = S.CONFIGS[kind](seed=sh["seed"])
    prop = perturbed_proposals([p])[0]
    hs = O.HostStruct(p)
    pp = np.ascontiguousarray(prop)
    e0, ne = int(p.band_start[band]), int(p.band_N[band])
    pairs = int(np.sum(p.exposure_N[e0:e0 + ne].astype(np.int64))) * int(p.n_sources) * int(p.n_psf_per_source[band])
    t = time.perf_counter()
    if use_ref:
        O.ref_module().EvaluateProposal(band, hs.ptr, pp.ctypes.data)
    else:
        import ctypes
        c = ctypes.c_double()
        g = np.zeros(30 * 7, np.float32)
        O.lib().fpo_evaluate_band_f32(hs.ptr, pp.ctypes.data, band, ctypes.addressof(c), g.ctypes.data, 1)
    return pairs, time.perf_counter() - t


def cpu_tasks(args, rank, use_ref):
    tasks = []
    for kind, sh in workload_shapes(args, rank):
        nb = len(sh["exp_per_band"]) if kind == "batched" else None
        if nb is None:
            from forcepho_b200 import synthetic as S
            nb = S.CONFIGS[kind](seed=sh["seed"]).n_bands
        for b in range(nb):
            tasks.append((kind, sh, b, use_ref))
    return tasks


def precision_sample(patches, n_check=4, max_pairs=6e8, seed=11):
    """A seeded spread of patch sizes for the precision leg: one patch drawn
    from each quantile band of n_pairs among the patches the single-threaded
    reference kernel evaluates in seconds (n_pairs <= max_pairs)."""
    cand = sorted((p.n_pairs(), i) for i, p in enumerate(patches) if p.n_pairs() <= max_pairs)
    if not cand:
        return []
    rng = np.random.default_rng(seed)
    edges = np.linspace(0, len(cand), n_check + 1).astype(int)
    return sorted(cand[int(rng.integers(a, b))][1] for a, b in zip(edges[:-1], edges[1:]) if b > a)


def cpu_precision(patches, proposals, results, n_check=4):
    """Part of the CPU-baseline leg, untimed: a seeded spread of patch sizes
    from the timed batch (``precision_sample``), with the exact inputs the GPU
    saw, evaluated by the FP64 oracle and by the reference CPU kernel.

    chi2 errors are raw, |dchi2| / |chi2| per band (with the floor RAW_FLOOR of
    sum (r^2 + d^2) ierr^2 for bands whose chi2 has cancelled), and scaled,
    |dchi2| / sum (r^2 + d^2) ierr^2; gradient errors per parameter column,
    normwise.  Three comparisons on the same patches: GPU vs FP64, GPU vs the
    reference kernel, and the reference kernel vs FP64, so that the part of
    the GPU-vs-reference gap that is the reference's own FP32 error shows."""
    from oracle import oracle as O
    picked = precision_sample(patches, n_check)
    pairs = {"gpu_vs_f64": ("gpu", "f64"), "gpu_vs_reference": ("gpu", "ref"), "reference_vs_f64": ("ref", "f64")}
    worst = {k: {"chi2_relerr_max": 0.0, "chi2_err_over_scale_max": 0.0, "grad_colnorm_relerr_max": 0.0}
             for k in pairs}
    gap_explained = True
    for i in picked:
        p, prop = patches[i], proposals[i]
        c_g, g_g = results[i]
        c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
        cref, gref, _ = O.ref_evaluate(p, prop)
        vals = {"gpu": (np.asarray(c_g, np.float64), g_g), "f64": (c64, g64), "ref": (cref, gref)}
        for b in range(p.n_bands):
            e0, ne = int(p.band_start[b]), int(p.band_N[b])
            s0 = int(p.exposure_start[e0])
            s1 = int(p.exposure_start[e0 + ne - 1] + p.exposure_N[e0 + ne - 1])
            d = p.data[s0:s1].astype(np.float64) * p.ierr[s0:s1]
            r = r64[s0:s1] * p.ierr[s0:s1]
            sc = float(np.sum(d * d + r * r))
            for name, (a, ref) in pairs.items():
                diff = abs(vals[a][0][b] - vals[ref][0][b])
                w = worst[name]
                w["chi2_relerr_max"] = max(w["chi2_relerr_max"], diff / max(abs(vals[ref][0][b]), RAW_FLOOR * sc))
                w["chi2_err_over_scale_max"] = max(w["chi2_err_over_scale_max"], diff / sc)
            gap = abs(c_g[b] - cref[b])
            gap_explained &= bool(gap <= abs(cref[b] - c64[b]) + 1e-6 * max(abs(c64[b]), RAW_FLOOR * sc))
        for name, (a, ref) in pairs.items():
            ga, gr = vals[a][1], vals[ref][1]
            for k in range(7):
                den = np.linalg.norm(gr[..., k])
                if den > 0:
                    worst[name]["grad_colnorm_relerr_max"] = max(
                        worst[name]["grad_colnorm_relerr_max"], float(np.linalg.norm(ga[..., k] - gr[..., k]) / den))
    out = {"patches": picked, "pairs_per_patch": [int(patches[i].n_pairs()) for i in picked],
           "chi2_relerr": "max over bands of |dchi2| / max(|chi2|, 1e-2 sum (r^2+d^2) ierr^2)",
           "gpu_gap_to_reference_within_reference_error": gap_explained}
    out.update(worst)
    # the names of earlier records
    out["vs_f64"], out["vs_reference"], out["ref_vs_f64"] = (worst["gpu_vs_f64"], worst["gpu_vs_reference"],
                                                              worst["reference_vs_f64"])
    return out


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def _item_pairs(t):
    kind, sh, b = t[0], t[1], t[2]
    if kind != "batched":
        return None
    e0 = sum(sh["exp_per_band"][:b])
    npx = sum(((n + 31) // 32) * 32 for n in sh["exp_pix"][e0:e0 + sh["exp_per_band"][b]])
    return npx * sh["n_sources"] * 36


def cpu_measure(args, rank, seconds, cores=None, seed=0, single_core=True):
    """pairs/s of the reference CPU kernel on a seeded random sample of the
    workload's (patch, band) items, sized to about ``seconds`` of work on
    ``cores`` processes (a spawn pool: the pybind call holds the GIL).

    ``value`` counts kernel time only: cores x sum(pairs) / sum(per-call
    seconds), every call timed inside a worker while all workers are busy (the
    patch construction of each item is not part of the reference's kernel).
    ``wall_value`` is sum(pairs) / pool wall time, construction included.
    ``single_core``: the best of 5 calls on one mid-size item, alone."""
    import multiprocessing as mp
    from oracle import oracle as O
    use_ref = O.ref_available()
    cores = cores or (os.cpu_count() or 1)
    tasks = cpu_tasks(args, rank, use_ref)
    rng = np.random.default_rng(1000 + seed)
    order = rng.permutation(len(tasks))
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_cpu_worker_init, initargs=(ROOT,)) as pool:
        sized = [(t, _item_pairs(t)) for t in tasks]
        known = [x for x in sized if x[1] is not None]
        # calibrate on one small item, then size the sample to the time budget
        probe = min(known, key=lambda x: x[1])[0] if known else tasks[0]
        pairs0, t0 = pool.apply(_cpu_item, (probe,))
        rate1 = pairs0 / max(t0, 1e-6)
        budget_pairs = rate1 * cores * seconds
        sample, acc = [], 0
        for k in order:
            if acc >= budget_pairs:
                break
            t, n = sized[int(k)]
            sample.append(t)
            acc = acc + n if n is not None else budget_pairs
        wall = time.perf_counter()
        res = pool.map(_cpu_item, sample, chunksize=1)
        wall = time.perf_counter() - wall
        one = None
        if single_core:
            mid = sorted(known, key=lambda x: x[1])[len(known) // 2][0] if known else tasks[0]
            runs = [pool.apply(_cpu_item, (mid,)) for _ in range(5)]
            one = max(r[0] / r[1] for r in runs)
    pairs = sum(r[0] for r in res)
    busy = sum(r[1] for r in res)
    out = {"value": cores * pairs / busy, "unit": UNIT, "cores": cores, "kind": "reference" if use_ref else "port",
           "cpu_model": cpu_model(), "wall_value": pairs / wall,
           "sample": "%d (patch, band) items of the %s workload drawn at random (seed %d), %.3g pairs; kernel time "
                     "%.1f s over %d processes (%.1f s wall, patch construction included); data noise-only "
                     "(work does not depend on pixel values)"
                     % (len(sample), args.workload, 1000 + seed, pairs, busy, cores, wall),
           "pairs": pairs, "seconds": busy / cores}
    if one is not None:
        out["single_core_best_of_5"] = one
    return out


# ----------------------------------------------------------------------------
# arms
# ----------------------------------------------------------------------------
def config_of(args, n_patches, extra=None):
    c = {"workload": args.workload, "patches_per_gpu": n_patches,
         "shape_draws": "sources U{1..30}, bands U{1..8}, exposures/band U{1..4}, pixels/exposure U{32^2..256^2}"
         if args.workload == "batched" else args.workload,
         "psf": "4 Gaussians x 9 Sersic radii" if args.workload == "batched" else "per workload",
         "l2": "inputs larger than L2 (pixel arrays of the batch exceed 126 MB)"}
    if extra:
        c.update(extra)
    return c


def run_reference(args):
    rank, world, _ = dist_env()
    if world > 1 and rank != 0:
        return
    per_step = max(3.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    samples = []
    for i in range(args.warmup + args.steps):
        r = cpu_measure(args, 0, per_step, seed=i, single_core=(i == args.warmup + args.steps - 1))
        if i >= args.warmup:
            samples.append(r)
    pairs = sum(s["pairs"] for s in samples)
    secs = sum(s["seconds"] for s in samples)
    val = pairs / secs
    cb = dict(samples[-1])
    cb["value"] = val
    out = {"metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / len(samples),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic", "config": config_of(args, args.patches),
           "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "cpu_model",
                                                "single_core_best_of_5") if k in cb},
           "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        # ranks that wait for each other end with an error within 5 minutes; rank 0's
        # CPU legs (about a minute) run while the others wait at the last barrier
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    from forcepho_b200 import _native as N
    from forcepho_b200.batch import BatchedProposer
    from forcepho_b200.proposal import PlainProposer
    import ctypes

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t)
        return float(t.item())

    t_setup = time.perf_counter()
    patches = make_patches(args, rank)
    for p in patches:
        p.return_residual = False
        p.send_to_device()
    proposals = perturbed_proposals(patches)
    tp = args.tile_pixels or 1024
    # one tile size for the batch (3 sizes x 2 CTA counts); the per-class tuner
    # (--tile-classes) measured no gain on this workload
    tune = False if args.no_autotune or args.tile_pixels else ("classes" if args.tile_classes else True)
    bp = BatchedProposer(patches, tile_pixels=tp, autotune=tune)
    bp.set_proposals_async(proposals)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup
    n_pairs = bp.n_pairs
    stream = torch.cuda.current_stream()

    # peaks of this device (roofline denominators)
    L = N.load()
    scratch = torch.zeros(256, dtype=torch.float32, device="cuda")
    fp32_tflops, ex2_rate = ctypes.c_double(), ctypes.c_double()
    N.check(L.fp_measure_peaks(ctypes.c_void_p(scratch.data_ptr()), ctypes.byref(fp32_tflops),
                               ctypes.byref(ex2_rate), ctypes.c_void_p(stream.cuda_stream)), "fp_measure_peaks")

    # census: pairs evaluated after culling, pairs within the cutoff
    evaluated, active, dropped = bp.count_pairs()

    # ---- device-resident timing: graph replay of the whole evaluation ----
    for _ in range(args.warmup):
        bp.run(stream)
    torch.cuda.synchronize()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    props_dev = torch.cuda.get_device_properties(dev)
    gpu_id = ("GPU-" + str(props_dev.uuid)) if getattr(props_dev, "uuid", None) else str(dev)
    with ClockSampler(gpu_id) as clk:
        torch.cuda.synchronize()
        barrier()
        ev0.record(stream)
        torch.cuda.nvtx.range_push("bench_timed")     # lets ncu --nvtx-include select the timed steps
        for _ in range(args.steps):
            bp.run(stream)
        torch.cuda.nvtx.range_pop()
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    ms_max = max_over_ranks(ms)
    total_pairs = sum_over_ranks(float(n_pairs))
    total_patches = sum_over_ranks(float(len(patches)))
    value = total_pairs / (ms_max * 1e-3)
    clocks = clk.summary()

    # ---- the tile kernel alone (roofline) ----
    lp_tiles = N.Launch(bp.launch.tile_pixels, bp.launch.ctas_per_sm, bp.launch.flags, N.PHASE_TILES)
    bp.plan.evaluate(bp.launch, stream=stream)          # setup tables current
    for _ in range(2):
        bp.plan.evaluate(lp_tiles, stream=stream)
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0.record(stream)
    torch.cuda.nvtx.range_push("bench_tile_kernel")
    for _ in range(args.steps):
        bp.plan.evaluate(lp_tiles, stream=stream)
    torch.cuda.nvtx.range_pop()
    k1.record(stream)
    k1.synchronize()
    tile_ms = k0.elapsed_time(k1) / args.steps
    achieved = FLOPS_PER_PAIR * active / (tile_ms * 1e-3) / 1e12
    roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_tflops.value, "unit": "TFLOP/s",
                "frac": achieved / fp32_tflops.value,
                "traffic": (TILE_TRAFFIC.get((args.workload, args.patches, bp.tile_pixels))
                            if len(bp.tile_classes) == 1 else None),
                "kernel": "tile_kernel<%d>" % (bp.tile_pixels // 256),
                "kernel_ms": tile_ms, "share_of_step": tile_ms / ms,
                "peak_source": "measured in this run: FFMA-chain kernel (fp_measure_peaks), not in MEASURED_PEAKS.json",
                "work": "84 FP32 flops per pair within the MAX_EXP_ARG cutoff (%d of %d pairs); the culled kernel "
                        "evaluates %d pairs" % (active, n_pairs, evaluated),
                "ex2": {"achieved_per_s": EX2_PER_PAIR * active / (tile_ms * 1e-3), "peak_per_s": ex2_rate.value,
                        "frac": EX2_PER_PAIR * active / (tile_ms * 1e-3) / ex2_rate.value},
                "hbm_gbs": 16.0 * sum(int(np.sum(p.exposure_N)) for p in patches) / (tile_ms * 1e-3) / 1e9}
    roofline["hbm"] = hbm_fraction(roofline["traffic"], roofline["hbm_gbs"], tile_ms)

    # ---- end to end through the public API (host proposals in, results out) ----
    for _ in range(2):
        bp.evaluate_proposals(proposals)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    torch.cuda.nvtx.range_push("bench_e2e")
    for _ in range(args.steps):
        res = bp.evaluate_proposals(proposals)
    torch.cuda.nvtx.range_pop()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    e2e = {"value": total_pairs / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": bp.h2d_bytes,
           "d2h_bytes_per_step": bp.d2h_bytes, "ms_per_step": e2e_ms,
           "lnlike_grad_evals_per_s": total_patches / (e2e_ms * 1e-3),
           "api": "BatchedProposer.evaluate_proposals (pinned H2D of proposals, graph replay, D2H of chi2 + "
                  "Response records, host sync)"}

    # ---- the plain one-launch-per-patch comparator on the same patches ----
    plain = PlainProposer()
    d_prop = torch.zeros((len(patches), 30 * 264), dtype=torch.uint8, device="cuda")
    d_prop.copy_(bp.plan.proposals.view(len(patches), -1))
    d_chi2 = torch.zeros((len(patches), 30), dtype=torch.float64, device="cuda")
    d_resp = torch.zeros((len(patches), 30, 210), dtype=torch.float32, device="cuda")

    def plain_step():
        for i, p in enumerate(patches):
            plain.launch(p, d_prop[i].data_ptr(), d_chi2[i].data_ptr(), d_resp[i].data_ptr(), stream)

    plain_step()
    torch.cuda.synchronize()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    for _ in range(args.plain_steps):
        plain_step()
    q1.record(stream)
    q1.synchronize()
    plain_ms = max_over_ranks(q0.elapsed_time(q1) / args.plain_steps)
    # equal results: batched vs plain on every patch
    bres = bp.evaluate_proposals(proposals)
    pc, pr = d_chi2.cpu().numpy(), d_resp.cpu().numpy()
    worst_c, worst_raw, worst_g = 0.0, 0.0, 0.0
    for i, p in enumerate(patches):
        c_b, g_b = bres[i]
        c_p = pc[i, :p.n_bands]
        g_p = pr[i].reshape(30, 30, 7)[:p.n_bands, :int(p.n_sources)]
        dd = (p.data.astype(np.float64) * p.ierr) ** 2
        scale = float(np.sum(dd)) + 1e-300
        worst_c = max(worst_c, float(np.max(np.abs(c_b - c_p)) / scale))
        for b in range(p.n_bands):
            e0, ne = int(p.band_start[b]), int(p.band_N[b])
            s0 = int(p.exposure_start[e0])
            s1 = int(p.exposure_start[e0 + ne - 1] + p.exposure_N[e0 + ne - 1])
            # chi2 = sum (r^2 - d^2) ierr^2, so sum (r^2 + d^2) ierr^2 = chi2 + 2 sum d^2 ierr^2
            sc_b = float(c_b[b]) + 2.0 * float(np.sum(dd[s0:s1]))
            worst_raw = max(worst_raw, abs(float(c_b[b]) - float(c_p[b])) / max(abs(float(c_b[b])), RAW_FLOOR * sc_b,
                                                                                  1e-300))
        den = np.linalg.norm(g_b) + 1e-30
        worst_g = max(worst_g, float(np.linalg.norm(g_b - g_p) / den))
    plain_out = {"value": total_pairs / (plain_ms * 1e-3), "unit": UNIT, "ms_per_step": plain_ms,
                 "launches_per_step": len(patches), "speedup_batched_over_plain": plain_ms / ms_max,
                 "max_chi2_relerr_vs_batched": worst_raw, "max_chi2_diff_over_scale_vs_batched": worst_c,
                 "max_grad_normdiff_vs_batched": worst_g}

    cpu = None
    precision = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_measure(args, rank, args.cpu_seconds)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample", "cpu_model", "wall_value",
                                    "single_core_best_of_5") if k in cpu}
        precision = cpu_precision(patches, proposals, bres)
    if rank == 0:
        # every patch of this rank's batch against the device FP64 evaluation
        f64w = f64_whole(patches, proposals, bres)
        precision = dict(precision or {}, vs_device_f64_whole_batch=f64w)

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": config_of(args, len(patches), {"tile_pixels": bp.tile_pixels,
                                                        "tile_classes": bp.tile_classes,
                                                        "ctas_per_sm": bp.launch.ctas_per_sm,
                                                        "pairs_per_step_per_gpu": n_pairs,
                                                        "parallelism": "replicas-%d (independent patch batches)"
                                                                       % world}),
               "lnlike_grad_evals_per_s": total_patches / (ms_max * 1e-3),
               "e2e": e2e, "plain": plain_out, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
               "precision": precision,
               "gpu_launches": 3 * args.steps,
               "pairs": {"total": n_pairs, "evaluated_after_cull": evaluated, "within_cutoff": active,
                         "within_cutoff_but_culled": dropped},
               "autotune": [list(r[1:]) for r in bp.tune_log], "setup_s": setup_s}
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def run_hmc(args):
    """Device-resident HMC on patches of the limits distribution (30 sources,
    8 bands x 4 exposures of 256x256 px, 6-Gaussian PSFs): --patches of them
    (128 unless given), --hmc-steps leapfrog steps per trajectory, --warmup
    adapting trajectories (dual-averaging step sizes per patch; the diagonal
    mass matrix re-estimated from the draws of the warm-up's second half, then
    the step sizes adapted again), then --steps timed trajectories
    (CUDA-graph replays).  Precision study (CPU leg, untimed): at seeded chain
    positions recorded during the timed trajectories (device copies), chi2 and
    every gradient component of seeded patches against the FP64 oracle and the
    reference CPU kernel at the same proposals."""
    import torch
    from forcepho_b200 import synthetic as S
    from forcepho_b200.batch import render_models
    from forcepho_b200.hmc import DeviceHMC
    from forcepho_b200.proposal import B200Proposer
    from forcepho_b200.structs import source_struct_dtype
    torch.cuda.set_device(0)
    n = 128 if args.patches == 512 else args.patches
    rng = np.random.default_rng(5)
    t0 = time.perf_counter()
    patches = [S.config_limits(seed=int(rng.integers(2 ** 31))) for _ in range(n)]
    models = render_models(patches)
    theta0 = []
    for p, m in zip(patches, models):
        r = np.random.default_rng(int(rng.integers(2 ** 31)))
        S.add_noise(p, r, r.uniform(0.5, 2.0, p.n_exp), m)
        p.return_residual = False
        p.send_to_device()
        th = p.scene.get_all_source_params().reshape(int(p.n_sources), -1).copy()
        th[:, :p.n_bands] *= r.uniform(0.9, 1.1, th[:, :p.n_bands].shape)   # start off the truth
        theta0.append(th.reshape(-1))
    n_final = max(10, args.warmup // 4)          # step-size adaptation after the mass-matrix update
    n_traj = args.warmup + n_final + args.steps + 2
    h = DeviceHMC(patches, theta0, n_steps=args.hmc_steps, max_traj=n_traj, step_size=0.05)
    h.estimate_inv_mass()
    setup_s = time.perf_counter() - t0
    # warm-up: step sizes, then the mass matrix from the second half's draws, then step sizes again
    tw = time.perf_counter()
    w1 = args.warmup // 2
    h.run(w1, adapt=True, target=0.8)
    h.end_adaptation()
    w2 = args.warmup - w1
    draws = torch.zeros((w2, h.n_params), dtype=torch.float64, device=h.device)
    h.run(w2, adapt=True, target=0.8, record={t: draws[t] for t in range(w2)})
    h.end_adaptation()
    if w2 >= 10:
        h.adapt_mass_from(draws)
        h.start_adaptation(0.8)
        h.run(n_final, adapt=True, target=0.8)
        h.end_adaptation()
    torch.cuda.synchronize()
    warm_s = time.perf_counter() - tw
    acc0 = h.accepted.clone()
    # seeded chain positions to check (trajectory index within the timed run)
    prng = np.random.default_rng(17)
    rec_t = sorted(set(int(t) for t in prng.integers(0, max(args.steps, 1), 4)))
    record = {t: torch.zeros(h.n_params, dtype=torch.float64, device=h.device) for t in rec_t}
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    props_dev = torch.cuda.get_device_properties(0)
    gpu_id = ("GPU-" + str(props_dev.uuid)) if getattr(props_dev, "uuid", None) else "0"
    with ClockSampler(gpu_id) as clk:
        torch.cuda.nvtx.range_push("bench_timed")
        e0.record(stream)
        h.run(args.steps, record=record)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = e0.elapsed_time(e1)
    grad_evals = n * args.hmc_steps * args.steps
    pairs = h.plan.n_pairs * args.hmc_steps * args.steps
    acc = ((h.accepted - acc0).double() / args.steps).cpu().numpy()
    de = h.energy_error.cpu().numpy()
    eps = h.eps.cpu().numpy()
    out = {"metric": METRIC, "value": pairs / (ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "hmc", "patches": n, "leapfrog_steps": args.hmc_steps,
                      "trajectories_timed": args.steps,
                      "patch": "30 sources, 8 bands x 4 exposures of 256x256 px, 6-Gaussian PSFs",
                      "mass_matrix": "diagonal: Hessian-diagonal estimate, then the variance of the warm-up's "
                                     "second-half draws",
                      "step_size": "per patch, dual averaging towards acceptance 0.8 during warm-up, averaged "
                                   "step size after",
                      "step": "a trajectory of every patch (graph replay)"},
           "gradient_evals_per_s": grad_evals / (ms * 1e-3),
           "trajectories_per_s": n * args.steps / (ms * 1e-3),
           "acceptance_mean": float(acc.mean()), "acceptance_min": float(acc.min()),
           "energy_error_abs_median": float(np.median(np.abs(de))),
           "step_size_median": float(np.median(eps)), "step_size_range": [float(eps.min()), float(eps.max())],
           "clocks": clk.summary(), "setup_s": setup_s, "warmup_s": warm_s,
           "gpu_launches": args.steps * (6 * args.hmc_steps + 2)}
    if not args.no_cpu:
        from oracle import oracle as O
        # proposals at the recorded positions (device splines and transform), for
        # seeded patches; GPU results from the proposer on those exact records
        picks = sorted(set(int(i) for i in prng.integers(0, n, 3)))
        rows = []
        worst = {"gpu_vs_f64": [0.0, 0.0, 0.0], "gpu_vs_reference": [0.0, 0.0, 0.0],
                 "reference_vs_f64": [0.0, 0.0, 0.0]}
        bands = (0, 5)
        for t in rec_t:
            h.z.copy_(record[t])
            h.positions()
            props_all = h.proposals()
            for i in picks:
                p = patches[i]
                prop = np.ascontiguousarray(props_all[i][:int(p.n_sources)]).view(source_struct_dtype)
                chi2, dchi2 = B200Proposer().evaluate_proposal(prop, patch=p)
                c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True, bands=bands)
                cref, gref, _ = O.ref_evaluate(p, prop, bands=bands)
                vals = {"gpu": (chi2, dchi2), "f64": (c64, g64), "reference": (cref, gref)}
                row = {"trajectory": t, "patch": i}
                for key, (a, b) in (("gpu_vs_f64", ("gpu", "f64")), ("gpu_vs_reference", ("gpu", "reference")),
                                    ("reference_vs_f64", ("reference", "f64"))):
                    ca, ga = vals[a]
                    cb, gb = vals[b]
                    cre = max(abs(ca[bb] - cb[bb]) / abs(cb[bb]) for bb in bands)
                    cols = component_errors(np.asarray(ga)[list(bands)], np.asarray(gb)[list(bands)])
                    gn = max(c["norm"] for c in cols)
                    gc = max(c["comp_max"] for c in cols)
                    row[key] = {"chi2_relerr": cre, "grad_colnorm": gn, "grad_comp_max": gc}
                    w = worst[key]
                    w[0], w[1], w[2] = max(w[0], cre), max(w[1], gn), max(w[2], gc)
                rows.append(row)
        out["precision"] = {"positions": rows, "bands": list(bands),
                            "worst": {k: {"chi2_relerr": v[0], "grad_colnorm": v[1], "grad_comp_max": v[2]}
                                      for k, v in worst.items()},
                            "state": "chain positions recorded during the timed trajectories"}
    print(json.dumps(out), flush=True)


def run_nuts_bench(args):
    """Lockstep NUTS on patches of the limits distribution: --patches of them
    (16 unless given), --warmup adapting transitions (untimed), then --steps
    kept transitions timed by wall clock: the loop is host-driven, one host
    synchronisation per leapfrog step of the whole batch."""
    import torch
    from forcepho_b200 import synthetic as S
    from forcepho_b200.batch import render_models
    from forcepho_b200.hmc import DeviceHMC
    from forcepho_b200.nuts import BatchedNUTS, DevicePosterior
    torch.cuda.set_device(0)
    n = 16 if args.patches == 512 else args.patches
    rng = np.random.default_rng(6)
    t0 = time.perf_counter()
    patches = [S.config_limits(seed=int(rng.integers(2 ** 31))) for _ in range(n)]
    models = render_models(patches)
    theta0 = []
    for p, m in zip(patches, models):
        r = np.random.default_rng(int(rng.integers(2 ** 31)))
        S.add_noise(p, r, r.uniform(0.5, 2.0, p.n_exp), m)
        p.return_residual = False
        p.send_to_device()
        th = p.scene.get_all_source_params().reshape(int(p.n_sources), -1).copy()
        th[:, :p.n_bands] *= r.uniform(0.9, 1.1, th[:, :p.n_bands].shape)
        theta0.append(th.reshape(-1))
    h = DeviceHMC(patches, theta0, n_steps=1, max_traj=1)
    var = h.estimate_inv_mass().cpu().numpy()
    post = DevicePosterior(h)
    z0 = post.start()
    nuts = BatchedNUTS(post, post.sizes, init_mean=z0, init_cov=[var[sl] for sl in h.slices],
                       max_treedepth=args.nuts_depth, seed=1)
    setup_s = time.perf_counter() - t0
    tw = time.perf_counter()
    _, _ = nuts.sample(z0, 0, tune=args.warmup, discard_tuned_samples=True)
    warm_s = time.perf_counter() - tw
    z, lnp, g = nuts.state                 # the adapted chains continue into the kept transitions
    torch.cuda.synchronize()
    ev0 = nuts.n_evals
    props_dev = torch.cuda.get_device_properties(0)
    gpu_id = ("GPU-" + str(props_dev.uuid)) if getattr(props_dev, "uuid", None) else "0"
    stats = []
    with ClockSampler(gpu_id) as clk:
        t1 = time.perf_counter()
        for _ in range(args.steps):
            z, lnp, g, st = nuts.iterate(z, lnp, g, tune=False)
            stats.append(st)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t1
    evals = nuts.n_evals - ev0
    live_leaves = float(sum(st["n_steps"].sum() for st in stats))
    pairs = h.plan.n_pairs * evals
    out = {"metric": METRIC, "value": pairs / wall, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "nuts", "patches": n, "max_treedepth": args.nuts_depth,
                      "patch": "30 sources, 8 bands x 4 exposures of 256x256 px, 6-Gaussian PSFs",
                      "mass_matrix": "diagonal, adapted; started from the Hessian-diagonal estimate",
                      "step": "one NUTS transition of every patch (wall clock, host-driven)"},
           "batched_gradient_evals": evals, "gradient_evals_per_s": n * evals / wall,
           "useful_fraction": live_leaves / (n * evals), "useful_gradient_evals_per_s": live_leaves / wall,
           "tree_depth_mean": float(np.mean([st["depth"] for st in stats])),
           "mean_tree_accept": float(np.mean([st["mean_tree_accept"] for st in stats])),
           "divergences": int(sum(st["diverging"].sum() for st in stats)),
           "clocks": clk.summary(), "setup_s": setup_s, "warmup_s": warm_s}
    print(json.dumps(out), flush=True)


def run_autograd(args):
    """The differentiable path: forward (chi2 per band) and backward (the
    vector-Jacobian product) through ``PatchChi2`` on the limits patch (30
    sources, 8 bands x 4 exposures of 256x256 px: 420 parameters) and through
    ``BatchChi2`` on the batched workload's patches, timed with CUDA events
    over --steps forward+backward passes after --warmup; theta stays on the
    device throughout."""
    import torch
    from forcepho_b200 import synthetic as S
    from forcepho_b200.autograd import BatchChi2, PatchChi2
    torch.cuda.set_device(0)
    out = {"metric": "forward+backward passes of the differentiable chi2", "unit": "pixel-Gaussian evals/s",
           "steps": args.steps, "warmup": args.warmup, "data": "synthetic", "higher_is_better": True, "cases": {}}
    lim = S.config_limits(seed=3)
    lim.return_residual = False
    lim.send_to_device()
    import copy
    bargs = copy.copy(args)
    bargs.workload = "batched"
    patches = make_patches(bargs, 0)
    for p in patches:
        p.return_residual = False
        p.send_to_device()
    for name, fn, pats in (("limits", PatchChi2(lim), [lim]), ("batched", BatchChi2(patches), patches)):
        th = np.concatenate([p.scene.get_all_source_params() for p in pats])
        theta = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
        w = torch.ones(fn.n_rows, dtype=torch.float64, device="cuda")

        def step():
            theta.grad = None
            (fn(theta) * w).sum().backward()

        for _ in range(max(args.warmup, 3)):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        pairs = sum(p.n_pairs() for p in pats)
        out["cases"][name] = {"patches": len(pats), "parameters": fn.n_params, "ms_per_pass": ms,
                              "value": pairs / (ms * 1e-3), "pairs_per_pass": pairs}
    print(json.dumps(out), flush=True)


def run_single(args):
    """Single-patch call latency, as forcepho's own samplers call the kernel
    (one proposal per call, host proposal in, results out): the Python
    proposer (one CUDA-graph replay per call), the reference's kernel ABI
    (fp_evaluate_proposal: struct and index-array read-backs, then the tiled
    launches on the library's cached plan) and the plain comparator, on the
    small (64x64 px, one source) and multiband (16 sources, 5 bands x 2
    exposures of 150x150 px) patches.  --steps calls per path after --warmup."""
    import ctypes
    import torch
    from forcepho_b200 import _native as N
    from forcepho_b200 import synthetic as S
    from forcepho_b200.kernel_limits import MAXSOURCES, NPARAMS
    from forcepho_b200.proposal import B200Proposer, PlainProposer
    torch.cuda.set_device(0)
    L = N.load()
    steps = max(args.steps, 50)
    out = {"metric": "single-patch lnlike+grad call latency", "unit": "us per call", "steps": steps,
           "warmup": args.warmup, "higher_is_better": False, "data": "synthetic", "patches": {}}
    for name in ("small", "multiband"):
        p = S.CONFIGS[name](seed=1)
        p.return_residual = False
        p.send_to_device()
        prop = perturbed_proposals([p])[0]
        nb, ns = p.n_bands, int(p.n_sources)
        pin_prop = torch.from_numpy(prop.view(np.uint8).copy()).pin_memory()
        d_prop = torch.empty_like(pin_prop, device="cuda")
        d_chi2 = torch.zeros(nb, dtype=torch.float64, device="cuda")
        d_resp = torch.zeros((nb, MAXSOURCES * NPARAMS), dtype=torch.float32, device="cuda")
        h_chi2 = torch.zeros(nb, dtype=torch.float64).pin_memory()
        h_resp = torch.zeros((nb, MAXSOURCES * NPARAMS), dtype=torch.float32).pin_memory()
        stream = torch.cuda.current_stream()

        def abi_call():
            d_prop.copy_(pin_prop, non_blocking=True)
            N.check(L.fp_evaluate_proposal(p.device_patch_ptr, d_prop.data_ptr(), ns, nb, d_chi2.data_ptr(),
                                           d_resp.data_ptr(), ctypes.c_void_p(stream.cuda_stream)),
                    "fp_evaluate_proposal")
            h_chi2.copy_(d_chi2, non_blocking=True)
            h_resp.copy_(d_resp, non_blocking=True)
            stream.synchronize()

        tiled, plain = B200Proposer(), PlainProposer()
        paths = {"proposer_graph": lambda: tiled.evaluate_proposal(prop, patch=p),
                 "reference_abi": abi_call,
                 "plain": lambda: plain.evaluate_proposal(prop, patch=p)}
        res = {}
        for key, fn in paths.items():
            for _ in range(max(args.warmup, 3)):
                fn()
            t = time.perf_counter()
            for _ in range(steps):
                fn()
            res[key] = 1e6 * (time.perf_counter() - t) / steps
        res["pairs"] = int(p.n_pairs())
        out["patches"][name] = res
    print(json.dumps(out), flush=True)


def component_errors(g, gref, rel_floor=1e-3):
    """Per parameter column k: the normwise error ||g - gref|| / ||gref|| and
    the largest and median error of single components |g - gref| / |gref|
    over the components with |gref| >= rel_floor * max |gref| of the column."""
    g = np.asarray(g, np.float64)
    gref = np.asarray(gref, np.float64)
    out = []
    for k in range(gref.shape[-1]):
        a, b = g[..., k].ravel(), gref[..., k].ravel()
        den = np.linalg.norm(b)
        if den == 0:
            out.append({"norm": 0.0, "comp_max": 0.0, "comp_median": 0.0})
            continue
        big = np.abs(b) >= rel_floor * np.abs(b).max()
        ce = np.abs(a[big] - b[big]) / np.abs(b[big])
        out.append({"norm": float(np.linalg.norm(a - b) / den), "comp_max": float(ce.max()),
                    "comp_median": float(np.median(ce))})
    return out


def run_precision(args):
    """Error of the loaded library against the FP64 oracle: chi2 (raw,
    per band) and every gradient component, on the limits-size patch (two
    bands) and on a seeded spread of the batched workload's patches.  Run once
    per precision variant (FORCEPHO_B200_VARIANT unset: FP32 runs flushed to
    FP64; =kahan: FP32 + Kahan) on the same inputs."""
    import torch
    from forcepho_b200 import synthetic as S
    from forcepho_b200 import _native as N
    from forcepho_b200.proposal import B200Proposer
    from oracle import oracle as O
    torch.cuda.set_device(0)
    N.load()
    variant = os.environ.get("FORCEPHO_B200_VARIANT", "") or "fp32-runs-flushed-to-fp64"
    cases = []
    lim = S.config_limits(seed=3)
    cases.append(("limits", lim, perturbed_proposals([lim])[0], (0, 4)))
    shapes = S.batched_shapes(seed=4, n_patches=args.patches)
    pats = []
    for sh in shapes:
        rng = np.random.default_rng(sh["seed"])
        p = S.make_patch(rng, n_sources=sh["n_sources"], exp_per_band=sh["exp_per_band"], exp_pix=sh["exp_pix"],
                         n_psf=4, source_params=S._broad_source, raster_width=256)
        p._rng = rng
        pats.append(p)
    for i in precision_sample(pats, 4, max_pairs=2e9):
        p = pats[i]
        S.add_noise(p, p._rng, p._rng.uniform(0.5, 2.0, p.n_exp), O.render(p, p.scene.get_proposal()))
        cases.append(("batched[%d]" % i, p, perturbed_proposals([p])[0], None))
    rows = []
    worst = {"chi2_relerr": 0.0, "grad_norm": 0.0, "grad_comp_max": 0.0}
    for name, p, prop, bands in cases:
        p.return_residual = False
        p.send_to_device()
        chi2, dchi2 = B200Proposer().evaluate_proposal(prop, patch=p)
        c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True, bands=bands)
        bl = list(range(p.n_bands)) if bands is None else list(bands)
        sc = []
        for b in bl:
            e0, ne = int(p.band_start[b]), int(p.band_N[b])
            s0 = int(p.exposure_start[e0])
            s1 = int(p.exposure_start[e0 + ne - 1] + p.exposure_N[e0 + ne - 1])
            d = p.data[s0:s1].astype(np.float64) * p.ierr[s0:s1]
            r = r64[s0:s1] * p.ierr[s0:s1]
            sc.append(float(np.sum(d * d + r * r)))
        ce = [abs(chi2[b] - c64[b]) / max(abs(c64[b]), RAW_FLOOR * s_) for b, s_ in zip(bl, sc)]
        cols = component_errors(dchi2[bl], g64[bl])
        rows.append({"patch": name, "pairs": int(p.n_pairs()), "bands": bl, "chi2_relerr": ce,
                     "grad": dict(zip(PARAM_NAMES, cols))})
        worst["chi2_relerr"] = max(worst["chi2_relerr"], max(ce))
        worst["grad_norm"] = max(worst["grad_norm"], max(c["norm"] for c in cols))
        worst["grad_comp_max"] = max(worst["grad_comp_max"], max(c["comp_max"] for c in cols))
        p.free()
    print(json.dumps({"metric": "error vs FP64 oracle", "variant": variant, "library": N.lib_path(),
                      "worst": worst, "cases": rows}), flush=True)
    print(json.dumps(precision_full(args, variant)), flush=True)


def f64_whole(patches, proposals, results):
    """Batched FP32 results (one (chi2, dchi2) per patch) against the device
    FP64 evaluation (fp_evaluate_proposal_f64, held to the FP64 oracle at
    1e-11 by the tests) on every patch: worst raw chi2 per band, against
    max(|chi2|, RAW_FLOOR sum (r^2 + d^2) ierr^2) with sum (r^2 + d^2) ierr^2
    = chi2_f64 + 2 sum d^2 ierr^2, and worst gradient column."""
    import torch
    from forcepho_b200.proposal import F64Proposer
    f64 = F64Proposer()
    t0 = time.perf_counter()
    worst = {"chi2_relerr": 0.0, "grad_norm": 0.0, "grad_comp_max": 0.0}
    where = {}
    for i, (p, prop) in enumerate(zip(patches, proposals)):
        c64, g64 = f64.evaluate_proposal(prop, patch=p)
        c32, g32 = results[i]
        dd = (p.data.astype(np.float64) * p.ierr) ** 2
        for b in range(p.n_bands):
            e0, ne = int(p.band_start[b]), int(p.band_N[b])
            s0 = int(p.exposure_start[e0])
            s1 = int(p.exposure_start[e0 + ne - 1] + p.exposure_N[e0 + ne - 1])
            sc = c64[b] + 2.0 * float(np.sum(dd[s0:s1]))
            e = abs(c32[b] - c64[b]) / max(abs(c64[b]), RAW_FLOOR * sc, 1e-300)
            if e > worst["chi2_relerr"]:
                worst["chi2_relerr"], where["chi2_relerr"] = e, [i, b]
        for name, c in zip(PARAM_NAMES, component_errors(g32, g64)):
            for k in ("norm", "comp_max"):
                key = "grad_" + k
                if c[k] > worst[key]:
                    worst[key], where[key] = c[k], [i, name]
    torch.cuda.synchronize()
    return {"patches": len(patches), "worst": worst, "worst_at": where,
            "f64_seconds": time.perf_counter() - t0}


def precision_full(args, variant):
    """The whole batched workload (every patch, the bench's proposals) through
    the batched FP32 path, against the device FP64 evaluation."""
    from forcepho_b200.batch import BatchedProposer
    patches = make_patches(argparse.Namespace(**{**vars(args), "workload": "batched"}), 0)
    for p in patches:
        p.return_residual = False
        p.send_to_device()
    proposals = perturbed_proposals(patches)
    bp = BatchedProposer(patches, tile_pixels=args.tile_pixels or 1024, autotune=False)
    got = bp.evaluate_proposals(proposals)
    out = {"metric": "error vs device FP64 (whole workload)", "variant": variant, "workload": "batched",
           "pairs": int(bp.n_pairs)}
    out.update(f64_whole(patches, proposals, got))
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "hmc":
        run_hmc(args)
    elif args.workload == "nuts":
        run_nuts_bench(args)
    elif args.workload == "single":
        run_single(args)
    elif args.workload == "precision":
        run_precision(args)
    elif args.workload == "autograd":
        run_autograd(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
