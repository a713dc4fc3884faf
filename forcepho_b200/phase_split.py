"""Phase split of the tile kernel on the bench's batched workload.

    python -m forcepho_b200.build --phase-timers
    python -m forcepho_b200.phase_split [--patches 512] [--tile-pixels 1024] [--ctas 4]

Loads the diagnostic library ``lib/libforcepho_b200_phases.so`` (the same
kernels with clock64 counters read by thread 0 of each CTA at the barriers
between phases), evaluates the workload three times and prints one JSON line:
tiles per evaluation, clock cycles per tile and the share of CTA time in the
cull, the forward pass with the residual, the adjoint, and the per-tile
partials.  The counters add one barrier per tile; the normal library has none
of them.
"""

import argparse
import ctypes
import json
import os
import sys


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--patches", type=int, default=512)
    ap.add_argument("--tile-pixels", type=int, default=1024)
    ap.add_argument("--ctas", type=int, default=4)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()

    from . import build as B
    if not os.path.exists(B.PHASES_LIB):
        raise SystemExit("%s is missing: run python -m forcepho_b200.build --phase-timers" % B.PHASES_LIB)
    B.LIB = B.PHASES_LIB                      # every ctypes call below goes to the diagnostic build
    import torch
    from . import _native as N
    N.load(build_if_missing=False)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import types
    import bench
    from .batch import BatchedProposer

    torch.cuda.set_device(0)
    wl = types.SimpleNamespace(workload="batched", patches=args.patches)
    patches = bench.make_patches(wl, 0)
    for p in patches:
        p.return_residual = False
        p.send_to_device()
    bp = BatchedProposer(patches, tile_pixels=args.tile_pixels, ctas_per_sm=args.ctas, use_graph=False)
    bp.set_proposals_async(bench.perturbed_proposals(patches))
    lp = N.Launch(bp.launch.tile_pixels, bp.launch.ctas_per_sm, bp.launch.flags, N.PHASE_TILES)
    bp.plan.evaluate(bp.launch)               # setup (Gaussian tables) once
    L = ctypes.CDLL(B.PHASES_LIB)
    buf = (ctypes.c_ulonglong * 8)()
    N.check(L.fp_debug_phases(buf, 1), "fp_debug_phases")
    for _ in range(args.reps):
        bp.plan.evaluate(lp)
    N.check(L.fp_debug_phases(buf, 1), "fp_debug_phases")
    v = list(buf)
    total = max(v[7], 1)
    names = ["cull", "forward+residual", "adjoint", "partials"]
    print(json.dumps({"patches": args.patches, "tile_pixels": args.tile_pixels, "ctas_per_sm": args.ctas,
                      "tiles_per_evaluation": v[5] / args.reps, "cycles_per_tile": v[7] / max(v[5], 1),
                      "share": {n: v[i + 1] / total for i, n in enumerate(names)}}))


if __name__ == "__main__":
    main()
