"""Compile the CUDA library ``forcepho_b200/lib/libforcepho_b200.so`` in-tree.

    python -m forcepho_b200.build [--verbose] [--phase-timers]

nvcc builds every ``csrc/*.cu`` for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) into one shared library exporting the C ABI
of ``include/forcepho_b200.h``.  The library is rebuilt only when a source or
header is newer than it (or with ``force=True``).  ``--phase-timers`` builds
the diagnostic variant ``libforcepho_b200_phases.so`` instead (clock64 counters
at the tile kernel's phase boundaries; ``python -m forcepho_b200.phase_split``).
"""

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libforcepho_b200.so")
DEFAULT_LIB = LIB
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "-shared", "--expt-relaxed-constexpr", "-I", INCLUDE]


def nvcc():
    for cand in [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc"]:
        if cand and os.path.exists(cand):
            return cand
    return "nvcc"


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force=False, verbose=False, extra=(), out=None):
    """Build the library (or, with ``out``, a variant of it at that path) if
    needed; returns its path."""
    lib = out or LIB
    if not force and lib == LIB and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = lib + ".tmp"
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + list(extra) + ["-o", tmp] + sources() + ["-lcudart"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode:
        raise RuntimeError("nvcc failed building %s (exit %d)" % (lib, r.returncode))
    os.replace(tmp, lib)
    return lib


# diagnostic variant: the tile kernel with per-phase clock64 counters
# (fp_debug_phases); forcepho_b200.phase_split reports them
PHASES_LIB = os.path.join(LIBDIR, "libforcepho_b200_phases.so")


def build_phase_timers(verbose=False):
    return build(force=True, verbose=verbose, extra=["-DFP_PHASE_TIMERS"], out=PHASES_LIB)


# precision variant: per-thread FP32 + Kahan sums in the pixel loops (model,
# chi2 terms, adjoint moments) instead of FP32 runs flushed to FP64; the
# comparison of the two schemes (bench.py --workload precision) loads it with
# FORCEPHO_B200_VARIANT=kahan
KAHAN_LIB = os.path.join(LIBDIR, "libforcepho_b200_kahan.so")


def build_kahan(verbose=False):
    return build(force=True, verbose=verbose, extra=["-DFP_KAHAN"], out=KAHAN_LIB)


def variant_lib():
    """The library _native loads: the normal build, or the variant named by
    $FORCEPHO_B200_VARIANT ("kahan")."""
    v = os.environ.get("FORCEPHO_B200_VARIANT", "")
    if v == "kahan":
        return KAHAN_LIB
    if v:
        raise ValueError("FORCEPHO_B200_VARIANT=%r: known variants are 'kahan'" % v)
    return LIB


if __name__ == "__main__":
    if "--phase-timers" in sys.argv:
        print(build_phase_timers(verbose="--verbose" in sys.argv))
    elif "--kahan" in sys.argv:
        print(build_kahan(verbose="--verbose" in sys.argv))
    else:
        build(force=True, verbose="--verbose" in sys.argv)
        print(LIB)
