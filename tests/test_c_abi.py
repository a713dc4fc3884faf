"""The C ABI from a C host (tests/c/abi_example.c): the header compiles as
plain C99, the program links against the library, plans a patch on the host
and gets the library's error codes and messages, with no GPU."""

import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_c_host_plans_a_patch_through_the_abi(tmp_path):
    from forcepho_b200 import _native as N
    N.load()
    libdir = os.path.dirname(N.lib_path())
    exe = str(tmp_path / "abi_example")
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                         os.path.join(ROOT, "tests", "c", "abi_example.c"), "-L", libdir, "-lforcepho_b200",
                         "-Wl,-rpath," + libdir, "-o", exe], capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    out = run.stdout
    assert "sizes 152 264 840 28" in out
    m = re.search(r"plan tiles (\d+) gauss (\d+) pairs (\d+) perm (\d+) pixels_in_tiles (\d+)", out)
    assert m, out
    tiles, gauss, pairs, perm, seen = map(int, m.groups())
    assert gauss == 2 * 3 * 9 and pairs == 2 * 960 * 27 and perm == 1920 and seen == 1920
    assert tiles >= 2 * 4                      # 40x24 pixels in 16x16 cells per exposure
    assert "null call rc -1" in out and "NULL" in out
