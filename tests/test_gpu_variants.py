"""The FP32 + Kahan precision variant of the library (built by
``python -m forcepho_b200.build --kahan``, loaded with
FORCEPHO_B200_VARIANT=kahan): its results stay within the tiled path's
tolerances of the FP64 oracle.  A process loads one library, so the variant
runs in a child process."""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
from forcepho_b200 import _native as N, synthetic as S
from forcepho_b200.proposal import B200Proposer
from oracle import oracle as O
from tolerances import band_scales, chi2_raw_err, grad_err
p = S.config_multiband(seed=13, render=O.render, n_sources=6, n_bands=3, exp_per_band=2, size=64)
p.return_residual = False
p.send_to_device()
prop = p.scene.get_proposal().copy()
prop["q"] = np.clip(prop["q"] * 0.95, 0.2, 0.99)
chi2, dchi2 = B200Proposer().evaluate_proposal(prop, patch=p)
c64, g64, r64 = O.evaluate(p, prop, precision="f64", return_residual=True)
print(json.dumps({"lib": N.lib_path(), "chi2": chi2_raw_err(chi2, c64, band_scales(p, r64)),
                  "grad": grad_err(dchi2, g64)}))
"""


def test_kahan_variant_matches_the_fp64_oracle():
    from forcepho_b200 import build as B
    from tolerances import CHI2_F64, GRAD_F64
    if not os.path.exists(B.KAHAN_LIB):
        pytest.skip("the FP32 + Kahan variant is not built")
    env = dict(os.environ, FORCEPHO_B200_VARIANT="kahan")
    out = subprocess.run([sys.executable, "-c", CHILD, ROOT], env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["lib"].endswith("libforcepho_b200_kahan.so")
    assert r["chi2"] < CHI2_F64 and r["grad"] < GRAD_F64, r
