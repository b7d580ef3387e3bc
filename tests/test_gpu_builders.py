"""Table-builder forms of the tensor-core path: the warp-per-harmonic
builders (default), the block-per-harmonic builders and the direct builders
(one FP64 sincos per entry) fill the R, S and C images for the same fields.
The two factored forms run the same FP64 operations per entry, so every
field must be bit-identical between them; the direct form rounds its phases
differently and must agree within the tensor-core tolerance of the FP64
oracle's own agreement (rel-RMS 1e-5)."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent


def _run(form, tmp_path):
    env = dict(os.environ)
    env.pop("SCARF3D_B200_TABLE_BUILDER", None)
    if form:
        env["SCARF3D_B200_TABLE_BUILDER"] = form
    out = tmp_path / f"{form or 'warps'}.npz"
    r = subprocess.run([sys.executable, str(HERE / "builder_fields.py"), str(out)], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return dict(np.load(out))


@pytest.fixture(scope="module")
def forms(tmp_path_factory):
    d = tmp_path_factory.mktemp("builders")
    return {f: _run(f, d) for f in ("", "block", "direct")}


def test_warp_and_block_builders_give_identical_fields(forms):
    warps, block = forms[""], forms["block"]
    assert warps.keys() == block.keys()
    for k in warps:
        assert np.all(np.isfinite(warps[k])), k
        assert np.array_equal(warps[k].view(np.uint32), block[k].view(np.uint32)), k


def test_direct_builders_agree_within_tolerance(forms):
    warps, direct = forms[""], forms["direct"]
    for k in warps:
        assert np.all(np.isfinite(direct[k])), k
        assert rel_rms(direct[k], warps[k]) <= 1e-5, k
