"""Accuracy of the tensor-core form against the FP64 oracle at harmonic counts
where tensor-core accumulation error matters (sampled points; the oracle is
exact FP64 over the identical FP32 harmonic table)."""
import ctypes

import numpy as np
import pytest

from srm_cases import iarr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _run_tc(lib, s, fs, n, ds, tab):
    out = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
    dt = torch.from_numpy(tab.reshape(-1).copy()).cuda()
    wb = lib.tc_workspace_bytes(s.ndim, n, len(tab))
    work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    lib.check(lib.lib.scarf_srm_tc_structured(ctypes.byref(s), iarr(fs), iarr(n), float(ds),
                                              ctypes.c_void_p(dt.data_ptr()), len(tab),
                                              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(work.data_ptr()),
                                              wb, None))
    return out


@pytest.mark.parametrize("nharm,n", [(8000, (128, 96, 64)), (20000, (64, 64, 48))])
def test_tc_vs_fp64_large_harmonic_count(lib, orc, nharm, n):
    kw = dict(acf=0, nharm=nharm, seed=1234, hurst=0.5, sigma=0.05, ds=25.0, cl=[3000.0, 3000.0, 1000.0])
    fs = [1, 1, 1]
    fe = list(n)
    op = orc.structured_params(fs=fs, fe=fe, **kw)
    p = lib.make_params(nc=list(op.nc), fc=list(op.fc), **kw)
    s = lib.compute_setup(p)
    tab, _ = lib.sample(p, s)
    out = _run_tc(lib, s, fs, list(n), kw["ds"], tab)
    fstd = float(out.double().std().item())
    rng = np.random.default_rng(1)
    idx = np.sort(rng.choice(int(np.prod(n)), size=256, replace=False)).astype(np.int64)
    got = out[torch.from_numpy(idx).cuda()].cpu().numpy().astype(np.float64)
    ref = orc.sum_structured(orc.setup(op), fs, list(n), kw["ds"], tab, idx=idx, f64=True)
    err = float(np.sqrt(np.mean((got - ref) ** 2)) / fstd)
    assert err <= 1e-5, err
