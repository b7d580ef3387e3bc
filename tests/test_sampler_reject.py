"""The device scan's certain-reject table (host code, no GPU): a pair whose
second raw draw y2 reaches its bin's threshold must fail the full rejection
test r2 < d(u) (1 + margin) for every first draw y1 of the bin, as the
reference's loop evaluates it (scarflib_srm.f90:734-745: u from r(1), d from
srm_fn, accept on r(2) < d). Checked here with the host's FP32 spectrum at
both ends of every bin and at random draws inside it, over the 256-field
batch's spectra and the single-field configurations."""
import numpy as np
import pytest

import scarf3d_b200 as sb
from scarf3d_b200.workloads import batched_fields

INV_M = float.fromhex("0x1.00000002p-31")  # 1 / (2^31 - 1), rounded to double
MARGIN = np.float32(2e-5)


def to_u01(y):
    return (np.asarray(y, np.float64) * INV_M).astype(np.float32)


def decision_bound(p, s, y1):
    """d(u) (1 + margin) in the scan's FP32 order for first draws y1."""
    r1 = to_u01(y1)
    w = np.float32(np.float32(s.kmax) - np.float32(s.kmin))
    u = (r1 * w).astype(np.float32) + np.float32(s.kmin)
    u = u.astype(np.float32)
    if p.acf == 0:
        fv = np.float32(1.0) / np.power((np.float32(1.0) + u * u).astype(np.float32), np.float32(s.nu))
    else:
        fv = np.exp((np.float32(-0.25) * (u * u).astype(np.float32)).astype(np.float32))
    srm = u.astype(np.float64) * fv.astype(np.float32).astype(np.float64)
    if s.ndim == 3:
        srm = srm * u.astype(np.float64)
    d = (srm * np.float64(np.float32(s.cnst))).astype(np.float32)
    return (d * (np.float32(1.0) + MARGIN)).astype(np.float32)


def spectra():
    out = [(f["params"], f["setup"]) for f in batched_fields(count=48)]
    for acf, hurst, cl, ds in [(0, 0.5, [3000.0, 3000.0, 1000.0], 25.0), (0, 0.25, [2000.0] * 3, 50.0),
                               (1, 0.0, [1500.0, 1500.0, 500.0], 100.0), (0, 0.3, [5000.0, 5000.0, 2000.0], 10.0),
                               (0, 0.1, [800.0, 500.0, 0.0], 50.0), (1, 0.0, [800.0, 600.0, 0.0], 50.0)]:
        n = [128, 128, 64 if cl[2] > 0 else 1]
        fc = [float(np.float32(v - 1) * np.float32(ds)) for v in n]
        p = sb.make_params(acf=acf, nharm=100, seed=1, hurst=hurst, sigma=0.05, ds=ds, cl=cl, nc=[0.0] * 3, fc=fc)
        out.append((p, sb.compute_setup(p)))
    return out


@pytest.mark.parametrize("idx", range(54))
def test_reject_table_bounds_the_decision(idx):
    p, s = spectra()[idx]
    thr = sb.sampler_reject_table(p, s)
    rng = np.random.default_rng(idx)
    m = 2 ** 31 - 1
    for b in range(256):
        if thr[b] == 0xFFFFFFFF:
            continue
        lo, hi = b << 23, min((b + 1) << 23, m) - 1
        y1 = np.concatenate([[lo, hi], rng.integers(lo, hi + 1, 256)])
        # every y2 >= thr[b] gives r2 >= to_u01(thr[b]): the full test rejects
        assert to_u01(thr[b]) >= decision_bound(p, s, y1).max(), (b, int(thr[b]))


def test_reject_table_is_tight():
    """Most rejections are taken early: the pairs left for the full test are
    within a small factor of the accepted ones (which it must keep)."""
    for p, s in spectra()[:16]:
        thr = sb.sampler_reject_table(p, s).astype(np.float64)
        survive = np.minimum(thr, 2 ** 31 - 1) / (2 ** 31 - 1)
        acc = s.intg_band * s.cnst / (s.kmax - s.kmin)
        assert survive.mean() <= 3.0 * acc + 1e-3, (survive.mean(), acc)
