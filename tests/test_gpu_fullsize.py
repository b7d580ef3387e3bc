"""Full-size workloads on the GPU, checked point by point over the whole field
against the FP64 sum over the identical harmonic table (oracle/gpu_fp64.py,
itself pinned to the CPU FP64 oracle below), at sampled points against the
CPU oracle (FP32 restatement and FP64), and through size-independent
properties (determinism, statistics)."""
import ctypes

import numpy as np
import pytest

import oracle
import scarf3d_b200 as sb
from oracle import gpu_fp64
from srm_cases import iarr, random_points, structured_case

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _sampled_errors(field_dev, ref_fn, npts, count=256, seed=0):
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(npts, size=count, replace=False)).astype(np.int64)
    got = field_dev[torch.from_numpy(idx).cuda()].cpu().numpy().astype(np.float64)
    fstd = float(field_dev.double().std().item())
    r64 = ref_fn(idx, True)
    r32 = ref_fn(idx, False).astype(np.float64)
    e64 = float(np.sqrt(np.mean((got - r64) ** 2)) / fstd)
    e32 = float(np.sqrt(np.mean((got - r32) ** 2)) / fstd)
    return e64, e32, float(np.max(np.abs(got - r64)))


def _structured(n, ds, kw, seed, nharm, form, dh=None):
    fs = [1, 1, 1]
    op = oracle.structured_params(fs=fs, fe=list(n), acf=kw["acf"], nharm=nharm, seed=seed, hurst=kw["hurst"],
                                  sigma=kw["sigma"], ds=ds, dh=dh, cl=kw["cl"])
    p = sb.make_params(nc=list(op.nc), fc=list(op.fc), acf=kw["acf"], nharm=nharm, seed=seed, hurst=kw["hurst"],
                       sigma=kw["sigma"], ds=ds, dh=dh, cl=kw["cl"])
    s = sb.compute_setup(p)
    tab, _ = sb.sample(p, s)
    d_tab = torch.from_numpy(tab.reshape(-1).copy()).cuda()
    npts = int(np.prod(n))
    out = torch.empty(npts, dtype=torch.float32, device="cuda")
    if form == "tc":
        wb = sb.tc_workspace_bytes(3, list(n), len(tab))
        work = torch.empty(wb, dtype=torch.uint8, device="cuda")
        sb.check(sb.lib.scarf_srm_tc_structured(ctypes.byref(s), iarr(fs), iarr(n), ds,
                                                ctypes.c_void_p(d_tab.data_ptr()), len(tab),
                                                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(work.data_ptr()),
                                                wb, None))
    else:
        sb.check(sb.lib.scarf_srm_direct_structured(ctypes.byref(s), iarr(fs), iarr(n), ds,
                                                    ctypes.c_void_p(d_tab.data_ptr()), len(tab),
                                                    ctypes.c_void_p(out.data_ptr()), None))
    so = oracle.setup(op)

    def ref(idx, f64):
        return oracle.sum_structured(so, fs, list(n), ds, tab, idx=idx, f64=f64)

    def full():
        return gpu_fp64.compare_structured(out, so, fs, list(n), ds, tab)

    ref.full = full
    ref.tab = tab
    ref.setup = so
    return out, ref, npts


# --------------------------------------------------- the FP64 full-field checker
@pytest.mark.parametrize("name", ["vk3d", "vk3d_rot_offset", "vk3d_dh_lt_ds", "gs2d"])
def test_fp64_checker_matches_cpu_fp64_oracle_structured(name):
    case = structured_case(name)
    so = oracle.setup(case["op"])
    tab, _ = oracle.sample(case["op"], so)
    ref = oracle.sum_structured(so, case["fs"], case["n"], case["ds"], tab, f64=True)
    got = gpu_fp64.structured_field(so, case["fs"], case["n"], case["ds"], tab).cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-11 * ref.std()


def test_fp64_checker_matches_cpu_fp64_oracle_points():
    x, y, z = random_points(5000)
    p = oracle.params(acf=1, nharm=400, seed=7, sigma=0.1, ds=100.0, cl=[1500.0, 1500.0, 500.0],
                      nc=[float(a.min()) for a in (x, y, z)], fc=[float(a.max()) for a in (x, y, z)], alpha=25.0)
    s = oracle.setup(p)
    tab, _ = oracle.sample(p, s)
    ref = oracle.sum_points(s, x, y, z, tab, f64=True)
    dx, dy, dz = (torch.from_numpy(a.copy()).cuda() for a in (x, y, z))
    got = gpu_fp64.points_field(s, dx, dy, dz, tab).cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-11 * ref.std()


def test_plain_config_128cubed_direct():
    """128^3 at 50 m, von Karman H=0.25, cl 2000 m, sigma 0.05, 5000 harmonics, seed 1234."""
    kw = dict(acf=0, hurst=0.25, sigma=0.05, cl=[2000.0, 2000.0, 2000.0])
    out, ref, npts = _structured((128, 128, 128), 50.0, kw, 1234, 5000, "direct")
    e64, e32, _ = _sampled_errors(out, ref, npts)
    assert e32 <= 1e-6
    assert e64 <= 5e-5
    full = ref.full()  # every point against the FP64 sum
    assert full["points"] == npts and full["rel_rms"] <= 5e-5, full


def test_precision_config_512cubed_tc_and_determinism():
    """512^3 at 25 m, von Karman H=0.5, cl 3000/3000/1000 m, 20000 harmonics."""
    kw = dict(acf=0, hurst=0.5, sigma=0.05, cl=[3000.0, 3000.0, 1000.0])
    out, ref, npts = _structured((512, 512, 512), 25.0, kw, 1234, 20000, "tc")
    first = out.clone()
    e64, e32, emax = _sampled_errors(out, ref, npts, count=192)
    assert e64 <= 1e-5, e64
    full = ref.full()  # every one of the 1.3e8 points against the FP64 sum
    assert full["points"] == npts and full["rel_rms"] <= 1e-5, full
    assert full["max_abs"] <= 1e-4 * full["std_ref"], full
    # the FP64 checker agrees with the CPU FP64 oracle at 2 000 sampled points
    idx = np.sort(np.random.default_rng(3).choice(npts, size=2000, replace=False)).astype(np.int64)
    g64 = gpu_fp64.structured_field(ref.setup, [1, 1, 1], [512, 512, 512], 25.0, ref.tab).cpu().numpy()[idx]
    assert np.max(np.abs(g64 - ref(idx, True))) <= 1e-10 * full["std_ref"]
    out2, _, _ = _structured((512, 512, 512), 25.0, kw, 1234, 20000, "tc")
    assert torch.equal(first, out2)  # fixed reduction order: bitwise reproducible


def test_precision_config_512cubed_direct_full_field():
    """The plain FP32 direct sum at 512^3 x 20 000, every point against FP64."""
    kw = dict(acf=0, hurst=0.5, sigma=0.05, cl=[3000.0, 3000.0, 1000.0])
    out, ref, npts = _structured((512, 512, 512), 25.0, kw, 1234, 20000, "direct")
    full = ref.full()
    assert full["points"] == npts and full["rel_rms"] <= 5e-5, full


def test_unstructured_config_2M_points_gaussian():
    """2 000 000 points uniform in a 20 x 20 x 10 km box (FP32, numpy default_rng(7)),
    Gaussian ACF, cl 1500/1500/500 m, sigma 0.1, 10000 harmonics, dh 100 m."""
    rng = np.random.default_rng(7)
    pts = (rng.random((3, 2_000_000)) * np.array([20000.0, 20000.0, 10000.0])[:, None]).astype(np.float32)
    x, y, z = pts
    sb.set_nharm(10000)
    try:
        sb.scarf_initialize(x=x, y=y, z=z, dh=100.0, acf=1, cl=[1500.0, 1500.0, 500.0], sigma=0.1, method=1)
        dev = torch.empty(len(x), dtype=torch.float32, device="cuda")
        _, stats = sb.scarf_execute(7, dev)
    finally:
        sb.scarf_finalize()
        sb.set_nharm(10000)
    nc = [float(a.min()) for a in (x, y, z)]
    fc = [float(a.max()) for a in (x, y, z)]
    p = oracle.params(acf=1, nharm=10000, seed=7, sigma=0.1, ds=100.0, cl=[1500.0, 1500.0, 500.0], nc=nc, fc=fc)
    s = oracle.setup(p)
    tab, _ = oracle.sample(p, s)

    def ref(idx, f64):
        return oracle.sum_points(s, x, y, z, tab, idx=idx, f64=f64)

    e64, e32, _ = _sampled_errors(dev, ref, len(x))
    assert e32 <= 1e-6
    assert abs(stats[2] / float(dev.double().std().item()) - 1) < 1e-5
    dx, dy, dz = (torch.from_numpy(a.copy()).cuda() for a in (x, y, z))
    full = gpu_fp64.compare_points(dev, s, dx, dy, dz, tab)  # all 2e6 points against FP64
    assert full["points"] == len(x) and full["rel_rms"] <= 5e-5, full


def test_large_config_2048x2048x512_tc():
    """2048 x 2048 x 512 at 10 m (8.6 GB field), von Karman H=0.3, cl 5000/5000/2000 m,
    sigma 0.08, 50000 harmonics, FP64 phase tables and FP64 statistics."""
    n = [2048, 2048, 512]
    fs, fe = [1, 1, 1], n
    sb.set_nharm(50000)
    sb.set_form(sb.FORM_TC)
    try:
        sb.scarf_initialize(fs=fs, fe=fe, ds=10.0, acf=0, cl=[5000.0, 5000.0, 2000.0], sigma=0.08, method=1,
                            hurst=0.3)
        dev = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
        _, stats = sb.scarf_execute(1234, dev)
    finally:
        sb.scarf_finalize()
        sb.set_nharm(10000)
        sb.set_form(sb.FORM_AUTO)
    op = oracle.structured_params(acf=0, nharm=50000, seed=1234, hurst=0.3, sigma=0.08, ds=10.0,
                                  cl=[5000.0, 5000.0, 2000.0], fs=fs, fe=fe)
    so = oracle.setup(op)
    tab, _ = oracle.sample(op, so)

    def ref(idx, f64):
        return oracle.sum_structured(so, fs, n, 10.0, tab, idx=idx, f64=f64)

    e64, _, _ = _sampled_errors(dev, ref, int(np.prod(n)), count=96)
    assert e64 <= 1e-5, e64
    full = gpu_fp64.compare_structured(dev, so, fs, n, 10.0, tab)  # all 2.1e9 points against FP64
    assert full["points"] == int(np.prod(n)) and full["rel_rms"] <= 1e-5, full
    std = float(dev.double().std().item())
    mean = float(dev.double().mean().item())
    assert abs(stats[2] / std - 1) < 1e-5
    assert abs(stats[3] - mean) < 1e-5 * std
