"""GPU parity of the device kernels, called through the C ABI, against the
CPU oracle on the same harmonic tables (bit-exact host setup/sampler is
checked on the CPU in test_host_parity.py)."""
import ctypes

import numpy as np
import pytest

from conftest import rel_rms
from srm_cases import iarr, random_points, structured_case

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _direct_structured(lib, case, tab):
    s = lib.compute_setup(case["pp"])
    n = case["n"]
    out = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
    dt = _dev(tab.reshape(-1))
    lib.check(lib.lib.scarf_srm_direct_structured(ctypes.byref(s), iarr(case["fs"]), iarr(n), float(case["ds"]),
                                                  ctypes.c_void_p(dt.data_ptr()), len(tab),
                                                  ctypes.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _tc_structured(lib, case, tab):
    s = lib.compute_setup(case["pp"])
    n = case["n"]
    out = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
    dt = _dev(tab.reshape(-1))
    wb = lib.tc_workspace_bytes(s.ndim, n, len(tab))
    assert wb > 0
    work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    lib.check(lib.lib.scarf_srm_tc_structured(ctypes.byref(s), iarr(case["fs"]), iarr(n), float(case["ds"]),
                                              ctypes.c_void_p(dt.data_ptr()), len(tab),
                                              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(work.data_ptr()),
                                              wb, None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name", ["vk3d", "gs3d_aniso", "vk3d_rot_offset", "vk3d_dh_lt_ds", "gs2d"])
def test_direct_structured_matches_fp32_restatement(lib, orc, name):
    case = structured_case(name)
    s_o = orc.setup(case["op"])
    tab, _ = lib.sample(case["pp"], lib.compute_setup(case["pp"]))
    got = _direct_structured(lib, case, tab)
    ref32 = orc.sum_structured(s_o, case["fs"], case["n"], case["ds"], tab)
    ref64 = orc.sum_structured(s_o, case["fs"], case["n"], case["ds"], tab, f64=True)
    # Same operations in the same order; only sinf/cosf ulps differ.
    assert rel_rms(got, ref32) <= 1e-6
    assert np.max(np.abs(got - ref32)) <= 1e-5 * ref32.std()
    assert rel_rms(got, ref64) <= 1e-4


def test_direct_points_matches_fp32_restatement(lib, orc):
    case = structured_case("gs3d_aniso", nharm=700)
    s = lib.compute_setup(case["pp"])
    s_o = orc.setup(case["op"])
    tab, _ = lib.sample(case["pp"], s)
    x, y, z = random_points(1001, box=(4000.0, 2400.0, 2000.0))
    out = torch.empty(len(x), dtype=torch.float32, device="cuda")
    dx, dy, dz, dt = _dev(x), _dev(y), _dev(z), _dev(tab.reshape(-1))
    lib.check(lib.lib.scarf_srm_direct_points(ctypes.byref(s), ctypes.c_void_p(dx.data_ptr()),
                                              ctypes.c_void_p(dy.data_ptr()), ctypes.c_void_p(dz.data_ptr()),
                                              len(x), ctypes.c_void_p(dt.data_ptr()), len(tab),
                                              ctypes.c_void_p(out.data_ptr()), None))
    got = out.cpu().numpy()
    ref32 = orc.sum_points(s_o, x, y, z, tab)
    assert rel_rms(got, ref32) <= 1e-6


def test_direct_unaligned_table_and_tail(lib, orc):
    """Table base not 16-byte aligned (plain-load path) and a partial tile."""
    case = structured_case("vk3d", nharm=517)
    s = lib.compute_setup(case["pp"])
    s_o = orc.setup(case["op"])
    tab, _ = lib.sample(case["pp"], s)
    n = case["n"]
    buf = torch.zeros(tab.size + 1, dtype=torch.float32, device="cuda")
    buf[1:] = torch.from_numpy(tab.reshape(-1)).cuda()
    out = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
    lib.check(lib.lib.scarf_srm_direct_structured(ctypes.byref(s), iarr(case["fs"]), iarr(n), float(case["ds"]),
                                                  ctypes.c_void_p(buf.data_ptr() + 4), len(tab),
                                                  ctypes.c_void_p(out.data_ptr()), None))
    got = out.cpu().numpy()
    ref32 = orc.sum_structured(s_o, case["fs"], n, case["ds"], tab)
    assert rel_rms(got, ref32) <= 1e-6


@pytest.mark.parametrize("name", ["vk3d", "gs3d_aniso", "vk3d_rot_offset", "vk3d_dh_lt_ds", "gs2d", "vk2d"])
def test_tc_matches_fp64_oracle(lib, orc, name):
    case = structured_case(name)
    s_o = orc.setup(case["op"])
    tab, _ = lib.sample(case["pp"], lib.compute_setup(case["pp"]))
    got = _tc_structured(lib, case, tab)
    ref64 = orc.sum_structured(s_o, case["fs"], case["n"], case["ds"], tab, f64=True)
    err = rel_rms(got, ref64)
    assert err <= 1e-5, err
    assert np.max(np.abs(got - ref64)) <= 2e-4 * ref64.std()


def test_tc_agrees_with_direct(lib, orc):
    case = structured_case("vk3d_rot_offset")
    tab, _ = lib.sample(case["pp"], lib.compute_setup(case["pp"]))
    tc = _tc_structured(lib, case, tab)
    direct = _direct_structured(lib, case, tab)
    assert rel_rms(tc, direct) <= 1e-4


@pytest.mark.parametrize("mode,tol", [(1, 1e-6), (0, 3e-7)])
def test_direct_sincos_modes_on_large_phases(lib, orc, mode, tol):
    """Points over 20 x 20 x 10 km with 1500/500 m correlation lengths put
    the phases at thousands of radians: the fast mode (Cody-Waite reduction
    to [-pi, pi] + SFU sin/cos) stays within 1e-6 of the FP32 restatement,
    CUDA's sincosf within 3e-7."""
    x, y, z = random_points(20000, seed=11)
    kw = dict(acf=1, nharm=3000, seed=7, hurst=0.0, sigma=0.1, ds=100.0, cl=[1500.0, 1500.0, 500.0])
    nc = [float(a.min()) for a in (x, y, z)]
    fc = [float(a.max()) for a in (x, y, z)]
    pp = lib.make_params(nc=nc, fc=fc, **kw)
    s = lib.compute_setup(pp)
    tab, _ = lib.sample(pp, s)
    so = orc.setup(orc.params(nc=nc, fc=fc, **kw))
    dx, dy, dz, dt = (_dev(a) for a in (x, y, z, tab.reshape(-1)))
    out = torch.empty(len(x), dtype=torch.float32, device="cuda")
    try:
        lib.set_direct_sincos(mode)
        lib.check(lib.lib.scarf_srm_direct_points(ctypes.byref(s), ctypes.c_void_p(dx.data_ptr()),
                                                  ctypes.c_void_p(dy.data_ptr()), ctypes.c_void_p(dz.data_ptr()),
                                                  len(x), ctypes.c_void_p(dt.data_ptr()), len(tab),
                                                  ctypes.c_void_p(out.data_ptr()), None))
    finally:
        lib.set_direct_sincos(1)
    got = out.cpu().numpy()
    ref32 = orc.sum_points(so, x, y, z, tab)
    assert rel_rms(got, ref32) <= tol
    assert np.max(np.abs(got - ref32)) <= 1e-5 * ref32.std()
