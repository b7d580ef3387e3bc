"""The allocation-free tensor-core entry point (scarf_srm_tc_structured_noalloc).

It exists for callers that cannot allocate device memory when they need a
field -- their device memory belongs to another allocator, or a per-step
cudaMalloc/cudaFree synchronisation is unacceptable -- and keeps its scratch
in a fixed 64 MiB device array instead of a caller workspace. These tests
call it through the C ABI and check it against the allocating entry point
(scarf_srm_tc_structured, same plan, so bit for bit) and against the FP64
oracle, on two calls in a row, so the second call also shows that the shared
scratch left by the first does not leak into results. Every kernel form is
covered, a 2-D grid, and a grid whose scratch fills the array to within a
few hundred bytes (where a layout error at the end of the array would show).
"""
import ctypes

import numpy as np
import pytest

import oracle
import scarf3d_b200 as sb
from conftest import rel_rms
from srm_cases import iarr, structured_case

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

VARIANTS = [sb.TC_SINGLE, sb.TC_SINGLE_TMEM_A, sb.TC_PAIR]


@pytest.fixture(autouse=True)
def _restore_variant():
    yield
    sb.set_tc_variant(sb.TC_SINGLE)


def _inputs(lib, name, nharm):
    case = structured_case(name, nharm=nharm)
    s = lib.compute_setup(case["pp"])
    tab, _ = lib.sample(case["pp"], s)
    return case, s, tab


def _with_workspace(lib, s, fs, n, ds, d_tab, nh):
    out = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
    wb = lib.tc_workspace_bytes(s.ndim, n, nh)
    work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    lib.check(lib.lib.scarf_srm_tc_structured(ctypes.byref(s), iarr(fs), iarr(n), float(ds),
                                              ctypes.c_void_p(d_tab.data_ptr()), nh,
                                              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(work.data_ptr()),
                                              wb, None))
    return out.cpu().numpy()


def _no_alloc(lib, s, fs, n, ds, d_tab, nh):
    out = torch.full((int(np.prod(n)),), float("nan"), dtype=torch.float32, device="cuda")
    lib.check(lib.lib.scarf_srm_tc_structured_noalloc(ctypes.byref(s), iarr(fs), iarr(n), float(ds),
                                                      ctypes.c_void_p(d_tab.data_ptr()), nh,
                                                      ctypes.c_void_p(out.data_ptr()), None))
    return out.cpu().numpy()


def _same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("variant", VARIANTS)
def test_no_alloc_matches_allocating_entry_point_two_calls_in_a_row(lib, variant):
    # A larger 3-D block, then a smaller rotated/offset one, then a 2-D grid:
    # each call after the first runs on scratch still holding the previous
    # call's tables.
    sb.set_tc_variant(variant)
    for name, nharm in (("gs3d_aniso", 700), ("vk3d_rot_offset", 333), ("gs2d", 260)):
        case, s, tab = _inputs(lib, name, nharm)
        d_tab = torch.from_numpy(tab.reshape(-1).copy()).cuda()
        args = (s, case["fs"], case["n"], case["ds"], d_tab, len(tab))
        ref = _with_workspace(lib, *args)
        got = _no_alloc(lib, *args)
        again = _no_alloc(lib, *args)
        assert np.all(np.isfinite(got))
        assert _same_bits(got, ref)
        assert _same_bits(again, ref)
        ref64 = oracle.sum_structured(oracle.setup(case["op"]), case["fs"], case["n"], case["ds"], tab, f64=True)
        assert rel_rms(got, ref64) <= 1e-5


def test_no_alloc_at_the_edge_of_its_scratch(lib):
    # 48 x 40 x 36 points with 61 680 harmonic rows leaves 768 bytes of the
    # 64 MiB array unused; one row more no longer fits.
    cap = int(lib.lib.scarf_srm_tc_noalloc_capacity_bytes())
    case, s, tab = _inputs(lib, "vk3d", 700)
    n, fs, nh = [48, 40, 36], [1, 1, 1], 61680
    need = lib.tc_workspace_bytes(3, n, nh)
    assert 0 < cap - need <= 4096
    assert lib.tc_workspace_bytes(3, n, nh + 1) > cap
    big = np.resize(tab, (nh, tab.shape[1])).astype(np.float32)
    d_tab = torch.from_numpy(np.ascontiguousarray(big.reshape(-1))).cuda()
    args = (s, fs, n, case["ds"], d_tab, nh)
    ref = _with_workspace(lib, *args)
    for _ in range(2):
        got = _no_alloc(lib, *args)
        assert np.all(np.isfinite(got))
        assert _same_bits(got, ref)


def test_no_alloc_rejects_grids_beyond_its_scratch(lib):
    case, s, tab = _inputs(lib, "vk3d", 300)
    d_tab = torch.from_numpy(tab.reshape(-1).copy()).cuda()
    cap = int(lib.lib.scarf_srm_tc_noalloc_capacity_bytes())
    for big, nh in (([1024, 1024, 256], 20000), ([48, 40, 36], 61681)):
        assert lib.tc_workspace_bytes(3, big, nh) > cap
        out = torch.empty(16, dtype=torch.float32, device="cuda")  # never written: the call is rejected first
        rc = lib.lib.scarf_srm_tc_structured_noalloc(ctypes.byref(s), iarr([1, 1, 1]), iarr(big), 25.0,
                                                     ctypes.c_void_p(d_tab.data_ptr()), nh,
                                                     ctypes.c_void_p(out.data_ptr()), None)
        assert rc == lib.SCARF_ERR_ARG
        assert "64 MiB" in lib.last_error()
