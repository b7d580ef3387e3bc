"""The allocation-free tensor-core entry point (scarf_srm_tc_structured_noalloc).

It exists for callers that cannot allocate device memory when they need a
field -- their device memory belongs to another allocator, or a per-step
cudaMalloc/cudaFree synchronisation is unacceptable -- and keeps its scratch
in a fixed 64 MiB device array instead of a caller workspace. These tests
call it through the C ABI and check it against the allocating entry point
(scarf_srm_tc_structured) on two calls in a row, so the second call also
shows that the shared scratch left by the first does not leak into results.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_rms
from srm_cases import iarr, structured_case

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _inputs(lib, name, nharm):
    case = structured_case(name, nharm=nharm)
    s = lib.compute_setup(case["pp"])
    tab, _ = lib.sample(case["pp"], s)
    d_tab = torch.from_numpy(tab.reshape(-1).copy()).cuda()
    return case, s, tab, d_tab


def _with_workspace(lib, case, s, d_tab, nh):
    n = case["n"]
    out = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
    wb = lib.tc_workspace_bytes(s.ndim, n, nh)
    work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    lib.check(lib.lib.scarf_srm_tc_structured(ctypes.byref(s), iarr(case["fs"]), iarr(n), float(case["ds"]),
                                              ctypes.c_void_p(d_tab.data_ptr()), nh,
                                              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(work.data_ptr()),
                                              wb, None))
    return out.cpu().numpy()


def _no_alloc(lib, case, s, d_tab, nh):
    n = case["n"]
    out = torch.full((int(np.prod(n)),), float("nan"), dtype=torch.float32, device="cuda")
    lib.check(lib.lib.scarf_srm_tc_structured_noalloc(ctypes.byref(s), iarr(case["fs"]), iarr(n),
                                                      float(case["ds"]), ctypes.c_void_p(d_tab.data_ptr()), nh,
                                                      ctypes.c_void_p(out.data_ptr()), None))
    return out.cpu().numpy()


def test_no_alloc_matches_allocating_entry_point_two_calls_in_a_row(lib):
    # First a larger 3-D block, then a smaller rotated/offset one: the second
    # call runs on scratch still holding the first call's tables.
    for name, nharm in (("gs3d_aniso", 700), ("vk3d_rot_offset", 333)):
        case, s, tab, d_tab = _inputs(lib, name, nharm)
        ref = _with_workspace(lib, case, s, d_tab, len(tab))
        got = _no_alloc(lib, case, s, d_tab, len(tab))
        assert np.all(np.isfinite(got))
        assert rel_rms(got, ref) <= 1e-6


def test_no_alloc_rejects_grids_beyond_its_scratch(lib):
    case, s, tab, d_tab = _inputs(lib, "vk3d", 300)
    cap = int(lib.lib.scarf_srm_tc_noalloc_capacity_bytes())
    big = [1024, 1024, 256]
    assert lib.tc_workspace_bytes(3, big, 20000) > cap
    out = torch.empty(16, dtype=torch.float32, device="cuda")  # never written: the call is rejected first
    rc = lib.lib.scarf_srm_tc_structured_noalloc(ctypes.byref(s), iarr([1, 1, 1]), iarr(big), 25.0,
                                                 ctypes.c_void_p(d_tab.data_ptr()), 20000,
                                                 ctypes.c_void_p(out.data_ptr()), None)
    assert rc == lib.SCARF_ERR_ARG
    assert "64 MiB" in lib.last_error()
