"""Failure paths on the GPU, made without faulting it: (1) the bounded waits
that every pipeline kernel relies on run out on an mbarrier that nothing
arrives on, report the timeout through the status word, and leave the
context usable; (2) a device-memory cap makes the library's own allocations
fail with SCARF_ERR_NOMEM, and the next call after the cap is lifted gives
the same field as a call that never failed."""
import ctypes

import numpy as np
import pytest

import oracle
import scarf3d_b200 as sb
from conftest import rel_rms
from srm_cases import structured_case

pytestmark = pytest.mark.gpu


def _run_case(name):
    c = structured_case(name)
    sb.set_nharm(c["kw"]["nharm"])
    try:
        sb.scarf_initialize(fs=c["fs"], fe=c["fe"], ds=c["ds"], acf=c["kw"]["acf"], cl=c["kw"]["cl"],
                            sigma=c["kw"]["sigma"], method=1, hurst=c["kw"]["hurst"], dh=c["kw"]["dh"],
                            nc=list(c["op"].nc), fc=list(c["op"].fc), alpha=c["kw"]["alpha"],
                            beta=c["kw"]["beta"], gamma=c["kw"]["gamma"])
        field, stats = sb.scarf_execute(c["kw"]["seed"])
        held = sb.device_memory_in_use()  # scarf_finalize frees the library's buffers again
    finally:
        sb.scarf_finalize()
        sb.set_nharm(10000)
    return c, np.asarray(field, np.float32), stats, held


def test_bounded_wait_runs_out_and_the_context_survives():
    r = sb.selftest_wait_limit(4)
    assert r["status"] == 1  # the timeout code
    assert 2.0 <= r["waited_s"] < 6.0  # the 2 s limit, and not much more
    c, field, _, _ = _run_case("vk3d")
    so = oracle.setup(c["op"])
    ref = oracle.sum_structured(so, c["fs"], c["n"], c["ds"], oracle.sample(c["op"], so)[0], f64=True)
    assert rel_rms(field, ref) <= 1e-5


def test_memory_cap_fails_cleanly_and_the_next_call_recovers():
    sb.release_device_memory()
    assert sb.device_memory_in_use() == 0
    _, small, _, held = _run_case("vk3d")  # 17 x 13 x 11: what the library holds during the call
    big_case, big_ref, big_stats, big_held = _run_case("vk3d_rot_offset")  # 56 x 48 x 32
    assert big_case["n"] == [56, 48, 32] and big_held > held > 0
    sb.release_device_memory()
    try:
        sb.set_device_memory_cap(held)
        with pytest.raises(sb.ScarfError) as e:
            _run_case("vk3d_rot_offset")  # its buffers would pass the cap
        assert e.value.code == sb.SCARF_ERR_NOMEM
        assert "memory" in sb.last_error()
        assert sb.device_memory_in_use() <= held
        # the library stays usable under the cap: a failed call may keep some
        # of what it allocated, so free that first
        sb.release_device_memory()
        _, again_small, _, _ = _run_case("vk3d")
        assert np.array_equal(again_small.view(np.uint32), small.view(np.uint32))
    finally:
        sb.set_device_memory_cap(0)
    _, big, stats, _ = _run_case("vk3d_rot_offset")
    assert np.array_equal(big.view(np.uint32), big_ref.view(np.uint32))
    assert np.array_equal(np.asarray(stats, np.float32)[2:4], np.asarray(big_stats, np.float32)[2:4])
