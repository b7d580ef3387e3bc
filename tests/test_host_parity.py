"""Product host code (setup scalars, quadrature, sampler) through the C ABI
against the oracle, bit for bit (no GPU needed)."""
import ctypes

import numpy as np
import pytest

import oracle
import scarf3d_b200 as sb


def _random_cases(count, seed=123):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        three = bool(rng.random() < 0.7)
        acf = int(rng.integers(0, 2))
        ds = float(rng.choice([10.0, 25.0, 50.0, 100.0]))
        n = [int(v) for v in rng.integers(32, 257, size=3 if three else 2)]
        cl = [float(v) for v in rng.uniform(500.0, 5000.0, size=3 if three else 2)]
        dh = ds if rng.random() < 0.7 else ds * float(rng.uniform(0.4, 1.0))
        kw = dict(acf=acf, nharm=int(rng.integers(50, 400)), seed=int(rng.integers(-2**31, 2**31 - 1)),
                  hurst=float(rng.uniform(0.05, 0.95)), sigma=float(rng.uniform(0.01, 0.2)), ds=ds, dh=dh, cl=cl,
                  alpha=float(rng.uniform(-90, 90)) if rng.random() < 0.5 else 0.0,
                  beta=float(rng.uniform(-45, 45)) if rng.random() < 0.3 else 0.0,
                  gamma=float(rng.uniform(-45, 45)) if rng.random() < 0.3 else 0.0)
        out.append((kw, [1] * len(n), n))
    return out


CASES = _random_cases(24)


def _pair(kw, fs, fe):
    op = oracle.structured_params(fs=fs, fe=fe, **kw)
    pp = sb.make_params(nc=list(op.nc), fc=list(op.fc), **kw)
    return op, pp


@pytest.mark.parametrize("case", range(len(CASES)))
def test_setup_and_sampler_bit_exact(case):
    kw, fs, fe = CASES[case]
    op, pp = _pair(kw, fs, fe)
    so = oracle.setup(op)
    acc = so.intg_band * so.cnst / max(so.kmax - so.kmin, 1e-30)
    ps = sb.compute_setup(pp)
    for f, _ in oracle.OrcSetup._fields_:
        assert np.array_equal(np.asarray(getattr(so, f)), np.asarray(getattr(ps, f))), f
    if acc < 1e-6:
        pytest.skip("spectrum mass in [kmin, kmax] too small for rejection sampling")
    if kw["nharm"] / acc > 3e6:
        pytest.skip("sampler comparison would take the (slow) oracle generator over a minute")
    ref, ref_pairs = oracle.sample(op, so)
    for threads in (1, 3, 8):
        sb.set_host_threads(threads)
        got, pairs = sb.sample(pp, ps)
        assert pairs == ref_pairs
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    sb.set_host_threads(0)


def test_parallel_sampler_long_stream():
    kw = dict(acf=0, nharm=20000, seed=1234, hurst=0.5, sigma=0.05, ds=25.0, cl=[3000.0, 3000.0, 1000.0])
    op, pp = _pair(kw, [1, 1, 1], [512, 512, 512])
    ref, ref_pairs = oracle.sample(op, oracle.setup(op))
    sb.set_host_threads(8)
    got, pairs = sb.sample(pp, sb.compute_setup(pp))
    sb.set_host_threads(0)
    assert pairs == ref_pairs and np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_uniform_source_hook_reproduces_a_supplied_stream():
    """A caller-supplied set_seed/srng (here the oracle's generator, standing
    in for the reference's prng.cpp) drives the product's sampler exactly."""
    state = (ctypes.c_int64 * 2)()
    SEED = ctypes.CFUNCTYPE(None, ctypes.c_int)
    SRNG = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_float))

    @SEED
    def set_seed(seed):
        oracle.L.orc_rng_seed(state, seed)

    @SRNG
    def srng(out):
        out[0] = oracle.L.orc_u01(oracle.L.orc_rng_next(state))
        out[1] = oracle.L.orc_u01(oracle.L.orc_rng_next(state))

    kw = dict(acf=1, nharm=300, seed=77, hurst=0.0, sigma=0.1, ds=100.0, cl=[1500.0, 1500.0, 500.0])
    op, pp = _pair(kw, [1, 1, 1], [40, 24, 20])
    ref, ref_pairs = oracle.sample(op, oracle.setup(op))
    sb.check(sb.lib.scarf_set_uniform_source(ctypes.cast(set_seed, ctypes.c_void_p),
                                             ctypes.cast(srng, ctypes.c_void_p)))
    try:
        got, pairs = sb.sample(pp, sb.compute_setup(pp))
    finally:
        sb.check(sb.lib.scarf_set_uniform_source(None, None))
    assert pairs == ref_pairs and np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_infeasible_rejection_sampling_is_refused():
    # Gaussian spectrum whose bulk lies below kmin (grid span small against cl).
    kw = dict(acf=1, nharm=64, seed=1, hurst=0.0, sigma=0.05, ds=50.0, cl=[2000.0, 1200.0])
    op, pp = _pair(kw, [1, 1], [24, 18])
    s = sb.compute_setup(pp)
    assert s.info0 == 1.0  # the reference's "domain too small" flag
    tab = np.zeros((64, 5), np.float32)
    rc = sb.lib.scarf_srm_sample(ctypes.byref(pp), ctypes.byref(s), tab.ctypes.data_as(ctypes.c_void_p), None, None)
    assert rc == sb.SCARF_ERR_ARG
    assert "acceptance rate" in sb.last_error()


def test_threaded_sampler_after_fork():
    # The threaded host sampler runs on a persistent worker pool; a child
    # made by fork() has none of the parent's workers and must build its own
    # (a pool inherited as is would wait for threads that do not exist).
    import os
    fc = [float(np.float32(127) * np.float32(50.0))] * 3
    p = sb.make_params(nc=[0.0] * 3, fc=fc, nharm=2000, acf=0, seed=7, hurst=0.3, sigma=0.05, ds=50.0,
                       cl=[2000.0] * 3)
    s = sb.compute_setup(p)
    sb.lib.scarf_set_host_threads(4)
    try:
        ref, _ = sb.sample(p, s)  # the parent's pool now has workers
        pid = os.fork()
        if pid == 0:  # child: same table, then leave without running pytest's teardown
            try:
                tab, _ = sb.sample(p, s)
                os._exit(0 if np.array_equal(tab.view(np.uint32), ref.view(np.uint32)) else 3)
            except BaseException:  # noqa: BLE001
                os._exit(4)
        _, status = os.waitpid(pid, 0)
        assert os.waitstatus_to_exitcode(status) == 0
        again, _ = sb.sample(p, s)  # and the parent's pool still works
        assert np.array_equal(again.view(np.uint32), ref.view(np.uint32))
    finally:
        sb.lib.scarf_set_host_threads(0)
