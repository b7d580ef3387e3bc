"""The device-assisted harmonic sampler is bit-identical to the serial host
sampling loop (scarflib_srm.f90:731-778): same table, same number of uniform
pairs consumed, for many parameter sets, multi-pass streams and the execute
path."""
import numpy as np
import pytest

import oracle
import scarf3d_b200 as sb
from test_host_parity import CASES

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _compare(pp):
    s = sb.compute_setup(pp)
    acc = s.intg_band * s.cnst / max(s.kmax - s.kmin, 1e-30)
    if acc < 1e-6:
        pytest.skip("infeasible rejection sampling")
    sb.set_host_threads(8)
    host, hp = sb.sample(pp, s)
    sb.set_host_threads(0)
    dev, dpairs, undecided = sb.sample_device(pp, s)
    assert dpairs == hp
    assert np.array_equal(dev.view(np.uint32), host.view(np.uint32))
    return undecided


@pytest.mark.parametrize("case", range(len(CASES)))
def test_device_sampler_matches_host_random_cases(case):
    kw, fs, fe = CASES[case]
    op = oracle.structured_params(fs=fs, fe=fe, **kw)
    _compare(sb.make_params(nc=list(op.nc), fc=list(op.fc), **kw))


@pytest.mark.parametrize("kw,fe", [
    (dict(acf=0, nharm=5000, seed=1234, hurst=0.25, sigma=0.05, ds=50.0, cl=[2000.0] * 3), [128, 128, 128]),
    (dict(acf=0, nharm=20000, seed=1234, hurst=0.5, sigma=0.05, ds=25.0, cl=[3000.0, 3000.0, 1000.0]),
     [512, 512, 512]),
    (dict(acf=0, nharm=50000, seed=1234, hurst=0.3, sigma=0.08, ds=10.0, cl=[5000.0, 5000.0, 2000.0]),
     [2048, 2048, 512]),
    (dict(acf=1, nharm=4000, seed=9, hurst=0.0, sigma=0.1, ds=100.0, dh=40.0, cl=[1500.0, 1500.0, 500.0]),
     [200, 200, 100]),
])
def test_device_sampler_matches_host_configs(kw, fe):
    op = oracle.structured_params(fs=[1, 1, 1], fe=fe, **kw)
    _compare(sb.make_params(nc=list(op.nc), fc=list(op.fc), **kw))


def test_device_sampler_low_acceptance_multi_pass():
    # Gaussian spectrum with kmin well inside its tail: acceptance ~1e-5,
    # hundreds of thousands of pairs per harmonic.
    kw = dict(acf=1, nharm=300, seed=77, hurst=0.0, sigma=0.05, ds=50.0, cl=[2000.0, 2000.0, 2000.0])
    op = oracle.structured_params(fs=[1, 1, 1], fe=[48, 48, 48], **kw)
    pp = sb.make_params(nc=list(op.nc), fc=list(op.fc), **kw)
    s = sb.compute_setup(pp)
    acc = s.intg_band * s.cnst / (s.kmax - s.kmin)
    assert 1e-6 < acc < 1e-3
    _compare(pp)
    # Force many short passes: the walk must chain them seamlessly.
    sb.check(sb.lib.scarf_set_sampler_pass_pairs(100_003))
    try:
        _compare(pp)
    finally:
        sb.check(sb.lib.scarf_set_sampler_pass_pairs(0))


def test_device_sampler_matches_the_oracle():
    kw = dict(acf=0, nharm=3000, seed=4321, hurst=0.7, sigma=0.05, ds=50.0, cl=[2500.0, 1500.0, 1000.0],
              alpha=25.0)
    op = oracle.structured_params(fs=[1, 1, 1], fe=[100, 90, 80], **kw)
    ref, ref_pairs = oracle.sample(op, oracle.setup(op))
    pp = sb.make_params(nc=list(op.nc), fc=list(op.fc), **kw)
    dev, pairs, _ = sb.sample_device(pp, sb.compute_setup(pp))
    assert pairs == ref_pairs and np.array_equal(dev.view(np.uint32), ref.view(np.uint32))


def test_execute_device_and_host_samplers_give_the_same_field():
    sb.set_nharm(2000)
    try:
        sb.scarf_initialize(fs=[1, 1, 1], fe=[64, 48, 40], ds=50.0, acf=0, cl=[2000.0] * 3, sigma=0.05, method=1,
                            hurst=0.25)
        sb.set_sampler(sb.SAMPLER_HOST)
        a, sa = sb.scarf_execute(1235)
        sb.set_sampler(sb.SAMPLER_DEVICE)
        b, sbb = sb.scarf_execute(1235)
        assert np.array_equal(a, b) and np.array_equal(sa[:4], sbb[:4])
    finally:
        sb.set_sampler(sb.SAMPLER_AUTO)
        sb.scarf_finalize()
        sb.set_nharm(10000)


def _batch_fields():
    out = []
    for kw, fs, fe in CASES:
        op = oracle.structured_params(fs=fs, fe=fe, **kw)
        pp = sb.make_params(nc=list(op.nc), fc=list(op.fc), **kw)
        s = sb.compute_setup(pp)
        if s.intg_band * s.cnst / max(s.kmax - s.kmin, 1e-30) >= 1e-6:
            out.append((pp, s))
    kw = dict(acf=1, nharm=300, seed=77, hurst=0.0, sigma=0.05, ds=50.0, cl=[2000.0, 2000.0, 2000.0])
    op = oracle.structured_params(fs=[1, 1, 1], fe=[48, 48, 48], **kw)
    pp = sb.make_params(nc=list(op.nc), fc=list(op.fc), **kw)
    out.append((pp, sb.compute_setup(pp)))  # low acceptance (~1e-5)
    return out


def test_batched_device_sampler_matches_per_field_sampler():
    fields = _batch_fields()
    tabs, used, _ = sb.sample_device_batch([f[0] for f in fields], [f[1] for f in fields])
    for (pp, s), t, u in zip(fields, tabs, used):
        ref, ref_pairs, _ = sb.sample_device(pp, s)
        assert u == ref_pairs
        assert np.array_equal(t.view(np.uint32), ref.view(np.uint32))


def test_batched_device_sampler_writes_into_caller_arrays():
    # Tables written in place into views of one buffer equal those of
    # library-allocated arrays; the views keep the rows beyond `kept` untouched.
    fields = _batch_fields()
    ps, ss = [f[0] for f in fields], [f[1] for f in fields]
    ref, ref_used, _ = sb.sample_device_batch(ps, ss)
    offs = np.concatenate([[0], np.cumsum([5 * p.nharm + 20 for p in ps])])
    buf = np.full(int(offs[-1]), -7.0, np.float32)
    views = [buf[offs[i]:offs[i + 1]] for i in range(len(ps))]
    got, used, _ = sb.sample_device_batch(ps, ss, out=views)
    assert list(used) == list(ref_used)
    for i, (g, r) in enumerate(zip(got, ref)):
        assert np.array_equal(g.view(np.uint32), r.view(np.uint32))
        assert np.shares_memory(g, buf)
        assert np.all(buf[offs[i] + 5 * ps[i].nharm:offs[i + 1]] == -7.0)


def test_batched_device_sampler_redoes_fields_whose_slots_overflowed(monkeypatch):
    # One candidate slot per scan thread: most threads overflow, their fields
    # are redone with their own passes, and the tables must not change.
    fields = _batch_fields()
    ref = sb.sample_device_batch([f[0] for f in fields], [f[1] for f in fields])
    monkeypatch.setenv("SCARF3D_B200_SAMPLER_SLOT_CAP", "1")
    got = sb.sample_device_batch([f[0] for f in fields], [f[1] for f in fields])
    for t, r in zip(got[0], ref[0]):
        assert np.array_equal(t.view(np.uint32), r.view(np.uint32))
    assert list(got[1]) == list(ref[1])


def test_batched_device_sampler_chains_further_passes():
    fields = _batch_fields()
    sb.check(sb.lib.scarf_set_sampler_pass_pairs(1_000_003))  # first passes run short
    try:
        tabs, used, _ = sb.sample_device_batch([f[0] for f in fields], [f[1] for f in fields])
    finally:
        sb.check(sb.lib.scarf_set_sampler_pass_pairs(0))
    for (pp, s), t, u in zip(fields, tabs, used):
        sb.set_host_threads(8)
        host, hp = sb.sample(pp, s)
        sb.set_host_threads(0)
        assert u == hp
        assert np.array_equal(t.view(np.uint32), host.view(np.uint32))


def test_batched_device_sampler_on_the_many_realisation_workload():
    # Against the host loop, which evaluates the full test for every pair
    # (the scan drops most pairs early on its reject table).
    from scarf3d_b200.workloads import batched_fields
    spec = batched_fields(count=24)
    tabs, used, _ = sb.sample_device_batch([f["params"] for f in spec], [f["setup"] for f in spec])
    sb.set_host_threads(16)
    try:
        for f, t, u in zip(spec, tabs, used):
            ref, ref_pairs = sb.sample(f["params"], f["setup"])
            assert u == ref_pairs and np.array_equal(t.view(np.uint32), ref.view(np.uint32))
    finally:
        sb.set_host_threads(0)


def test_batched_device_sampler_names_an_infeasible_field():
    fields = _batch_fields()[:3]
    kw = dict(acf=1, nharm=100, seed=5, hurst=0.0, sigma=0.05, ds=50.0, cl=[2000.0, 2000.0, 2000.0])
    op = oracle.structured_params(fs=[1, 1, 1], fe=[12, 12, 12], **kw)
    bad = sb.make_params(nc=list(op.nc), fc=list(op.fc), **kw)
    ps = [f[0] for f in fields] + [bad]
    ss = [f[1] for f in fields] + [sb.compute_setup(bad)]
    with pytest.raises(sb.ScarfError, match="field 3"):
        sb.sample_device_batch(ps, ss)
