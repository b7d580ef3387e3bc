"""scarf_execute end to end (C ABI, GPU) against the CPU oracle's execute:
field, stats[8], rescale, taper, host and device output, both summation
forms, structured and unstructured meshes."""
import ctypes

import numpy as np
import pytest

import oracle
import scarf3d_b200 as sb
from conftest import rel_rms
from srm_cases import random_points

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

KW3 = dict(acf=0, hurst=0.25, sigma=0.05, ds=50.0, cl=[2000.0, 2000.0, 2000.0])


@pytest.fixture(autouse=True)
def _reset():
    sb.set_nharm(400)
    sb.set_form(sb.FORM_AUTO)
    yield
    sb.scarf_finalize()
    sb.set_nharm(10000)
    sb.set_form(sb.FORM_AUTO)


def _oracle_execute(fs, fe, seed, nharm, poi=None, mute=-999.0, taper=-999.0, rescale=0, **kw):
    p = oracle.structured_params(acf=kw["acf"], nharm=nharm, seed=seed, hurst=kw["hurst"], sigma=kw["sigma"],
                                 ds=kw["ds"], cl=kw["cl"], fs=fs, fe=fe, rescale=rescale,
                                 alpha=kw.get("alpha", 0.0), beta=kw.get("beta", 0.0), gamma=kw.get("gamma", 0.0))
    return oracle.execute_structured(p, fs + [1] * (3 - len(fs)), fe + [1] * (3 - len(fe)), poi=poi, mute=mute,
                                     taper=taper, nthreads=8), p


@pytest.mark.parametrize("form,tol", [(sb.FORM_DIRECT, 1e-6), (sb.FORM_TC, 2e-5)])
def test_execute_structured_matches_oracle(form, tol):
    fs, fe = [1, 1, 1], [48, 40, 36]
    sb.set_form(form)
    sb.scarf_initialize(fs=fs, fe=fe, acf=KW3["acf"], ds=KW3["ds"], cl=KW3["cl"], sigma=KW3["sigma"], method=1,
                        hurst=KW3["hurst"])
    field, stats = sb.scarf_execute(1235)
    (ref, info), _ = _oracle_execute(fs, fe, 1235, 400, **KW3)
    assert rel_rms(field, ref) <= tol
    assert stats[0] == info[0] and stats[1] == info[1]
    assert abs(stats[2] / info[2] - 1) <= 10 * tol
    assert abs(stats[3] - info[3]) <= 10 * tol * info[2]
    assert stats[4] > 0 and stats[5] > 0 and stats[6] == 0 and stats[7] == 0


def test_execute_rescale_and_taper_structured():
    fs, fe = [1, 1, 1], [40, 32, 24]
    poi = np.array([[700.0, 500.0, 400.0], [1500.0, 1200.0, 900.0]], np.float32)
    sb.set_form(sb.FORM_DIRECT)
    sb.scarf_initialize(fs=fs, fe=fe, acf=0, ds=50.0, cl=[2000.0] * 3, sigma=0.05, method=1, hurst=0.25,
                        rescale=1, poi=poi, mute=300.0, taper=500.0, alpha=30.0, beta=-10.0)
    field, stats = sb.scarf_execute(1235)
    (ref, info), _ = _oracle_execute(fs, fe, 1235, 400, poi=poi, mute=300.0, taper=500.0, rescale=1,
                                     alpha=30.0, beta=-10.0, **dict(KW3))
    assert stats[2] == np.float32(0.05) and stats[3] == 0.0
    assert np.array_equal(field == 0.0, ref == 0.0)  # identical mute decisions
    assert rel_rms(field, ref) <= 1e-6


def test_execute_device_output_equals_host_output():
    fs, fe = [3, 2, 5], [50, 37, 29]
    sb.scarf_initialize(fs=fs, fe=fe, acf=1, ds=100.0, cl=[1500.0, 1500.0, 500.0], sigma=0.1, method=1)
    host, st_h = sb.scarf_execute(7)
    dev = torch.empty(host.size, dtype=torch.float32, device="cuda")
    _, st_d = sb.scarf_execute(7, dev)
    assert np.array_equal(dev.cpu().numpy(), host)
    assert np.array_equal(st_h[:4], st_d[:4])


def test_execute_2d_structured_tc():
    fs, fe = [1, 1], [300, 200]
    kw = dict(acf=1, hurst=0.0, sigma=0.05, ds=50.0, cl=[2000.0, 1200.0], alpha=20.0)
    sb.scarf_initialize(fs=fs, fe=fe, method=1, **kw)
    field, stats = sb.scarf_execute(1235)
    (ref, info), p = _oracle_execute(fs, fe, 1235, 400, **kw)
    s = oracle.setup(p)
    tab, _ = oracle.sample(p, s)
    ref64 = oracle.sum_structured(s, [1, 1, 1], [300, 200, 1], 50.0, tab, f64=True)
    assert rel_rms(field, ref64) <= 1e-5
    assert rel_rms(field, ref) <= 2e-5


def _oracle_points(x, y, z, seed, nharm, acf, hurst, sigma, dh, cl):
    nd = len(cl)
    nc = [float(a.min()) for a in (x, y, z)][:nd] + [0.0] * (3 - nd)
    fc = [float(a.max()) for a in (x, y, z)][:nd] + [0.0] * (3 - nd)
    p = oracle.params(acf=acf, nharm=nharm, seed=seed, hurst=hurst, sigma=sigma, ds=dh, dh=dh, cl=cl, nc=nc, fc=fc)
    s = oracle.setup(p)
    tab, _ = oracle.sample(p, s)
    return oracle.sum_points(s, x, y, z, tab), s, tab


def test_execute_unstructured_3d():
    x, y, z = random_points(5003, box=(6000.0, 5000.0, 3000.0), seed=3)
    sb.scarf_initialize(x=x, y=y, z=z, dh=100.0, acf=1, cl=[1500.0, 1500.0, 500.0], sigma=0.1, method=1)
    field, stats = sb.scarf_execute(7)
    ref, s, tab = _oracle_points(x, y, z, 7, 400, 1, 0.0, 0.1, 100.0, [1500.0, 1500.0, 500.0])
    assert rel_rms(field, ref) <= 1e-6
    assert abs(stats[2] / np.sqrt(oracle.variance(ref)) - 1) < 1e-5


def test_execute_unstructured_2d_zero_z():
    x, y, _ = random_points(3001, box=(8000.0, 6000.0, 1.0), seed=4)
    sb.scarf_initialize(x=x, y=y, dh=50.0, acf=0, cl=[2000.0, 2000.0], sigma=0.05, method=1, hurst=0.25)
    field, _ = sb.scarf_execute(11)
    ref, _, _ = _oracle_points(x, y, np.zeros_like(x), 11, 400, 0, 0.25, 0.05, 50.0, [2000.0, 2000.0])
    assert rel_rms(field, ref) <= 1e-6


def test_unstructured_taper_follows_reference_unless_requested():
    """The reference never tapers unstructured meshes (poi is assigned into a
    0x0 array, scarflib.f90:273,283); SCARF_TAPER_UNSTRUCTURED applies it."""
    x, y, z = random_points(4000, box=(4000.0, 4000.0, 2000.0), seed=5)
    poi = np.array([[2000.0, 2000.0, 1000.0]], np.float32)
    sb.scarf_initialize(x=x, y=y, z=z, dh=100.0, acf=0, cl=[1500.0] * 3, sigma=0.05, method=1, hurst=0.5,
                        poi=poi, mute=400.0, taper=600.0)
    plain, _ = sb.scarf_execute(9)
    tapered, _ = sb.scarf_execute(9, flags=sb.TAPER_UNSTRUCTURED)
    ref, _, _ = _oracle_points(x, y, z, 9, 400, 0, 0.5, 0.05, 100.0, [1500.0] * 3)
    assert rel_rms(plain, ref) <= 1e-6
    exp = ref.copy()
    oracle.taper_points(x, y, z, exp, poi[0], 400.0, 600.0)
    assert np.array_equal(tapered == 0.0, exp == 0.0)
    assert rel_rms(tapered, exp) <= 1e-6


def test_infeasible_domain_returns_an_error():
    sb.scarf_initialize(fs=[1, 1], fe=[24, 18], ds=50.0, acf=1, cl=[2000.0, 1200.0], sigma=0.05, method=1)
    with pytest.raises(sb.ScarfError) as e:
        sb.scarf_execute(1)
    assert e.value.code == sb.SCARF_ERR_ARG


@pytest.mark.parametrize("fs,fe,items", [
    ([2, 3, 1], [150, 130, 290], 3),    # ragged row blocks and column tiles, many slabs
    ([1, 1, 1], [64, 64, 520], 1),      # default slab size, three column tiles
    ([1, 1], [300, 600], 2),            # 2D: three column tiles along y
])
def test_execute_overlapped_output_matches_serial(fs, fe, items):
    kw = dict(acf=0, hurst=0.25, sigma=0.05, ds=50.0, cl=[2000.0] * len(fe), method=1)
    sb.set_form(sb.FORM_TC)
    sb.scarf_initialize(fs=fs, fe=fe, **kw)
    try:
        sb.set_output_overlap(0)
        serial, st0 = sb.scarf_execute(4321)
        sb.set_output_overlap(items)
        overlapped, st1 = sb.scarf_execute(4321)
    finally:
        sb.set_output_overlap(1)
    assert np.array_equal(overlapped.view(np.uint32), serial.view(np.uint32))
    assert np.array_equal(st0[:4], st1[:4])


def test_execute_overlap_falls_back_when_rescaling():
    fs, fe = [1, 1, 1], [96, 80, 300]
    sb.set_form(sb.FORM_TC)
    sb.scarf_initialize(fs=fs, fe=fe, acf=1, ds=50.0, cl=[1500.0] * 3, sigma=0.05, method=1, rescale=1)
    try:
        sb.set_output_overlap(0)
        a, sa = sb.scarf_execute(99)
        sb.set_output_overlap(2)
        b, sbb = sb.scarf_execute(99)
    finally:
        sb.set_output_overlap(1)
    assert np.array_equal(a, b) and np.array_equal(sa[:4], sbb[:4])
    assert sbb[2] == np.float32(0.05)


@pytest.mark.parametrize("form,rescale,method", [(sb.FORM_TC, 0, 1), (sb.FORM_TC, 1, 1), (sb.FORM_DIRECT, 0, 1),
                                                 (sb.FORM_AUTO, 0, 0)])
def test_execute_pageable_and_page_locked_outputs_agree(form, rescale, method):
    """Pageable host fields go through the page-locked bounce ring (in slabs
    while the tensor-core kernel runs, or in whole after it); page-locked
    fields are copied directly; both equal the device output bit for bit."""
    fs, fe = [1, 1, 1], [130, 96, 290]
    sb.set_form(form)
    sb.scarf_initialize(fs=fs, fe=fe, acf=0, hurst=0.25, sigma=0.05, ds=50.0, cl=[2000.0] * 3, method=method,
                        rescale=rescale)
    npts = int(np.prod([e - s + 1 for s, e in zip(fs, fe)]))
    sb.set_output_overlap(2)
    try:
        dev = torch.empty(npts, dtype=torch.float32, device="cuda")
        _, sd = sb.scarf_execute(77, dev)
        pageable = np.full(npts, np.nan, np.float32)
        _, sp = sb.scarf_execute(77, pageable)
        pinned = torch.full((npts,), float("nan"), dtype=torch.float32, pin_memory=True)
        _, sl = sb.scarf_execute(77, pinned.numpy())
    finally:
        sb.set_output_overlap(1)
    ref = dev.cpu().numpy()
    assert np.array_equal(pageable.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(pinned.numpy().view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(sd[:4], sp[:4]) and np.array_equal(sd[:4], sl[:4])
