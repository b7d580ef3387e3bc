"""The three forms of the tensor-core sum (one CTA per 128-row tile with A in
shared memory, the same with A in tensor memory, and CTA pairs issuing
cta_group::2 MMAs over 256-row tiles) compute the same products in the same
accumulation order per output point: their fields are bit-identical, and
each agrees with the FP64 oracle within the tensor-core tolerance."""
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


def _run(variant, s, fs, n, ds, tab):
    sb.set_tc_variant(variant)
    out = torch.full((int(np.prod(n)),), float("nan"), dtype=torch.float32, device="cuda")
    d_tab = torch.from_numpy(np.ascontiguousarray(tab.reshape(-1))).cuda()
    wb = sb.tc_workspace_bytes(s.ndim, n, len(tab))
    assert wb > 0
    work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    sb.check(sb.lib.scarf_srm_tc_structured(ctypes.byref(s), iarr(fs), iarr(n), float(ds),
                                            ctypes.c_void_p(d_tab.data_ptr()), len(tab),
                                            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(work.data_ptr()),
                                            wb, None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name", ["vk3d", "gs3d_aniso", "vk3d_rot_offset", "gs2d", "vk2d"])
def test_variants_bit_identical_on_oracle_cases(name):
    case = structured_case(name)
    s = sb.compute_setup(case["pp"])
    tab, _ = sb.sample(case["pp"], s)
    fields = [_run(v, s, case["fs"], case["n"], case["ds"], tab) for v in VARIANTS]
    for f in fields:
        assert np.all(np.isfinite(f))
        assert np.array_equal(f.view(np.uint32), fields[0].view(np.uint32))
    ref64 = oracle.sum_structured(oracle.setup(case["op"]), case["fs"], case["n"], case["ds"], tab, f64=True)
    assert rel_rms(fields[0], ref64) <= 1e-5


@pytest.mark.parametrize("n,nharm", [
    ([150, 130, 290], 700),   # ragged row blocks (odd count along j) and two column tiles
    ([40, 7, 520], 333),      # two row blocks along j (one pair); three column tiles
    ([330, 4, 200], 500),     # one row block along j: pairs split along i (odd count)
    ([16, 16, 16], 100),      # smaller than one pair tile
])
def test_variants_bit_identical_on_ragged_grids(n, nharm):
    kw = dict(acf=0, nharm=nharm, seed=77, hurst=0.3, sigma=0.05, ds=40.0, cl=[1500.0, 1500.0, 1500.0])
    fc = [float(np.float32(v - 1) * np.float32(40.0)) for v in n]
    p = sb.make_params(nc=[0.0, 0.0, 0.0], fc=fc, **kw)
    s = sb.compute_setup(p)
    tab, _ = sb.sample(p, s)
    fields = [_run(v, s, [1, 1, 1], n, 40.0, tab) for v in VARIANTS]
    for f in fields:
        assert np.all(np.isfinite(f))
        assert np.array_equal(f.view(np.uint32), fields[0].view(np.uint32))


def test_pair_form_batch_matches_single_form():
    shapes = [(48, 32, 64), (80, 16, 32), (17, 23, 40), (64, 64, 256), (40, 8, 300), (33, 40, 31)]
    entries, fields = [], []
    for f, n in enumerate(shapes):
        cl = [float(min(2000.0, max(300.0, (m - 1) * 50.0 / 3.5))) for m in n]
        kw = dict(acf=f % 2, nharm=150 + 41 * f, seed=900 + f, hurst=0.3 if f % 2 == 0 else 0.0, sigma=0.05,
                  ds=50.0, cl=cl)
        op = oracle.structured_params(fs=[1, 1, 1], fe=list(n), **kw)
        p = sb.make_params(nc=list(op.nc), fc=list(op.fc), **kw)
        s = sb.compute_setup(p)
        tab, _ = sb.sample(p, s)
        d_tab = torch.from_numpy(tab.reshape(-1).copy()).cuda()
        out = torch.full((int(np.prod(n)),), float("nan"), dtype=torch.float32, device="cuda")
        fields.append(dict(n=list(n), s=s, tab=tab, out=out, d_tab=d_tab))
        entries.append(dict(setup=s, fs=[1, 1, 1], n=list(n), ds=50.0, d_table=d_tab.data_ptr(), nh=len(tab),
                            d_field=out.data_ptr()))
    sb.set_tc_variant(sb.TC_PAIR)
    batch = sb.TcBatch(entries, lambda nb: torch.empty(nb, dtype=torch.uint8, device="cuda"))
    batch.launch()
    batch.wait()
    for f in fields:
        got = f["out"].cpu().numpy()
        ref = _run(sb.TC_SINGLE, f["s"], [1, 1, 1], f["n"], 50.0, f["tab"])
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_unknown_variant_is_rejected():
    with pytest.raises(sb.ScarfError):
        sb.set_tc_variant(7)


@pytest.mark.parametrize("n", [[64, 200, 40], [96, 130, 33], [40, 257, 100], [257, 40, 64], [300, 96, 17]])
def test_long_axis_grids_take_it_as_the_column_axis(n):
    # The device-field entry point lets the longest axis be the column
    # axis: the field must still agree with the FP64 oracle in the caller's
    # x-fastest layout, for every kernel form.
    kw = dict(acf=0, nharm=600, seed=31, hurst=0.3, sigma=0.05, ds=40.0, cl=[1500.0, 1500.0, 1500.0])
    fc = [float(np.float32(v - 1) * np.float32(40.0)) for v in n]
    p = sb.make_params(nc=[0.0, 0.0, 0.0], fc=fc, **kw)
    s = sb.compute_setup(p)
    tab, _ = sb.sample(p, s)
    fields = [_run(v, s, [1, 1, 1], n, 40.0, tab) for v in VARIANTS]
    for f in fields:
        assert np.array_equal(f.view(np.uint32), fields[0].view(np.uint32))
    op = oracle.params(acf=0, nharm=600, seed=31, hurst=0.3, sigma=0.05, ds=40.0, dh=40.0, cl=[1500.0] * 3,
                       nc=[0.0] * 3, fc=fc)
    ref64 = oracle.sum_structured(oracle.setup(op), [1, 1, 1], n, 40.0, tab, f64=True)
    assert rel_rms(fields[0], ref64) <= 1e-5


@pytest.mark.parametrize("nharm", [1, 15, 17])
@pytest.mark.parametrize("fs,n", [
    ([1, 1, 1], [1, 1, 1]),        # a single point
    ([20, 5, 33], [1, 9, 1]),      # one line along y inside a larger domain
    ([3, 40, 7], [33, 1, 1]),      # one line along x (x becomes the column axis)
    ([9, 9, 1], [1, 1, 300]),      # one line along z, two column tiles
    ([2, 60, 61], [2, 3, 5]),      # a corner block smaller than one row tile
])
def test_degenerate_blocks_and_tiny_harmonic_counts(fs, n, nharm):
    # Blocks of one point or one line of a 64 x 64 x 320 domain (a rank's sub-block),
    # with harmonic counts below, at and just above one 16-harmonic stage:
    # every kernel form agrees bit for bit and with the FP64 oracle.
    kw = dict(acf=0, nharm=nharm, seed=5, hurst=0.4, sigma=0.05, ds=50.0, cl=[800.0, 800.0, 800.0])
    fc = [float(np.float32(m - 1) * np.float32(50.0)) for m in (64, 64, 320)]
    p = sb.make_params(nc=[0.0, 0.0, 0.0], fc=fc, **kw)
    s = sb.compute_setup(p)
    tab, _ = sb.sample(p, s)
    fields = [_run(v, s, fs, n, 50.0, tab) for v in VARIANTS]
    for f in fields:
        assert np.all(np.isfinite(f))
        assert np.array_equal(f.view(np.uint32), fields[0].view(np.uint32))
    op = oracle.params(acf=0, nharm=nharm, seed=5, hurst=0.4, sigma=0.05, ds=50.0, dh=50.0, cl=[800.0] * 3,
                       nc=[0.0] * 3, fc=fc)
    ref64 = oracle.sum_structured(oracle.setup(op), fs, n, 50.0, tab, f64=True)
    # absolute bound: 1e-4 of sigma (the bench's 512^3 field sees ~1e-5)
    assert float(np.max(np.abs(fields[0].astype(np.float64) - ref64))) <= 1e-4 * 0.05


@pytest.mark.parametrize("variant", VARIANTS)
def test_operand_precision_settings_against_fp64(variant):
    """Both 3-product splits meet 1e-5 against FP64 (BF16, the default, keeps
    fewer bits than FP16 and comes out a little worse); dropping the hi.lo
    product loses the B correction and misses it (measured, not assumed)."""
    case = structured_case("vk3d_rot_offset", nharm=1500)
    s = sb.compute_setup(case["pp"])
    tab, _ = sb.sample(case["pp"], s)
    ref64 = oracle.sum_structured(oracle.setup(case["op"]), case["fs"], case["n"], case["ds"], tab, f64=True)
    err = {}
    try:
        for otype, terms in ((sb.TC_FP16, 3), (sb.TC_BF16, 3), (sb.TC_FP16, 2), (sb.TC_BF16, 2)):
            sb.set_tc_precision(otype, terms)
            f = _run(variant, s, case["fs"], case["n"], case["ds"], tab)
            assert np.all(np.isfinite(f))
            err[(otype, terms)] = rel_rms(f, ref64)
    finally:
        sb.set_tc_precision()
    assert err[(sb.TC_FP16, 3)] <= 1e-5
    assert err[(sb.TC_BF16, 3)] <= 1e-5
    assert err[(sb.TC_BF16, 3)] > err[(sb.TC_FP16, 3)]
    assert err[(sb.TC_FP16, 2)] > 1e-5
    assert err[(sb.TC_BF16, 2)] > err[(sb.TC_FP16, 2)]


@pytest.mark.parametrize("variant", [sb.TC_SINGLE, sb.TC_SINGLE_TMEM_A])
@pytest.mark.parametrize("split", [2, 3, 8])
def test_harmonic_split_matches_unsplit_and_fp64(variant, split, monkeypatch):
    """Splitting the harmonics over several work items per tile (partial sums
    reduced in segment order after the kernel) gives the unsplit sum up to
    FP32 rounding, the FP64 oracle within the tensor-core tolerance, and the
    same bits on every run."""
    case = structured_case("gs3d_aniso", nharm=900)
    s = sb.compute_setup(case["pp"])
    tab, _ = sb.sample(case["pp"], s)
    base = _run(variant, s, case["fs"], case["n"], case["ds"], tab)
    monkeypatch.setenv("SCARF3D_B200_TC_SPLIT", str(split))
    assert sb.tc_plan_info(3, case["n"], len(tab))["split"] == split
    a = _run(variant, s, case["fs"], case["n"], case["ds"], tab)
    b = _run(variant, s, case["fs"], case["n"], case["ds"], tab)
    assert np.all(np.isfinite(a))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert rel_rms(a, base) <= 1e-5  # two tensor-core sums, each within ~4e-6 of FP64
    ref64 = oracle.sum_structured(oracle.setup(case["op"]), case["fs"], case["n"], case["ds"], tab, f64=True)
    assert rel_rms(a, ref64) <= 1e-5


def test_autotuner_offers_splits_for_small_grids():
    """A grid with fewer tiles than SMs gets split candidates; whatever the
    tuner records is followed by the device-field entry point and agrees with
    the FP64 oracle."""
    case = structured_case("gs3d_aniso", nharm=2000)
    s = sb.compute_setup(case["pp"])
    tab, _ = sb.sample(case["pp"], s)
    d_tab = torch.from_numpy(np.ascontiguousarray(tab.reshape(-1))).cuda()
    try:
        t = sb.tc_autotune(s, case["fs"], case["n"], case["ds"], d_tab.data_ptr(), len(tab))
        sb.set_tc_autotune(1)
        info = sb.tc_plan_info(3, case["n"], len(tab))
        assert info["split"] == t["split"] >= 1
        sb.set_tc_variant(t["variant"])
        f = _run(t["variant"], s, case["fs"], case["n"], case["ds"], tab)
    finally:
        sb.set_tc_autotune(0)
    ref64 = oracle.sum_structured(oracle.setup(case["op"]), case["fs"], case["n"], case["ds"], tab, f64=True)
    assert rel_rms(f, ref64) <= 1e-5
