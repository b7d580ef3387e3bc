"""Autotuning of the tensor-core form: a tuning times the candidate plans on
the caller's grid and table and records the fastest for the grid's shape
bucket; with tuned plans enabled the entry points follow it (and only for
that bucket), the recorded choice survives in the cache file for a new
process, and every tuned plan still computes the field within the
tensor-core tolerance of the FP64 oracle."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
import scarf3d_b200 as sb
from conftest import rel_rms

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
KW = dict(acf=0, seed=41, hurst=0.3, sigma=0.05, ds=40.0, cl=[1500.0, 1500.0, 1500.0])


@pytest.fixture(autouse=True)
def _reset():
    yield
    sb.set_tc_autotune(0)
    sb.set_tc_tune_cache(None)
    sb.set_tc_variant(sb.TC_SINGLE)


def _case(n, nharm=600):
    fc = [float(np.float32(v - 1) * np.float32(40.0)) for v in n]
    p = sb.make_params(nc=[0.0, 0.0, 0.0], fc=fc, nharm=nharm, **KW)
    s = sb.compute_setup(p)
    tab, _ = sb.sample(p, s)
    op = oracle.params(nharm=nharm, dh=40.0, nc=[0.0] * 3, fc=fc, **KW)
    return s, tab, op


def _tc(s, n, tab):
    return _tc_nd(s, n, tab, 3)


def _tc_nd(s, n, tab, ndim):
    d_tab = torch.from_numpy(np.ascontiguousarray(tab.reshape(-1))).cuda()
    out = torch.full((int(np.prod(n)),), float("nan"), dtype=torch.float32, device="cuda")
    wb = sb.tc_workspace_bytes(ndim, n, len(tab))
    work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    import ctypes
    from srm_cases import iarr
    sb.check(sb.lib.scarf_srm_tc_structured(ctypes.byref(s), iarr([1, 1, 1]), iarr(n), 40.0,
                                            ctypes.c_void_p(d_tab.data_ptr()), len(tab),
                                            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(work.data_ptr()),
                                            wb, None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_tuning_is_recorded_and_followed(tmp_path):
    n = [72, 48, 200]
    s, tab, op = _case(n)
    cache = tmp_path / "tune.txt"
    sb.set_tc_tune_cache(cache)
    d_tab = torch.from_numpy(np.ascontiguousarray(tab.reshape(-1))).cuda()
    t = sb.tc_autotune(s, [1, 1, 1], n, 40.0, d_tab.data_ptr(), len(tab))
    assert t["variant"] in (sb.TC_SINGLE, sb.TC_PAIR, sb.TC_SINGLE_TMEM_A)
    assert t["tile_j"] in (1, 2, 4, 8, 16) and t["ms"] > 0.0
    default = sb.tc_plan_info(3, n, len(tab))
    other_default = sb.tc_plan_info(3, [200, 48, 72], len(tab))
    sb.set_tc_autotune(1)
    tuned = sb.tc_plan_info(3, n, len(tab))
    assert (tuned["variant"], tuned["tile_j"], tuned["permute"]) == (t["variant"], t["tile_j"], t["permute"])
    # another bucket keeps the default plan
    assert sb.tc_plan_info(3, [200, 48, 72], len(tab)) == other_default
    field = _tc(s, n, tab)
    ref64 = oracle.sum_structured(oracle.setup(op), [1, 1, 1], n, 40.0, tab, f64=True)
    assert rel_rms(field, ref64) <= 1e-5
    sb.set_tc_autotune(0)
    assert sb.tc_plan_info(3, n, len(tab)) == default
    assert cache.read_text().strip().count("\n") == 0  # one entry written


def test_every_candidate_plan_computes_the_field():
    # The tuner may pick any (form, row tile, column axis): each must agree
    # with the FP64 oracle. Entries are forced through the cache file.
    n = [96, 24, 40]  # x longest: permuting plans take it as the column axis
    s, tab, op = _case(n, nharm=300)
    ref64 = oracle.sum_structured(oracle.setup(op), [1, 1, 1], n, 40.0, tab, f64=True)
    d_tab = torch.from_numpy(np.ascontiguousarray(tab.reshape(-1))).cuda()
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        cache = Path(d) / "t.txt"
        sb.set_tc_tune_cache(cache)
        sb.tc_autotune(s, [1, 1, 1], n, 40.0, d_tab.data_ptr(), len(tab))
        key = cache.read_text().split()[0]
        fields = []
        for variant in (sb.TC_SINGLE, sb.TC_PAIR, sb.TC_SINGLE_TMEM_A):
            for tj in (1, 2, 4, 8, 16):
                for perm in (0, 1):
                    cache.write_text(f"{key} {variant} {tj} {perm} 1.0\n")
                    sb.set_tc_tune_cache(cache)
                    sb.set_tc_autotune(1)
                    info = sb.tc_plan_info(3, n, len(tab))
                    assert (info["variant"], info["tile_j"]) == (variant, tj)
                    f = _tc(s, n, tab)
                    assert np.all(np.isfinite(f))
                    assert rel_rms(f, ref64) <= 1e-5, (variant, tj, perm)
                    fields.append(((variant, tj, info["permute"]), f))
        # the same column axis gives the same bits whatever the form and row tile
        for perm in (0, 1):
            same = [f for (v, tj, p), f in fields if p == perm]
            for f in same[1:]:
                assert np.array_equal(f.view(np.uint32), same[0].view(np.uint32))


def test_cache_file_serves_a_new_process(tmp_path):
    n = [64, 40, 128]
    s, tab, _ = _case(n, nharm=200)
    cache = tmp_path / "tune.txt"
    sb.set_tc_tune_cache(cache)
    d_tab = torch.from_numpy(np.ascontiguousarray(tab.reshape(-1))).cuda()
    t = sb.tc_autotune(s, [1, 1, 1], n, 40.0, d_tab.data_ptr(), len(tab))
    code = (
        "import sys; sys.path.insert(0, %r); import scarf3d_b200 as sb; "
        "sb.set_tc_tune_cache(%r); sb.set_tc_autotune(1); print(sb.tc_plan_info(3, %r, %d))"
        % (str(ROOT), str(cache), n, len(tab)))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout
    info = eval(out.strip().splitlines()[-1])
    assert (info["variant"], info["tile_j"], info["permute"]) == (t["variant"], t["tile_j"], t["permute"])


def test_execute_follows_a_fixed_column_tuning():
    fs, fe = [1, 1, 1], [48, 40, 64]
    n = [fe[c] - fs[c] + 1 for c in range(3)]
    s, tab, op = _case(n, nharm=400)
    d_tab = torch.from_numpy(np.ascontiguousarray(tab.reshape(-1))).cuda()
    t = sb.tc_autotune(s, fs, n, 40.0, d_tab.data_ptr(), len(tab), fixed_columns=True)
    assert t["permute"] == 0
    sb.set_tc_autotune(1)
    sb.set_nharm(400)
    try:
        sb.scarf_initialize(fs=fs, fe=fe, ds=40.0, acf=0, cl=KW["cl"], sigma=0.05, method=1, hurst=0.3,
                            nc=[0.0] * 3, fc=[float(np.float32(v - 1) * np.float32(40.0)) for v in n])
        field, _ = sb.scarf_execute(41)
    finally:
        sb.scarf_finalize()
        sb.set_nharm(10000)
    ref64 = oracle.sum_structured(oracle.setup(op), fs, n, 40.0, tab, f64=True)
    assert rel_rms(field, ref64) <= 1e-5


def test_batch_tuning_returns_a_plan_that_runs():
    shapes = [(48, 32, 64), (80, 16, 32), (32, 40, 48), (64, 64, 128)]
    entries, outs, keep = [], [], []
    for f, n in enumerate(shapes):
        s, tab, _ = _case(list(n), nharm=150 + 50 * f)
        d = torch.from_numpy(np.ascontiguousarray(tab.reshape(-1))).cuda()
        o = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
        keep += [d]
        outs.append(o)
        entries.append(dict(setup=s, fs=[1, 1, 1], n=list(n), ds=40.0, d_table=d.data_ptr(), nh=len(tab),
                            d_field=o.data_ptr()))
    alloc = lambda nb: torch.empty(nb, dtype=torch.uint8, device="cuda")  # noqa: E731
    b = sb.TcBatch(entries, alloc)
    b.launch()
    b.wait()
    ref = [o.cpu().numpy().copy() for o in outs]
    t = sb.tc_batch_autotune(entries)
    assert t["variant"] in (sb.TC_SINGLE, sb.TC_PAIR) and t["tile_j"] in (1, 2, 4, 8, 16) and t["ms"] > 0
    sb.set_tc_variant(t["variant"])
    for e in entries:
        e["tile_j"] = t["tile_j"]
    for o in outs:
        o.fill_(float("nan"))
    b2 = sb.TcBatch(entries, alloc)
    b2.launch()
    b2.wait()
    for o, r in zip(outs, ref):
        assert np.array_equal(o.cpu().numpy().view(np.uint32), r.view(np.uint32))


def test_two_dimensional_grid_tuning():
    # 2-D grids: the single z plane is the row-slow axis, so row tiles with
    # tile_j > 1 waste rows; the tuner must offer tile_j = 1 (the default).
    n = [300, 200, 1]
    fc = [float(np.float32(v - 1) * np.float32(40.0)) for v in n[:2]] + [0.0]
    kw = dict(KW, cl=[1500.0, 1500.0, 0.0])
    p = sb.make_params(nc=[0.0, 0.0, 0.0], fc=fc, nharm=300, **kw)
    s = sb.compute_setup(p)
    tab, _ = sb.sample(p, s)
    d_tab = torch.from_numpy(np.ascontiguousarray(tab.reshape(-1))).cuda()
    default = sb.tc_plan_info(2, n, len(tab))
    assert default["tile_j"] == 1
    t = sb.tc_autotune(s, [1, 1, 1], n, 40.0, d_tab.data_ptr(), len(tab))
    sb.set_tc_autotune(1)
    field = _tc_nd(s, n, tab, 2)
    op = oracle.params(nharm=300, dh=40.0, nc=[0.0] * 3, fc=fc, **kw)
    ref64 = oracle.sum_structured(oracle.setup(op), [1, 1, 1], n, 40.0, tab, f64=True)
    assert rel_rms(field, ref64) <= 1e-5
    assert t["tile_j"] in (1, 2, 4, 8, 16)
