"""The FIM path (method 0, the reference's default) through scarf_execute on
the GPU, against the CPU restatement (oracle/fim.py): internal grid flags,
statistics of the internal grid, and every external point, for structured
grids (3-D and 2-D, padded or not, filtered when ds != dh, rescaled and
tapered) and point sets. The transform differs only in rounding (cuFFT
single precision against numpy double precision), so fields agree to
~1e-7 of their standard deviation; the tolerance is 1e-5."""
import numpy as np
import pytest

import scarf3d_b200 as sb
from conftest import rel_rms
from oracle import fim
from srm_cases import random_points

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(autouse=True)
def _reset():
    yield
    sb.scarf_finalize()


STRUCTURED = [
    # fs, fe, ds, dh, acf, cl, sigma, hurst, seed, pad, rescale, poi/mute/taper
    dict(fs=[1, 1, 1], fe=[40, 32, 24], ds=50.0, dh=None, acf=0, cl=[500.0, 500.0, 500.0], sigma=0.05, hurst=0.25,
         seed=1235, pad=0),
    dict(fs=[1, 1, 1], fe=[48, 40, 36], ds=50.0, dh=None, acf=1, cl=[400.0, 300.0, 200.0], sigma=0.1, hurst=0.0,
         seed=7, pad=1),
    dict(fs=[3, 2, 5], fe=[40, 30, 28], ds=25.0, dh=50.0, acf=0, cl=[600.0, 600.0, 300.0], sigma=0.05, hurst=0.5,
         seed=99, pad=1),
    dict(fs=[1, 1], fe=[96, 70], ds=50.0, dh=None, acf=0, cl=[800.0, 500.0], sigma=0.05, hurst=0.3, seed=3, pad=0),
    dict(fs=[1, 1], fe=[64, 64], ds=50.0, dh=None, acf=1, cl=[600.0, 600.0], sigma=0.05, hurst=0.0, seed=-7, pad=1),
    dict(fs=[1, 1, 1], fe=[40, 36, 30], ds=50.0, dh=None, acf=0, cl=[500.0, 500.0, 400.0], sigma=0.05, hurst=0.25,
         seed=11, pad=0, rescale=1, poi=[[700.0, 600.0, 500.0], [1500.0, 900.0, 1100.0]], mute=200.0, taper=400.0),
]


def _execute_structured(c):
    kw = dict(fs=c["fs"], fe=c["fe"], ds=c["ds"], acf=c["acf"], cl=c["cl"], sigma=c["sigma"], method=0,
              hurst=c["hurst"], pad=c.get("pad", 0), rescale=c.get("rescale", 0))
    if c.get("dh"):
        kw["dh"] = c["dh"]
    if c.get("poi") is not None:
        kw.update(poi=np.asarray(c["poi"], np.float32), mute=c["mute"], taper=c["taper"])
    sb.scarf_initialize(**kw)
    n = [e - s + 1 for s, e in zip(c["fs"], c["fe"])]
    dev = torch.full((int(np.prod(n)),), float("nan"), dtype=torch.float32, device="cuda")
    _, stats = sb.scarf_execute(c["seed"], dev)
    host, stats_h = sb.scarf_execute(c["seed"])
    sb.scarf_finalize()
    return dev.cpu().numpy(), stats, np.asarray(host), stats_h


@pytest.mark.parametrize("case", range(len(STRUCTURED)))
def test_fim_structured_matches_oracle(case):
    c = STRUCTURED[case]
    got, stats, host, stats_h = _execute_structured(c)
    ref, info, det = fim.execute_structured(fs=c["fs"], fe=c["fe"], ds=c["ds"], dh=c.get("dh"), acf=c["acf"],
                                            cl=c["cl"], sigma=c["sigma"], hurst=c["hurst"], seed=c["seed"],
                                            pad=c.get("pad", 0), rescale=c.get("rescale", 0), poi=c.get("poi"),
                                            mute=c.get("mute", -999.0), taper=c.get("taper", -999.0))
    assert np.all(np.isfinite(got))
    assert np.array_equal(host.view(np.uint32), got.view(np.uint32))  # host and device output alike
    assert rel_rms(got, ref) <= TOL, rel_rms(got, ref)
    assert stats[0] == info[0] and stats[1] == info[1]
    assert abs(stats[2] / info[2] - 1) <= 10 * TOL
    assert abs(stats[3] - info[3]) <= 10 * TOL * info[2]
    assert stats[4] > 0 and stats[6] > 0  # spectrum and transform times
    assert np.array_equal(stats[:4], stats_h[:4])
    if c.get("poi") is not None:
        assert np.array_equal(got == 0.0, ref == 0.0)  # the same muted points


def test_fim_points_3d_and_2d():
    x, y, z = random_points(6000, box=(3000.0, 2500.0, 1500.0), seed=5)
    for cl, zz in (([500.0, 500.0, 300.0], z), ([600.0, 400.0], None)):
        kw = dict(x=x, y=y, dh=50.0, acf=0, cl=cl, sigma=0.05, method=0, hurst=0.3, pad=1)
        if zz is not None:
            kw["z"] = zz
        sb.scarf_initialize(**kw)
        got, stats = sb.scarf_execute(21)
        sb.scarf_finalize()
        ref, info, _ = fim.execute_points(x=x, y=y, z=zz, dh=50.0, acf=0, cl=cl, sigma=0.05, hurst=0.3, seed=21,
                                          pad=1)
        assert rel_rms(got, ref) <= TOL, rel_rms(got, ref)
        assert stats[0] == info[0] and stats[1] == info[1]
        assert abs(stats[2] / info[2] - 1) <= 10 * TOL


def test_fim_is_deterministic_and_seeded():
    c = STRUCTURED[0]
    a, _, _, _ = _execute_structured(c)
    b, _, _, _ = _execute_structured(c)
    d, _, _, _ = _execute_structured(dict(c, seed=c["seed"] + 1))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert rel_rms(a, d) > 0.5


def test_cached_transform_plans_follow_the_grid():
    """The cuFFT plans kept from one call to the next are rebuilt when the
    internal grid changes and after scarf_release_device_memory: grids run in
    turn (A, B, A, release, A) give A's field bit for bit every time."""
    a, b = STRUCTURED[0], STRUCTURED[1]
    ref, st_ref, _, _ = _execute_structured(a)
    other, _, _, _ = _execute_structured(b)
    assert other.size != ref.size
    again, st_again, _, _ = _execute_structured(a)
    assert np.array_equal(again.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(st_again[:4], st_ref[:4])
    sb.check(sb.lib.scarf_release_device_memory())
    after, _, _, _ = _execute_structured(a)
    assert np.array_equal(after.view(np.uint32), ref.view(np.uint32))
