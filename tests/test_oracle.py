"""CPU oracle: golden fixtures, closed-form known answers and the reference's
invariants (no GPU). The oracle is parity-unpinned (the reference cannot be
built here), so these checks are what anchors it."""
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
from conftest import rel_rms

GOLDEN = Path(__file__).resolve().parent / "golden"


def _load_cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


MG = _load_cases()


@pytest.mark.parametrize("name", sorted(MG.CASES))
def test_oracle_reproduces_golden_fixture(name):
    ref = np.load(GOLDEN / f"{name}.npz")
    got = MG.build_case(MG.CASES[name])
    for key in ("setup", "ier", "table", "pairs", "field_f32", "execute_field", "execute_info", "n"):
        assert np.array_equal(np.asarray(got[key]).view(np.uint8), ref[key].view(np.uint8)), key
    np.testing.assert_allclose(got["field_f64"], ref["field_f64"], rtol=1e-12, atol=1e-15)


def test_uniform_stream_golden():
    ref = np.load(GOLDEN / "uniform_stream.npz")
    assert np.array_equal(oracle.raw_stream(1235, 64), ref["seed1235"])
    assert np.array_equal(oracle.raw_stream(-7, 64), ref["seed_neg7"])


def test_uniform_stream_is_unit_interval_and_uniform():
    raw = oracle.raw_stream(42, 20000)
    assert raw.max() < 2 ** 31 - 1
    u = np.array([oracle.L.orc_u01(int(y)) for y in raw[:5000]], np.float32)
    assert u.min() >= 0.0 and u.max() <= 1.0
    assert abs(u.mean() - 0.5) < 0.02 and abs(u.std() - math.sqrt(1 / 12)) < 0.01


def test_uniform_draw_is_a_double_draw_rounded_to_float():
    """uniform01_dist<> draws a double y/m in [0,1) (default result type) and
    srng stores it into a float (prng.cpp:152-165): the float is the double
    y * (1/m) rounded to nearest, so it can be 0 and can round up to 1."""
    m = 2 ** 31 - 1
    ys = [0, 1, 2, 255, 256, 1 << 20, m // 2, m - 65, m - 64, m - 2, m - 1]
    ys += [int(y) for y in oracle.raw_stream(5, 4000)]
    for y in ys:
        assert oracle.L.orc_u01(y) == np.float32(np.float64(y) * (1.0 / m))
    assert oracle.L.orc_u01(0) == 0.0
    assert oracle.L.orc_u01(m - 1) == 1.0


def test_negative_seed_is_reduced_as_a_signed_integer():
    """prng.cpp:147 turns the int seed into unsigned long; yarn2's seeding
    reads it back as a signed 64-bit value and reduces it into [0, m): seed -7
    starts from the state (m - 7, 1)."""
    m = 2 ** 31 - 1
    a1, a2, g = 1498809829, 1160990996, 123567893
    r0, r1 = m - 7, 1
    want = []
    for _ in range(8):
        r0, r1 = (a1 * r0 + a2 * r1) % m, r0
        want.append(0 if r0 == 0 else pow(g, r0, m))
    assert list(oracle.raw_stream(-7, 8)) == want


# ---------------------------------------------------------------- quadrature --
def _beta(a, b):
    return math.gamma(a) * math.gamma(b) / math.gamma(a + b)


@pytest.mark.parametrize("hurst", [0.1, 0.25, 0.5, 0.8])
def test_dqagi_vk3d_closed_form(hurst):
    nu = np.float32(hurst + 1.5)
    r, _, ier = oracle.dqagi(3, 0, float(nu))
    exact = 0.5 * _beta(1.5, float(nu) - 1.5)
    assert ier == 0
    assert abs(r / exact - 1) < 3e-5


@pytest.mark.parametrize("hurst", [0.1, 0.5, 0.9])
def test_dqagi_vk2d_closed_form(hurst):
    nu = np.float32(hurst + 1.0)
    r, _, ier = oracle.dqagi(2, 0, float(nu))
    exact = 1.0 / (2.0 * (float(nu) - 1.0))
    assert abs(r / exact - 1) < 3e-5


def test_dqagi_gaussian_closed_forms():
    r3, _, _ = oracle.dqagi(3, 1, 1.5)
    r2, _, _ = oracle.dqagi(2, 1, 1.0)
    assert abs(r3 / (2 * math.sqrt(math.pi)) - 1) < 1e-5
    assert abs(r2 / 2.0 - 1) < 1e-5


@pytest.mark.parametrize("a,b", [(1.5, 125.0), (2.0, 40.0), (0.3, 5.0)])
def test_dqng_band_closed_forms(a, b):
    # VK 3D with nu = 2 (Hurst 0.5): F(k) = (atan k - k/(1+k^2))/2.
    r, _, _ = oracle.dqng(3, 0, 2.0, a, b)
    F = lambda k: 0.5 * (math.atan(k) - k / (1 + k * k))  # noqa: E731
    assert abs(r / (F(b) - F(a)) - 1) < 2e-5
    # Gaussian 2D: 2 (exp(-a^2/4) - exp(-b^2/4)).
    r, _, _ = oracle.dqng(2, 1, 1.0, a, b)
    assert abs(r / (2 * (math.exp(-a * a / 4) - math.exp(-b * b / 4))) - 1) < 2e-5


# --------------------------------------------------------- setup and sampler --
def test_rotation_is_orthonormal_and_bar_is_rotated_half_span():
    p = oracle.structured_params(acf=0, nharm=10, seed=1, hurst=0.5, sigma=0.05, ds=50.0, cl=[2000.0] * 3,
                                 fs=[1, 1, 1], fe=[64, 48, 32], alpha=30.0, beta=-10.0, gamma=25.0)
    s = oracle.setup(p)
    m = np.array(s.m, np.float64).reshape(3, 3)
    np.testing.assert_allclose(m @ m.T, np.eye(3), atol=1e-6)
    half = (np.array(p.fc, np.float64) - np.array(p.nc, np.float64)) / 2
    np.testing.assert_allclose(np.array(s.bar), half - m @ half, rtol=1e-5, atol=1e-3)


def test_sampler_distributions():
    p = oracle.structured_params(acf=0, nharm=20000, seed=11, hurst=0.5, sigma=0.05, ds=25.0,
                                 cl=[3000.0, 3000.0, 1000.0], fs=[1, 1, 1], fe=[256, 256, 256])
    s = oracle.setup(p)
    tab, pairs = oracle.sample(p, s)
    assert len(tab) == 20000  # ds == dh: no harmonic above the corner wavenumber
    a, b = tab[:, 3].astype(np.float64), tab[:, 4].astype(np.float64)
    for x in (a, b):
        assert abs(x.mean()) < 0.03 and abs(x.std() - 1) < 0.03
    k = np.sqrt((tab[:, 0] * 3000.0) ** 2 + (tab[:, 1] * 3000.0) ** 2 + (tab[:, 2] * 1000.0) ** 2)
    assert k.min() >= s.kmin * (1 - 1e-5) and k.max() <= s.kmax * (1 + 1e-5)
    # Acceptance: about (kmax - kmin)/int_{kmin}^{kmax} pairs per harmonic, plus 3 more.
    expect = 20000 * ((s.kmax - s.kmin) / (s.intg_band * s.cnst) + 3)
    assert abs(pairs / expect - 1) < 0.05


def test_corner_wavenumber_drops_harmonics():
    p = oracle.structured_params(acf=0, nharm=2000, seed=5, hurst=0.3, sigma=0.05, ds=50.0, dh=20.0,
                                 cl=[2000.0, 2000.0, 800.0], fs=[1, 1, 1], fe=[32, 32, 32])
    s = oracle.setup(p)
    assert s.kc < s.kmax
    tab, _ = oracle.sample(p, s)
    assert 0 < len(tab) < 2000


# ---------------------------------------------------------------- invariants --
def _grid_case(**over):
    kw = dict(acf=0, nharm=200, seed=21, hurst=0.25, sigma=0.05, ds=50.0, cl=[2000.0, 2000.0, 1000.0],
              alpha=15.0, beta=5.0, gamma=-20.0)
    kw.update(over)
    fs, fe = [3, 2, 1], [26, 19, 14]
    p = oracle.structured_params(fs=fs, fe=fe, **kw)
    s = oracle.setup(p)
    tab, _ = oracle.sample(p, s)
    n = [fe[c] - fs[c] + 1 for c in range(3)]
    return p, s, tab, fs, fe, n, kw


def test_structured_equals_unstructured_on_same_points():
    p, s, tab, fs, fe, n, kw = _grid_case()
    ds = np.float32(kw["ds"])
    i, j, k = np.meshgrid(np.arange(n[0]), np.arange(n[1]), np.arange(n[2]), indexing="ij")
    x = (np.float32(1) * (i.ravel(order="F") + fs[0] - 1).astype(np.float32)) * ds
    y = (j.ravel(order="F") + fs[1] - 1).astype(np.float32) * ds
    z = (k.ravel(order="F") + fs[2] - 1).astype(np.float32) * ds
    a = oracle.sum_structured(s, fs, n, kw["ds"], tab)
    b = oracle.sum_points(s, x, y, z, tab)
    assert np.array_equal(a, b)


def test_slab_decomposition_is_invariant():
    """Ranks with the same seed and global corners reproduce the one-rank
    field on their own blocks (scarflib_srm.f90:627-628, 641-642)."""
    p, s, tab, fs, fe, n, kw = _grid_case()
    full = oracle.sum_structured(s, fs, n, kw["ds"], tab).reshape(n, order="F")
    parts = []
    for z0, z1 in ((1, 6), (7, 14)):
        fs_r, fe_r = [fs[0], fs[1], z0], [fe[0], fe[1], z1]
        n_r = [fe_r[c] - fs_r[c] + 1 for c in range(3)]
        p_r = oracle.structured_params(fs=fs_r, fe=fe_r, nc=list(p.nc), fc=list(p.fc), **kw)
        s_r = oracle.setup(p_r)
        tab_r, _ = oracle.sample(p_r, s_r)
        assert np.array_equal(tab_r, tab)
        parts.append(oracle.sum_structured(s_r, fs_r, n_r, kw["ds"], tab_r).reshape(n_r, order="F"))
    assert np.array_equal(np.concatenate(parts, axis=2), full)


def test_chan_merge_equals_whole_field_statistics():
    p, s, tab, fs, fe, n, kw = _grid_case()
    f = oracle.sum_structured(s, fs, n, kw["ds"], tab).reshape(n, order="F")
    parts = [f[:, :, :5].ravel(order="F"), f[:, :, 5:].ravel(order="F")]
    var = [oracle.variance(q) for q in parts]
    mu = [oracle.mean(q) for q in parts]
    v, m = oracle.parallel_variance(var, mu, [q.size for q in parts])
    whole = f.ravel(order="F")
    assert abs(v / oracle.variance(whole) - 1) < 1e-5
    assert abs(m - oracle.mean(whole)) < 1e-6 * math.sqrt(v)


def test_fp32_restatement_close_to_fp64_oracle():
    p, s, tab, fs, fe, n, kw = _grid_case(nharm=500)
    f32 = oracle.sum_structured(s, fs, n, kw["ds"], tab)
    f64 = oracle.sum_structured(s, fs, n, kw["ds"], tab, f64=True)
    assert rel_rms(f32, f64) < 2e-5


def test_rescale_sets_std_to_sigma_and_taper_mutes():
    kw = dict(acf=0, nharm=200, seed=3, hurst=0.25, sigma=0.05, ds=50.0, cl=[2000.0, 2000.0, 2000.0], rescale=1)
    fs, fe = [1, 1, 1], [24, 20, 16]
    p = oracle.structured_params(fs=fs, fe=fe, **kw)
    field, info = oracle.execute_structured(p, fs, fe)
    assert info[2] == np.float32(0.05) and info[3] == 0.0
    assert abs(oracle.variance(field) ** 0.5 / 0.05 - 1) < 1e-3
    poi = [[500.0, 400.0, 300.0]]
    f2, _ = oracle.execute_structured(p, fs, fe, poi=poi, mute=200.0, taper=300.0)
    n = [24, 20, 16]
    i, j, k = np.meshgrid(*[np.arange(v) for v in n], indexing="ij")
    d = np.sqrt(((i * 50.0 - 500) ** 2 + (j * 50.0 - 400) ** 2 + (k * 50.0 - 300) ** 2)).ravel(order="F")
    assert np.all(f2[d <= 199.0] == 0.0)
    outside = d > 501.0
    assert np.array_equal(f2[outside], field[outside])
    shell = (d > 201.0) & (d < 499.0)
    assert np.all(np.abs(f2[shell]) <= np.abs(field[shell]) + 1e-12)
