"""The FIM restatement on the CPU (oracle/fim.py, oracle/fim_oracle.c):
internal-grid arithmetic, the draw-to-point mapping of the block-split
uniform stream, the Hermitian planes and the properties of the field."""
import math

import numpy as np

import oracle
from oracle import fim


def test_internal_grid_known_answers():
    # 40 x 32 x 24 points at 50 m, no padding: span (n - 1) ds + dh -> n + 1
    # points, rounded up to even; the first node half a step before nc.
    npts, off, info = fim.grid(3, [0, 0, 0], [1950.0, 1550.0, 1150.0], 50.0, [500.0, 500.0, 500.0], 0)
    assert npts == [42, 34, 26]
    assert np.allclose(off, [-25.0, -25.0, -25.0])
    assert info[0] == 1.0  # 42 <= NINT(2 pi 500 / 50) = 63: domain too small
    assert info[1] == 0.0
    # padding adds NINT(cl / dh) nodes on each side
    npts, off, _ = fim.grid(3, [0, 0, 0], [1950.0, 1550.0, 1150.0], 50.0, [400.0, 300.0, 200.0], 1)
    assert npts == [58, 46, 34]
    assert np.allclose(off, [-425.0, -325.0, -225.0])
    # 2-D: one z node, its offset negated
    npts, off, _ = fim.grid(2, [0, 0, 0], [4750.0, 3450.0, 0.0], 50.0, [800.0, 500.0], 0)
    assert npts[2] == 1 and off[2] == 25.0


def test_phases_are_the_stream_in_x_fastest_order():
    npts = [8, 6, 4]
    spec = fim.spectrum(npts, 3, 50.0, 50.0, 1, [100.0, 100.0, 100.0], 1.0, 0.0, 1234)
    raw = oracle.raw_stream(1234, int(np.prod(npts)))
    u = np.array([oracle.L.orc_u01(int(v)) for v in raw], np.float32).reshape(4, 6, 8)
    # away from the Hermitian planes (i = 0, n1/2) every phase is 2 pi u
    for (k, j, i) in [(0, 1, 1), (2, 3, 2), (3, 5, 3), (1, 0, 1)]:
        h = np.float32(np.float32(u[k, j, i] * np.float32(2.0)) * np.float32(math.pi))
        c = spec[k, j, i]
        amp = abs(c)
        assert amp > 0
        assert abs(c.real - np.cos(h) * amp) <= 1e-6 * amp and abs(c.imag - np.sin(h) * amp) <= 1e-6 * amp


def test_hermitian_planes():
    npts = [10, 8, 6]
    spec = fim.spectrum(npts, 3, 50.0, 50.0, 0, [200.0, 200.0, 200.0], 0.05, 0.3, 5)
    n1, n2, n3 = npts
    for i in (0, n1 // 2):
        p = spec[:, :, i]
        assert p[0, 0].imag == 0.0
        for k in range(n3):
            for j in range(n2):
                if k > n3 // 2 or (k == n3 // 2 and j > n2 // 2):
                    assert p[k, j] == np.conj(p[(n3 - k) % n3, (n2 - j) % n2])
                if k == 0 and j > n2 // 2:
                    # the reference's unmirrored row (conjugated in place)
                    assert p[0, j] != np.conj(p[0, n2 - j])
    assert spec[0, 0, 0] == 0


def test_field_properties():
    f, info, det = fim.execute_structured(fs=[1, 1, 1], fe=[64, 64, 64], ds=50.0, acf=0, cl=[400.0] * 3,
                                          sigma=0.05, hurst=0.5, seed=1235, pad=1)
    internal = det["internal"]
    assert abs(float(info[3])) < 1e-6  # zero-mean: the DC term is removed
    assert 0.03 < float(info[2]) < 0.07  # std near sigma
    assert np.count_nonzero(f) == f.size
    # every external value is an internal node value
    assert np.isin(f, internal).all()
    f2, _, _ = fim.execute_structured(fs=[1, 1, 1], fe=[64, 64, 64], ds=50.0, acf=0, cl=[400.0] * 3, sigma=0.05,
                                      hurst=0.5, seed=1235, pad=1, rescale=1)
    assert abs(float(np.std(f2.astype(np.float64))) - 0.05) < 0.01


def test_library_internal_grid_equals_the_oracle():
    """The library's FIM grid (host code of the product) and the oracle's
    restatement agree bit for bit over random domains, steps and lengths."""
    import scarf3d_b200 as sb
    rng = np.random.default_rng(17)
    for _ in range(400):
        ndim = int(rng.integers(2, 4))
        nc = (rng.uniform(-5000.0, 5000.0, 3)).astype(np.float32)
        fc = (nc + rng.uniform(10.0, 30000.0, 3)).astype(np.float32)
        if ndim == 2:
            nc[2] = fc[2] = 0.0
        dh = np.float32(rng.uniform(5.0, 200.0))
        cl = rng.uniform(50.0, 5000.0, ndim).astype(np.float32)
        pad = int(rng.integers(0, 2))
        a = sb.fim_internal_grid(ndim, nc, fc, dh, cl, pad)
        b = fim.grid(ndim, nc, fc, dh, cl, pad)
        assert a[0] == b[0]
        assert np.array_equal(np.asarray(a[1]).view(np.uint32), np.asarray(b[1]).view(np.uint32))
        assert np.array_equal(a[2], b[2])
    assert sb.lib.scarf_fim_workspace_bytes(np.asarray([64, 64, 64], np.int32).ctypes.data, 2) > 64 * 64 * 33 * 8
