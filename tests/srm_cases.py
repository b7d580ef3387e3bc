"""Shared SRM parameter sets and helpers for the tests (parameters mirror the
reference's example drivers, examples/fortran/driver.f90:89-119, at small sizes)."""
from __future__ import annotations

import ctypes

import numpy as np

import oracle
import scarf3d_b200 as sb

# name: (acf, hurst, sigma, ds, dh, cl, fs, fe, angles(alpha,beta,gamma), nharm, seed)
STRUCTURED = {
    "vk3d": (0, 0.25, 0.05, 50.0, None, [2000.0, 2000.0, 2000.0], [1, 1, 1], [17, 13, 11], (0, 0, 0), 300, 1234),
    "gs3d_aniso": (1, 0.0, 0.1, 100.0, None, [1500.0, 1500.0, 500.0], [1, 1, 1], [40, 24, 20], (0, 0, 0), 250, 7),
    "vk3d_rot_offset": (0, 0.5, 0.05, 25.0, None, [3000.0, 3000.0, 1000.0], [5, 3, 2], [60, 50, 33], (30, -10, 5),
                        333, 99),
    "vk3d_dh_lt_ds": (0, 0.3, 0.08, 50.0, 20.0, [2000.0, 2000.0, 800.0], [1, 1, 1], [24, 20, 16], (0, 0, 0), 200,
                      11),
    "gs2d": (1, 0.0, 0.05, 50.0, None, [2000.0, 1200.0], [1, 1], [100, 70], (20, 0, 0), 260, 1235),
    "vk2d": (0, 0.25, 0.05, 50.0, None, [2000.0, 2000.0], [1, 1], [130, 64], (0, 0, 0), 128, 3),
}


def structured_case(name, nharm=None):
    acf, hurst, sigma, ds, dh, cl, fs, fe, ang, nh, seed = STRUCTURED[name]
    if nharm is not None:
        nh = nharm
    kw = dict(acf=acf, nharm=nh, seed=seed, hurst=hurst, sigma=sigma, ds=ds, dh=dh, cl=cl,
              alpha=ang[0], beta=ang[1], gamma=ang[2])
    op = oracle.structured_params(fs=fs, fe=fe, **kw)
    pp = sb.make_params(nc=list(op.nc), fc=list(op.fc), **kw)
    fs3 = list(fs) + [1] * (3 - len(fs))
    fe3 = list(fe) + [1] * (3 - len(fe))
    n = [fe3[c] - fs3[c] + 1 for c in range(3)]
    return dict(op=op, pp=pp, fs=fs3, fe=fe3, n=n, ds=ds, kw=kw, nd=len(cl))


def iarr(v):
    return (ctypes.c_int * 3)(*[int(x) for x in v])


def random_points(npts, box=(20000.0, 20000.0, 10000.0), seed=7):
    """Uniform points in a box, FP32 (numpy default_rng(seed))."""
    rng = np.random.default_rng(seed)
    pts = rng.random((3, npts)) * np.asarray(box)[:, None]
    return pts.astype(np.float32)
