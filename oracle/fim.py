"""FIM (Fourier integral method) oracle: the reference's scarf3d_structured_fim
and scarf3d_unstructured_fim (scarflib_fim.f90:141-1104) restated on the CPU.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA FIM
path, never by the product. Parity status: UNPINNED (no reference build or
golden vectors exist; the uniform stream is the documented one).

The single-precision steps (internal grid, spectrum, Hermitian planes,
nearest-node mapping, statistics, rescale, taper) run in the C oracle
(fim_oracle.c, srm_oracle.c) in the reference's operation order. The inverse
transform -- c2c along z and y, then c2r along x, unnormalised (FFTW_BACKWARD,
scarflib_fim.f90:1705-2315) -- is numpy's, in double precision, rounded to
single precision as the reference's FFTW output is single precision.
The DIP (rotated-axes) build option of the reference is not restated: the
rotation angles do not enter the FIM path, as in its default build.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import L, _i3, _ptr

_vp, _i64 = ctypes.c_void_p, ctypes.c_int64
L.orc_fim_grid.argtypes = [ctypes.c_int, _vp, _vp, ctypes.c_float, _vp, ctypes.c_int, _vp, _vp, _vp]
L.orc_fim_spectrum.argtypes = [_vp, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, _vp,
                               ctypes.c_float, ctypes.c_float, ctypes.c_int, _vp]
L.orc_fim_map_structured.argtypes = [_vp, _vp, ctypes.c_float, _vp, _vp, _vp, ctypes.c_float, _vp]
L.orc_fim_map_points.argtypes = [_vp, _vp, ctypes.c_float, _vp, _vp, _vp, _vp, _i64, ctypes.c_int, _vp]


def _f3(v):
    a = np.zeros(3, np.float32)
    a[:len(v)] = np.asarray(v, np.float32)
    return a


def grid(ndim, nc, fc, dh, cl, pad):
    """Internal grid: (npts[3], off_axis[3], info[0..1])."""
    npts = np.zeros(3, np.int32)
    off = np.zeros(3, np.float32)
    info = np.zeros(2, np.float32)
    ncv, fcv, clv = _f3(nc), _f3(fc), _f3(cl)
    L.orc_fim_grid(int(ndim), _ptr(ncv), _ptr(fcv), float(dh), _ptr(clv), int(pad), _ptr(npts), _ptr(off),
                   _ptr(info))
    return [int(v) for v in npts], off, info


def spectrum(npts, ndim, ds, dh, acf, cl, sigma, hurst, seed):
    """Half spectrum (n3, n2, n1/2+1) complex64 with the Hermitian planes."""
    n1, n2, n3 = npts
    n1h = n1 // 2 + 1
    spec = np.zeros((n3, n2, n1h, 2), np.float32)
    nv = np.asarray(npts, np.int32)
    L.orc_fim_spectrum(_ptr(nv), int(ndim), float(ds), float(dh), int(acf), _ptr(_f3(cl)), float(sigma),
                       float(hurst), int(seed), _ptr(spec))
    return spec[..., 0] + 1j * spec[..., 1].astype(np.float64)


def scaling(npts, ndim, dh):
    """1 / sqrt(n1 n2 n3 dh^n) in single precision (scarflib_fim.f90:1019)."""
    f = np.float32
    dh = f(dh)
    p = f(dh * dh) if ndim == 2 else f(f(dh * dh) * dh)
    v = f(f(f(f(npts[0]) * f(npts[1])) * f(npts[2])) * p)
    return f(f(1.0) / np.sqrt(v))


def internal_field(spec, npts, ndim, dh):
    """REAL(inverse transform) * scaling on the internal grid, (n3, n2, n1) float32."""
    n1, n2, n3 = npts
    if ndim == 3:
        r = np.fft.irfftn(spec.astype(np.complex128), s=(n3, n2, n1), axes=(0, 1, 2), norm="forward")
    else:
        r = np.fft.irfftn(spec[0].astype(np.complex128), s=(n2, n1), axes=(0, 1), norm="forward")[None]
    return (r.astype(np.float32) * scaling(npts, ndim, dh)).astype(np.float32)


def _post(buf, npts, ndim, dh, off, sigma, rescale, poi, mute, taper):
    """Statistics on the internal grid, rescale and taper (:1019-1070)."""
    from . import mean, rescale as orc_rescale, taper_structured, variance
    flat = np.ascontiguousarray(buf.reshape(-1))
    var = variance(flat)
    mu = mean(flat)
    info = np.zeros(4, np.float32)
    info[2] = np.sqrt(np.float32(var))
    info[3] = mu
    if rescale == 1:
        orc_rescale(flat, sigma, float(info[2]), float(info[3]))
        info[2] = sigma
        info[3] = 0.0
    if poi is not None:
        for pt in np.atleast_2d(np.asarray(poi, np.float32)):
            q = np.zeros(3, np.float32)
            for k in range(ndim):
                q[k] = np.float32(pt[k]) - off[k]
            taper_structured(dh, [1, 1, 1], npts, flat, q, mute, taper)
    return flat, info


def execute_structured(*, fs, fe, ds, dh=None, acf, cl, sigma, hurst=0.0, seed, pad=0, rescale=0, poi=None,
                       mute=-999.0, taper=-999.0, nc=None, fc=None):
    """(field, info[0..3], details) of scarf3d_structured_fim on one process."""
    ndim = 3 if len(cl) == 3 and cl[2] > 0 else 2
    fs3 = list(fs) + [1] * (3 - len(fs))
    fe3 = list(fe) + [1] * (3 - len(fe))
    dh = ds if dh is None else dh
    ds32 = np.float32(ds)
    if nc is None:
        nc = [np.float32(fs3[c] - 1) * ds32 for c in range(3)]
        fc = [np.float32(fe3[c] - 1) * ds32 for c in range(3)]
    npts, off, flags = grid(ndim, nc, fc, dh, cl, pad)
    spec = spectrum(npts, ndim, ds, dh, acf, cl, sigma, hurst, seed)
    buf = internal_field(spec, npts, ndim, dh)
    flat, info = _post(buf, npts, ndim, dh, off, sigma, rescale, poi, mute, taper)
    info[0:2] = flags
    n = [fe3[c] - fs3[c] + 1 for c in range(3)]
    field = np.zeros(int(np.prod(n)), np.float32)
    L.orc_fim_map_structured(_ptr(np.asarray(npts, np.int32)), _ptr(flat), float(dh), _ptr(off), _i3(fs3), _i3(fe3),
                             float(ds), _ptr(field))
    return field, info, dict(npts=npts, off_axis=off, internal=flat)


def execute_points(*, x, y, z=None, dh, ds=None, acf, cl, sigma, hurst=0.0, seed, pad=0, rescale=0, poi=None,
                   mute=-999.0, taper=-999.0):
    """(field, info[0..3], details) of scarf3d_unstructured_fim on one process."""
    ndim = 3 if len(cl) == 3 and cl[2] > 0 else 2
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    z = np.zeros_like(x) if z is None else np.ascontiguousarray(z, np.float32)
    ds = dh if ds is None else ds
    nc = [x.min(), y.min(), z.min()]
    fc = [x.max(), y.max(), z.max()]
    npts, off, flags = grid(ndim, nc, fc, dh, cl, pad)
    spec = spectrum(npts, ndim, ds, dh, acf, cl, sigma, hurst, seed)
    buf = internal_field(spec, npts, ndim, dh)
    flat, info = _post(buf, npts, ndim, dh, off, sigma, rescale, poi, mute, taper)
    info[0:2] = flags
    field = np.zeros(len(x), np.float32)
    L.orc_fim_map_points(_ptr(np.asarray(npts, np.int32)), _ptr(flat), float(dh), _ptr(off), _ptr(x), _ptr(y),
                         _ptr(z), len(x), int(ndim), _ptr(field))
    return field, info, dict(npts=npts, off_axis=off, internal=flat)
