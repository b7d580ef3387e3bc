"""ctypes wrapper of the CPU oracle (liboracle_srm.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg, always as the checker, never as the product path.
Parity status of the oracle: UNPINNED (see srm_oracle.h).
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "liboracle_srm.so"


class OrcParams(ctypes.Structure):
    _fields_ = [("ndim_hint", ctypes.c_int), ("acf", ctypes.c_int), ("nharm", ctypes.c_int),
                ("seed", ctypes.c_int), ("rescale", ctypes.c_int), ("hurst", ctypes.c_float),
                ("sigma", ctypes.c_float), ("ds", ctypes.c_float), ("dh", ctypes.c_float),
                ("cl", ctypes.c_float * 3), ("nc", ctypes.c_float * 3), ("fc", ctypes.c_float * 3),
                ("alpha", ctypes.c_float), ("beta", ctypes.c_float), ("gamma", ctypes.c_float)]


class OrcSetup(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("kmin", ctypes.c_float), ("kmax", ctypes.c_float),
                ("kc", ctypes.c_float), ("nu", ctypes.c_float), ("cnst", ctypes.c_float),
                ("scaling", ctypes.c_float), ("scaling0", ctypes.c_float), ("m", ctypes.c_float * 9),
                ("bar", ctypes.c_float * 3), ("info0", ctypes.c_float), ("info1", ctypes.c_float),
                ("intg_band", ctypes.c_float), ("intg_full", ctypes.c_float), ("ier_band", ctypes.c_int),
                ("ier_full", ctypes.c_int)]


def _load():
    if not LIB_PATH.exists():
        import subprocess
        subprocess.run(["make", "-C", str(_HERE), "-s"], check=True)
    L = ctypes.CDLL(str(LIB_PATH))
    vp, i64, ip = ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int)
    P, S = ctypes.POINTER(OrcParams), ctypes.POINTER(OrcSetup)
    L.orc_setup_compute.argtypes = [P, S]
    L.orc_sample.argtypes = [P, S, vp, ctypes.POINTER(i64)]
    L.orc_sum_structured_f32.argtypes = [S, ip, ip, ctypes.c_float, vp, ctypes.c_int, vp, i64, vp]
    L.orc_sum_structured_f64.argtypes = [S, ip, ip, ctypes.c_float, vp, ctypes.c_int, vp, i64, vp]
    L.orc_sum_points_f32.argtypes = [S, vp, vp, vp, vp, ctypes.c_int, vp, i64, vp]
    L.orc_sum_points_f64.argtypes = [S, vp, vp, vp, vp, ctypes.c_int, vp, i64, vp]
    L.orc_sum_structured_f32_mt.argtypes = [S, ip, ip, ctypes.c_float, vp, ctypes.c_int, vp, ctypes.c_int]
    L.orc_sum_points_f32_mt.argtypes = [S, vp, vp, vp, i64, vp, ctypes.c_int, vp, ctypes.c_int]
    L.orc_mean.argtypes = [vp, i64]
    L.orc_mean.restype = ctypes.c_float
    L.orc_variance.argtypes = [vp, i64]
    L.orc_variance.restype = ctypes.c_float
    L.orc_parallel_variance.argtypes = [vp, vp, vp, ctypes.c_int, vp, vp]
    L.orc_rescale.argtypes = [vp, i64, ctypes.c_float, ctypes.c_float, ctypes.c_float]
    L.orc_taper_structured.argtypes = [ctypes.c_float, ip, ip, vp, vp, ctypes.c_float, ctypes.c_float]
    L.orc_taper_points.argtypes = [vp, vp, vp, i64, vp, vp, ctypes.c_float, ctypes.c_float]
    L.orc_execute_structured.argtypes = [P, ip, ip, vp, ctypes.c_int, ctypes.c_float, ctypes.c_float, vp, vp,
                                         ctypes.c_int]
    L.orc_rng_seed.argtypes = [vp, ctypes.c_int]
    L.orc_rng_next.argtypes = [vp]
    L.orc_rng_next.restype = ctypes.c_uint32
    L.orc_u01.argtypes = [ctypes.c_uint32]
    L.orc_u01.restype = ctypes.c_float
    L.orc_fn_vk.argtypes = [ctypes.c_float, ctypes.c_float]
    L.orc_fn_vk.restype = ctypes.c_float
    L.orc_fn_gs.argtypes = [ctypes.c_float]
    L.orc_fn_gs.restype = ctypes.c_float
    L.orc_srm_fn.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_float]
    L.orc_srm_fn.restype = ctypes.c_double
    L.orc_dqng.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_double,
                           ctypes.c_double, ctypes.c_double, vp, vp, vp, vp]
    L.orc_dqagi.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_int,
                            ctypes.c_double, ctypes.c_double, ctypes.c_int, vp, vp, vp, vp, vp]
    return L


L = _load()


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def _i3(v):
    return (ctypes.c_int * 3)(*[int(x) for x in v])


def params(*, acf, nharm, seed, hurst=0.0, sigma=1.0, ds, dh=None, cl, nc, fc, rescale=0, alpha=0.0,
           beta=0.0, gamma=0.0) -> OrcParams:
    p = OrcParams()
    p.acf, p.nharm, p.seed, p.rescale = int(acf), int(nharm), int(seed), int(rescale)
    p.hurst, p.sigma, p.ds = float(hurst), float(sigma), float(ds)
    p.dh = float(dh if dh is not None else ds)
    cl3 = list(cl) + [0.0] * (3 - len(cl))
    for c in range(3):
        p.cl[c] = cl3[c]
        p.nc[c] = float(nc[c]) if c < len(nc) else 0.0
        p.fc[c] = float(fc[c]) if c < len(fc) else 0.0
    p.alpha, p.beta, p.gamma = float(alpha), float(beta), float(gamma)
    return p


def structured_params(*, acf, nharm, seed, hurst, sigma, ds, dh=None, cl, fs, fe, **kw) -> OrcParams:
    """Defaults of initialize_structured: nc/fc = (fs-1)*ds, (fe-1)*ds (scarflib.f90:157-158),
    computed in FP32 as the reference does."""
    nd = len(cl)
    fs3 = list(fs) + [1] * (3 - len(fs))
    fe3 = list(fe) + [1] * (3 - len(fe))
    ds32 = np.float32(ds)
    nc = [float(np.float32(fs3[c] - 1) * ds32) for c in range(3)]
    fc = [float(np.float32(fe3[c] - 1) * ds32) for c in range(3)]
    nc = kw.pop("nc", nc)
    fc = kw.pop("fc", fc)
    del nd
    return params(acf=acf, nharm=nharm, seed=seed, hurst=hurst, sigma=sigma, ds=ds, dh=dh, cl=cl, nc=nc, fc=fc,
                  **kw)


def setup(p: OrcParams) -> OrcSetup:
    s = OrcSetup()
    rc = L.orc_setup_compute(ctypes.byref(p), ctypes.byref(s))
    if rc:
        raise ValueError(f"oracle setup failed: {rc}")
    return s


def sample(p: OrcParams, s: OrcSetup) -> tuple[np.ndarray, int]:
    tab = np.zeros((max(p.nharm, 1), 5), np.float32)
    pairs = ctypes.c_int64()
    n = L.orc_sample(ctypes.byref(p), ctypes.byref(s), _ptr(tab), ctypes.byref(pairs))
    return tab[:n].copy(), pairs.value


def sum_structured(s: OrcSetup, fs, n, ds, tab, idx=None, f64=False) -> np.ndarray:
    """FP32 op-order restatement (f64=False) or FP64 oracle (f64=True) at the
    selected linear indices (default: all points)."""
    tab = np.ascontiguousarray(tab, np.float32)
    if idx is None:
        idx = np.arange(int(np.prod(n)), dtype=np.int64)
    idx = np.ascontiguousarray(idx, np.int64)
    out = np.zeros(len(idx), np.float64 if f64 else np.float32)
    fn = L.orc_sum_structured_f64 if f64 else L.orc_sum_structured_f32
    fn(ctypes.byref(s), _i3(fs), _i3(n), float(ds), _ptr(tab), len(tab), _ptr(idx), len(idx), _ptr(out))
    return out


def sum_points(s: OrcSetup, x, y, z, tab, idx=None, f64=False) -> np.ndarray:
    tab = np.ascontiguousarray(tab, np.float32)
    x, y, z = (np.ascontiguousarray(a, np.float32) for a in (x, y, z))
    if idx is None:
        idx = np.arange(len(x), dtype=np.int64)
    idx = np.ascontiguousarray(idx, np.int64)
    out = np.zeros(len(idx), np.float64 if f64 else np.float32)
    fn = L.orc_sum_points_f64 if f64 else L.orc_sum_points_f32
    fn(ctypes.byref(s), _ptr(x), _ptr(y), _ptr(z), _ptr(tab), len(tab), _ptr(idx), len(idx), _ptr(out))
    return out


def sum_structured_mt(s: OrcSetup, fs, n, ds, tab, nthreads=None) -> np.ndarray:
    tab = np.ascontiguousarray(tab, np.float32)
    out = np.zeros(int(np.prod(n)), np.float32)
    L.orc_sum_structured_f32_mt(ctypes.byref(s), _i3(fs), _i3(n), float(ds), _ptr(tab), len(tab), _ptr(out),
                                int(nthreads or os.cpu_count() or 1))
    return out


def sum_points_mt(s: OrcSetup, x, y, z, tab, nthreads=None) -> np.ndarray:
    tab = np.ascontiguousarray(tab, np.float32)
    x, y, z = (np.ascontiguousarray(a, np.float32) for a in (x, y, z))
    out = np.zeros(len(x), np.float32)
    L.orc_sum_points_f32_mt(ctypes.byref(s), _ptr(x), _ptr(y), _ptr(z), len(x), _ptr(tab), len(tab), _ptr(out),
                            int(nthreads or os.cpu_count() or 1))
    return out


def mean(f) -> float:
    f = np.ascontiguousarray(f, np.float32)
    return float(L.orc_mean(_ptr(f), f.size))


def variance(f) -> float:
    f = np.ascontiguousarray(f, np.float32)
    return float(L.orc_variance(_ptr(f), f.size))


def parallel_variance(var, avg, nset):
    v = np.ascontiguousarray(var, np.float32)
    a = np.ascontiguousarray(avg, np.float32)
    n = np.ascontiguousarray(nset, np.int32)
    vo = np.zeros(1, np.float32)
    ao = np.zeros(1, np.float32)
    L.orc_parallel_variance(_ptr(v), _ptr(a), _ptr(n), len(v), _ptr(vo), _ptr(ao))
    return float(vo[0]), float(ao[0])


def rescale(f: np.ndarray, sigma, std, mu) -> None:
    L.orc_rescale(_ptr(f), f.size, float(sigma), float(std), float(mu))


def taper_structured(dh, fs, fe, field: np.ndarray, poi, mute, taper) -> None:
    pt = np.ascontiguousarray(list(poi) + [0.0] * (3 - len(poi)), np.float32)
    L.orc_taper_structured(float(dh), _i3(fs), _i3(fe), _ptr(field), _ptr(pt), float(mute), float(taper))


def taper_points(x, y, z, field: np.ndarray, poi, mute, taper) -> None:
    x, y, z = (np.ascontiguousarray(a, np.float32) for a in (x, y, z))
    pt = np.ascontiguousarray(list(poi) + [0.0] * (3 - len(poi)), np.float32)
    L.orc_taper_points(_ptr(x), _ptr(y), _ptr(z), len(x), _ptr(field), _ptr(pt), float(mute), float(taper))


def execute_structured(p: OrcParams, fs, fe, poi=None, mute=-999.0, taper=-999.0, nthreads=None):
    """Whole structured execute on the CPU; returns (field, info[6])."""
    n = [int(e) - int(s_) + 1 for s_, e in zip(fs, fe)]
    field = np.zeros(int(np.prod(n)), np.float32)
    info = np.zeros(6, np.float32)
    if poi is not None:
        pa = np.ascontiguousarray(poi, np.float32)
        npoi = pa.shape[0] if pa.ndim == 2 else 1
        pp = _ptr(pa)
    else:
        pa, npoi, pp = None, 0, None
    rc = L.orc_execute_structured(ctypes.byref(p), _i3(fs), _i3(fe), pp, npoi, float(mute), float(taper),
                                  _ptr(field), _ptr(info), int(nthreads or os.cpu_count() or 1))
    if rc:
        raise ValueError(f"oracle execute failed: {rc}")
    return field, info


def raw_stream(seed: int, count: int) -> np.ndarray:
    """First `count` raw outputs of the uniform source after seeding."""
    st = (ctypes.c_int64 * 2)()
    L.orc_rng_seed(st, int(seed))
    return np.array([L.orc_rng_next(st) for _ in range(count)], np.uint32)


def dqng(ndim, acf, nu, a, b, epsabs=1e-8, epsrel=1e-5):
    r, e = ctypes.c_double(), ctypes.c_double()
    nev, ier = ctypes.c_int(), ctypes.c_int()
    L.orc_dqng(ndim, acf, nu, a, b, epsabs, epsrel, ctypes.byref(r), ctypes.byref(e), ctypes.byref(nev),
               ctypes.byref(ier))
    return r.value, e.value, ier.value


def dqagi(ndim, acf, nu, bound=0.0, inf=1, epsabs=1e-8, epsrel=1e-5, limit=500):
    r, e = ctypes.c_double(), ctypes.c_double()
    nev, ier, last = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.orc_dqagi(ndim, acf, nu, bound, inf, epsabs, epsrel, limit, ctypes.byref(r), ctypes.byref(e),
                ctypes.byref(nev), ctypes.byref(ier), ctypes.byref(last))
    return r.value, e.value, ier.value
