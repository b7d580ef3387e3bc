"""Python host interface of the B200 SRM library (libscarf3d_b200.so).

Mirrors SCARF3D's initialize / execute / finalize interface (scarflib.f90:48-62,
c_binding.c:62-150) with the same argument names and meaning, over the library's
C ABI (include/scarf3d.h, include/scarf3d_b200.h). There is no CPU fallback: if
the shared library is missing or fails to load, importing this package raises.
"""
from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("SCARF3D_B200_LIB", _HERE / "libscarf3d_b200.so"))

SCARF_OK = 0
SCARF_ERR_ARG = -1
SCARF_ERR_STATE = -2
SCARF_ERR_CUDA = -3
SCARF_ERR_UNSUPPORTED = -4
SCARF_ERR_DEVICE = -5
SCARF_ERR_NOMEM = -6

FORM_AUTO, FORM_DIRECT, FORM_TC = 0, 1, 2
FIELD_ON_DEVICE, TAPER_UNSTRUCTURED = 1, 2

EXPORTED_SYMBOLS = (
    # reference-compatible (include/scarf3d.h)
    "scarf_opt_init", "scarf_cart_initialize", "scarf_nocart_initialize", "scarf_execute",
    "scarf_finalize", "scarf_io_one", "scarf_io_slice",
    # extended (include/scarf3d_b200.h)
    "scarf_last_error", "scarf_set_nharm", "scarf_get_nharm", "scarf_set_form",
    "scarf_set_uniform_source", "scarf_set_stream", "scarf_set_host_threads", "scarf_set_kernel_timing",
    "scarf_last_kernel_ms", "scarf_set_device_memory_cap", "scarf_device_memory_in_use",
    "scarf_release_device_memory",
    "scarf_selftest_wait_limit", "scarf_set_tc_chunk", "scarf_set_tc_variant", "scarf_set_tc_precision",
    "scarf_set_direct_sincos", "scarf_fim_internal_grid", "scarf_fim_workspace_bytes",
    "scarf_set_output_overlap",
    "scarf_execute_ex", "scarf_ctx_create", "scarf_ctx_destroy", "scarf_ctx_make_current",
    "scarf_ctx_cart_initialize", "scarf_ctx_nocart_initialize", "scarf_ctx_execute", "scarf_ctx_finalize",
    "scarf_srm_compute_setup", "scarf_srm_sample", "scarf_srm_sample_device", "scarf_srm_sample_device_batch",
    "scarf_srm_sampler_reject_table", "scarf_set_sampler",
    "scarf_set_sampler_pass_pairs",
    "scarf_srm_direct_structured",
    "scarf_srm_direct_points", "scarf_srm_tc_workspace_bytes", "scarf_srm_tc_structured",
    "scarf_srm_tc_noalloc_capacity_bytes", "scarf_srm_tc_structured_noalloc",
    "scarf_srm_tc_batch_workspace_bytes", "scarf_srm_tc_batch_create", "scarf_srm_tc_batch_launch",
    "scarf_srm_tc_batch_wait", "scarf_srm_tc_batch_destroy", "scarf_srm_tc_batch_set_host_outputs",
    "scarf_set_tc_autotune", "scarf_set_tc_tune_cache", "scarf_srm_tc_autotune", "scarf_srm_tc_batch_autotune",
    "scarf_srm_tc_plan_info",
    "scarf_field_stats_workspace_bytes", "scarf_field_stats",
)


class ScarfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"scarf3d_b200 error {code}: {msg}")
        self.code = code


class ScarfOpt(ctypes.Structure):
    """struct scarf_opt (src/scarf3d.h:54-70), byte-for-byte."""
    _fields_ = [("method", ctypes.c_int), ("hurst", ctypes.c_float), ("dh", ctypes.c_float),
                ("ds", ctypes.c_float), ("poi", ctypes.POINTER(ctypes.c_float)), ("npoi", ctypes.c_int),
                ("mute", ctypes.c_float), ("taper", ctypes.c_float), ("rescale", ctypes.c_int),
                ("pad", ctypes.c_int), ("nc", ctypes.POINTER(ctypes.c_float)),
                ("fc", ctypes.POINTER(ctypes.c_float)), ("alpha", ctypes.c_float),
                ("beta", ctypes.c_float), ("gamma", ctypes.c_float)]


class SrmParams(ctypes.Structure):
    _fields_ = [("acf", ctypes.c_int), ("nharm", ctypes.c_int), ("seed", ctypes.c_int),
                ("rescale", ctypes.c_int), ("hurst", ctypes.c_float), ("sigma", ctypes.c_float),
                ("ds", ctypes.c_float), ("dh", ctypes.c_float), ("cl", ctypes.c_float * 3),
                ("nc", ctypes.c_float * 3), ("fc", ctypes.c_float * 3), ("alpha", ctypes.c_float),
                ("beta", ctypes.c_float), ("gamma", ctypes.c_float)]


class SrmSetup(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("kmin", ctypes.c_float), ("kmax", ctypes.c_float),
                ("kc", ctypes.c_float), ("nu", ctypes.c_float), ("cnst", ctypes.c_float),
                ("scaling", ctypes.c_float), ("scaling0", ctypes.c_float), ("m", ctypes.c_float * 9),
                ("bar", ctypes.c_float * 3), ("info0", ctypes.c_float), ("info1", ctypes.c_float),
                ("intg_band", ctypes.c_float), ("intg_full", ctypes.c_float), ("ier_band", ctypes.c_int),
                ("ier_full", ctypes.c_int)]


class TcField(ctypes.Structure):
    """scarf_tc_field: one structured field of a batched tensor-core launch."""
    _fields_ = [("setup", ctypes.POINTER(SrmSetup)), ("fs", ctypes.c_int * 3), ("n", ctypes.c_int * 3),
                ("ds", ctypes.c_float), ("d_table", ctypes.c_void_p), ("nh", ctypes.c_int),
                ("d_field", ctypes.c_void_p), ("tile_j", ctypes.c_int)]


class TcTuning(ctypes.Structure):
    """scarf_tc_tuning: a tuned plan choice of the tensor-core form."""
    _fields_ = [("variant", ctypes.c_int), ("tile_j", ctypes.c_int), ("permute", ctypes.c_int),
                ("ms", ctypes.c_float), ("split", ctypes.c_int)]


def _load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"scarf3d_b200: {LIB_PATH} is missing; build it with "
                          f"`python scarf3d_b200/build.py` (no CPU fallback exists)")
    lib = ctypes.CDLL(str(LIB_PATH))
    c_int, c_float, c_void_p, c_size_t, c_ll = (ctypes.c_int, ctypes.c_float, ctypes.c_void_p,
                                                ctypes.c_size_t, ctypes.c_longlong)
    fp = ctypes.POINTER(c_float)
    ip = ctypes.POINTER(c_int)
    sig = {
        "scarf_opt_init": (None, [ctypes.POINTER(ScarfOpt)]),
        "scarf_cart_initialize": (None, [c_int, ip, ip, c_float, c_int, fp, c_float, ctypes.POINTER(ScarfOpt)]),
        "scarf_nocart_initialize": (None, [c_int, c_int, fp, fp, fp, c_float, c_int, fp, c_float,
                                           ctypes.POINTER(ScarfOpt)]),
        "scarf_execute": (None, [c_int, c_void_p, fp]),
        "scarf_finalize": (None, []),
        "scarf_io_one": (None, [c_int, ip, c_void_p, ctypes.c_char_p, ip]),
        "scarf_io_slice": (None, [ip, ctypes.c_char_p, c_int, c_void_p, ctypes.c_char_p]),
        "scarf_last_error": (ctypes.c_char_p, []),
        "scarf_set_nharm": (c_int, [c_int]),
        "scarf_get_nharm": (c_int, []),
        "scarf_set_form": (c_int, [c_int]),
        "scarf_set_uniform_source": (c_int, [c_void_p, c_void_p]),
        "scarf_set_stream": (c_int, [c_void_p]),
        "scarf_set_host_threads": (c_int, [c_int]),
        "scarf_set_kernel_timing": (c_int, [c_int]),
        "scarf_last_kernel_ms": (c_float, []),
        "scarf_set_device_memory_cap": (c_int, [c_size_t]),
        "scarf_device_memory_in_use": (c_size_t, []),
        "scarf_release_device_memory": (c_int, []),
        "scarf_selftest_wait_limit": (c_int, [c_int, ctypes.POINTER(c_int), ctypes.POINTER(ctypes.c_double)]),
        "scarf_set_tc_chunk": (c_int, [c_int]),
        "scarf_set_tc_variant": (c_int, [c_int]),
        "scarf_set_tc_precision": (c_int, [c_int, c_int]),
        "scarf_set_direct_sincos": (c_int, [c_int]),
        "scarf_fim_internal_grid": (c_int, [c_int, c_void_p, c_void_p, ctypes.c_float, c_void_p, c_int, c_void_p,
                                            c_void_p, c_void_p]),
        "scarf_fim_workspace_bytes": (ctypes.c_size_t, [c_void_p, c_int]),
        "scarf_set_output_overlap": (c_int, [c_int]),
        "scarf_execute_ex": (c_int, [c_int, c_void_p, fp, c_int]),
        "scarf_ctx_create": (c_void_p, []),
        "scarf_ctx_destroy": (None, [c_void_p]),
        "scarf_ctx_make_current": (c_int, [c_void_p]),
        "scarf_ctx_cart_initialize": (c_int, [c_void_p, c_int, ip, ip, c_float, c_int, fp, c_float,
                                              ctypes.POINTER(ScarfOpt)]),
        "scarf_ctx_nocart_initialize": (c_int, [c_void_p, c_int, c_int, fp, fp, fp, c_float, c_int, fp, c_float,
                                                ctypes.POINTER(ScarfOpt)]),
        "scarf_ctx_execute": (c_int, [c_void_p, c_int, c_void_p, fp, c_int]),
        "scarf_ctx_finalize": (c_int, [c_void_p]),
        "scarf_srm_compute_setup": (c_int, [ctypes.POINTER(SrmParams), ctypes.POINTER(SrmSetup)]),
        "scarf_srm_sample": (c_int, [ctypes.POINTER(SrmParams), ctypes.POINTER(SrmSetup), c_void_p, ip,
                                     ctypes.POINTER(c_ll)]),
        "scarf_srm_sample_device": (c_int, [ctypes.POINTER(SrmParams), ctypes.POINTER(SrmSetup), c_void_p, ip,
                                            ctypes.POINTER(c_ll), ctypes.POINTER(c_ll), c_void_p]),
        "scarf_srm_sample_device_batch": (c_int, [c_int, c_void_p, c_void_p, c_void_p, ip, c_void_p,
                                                  ctypes.POINTER(c_ll), c_void_p]),
        "scarf_srm_sampler_reject_table": (c_int, [ctypes.POINTER(SrmParams), ctypes.POINTER(SrmSetup), c_void_p]),
        "scarf_set_sampler": (c_int, [c_int]),
        "scarf_set_sampler_pass_pairs": (c_int, [c_ll]),
        "scarf_srm_direct_structured": (c_int, [ctypes.POINTER(SrmSetup), ip, ip, c_float, c_void_p, c_int,
                                                c_void_p, c_void_p]),
        "scarf_srm_direct_points": (c_int, [ctypes.POINTER(SrmSetup), c_void_p, c_void_p, c_void_p, c_ll,
                                            c_void_p, c_int, c_void_p, c_void_p]),
        "scarf_srm_tc_workspace_bytes": (c_size_t, [c_int, ip, c_int]),
        "scarf_srm_tc_structured": (c_int, [ctypes.POINTER(SrmSetup), ip, ip, c_float, c_void_p, c_int,
                                            c_void_p, c_void_p, c_size_t, c_void_p]),
        "scarf_srm_tc_batch_workspace_bytes": (c_size_t, [ctypes.POINTER(TcField), c_int]),
        "scarf_srm_tc_batch_create": (c_int, [ctypes.POINTER(TcField), c_int, c_void_p, c_size_t,
                                              ctypes.POINTER(c_void_p)]),
        "scarf_srm_tc_batch_launch": (c_int, [c_void_p, c_void_p]),
        "scarf_srm_tc_batch_wait": (c_int, [c_void_p, c_void_p]),
        "scarf_srm_tc_batch_destroy": (None, [c_void_p]),
        "scarf_srm_tc_batch_set_host_outputs": (c_int, [c_void_p, c_void_p]),
        "scarf_srm_tc_noalloc_capacity_bytes": (c_size_t, []),
        "scarf_srm_tc_structured_noalloc": (c_int, [ctypes.POINTER(SrmSetup), ip, ip, c_float, c_void_p, c_int,
                                                    c_void_p, c_void_p]),
        "scarf_set_tc_autotune": (c_int, [c_int]),
        "scarf_srm_tc_plan_info": (c_int, [c_int, ip, c_int, ctypes.POINTER(TcTuning)]),
        "scarf_set_tc_tune_cache": (c_int, [ctypes.c_char_p]),
        "scarf_srm_tc_autotune": (c_int, [ctypes.POINTER(SrmSetup), ip, ip, c_float, c_void_p, c_int, c_int,
                                          c_void_p, ctypes.POINTER(TcTuning)]),
        "scarf_srm_tc_batch_autotune": (c_int, [ctypes.POINTER(TcField), c_int, c_void_p,
                                                ctypes.POINTER(TcTuning)]),
        "scarf_field_stats_workspace_bytes": (c_size_t, [c_ll]),
        "scarf_field_stats": (c_int, [c_void_p, c_ll, c_void_p, c_size_t, fp, fp, c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    return (lib.scarf_last_error() or b"").decode()


def check(rc: int) -> None:
    if rc != SCARF_OK:
        raise ScarfError(rc, last_error())


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _iptr(a):
    arr = (ctypes.c_int * len(a))(*[int(v) for v in a])
    return arr


def _fptr(a):
    return (ctypes.c_float * len(a))(*[float(v) for v in a])


# --------------------------------------------------------------------------
# Reference-style interface (scarflib.f90 generic procedures)
# --------------------------------------------------------------------------
class _MeshState:
    """Python-side companions of one context's mesh: the arrays the library
    borrows until finalize, and the field extent."""

    def __init__(self):
        self.keep: list = []
        self.n: tuple | None = None
        self.structured = True


_DEFAULT_MESH = _MeshState()
_tls = threading.local()


def _cur() -> _MeshState:
    """The calling thread's current context's mesh state (the default
    context's outside `with Context()`)."""
    return getattr(_tls, "mesh", _DEFAULT_MESH)


class Context:
    """One independent library instance (scarf_ctx): an initialised mesh, the
    execute settings (nharm, form, stream, sampler, ...) and the device buffers
    of its execute path. Several contexts hold different meshes at once.
    Inside `with ctx:` the calling thread's current context is ctx, so
    scarf_initialize, scarf_execute, scarf_finalize, set_nharm and the other
    per-context settings act on it."""

    def __init__(self):
        self._h = lib.scarf_ctx_create()
        if not self._h:
            raise ScarfError(SCARF_ERR_NOMEM, last_error())
        self._mesh = _MeshState()
        self._mesh._ctx_handle = self._h

    def __enter__(self):
        if not self._h:
            raise ScarfError(SCARF_ERR_STATE, "context is closed")
        check(lib.scarf_ctx_make_current(ctypes.c_void_p(self._h)))
        stack = getattr(_tls, "stack", None)
        if stack is None:
            stack = _tls.stack = []
        stack.append(_cur())
        _tls.mesh = self._mesh
        return self

    def __exit__(self, *exc):
        outer_mesh = _tls.stack.pop()
        _tls.mesh = outer_mesh
        outer = getattr(outer_mesh, "_ctx_handle", None)
        lib.scarf_ctx_make_current(ctypes.c_void_p(outer) if outer else None)
        return False

    def close(self):
        if self._h:
            lib.scarf_ctx_destroy(ctypes.c_void_p(self._h))
            self._h = None
            self._mesh = _MeshState()
            self._mesh._ctx_handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scarf_initialize(*, fs=None, fe=None, ds=None, x=None, y=None, z=None, dh=None, acf, cl, sigma,
                     method=1, hurst=0.0, poi=None, mute=0.0, taper=0.0, rescale=0, pad=0, nc=None,
                     fc=None, alpha=0.0, beta=0.0, gamma=0.0):
    """initialize_structured (fs, fe, ds given) or initialize_unstructured (x, y[, z], dh given).

    Optional arguments follow the C binding's rule: they count as given when
    > 0 (hurst, dh/ds, mute, taper, npoi), == 1 (method, rescale, pad) or != 0
    (angles); nc and fc must be given together.
    """
    opt = ScarfOpt()
    lib.scarf_opt_init(ctypes.byref(opt))
    opt.method = int(method)
    opt.hurst = float(hurst)
    opt.mute = float(mute)
    opt.taper = float(taper)
    opt.rescale = int(rescale)
    opt.pad = int(pad)
    opt.alpha, opt.beta, opt.gamma = float(alpha), float(beta), float(gamma)
    keep = []
    if poi is not None:
        p = _f32(poi)
        keep.append(p)
        opt.poi = p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        opt.npoi = p.shape[0] if p.ndim == 2 else 1
    if nc is not None and fc is not None:
        a, b = _f32(nc), _f32(fc)
        keep += [a, b]
        opt.nc = a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        opt.fc = b.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    clv = _f32(cl)
    keep.append(clv)
    nd = len(clv)
    if fs is not None:
        if dh is not None:
            opt.dh = float(dh)
        lib.scarf_cart_initialize(nd, _iptr(fs), _iptr(fe), float(ds), int(acf),
                                  clv.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(sigma),
                                  ctypes.byref(opt))
        _cur().structured = True
        _cur().n = tuple(int(e) - int(s) + 1 for s, e in zip(fs, fe))
    else:
        if ds is not None:
            opt.ds = float(ds)
        xs, ys = _f32(x), _f32(y)
        zs = _f32(z) if z is not None else None
        keep += [xs, ys] + ([zs] if zs is not None else [])
        fpz = zs.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if zs is not None else None
        lib.scarf_nocart_initialize(nd, len(xs), xs.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                    ys.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), fpz, float(dh), int(acf),
                                    clv.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(sigma),
                                    ctypes.byref(opt))
        _cur().structured = False
        _cur().n = (len(xs),)
    err = last_error()
    if err:
        raise ScarfError(SCARF_ERR_ARG, err)
    _cur().keep = keep  # the library borrows these until scarf_finalize


def scarf_execute(seed: int, field=None, *, flags: int = 0):
    """Run the SRM; returns (field, stats[8]). `field` may be a NumPy array
    (host) or an object exposing a CUDA device pointer via `data_ptr()`
    (torch tensor), float32, column-major extent n0 x n1 x n2 / npts."""
    if _cur().n is None:
        raise ScarfError(SCARF_ERR_STATE, "scarf_execute before scarf_initialize")
    stats = np.zeros(8, np.float32)
    if field is None:
        field = np.zeros(int(np.prod(_cur().n)), np.float32)
    if hasattr(field, "data_ptr"):
        ptr = field.data_ptr()
        flags |= FIELD_ON_DEVICE if field.is_cuda else 0
    else:
        if field.dtype != np.float32 or not field.flags["C_CONTIGUOUS"] and not field.flags["F_CONTIGUOUS"]:
            raise ValueError("field must be a contiguous float32 array")
        ptr = field.ctypes.data
    check(lib.scarf_execute_ex(int(seed), ctypes.c_void_p(ptr),
                               stats.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), int(flags)))
    return field, stats


def scarf_finalize():
    lib.scarf_finalize()
    _cur().keep = []
    _cur().n = None


def scarf_io(npts, field, filename: str, nwriters=None):
    nwr = _iptr([nwriters]) if nwriters else None
    f = _f32(field) if not hasattr(field, "ctypes") else field
    lib.scarf_io_one(len(npts), _iptr(npts), ctypes.c_void_p(f.ctypes.data), filename.encode(), nwr)


def scarf_io_slice(npts, axis: str, plane: int, field, filename: str):
    lib.scarf_io_slice(_iptr(npts), axis.encode(), int(plane), ctypes.c_void_p(field.ctypes.data),
                       filename.encode())


# --------------------------------------------------------------------------
# Building blocks
# --------------------------------------------------------------------------
def make_params(*, acf, nharm, seed, hurst=0.0, sigma=1.0, ds, dh=None, cl, nc, fc, rescale=0,
                alpha=0.0, beta=0.0, gamma=0.0) -> SrmParams:
    p = SrmParams()
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


def compute_setup(p: SrmParams) -> SrmSetup:
    s = SrmSetup()
    check(lib.scarf_srm_compute_setup(ctypes.byref(p), ctypes.byref(s)))
    return s


def sample(p: SrmParams, s: SrmSetup) -> tuple[np.ndarray, int]:
    """Harmonic table (n_kept x 5: v1, v2, v3, a, b) and the srng pairs used."""
    tab = np.zeros((max(p.nharm, 1), 5), np.float32)
    kept = ctypes.c_int()
    used = ctypes.c_longlong()
    check(lib.scarf_srm_sample(ctypes.byref(p), ctypes.byref(s), tab.ctypes.data_as(ctypes.c_void_p),
                               ctypes.byref(kept), ctypes.byref(used)))
    return tab[: kept.value].copy(), used.value


SAMPLER_AUTO, SAMPLER_HOST, SAMPLER_DEVICE = 0, 1, 2


def sample_device(p: SrmParams, s: SrmSetup, stream_handle: int | None = None):
    """Device-assisted sampler: (table, pairs used, pairs decided on the host)."""
    tab = np.zeros((max(p.nharm, 1), 5), np.float32)
    kept = ctypes.c_int()
    used = ctypes.c_longlong()
    open_ = ctypes.c_longlong()
    check(lib.scarf_srm_sample_device(ctypes.byref(p), ctypes.byref(s), tab.ctypes.data_as(ctypes.c_void_p),
                                      ctypes.byref(kept), ctypes.byref(used), ctypes.byref(open_),
                                      ctypes.c_void_p(stream_handle or 0)))
    return tab[: kept.value].copy(), used.value, open_.value


def sampler_reject_table(p: SrmParams, s: SrmSetup):
    """The device scan's certain-reject thresholds on the second raw draw,
    one per bin y1 >> 23 of the first (256 uint32; 0xFFFFFFFF = never)."""
    thr = np.zeros(256, np.uint32)
    check(lib.scarf_srm_sampler_reject_table(ctypes.byref(p), ctypes.byref(s), thr.ctypes.data_as(ctypes.c_void_p)))
    return thr


def sample_device_batch(params, setups, stream_handle: int | None = None, out=None):
    """Device-assisted sampler for many fields in one pass of launches:
    (list of tables, list of pairs used, pairs decided on the host). Each
    table is a view of its kept rows. `out` optionally gives the arrays to
    write into, one per field: float32, C-contiguous, at least nharm x 5
    (for example views of one page-locked buffer, ready for one upload)."""
    n = len(params)
    if len(setups) != n:
        raise ValueError("params and setups differ in length")
    p_arr = (SrmParams * n)(*params)
    s_arr = (SrmSetup * n)(*setups)
    if out is None:
        tabs = [np.empty((max(p.nharm, 1), 5), np.float32) for p in params]
    else:
        if len(out) != n:
            raise ValueError("out must hold one array per field")
        tabs = []
        for p, t in zip(params, out):
            t = np.asarray(t)
            if (t.dtype != np.float32 or not t.flags.c_contiguous or not t.flags.writeable
                    or t.size < 5 * max(p.nharm, 1)):
                raise ValueError("each out array must be writeable, C-contiguous float32 with room for "
                                 "nharm x 5 values")
            tabs.append(t.reshape(-1)[: 5 * max(p.nharm, 1)].reshape(-1, 5))
    ptrs = (ctypes.c_void_p * n)(*[t.ctypes.data for t in tabs])
    kept = (ctypes.c_int * n)()
    used = (ctypes.c_longlong * n)()
    open_ = ctypes.c_longlong()
    check(lib.scarf_srm_sample_device_batch(n, ctypes.cast(p_arr, ctypes.c_void_p), ctypes.cast(s_arr, ctypes.c_void_p),
                                            ctypes.cast(ptrs, ctypes.c_void_p), kept,
                                            ctypes.cast(used, ctypes.c_void_p), ctypes.byref(open_),
                                            ctypes.c_void_p(stream_handle or 0)))
    return [t[: kept[i]] for i, t in enumerate(tabs)], list(used), open_.value


def set_sampler(where: int):
    check(lib.scarf_set_sampler(int(where)))


def set_nharm(n: int):
    check(lib.scarf_set_nharm(int(n)))


def set_form(form: int):
    check(lib.scarf_set_form(int(form)))


TC_PAIR, TC_SINGLE, TC_SINGLE_TMEM_A = 0, 1, 2


def set_tc_variant(variant: int):
    """Tensor-core kernel form for plans made afterwards: TC_SINGLE (default),
    TC_PAIR (CTA pairs with cta_group::2 MMAs) or TC_SINGLE_TMEM_A."""
    check(lib.scarf_set_tc_variant(int(variant)))


TC_FP16, TC_BF16 = 0, 1
SINCOS_ACCURATE, SINCOS_FAST = 0, 1


def set_direct_sincos(mode: int):
    """sin/cos of the FP32 direct sum: SINCOS_FAST (default: Cody-Waite
    reduction + SFU) or SINCOS_ACCURATE (CUDA's sincosf)."""
    check(lib.scarf_set_direct_sincos(int(mode)))


def set_tc_precision(operand_type: int = 1, terms: int = 3):
    """Operand split of the tensor-core form for plans made afterwards:
    TC_BF16 (default) or TC_FP16 hi/lo parts, 3 (default) or 2 products."""
    check(lib.scarf_set_tc_precision(int(operand_type), int(terms)))


def fim_internal_grid(ndim: int, nc, fc, dh: float, cl, pad: int = 0):
    """(npts[3], off_axis[3], flags[2]) of the FIM's internal grid."""
    ncv = np.zeros(3, np.float32)
    fcv = np.zeros(3, np.float32)
    clv = np.zeros(3, np.float32)
    ncv[:len(nc)], fcv[:len(fc)], clv[:len(cl)] = nc, fc, cl
    npts = np.zeros(3, np.int32)
    off = np.zeros(3, np.float32)
    flags = np.zeros(2, np.float32)
    check(lib.scarf_fim_internal_grid(int(ndim), ncv.ctypes.data, fcv.ctypes.data, float(dh), clv.ctypes.data,
                                      int(pad), npts.ctypes.data, off.ctypes.data, flags.ctypes.data))
    return [int(v) for v in npts], off, flags


def set_device_memory_cap(nbytes: int):
    """Cap on the device memory the library allocates for itself (0: none);
    calls that would pass it raise ScarfError(SCARF_ERR_NOMEM)."""
    check(lib.scarf_set_device_memory_cap(int(nbytes)))


def device_memory_in_use() -> int:
    return int(lib.scarf_device_memory_in_use())


def release_device_memory():
    """Frees the device buffers the library keeps between calls."""
    check(lib.scarf_release_device_memory())


def selftest_wait_limit(blocks: int = 4) -> dict:
    """Runs the bounded-wait self-test (blocks wait on an mbarrier that nothing
    arrives on); returns the status word and the longest wait in seconds.
    Raises when the waits did not report the timeout as designed."""
    st = ctypes.c_int(-1)
    waited = ctypes.c_double(0.0)
    check(lib.scarf_selftest_wait_limit(int(blocks), ctypes.byref(st), ctypes.byref(waited)))
    return {"status": st.value, "waited_s": waited.value}


def set_tc_autotune(mode: int):
    """0: default plans; 1: plans follow recorded tunings of their shape bucket."""
    check(lib.scarf_set_tc_autotune(int(mode)))


def set_tc_tune_cache(path):
    """Append tunings to (and read them from) this text file; None: memory only."""
    check(lib.scarf_set_tc_tune_cache(None if path is None else str(path).encode()))


def tc_autotune(s: "SrmSetup", fs, n, ds: float, d_table: int, nh: int, fixed_columns: bool = False,
                stream_handle: int | None = None) -> dict:
    """Time the candidate plans of one grid on the device table `d_table`
    (device pointer, nh rows) and record the fastest for its shape bucket."""
    t = TcTuning()
    check(lib.scarf_srm_tc_autotune(ctypes.byref(s), _iptr(fs), _iptr(n), float(ds), ctypes.c_void_p(int(d_table)),
                                    int(nh), int(bool(fixed_columns)), ctypes.c_void_p(stream_handle or 0),
                                    ctypes.byref(t)))
    return {"variant": t.variant, "tile_j": t.tile_j, "permute": t.permute, "ms": t.ms, "split": t.split}


def tc_plan_info(ndim: int, n, nh: int) -> dict:
    """The plan the device-field tensor-core entry points would use now."""
    t = TcTuning()
    check(lib.scarf_srm_tc_plan_info(int(ndim), _iptr(n), int(nh), ctypes.byref(t)))
    return {"variant": t.variant, "tile_j": t.tile_j, "permute": t.permute, "split": t.split}


def set_output_overlap(items_per_slab: int = 1):
    """scarf_execute: copy finished field slabs (about items_per_slab work
    items each; 1 = default size) to the host while the kernel runs, or the
    whole field afterwards (0)."""
    check(lib.scarf_set_output_overlap(int(items_per_slab)))


def set_host_threads(n: int):
    check(lib.scarf_set_host_threads(int(n)))


def set_stream(stream_handle: int | None):
    check(lib.scarf_set_stream(ctypes.c_void_p(stream_handle or 0)))


def tc_workspace_bytes(ndim: int, n, nh: int) -> int:
    return int(lib.scarf_srm_tc_workspace_bytes(int(ndim), _iptr(n), int(nh)))


def _tc_field_array(entries, setups):
    arr = (TcField * len(entries))()
    for k, e in enumerate(entries):
        f = arr[k]
        f.setup = ctypes.pointer(setups[k])
        for c in range(3):
            f.fs[c] = int(e["fs"][c])
            f.n[c] = int(e["n"][c])
        f.ds = float(e["ds"])
        f.d_table = ctypes.c_void_p(int(e["d_table"]))
        f.nh = int(e["nh"])
        f.d_field = ctypes.c_void_p(int(e["d_field"]))
        f.tile_j = int(e.get("tile_j", 0))
    return arr


def tc_batch_autotune(entries, stream_handle: int | None = None) -> dict:
    """Time the candidate plans of a batch (the TcBatch entries; outputs are
    overwritten) and return the fastest {variant, tile_j, ms}."""
    setups = [e["setup"] for e in entries]
    arr = _tc_field_array(entries, setups)
    t = TcTuning()
    check(lib.scarf_srm_tc_batch_autotune(arr, len(entries), ctypes.c_void_p(stream_handle or 0), ctypes.byref(t)))
    return {"variant": t.variant, "tile_j": t.tile_j, "ms": t.ms}


class TcBatch:
    """Batched tensor-core launch over many structured fields.

    `entries` is a list of dicts with keys setup (SrmSetup), fs, n, ds,
    d_table (device pointer), nh, d_field (device pointer) and optional tile_j.
    `alloc(nbytes)` returns a device buffer object exposing data_ptr() (e.g. a
    torch.uint8 CUDA tensor) that stays alive with the batch.
    """

    def __init__(self, entries, alloc):
        self._setups = [e["setup"] for e in entries]
        arr = _tc_field_array(entries, self._setups)
        self._arr = arr
        self.bytes = int(lib.scarf_srm_tc_batch_workspace_bytes(arr, len(entries)))
        if self.bytes == 0:
            raise ScarfError(SCARF_ERR_ARG, "fields cannot share one batched launch")
        self.work = alloc(self.bytes)
        # held by the instance: module globals may already be gone when a
        # batch is collected at interpreter exit
        self._destroy = lib.scarf_srm_tc_batch_destroy
        self._h = ctypes.c_void_p()
        check(lib.scarf_srm_tc_batch_create(arr, len(entries), ctypes.c_void_p(self.work.data_ptr()), self.bytes,
                                            ctypes.byref(self._h)))

    def launch(self, stream_handle: int | None = None):
        check(lib.scarf_srm_tc_batch_launch(self._h, ctypes.c_void_p(stream_handle or 0)))

    def set_host_outputs(self, host_ptrs):
        """Host buffers (addresses, one per field, page-locked for full speed)
        that wait() fills field by field as the launch completes them; None
        turns the copy-out off."""
        if host_ptrs is None:
            check(lib.scarf_srm_tc_batch_set_host_outputs(self._h, None))
            self._host = None
            return
        arr = (ctypes.c_void_p * len(host_ptrs))(*[int(p) for p in host_ptrs])
        check(lib.scarf_srm_tc_batch_set_host_outputs(self._h, arr))
        self._host = arr

    def wait(self, stream_handle: int | None = None):
        check(lib.scarf_srm_tc_batch_wait(self._h, ctypes.c_void_p(stream_handle or 0)))

    def close(self):
        """Releases the batch's host-side state (its workspace belongs to the
        caller's allocation); later calls raise."""
        h = getattr(self, "_h", None)
        if h:
            self._destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        self.close()
