"""Library contexts (scarf_ctx), host side: each context keeps its own
initialised mesh and execute settings, the calling thread's current context
is what the reference-compatible entry points act on (the default one unless
another is made current), and destroying a context leaves the others intact.
The reference keeps a single global object (scarflib.f90:87)."""
import ctypes
import os

import numpy as np

import scarf3d_b200 as sb


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _ip(a):
    return np.asarray(a, np.int32).ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def test_settings_and_meshes_are_per_context():
    a, b = sb.Context(), sb.Context()
    try:
        with a:
            sb.set_nharm(777)
            sb.scarf_initialize(fs=[1, 1, 1], fe=[8, 6, 4], ds=50.0, acf=0, cl=[500.0] * 3, sigma=0.1, hurst=0.5)
            with b:
                assert sb.lib.scarf_get_nharm() == 10000
                sb.scarf_initialize(fs=[1, 1, 1], fe=[4, 4, 4], ds=50.0, acf=1, cl=[300.0] * 3, sigma=0.1)
                assert sb._cur().n == (4, 4, 4)
            assert sb.lib.scarf_get_nharm() == 777
            assert sb._cur().n == (8, 6, 4)
        assert sb.lib.scarf_get_nharm() == 10000
        assert sb._cur().n is None
    finally:
        a.close()
        b.close()


def test_io_follows_the_current_context(tmp_path):
    # scarf_io_one needs an initialised structured mesh: the context that has
    # one writes the file, the default context (none) refuses.
    ctx = sb.Context()
    field = np.arange(4 * 3 * 2, dtype=np.float32)
    try:
        with ctx:
            sb.scarf_initialize(fs=[1, 1, 1], fe=[4, 3, 2], ds=10.0, acf=0, cl=[100.0] * 3, sigma=0.1, hurst=0.5)
            path = str(tmp_path / "a.bin")
            sb.scarf_io([4, 3, 2], field, path)
            assert np.array_equal(np.fromfile(path, np.float32), field)
        path2 = str(tmp_path / "b.bin")
        sb.lib.scarf_io_one(3, _ip([4, 3, 2]), ctypes.c_void_p(field.ctypes.data), path2.encode(), None)
        assert not os.path.exists(path2)
        assert "initialized structured mesh" in sb.last_error()
    finally:
        ctx.close()


def test_explicit_context_entry_points():
    h = sb.lib.scarf_ctx_create()
    assert h
    try:
        cl = np.full(3, 400.0, np.float32)
        stats = np.zeros(8, np.float32)
        field = np.zeros(8, np.float32)
        # execute before initialize, on this context only
        rc = sb.lib.scarf_ctx_execute(ctypes.c_void_p(h), 1, ctypes.c_void_p(field.ctypes.data), _fp(stats), 0)
        assert rc == sb.SCARF_ERR_STATE
        assert sb.lib.scarf_ctx_cart_initialize(ctypes.c_void_p(h), 4, _ip([1, 1, 1]), _ip([2, 2, 2]), 10.0, 0,
                                                _fp(cl), 0.1, None) == sb.SCARF_ERR_ARG
        assert sb.lib.scarf_ctx_cart_initialize(ctypes.c_void_p(h), 3, _ip([1, 1, 1]), _ip([2, 2, 2]), 10.0, 0,
                                                _fp(cl), 0.1, None) == sb.SCARF_OK
        x = np.linspace(0, 100, 16).astype(np.float32)
        assert sb.lib.scarf_ctx_nocart_initialize(ctypes.c_void_p(h), 3, 16, _fp(x), _fp(x), None, 10.0, 0,
                                                  _fp(cl), 0.1, None) == sb.SCARF_ERR_ARG
        assert sb.lib.scarf_ctx_nocart_initialize(ctypes.c_void_p(h), 3, 16, _fp(x), _fp(x), _fp(x), 10.0, 0,
                                                  _fp(cl), 0.1, None) == sb.SCARF_OK
        assert sb.lib.scarf_ctx_finalize(ctypes.c_void_p(h)) == sb.SCARF_OK
        # the default context was untouched throughout
        assert sb.lib.scarf_execute_ex(1, ctypes.c_void_p(field.ctypes.data), _fp(stats), 0) == sb.SCARF_ERR_STATE
        assert sb.lib.scarf_ctx_execute(None, 1, ctypes.c_void_p(field.ctypes.data), _fp(stats), 0) == sb.SCARF_ERR_ARG
    finally:
        sb.lib.scarf_ctx_destroy(ctypes.c_void_p(h))


def test_destroying_the_current_context_returns_to_the_default():
    h = sb.lib.scarf_ctx_create()
    assert sb.lib.scarf_ctx_make_current(ctypes.c_void_p(h)) == sb.SCARF_OK
    sb.check(sb.lib.scarf_set_nharm(123))
    assert sb.lib.scarf_get_nharm() == 123
    sb.lib.scarf_ctx_destroy(ctypes.c_void_p(h))
    assert sb.lib.scarf_get_nharm() == 10000
    sb.lib.scarf_ctx_destroy(None)  # ignored


def test_contexts_from_a_c_program(tmp_path):
    """The context entry points as a C caller links them: two meshes kept at
    once, status codes, and the default context untouched."""
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    pkg = root / "scarf3d_b200"
    src = tmp_path / "ctx.c"
    src.write_text(r"""
#include <stdio.h>
#include "scarf3d.h"
#include "scarf3d_b200.h"
int main(void) {
  const int fs[3] = {1, 1, 1}, fa[3] = {8, 6, 4}, fb[3] = {4, 4, 4};
  const float cl[3] = {500.f, 500.f, 500.f};
  struct scarf_opt opt;
  scarf_opt_init(&opt);
  opt.method = 1;
  opt.hurst = 0.5f;
  scarf_ctx *a = scarf_ctx_create(), *b = scarf_ctx_create();
  if (!a || !b) return 1;
  if (scarf_ctx_cart_initialize(a, 3, fs, fa, 50.f, 0, cl, 0.1f, &opt) != SCARF_OK) return 2;
  if (scarf_ctx_cart_initialize(b, 3, fs, fb, 25.f, 1, cl, 0.1f, &opt) != SCARF_OK) return 3;
  scarf_ctx_make_current(a);
  if (scarf_set_nharm(321) != SCARF_OK || scarf_get_nharm() != 321) return 4;
  scarf_ctx_make_current(NULL);
  if (scarf_get_nharm() != 10000) return 5;
  float field[8], stats[8];
  if (scarf_execute_ex(1, field, stats, 0) != SCARF_ERR_STATE) return 6;  /* default: no mesh */
  if (scarf_ctx_finalize(b) != SCARF_OK) return 7;
  if (scarf_ctx_execute(b, 1, field, stats, 0) != SCARF_ERR_STATE) return 8;  /* b finalised */
  scarf_ctx_destroy(a);
  scarf_ctx_destroy(b);
  printf("ok\n");
  return 0;
}
""")
    exe = tmp_path / "ctx"
    subprocess.run(["gcc", "-std=c11", f"-I{root / 'include'}", str(src), f"-L{pkg}", "-lscarf3d_b200",
                    f"-Wl,-rpath,{pkg}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", (r.returncode, r.stdout, r.stderr)
