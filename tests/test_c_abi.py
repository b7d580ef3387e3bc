"""The C ABI on the CPU: every declared entry point is exported, the structs
match the C layout, error paths report status codes, the binary writers
produce the reference's raw column-major format, and the package refuses to
load without its shared library (no CPU fallback)."""
import ctypes
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import HAS_GPU

import scarf3d_b200 as sb

ROOT = Path(__file__).resolve().parent.parent
INCLUDE = ROOT / "include"


def _declared_functions():
    names = set()
    for h in INCLUDE.glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = text.split("namespace Scarf3D")[0]
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(scarf_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_every_declared_entry_point_is_exported():
    declared = _declared_functions()
    assert len(declared) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", str(sb.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = sorted(declared - exported)
    assert not missing, missing
    assert declared <= set(sb.EXPORTED_SYMBOLS) | {"scarf_srm_tc_noalloc_capacity_bytes"}
    for name in declared:
        assert getattr(sb.lib, name) is not None


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(r"""
#include <stddef.h>
#include <stdio.h>
#include "scarf3d.h"
#include "scarf3d_b200.h"
#define P(T, f) printf(#T "." #f " %zu\n", offsetof(struct T, f))
int main(void) {
  P(scarf_opt, method); P(scarf_opt, hurst); P(scarf_opt, dh); P(scarf_opt, ds); P(scarf_opt, poi);
  P(scarf_opt, npoi); P(scarf_opt, mute); P(scarf_opt, taper); P(scarf_opt, rescale); P(scarf_opt, pad);
  P(scarf_opt, nc); P(scarf_opt, fc); P(scarf_opt, alpha); P(scarf_opt, beta); P(scarf_opt, gamma);
  printf("scarf_opt.size %zu\n", sizeof(struct scarf_opt));
  printf("scarf_srm_params.size %zu\n", sizeof(scarf_srm_params));
  printf("scarf_srm_setup.size %zu\n", sizeof(scarf_srm_setup));
  P(scarf_srm_setup, m); P(scarf_srm_setup, ier_full);
  P(scarf_tc_tuning, variant); P(scarf_tc_tuning, tile_j); P(scarf_tc_tuning, permute); P(scarf_tc_tuning, ms);
  P(scarf_tc_tuning, split);
  printf("scarf_tc_tuning.size %zu\n", sizeof(scarf_tc_tuning));
  return 0;
}
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", f"-I{INCLUDE}", str(src), "-o", str(exe)], check=True)
    got = dict(ln.split() for ln in subprocess.run([str(exe)], capture_output=True, text=True,
                                                   check=True).stdout.splitlines())
    for fname, _ in sb.ScarfOpt._fields_:
        assert int(got[f"scarf_opt.{fname}"]) == getattr(sb.ScarfOpt, fname).offset, fname
    assert int(got["scarf_opt.size"]) == ctypes.sizeof(sb.ScarfOpt)
    assert int(got["scarf_srm_params.size"]) == ctypes.sizeof(sb.SrmParams)
    assert int(got["scarf_srm_setup.size"]) == ctypes.sizeof(sb.SrmSetup)
    assert int(got["scarf_srm_setup.m"]) == sb.SrmSetup.m.offset
    assert int(got["scarf_srm_setup.ier_full"]) == sb.SrmSetup.ier_full.offset
    for fname, _ in sb.TcTuning._fields_:
        assert int(got[f"scarf_tc_tuning.{fname}"]) == getattr(sb.TcTuning, fname).offset, fname
    assert int(got["scarf_tc_tuning.size"]) == ctypes.sizeof(sb.TcTuning)


def test_cpp_wrapper_compiles(tmp_path):
    src = tmp_path / "w.cpp"
    src.write_text(r"""
#include "scarf3d.h"
#include "scarf3d_b200.h"
int run(float* field, float* stats) {
  const int fs[3] = {1, 1, 1}, fe[3] = {8, 8, 8};
  const float cl[3] = {2000.f, 2000.f, 2000.f};
  Scarf3D::options.hurst = 0.25f;
  Scarf3D::Initialize<srm> S(3, fs, fe, 50.f, 0, cl, 0.05f);
  S.execute(1234, field, stats);
  return scarf_set_nharm(500);
}
""")
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", f"-I{INCLUDE}", str(src)], check=True)


def test_error_paths_without_a_gpu():
    sb.lib.scarf_finalize()
    stats = np.zeros(8, np.float32)
    field = np.zeros(8, np.float32)
    fp = stats.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    assert sb.lib.scarf_execute_ex(1, ctypes.c_void_p(field.ctypes.data), fp, 0) == sb.SCARF_ERR_STATE
    assert "before" in sb.last_error()
    # Both methods reach the device: without one, execute reports a CUDA error.
    for method in (0, 1):
        sb.scarf_initialize(fs=[1, 1, 1], fe=[2, 2, 2], ds=50.0, acf=0, cl=[2000.0] * 3, sigma=0.05, method=method)
        if not HAS_GPU:
            assert sb.lib.scarf_execute_ex(1, ctypes.c_void_p(field.ctypes.data), fp, 0) == sb.SCARF_ERR_CUDA
            assert sb.last_error()
        sb.scarf_finalize()
    assert sb.lib.scarf_set_nharm(0) == sb.SCARF_ERR_ARG
    assert sb.lib.scarf_set_form(7) == sb.SCARF_ERR_ARG
    assert sb.lib.scarf_set_uniform_source(ctypes.c_void_p(1), None) == sb.SCARF_ERR_ARG
    assert sb.lib.scarf_set_host_threads(-1) == sb.SCARF_ERR_ARG
    p = sb.make_params(acf=2, nharm=10, seed=1, ds=50.0, cl=[1.0, 1.0, 1.0], nc=[0, 0, 0], fc=[1, 1, 1])
    s = sb.SrmSetup()
    assert sb.lib.scarf_srm_compute_setup(ctypes.byref(p), ctypes.byref(s)) == sb.SCARF_ERR_UNSUPPORTED
    assert sb.tc_workspace_bytes(3, [0, 4, 4], 10) == 0


def test_nharm_default_is_the_reference_constant():
    # scarflib_srm.f90:90; checked in a fresh process (the setting is global).
    r = subprocess.run([sys.executable, "-c", "import scarf3d_b200 as s; print(s.lib.scarf_get_nharm())"],
                       cwd=str(ROOT), capture_output=True, text=True, check=True)
    assert r.stdout.strip() == "10000"


def test_io_one_writes_raw_column_major_blocks(tmp_path):
    """Two blocks of a 6x4x5 grid written by two 'ranks' assemble the global
    array in Fortran order (scarflib_common.f90:363-399)."""
    glob = np.arange(6 * 4 * 5, dtype=np.float32).reshape((6, 4, 5), order="F")
    fname = str(tmp_path / "field.bin")
    for z0, z1 in ((1, 2), (3, 5)):
        sb.scarf_initialize(fs=[1, 1, z0], fe=[6, 4, z1], ds=50.0, acf=0, cl=[2000.0] * 3, sigma=0.05)
        block = np.asfortranarray(glob[:, :, z0 - 1:z1]).ravel(order="F")
        sb.scarf_io([6, 4, 5], block, fname)
        sb.scarf_finalize()
    back = np.fromfile(fname, np.float32).reshape((6, 4, 5), order="F")
    assert np.array_equal(back, glob)


def test_io_slice_writes_one_plane(tmp_path):
    glob = np.arange(6 * 4 * 5, dtype=np.float32).reshape((6, 4, 5), order="F")
    sb.scarf_initialize(fs=[1, 1, 1], fe=[6, 4, 5], ds=50.0, acf=0, cl=[2000.0] * 3, sigma=0.05)
    flat = glob.ravel(order="F")
    for axis, plane, ref in (("x", 3, glob[2, :, :]), ("y", 2, glob[:, 1, :]), ("z", 5, glob[:, :, 4])):
        fname = str(tmp_path / f"slice_{axis}.bin")
        sb.scarf_io_slice([6, 4, 5], axis, plane, flat, fname)
        back = np.fromfile(fname, np.float32).reshape(ref.shape, order="F")
        assert np.array_equal(back, ref)
    sb.scarf_finalize()


def test_package_refuses_to_load_without_its_library():
    env = dict(os.environ, SCARF3D_B200_LIB="/nonexistent/libscarf3d_b200.so")
    r = subprocess.run([sys.executable, "-c", "import scarf3d_b200"], cwd=str(ROOT), env=env, capture_output=True,
                       text=True)
    assert r.returncode != 0 and "no CPU fallback" in r.stderr


def test_device_memory_cap_and_selftest_arguments_without_a_gpu():
    assert sb.device_memory_in_use() == 0
    sb.set_device_memory_cap(1 << 20)
    sb.set_device_memory_cap(0)
    st = ctypes.c_int(-1)
    waited = ctypes.c_double(-1.0)
    assert sb.lib.scarf_selftest_wait_limit(0, ctypes.byref(st), ctypes.byref(waited)) == sb.SCARF_ERR_ARG
    assert sb.lib.scarf_selftest_wait_limit(2000, None, None) == sb.SCARF_ERR_ARG
    assert "blocks" in sb.last_error()


def test_batch_sampler_output_arrays_are_validated():
    ps = [sb.make_params(nc=[0.0] * 3, fc=[1000.0] * 3, nharm=n, acf=0, seed=1, hurst=0.3, sigma=0.05, ds=50.0,
                         cl=[500.0] * 3) for n in (7, 13)]
    ss = [sb.SrmSetup(), sb.SrmSetup()]
    ro = np.zeros(35, np.float32)
    ro.flags.writeable = False
    for bad in ([np.zeros(35, np.float64), np.zeros(65, np.float32)],  # wrong type
                [np.zeros(30, np.float32), np.zeros(65, np.float32)],  # too small
                [ro, np.zeros(65, np.float32)],                        # read-only
                [np.zeros(35, np.float32)]):                           # one array short
        with pytest.raises(ValueError):
            sb.sample_device_batch(ps, ss, out=bad)


def test_tensor_core_plan_and_workspace_without_a_gpu():
    # 512^3 x 20 000 harmonics, default plan: one CTA, 16 x 8 row tiles, z the
    # column axis in 256-wide tiles; 1 250 stages of 16 harmonics. The R, S
    # and C images are 32 x 16 rows, 64 x 8 rows and 2 x 256 columns (hi and lo
    # halves of 64-byte rows) per stage, 8 bytes per R/S entry: 81.92 MB each,
    # plus 256 bytes of status and queue words.
    assert sb.tc_plan_info(3, [512, 512, 512], 20000) == {"variant": sb.TC_SINGLE, "tile_j": 8, "permute": 0,
                                                          "split": 1}
    stages = 20000 // 16
    image = stages * 16 * 512 * 8
    assert sb.tc_workspace_bytes(3, [512, 512, 512], 20000) == 3 * image + 256
    # one more stage adds one stage of each image
    per_stage = 16 * 512 * 8 * 3
    assert (sb.tc_workspace_bytes(3, [512, 512, 512], 20016) - sb.tc_workspace_bytes(3, [512, 512, 512], 20000)
            == per_stage)
    # 2-D grids keep one row of j per tile (tile_j 1)
    assert sb.tc_plan_info(2, [300, 200, 1], 300)["tile_j"] == 1
