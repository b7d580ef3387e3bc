"""The reference's Fortran BIND(C) layer (src/f_binding.f90) as a shim over the
library: the six routine names are exported, a C program written against
them (arguments by reference, optional ones as NULL pointers, fields as the
address of the caller's pointer, as src/c_binding.c calls them) links, and on
a GPU it produces exactly the field the library's own API produces."""
import importlib.util
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "scarf3d_b200"

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
typedef float real;
void struct_initialize(const int *nd, const int *fs, const int *fe, const real *ds, const int *acf, const real *cl,
                       const real *sigma, const int *method, const real *hurst, const real *dh, real **poi,
                       const int *np, const real *mute, const real *taper, const int *rescale, const int *pad,
                       const real *nc, const real *fc, const real *alpha, const real *beta, const real *gamma);
void execute(const int *seed, real **field, real *stats);
void finalize(void);
void io_one(const int *nd, const int *npts, real **field, const char *fout, const int *nwriters);
int main(int argc, char **argv) {
  const int nd = 3, fs[3] = {1, 1, 1}, fe[3] = {40, 32, 24}, acf = 0, method = 1, seed = 77;
  const real ds = 50.0f, cl[3] = {1500.0f, 1500.0f, 1000.0f}, sigma = 0.05f, hurst = 0.4f, alpha = 20.0f;
  struct_initialize(&nd, fs, fe, &ds, &acf, cl, &sigma, &method, &hurst, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                    NULL, NULL, &alpha, NULL, NULL);
  real *field = (real *)malloc(sizeof(real) * 40 * 32 * 24), stats[8];
  execute(&seed, &field, stats);
  const int npts[3] = {40, 32, 24};
  io_one(&nd, npts, &field, argv[1], NULL);
  printf("%.9g %.9g\n", stats[2], stats[3]);
  finalize();
  free(field);
  return 0;
}
"""


@pytest.fixture(scope="module")
def shim():
    spec = importlib.util.spec_from_file_location("scarf3d_b200_build", PKG / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    if not b.LIB.exists():
        pytest.skip("library not built")
    return b.build_fbind()


@pytest.fixture(scope="module")
def program(shim, tmp_path_factory):
    d = tmp_path_factory.mktemp("fbind")
    src = d / "prog.c"
    src.write_text(PROGRAM)
    exe = d / "prog"
    subprocess.run(["gcc", "-std=c11", str(src), f"-L{PKG}", "-lscarf3d_b200_fbind", "-lscarf3d_b200",
                    f"-Wl,-rpath,{PKG}", "-o", str(exe)], check=True)
    return exe


def test_shim_exports_the_fortran_binding_names(shim):
    out = subprocess.run(["nm", "-D", "--defined-only", str(shim)], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert {"struct_initialize", "unstruct_initialize", "execute", "finalize", "io_one", "io_slice"} <= exported


def test_c_program_links_against_the_shim(program):
    assert program.exists()


@pytest.mark.gpu
def test_c_program_through_the_shim_matches_the_library(program, tmp_path):
    import scarf3d_b200 as sb
    out = tmp_path / "field.bin"
    r = subprocess.run([str(program), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.fromfile(out, dtype=np.float32)
    std, mean = (float(v) for v in r.stdout.split())
    sb.scarf_initialize(fs=[1, 1, 1], fe=[40, 32, 24], ds=50.0, acf=0, cl=[1500.0, 1500.0, 1000.0], sigma=0.05,
                        method=1, hurst=0.4, alpha=20.0)
    try:
        ref, stats = sb.scarf_execute(77)
    finally:
        sb.scarf_finalize()
    assert np.array_equal(got.view(np.uint32), np.asarray(ref, np.float32).view(np.uint32))
    assert std == pytest.approx(float(stats[2]), rel=1e-6) and mean == pytest.approx(float(stats[3]), rel=1e-6,
                                                                                    abs=1e-9)
