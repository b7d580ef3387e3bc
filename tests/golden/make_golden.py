"""Generate the golden fixtures of the CPU oracle (tests/golden/*.npz).

The reference cannot be built or run in this environment or on the GPU host
(Fortran + MPI + TRNG4, all absent) and ships no golden vectors, so these
fixtures come from the oracle itself, whose uniform stream follows TRNG's
documented yarn2 seeding and uniform01_dist<> (double draw stored as float). They pin the oracle (setup scalars, harmonic table, FP32 op-order
field, FP64 field, statistics) against unintended changes; the product is
checked against them and against the live oracle.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

HERE = Path(__file__).resolve().parent

# name: structured case (parameters follow the reference's drivers,
# examples/fortran/driver.f90:89-119, at small sizes)
CASES = {
    "vk3d_iso": dict(acf=0, nharm=64, seed=1235, hurst=0.25, sigma=0.05, ds=50.0, cl=[2000.0, 2000.0, 2000.0],
                     fs=[1, 1, 1], fe=[16, 12, 10]),
    "gs3d_aniso": dict(acf=1, nharm=96, seed=7, hurst=0.0, sigma=0.1, ds=100.0, cl=[1500.0, 1500.0, 500.0],
                       fs=[1, 1, 1], fe=[20, 16, 12]),
    "vk3d_rot_offset_dh": dict(acf=0, nharm=80, seed=99, hurst=0.5, sigma=0.05, ds=25.0, dh=10.0,
                               cl=[3000.0, 3000.0, 1000.0], fs=[5, 3, 2], fe=[20, 14, 9], alpha=30.0,
                               beta=-10.0, gamma=5.0),
    "gs2d": dict(acf=1, nharm=64, seed=1235, hurst=0.0, sigma=0.05, ds=250.0, cl=[2000.0, 1200.0], fs=[1, 1],
                 fe=[24, 18], alpha=20.0),
    "vk2d_rescale_taper": dict(acf=0, nharm=64, seed=3, hurst=0.25, sigma=0.05, ds=50.0, cl=[2000.0, 2000.0],
                               fs=[1, 1], fe=[30, 20], rescale=1, poi=[[600.0, 400.0]], mute=100.0, taper=400.0),
}


def build_case(c: dict) -> dict:
    c = dict(c)
    fs, fe = c.pop("fs"), c.pop("fe")
    poi = c.pop("poi", None)
    mute = c.pop("mute", -999.0)
    taper = c.pop("taper", -999.0)
    fs3 = list(fs) + [1] * (3 - len(fs))
    fe3 = list(fe) + [1] * (3 - len(fe))
    n = [fe3[k] - fs3[k] + 1 for k in range(3)]
    p = oracle.structured_params(fs=fs, fe=fe, **c)
    s = oracle.setup(p)
    tab, pairs = oracle.sample(p, s)
    f32 = oracle.sum_structured(s, fs3, n, c["ds"], tab)
    f64 = oracle.sum_structured(s, fs3, n, c["ds"], tab, f64=True)
    field, info = oracle.execute_structured(p, fs3, fe3, poi=poi, mute=mute, taper=taper, nthreads=2)
    setup = np.array([s.kmin, s.kmax, s.kc, s.nu, s.cnst, s.scaling, s.scaling0, *s.m, *s.bar, s.info0, s.info1,
                      s.intg_band, s.intg_full], np.float32)
    return dict(setup=setup, ier=np.array([s.ier_band, s.ier_full], np.int32), table=tab,
                pairs=np.array([pairs], np.int64), field_f32=f32, field_f64=f64, execute_field=field,
                execute_info=info, n=np.array(n, np.int32))


def main():
    for name, c in CASES.items():
        out = build_case(c)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(name, {k: v.shape for k, v in out.items()})
    # Raw uniform stream of the restated generator for two seeds.
    np.savez_compressed(HERE / "uniform_stream.npz", seed1235=oracle.raw_stream(1235, 64),
                        seed_neg7=oracle.raw_stream(-7, 64))


if __name__ == "__main__":
    main()
