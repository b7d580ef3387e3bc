"""Synthetic SRM workloads used by the benchmark and the tests.

batched_fields(): the many-realisation configuration -- fields with grid
axes drawn log-uniformly between 32 and 256 points (each axis independently,
rounded to a multiple of 16), the ACF alternating von Karman (Hurst uniform
0.1-0.9) and Gaussian, correlation lengths uniform 500-5000 m per axis,
harmonic counts uniform 2 000-20 000, distinct seeds, ds = 50 m,
sigma = 0.05, drawn from a fixed meta-seed.

One rule is added to make every field computable: the SRM draws wavenumbers
by rejection in [kmin, kmax] with kmin = 2 pi max(cl / span); when a
correlation length is large against its axis' span (e.g. a Gaussian field
with cl = 5000 m on a 1550 m axis) the acceptance rate of that loop is
astronomically small and the reference's sampler never terminates
(scarflib_srm.f90:731-745). Correlation lengths of such fields are redrawn
until the acceptance rate is at least `min_acceptance`; the redraws come from
the same seeded stream, so the batch is reproducible.
"""
from __future__ import annotations

import math

import numpy as np


def _round16(v: float) -> int:
    return int(max(16, round(v / 16.0) * 16))


def batched_fields(count: int = 256, meta_seed: int = 20240, ds: float = 50.0, sigma: float = 0.05,
                   nharm_range=(2000, 20000), size_range=(32, 256), min_acceptance: float = 1e-4):
    import scarf3d_b200 as sb
    rng = np.random.default_rng(meta_seed)
    lo, hi = math.log(size_range[0]), math.log(size_range[1])
    fields = []
    for f in range(count):
        n = [min(size_range[1], _round16(math.exp(rng.uniform(lo, hi)))) for _ in range(3)]
        acf = f % 2  # alternate von Karman / Gaussian
        hurst = float(rng.uniform(0.1, 0.9)) if acf == 0 else 0.0
        nharm = int(rng.integers(nharm_range[0], nharm_range[1] + 1))
        ds32 = np.float32(ds)
        fc = [float(np.float32(n[c] - 1) * ds32) for c in range(3)]
        for _ in range(1000):
            cl = [float(v) for v in rng.uniform(500.0, 5000.0, size=3)]
            p = sb.make_params(acf=acf, nharm=nharm, seed=1000 + f, hurst=hurst, sigma=sigma, ds=ds, cl=cl,
                               nc=[0.0, 0.0, 0.0], fc=fc)
            s = sb.compute_setup(p)
            acc = s.intg_band * s.cnst / max(s.kmax - s.kmin, 1e-30)
            if acc >= min_acceptance:
                break
        fields.append(dict(n=n, acf=acf, hurst=hurst, cl=cl, sigma=sigma, nharm=nharm, seed=1000 + f, ds=ds,
                           params=p, setup=s))
    return fields


def work_pt_harm(fields) -> float:
    return float(sum(int(np.prod(f["n"])) * f["nharm"] for f in fields))
