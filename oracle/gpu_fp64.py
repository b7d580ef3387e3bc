"""FP64 evaluation of the SRM sum on the GPU: a full-field checker.

TEST INFRASTRUCTURE ONLY, like the CPU oracle beside it: imported by tests/
and by bench.py's accuracy legs (outside every timed region), always as the
checker, never as the product path. It evaluates the same sum as the CPU FP64
oracle (orc_sum_structured_f64 / orc_sum_points_f64, which follow
scarflib_srm.f90:794-809 and :397-406 with normalisation :843-851) over the
same FP32 harmonic table, every operation in FP64, through torch on the GPU
so that whole fields of 1e8-1e9 points can be compared point by point where
the CPU oracle would take hours. The tests pin it against the CPU FP64 oracle
(agreement ~1e-12 relative).

Structured grids use the factorisation of the phase, exact in real
arithmetic: with P = M x + bar (M, bar: the setup's FP32 rotation and offset,
promoted), v . P = kx x + ky y + kz z + c where k_c = sum_r v_r M[r][c] and
c = sum_r v_r bar_r, so

    a sin(v.P) + b cos(v.P) = Re[(b - i a) e^{i(kx x + c)} e^{i ky y} e^{i kz z}],

and a block of rows (i, j) against every column k is one FP64 real GEMM of
K = 2 nh (cuBLAS DGEMM). Phases are formed in FP64 from FP64 coordinates
(i + fs - 2) ds. Unstructured sets are summed directly in FP64 (sin, cos of
the FP64 phase per point and harmonic).
"""
from __future__ import annotations

import math

import numpy as np


def _torch():
    import torch
    return torch


def _setup_arrays(setup):
    m = np.asarray(list(setup.m), np.float64).reshape(3, 3)
    bar = np.asarray(list(setup.bar), np.float64)
    return m, bar, float(setup.scaling)


def _wavenumbers(tab, m, bar, device):
    """(kx, ky, kz, c, a, b) in FP64 on the device from the FP32 table."""
    torch = _torch()
    t = torch.as_tensor(np.ascontiguousarray(np.asarray(tab, np.float32).reshape(-1, 5)), device=device)
    t = t.to(torch.float64)
    v = t[:, 0:3]
    mm = torch.as_tensor(m, device=device)
    k = v @ mm                        # k[:, c] = sum_r v_r M[r][c]
    c = v @ torch.as_tensor(bar, device=device)
    return k[:, 0], k[:, 1], k[:, 2], c, t[:, 3], t[:, 4]


class _Stats:
    """Running FP64 sums for rel-RMS (normalised by the reference's std) and max-abs."""

    def __init__(self):
        self.n = 0
        self.sd2 = 0.0
        self.sr = 0.0
        self.sr2 = 0.0
        self.maxabs = 0.0

    def add(self, got, ref):
        torch = _torch()
        d = got.to(torch.float64) - ref
        self.n += ref.numel()
        self.sd2 += float((d * d).sum())
        self.sr += float(ref.sum())
        self.sr2 += float((ref * ref).sum())
        self.maxabs = max(self.maxabs, float(d.abs().max()))

    def result(self):
        mean = self.sr / self.n
        var = max(self.sr2 / self.n - mean * mean, 0.0)
        std = math.sqrt(var)
        return {"rel_rms": math.sqrt(self.sd2 / self.n) / std, "max_abs": self.maxabs, "std_ref": std,
                "mean_ref": mean, "points": self.n}


def _structured_blocks(setup, fs, n, ds, tab, device, budget_bytes):
    """Yield (k0, k1, j0, j1, block) with block[k - k0, j - j0, i] the FP64
    field (scaled) of rows j0..j1-1 of every x at columns k0..k1-1, covering
    the whole grid; column axis z (3-D) or y (2-D: one z plane)."""
    torch = _torch()
    m, bar, scaling = _setup_arrays(setup)
    kx, ky, kz, c, a, b = _wavenumbers(tab, m, bar, device)
    nh = kx.numel()
    f64 = torch.float64
    ax = [(torch.arange(n[d], device=device, dtype=f64) + float(fs[d] - 1)) * float(ds) for d in range(3)]
    # x factor with the amplitude and constant phase: (b - i a) e^{i(kx x + c)}
    th = kx[:, None] * ax[0][None, :] + c[:, None]
    cx, sx = torch.cos(th), torch.sin(th)
    xr = b[:, None] * cx + a[:, None] * sx
    xi = b[:, None] * sx - a[:, None] * cx
    del th, cx, sx
    th = ky[:, None] * ax[1][None, :]
    yr, yi = torch.cos(th), torch.sin(th)
    th = kz[:, None] * ax[2][None, :]
    zr, zi = torch.cos(th), torch.sin(th)
    del th
    # columns: z (nz) against rows (j, i); B = [Re Z; -Im Z] of shape (2 nh, nz)
    bmat = torch.cat([zr, -zi], 0)
    nx, ny, nz = n
    per_row = 2 * nh * nx * 8 * 3  # P (re, im) and its K-major copy
    nj = max(1, min(ny, budget_bytes // max(per_row, 1)))
    for j0 in range(0, ny, nj):
        j1 = min(ny, j0 + nj)
        pr = xr[:, None, :] * yr[:, j0:j1, None] - xi[:, None, :] * yi[:, j0:j1, None]
        pi = xr[:, None, :] * yi[:, j0:j1, None] + xi[:, None, :] * yr[:, j0:j1, None]
        amat = torch.cat([pr.reshape(nh, -1), pi.reshape(nh, -1)], 0)  # (2 nh, nj*nx)
        del pr, pi
        f = (amat.t() @ bmat) * scaling   # ((j,i), k)
        del amat
        yield j0, j1, f.t().reshape(nz, j1 - j0, nx)


def structured_field(setup, fs, n, ds, tab, device="cuda", budget_bytes=2 << 30):
    """The whole FP64 field, Fortran order (x fastest), as a device tensor."""
    torch = _torch()
    out = torch.empty((n[2], n[1], n[0]), dtype=torch.float64, device=device)
    for j0, j1, blk in _structured_blocks(setup, fs, n, ds, tab, device, budget_bytes):
        out[:, j0:j1, :] = blk
    return out.reshape(-1)


def compare_structured(field, setup, fs, n, ds, tab, budget_bytes=2 << 30):
    """rel-RMS (by the FP64 field's std) and max-abs of `field` (a device
    tensor of n0*n1*n2 FP32 values, x fastest) against the FP64 sum, block by
    block without holding the FP64 field."""
    torch = _torch()
    fv = field.reshape(n[2], n[1], n[0])
    st = _Stats()
    with torch.no_grad():
        for j0, j1, blk in _structured_blocks(setup, fs, n, ds, tab, field.device, budget_bytes):
            st.add(fv[:, j0:j1, :], blk)
    return st.result()


def _points_blocks(setup, x, y, z, tab, device, chunk):
    torch = _torch()
    m, bar, scaling = _setup_arrays(setup)
    kx, ky, kz, c, a, b = _wavenumbers(tab, m, bar, device)
    kmat = torch.stack([kx, ky, kz, c], 0)  # (4, nh)
    f64 = torch.float64
    npts = int(x.numel())
    for p0 in range(0, npts, chunk):
        p1 = min(npts, p0 + chunk)
        P = torch.stack([x[p0:p1].to(f64), y[p0:p1].to(f64), z[p0:p1].to(f64),
                         torch.ones(p1 - p0, dtype=f64, device=device)], 1)
        arg = P @ kmat
        f = (torch.sin(arg) @ a + torch.cos(arg) @ b) * scaling
        yield p0, p1, f


def points_field(setup, x, y, z, tab, chunk=8192):
    """FP64 field at the points x, y, z (device FP32 tensors)."""
    torch = _torch()
    out = torch.empty(int(x.numel()), dtype=torch.float64, device=x.device)
    with torch.no_grad():
        for p0, p1, f in _points_blocks(setup, x, y, z, tab, x.device, chunk):
            out[p0:p1] = f
    return out


def compare_points(field, setup, x, y, z, tab, chunk=8192):
    torch = _torch()
    st = _Stats()
    with torch.no_grad():
        for p0, p1, f in _points_blocks(setup, x, y, z, tab, x.device, chunk):
            st.add(field[p0:p1], f)
    return st.result()
