"""Decomposition invariance of the product on one GPU: the multi-rank SRM.

The reference splits a grid over MPI ranks; every rank seeds the generator
alike and draws the same harmonics (scarflib_srm.f90:627-628), takes the
global extent from an allreduce (:641-642) and evaluates its own block; the
statistics of the blocks are merged with Chan's formula after an allgather
(:887-892, scarflib_common.f90:823-875). Here each "rank" is one
scarf_execute over a z-slab with the global nc/fc, run one after another on
the same GPU; the slabs, concatenated, must give the whole-grid field (bit for
bit with the direct sum, within 1e-6 with the tensor-core form, whose per-axis
phase tables are rebuilt from the slab's own offset), and the Chan merge of
the slabs' (variance, mean, count) must give the whole grid's statistics --
the route multi-GPU runs take (scarf3d_b200.distributed).
"""
import numpy as np
import pytest

import scarf3d_b200 as sb
from conftest import rel_rms
from scarf3d_b200.distributed import chan_merge

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

N = [48, 40, 36]
DS = 50.0
KW = dict(acf=0, hurst=0.25, sigma=0.05, cl=[2000.0, 1500.0, 1000.0])


@pytest.fixture(autouse=True)
def _reset():
    sb.set_nharm(400)
    yield
    sb.scarf_finalize()
    sb.set_nharm(10000)
    sb.set_form(sb.FORM_AUTO)


def _global_extent():
    ds32 = np.float32(DS)
    nc = np.zeros(3, np.float32)
    fc = np.array([np.float32(n - 1) * ds32 for n in N], np.float32)
    return nc, fc


def _execute(fs, fe, seed=1235, alpha=0.0):
    nc, fc = _global_extent()
    sb.scarf_initialize(fs=fs, fe=fe, ds=DS, method=1, nc=nc, fc=fc, alpha=alpha, **KW)
    n = [e - s + 1 for s, e in zip(fs, fe)]
    dev = torch.empty(int(np.prod(n)), dtype=torch.float32, device="cuda")
    try:
        _, stats = sb.scarf_execute(seed, dev)
    finally:
        sb.scarf_finalize()
    return dev.cpu().numpy(), stats.copy()


@pytest.mark.parametrize("form", [sb.FORM_DIRECT, sb.FORM_TC])
@pytest.mark.parametrize("cuts", [[18], [17], [12, 24], [5, 21, 30]])
@pytest.mark.parametrize("alpha", [0.0, 30.0])
def test_z_slabs_reassemble_the_whole_grid(form, cuts, alpha):
    sb.set_form(form)
    whole, wstats = _execute([1, 1, 1], N, alpha=alpha)
    bounds = [1] + [c + 1 for c in cuts] + [N[2] + 1]
    parts, var, mean, cnt = [], [], [], []
    for z0, z1 in zip(bounds[:-1], bounds[1:]):
        f, st = _execute([1, 1, z0], [N[0], N[1], z1 - 1], alpha=alpha)
        parts.append(f)
        var.append(np.float32(st[2]) ** 2)
        mean.append(st[3])
        cnt.append(f.size)
        assert st[0] == wstats[0] and st[1] == wstats[1]  # domain flags come from the global extent
    joined = np.concatenate(parts)  # z is the slowest axis: slabs follow one another
    assert joined.shape == whole.shape
    if form == sb.FORM_DIRECT:
        assert np.array_equal(joined.view(np.uint32), whole.view(np.uint32))
    else:
        assert rel_rms(joined, whole) <= 1e-6
    mvar, mmean = chan_merge(var, mean, cnt)
    wvar = float(np.float32(wstats[2]) ** 2)
    assert abs(mvar / wvar - 1.0) <= 2e-6
    assert abs(mmean - float(wstats[3])) <= 2e-6 * float(wstats[2])
