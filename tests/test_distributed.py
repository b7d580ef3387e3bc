"""Multi-rank host logic on the CPU (gloo, world size 2): every rank draws the
same harmonics and evaluates its own z-slab; the global statistics are the
Chan merge of the per-rank (variance, mean, count), gathered in rank order."""
import datetime
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from scarf3d_b200.distributed import chan_merge, merge_stats_across_ranks, slab_bounds  # noqa: E402

NX, NY, NZ = 20, 16, 13
KW = dict(acf=0, nharm=150, seed=31, hurst=0.3, sigma=0.05, ds=50.0, cl=[2000.0, 2000.0, 1000.0], alpha=10.0)


# The ranks meet through a file store in the test's own directory: no port
# to pick, so no port another process can take between the pick and the bind.
def _init(rank, world, store, seconds):
    dist.init_process_group("gloo", init_method=f"file://{store}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=seconds))


def _global_corners():
    ds = np.float32(KW["ds"])
    return [0.0, 0.0, 0.0], [float(np.float32(NX - 1) * ds), float(np.float32(NY - 1) * ds),
                             float(np.float32(NZ - 1) * ds)]


def _slab_field(rank, world):
    import oracle
    z0, z1 = slab_bounds(NZ, world, rank)
    fs, fe = [1, 1, z0], [NX, NY, z1]
    nc, fc = _global_corners()
    p = oracle.structured_params(fs=fs, fe=fe, nc=nc, fc=fc, **KW)
    s = oracle.setup(p)
    tab, _ = oracle.sample(p, s)
    n = [fe[c] - fs[c] + 1 for c in range(3)]
    return oracle.sum_structured(s, fs, n, KW["ds"], tab), n


def _worker(rank, world, store, out):
    _init(rank, world, store, 60)
    import oracle
    f, n = _slab_field(rank, world)
    var, mean = oracle.variance(f), oracle.mean(f)
    gv, gm = merge_stats_across_ranks(var, mean, f.size)
    pieces = [torch.zeros(NX * NY * NZ, dtype=torch.float32) for _ in range(world)]
    padded = torch.zeros(NX * NY * NZ, dtype=torch.float32)
    padded[: f.size] = torch.from_numpy(f)
    dist.all_gather(pieces, padded)
    sizes = [NX * NY * (slab_bounds(NZ, world, r)[1] - slab_bounds(NZ, world, r)[0] + 1) for r in range(world)]
    if rank == 0:
        whole = np.concatenate([pieces[r][: sizes[r]].numpy() for r in range(world)])
        out.put((gv, gm, whole))
    dist.barrier()
    dist.destroy_process_group()


def test_slab_bounds_cover_the_axis():
    for nz in (1, 7, 13, 512):
        for world in (1, 2, 3, 8):
            spans = [slab_bounds(nz, world, r) for r in range(world)]
            assert spans[0][0] == 1 and spans[-1][1] == nz
            for a, b in zip(spans, spans[1:]):
                assert b[0] == a[1] + 1


def test_chan_merge_single_set_is_identity():
    v, m = chan_merge([np.float32(0.25)], [np.float32(-0.5)], [1000])
    assert v == np.float32(0.25) and m == np.float32(-0.5)


def test_two_rank_slabs_reproduce_single_rank_field_and_stats(tmp_path):
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    store = str(tmp_path / "store")
    procs = [ctx.Process(target=_worker, args=(r, 2, store, q)) for r in range(2)]
    for p in procs:
        p.start()
    gv, gm, whole = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full, _ = _slab_field(0, 1)
    assert np.array_equal(whole, full)  # decomposition invariance, bit for bit
    assert abs(gv / oracle.variance(full) - 1) < 1e-5
    assert abs(gm - oracle.mean(full)) <= 1e-6 * np.sqrt(gv)


def _leaving_worker(rank, world, store, out):
    # Rank 1 leaves between steps (after the group is up, before the merge);
    # rank 0 must get an error from its next collective, not wait for good.
    import time
    _init(rank, world, store, 5)
    if rank == 1:
        os._exit(0)
    t0 = time.monotonic()
    try:
        merge_stats_across_ranks(1.0, 0.0, 10)
        out.put(("merged", time.monotonic() - t0))
    except Exception as e:  # noqa: BLE001 - any error is the expected outcome
        out.put(("error", time.monotonic() - t0, type(e).__name__))
    os._exit(0)


def test_a_rank_that_leaves_makes_the_merge_fail_instead_of_hang(tmp_path):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    store = str(tmp_path / "store")
    procs = [ctx.Process(target=_leaving_worker, args=(r, 2, store, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == "error", res
    assert res[1] < 60.0  # bounded by the process group's timeout
