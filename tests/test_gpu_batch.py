"""Batched tensor-core form: many fields in one persistent launch (device work
queue), checked field by field against the single-field path and the FP64
oracle, and replayed from a CUDA graph."""
import ctypes

import numpy as np
import pytest

import oracle
import scarf3d_b200 as sb
from conftest import rel_rms
from srm_cases import iarr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SHAPES = [(48, 32, 64), (80, 16, 32), (32, 48, 48), (96, 64, 16), (17, 23, 40), (64, 64, 256), (40, 8, 300),
          (128, 16, 48), (33, 40, 31), (16, 16, 16)]


def _fields(nh_base=120):
    out = []
    for f, n in enumerate(SHAPES):
        acf = f % 2
        # correlation lengths about a quarter of each axis' span keep the
        # rejection sampler's acceptance high for both spectra
        cl = [float(min(2000.0, max(300.0, (m - 1) * 50.0 / (3.5 + 0.2 * f)))) for m in n]
        kw = dict(acf=acf, nharm=nh_base + 37 * f, seed=500 + f, hurst=0.2 + 0.06 * f if acf == 0 else 0.0,
                  sigma=0.05, ds=50.0, cl=cl)
        op = oracle.structured_params(fs=[1, 1, 1], fe=list(n), **kw)
        p = sb.make_params(nc=list(op.nc), fc=list(op.fc), **kw)
        s = sb.compute_setup(p)
        tab, _ = sb.sample(p, s)
        d_tab = torch.from_numpy(tab.reshape(-1).copy()).cuda()
        field = torch.full((int(np.prod(n)),), float("nan"), dtype=torch.float32, device="cuda")
        out.append(dict(n=list(n), fs=[1, 1, 1], ds=50.0, setup=s, tab=tab, d_table=d_tab, field=field, op=op, kw=kw))
    return out


def _entries(fields):
    return [dict(setup=f["setup"], fs=f["fs"], n=f["n"], ds=f["ds"], d_table=f["d_table"].data_ptr(),
                 nh=len(f["tab"]), d_field=f["field"].data_ptr()) for f in fields]


def _alloc(nbytes):
    return torch.empty(nbytes, dtype=torch.uint8, device="cuda")


def _single(f):
    out = torch.empty_like(f["field"])
    wb = sb.tc_workspace_bytes(3, f["n"], len(f["tab"]))
    work = _alloc(wb)
    sb.check(sb.lib.scarf_srm_tc_structured(ctypes.byref(f["setup"]), iarr(f["fs"]), iarr(f["n"]), f["ds"],
                                            ctypes.c_void_p(f["d_table"].data_ptr()), len(f["tab"]),
                                            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(work.data_ptr()),
                                            wb, None))
    return out


def test_batch_matches_single_field_path_and_oracle():
    fields = _fields()
    batch = sb.TcBatch(_entries(fields), _alloc)
    batch.launch()
    batch.wait()
    for f in fields:
        got = f["field"].cpu().numpy()
        assert np.all(np.isfinite(got))
        ref = _single(f).cpu().numpy()
        assert np.array_equal(got, ref)  # same tiles, same arithmetic order
        r64 = oracle.sum_structured(oracle.setup(f["op"]), f["fs"], f["n"], f["ds"], f["tab"], f64=True)
        assert rel_rms(got, r64) <= 1e-5


def test_batch_replays_from_a_cuda_graph():
    fields = _fields(nh_base=80)
    batch = sb.TcBatch(_entries(fields), _alloc)
    batch.launch()
    batch.wait()
    eager = [f["field"].clone() for f in fields]
    for f in fields:
        f["field"].fill_(float("nan"))
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        batch.launch(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        batch.wait()
        for f, e in zip(fields, eager):
            assert torch.equal(f["field"], e)
    del g


def test_batch_copies_fields_to_host_buffers_as_they_complete():
    # Host outputs: wait() copies every field to its page-locked host buffer
    # (field by field as the launch raises its flags), eagerly and from a
    # graph replay, twice in a row; None turns the copy-out off again.
    fields = _fields(nh_base=90)
    batch = sb.TcBatch(_entries(fields), _alloc)
    batch.launch()
    batch.wait()
    ref = [f["field"].cpu().clone() for f in fields]
    hosts = [torch.full((f["field"].numel(),), float("nan"), dtype=torch.float32, pin_memory=True) for f in fields]
    batch.set_host_outputs([h.data_ptr() for h in hosts])
    batch.launch()
    batch.wait()
    for h, r in zip(hosts, ref):
        assert torch.equal(h, r)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        batch.launch(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        for h in hosts:
            h.fill_(float("nan"))
        g.replay()
        batch.wait(torch.cuda.current_stream().cuda_stream)
        for h, r in zip(hosts, ref):
            assert torch.equal(h, r)
    del g
    batch.set_host_outputs(None)
    for h in hosts:
        h.fill_(float("nan"))
    batch.launch()
    batch.wait()
    assert all(torch.isnan(h).all() for h in hosts)


def test_batch_rejects_mixed_row_tiles():
    fields = _fields()[:2]
    entries = _entries(fields)
    entries[1]["tile_j"] = 2
    with pytest.raises(sb.ScarfError):
        sb.TcBatch(entries, _alloc)


def test_batch_of_the_many_realisation_workload_small_harmonics():
    """The 256-field workload's shapes and spectra (harmonics capped at 64 to
    keep the oracle check fast): every field against the FP64 oracle at
    sampled points."""
    from scarf3d_b200.workloads import batched_fields
    spec = batched_fields(count=64, nharm_range=(48, 64))
    fields = []
    for f in spec:
        tab, _ = sb.sample(f["params"], f["setup"])
        fields.append(dict(n=f["n"], fs=[1, 1, 1], ds=f["ds"], setup=f["setup"], tab=tab,
                           d_table=torch.from_numpy(tab.reshape(-1).copy()).cuda(),
                           field=torch.empty(int(np.prod(f["n"])), dtype=torch.float32, device="cuda"),
                           params=f["params"]))
    batch = sb.TcBatch(_entries(fields), _alloc)
    batch.launch()
    batch.wait()
    rng = np.random.default_rng(3)
    for f in fields:
        npts = int(np.prod(f["n"]))
        idx = np.sort(rng.choice(npts, size=min(64, npts), replace=False)).astype(np.int64)
        p = f["params"]
        op = oracle.params(acf=p.acf, nharm=p.nharm, seed=p.seed, hurst=p.hurst, sigma=p.sigma, ds=p.ds,
                           cl=list(p.cl), nc=list(p.nc), fc=list(p.fc))
        r64 = oracle.sum_structured(oracle.setup(op), [1, 1, 1], f["n"], f["ds"], f["tab"], idx=idx, f64=True)
        got = f["field"][torch.from_numpy(idx).cuda()].cpu().numpy()
        fstd = float(f["field"].double().std().item())
        assert np.sqrt(np.mean((got - r64) ** 2)) / fstd <= 1e-5
