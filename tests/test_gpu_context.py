"""Library contexts on the GPU: meshes initialised in separate contexts give,
executed in any interleaving and from several threads at once, the same fields
and statistics bit for bit as one after another on the default context."""
import threading

import numpy as np
import pytest

import scarf3d_b200 as sb

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MESHES = [
    dict(fs=[1, 1, 1], fe=[40, 32, 24], ds=50.0, acf=0, cl=[800.0, 800.0, 600.0], sigma=0.05, hurst=0.4),
    dict(fs=[1, 1, 1], fe=[24, 36, 20], ds=40.0, acf=1, cl=[500.0, 700.0, 400.0], sigma=0.1),
    dict(fs=[1, 1, 1], fe=[32, 32, 32], ds=25.0, acf=0, cl=[300.0, 300.0, 300.0], sigma=0.08, hurst=0.7, rescale=1),
]
NHARM = [300, 500, 700]
SEEDS = [11, 22, 33]


def _run_default(m, nh, seed):
    sb.set_nharm(nh)
    try:
        sb.scarf_initialize(method=1, **m)
        f, st = sb.scarf_execute(seed)
        return f.copy(), st.copy()
    finally:
        sb.scarf_finalize()
        sb.set_nharm(10000)


def test_contexts_interleaved_match_the_default_context():
    ref = [_run_default(m, nh, sd) for m, nh, sd in zip(MESHES, NHARM, SEEDS)]
    ctxs = [sb.Context() for _ in MESHES]
    try:
        for c, m, nh in zip(ctxs, MESHES, NHARM):
            with c:
                sb.set_nharm(nh)
                sb.scarf_initialize(method=1, **m)
        for rnd in range(2):
            for i in (2, 0, 1) if rnd else (0, 1, 2):
                with ctxs[i]:
                    f, st = sb.scarf_execute(SEEDS[i])
                assert np.array_equal(f.view(np.uint32), ref[i][0].view(np.uint32))
                assert np.array_equal(st[:4], ref[i][1][:4])
    finally:
        for c in ctxs:
            c.close()


def test_contexts_on_separate_threads():
    ref = [_run_default(m, nh, sd) for m, nh, sd in zip(MESHES, NHARM, SEEDS)]
    out = [None] * len(MESHES)
    errors = []

    def work(i):
        try:
            with sb.Context() as c:
                sb.set_nharm(NHARM[i])
                sb.scarf_initialize(method=1, **MESHES[i])
                res = []
                for _ in range(3):
                    f, st = sb.scarf_execute(SEEDS[i])
                    res.append((f.copy(), st.copy()))
                out[i] = res
            c.close()
        except Exception as e:  # reported on the main thread
            errors.append(e)

    ths = [threading.Thread(target=work, args=(i,)) for i in range(len(MESHES))]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    assert not errors, errors
    for i, res in enumerate(out):
        for f, st in res:
            assert np.array_equal(f.view(np.uint32), ref[i][0].view(np.uint32))
            assert np.array_equal(st[:4], ref[i][1][:4])
