"""Unstructured meshes: the library page-locks the borrowed coordinate arrays
from scarf_nocart_initialize to scarf_finalize (so each execute's upload is an
asynchronous copy beside the sampling) and releases them again; arrays that
share pages are registered as one range, and arrays the caller page-locked
itself are copied as they are, with the same field bit for bit."""
import numpy as np
import pytest

import scarf3d_b200 as sb

torch = pytest.importorskip("torch")
rt = pytest.importorskip("cuda.bindings.runtime")
pytestmark = pytest.mark.gpu

KW = dict(dh=100.0, acf=1, cl=[1500.0, 1500.0, 500.0], sigma=0.1, method=1)
N = 50_000


def _mem_type(a):
    err, attr = rt.cudaPointerGetAttributes(a.ctypes.data)
    assert err == rt.cudaError_t.cudaSuccess
    return attr.type


def _points(seed=3):
    rng = np.random.default_rng(seed)
    return [np.ascontiguousarray(rng.random(N, dtype=np.float32) * L) for L in (20000.0, 20000.0, 10000.0)]


def _run(x, y, z, seed=7):
    sb.set_nharm(800)
    try:
        sb.scarf_initialize(x=x, y=y, z=z, **KW)
        types = [_mem_type(a) for a in (x, y, z)]
        f1, st = sb.scarf_execute(seed)
        f2, _ = sb.scarf_execute(seed)
        assert np.array_equal(f1.view(np.uint32), f2.view(np.uint32))
        return f1.copy(), st.copy(), types
    finally:
        sb.scarf_finalize()
        sb.set_nharm(10000)


def test_coordinates_are_page_locked_for_the_life_of_the_mesh():
    x, y, z = _points()
    assert all(_mem_type(a) == rt.cudaMemoryType.cudaMemoryTypeUnregistered for a in (x, y, z))
    f, st, types = _run(x, y, z)
    assert all(t == rt.cudaMemoryType.cudaMemoryTypeHost for t in types)
    # released at finalize
    assert all(_mem_type(a) == rt.cudaMemoryType.cudaMemoryTypeUnregistered for a in (x, y, z))
    # and a re-initialised mesh over the same arrays gives the same field
    f2, st2, _ = _run(x, y, z)
    assert np.array_equal(f.view(np.uint32), f2.view(np.uint32))
    assert np.array_equal(st[:4], st2[:4])


def test_shared_pages_and_caller_locked_arrays_give_the_same_field():
    x, y, z = _points()
    ref, st_ref, _ = _run(x, y, z)
    # one buffer: the three arrays share pages at their boundaries
    buf = np.concatenate([x, y, z])
    parts = (buf[:N], buf[N:2 * N], buf[2 * N:])
    f, st, types = _run(*parts)
    assert np.array_equal(f.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(st[:4], st_ref[:4])
    assert all(t == rt.cudaMemoryType.cudaMemoryTypeHost for t in types)
    assert all(_mem_type(a) == rt.cudaMemoryType.cudaMemoryTypeUnregistered for a in parts)
    # arrays the caller page-locked itself stay locked after finalize
    pinned = [torch.from_numpy(a.copy()).pin_memory().numpy() for a in (x, y, z)]
    f, st, types = _run(*pinned)
    assert np.array_equal(f.view(np.uint32), ref.view(np.uint32))
    assert all(_mem_type(a) == rt.cudaMemoryType.cudaMemoryTypeHost for a in pinned)
