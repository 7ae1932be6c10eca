"""hdb_sort_edges_noalloc: the MST edge sort for callers that cannot allocate
device memory (a host framework that owns every device byte, or a device that
is already full).  It must give exactly what the reference's stable sort by
weight gives (the oracle's sort_edges) and what hdb_sort_edges gives, call
after call, although all calls share one static scratch array -- and a call
must not allocate.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_EDGES = 1 << 18


def _edges(m, seed):
    rng = np.random.default_rng(seed)
    e = np.zeros((m, 3), np.int32)
    e[:, 0] = np.arange(m)
    e[:, 1] = rng.integers(0, 1 << 20, m)
    w = (rng.integers(0, 400, m).astype(np.float32) / 13.0)  # many equal weights
    w[rng.integers(0, m, 50)] = -0.0  # -0.0 and +0.0 are equal weights
    w[rng.integers(0, m, 50)] = 0.0
    e[:, 2] = w.view(np.int32)
    return e


def test_noalloc_sort_matches_the_reference_sort_twice_in_a_row(oracle):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpu_hdbscan_b200 import Context, _lib
    L = _lib.load()
    ctx = Context(0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # warm-up: m = 0 places the static array on the device and sorts nothing;
    # a small sort then loads the sort's kernels (lazy module loading)
    assert L.hdb_sort_edges_noalloc(None, 0, stream) == _lib.HDB_OK, L.hdb_last_error()
    w = torch.from_numpy(_edges(1000, 0)).cuda()
    assert L.hdb_sort_edges_noalloc(C.c_void_p(w.data_ptr()), 1000, stream) == _lib.HDB_OK
    for seed, m in ((1, 200_000), (2, 150_001)):  # the second call sees the first's leftovers
        e = _edges(m, seed)
        want = oracle.sort_edges(e.copy().view(oracle.MST_EDGE).reshape(-1))
        ref = torch.from_numpy(e.copy()).cuda()
        ctx.sort_edges(ref)
        got = torch.from_numpy(e.copy()).cuda()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        alloc0 = torch.cuda.memory_allocated()
        st = L.hdb_sort_edges_noalloc(C.c_void_p(got.data_ptr()), m, stream)
        torch.cuda.synchronize()
        assert st == _lib.HDB_OK, L.hdb_last_error()
        # the call allocated nothing: neither torch's pool nor the device saw a change
        assert torch.cuda.mem_get_info()[0] == free0
        assert torch.cuda.memory_allocated() == alloc0
        g = got.cpu().numpy()
        np.testing.assert_array_equal(g, want.view(np.int32).reshape(-1, 3))  # bit for bit
        np.testing.assert_array_equal(g, ref.cpu().numpy())
    ctx.close()


def test_noalloc_sort_rejects_more_than_its_static_limit():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpu_hdbscan_b200 import _lib
    L = _lib.load()
    buf = torch.zeros((MAX_EDGES + 1, 3), dtype=torch.int32, device="cuda")
    st = L.hdb_sort_edges_noalloc(C.c_void_p(buf.data_ptr()), MAX_EDGES + 1, None)
    assert st == _lib.HDB_ERR_ARG
    assert b"262144" in L.hdb_last_error()
    assert L.hdb_sort_edges_noalloc(None, 0, None) == _lib.HDB_OK
