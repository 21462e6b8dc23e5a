"""The no-allocation entry point (lqg_search_exact_noalloc) through the C ABI.

It exists for callers that cannot let a library allocate GPU memory (device
memory reserved by another allocator, or loops that must not stall on
cudaMalloc/cudaFree). It must give exactly what lqg_search_exact_device gives
— ids, pools, statistics — on two calls in a row, since every call reuses the
same fixed work array. This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(lib, fn, h, q, m, k, ef, bufs, stream):
    ids, pid, pdd, st = bufs
    for t in bufs:
        t.fill_(0)
    r = fn(h, q.data_ptr(), m, None, k, None, ef, ids.data_ptr(), k, pid.data_ptr(),
           pdd.data_ptr(), ef, st.data_ptr(), stream)
    assert r == 0, lib.lqg_last_error().decode()
    return [t.cpu().numpy().copy() for t in bufs]


@pytest.mark.parametrize("case,ef,k", [("mix128d64", 100, 10), ("bin40", 200, 50), ("u48", 50, 1)])
def test_noalloc_equals_exact_entry_point_on_two_calls(golden, case, ef, k):
    import torch

    import liteqg_b200
    from liteqg_b200._capi import lib

    g = golden[case]
    ix = liteqg_b200.Index("QG", "L2", g["n"], g["dim"], g["deg"])
    ix.load(g["path"])
    q = torch.from_numpy(np.ascontiguousarray(g["queries"])).cuda()
    m = q.shape[0]

    def bufs():
        return (torch.empty((m, k), dtype=torch.int32, device="cuda"),
                torch.empty((m, ef), dtype=torch.int32, device="cuda"),
                torch.empty((m, ef), dtype=torch.float32, device="cuda"),
                torch.empty((m, 4), dtype=torch.int32, device="cuda"))

    stream = torch.cuda.current_stream().cuda_stream
    L = lib()
    want = _run(L, L.lqg_search_exact_device, ix.handle, q, m, k, ef, bufs(), stream)
    assert L.lqg_stream_status(ix.handle, stream) == 0
    for _ in range(2):
        got = _run(L, L.lqg_search_exact_noalloc, ix.handle, q, m, k, ef, bufs(), stream)
        for a, b in zip(got, want):
            assert np.array_equal(a, b)
    # and the reference's own ids, from the golden file
    if (ef, k) in g["expected"]:
        assert np.array_equal(got[0].view(np.uint32), g["expected"][(ef, k)])


def test_noalloc_rejects_ef_beyond_its_work_area(golden):
    import torch

    import liteqg_b200
    from liteqg_b200._capi import lib

    g = golden["u48"]
    ix = liteqg_b200.Index("QG", "L2", g["n"], g["dim"], g["deg"])
    ix.load(g["path"])
    q = torch.from_numpy(np.ascontiguousarray(g["queries"])).cuda()
    ids = torch.empty((q.shape[0], 10), dtype=torch.int32, device="cuda")
    L = lib()
    r = L.lqg_search_exact_noalloc(ix.handle, q.data_ptr(), q.shape[0], None, 10, None, 600,
                                   ids.data_ptr(), 10, None, None, 0, None, None)
    assert r == LQG_ERR_ARG and b"512" in L.lqg_last_error()


LQG_ERR_ARG = 1
LQG_ERR_CAPACITY = 6
NOALLOC_VISITED = 8192  # visited nodes per query the fixed work area holds


def _random_graph_index(tmp_path, n=20000, dim=48, deg=32, seed=11):
    """An index file with random neighbour lists: searches at large ef visit
    most of the graph, so they outgrow the fixed work area."""
    from oracle.oracle import IndexArrays, sq8_quantize, write_index

    rng = np.random.default_rng(seed)
    x = rng.random((n, dim), dtype=np.float32)
    nb = rng.integers(0, n, (n, deg)).astype(np.uint32)
    codes, params = sq8_quantize(x)
    ix = IndexArrays(n, dim, deg, 0, x, nb, codes, params)
    path = str(tmp_path / "random_graph.idx")
    write_index(path, ix)
    return path, ix, rng.random((16, dim), dtype=np.float32)


def test_noalloc_overflow_is_reported_per_query(tmp_path):
    """A query that needs more than the fixed work area gets LQG_NO_ID and the
    call returns LQG_ERR_CAPACITY; every other query of the same batch (a
    per-query ef array: small and large ef mixed) equals
    lqg_search_exact_device, whose allocated work area holds them all."""
    import torch

    import liteqg_b200
    from liteqg_b200._capi import lib
    from oracle.oracle import Oracle

    path, arrays, qh = _random_graph_index(tmp_path)
    m, k = qh.shape[0], 10
    efq = np.array([512, 16] * (m // 2), dtype=np.uint32)
    want_or = Oracle(arrays).search(qh, k, efq.astype(np.int32))
    visited = want_or.evals.astype(np.int64) + 1  # the entry point and every evaluated node
    assert visited.max() > NOALLOC_VISITED and visited.min() < NOALLOC_VISITED // 2
    ix = liteqg_b200.Index("QG", "L2", arrays.n, arrays.dim, arrays.deg)
    ix.load(path)
    q = torch.from_numpy(qh).cuda()
    e_dev = torch.from_numpy(efq.view(np.int32)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    L = lib()

    def call(fn):
        ids = torch.zeros((m, k), dtype=torch.int32, device="cuda")
        r = fn(ix.handle, q.data_ptr(), m, None, k, e_dev.data_ptr(), 512, ids.data_ptr(), k,
               None, None, 0, None, stream)
        return r, ids.cpu().numpy().view(np.uint32)

    r0, want = call(L.lqg_search_exact_device)
    assert r0 == 0 and L.lqg_stream_status(ix.handle, stream) == 0, L.lqg_last_error()
    assert np.array_equal(want, want_or.compat)
    for _ in range(2):
        r, got = call(L.lqg_search_exact_noalloc)
        assert r == LQG_ERR_CAPACITY, L.lqg_last_error()
        over = visited > NOALLOC_VISITED
        fits = visited <= NOALLOC_VISITED - 64
        assert (got[over] == 0xFFFFFFFF).all()
        assert np.array_equal(got[fits], want[fits])
        assert fits.sum() + over.sum() == m
