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
    assert r == 1 and b"512" in L.lqg_last_error()
