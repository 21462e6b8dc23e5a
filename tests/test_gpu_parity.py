"""GPU parity: the B200 kernels against the reference's outputs and the oracle.

Every search here goes through the C ABI (liblqg.so) via liteqg_b200.Index.
The bar is bit-exact: ids equal, FP32 pool distances equal, and the exact
kernel's pops/evaluations equal the oracle's.
"""
import numpy as np
import pytest

from oracle.oracle import SENTINEL, IndexArrays, Oracle, read_index, write_index

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lqg():
    import liteqg_b200

    return liteqg_b200


def open_index(lqg, g):
    """An index on the fast kernel's path (tuning mode 1: fast kernel, heap
    kernel for tied queries, exact kernel for capacity spills)."""
    ix = lqg.Index("QG", "L2", g["n"], g["dim"], g["deg"])
    ix.load(g["path"])
    ix.set_tuning(mode=1, lanes_per_cand=4, heap_scap=1024)
    return ix


def test_golden_plain_single_query(lqg, golden):
    """Index.search(query, k) one query per call == the reference, every (ef, k)."""
    for name, g in golden.items():
        ix = open_index(lqg, g)
        for (ef, k), want in g["expected"].items():
            ix.set_ef(ef)
            got = np.stack([ix.search(q, k) for q in g["queries"]])
            assert got.dtype == np.uint32
            assert np.array_equal(got, want), (name, ef, k)


def test_golden_batched(lqg, golden):
    for name, g in golden.items():
        ix = open_index(lqg, g)
        for (ef, k), want in g["expected"].items():
            ix.set_ef(ef)
            got = ix.search(g["queries"], k)
            assert np.array_equal(got, want), (name, ef, k)


def _oracle_for(g):
    return Oracle(read_index(g["path"], g["n"], g["dim"], g["deg"]))


def test_pool_distances_and_counts_bit_exact(lqg, golden):
    """Full pools (ids, FP32 distances) and pops equal the oracle's."""
    for name, g in golden.items():
        ix = open_index(lqg, g)
        o = _oracle_for(g)
        for ef in (10, 33, 100, 200):
            want = o.search(g["queries"], 10, ef)
            ids, (pid, pd), st = ix.search(g["queries"], 10, ef=ef, return_pool=True,
                                           return_stats=True)
            assert np.array_equal(ids, want.compat), (name, ef)
            for i in range(len(ids)):
                p = want.pool_n[i]
                assert st[i, 3] == p
                assert np.array_equal(pid[i, :p], want.pool_ids[i, :p]), (name, ef, i)
                assert np.array_equal(pd[i, :p], want.pool_d[i, :p]), (name, ef, i)
                assert (pid[i, p:] == SENTINEL).all()
                assert st[i, 0] == want.pops[i], (name, ef, i)
                if st[i, 2] == 2:  # global exact kernel: the reference's evaluation count
                    assert st[i, 1] == want.evals[i]
                else:  # fast/heap kernels may re-evaluate forgotten nodes, never fewer
                    assert st[i, 1] >= want.evals[i] + 1


def test_tie_heavy_case_goes_through_exact_kernel(lqg, golden):
    g = golden["bin40"]
    ix = open_index(lqg, g)
    ids, st = ix.search(g["queries"], 10, ef=100, return_stats=True)
    assert (st[:, 2] >= 1).sum() > len(ids) // 2
    assert np.array_equal(ids, g["expected"][(100, 10)])


def _device(lqg, ix, g, exact, ef, k, kq=None, efq=None):
    import torch

    q = torch.from_numpy(np.ascontiguousarray(g["queries"])).cuda()
    m = q.shape[0]
    ids = torch.full((m, k), -1, dtype=torch.int32, device="cuda")
    pstride = ef
    pid = torch.full((m, pstride), -1, dtype=torch.int32, device="cuda")
    pdd = torch.full((m, pstride), float("inf"), dtype=torch.float32, device="cuda")
    st = torch.zeros((m, 4), dtype=torch.int32, device="cuda")
    kt = torch.from_numpy(kq).cuda() if kq is not None else None
    et = torch.from_numpy(efq).cuda() if efq is not None else None
    s = torch.cuda.current_stream()
    ix.search_device(q.data_ptr(), m, k, ids.data_ptr(), k, ef=ef,
                     ef_ptr=et.data_ptr() if et is not None else 0,
                     k_ptr=kt.data_ptr() if kt is not None else 0,
                     pool_ids_ptr=pid.data_ptr(), pool_d_ptr=pdd.data_ptr(), pstride=pstride,
                     stats_ptr=st.data_ptr(), stream=s.cuda_stream, exact=exact)
    ix.stream_status(s.cuda_stream)
    v = lambda t: t.cpu().numpy().view(np.uint32) if t.dtype == torch.int32 else t.cpu().numpy()
    return v(ids), v(pid), v(pdd), v(st)


def test_exact_kernel_alone_matches_oracle(lqg, golden):
    for name, g in golden.items():
        ix = open_index(lqg, g)
        o = _oracle_for(g)
        want = o.search(g["queries"], 50, 100)
        ids, pid, pd, st = _device(lqg, ix, g, True, 100, 50)
        assert np.array_equal(ids, want.compat), name
        assert np.array_equal(st[:, 0], want.pops) and np.array_equal(st[:, 1], want.evals)
        assert (st[:, 2] == 2).all()
        for i in range(len(ids)):
            p = want.pool_n[i]
            assert np.array_equal(pid[i, :p], want.pool_ids[i, :p])
            assert np.array_equal(pd[i, :p], want.pool_d[i, :p])


def test_uneven_batch_per_query_ef_and_k(lqg, golden):
    rng = np.random.default_rng(5)
    for name, g in golden.items():
        ix = open_index(lqg, g)
        o = _oracle_for(g)
        m = len(g["queries"])
        efq = rng.choice([1, 7, 32, 64, 100, 256, 512], size=m).astype(np.uint32)
        kq = rng.choice([1, 10, 100], size=m).astype(np.uint32)
        ids, pid, pd, st = _device(lqg, ix, g, False, 512, 100, kq=kq, efq=efq)
        want = o.search(g["queries"], kq.astype(np.int32), efq.astype(np.int32))
        for i in range(m):
            k = int(kq[i])
            assert np.array_equal(ids[i, :k], want.compat[i, :k]), (name, i, efq[i], k)


@pytest.mark.parametrize("g_lanes", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("vbits", [8, 13])
def test_tuning_does_not_change_results(lqg, golden, g_lanes, vbits):
    g = golden["mix128d64"]
    ix = open_index(lqg, g)
    ix.set_tuning(lanes_per_cand=g_lanes, visited_bits=vbits, warps_per_block=4)
    for ef, k in ((50, 10), (200, 50)):
        ix.set_ef(ef)
        assert np.array_equal(ix.search(g["queries"], k), g["expected"][(ef, k)])


def _knn_graph(x, deg):
    sq = (x.astype(np.float64) ** 2).sum(1)
    n = len(x)
    nb = np.empty((n, deg), np.uint32)
    for s in range(0, n, 2048):
        d = sq[s:s + 2048, None] + sq[None, :] - 2 * x[s:s + 2048].astype(np.float64) @ x.T.astype(np.float64)
        d[np.arange(d.shape[0]), np.arange(s, s + d.shape[0])] = np.inf
        nb[s:s + 2048] = np.argpartition(d, deg, axis=1)[:, :deg]
    return nb


@pytest.mark.parametrize("dim,deg", [(128, 32), (96, 64), (40, 32)])
def test_larger_index_matches_oracle(lqg, tmp_path, dim, deg):
    """12k nodes, exact-kNN graph, 400 queries, ef up to 256, k up to 100."""
    from oracle.oracle import sq8_quantize

    rng = np.random.default_rng(dim)
    n = 12000
    cent = rng.uniform(0, 255, (64, dim))
    x = np.clip(np.rint(cent[rng.integers(0, 64, n)] + rng.normal(0, 20, (n, dim))), 0, 255).astype(np.float32)
    codes, params = sq8_quantize(x, 2)
    arr = IndexArrays(n, dim, deg, int(rng.integers(0, n)), x, _knn_graph(x, deg), codes, params)
    path = str(tmp_path / "big.idx")
    write_index(path, arr)
    ix = lqg.Index("QG", "L2", n, dim, deg)
    ix.load(path)
    ix.set_tuning(mode=1, lanes_per_cand=4, heap_scap=1024)
    o = Oracle(arr)
    q = np.clip(np.rint(cent[rng.integers(0, 64, 400)] + rng.normal(0, 20, (400, dim))), 0, 255).astype(np.float32)
    for ef, k in ((64, 10), (128, 100), (256, 10)):
        want = o.search(q, k, ef)
        got, (pid, pd) = ix.search(q, k, ef=ef, return_pool=True)
        assert np.array_equal(got, want.compat), (ef, k)
        assert np.array_equal(pd, want.pool_d), (ef, k)


def test_error_paths(lqg, golden, tmp_path):
    g = golden["u48"]
    ix = lqg.Index("QG", "L2", g["n"], g["dim"], g["deg"])
    with pytest.raises(lqg.symphonyqg.LqgError, match="LQG_ERR_STATE"):
        ix.search(g["queries"][0], 10)
    bad = tmp_path / "short.idx"
    bad.write_bytes(open(g["path"], "rb").read()[:-3])
    with pytest.raises(lqg.symphonyqg.LqgError, match="LQG_ERR_IO"):
        ix.load(str(bad))
    arr = read_index(g["path"], g["n"], g["dim"], g["deg"])
    arr.nbrs[5, 3] = g["n"] + 7
    p = str(tmp_path / "corrupt.idx")
    write_index(p, arr)
    with pytest.raises(lqg.symphonyqg.LqgError, match="LQG_ERR_CORRUPT"):
        ix.load(p)
    ix.load(g["path"])
    with pytest.raises(lqg.symphonyqg.LqgError, match="LQG_ERR_STATE"):
        ix.search(g["queries"][0], 10)
    ix.set_ef(20)
    assert np.array_equal(ix.search(g["queries"][0], 10), g["expected"][(20, 10)][0])
    with pytest.raises(lqg.symphonyqg.LqgError, match="LQG_ERR_ARG"):
        ix.set_ef(513)


def test_save_roundtrip_bytes(lqg, golden, tmp_path):
    g = golden["mix128d64"]
    ix = open_index(lqg, g)
    p = str(tmp_path / "s.idx")
    ix.save(p)
    assert open(p, "rb").read() == open(g["path"], "rb").read()


@pytest.mark.parametrize("mode,scap", [(2, 1024), (2, 256), (1, 256)])
def test_heap_kernel_modes_match_reference(lqg, golden, mode, scap):
    """mode 2: the heap kernel runs every query; scap 256 forces spills to the
    global exact kernel. All paths give the reference's ids and pools."""
    for name, g in golden.items():
        ix = open_index(lqg, g)
        ix.set_tuning(mode=mode, heap_scap=scap)
        o = _oracle_for(g)
        for (ef, k), want in g["expected"].items():
            ix.set_ef(ef)
            got, (pid, pd), st = ix.search(g["queries"], k, ef=ef, return_pool=True,
                                           return_stats=True)
            assert np.array_equal(got, want), (name, ef, k, mode, scap)
            if k == 10:
                w = o.search(g["queries"], k, ef)
                assert np.array_equal(pd, w.pool_d) and np.array_equal(st[:, 0], w.pops)
        if mode == 2:
            assert (st[:, 2] >= 1).all()


@pytest.mark.parametrize("dim,deg", [(128, 32), (96, 64)])
def test_heap_kernel_larger_index(lqg, tmp_path, dim, deg):
    from oracle.oracle import sq8_quantize

    rng = np.random.default_rng(dim + 1)
    n = 12000
    cent = rng.uniform(0, 255, (64, dim))
    x = np.clip(np.rint(cent[rng.integers(0, 64, n)] + rng.normal(0, 20, (n, dim))), 0, 255).astype(np.float32)
    codes, params = sq8_quantize(x, 2)
    arr = IndexArrays(n, dim, deg, int(rng.integers(0, n)), x, _knn_graph(x, deg), codes, params)
    path = str(tmp_path / "big.idx")
    write_index(path, arr)
    ix = lqg.Index("QG", "L2", n, dim, deg)
    ix.load(path)
    ix.set_tuning(mode=2)
    o = Oracle(arr)
    q = np.clip(np.rint(cent[rng.integers(0, 64, 300)] + rng.normal(0, 20, (300, dim))), 0, 255).astype(np.float32)
    for ef, k in ((64, 10), (256, 100), (512, 10)):
        want = o.search(q, k, ef)
        got, (pid, pd) = ix.search(q, k, ef=ef, return_pool=True)
        assert np.array_equal(got, want.compat), (ef, k)
        assert np.array_equal(pd, want.pool_d), (ef, k)
