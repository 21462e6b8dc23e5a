"""GPU parity of the replay (tuning mode 3), split (mode 4) and batch (mode 5)
kernels through the C ABI.

Mode 3: search warps run the sorted-pool form of the reference's loop and log
every search-pool operation; a replay lane runs the reference's libstdc++
search heap from the log, checks each step, and answers when equal distances
make the heap layout decide. Mode 4: each search warp runs the exact search
heap itself and keeps only a sorted array for the bound. Mode 5: as mode 4,
with the sorted pool in shared memory and every expansion's candidates
accepted or rejected at once from a rank count. Mode 6: as mode 5 with no
search heap until a pop meets equal smallest distances; the heap is then
rebuilt from the logs, every replayed pop checked. In all, the result
heap is replayed afterwards from a per-query log by one warp per query,
which checks every acceptance and writes the output. Bar: ids, FP32 pools and
pop counts bit-exact against the reference's golden outputs and the oracle;
queries only reach the exact global-memory kernel (stats flag 2) when a pool
outgrows its capacity.
"""
import numpy as np
import pytest

from oracle.oracle import SENTINEL, IndexArrays, Oracle, read_index, write_index

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lqg():
    import liteqg_b200

    return liteqg_b200


OFF = 0xFFFFFFFF  # small_batch: never the query-per-block form


# (tuning mode, replay_all[, small_batch]): the split kernel writes unambiguous
# outputs from its sorted array; replay_all=1 sends every query through the
# checked result replay pass instead, so both paths are covered. Batches of
# these sizes run the batch kernels' query-per-block form (4 warps per query)
# unless small_batch is OFF, which keeps one warp per query.
@pytest.fixture(params=[(3, 0), (4, 0), (4, 1), (5, 0), (5, 1), (5, 0, OFF), (6, 0), (6, 1),
                        (6, 0, OFF), (6, 1, OFF)],
                ids=["replay", "split", "split-replay-all", "batch", "batch-replay-all",
                     "batch-warp", "lazy", "lazy-replay-all", "lazy-warp", "lazy-warp-replay-all"])
def mode(request):
    return request.param


def open_index(lqg, g, mode, **tune):
    ix = lqg.Index("QG", "L2", g["n"], g["dim"], g["deg"])
    ix.load(g["path"])
    ix.set_tuning(mode=mode[0], replay_all=mode[1], small_batch=mode[2] if len(mode) > 2 else 0,
                  **tune)
    return ix


def _oracle_for(g):
    return Oracle(read_index(g["path"], g["n"], g["dim"], g["deg"]))


def test_replay_golden_every_ef_k(lqg, golden, mode):
    """The reference's own outputs, every (ef, k) of the fixtures, batched and single."""
    for name, g in golden.items():
        ix = open_index(lqg, g, mode)
        for (ef, k), want in g["expected"].items():
            ix.set_ef(ef)
            got = ix.search(g["queries"], k)
            assert np.array_equal(got, want), (name, ef, k)
            one = ix.search(g["queries"][3], k)
            assert np.array_equal(one, want[3]), (name, ef, k)


def test_replay_pools_and_pops_bit_exact(lqg, golden, mode):
    for name, g in golden.items():
        ix = open_index(lqg, g, mode)
        o = _oracle_for(g)
        for ef in (10, 33, 100, 200, 480):
            want = o.search(g["queries"], 10, ef)
            ids, (pid, pd), st = ix.search(g["queries"], 10, ef=ef, return_pool=True,
                                           return_stats=True)
            assert np.array_equal(ids, want.compat), (name, ef)
            for i in range(len(ids)):
                p = want.pool_n[i]
                assert st[i, 3] == p, (name, ef, i)
                assert np.array_equal(pid[i, :p], want.pool_ids[i, :p]), (name, ef, i)
                assert np.array_equal(pd[i, :p], want.pool_d[i, :p]), (name, ef, i)
                assert (pid[i, p:] == SENTINEL).all()
                assert st[i, 0] == want.pops[i], (name, ef, i)
                assert st[i, 1] >= want.evals[i] + (0 if st[i, 2] == 2 else 1)
            if name != "bin40":
                # no pool outgrew its capacity: every query stayed in the replay kernel
                assert (st[:, 2] == 0).all(), (name, ef, int((st[:, 2] != 0).sum()))


@pytest.mark.parametrize("g_lanes,vbits,swarps,scap", [
    (4, 10, 15, 512), (2, 8, 4, 256), (8, 13, 1, 2048), (4, 9, 7, 1024), (2, 12, 15, 256)])
def test_replay_tuning_does_not_change_results(lqg, golden, mode, g_lanes, vbits, swarps, scap):
    for name in ("mix128d64", "bin40"):
        g = golden[name]
        ix = open_index(lqg, g, mode, lanes_per_cand=g_lanes, visited_bits=vbits,
                        replay_warps=swarps, heap_warps=min(swarps, 5), heap_scap=scap)
        for ef, k in ((20, 10), (50, 50), (200, 10)):
            ix.set_ef(ef)
            assert np.array_equal(ix.search(g["queries"], k), g["expected"][(ef, k)]), (name, ef, k)


def test_replay_tie_heavy_binary_vectors(lqg, golden, mode):
    """Binary vectors: every query meets equal distances at the pop and the bound."""
    g = golden["bin40"]
    ix = open_index(lqg, g, mode)
    o = _oracle_for(g)
    for ef in (20, 100, 200):
        want = o.search(g["queries"], 50, ef)
        ids, (pid, pd), st = ix.search(g["queries"], 50, ef=ef, return_pool=True,
                                       return_stats=True)
        assert np.array_equal(ids, want.compat), ef
        assert np.array_equal(pd, want.pool_d), ef
        assert np.array_equal(pid, want.pool_ids), ef
        assert np.array_equal(st[:, 0], want.pops), ef


def _device(ix, q, ef, k, kq=None, efq=None):
    import torch

    qt = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    m = qt.shape[0]
    ids = torch.full((m, k), -1, dtype=torch.int32, device="cuda")
    st = torch.zeros((m, 4), dtype=torch.int32, device="cuda")
    kt = torch.from_numpy(kq).cuda() if kq is not None else None
    et = torch.from_numpy(efq).cuda() if efq is not None else None
    s = torch.cuda.current_stream()
    ix.search_device(qt.data_ptr(), m, k, ids.data_ptr(), k, ef=ef,
                     ef_ptr=et.data_ptr() if et is not None else 0,
                     k_ptr=kt.data_ptr() if kt is not None else 0,
                     stats_ptr=st.data_ptr(), stream=s.cuda_stream)
    ix.stream_status(s.cuda_stream)
    return ids.cpu().numpy().view(np.uint32), st.cpu().numpy()


def _knn_graph(x, deg):
    sq = (x.astype(np.float64) ** 2).sum(1)
    n = len(x)
    nb = np.empty((n, deg), np.uint32)
    for s in range(0, n, 2048):
        d = sq[s:s + 2048, None] + sq[None, :] - 2 * x[s:s + 2048].astype(np.float64) @ x.T.astype(np.float64)
        d[np.arange(d.shape[0]), np.arange(s, s + d.shape[0])] = np.inf
        nb[s:s + 2048] = np.argpartition(d, deg, axis=1)[:, :deg]
    return nb


@pytest.mark.parametrize("dim,deg,integer", [(128, 32, True), (96, 64, True), (64, 32, False),
                                             (288, 64, False), (33, 32, True), (130, 32, False),
                                             (64, 96, True), (48, 128, False)])
def test_replay_larger_index_uneven_batch(lqg, tmp_path, mode, dim, deg, integer):
    """12k nodes, exact-kNN graph; per-query ef in {1..512} and k in {1, 10, 100}."""
    from oracle.oracle import sq8_quantize

    rng = np.random.default_rng(dim + deg)
    n = 12000
    if integer:
        cent = rng.uniform(0, 255, (64, dim))
        gen = lambda m: np.clip(np.rint(cent[rng.integers(0, 64, m)] + rng.normal(0, 20, (m, dim))),
                                0, 255).astype(np.float32)
    else:
        gen = lambda m: rng.random((m, dim), dtype=np.float32)
    x = gen(n)
    codes, params = sq8_quantize(x, 2)
    arr = IndexArrays(n, dim, deg, int(rng.integers(0, n)), x, _knn_graph(x, deg), codes, params)
    path = str(tmp_path / "big.idx")
    write_index(path, arr)
    ix = lqg.Index("QG", "L2", n, dim, deg)
    ix.load(path)
    ix.set_tuning(mode=mode[0], replay_all=mode[1], small_batch=mode[2] if len(mode) > 2 else 0)
    o = Oracle(arr)
    q = gen(400)
    efq = rng.choice([1, 7, 32, 64, 100, 256, 512], size=len(q)).astype(np.uint32)
    kq = rng.choice([1, 10, 100], size=len(q)).astype(np.uint32)
    ids, st = _device(ix, q, 512, 100, kq=kq, efq=efq)
    want = o.search(q, kq.astype(np.int32), efq.astype(np.int32))
    for i in range(len(q)):
        k = int(kq[i])
        assert np.array_equal(ids[i, :k], want.compat[i, :k]), (i, efq[i], k)
    assert np.array_equal(st[:, 0], want.pops)
    assert (st[:, 2] == 0).mean() > 0.95, int((st[:, 2] != 0).sum())
    for ef, k in ((64, 10), (256, 100)):
        w = o.search(q, k, ef)
        got, (pid, pd) = ix.search(q, k, ef=ef, return_pool=True)
        assert np.array_equal(got, w.compat), (ef, k)
        assert np.array_equal(pd, w.pool_d), (ef, k)
        assert np.array_equal(pid, w.pool_ids), (ef, k)


@pytest.mark.parametrize("work_mode", [2, 6])
def test_large_batch_work_order(lqg, tmp_path, work_mode):
    """8,000 queries (more than the launch's resident warps, so the batch is
    reordered longest-expected first) with per-query ef and k: ids and pops
    equal the oracle's, query by query, in the heap kernel's path (mode 2) and
    the batch kernel's (mode 6)."""
    from oracle.oracle import sq8_quantize

    rng = np.random.default_rng(77)
    n, dim, deg = 6000, 64, 32
    cent = rng.uniform(0, 255, (32, dim))
    gen = lambda m: np.clip(np.rint(cent[rng.integers(0, 32, m)] + rng.normal(0, 20, (m, dim))),
                            0, 255).astype(np.float32)
    x = gen(n)
    codes, params = sq8_quantize(x, 2)
    arr = IndexArrays(n, dim, deg, int(rng.integers(0, n)), x, _knn_graph(x, deg), codes, params)
    path = str(tmp_path / "wo.idx")
    write_index(path, arr)
    ix = lqg.Index("QG", "L2", n, dim, deg)
    ix.load(path)
    ix.set_tuning(mode=work_mode)
    q = gen(8000)
    efq = rng.choice([10, 32, 64, 128], size=len(q)).astype(np.uint32)
    kq = rng.choice([1, 10], size=len(q)).astype(np.uint32)
    ids, st = _device(ix, q, 128, 10, kq=kq, efq=efq)
    want = Oracle(arr).search(q, kq.astype(np.int32), efq.astype(np.int32))
    for i in range(len(q)):
        k = int(kq[i])
        assert np.array_equal(ids[i, :k], want.compat[i, :k]), (i, efq[i], k)
    assert np.array_equal(st[:, 0], want.pops)


@pytest.mark.parametrize("fix_mode", [1, 2, 4, 5, 6])
def test_repeated_ids_across_list_words(lqg, tmp_path, fix_mode):
    """Degree 64 (two 32-id words per list) with ids repeated across the words
    and a 256-slot visited cache, so a kept id's slot is often taken by
    another id of the same expansion: every node is still a candidate once
    per expansion, as the reference's visited set makes it (ids, pools and
    pops equal the oracle's), in every kernel mode."""
    from oracle.oracle import sq8_quantize

    rng = np.random.default_rng(64)
    n, dim, deg = 5000, 64, 64
    cent = rng.uniform(0, 255, (16, dim))
    gen = lambda m: np.clip(np.rint(cent[rng.integers(0, 16, m)] + rng.normal(0, 25, (m, dim))),
                            0, 255).astype(np.float32)
    x = gen(n)
    nb = _knn_graph(x, deg)
    # the second word repeats a third of the first word's ids at random slots
    for i in range(n):
        src = rng.choice(32, 11, replace=False)
        dst = 32 + rng.choice(32, 11, replace=False)
        nb[i, dst] = nb[i, src]
    codes, params = sq8_quantize(x, 2)
    arr = IndexArrays(n, dim, deg, int(rng.integers(0, n)), x, nb, codes, params)
    path = str(tmp_path / "rep.idx")
    write_index(path, arr)
    ix = lqg.Index("QG", "L2", n, dim, deg)
    ix.load(path)
    ix.set_tuning(mode=fix_mode, visited_bits=8)
    o = Oracle(arr)
    q = gen(300)
    for ef in (32, 128):
        want = o.search(q, 10, ef)
        ids, (pid, pd), st = ix.search(q, 10, ef=ef, return_pool=True, return_stats=True)
        assert np.array_equal(ids, want.compat), ef
        assert np.array_equal(pd, want.pool_d), ef
        assert np.array_equal(st[:, 0], want.pops), ef


@pytest.mark.parametrize("hd_mode,small", [(2, 0), (4, 0), (5, 0), (6, 0), (6, OFF)])
def test_high_dimension_degree_64_uneven_batch(lqg, tmp_path, hd_mode, small):
    """The uneven high-dimension workload's shape at 12k nodes: D = 960
    (960-byte code rows, the long code-load window), degree 64, a float
    Gaussian mixture (centres N(0, 1), sigma 0.3), an exact-kNN graph, and one
    batch with per-query ef up to 512 and k in {1, 10, 100}: ids, pops and
    FP32 pools equal the oracle's in the heap kernel (mode 2, the tuner's
    choice there), the split kernel (4) and the batch kernels (5, 6; 300
    queries run one query per block of 4 warps, and with small_batch OFF one
    per warp)."""
    from oracle.oracle import sq8_quantize

    rng = np.random.default_rng(960)
    n, dim, deg = 12000, 960, 64
    cent = rng.normal(0.0, 1.0, (8, dim))  # 1,500 nodes per cluster: every pool fills
    gen = lambda m: (cent[rng.integers(0, 8, m)] + rng.normal(0.0, 0.3, (m, dim))).astype(np.float32)
    x = gen(n)
    codes, params = sq8_quantize(x)
    arr = IndexArrays(n, dim, deg, int(rng.integers(0, n)), x, _knn_graph(x, deg), codes, params)
    path = str(tmp_path / "hd.idx")
    write_index(path, arr)
    ix = lqg.Index("QG", "L2", n, dim, deg)
    ix.load(path)
    ix.set_tuning(mode=hd_mode, lanes_per_cand=2, heap_scap=512, small_batch=small)
    o = Oracle(arr)
    q = gen(300)
    efq = rng.choice([32, 64, 128, 256, 512], size=len(q)).astype(np.uint32)
    kq = rng.choice([1, 10, 100], size=len(q)).astype(np.uint32)
    ids, st = _device(ix, q, 512, 100, kq=kq, efq=efq)
    want = o.search(q, kq.astype(np.int32), efq.astype(np.int32))
    for i in range(len(q)):
        k = int(kq[i])
        assert np.array_equal(ids[i, :k], want.compat[i, :k]), (i, efq[i], k)
    assert np.array_equal(st[:, 0], want.pops)
    for ef, k in ((64, 10), (512, 100)):
        w = o.search(q[:100], k, ef)
        got, (pid, pd), st2 = ix.search(q[:100], k, ef=ef, return_pool=True, return_stats=True)
        assert np.array_equal(got, w.compat), (ef, k)
        assert np.array_equal(pd, w.pool_d), (ef, k)
        assert np.array_equal(pid, w.pool_ids), (ef, k)
        assert np.array_equal(st2[:, 0], w.pops), (ef, k)
