"""Serving loop: results in a continuous-batching mix equal each query alone."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("streams,max_batch", [(3, 8), (1, 64), (4, 0)])
def test_server_results_equal_alone(golden, streams, max_batch):
    import liteqg_b200
    from liteqg_b200.serving import Server

    g = golden["mix128d64"]
    ix = liteqg_b200.Index("QG", "L2", g["n"], g["dim"], g["deg"])
    ix.load(g["path"])
    rng = np.random.default_rng(streams)
    q = np.concatenate([g["queries"]] * 3)
    m = len(q)
    ks = rng.choice([1, 10, 50], m).astype(np.uint32)
    efs = rng.choice([20, 50, 100, 200], m).astype(np.uint32)
    arrivals = np.cumsum(rng.exponential(1e6 / 20000.0, m))  # Poisson, 20k requests/s
    with Server(ix, streams=streams, max_batch=max_batch) as srv:
        ids, lat = srv.replay(q, ks, efs, arrivals)
        st = srv.stats()
    assert st["completed"] == m and st["batches"] >= 1
    assert (lat > 0).all() and st["p99_us"] >= st["p50_us"] > 0
    for i in range(m):
        k, ef = int(ks[i]), int(efs[i])
        alone = ix.search(q[i:i + 1], k, ef=ef)[0]
        assert np.array_equal(ids[i, :k], alone), (i, k, ef)
        if (ef, k) in g["expected"]:
            assert np.array_equal(ids[i, :k], g["expected"][(ef, k)][i % len(g["queries"])])


def test_server_concurrent_submitters(golden):
    import liteqg_b200
    from liteqg_b200.serving import Server

    g = golden["bin40"]
    ix = liteqg_b200.Index("QG", "L2", g["n"], g["dim"], g["deg"])
    ix.load(g["path"])
    ix.set_ef(100)
    out = {}
    with Server(ix, streams=2, max_batch=16) as srv:
        def worker(t):
            for i in range(t, len(g["queries"]), 4):
                tk = srv.submit(g["queries"][i], 10)
                out[i] = srv.wait(tk, 10)[0]
        th = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    want = g["expected"][(100, 10)]
    for i, ids in out.items():
        assert np.array_equal(ids, want[i])


def test_server_admission_by_ef_class(golden):
    """A small device budget: each batch holds only requests of one ef class
    or smaller ones, as many as fit the class's footprint; results still equal
    each query searched alone, for every class mixed in one stream of requests."""
    import liteqg_b200
    from liteqg_b200.serving import Server

    g = golden["u48"]
    ix = liteqg_b200.Index("QG", "L2", g["n"], g["dim"], g["deg"])
    ix.load(g["path"])
    rng = np.random.default_rng(5)
    q = np.concatenate([g["queries"]] * 4)
    m = len(q)
    ks = rng.choice([1, 10, 50], m).astype(np.uint32)
    efs = rng.choice([16, 64, 100, 200, 300, 512], m).astype(np.uint32)
    # about 40 ef-64 requests or 5 ef-512 requests per context
    with Server(ix, streams=2, state_budget=2 * 40 * (48 * 4 + 100 * 4 + 12 + 1024 * 24)) as srv:
        ids, lat = srv.replay(q, ks, efs, None)
        st = srv.stats()
    assert st["completed"] == m
    assert st["batches"] >= m // 40
    for i in range(m):
        k, ef = int(ks[i]), int(efs[i])
        assert np.array_equal(ids[i, :k], ix.search(q[i:i + 1], k, ef=ef)[0]), (i, k, ef)
