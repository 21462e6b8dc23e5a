"""GPU index builder: valid graph, reference-exact SQ8 encoding, usable recall."""
import numpy as np
import pytest

from oracle.oracle import Oracle, read_index, sq8_quantize

pytestmark = pytest.mark.gpu


def _recall(pool, gt, k):
    return np.mean([len(set(pool[i, :k]) & set(gt[i, :k])) / k for i in range(len(gt))])


@pytest.mark.parametrize("n,dim,deg", [(20000, 64, 32), (8000, 96, 64), (5000, 40, 32)])
def test_build_graph_valid_and_searchable(tmp_path, n, dim, deg):
    import liteqg_b200

    rng = np.random.default_rng(n + dim)
    x = rng.random((n, dim), dtype=np.float32)
    q = rng.random((200, dim), dtype=np.float32)
    ix = liteqg_b200.Index("QG", "L2", n, dim, deg)
    ix.build_index(x, 100, num_iter=3)
    entry, vec, nb, codes, params = ix.get_arrays()
    assert np.array_equal(vec, x)
    # graph: exactly deg distinct ids per node, none the node itself
    assert nb.shape == (n, deg) and int(nb.max()) < n
    srt = np.sort(nb, axis=1)
    assert not (srt[:, 1:] == srt[:, :-1]).any()
    assert not (nb == np.arange(n, dtype=np.uint32)[:, None]).any()
    # SQ8 encoding equals the reference encoder (pinned by the oracle tests)
    c2, p2 = sq8_quantize(x, 2)
    assert np.array_equal(codes, c2) and np.array_equal(params.view(np.uint32), p2.view(np.uint32))
    # entry point: nearest point to the centroid
    cen = (x.astype(np.float64).sum(0) / n).astype(np.float32)
    d = ((x - cen) ** 2).sum(1)
    assert d[entry] <= d.min() * (1 + 1e-5)
    # searching the built index is exact against the oracle, and recall is high
    path = str(tmp_path / "b.idx")
    ix.save(path)
    o = Oracle(read_index(path, n, dim, deg))
    got, (pid, pd) = ix.search(q, 10, ef=64, return_pool=True)
    want = o.search(q, 10, 64)
    assert np.array_equal(got, want.compat)
    gt = np.argsort(((q[:, None, :].astype(np.float64) - x[None].astype(np.float64)) ** 2).sum(-1), 1)[:, :10]
    # quality: at least what the exact deg-NN graph gives on the same data
    from oracle.oracle import IndexArrays
    from tests.test_gpu_parity import _knn_graph

    knn = IndexArrays(n, dim, deg, entry, x, _knn_graph(x, deg), codes, params)
    kr = Oracle(knn).search(q, 10, 64)
    r_built, r_knn = _recall(pid, gt, 10), _recall(kr.pool_ids, gt, 10)
    assert r_built >= r_knn - 0.02, (r_built, r_knn)


def test_build_is_deterministic():
    import liteqg_b200

    x = np.random.default_rng(3).random((6000, 48), dtype=np.float32)
    a = liteqg_b200.Index("QG", "L2", 6000, 48, 32)
    b = liteqg_b200.Index("QG", "L2", 6000, 48, 32)
    a.build_index(x, 64, 2)
    b.build_index(x, 64, 2)
    assert np.array_equal(a.get_arrays()[2], b.get_arrays()[2])


def test_build_rejects_bad_shapes():
    import liteqg_b200

    ix = liteqg_b200.Index("QG", "L2", 100, 64, 32)
    with pytest.raises(ValueError, match="different with initialization"):
        ix.build_index(np.zeros((99, 64), np.float32), 50)
    with pytest.raises(ValueError, match=">= 3"):
        ix.build_index(np.zeros((100, 64), np.float32), 50, num_iter=1)


def test_build_search_path_links_reach_every_cluster():
    """Clustered data (96 well-separated clusters): without search-path links
    the clusters far from the entry point stay hard to reach; with them
    (path_take, far_budget) recall at a small ef rises. The graph stays valid
    and deterministic, and searching it stays exact against the oracle."""
    import liteqg_b200

    rng = np.random.default_rng(11)
    n, dim, deg, nc = 24000, 48, 32, 96
    cent = rng.uniform(0, 255, (nc, dim))
    gen = lambda m: np.clip(np.rint(cent[rng.integers(0, nc, m)] + rng.normal(0, 12, (m, dim))),
                            0, 255).astype(np.float32)
    x, q = gen(n), gen(300)
    gt = np.argsort(((q[:, None, :].astype(np.float64) - x[None].astype(np.float64)) ** 2).sum(-1), 1)[:, :10]
    rec = {}
    for name, kw in (("random", dict(random_edges=4)),
                     ("path", dict(random_edges=4, path_take=64, far_budget=4))):
        ix = liteqg_b200.Index("QG", "L2", n, dim, deg)
        ix.build_index(x, 100, num_iter=3, **kw)
        nb = ix.get_arrays()[2]
        srt = np.sort(nb, axis=1)
        assert not (srt[:, 1:] == srt[:, :-1]).any() and int(nb.max()) < n
        _, (pid, _) = ix.search(q, 10, ef=32, return_pool=True)
        rec[name] = _recall(pid, gt, 10)
        if name == "path":
            again = liteqg_b200.Index("QG", "L2", n, dim, deg)
            again.build_index(x, 100, num_iter=3, **kw)
            assert np.array_equal(again.get_arrays()[2], nb)
    assert rec["path"] >= rec["random"], rec
    assert rec["path"] >= 0.9, rec


@pytest.mark.parametrize("kind", ["uniform", "int_mixture", "gauss_mixture"])
def test_tensor_core_prune_builds_the_fp32_graph(kind):
    """pair_kernel 1 (BF16 tcgen05 Gram matrices, FP32 re-check of decisions
    near their threshold) builds exactly the graph of pair_kernel 0 (FP32 on
    CUDA cores): no pruned edge differs."""
    import liteqg_b200

    rng = np.random.default_rng(17)
    n, dim, deg = 12000, 128, 32
    if kind == "uniform":
        x = rng.random((n, dim), dtype=np.float32)
    elif kind == "int_mixture":
        c = rng.uniform(0, 255, (48, dim))
        x = np.clip(np.rint(c[rng.integers(0, 48, n)] + rng.normal(0, 20, (n, dim))), 0, 255).astype(np.float32)
    else:
        c = rng.normal(0, 1, (48, dim))
        x = (c[rng.integers(0, 48, n)] + rng.normal(0, 0.3, (n, dim))).astype(np.float32)
    graphs, reps = [], []
    for pk in (0, 1):
        ix = liteqg_b200.Index("QG", "L2", n, dim, deg)
        reps.append(ix.build_index(x, 100, num_iter=3, random_edges=4, path_take=32, far_budget=4,
                                   pair_kernel=pk))
        graphs.append(ix.get_arrays()[2])
    assert np.array_equal(graphs[0], graphs[1]), int((graphs[0] != graphs[1]).any(1).sum())
    assert reps[0]["rechecks"] == 0 and reps[1]["prune_ms"] > 0


def test_sq8_params_keep_the_reference_zero():
    """Rounded integer data holds both -0.0 and 0.0: the minimum's sign is the
    one the reference's compiled std::min keeps (the last of the equal values
    over the rows in order, sq8.hpp:13-17), so the saved file matches the
    reference's bytes; the fixture is the reference's own encoder output."""
    import os

    import liteqg_b200

    from tests.golden.make_sq8_golden import signed_zero_data

    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                             "sq8_signed_zero.npz"))
    assert np.array_equal(signed_zero_data().view(np.uint32), z["x"].view(np.uint32))
    rng = np.random.default_rng(8)
    n, dim = 6000, 48
    x = np.clip(np.rint(rng.normal(0.0, 3.0, (n, dim))), 0, 255).astype(np.float32)
    x[-1, : dim // 2] = -0.0  # the last row decides for half of the columns
    x[-1, dim // 2:] = 0.0
    x[-2, dim // 2:] = -0.0
    assert (np.signbit(x) & (x == 0)).any(0).all()
    for data in (z["x"], x):
        ix = liteqg_b200.Index("QG", "L2", len(data), dim, 32)
        ix.build_index(data, 64, num_iter=2)
        _, _, _, codes, params = ix.get_arrays()
        c2, p2 = sq8_quantize(data, 2)
        assert np.array_equal(codes, c2)
        assert np.array_equal(params.view(np.uint32), p2.view(np.uint32))
        ix.close()
    assert np.array_equal(params.view(np.uint32)[:, 0] >> 31, (np.arange(dim) < dim // 2))
