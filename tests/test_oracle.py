"""The CPU oracle, pinned against the reference's own outputs (no GPU)."""
import numpy as np
import pytest

from oracle.oracle import SENTINEL, Oracle, RefHarness, read_index, ref_available, sq8_quantize, write_index


def test_oracle_matches_golden(golden):
    """Bit-exact compat ids vs the reference's search on its own saved index."""
    for name, g in golden.items():
        ix = read_index(g["path"], g["n"], g["dim"], g["deg"])
        o = Oracle(ix)
        for (ef, k), want in g["expected"].items():
            got = o.search(g["queries"], k, ef, nthreads=2)
            assert np.array_equal(got.compat, want), (name, ef, k)


def test_golden_has_ties_and_unwritten_slots(golden):
    """The fixtures exercise the cases where heap order and short pools matter."""
    g = golden["bin40"]
    ix = read_index(g["path"], g["n"], g["dim"], g["deg"])
    r = Oracle(ix).search(g["queries"], 10, 100)
    tied = sum(len(np.unique(r.pool_d[i, : r.pool_n[i]])) < r.pool_n[i] for i in range(len(r.pool_n)))
    assert tied > len(r.pool_n) // 2
    assert (golden["u48"]["expected"][(10, 50)] == SENTINEL).any()


def test_pool_is_consistent_with_compat(golden):
    g = golden["u48"]
    ix = read_index(g["path"], g["n"], g["dim"], g["deg"])
    o = Oracle(ix)
    r = o.search(g["queries"], 10, 50)
    for i in range(len(r.pool_n)):
        p = r.pool_n[i]
        assert p == 50
        assert np.array_equal(r.compat[i], r.pool_ids[i, p - 10 : p])
        assert np.all(np.diff(r.pool_d[i, :p]) >= 0)
        d = o.sq8_l2(g["queries"][i], r.pool_ids[i, :p])
        assert np.array_equal(d, r.pool_d[i, :p])


def test_encoder_matches_reference_file(golden):
    """SQ8 encode restatement == the codes/params inside the reference's file."""
    for name, g in golden.items():
        ix = read_index(g["path"], g["n"], g["dim"], g["deg"])
        codes, params = sq8_quantize(ix.vectors, recip=2)
        assert np.array_equal(codes, ix.codes), name
        assert np.array_equal(params, ix.params), name


def test_encoder_signed_zero_matches_reference_golden():
    """-0.0 and 0.0 in every column: the oracle keeps the same one as the
    reference's compiled std::min (the last of the equal values), so the
    params' bytes agree (fixture: tests/golden/make_sq8_golden.py)."""
    import os

    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                             "sq8_signed_zero.npz"))
    codes, params = sq8_quantize(z["x"], recip=2)
    assert np.array_equal(codes, z["codes"])
    assert np.array_equal(params.view(np.uint32), z["params"].view(np.uint32))
    assert np.signbit(params[:24, 0]).all() and not np.signbit(params[24:, 0]).any()


@pytest.mark.skipif(not ref_available(), reason="compiled reference (oracle/_ref) not present")
def test_encoder_signed_zero_matches_reference_random():
    rng = np.random.default_rng(11)
    h = RefHarness()
    for trial in range(4):
        x = np.clip(np.rint(rng.normal(0.0, 2.0, (700, 40))), 0, 9).astype(np.float32)
        c1, p1 = h.sq8_quantize(x)
        c2, p2 = sq8_quantize(x, recip=2)
        assert np.array_equal(c1, c2) and np.array_equal(p1.view(np.uint32), p2.view(np.uint32))


def test_index_roundtrip(golden, tmp_path):
    g = golden["mix128d64"]
    ix = read_index(g["path"], g["n"], g["dim"], g["deg"])
    p = str(tmp_path / "rt.idx")
    write_index(p, ix)
    assert open(p, "rb").read() == open(g["path"], "rb").read()


@pytest.mark.skipif(not ref_available(), reason="compiled reference (oracle/_ref) not present")
def test_oracle_matches_reference_random(tmp_path):
    """Fresh reference builds, uniform and duplicate-heavy data, several ef/k."""
    h = RefHarness()
    rng = np.random.default_rng(7)
    base = rng.random((600, 64), dtype=np.float32)
    for name, data in (("u", rng.random((1500, 64), dtype=np.float32)),
                       ("dup", np.concatenate([base, base, base[:300]]))):
        path = str(tmp_path / f"{name}.idx")
        h.build(data, 32, 80, 3, path, nthreads=2)
        ref = h.open(path, data.shape[0], 64, 32)
        o = Oracle(read_index(path, data.shape[0], 64, 32))
        q = rng.random((60, 64), dtype=np.float32)
        for ef, k in ((16, 10), (64, 10), (128, 100)):
            assert np.array_equal(ref.search(q, k, ef, nthreads=2), o.search(q, k, ef).compat), (name, ef, k)
        ref.close()


@pytest.mark.skipif(not ref_available(), reason="compiled reference (oracle/_ref) not present")
def test_distance_matches_reference():
    h = RefHarness()
    rng = np.random.default_rng(3)
    for dim in (33, 48, 64, 96, 128, 130):
        data = rng.normal(size=(500, dim)).astype(np.float32) * 7
        codes, params = h.sq8_quantize(data)
        ix = type("I", (), {})()
        q = rng.normal(size=dim).astype(np.float32)
        want = h.sq8_l2(q, codes, params)
        from oracle.oracle import IndexArrays
        arr = IndexArrays(500, dim, 32, 0, data, np.zeros((500, 32), np.uint32), codes, params)
        got = Oracle(arr).sq8_l2(q, np.arange(500))
        assert np.array_equal(got, want), dim
