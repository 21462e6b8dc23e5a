"""The FastScan/RaBitQ oracle (oracle/fs_oracle.c), pinned without a GPU.

Against the golden fixtures (tests/golden/fs_*.npz, made by the reference's
own rotator, RaBitQ encoder and search_qg) always; piece by piece against the
reference's functions compiled into oracle/_ref where that library exists.
"""
import os

import numpy as np
import pytest

from oracle.oracle import FsArrays, FsOracle, RefFastScan, fs_encode, padded_dim, ref_available

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FS_CASES = ("fs40", "fs100d64")


def load_fs_golden(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    n, dim, deg = int(z["n"]), int(z["dim"]), int(z["deg"])
    P = padded_dim(dim)
    o = FsOracle()
    codes = np.stack([o.unpack(z["packed"][i], deg, P) for i in range(n)])
    fs = FsArrays(n, dim, deg, int(z["entry"]), z["vectors"], z["nbrs"], codes, z["factors"],
                  z["diag"])
    exp = {}
    for key in z.files:
        if key.startswith("ids_ef"):
            ef, k = key[6:].split("_k")
            exp[(int(ef), int(k))] = z[key]
    return fs, z["queries"], exp, z["packed"]


@pytest.mark.parametrize("name", FS_CASES)
def test_fs_oracle_matches_reference_golden(name):
    """Bit-exact ids vs the reference's search_qg on the same rows."""
    fs, q, exp, _ = load_fs_golden(name)
    o = FsOracle(fs)
    for (ef, k), want in exp.items():
        got, st = o.search(q, k, ef, nthreads=2)
        assert np.array_equal(got, want), (name, ef, k)


def test_fs_golden_covers_short_results():
    """ef < k: the results are topped up by update_results (qg.hpp:395-418)."""
    fs, q, exp, _ = load_fs_golden("fs40")
    _, st = FsOracle(fs).search(q, 20, 5)
    assert (st[:, 2] > 0).all()


@pytest.mark.parametrize("name", FS_CASES)
def test_fs_pack_unpack_round_trip(name):
    fs, _, _, packed = load_fs_golden(name)
    o = FsOracle()
    for i in range(0, fs.n, 97):
        assert np.array_equal(o.pack(fs.codes[i]), packed[i])


needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


def _diag(rng, P):
    return ((rng.integers(0, 2, P) * 2 - 1) / np.sqrt(np.float32(P))).astype(np.float32)


@needs_ref
@pytest.mark.parametrize("dim", [33, 40, 64, 100, 128, 960, 2048])
def test_rotation_and_query_prepare_bit_exact(dim):
    rng = np.random.default_rng(dim)
    P = padded_dim(dim)
    diag = _diag(rng, P)
    x = (rng.normal(0, 1, (64, dim)) * rng.uniform(0.01, 100)).astype(np.float32)
    o, r = FsOracle(), RefFastScan()
    rot = o.rotate(x, diag)
    assert np.array_equal(rot, r.rotate(x, diag))
    for i in range(len(x)):
        l1, w1, lo1, s1 = o.query_prepare(rot[i])
        l2, w2, lo2, s2 = r.query_prepare(x[i], diag)
        assert np.array_equal(l1, l2) and (w1, lo1, s1) == (w2, lo2, s2), i


@needs_ref
@pytest.mark.parametrize("dim,deg", [(40, 32), (128, 32), (100, 64), (960, 64), (2048, 32)])
def test_rabitq_codes_and_scan(dim, deg):
    """Codes bit-exact; factors within 2e-4 of the largest factor of their kind
    (the reference reduces in FP32 with Eigen, the oracle in FP64; triple_x is
    a difference of similar terms, so a relative bound per value would not
    hold near zero); the scanner's estimates (integer
    accumulators, 16-bit sign extension, the estimator) bit-exact on the
    reference's own codes and factors."""
    rng = np.random.default_rng(dim + deg)
    P = padded_dim(dim)
    diag = _diag(rng, P)
    o, r = FsOracle(), RefFastScan()
    for trial in range(3):
        x = (rng.normal(0, 1, (deg + 1, dim)) * 10).astype(np.float32)
        rot = o.rotate(x, diag)
        bits, fac = o.rabitq(rot[1:], rot[0])
        packed_ref, fac_ref = r.rabitq(rot[1:], rot[0])
        assert np.array_equal(o.pack(bits), packed_ref)
        scale = np.abs(fac_ref).max(axis=1, keepdims=True)  # per factor kind
        assert (np.abs(fac - fac_ref) <= 2e-4 * scale).all()
        for _ in range(10):
            q = (rng.normal(0, 1, dim) * 10).astype(np.float32)
            lut, w, lo, sq = o.query_prepare(o.rotate(q, diag)[0])
            sqr_y = np.float32(rng.uniform(0, 1000))
            mine = o.estimate(o.accumulate(bits, lut), sq, w, lo, sqr_y, fac_ref)
            ref = r.scan(lut, sqr_y, lo, w, sq, packed_ref, fac_ref, deg)
            assert np.array_equal(mine.view(np.uint32), ref.view(np.uint32))


@needs_ref
def test_search_bit_exact_on_oracle_encoded_index():
    """An index encoded by the oracle (FP64 factors): the reference's search_qg
    and the oracle return the same ids."""
    from tests.golden.make_fs_golden import knn_graph

    rng = np.random.default_rng(9)
    n, dim, deg = 1500, 128, 32
    P = padded_dim(dim)
    cent = rng.normal(0, 1, (10, dim))
    x = (cent[rng.integers(0, 10, n)] + rng.normal(0, 0.5, (n, dim))).astype(np.float32)
    q = (cent[rng.integers(0, 10, 100)] + rng.normal(0, 0.5, (100, dim))).astype(np.float32)
    diag = _diag(rng, P)
    nb = knn_graph(x, deg)
    codes, fac = fs_encode(x, nb, diag)
    fs = FsArrays(n, dim, deg, 3, x, nb, codes, fac, diag)
    o, r = FsOracle(fs), RefFastScan()
    for ef, k in ((10, 10), (64, 10), (128, 100), (7, 30)):
        assert np.array_equal(o.search(q, k, ef)[0], r.search(fs, q, k, ef)), (ef, k)
