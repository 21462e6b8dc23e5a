"""GPU parity of the FastScan/RaBitQ search (upstream search_qg) through the C ABI.

Bar: ids bit-exact against the reference's own search_qg (golden fixtures,
tests/golden/fs_*.npz, whose codes and factors the reference's rabitq_codes
wrote) and against the oracle (fs_oracle.c) on GPU-encoded indexes, with the
oracle's pop and evaluation counts; the GPU encoder's codes bit-exact against
the oracle's and its factors within 1e-5 of the largest of their kind.
"""
import os

import numpy as np
import pytest

from oracle.oracle import FsArrays, FsOracle, fs_encode, padded_dim, sq8_quantize

from .test_fs_oracle import FS_CASES, load_fs_golden

pytestmark = pytest.mark.gpu


def _index_from(fs: FsArrays):
    import liteqg_b200

    ix = liteqg_b200.Index("QG", "L2", fs.n, fs.dim, fs.deg)
    codes, params = sq8_quantize(fs.vectors)
    ix.set_arrays(fs.entry, fs.vectors, fs.nbrs, codes, params)
    return ix


def _knn(x, deg):
    sq = (x.astype(np.float64) ** 2).sum(1)
    n = len(x)
    nb = np.empty((n, deg), np.uint32)
    for s in range(0, n, 2048):
        d = sq[s:s + 2048, None] + sq[None, :] - 2 * x[s:s + 2048].astype(np.float64) @ x.T.astype(np.float64)
        d[np.arange(d.shape[0]), np.arange(s, s + d.shape[0])] = np.inf
        nb[s:s + 2048] = np.argpartition(d, deg, axis=1)[:, :deg]
    return nb


@pytest.mark.parametrize("name", FS_CASES)
def test_fastscan_golden_every_ef_k(name):
    """The reference's own codes, factors and search_qg outputs: batched and
    one query per call, every (ef, k) of the fixture, stats equal the oracle's."""
    fs, q, exp, packed = load_fs_golden(name)
    ix = _index_from(fs)
    ix.set_fastscan_arrays(fs.diag, packed, fs.factors)
    o = FsOracle(fs)
    for (ef, k), want in exp.items():
        got, st = ix.search_fastscan(q, k, ef=ef, return_stats=True)
        assert np.array_equal(got, want), (name, ef, k)
        _, ost = o.search(q, k, ef)
        assert np.array_equal(st.astype(np.int32), ost), (name, ef, k)
        ix.set_ef(ef)
        assert np.array_equal(ix.search_fastscan(q[7], k), want[7]), (name, ef, k)


@pytest.mark.parametrize("dim,deg,n", [(128, 32, 4000), (100, 64, 3000), (960, 64, 2500),
                                       (48, 32, 3000), (2048, 32, 800)])
def test_fastscan_gpu_encoder_and_search(dim, deg, n):
    """lqg_fs_build on a kNN graph: codes bit-exact against the oracle's
    encoder, factors within 1e-5 of the largest of their kind (both reduce in
    FP64, in different orders); then per-query ef and k in one batch: ids and
    counts equal the oracle's on the GPU-encoded section."""
    rng = np.random.default_rng(dim * 7 + deg)
    cent = rng.normal(0, 1, (12, dim))
    gen = lambda m: (cent[rng.integers(0, 12, m)] + rng.normal(0, 0.5, (m, dim))).astype(np.float32)
    x = gen(n)
    nb = _knn(x, deg)
    fs0 = FsArrays(n, dim, deg, int(rng.integers(0, n)), x, nb, None, None, None)
    ix = _index_from(fs0)
    ix.fastscan_build(seed=dim)
    diag, packed, fac = ix.fastscan_arrays()
    P = padded_dim(dim)
    assert diag.shape == (P,) and np.allclose(np.abs(diag), 1 / np.sqrt(P))
    o = FsOracle()
    codes, fac_o = fs_encode(x, nb, diag, o)
    got_codes = np.stack([o.unpack(packed[i], deg, P) for i in range(n)])
    assert np.array_equal(got_codes, codes)
    scale = np.abs(fac_o).max(axis=(0, 2), keepdims=True)
    assert (np.abs(fac - fac_o) <= 1e-5 * scale).all()
    fs = FsArrays(n, dim, deg, fs0.entry, x, nb, got_codes, fac, diag)
    q = gen(300)
    efq = rng.choice([1, 10, 32, 64, 100, 256, 512], len(q)).astype(np.uint32)
    kq = rng.choice([1, 10, 100], len(q)).astype(np.int32)
    want, wst = FsOracle(fs).search(q, kq, efq.astype(np.int32))
    import torch

    qt = torch.from_numpy(q).cuda()
    ids = torch.full((len(q), 100), -1, dtype=torch.int32, device="cuda")
    st = torch.zeros((len(q), 4), dtype=torch.int32, device="cuda")
    et = torch.from_numpy(efq.view(np.int32)).cuda()
    kt = torch.from_numpy(kq).cuda()
    s = torch.cuda.current_stream()
    ix.search_fastscan_device(qt.data_ptr(), len(q), 0, ids.data_ptr(), 100, ef=512,
                              ef_ptr=et.data_ptr(), k_ptr=kt.data_ptr(), stats_ptr=st.data_ptr(),
                              stream=s.cuda_stream)
    ix.fastscan_status(s.cuda_stream)
    got = ids.cpu().numpy().view(np.uint32)
    for i in range(len(q)):
        assert np.array_equal(got[i, :kq[i]], want[i, :kq[i]]), (i, efq[i], kq[i])
    assert np.array_equal(st.cpu().numpy(), wst)


def test_fastscan_section_save_load(tmp_path):
    """The section round-trips through the index file; the reference's loader
    still reads the file (its bytes come first) and searches it unchanged."""
    import liteqg_b200
    from oracle.oracle import RefHarness, ref_available

    fs, q, exp, packed = load_fs_golden("fs40")
    ix = _index_from(fs)
    ix.set_fastscan_arrays(fs.diag, packed, fs.factors)
    path = str(tmp_path / "fs.idx")
    ix.save(path)
    ix2 = liteqg_b200.Index("QG", "L2", fs.n, fs.dim, fs.deg)
    ix2.load(path)
    d2, p2, f2 = ix2.fastscan_arrays()
    assert np.array_equal(d2, fs.diag) and np.array_equal(p2, packed)
    assert np.array_equal(f2, fs.factors)
    assert np.array_equal(ix2.search_fastscan(q, 10, ef=64), exp[(64, 10)])
    # the SQ8 path and the reference's loader on the same file
    ix.set_ef(50)
    ix2.set_ef(50)
    assert np.array_equal(ix2.search(q, 10), ix.search(q, 10))
    if ref_available():
        r = RefHarness().open(path, fs.n, fs.dim, fs.deg)
        assert np.array_equal(r.search(q, 10, 50), ix2.search(q, 10))


def test_fastscan_requires_a_section():
    import liteqg_b200
    from liteqg_b200._capi import LqgError

    fs, q, _, _ = load_fs_golden("fs40")
    ix = _index_from(fs)
    with pytest.raises(LqgError, match="FastScan section"):
        ix.search_fastscan(q, 10, ef=10)
    ix.fastscan_build()
    ix.search_fastscan(q, 10, ef=10)
    # a new graph makes the section stale
    ix.set_arrays(fs.entry, fs.vectors, fs.nbrs, *sq8_quantize(fs.vectors))
    with pytest.raises(LqgError, match="FastScan section"):
        ix.search_fastscan(q, 10, ef=10)
