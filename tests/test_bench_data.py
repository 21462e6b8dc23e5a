"""bench.py's prebuilt-graph transport (no GPU): packed ids round-trip, and
the reference arm's CPU-only assembly of an index file reproduces the built
file byte for byte (SHA-256), or refuses when a part is missing."""
import os

import numpy as np
import pytest

import bench
from oracle.oracle import IndexArrays, RefHarness, ref_available, sq8_quantize, write_index


@pytest.mark.parametrize("n", [3, 1000, 1_000_000, 10_000_000])
def test_pack_unpack_ids(n):
    bits = bench._id_bits(n)
    ids = np.random.default_rng(n).integers(0, n, (1001, 32)).astype(np.uint32)
    buf = bench._pack_ids(ids, bits)
    assert len(buf) == (ids.size + ids.size % 2) * bits // 8
    assert np.array_equal(bench._unpack_ids(buf, bits, ids.size), ids.reshape(-1))


def test_assemble_matches_built_file(tmp_path, monkeypatch):
    monkeypatch.setenv("LQG_BENCH_CACHE", str(tmp_path / "cache"))
    name = "small-100k64"
    w = dict(bench.WORKLOADS[name], n=5000, nq=50)
    base = bench.gen_data(w, "base")
    if ref_available():
        codes, params = RefHarness().sq8_quantize(base)
    else:
        codes, params = sq8_quantize(base)
    nb = np.random.default_rng(1).integers(0, w["n"], (w["n"], w["deg"])).astype(np.uint32)
    write_index(bench.index_path(name, w), IndexArrays(w["n"], w["dim"], w["deg"], 17, base, nb,
                                                       codes, params))
    gt = np.random.default_rng(2).integers(0, w["n"], (w["nq"], 100))
    np.save(bench.gt_path(name, w, 0, w["nq"]), gt)
    ship = tmp_path / "ship"
    for p in range(2):
        bench.export_shipped(name, w, p, 2, str(ship))
    sha = bench._sha256(bench.index_path(name, w))
    os.remove(bench.index_path(name, w))
    os.remove(bench.gt_path(name, w, 0, w["nq"]))
    monkeypatch.setattr(bench, "DATA_DIR", str(ship))
    assert bench.assemble_shipped(name, w, base) is not None
    assert bench._sha256(bench.index_path(name, w)) == sha
    assert np.array_equal(np.load(bench.gt_path(name, w, 0, w["nq"])), gt)
    # a missing part: no assembly
    os.remove(bench.index_path(name, w))
    os.remove(next(ship.glob("*.nbrs1of2.bin")))
    assert bench.assemble_shipped(name, w, base) is None
