"""Generates the golden fixtures under tests/golden/ from the reference itself.

Run where the reference sources were available to ``make -C oracle ref``
(``oracle/_ref/`` present). For each case it:
  1. builds an index with the reference's own builder (QGBuilder through
     ``oracle/_ref/libref_harness.so``) and keeps the exact file it saved
     (gzipped) — the reference's file layout, byte for byte;
  2. draws queries from a fixed seed;
  3. records what the reference's ``QuantizedGraph::search`` writes for each
     (ef, k) pair, with the slots it leaves unwritten filled with 0xFFFFFFFF;
  4. cross-checks a subset through the reference's unmodified pybind module
     (``oracle/_ref/symphonyqg*.so``, ``Index.load/set_ef/search``), where
     every slot is written (k <= pool size).

The reference builder seeds itself from std::random_device, so a rerun gives
different graphs; the committed files are the fixtures.

usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import gzip
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import RefHarness, SENTINEL, read_index  # noqa: E402

EFS = (10, 20, 50, 100, 200)
KS = (1, 10, 50)
NQ = 100


def mixture(rng, n, dim, nclusters, lo, hi, sigma):
    centres = rng.uniform(lo, hi, size=(nclusters, dim))
    lab = rng.integers(0, nclusters, size=n)
    x = centres[lab] + rng.normal(0.0, sigma, size=(n, dim))
    return np.clip(np.rint(x), lo, hi).astype(np.float32)


CASES = {
    # name: (data, queries, degree_bound, EF)
    "u48": lambda: (np.random.default_rng(10).random((1000, 48), dtype=np.float32),
                    np.random.default_rng(11).random((NQ, 48), dtype=np.float32), 32, 100),
    "bin40": lambda: (np.random.default_rng(12).integers(0, 2, (800, 40)).astype(np.float32),
                      np.random.default_rng(13).integers(0, 2, (NQ, 40)).astype(np.float32),
                      32, 100),
    "mix128d64": lambda: (mixture(np.random.default_rng(14), 1000, 128, 16, 0, 255, 20.0),
                          mixture(np.random.default_rng(15), NQ, 128, 16, 0, 255, 20.0), 64, 100),
}


def main():
    h = RefHarness()
    import importlib.util

    so = [f for f in os.listdir(os.path.join(ROOT, "oracle", "_ref")) if f.startswith("symphonyqg")]
    spec = importlib.util.spec_from_file_location("symphonyqg", os.path.join(ROOT, "oracle", "_ref", so[0]))
    symqg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(symqg)

    tmp = tempfile.mkdtemp()
    try:
        for name, make in CASES.items():
            data, queries, deg, efb = make()
            n, dim = data.shape
            path = os.path.join(tmp, name + ".idx")
            h.build(data, deg, efb, 3, path, nthreads=4)
            ref = h.open(path, n, dim, deg)
            out = {"queries": queries, "n": n, "dim": dim, "deg": deg}
            for ef in EFS:
                for k in KS:
                    out[f"ids_ef{ef}_k{k}"] = ref.search(queries, k, ef, nthreads=1)
            ref.close()
            # the reference's own Python API on the same file
            ix = symqg.Index("QG", "L2", n, dim, deg)
            ix.load(path)
            for ef in EFS:
                ix.set_ef(ef)
                k = min(10, ef)
                got = np.stack([ix.search(queries[i], k) for i in range(NQ)])
                want = out[f"ids_ef{ef}_k{k}"] if k in KS else None
                if want is not None and not np.array_equal(got, want):
                    raise SystemExit(f"{name}: pybind and harness disagree at ef={ef}")
            arrays = read_index(path, n, dim, deg)
            assert int(np.max(arrays.nbrs)) < n
            with open(path, "rb") as f, gzip.open(os.path.join(HERE, name + ".idx.gz"), "wb", 9) as g:
                shutil.copyfileobj(f, g)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
            print(name, "written")
    finally:
        shutil.rmtree(tmp)
    assert SENTINEL == 0xFFFFFFFF


if __name__ == "__main__":
    main()
