"""Generates the FastScan/RaBitQ golden fixtures (tests/golden/fs_*.npz) from
the reference's own code, compiled from its sources into oracle/_ref.

The fork's search no longer calls its FastScan path (symqglib/qg/qg.hpp:241)
and its builder never writes RaBitQ codes, so the fixtures run the upstream
pieces it still carries on real data:
  1. a seeded clustered data set and its exact k-nearest-neighbour graph
     (numpy, FP64) stand in for a built graph;
  2. a seeded +-1/sqrt(P) rotation diagonal is loaded into the reference's
     FHTRotator, which rotates every vector (utils/rotator.hpp:89-114);
  3. the reference's rabitq_codes (quantization/rabitq.hpp:23-108) encodes
     each node's neighbours around the node: packed FastScan codes and the
     three factors, exactly as upstream stores them in a row;
  4. the reference's QuantizedGraph::search_qg (qg.hpp:252-287) runs on an
     index laid out as upstream's rows, for each (ef, k) below.
The arrays and the reference's ids are stored; the oracle and the GPU kernel
are checked against them.

usage: python tests/golden/make_fs_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import FsArrays, FsOracle, RefFastScan, padded_dim  # noqa: E402

EF_K = ((1, 1), (5, 20), (10, 10), (20, 10), (64, 10), (100, 50), (200, 10))
NQ = 100

CASES = {
    # name: (n, dim, deg, clusters, sigma, seed)
    "fs40": (1000, 40, 32, 12, 0.6, 20),
    "fs100d64": (600, 100, 64, 8, 0.5, 21),
}


def knn_graph(x, deg):
    sq = (x.astype(np.float64) ** 2).sum(1)
    d = sq[:, None] + sq[None, :] - 2.0 * x.astype(np.float64) @ x.T.astype(np.float64)
    np.fill_diagonal(d, np.inf)
    return np.argsort(d, axis=1, kind="stable")[:, :deg].astype(np.uint32)


def main():
    r = RefFastScan()
    o = FsOracle()
    for name, (n, dim, deg, nc, sigma, seed) in CASES.items():
        rng = np.random.default_rng(seed)
        P = padded_dim(dim)
        cent = rng.normal(0.0, 1.0, (nc, dim))
        x = (cent[rng.integers(0, nc, n)] + rng.normal(0.0, sigma, (n, dim))).astype(np.float32)
        q = (cent[rng.integers(0, nc, NQ)] + rng.normal(0.0, sigma, (NQ, dim))).astype(np.float32)
        diag = ((rng.integers(0, 2, P) * 2 - 1) / np.sqrt(np.float32(P))).astype(np.float32)
        nb = knn_graph(x, deg)
        rot = r.rotate(x, diag)
        packed = np.empty((n, deg * P // 8), np.uint8)
        fac = np.empty((n, 3, deg), np.float32)
        for i in range(n):
            packed[i], fac[i] = r.rabitq(rot[nb[i]], rot[i])
        codes = np.stack([o.unpack(packed[i], deg, P) for i in range(n)])
        entry = int(rng.integers(0, n))
        fs = FsArrays(n, dim, deg, entry, x, nb, codes, fac, diag)
        out = dict(n=n, dim=dim, deg=deg, entry=entry, vectors=x, nbrs=nb, packed=packed,
                   factors=fac, diag=diag, queries=q)
        for ef, k in EF_K:
            out[f"ids_ef{ef}_k{k}"] = r.search(fs, q, k, ef, nthreads=4)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, {kk: v.shape for kk, v in out.items() if hasattr(v, "shape")})


if __name__ == "__main__":
    main()
