"""Autotuner for the search kernels' launch shape and policy.

Times a small grid of `lqg_tuning` settings (kernel mode: 1 fast + heap for
tied queries, 2 heap, 4 split, 5 batch, 6 batch with a lazy search heap;
lanes per candidate, visited-cache size, warps per block, shared-memory
search-pool slots) on the caller's queries with CUDA events, keeps the
fastest, and caches the choice in a JSON file keyed on (N, D, degree, ef, k),
so later runs on the same kind of index start from it. Every setting returns
the same ids (the kernels are exact under all of them); only time differs.
"""
from __future__ import annotations

import json
import os

import numpy as np

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "liteqg_b200", "tuning.json")

# (mode, lanes_per_cand, visited_bits, warps_per_block, heap_warps, heap_scap)
CANDIDATES = [
    (6, 2, 10, 8, 4, 256),
    (6, 4, 10, 8, 4, 256),
    (6, 2, 10, 8, 5, 256),
    (6, 4, 10, 8, 5, 256),
    (6, 2, 10, 8, 4, 512),
    (6, 2, 9, 8, 5, 256),
    (5, 2, 10, 8, 4, 256),
    (5, 4, 10, 8, 4, 256),
    (5, 2, 10, 8, 4, 512),
    (5, 4, 10, 8, 4, 512),
    (5, 2, 11, 8, 4, 512),
    (5, 2, 10, 8, 5, 256),
    (5, 4, 10, 8, 5, 256),
    (4, 2, 10, 8, 4, 256),
    (4, 2, 10, 8, 4, 512),
    (4, 4, 10, 8, 4, 512),
    (4, 4, 10, 8, 4, 256),
    (4, 2, 11, 8, 4, 512),
    (4, 2, 10, 8, 5, 256),
    (1, 4, 10, 8, 4, 1024),
    (2, 4, 10, 8, 4, 1024),
    (2, 4, 10, 8, 4, 512),
    (2, 4, 11, 8, 4, 512),
    (2, 4, 9, 8, 4, 1024),
    (2, 4, 10, 8, 2, 1024),
    (2, 8, 10, 8, 4, 1024),
    (2, 2, 10, 8, 4, 1024),
    (2, 4, 10, 8, 4, 2048),
    (1, 8, 10, 8, 4, 1024),
    (1, 4, 11, 4, 4, 1024),
]


def _key(ix, ef, k) -> str:
    return f"N{ix.num_elements}-D{ix.dimension}-deg{ix.degree_bound}-ef{ef}-k{k}"


def load_cached(ix, ef: int, k: int, path: str = DEFAULT_CACHE):
    try:
        with open(path) as f:
            return json.load(f).get(_key(ix, ef, k))
    except (OSError, ValueError):
        return None


def tune(ix, queries: np.ndarray, ef: int, k: int, reps: int = 3, path: str | None = DEFAULT_CACHE,
         candidates=CANDIDATES, device: int = 0) -> dict:
    """Times each candidate on `queries` (device-resident copy) and applies the best."""
    import torch

    dev = torch.device("cuda", device)
    stream = torch.cuda.current_stream(dev)
    q = torch.from_numpy(np.ascontiguousarray(queries, dtype=np.float32)).to(dev)
    m = q.shape[0]
    ids = torch.empty((m, k), dtype=torch.int32, device=dev)
    results = []
    for c in candidates:
        mode, g, vb, wpb, hw, scap = c
        try:
            ix.set_tuning(lanes_per_cand=g, visited_bits=vb, warps_per_block=wpb, mode=mode,
                          heap_warps=hw, heap_scap=scap)
        except Exception:
            continue
        ix.search_device(q.data_ptr(), m, k, ids.data_ptr(), k, ef=ef, stream=stream.cuda_stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            ix.search_device(q.data_ptr(), m, k, ids.data_ptr(), k, ef=ef,
                             stream=stream.cuda_stream)
        b.record(stream)
        b.synchronize()
        ix.stream_status(stream.cuda_stream)
        results.append((a.elapsed_time(b) / reps, c))
    results.sort()
    best_ms, best = results[0]
    mode, g, vb, wpb, hw, scap = best
    choice = dict(mode=mode, lanes_per_cand=g, visited_bits=vb, warps_per_block=wpb,
                  heap_warps=hw, heap_scap=scap, ms=best_ms, queries=m)
    ix.set_tuning(lanes_per_cand=g, visited_bits=vb, warps_per_block=wpb, mode=mode,
                  heap_warps=hw, heap_scap=scap)
    if path:
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            table = {}
            if os.path.exists(path):
                with open(path) as f:
                    table = json.load(f)
            table[_key(ix, ef, k)] = choice
            with open(path, "w") as f:
                json.dump(table, f, indent=1)
        except (OSError, ValueError):
            pass
    choice["all"] = [(round(t, 4), list(c)) for t, c in results]
    return choice


def apply(ix, choice: dict) -> None:
    ix.set_tuning(lanes_per_cand=choice["lanes_per_cand"], visited_bits=choice["visited_bits"],
                  warps_per_block=choice["warps_per_block"], mode=choice["mode"],
                  heap_warps=choice["heap_warps"], heap_scap=choice["heap_scap"])
