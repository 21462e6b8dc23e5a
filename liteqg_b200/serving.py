"""Continuous-batching serving loop over one resident index (lqg_server_* C ABI).

    srv = Server(index, streams=4)
    t = srv.submit(query, k=10, ef=128)       # from any thread
    ids, latency_us = srv.wait(t)
    ids, lat = srv.replay(queries, k, ef, arrival_us)   # open-loop driver in C++
    srv.stats()   # completed, batches, mean batch, p50/p99 latency (us), QPS

Requests that arrive while batches are on the GPU are admitted into the next
free stream context and overlap with them; each result equals a search of
that query alone (same kernels, its own k and ef).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import ServerConfig, ServerStats, check, lib


class Server:
    def __init__(self, index, streams: int = 4, max_batch: int = 0, state_budget: int = 0,
                 max_k: int = 100, max_ef: int = 512):
        self.index = index
        self.max_k = int(max_k)
        cfg = ServerConfig(streams, max_batch, state_budget, max_k, max_ef)
        h = C.c_void_p()
        check(lib().lqg_server_start(index.handle, C.byref(cfg), C.byref(h)))
        self._h = h

    def submit(self, query, k: int, ef: int = 0) -> int:
        q = np.ascontiguousarray(query, dtype=np.float32).reshape(-1)
        t = C.c_uint64()
        check(lib().lqg_server_submit(self._h, q.ctypes.data_as(C.c_void_p), int(k), int(ef),
                                      C.byref(t)))
        return int(t.value)

    def wait(self, ticket: int, k: int, timeout_us: int = -1):
        ids = np.empty(int(k), dtype=np.uint32)
        lat = C.c_double()
        check(lib().lqg_server_wait(self._h, ticket, ids.ctypes.data_as(C.c_void_p),
                                    int(timeout_us), C.byref(lat)))
        return ids, float(lat.value)

    def replay(self, queries, k, ef, arrival_us=None):
        q = np.ascontiguousarray(queries, dtype=np.float32)
        m = q.shape[0]
        ka = np.ascontiguousarray(np.broadcast_to(np.asarray(k, dtype=np.uint32), (m,)))
        ea = np.ascontiguousarray(np.broadcast_to(np.asarray(ef, dtype=np.uint32), (m,)))
        kstride = int(ka.max()) if m else 1
        ids = np.full((m, kstride), 0xFFFFFFFF, dtype=np.uint32)
        lat = np.zeros(m, dtype=np.float64)
        arr = None if arrival_us is None else np.ascontiguousarray(arrival_us, dtype=np.float64)
        p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        check(lib().lqg_server_replay(self._h, p(q), m, p(ka), p(ea), p(arr), p(ids), kstride,
                                      p(lat)))
        return ids, lat

    def stats(self) -> dict:
        s = ServerStats()
        check(lib().lqg_server_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def reset_stats(self) -> None:
        check(lib().lqg_server_reset_stats(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().lqg_server_stop(self._h)
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
