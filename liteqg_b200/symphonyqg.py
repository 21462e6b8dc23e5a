"""``symphonyqg.Index`` on a B200: the reference's Python API over the C ABI.

Mirrors python/bindings.cpp:35-125 of LiteQG: the same constructor
(``index_type``, ``metric``, ``num_elements``, ``dimension``,
``degree_bound=32``), ``load``/``save`` of the same file, ``set_ef``,
``build_index(data, EF, num_iter=3, num_thread)``, and ``search(query, k)``
returning ``uint32[k]`` with exactly the reference's ids.

Differences, all additive or fail-loud:
* ``search`` with a 2-D ``[M, D]`` query block and ``M > 1`` searches every row
  in one batched launch and returns ``uint32[M, k]`` (the reference reads only
  row 0, bindings.cpp:95). Keyword ``ef`` (int or per-row array) overrides
  ``set_ef``; ``return_pool=True`` also returns the full ascending pool
  ``(ids[M, ef], dists[M, ef])``; ``return_stats=True`` returns per-query
  ``[pops, distance computations, exact-path flag, pool size]``.
* Invalid arguments raise ``ValueError``/``LqgError`` with the reference's
  message, where the reference prints to stderr and leaves an unusable
  object (bindings.cpp:45-60, 80-86).
* Output slots the reference leaves uninitialised (pool smaller than k) hold
  0xFFFFFFFF.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import LQG_NO_ID, BuildReport, LqgError, Tuning, check, lib

UINT_MAX = 0xFFFFFFFF


def _as_f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=np.float32)


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Index:
    def __init__(self, index_type: str, metric: str, num_elements: int, dimension: int,
                 degree_bound: int = 32, device: int = 0):
        h = C.c_void_p()
        st = lib().lqg_create(str(index_type).encode(), str(metric).encode(), int(num_elements),
                              int(dimension), int(degree_bound), int(device), C.byref(h))
        if st != _capi.LQG_OK:
            msg = lib().lqg_last_error().decode()
            if st == 1:
                raise ValueError(msg)
            raise LqgError(st, msg)
        self._h = h
        self.num_elements = int(num_elements)
        self.dimension = int(dimension)
        self.degree_bound = int(degree_bound)
        self.device = int(device)

    # -- lifetime --------------------------------------------------------
    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().lqg_free(h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise ValueError("index is closed")
        return self._h

    # -- reference API ---------------------------------------------------
    def load(self, filename: str) -> None:
        check(lib().lqg_load(self.handle, str(filename).encode()))

    def save(self, filename: str) -> None:
        check(lib().lqg_save(self.handle, str(filename).encode()))

    def set_ef(self, EF: int) -> None:
        check(lib().lqg_set_ef(self.handle, int(EF)))

    def build_index(self, data, EF: int, num_iter: int = 3, num_thread: int = UINT_MAX,
                    seed: int = 0, random_edges: int | None = None,
                    alpha: float = 1.0, path_take: int = 0, far_budget: int = 0,
                    pair_kernel: int = 1) -> dict:
        """Builds on the GPU (``num_thread`` is accepted and unused).

        ``random_edges`` slots of each neighbour list hold seeded random
        long-range links (default ``degree_bound // 8``); ``alpha`` >= 1 is
        the prune's occlusion factor (1 = the reference's heuristic);
        ``path_take`` search-path nodes join each node's candidates and
        ``far_budget`` slots are held for long links; ``pair_kernel`` 1 runs
        the prune's distance matrices as BF16 tcgen05 GEMMs with FP32
        re-checks, 0 in FP32 on CUDA cores (same graph; see lqg_build_ex).
        Returns the build report (prune/build ms, FP32 re-checks)."""
        items = _as_f32(data)
        if items.ndim == 1:
            items = items.reshape(1, -1)
        if items.ndim != 2 or items.shape != (self.num_elements, self.dimension):
            raise ValueError(
                "The shape of data is different with initialization! Expected shape: "
                f"({self.num_elements}, {self.dimension}), but got: {tuple(items.shape)}")
        if num_iter <= 1:
            raise ValueError("The number of iter for building qg should >= 3")
        re = self.degree_bound // 8 if random_edges is None else int(random_edges)
        rep = BuildReport()
        check(lib().lqg_build_ex(self.handle, _p(items), int(EF), int(num_iter), int(seed), re,
                                 float(alpha), int(path_take), int(far_budget), int(pair_kernel),
                                 C.byref(rep)))
        return {f: getattr(rep, f) for f, _ in BuildReport._fields_}

    def search(self, query, k: int, ef=None, return_pool: bool = False,
               return_stats: bool = False):
        q = _as_f32(query)
        k = int(k)
        if q.ndim == 1:
            q = q.reshape(1, -1)
            single = True
        elif q.ndim == 2:
            single = q.shape[0] == 1
        else:
            raise ValueError("Input data has an incorrect shape. Data must be a 1D or 2D array.")
        if q.shape[1] != self.dimension:
            raise ValueError(f"query dimension {q.shape[1]} != index dimension {self.dimension}")
        if k < 0:
            raise ValueError("k must be >= 0")
        if single and ef is None and not return_pool and not return_stats:
            out = np.full(k, LQG_NO_ID, dtype=np.uint32)
            if k:
                check(lib().lqg_search(self.handle, _p(q), k, _p(out)))
            return out
        m = q.shape[0]
        ef_arr, ef0 = None, 0
        if ef is not None:
            if np.ndim(ef) == 0:
                ef0 = int(ef)
            else:
                ef_arr = np.ascontiguousarray(ef, dtype=np.uint32)
                if ef_arr.shape != (m,):
                    raise ValueError("per-query ef must have one value per query row")
                ef0 = int(ef_arr.max()) if m else 1
        kstride = max(k, 1)
        ids = np.full((m, kstride), LQG_NO_ID, dtype=np.uint32)
        pstride = 0
        pool_ids = pool_d = None
        if return_pool:
            pstride = int(ef0 if ef is not None else self.get_ef())
            pool_ids = np.full((m, pstride), LQG_NO_ID, dtype=np.uint32)
            pool_d = np.full((m, pstride), np.inf, dtype=np.float32)
        stats = np.zeros((m, 4), dtype=np.uint32) if return_stats else None
        if m:
            check(lib().lqg_search_batch(
                self.handle, _p(q), m, None, k, _p(ef_arr), ef0, _p(ids), kstride,
                _p(pool_ids), _p(pool_d), pstride, _p(stats), None))
        ids = ids[:, :k]
        res = ids[0] if (single and q.shape[0] == 1 and np.ndim(query) == 1) else ids
        extra = []
        if return_pool:
            extra.append((pool_ids, pool_d))
        if return_stats:
            extra.append(stats)
        return (res, *extra) if extra else res

    # -- additions -------------------------------------------------------
    def get_ef(self) -> int:
        ef = C.c_uint32()
        check(lib().lqg_info(self.handle, None, None, None, None, C.byref(ef)))
        return int(ef.value)

    def entry_point(self) -> int:
        e = C.c_uint32()
        check(lib().lqg_info(self.handle, None, None, None, C.byref(e), None))
        return int(e.value)

    def set_arrays(self, entry: int, vectors, nbrs, codes, params) -> None:
        v = None if vectors is None else _as_f32(vectors)
        nb = np.ascontiguousarray(nbrs, dtype=np.uint32)
        cd = np.ascontiguousarray(codes, dtype=np.uint8)
        pr = _as_f32(params)
        n, d, g = self.num_elements, self.dimension, self.degree_bound
        if nb.shape != (n, g) or cd.shape != (n, d) or pr.reshape(-1).shape != (2 * d,):
            raise ValueError("array shapes do not match the index")
        if v is not None and v.shape != (n, d):
            raise ValueError("vectors shape does not match the index")
        check(lib().lqg_set_arrays(self.handle, int(entry), _p(v), _p(nb), _p(cd), _p(pr)))

    def get_arrays(self):
        n, d, g = self.num_elements, self.dimension, self.degree_bound
        e = C.c_uint32()
        v = np.empty((n, d), np.float32)
        nb = np.empty((n, g), np.uint32)
        cd = np.empty((n, d), np.uint8)
        pr = np.empty((d, 2), np.float32)
        check(lib().lqg_get_arrays(self.handle, C.byref(e), _p(v), _p(nb), _p(cd), _p(pr)))
        return int(e.value), v, nb, cd, pr

    def set_tuning(self, lanes_per_cand=0, visited_bits=0, warps_per_block=0,
                   blocks_per_sm=0, mode=0, heap_warps=0, heap_scap=0,
                   replay_warps=0, replay_all=0, small_batch=0) -> None:
        """Launch shape (lqg_set_tuning; 0 keeps a field). small_batch: batches
        of at most this many queries run one query per block of 4 warps
        (_capi.SMALL_BATCH_AUTO: as many as fit at once; SMALL_BATCH_OFF: never)."""
        t = Tuning(lanes_per_cand, visited_bits, warps_per_block, blocks_per_sm, mode,
                   heap_warps, heap_scap, replay_warps, replay_all, small_batch)
        check(lib().lqg_set_tuning(self.handle, C.byref(t)))

    def get_tuning(self) -> dict:
        t = Tuning()
        check(lib().lqg_get_tuning(self.handle, C.byref(t)))
        return {f: int(getattr(t, f)) for f, _ in Tuning._fields_}

    # -- FastScan / RaBitQ search (upstream search_qg) -------------------
    def fastscan_build(self, seed: int = 0) -> None:
        """Writes the FastScan section for the current graph: a seeded rotation,
        and per node the RaBitQ codes and factors of its neighbours."""
        check(lib().lqg_fs_build(self.handle, int(seed)))

    def fastscan_arrays(self):
        """(diag[P], packed[N][deg*P/8] in upstream's FastScan block layout,
        factors[N][3][deg])."""
        P = C.c_uint32()
        check(lib().lqg_fs_get_arrays(self.handle, C.byref(P), None, None, None))
        n, g = self.num_elements, self.degree_bound
        diag = np.empty(P.value, np.float32)
        packed = np.empty((n, g * P.value // 8), np.uint8)
        fac = np.empty((n, 3, g), np.float32)
        check(lib().lqg_fs_get_arrays(self.handle, None, _p(diag), _p(packed), _p(fac)))
        return diag, packed, fac

    def set_fastscan_arrays(self, diag, packed, factors) -> None:
        d = _as_f32(diag)
        pk = np.ascontiguousarray(packed, dtype=np.uint8)
        fc = _as_f32(factors)
        P = 1
        while P < self.dimension:
            P <<= 1
        n, g = self.num_elements, self.degree_bound
        if d.shape != (P,) or pk.size != n * g * P // 8 or fc.size != n * 3 * g:
            raise ValueError("FastScan array shapes do not match the index")
        check(lib().lqg_fs_set_arrays(self.handle, _p(d), _p(pk), _p(fc)))

    def search_fastscan(self, query, k: int, ef=None, return_stats: bool = False):
        """Upstream's search_qg: the k nearest popped nodes by exact distance.
        ``ef`` (int or per-row array) overrides set_ef. A 1-D query returns
        uint32[k]; a 2-D block uint32[M, k]. Slots the reference's result
        buffer never fills hold 0, as in the reference."""
        q = _as_f32(query)
        one = q.ndim == 1
        if one:
            q = q.reshape(1, -1)
        if q.ndim != 2 or q.shape[1] != self.dimension:
            raise ValueError("query must be [D] or [M, D] with D the index dimension")
        k = int(k)
        if k < 1:
            raise ValueError("k must be >= 1")
        m = q.shape[0]
        ef_arr, ef0 = None, 0
        if ef is not None:
            if np.ndim(ef) == 0:
                ef0 = int(ef)
            else:
                ef_arr = np.ascontiguousarray(ef, dtype=np.uint32)
                if ef_arr.shape != (m,):
                    raise ValueError("per-query ef must have one value per query row")
                ef0 = int(ef_arr.max()) if m else 1
        ids = np.full((m, k), LQG_NO_ID, dtype=np.uint32)
        stats = np.zeros((m, 4), dtype=np.uint32) if return_stats else None
        if m:
            check(lib().lqg_fs_search_batch(self.handle, _p(q), m, None, k, _p(ef_arr), ef0,
                                            _p(ids), k, _p(stats), None))
        res = ids[0] if one else ids
        return (res, stats) if return_stats else res

    def search_fastscan_device(self, q_ptr: int, m: int, k: int, ids_ptr: int, kstride: int,
                               ef: int = 0, ef_ptr: int = 0, k_ptr: int = 0, stats_ptr: int = 0,
                               stream: int = 0) -> None:
        check(lib().lqg_fs_search_batch_device(self.handle, q_ptr, m, k_ptr or None, k,
                                               ef_ptr or None, ef, ids_ptr, kstride,
                                               stats_ptr or None, stream or None))

    def fastscan_status(self, stream: int = 0) -> None:
        check(lib().lqg_fs_stream_status(self.handle, stream or None))

    # Device-pointer entry points (pointers as ints; stream as int handle).
    def search_device(self, q_ptr: int, m: int, k: int, ids_ptr: int, kstride: int, ef: int = 0,
                      ef_ptr: int = 0, k_ptr: int = 0, pool_ids_ptr: int = 0,
                      pool_d_ptr: int = 0, pstride: int = 0, stats_ptr: int = 0,
                      stream: int = 0, exact: bool = False) -> None:
        f = lib().lqg_search_exact_device if exact else lib().lqg_search_batch_device
        check(f(self.handle, q_ptr, m, k_ptr or None, k, ef_ptr or None, ef, ids_ptr, kstride,
                pool_ids_ptr or None, pool_d_ptr or None, pstride, stats_ptr or None,
                stream or None))

    def set_kernel_events(self, start: int = 0, stop: int = 0) -> None:
        """cudaEvent_t handles (ints) recorded around each fast-kernel launch."""
        check(lib().lqg_set_kernel_events(self.handle, start or None, stop or None))

    def stream_status(self, stream: int = 0) -> None:
        check(lib().lqg_stream_status(self.handle, stream or None))
