"""Test infrastructure: Python access to the CPU checkers.

* ``Oracle`` wraps ``oracle/_lib/liblqg_oracle.so`` (the plain-C restatement of
  the reference's query path, ``lqg_oracle.c``).
* ``RefHarness`` wraps ``oracle/_ref/libref_harness.so``: the reference's own
  ``QuantizedGraph::search`` / ``QGBuilder`` compiled from its sources by
  ``oracle/Makefile`` (present only where the reference sources were available
  at build time, or where the built file travelled with the repository).
* ``read_index`` / ``write_index`` parse and write the reference's index file
  (``symqglib/qg/qg.hpp:206-224``): ``u32 entry`` | ``f32 data[N][D+deg]`` (raw
  vector, then ``deg`` u32 neighbour ids bit-cast into the row) |
  ``u8 codes[N][D]`` | ``f32 params[D][2]`` (min, scale). No header.

Only tests/, ``__graft_entry__.smoke`` and bench.py's CPU-baseline legs import
this module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_lib", "liblqg_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_harness.so")

SENTINEL = 0xFFFFFFFF


def index_nbytes(n: int, dim: int, deg: int) -> int:
    return 4 + 4 * n * (dim + deg) + n * dim + 8 * dim


@dataclass
class IndexArrays:
    n: int
    dim: int
    deg: int
    entry: int
    vectors: np.ndarray  # f32 [n, dim] (raw vectors as stored)
    nbrs: np.ndarray  # u32 [n, deg]
    codes: np.ndarray  # u8 [n, dim]
    params: np.ndarray  # f32 [dim, 2]


def read_index(path: str, n: int, dim: int, deg: int) -> IndexArrays:
    size = os.path.getsize(path)
    want = index_nbytes(n, dim, deg)
    if size != want:
        raise ValueError(f"{path}: {size} bytes, expected {want} for n={n} dim={dim} deg={deg}")
    raw = np.fromfile(path, dtype=np.uint8)
    entry = int(raw[:4].view(np.uint32)[0])
    off = 4
    rows = raw[off : off + 4 * n * (dim + deg)].view(np.uint32).reshape(n, dim + deg)
    off += 4 * n * (dim + deg)
    codes = raw[off : off + n * dim].reshape(n, dim)
    off += n * dim
    params = raw[off : off + 8 * dim].view(np.float32).reshape(dim, 2)
    return IndexArrays(
        n, dim, deg, entry,
        np.ascontiguousarray(rows[:, :dim]).view(np.float32),
        np.ascontiguousarray(rows[:, dim:]),
        np.ascontiguousarray(codes),
        np.ascontiguousarray(params),
    )


def write_index(path: str, ix: IndexArrays) -> None:
    rows = np.empty((ix.n, ix.dim + ix.deg), dtype=np.uint32)
    rows[:, : ix.dim] = np.ascontiguousarray(ix.vectors, dtype=np.float32).view(np.uint32)
    rows[:, ix.dim :] = ix.nbrs
    with open(path, "wb") as f:
        f.write(np.uint32(ix.entry).tobytes())
        f.write(rows.tobytes())
        f.write(np.ascontiguousarray(ix.codes, dtype=np.uint8).tobytes())
        f.write(np.ascontiguousarray(ix.params, dtype=np.float32).tobytes())


class _LqgoIndex(C.Structure):
    _fields_ = [
        ("nbrs", C.c_void_p),
        ("codes", C.c_void_p),
        ("params", C.c_void_p),
        ("n", C.c_uint64),
        ("dim", C.c_uint32),
        ("deg", C.c_uint32),
        ("entry", C.c_uint32),
        ("lanes", C.c_int),
    ]


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class SearchResult:
    compat: np.ndarray  # u32 [m, kmax]  what the reference search() writes
    pool_ids: np.ndarray | None  # u32 [m, efmax] ascending pool
    pool_d: np.ndarray | None  # f32 [m, efmax]
    pool_n: np.ndarray | None  # i32 [m]
    pops: np.ndarray | None
    evals: np.ndarray | None


class Oracle:
    """CPU restatement of the reference search over one index."""

    def __init__(self, ix: IndexArrays, lanes: int = 16):
        if not os.path.exists(ORACLE_SO):
            raise FileNotFoundError(f"{ORACLE_SO} not built (make -C oracle)")
        self.lib = C.CDLL(ORACLE_SO)
        self.lib.lqgo_search_batch.restype = C.c_int
        self.lib.lqgo_sq8_l2.restype = C.c_float
        self.ix = ix
        self._keep = (
            np.ascontiguousarray(ix.nbrs, dtype=np.uint32),
            np.ascontiguousarray(ix.codes, dtype=np.uint8),
            np.ascontiguousarray(ix.params, dtype=np.float32),
        )
        self.c = _LqgoIndex(
            _ptr(self._keep[0]), _ptr(self._keep[1]), _ptr(self._keep[2]),
            ix.n, ix.dim, ix.deg, ix.entry, lanes,
        )

    def search(self, q, k, ef, nthreads: int = 0, pool: bool = True) -> SearchResult:
        q = np.ascontiguousarray(np.atleast_2d(q), dtype=np.float32)
        m = q.shape[0]
        ka = np.broadcast_to(np.asarray(k, dtype=np.int32), (m,)).copy()
        ea = np.broadcast_to(np.asarray(ef, dtype=np.int32), (m,)).copy()
        kmax, efmax = int(ka.max()), int(max(ea.max(), 1))
        compat = np.full((m, kmax), SENTINEL, dtype=np.uint32)
        pid = np.full((m, efmax), SENTINEL, dtype=np.uint32) if pool else None
        pd = np.full((m, efmax), np.inf, dtype=np.float32) if pool else None
        pn = np.zeros(m, dtype=np.int32)
        pops = np.zeros(m, dtype=np.int32)
        evals = np.zeros(m, dtype=np.int32)
        r = self.lib.lqgo_search_batch(
            C.byref(self.c), _ptr(q), C.c_int64(m), _ptr(ka), 0, _ptr(ea), 0,
            kmax, efmax, _ptr(compat), _ptr(pid), _ptr(pd), _ptr(pn), _ptr(pops),
            _ptr(evals), nthreads,
        )
        if r != 0:
            raise MemoryError("oracle search failed")
        return SearchResult(compat, pid, pd, pn, pops, evals)

    def sq8_l2(self, q, ids) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.float32)
        codes = self._keep[1]
        out = np.empty(len(ids), dtype=np.float32)
        for i, v in enumerate(ids):
            out[i] = self.lib.lqgo_sq8_l2(
                _ptr(q), _ptr(codes[v]), _ptr(self._keep[2]), self.ix.dim, self.c.lanes
            )
        return out


def sq8_quantize(data: np.ndarray, recip: int = 0):
    """The oracle's restatement of the reference SQ8 encoder."""
    lib = C.CDLL(ORACLE_SO)
    data = np.ascontiguousarray(data, dtype=np.float32)
    n, dim = data.shape
    codes = np.empty((n, dim), dtype=np.uint8)
    params = np.empty((dim, 2), dtype=np.float32)
    lib.lqgo_sq8_quantize(_ptr(data), C.c_uint64(dim), C.c_uint64(n), _ptr(codes), _ptr(params), recip)
    return codes, params


def ref_available() -> bool:
    return os.path.exists(REF_SO)


class RefHarness:
    """The reference's own search/build code (compiled from its sources)."""

    def __init__(self):
        if not ref_available():
            raise FileNotFoundError(f"{REF_SO} not built (make -C oracle ref)")
        self.lib = C.CDLL(REF_SO)
        self.lib.ref_open.restype = C.c_void_p
        self.lib.ref_open.argtypes = [C.c_char_p, C.c_uint64, C.c_uint64, C.c_uint64]
        self.lib.ref_close.argtypes = [C.c_void_p]
        self.lib.ref_entry_point.restype = C.c_uint32
        self.lib.ref_entry_point.argtypes = [C.c_void_p]
        self.lib.ref_search.argtypes = [
            C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p, C.c_int,
        ]
        self.lib.ref_build.argtypes = [
            C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
            C.c_int, C.c_char_p,
        ]
        self.lib.ref_sq8_quantize.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p]
        self.lib.ref_sq8_l2.argtypes = [
            C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p,
        ]

    def isa_lanes(self) -> int:
        return int(self.lib.ref_isa())

    def build(self, data, deg, ef_build, num_iter, path, nthreads=0):
        data = np.ascontiguousarray(data, dtype=np.float32)
        n, dim = data.shape
        self.lib.ref_build(_ptr(data), n, dim, deg, ef_build, num_iter, nthreads, path.encode())

    def open(self, path, n, dim, deg):
        return _RefIndex(self, path, n, dim, deg)

    def sq8_quantize(self, data):
        data = np.ascontiguousarray(data, dtype=np.float32)
        n, dim = data.shape
        codes = np.empty((n, dim), dtype=np.uint8)
        params = np.empty((dim, 2), dtype=np.float32)
        self.lib.ref_sq8_quantize(_ptr(data), dim, n, _ptr(codes), _ptr(params))
        return codes, params

    def sq8_l2(self, q, codes, params):
        q = np.ascontiguousarray(q, dtype=np.float32)
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        params = np.ascontiguousarray(params, dtype=np.float32)
        out = np.empty(codes.shape[0], dtype=np.float32)
        self.lib.ref_sq8_l2(_ptr(q), _ptr(codes), codes.shape[0], codes.shape[1], _ptr(params), _ptr(out))
        return out


class _RefIndex:
    def __init__(self, h: RefHarness, path, n, dim, deg):
        self.h, self.dim = h, dim
        self.handle = h.lib.ref_open(path.encode(), n, dim, deg)

    def entry(self) -> int:
        return int(self.h.lib.ref_entry_point(self.handle))

    def search(self, q, k, ef, nthreads=0) -> np.ndarray:
        """Reference search() per query; unwritten slots stay SENTINEL."""
        q = np.ascontiguousarray(np.atleast_2d(q), dtype=np.float32)
        out = np.full((q.shape[0], k), SENTINEL, dtype=np.uint32)
        self.h.lib.ref_search(self.handle, _ptr(q), q.shape[0], k, ef, _ptr(out), nthreads)
        return out

    def close(self):
        if self.handle:
            self.h.lib.ref_close(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
