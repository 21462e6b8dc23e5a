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


# ---- upstream FastScan / RaBitQ path --------------------------------------

class _FsoIndex(C.Structure):
    _fields_ = [
        ("vectors", C.c_void_p),
        ("nbrs", C.c_void_p),
        ("codes", C.c_void_p),
        ("factors", C.c_void_p),
        ("diag", C.c_void_p),
        ("n", C.c_uint64),
        ("dim", C.c_uint32),
        ("P", C.c_uint32),
        ("deg", C.c_uint32),
        ("entry", C.c_uint32),
    ]


def padded_dim(dim: int) -> int:
    p = 1
    while p < dim:
        p <<= 1
    return p


@dataclass
class FsArrays:
    """A FastScan index: graph + raw vectors + per-node neighbour codes/factors.
    codes [n][deg][P/8] (byte b: 4-dimension groups 2b low nibble, 2b+1 high
    nibble, the group's first dimension on the nibble's bit 3); factors
    [n][3][deg] (triple_x, factor_dq, factor_vq); diag [P]."""
    n: int
    dim: int
    deg: int
    entry: int
    vectors: np.ndarray
    nbrs: np.ndarray
    codes: np.ndarray
    factors: np.ndarray
    diag: np.ndarray

    @property
    def P(self) -> int:
        return padded_dim(self.dim)


class FsOracle:
    """CPU restatement of the upstream sorted-buffer FastScan search (fs_oracle.c)."""

    def __init__(self, fs: FsArrays | None = None):
        self.lib = C.CDLL(ORACLE_SO)
        self.lib.fso_l2.restype = C.c_float
        self.lib.fso_search_batch.restype = C.c_int
        self.fs = fs
        if fs is not None:
            self._keep = (np.ascontiguousarray(fs.vectors, np.float32),
                          np.ascontiguousarray(fs.nbrs, np.uint32),
                          np.ascontiguousarray(fs.codes, np.uint8),
                          np.ascontiguousarray(fs.factors, np.float32),
                          np.ascontiguousarray(fs.diag, np.float32))
            self.c = _FsoIndex(*[_ptr(a) for a in self._keep], fs.n, fs.dim, fs.P, fs.deg,
                               fs.entry)

    def rotate(self, x, diag):
        x = np.ascontiguousarray(np.atleast_2d(x), np.float32)
        diag = np.ascontiguousarray(diag, np.float32)
        P = len(diag)
        out = np.empty((x.shape[0], P), np.float32)
        for i in range(x.shape[0]):
            self.lib.fso_rotate(_ptr(x[i]), x.shape[1], P, _ptr(diag), _ptr(out[i]))
        return out

    def query_prepare(self, rot):
        rot = np.ascontiguousarray(rot, np.float32)
        P = len(rot)
        lut = np.empty(P * 4, np.uint8)
        w, lo, sq = C.c_float(), C.c_float(), C.c_int32()
        self.lib.fso_query_prepare(_ptr(rot), P, _ptr(lut), C.byref(w), C.byref(lo), C.byref(sq))
        return lut, w.value, lo.value, sq.value

    def rabitq(self, rot_nb, rot_c):
        rot_nb = np.ascontiguousarray(rot_nb, np.float32)
        rot_c = np.ascontiguousarray(rot_c, np.float32)
        deg, P = rot_nb.shape
        bits = np.empty((deg, P // 8), np.uint8)
        fac = np.empty((3, deg), np.float32)
        self.lib.fso_rabitq(_ptr(rot_nb), _ptr(rot_c), deg, P, _ptr(bits), _ptr(fac))
        return bits, fac

    def pack(self, bits):
        bits = np.ascontiguousarray(bits, np.uint8)
        ncode, rowb = bits.shape
        out = np.empty(ncode * rowb, np.uint8)
        self.lib.fso_pack_codes(_ptr(bits), ncode, rowb * 8, _ptr(out))
        return out

    def unpack(self, packed, ncode, P):
        packed = np.ascontiguousarray(packed, np.uint8)
        bits = np.empty((ncode, P // 8), np.uint8)
        self.lib.fso_unpack_codes(_ptr(packed), ncode, P, _ptr(bits))
        return bits

    def accumulate(self, bits, lut):
        bits = np.ascontiguousarray(bits, np.uint8)
        lut = np.ascontiguousarray(lut, np.uint8)
        ncode, rowb = bits.shape
        res = np.empty(ncode, np.uint16)
        self.lib.fso_accumulate(_ptr(bits), ncode, rowb * 8, _ptr(lut), _ptr(res))
        return res

    def estimate(self, res, sumq, width, lower, sqr_y, factors):
        res = np.ascontiguousarray(res, np.uint16)
        factors = np.ascontiguousarray(factors, np.float32)
        out = np.empty(len(res), np.float32)
        self.lib.fso_estimate(_ptr(res), len(res), C.c_int32(sumq), C.c_float(width),
                              C.c_float(lower), C.c_float(sqr_y), _ptr(factors), _ptr(out))
        return out

    def l2(self, a, b):
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        return float(self.lib.fso_l2(_ptr(a), _ptr(b), len(a)))

    def search(self, q, k, ef, nthreads: int = 0):
        """ids [m][max k] (the reference's copy-out; never-filled slots 0) and
        stats [m][4]: buffer pops, exact evaluations of popped nodes, exact
        evaluations in update_results, result count."""
        q = np.ascontiguousarray(np.atleast_2d(q), np.float32)
        m = q.shape[0]
        ka = np.broadcast_to(np.asarray(k, np.int32), (m,)).copy()
        ea = np.broadcast_to(np.asarray(ef, np.int32), (m,)).copy()
        kmax = int(ka.max())
        ids = np.zeros((m, kmax), np.uint32)
        st = np.zeros((m, 4), np.int32)
        r = self.lib.fso_search_batch(C.byref(self.c), _ptr(q), C.c_int64(m), _ptr(ka), _ptr(ea),
                                      _ptr(ids), kmax, _ptr(st), nthreads)
        if r != 0:
            raise MemoryError("FastScan oracle search failed")
        return ids, st


def fs_encode(vectors, nbrs, diag, oracle: FsOracle | None = None):
    """Per-node neighbour codes and factors of a graph (oracle restatement)."""
    o = oracle or FsOracle()
    vectors = np.ascontiguousarray(vectors, np.float32)
    n, dim = vectors.shape
    deg = nbrs.shape[1]
    P = len(diag)
    rot = o.rotate(vectors, diag)
    codes = np.empty((n, deg, P // 8), np.uint8)
    fac = np.empty((n, 3, deg), np.float32)
    for i in range(n):
        codes[i], fac[i] = o.rabitq(rot[nbrs[i]], rot[i])
    return codes, fac


class RefFastScan:
    """The reference's own upstream FastScan/RaBitQ functions (oracle/_ref)."""

    def __init__(self):
        self.lib = C.CDLL(REF_SO)
        self.lib.ref_fs_open.restype = C.c_void_p
        self.lib.ref_fs_open.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32] + \
            [C.c_void_p] * 5
        self.lib.ref_fs_close.argtypes = [C.c_void_p]
        self.lib.ref_fs_search.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int,
                                           C.c_void_p, C.c_int]
        self.lib.ref_fs_rotate.argtypes = [C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint64,
                                           C.c_void_p]
        self.lib.ref_fs_query_prepare.argtypes = [C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        self.lib.ref_fs_rabitq.argtypes = [C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p]
        self.lib.ref_fs_scan.argtypes = [C.c_uint64, C.c_uint64, C.c_void_p, C.c_float,
                                         C.c_float, C.c_float, C.c_int32, C.c_void_p, C.c_void_p,
                                         C.c_void_p]

    def rotate(self, x, diag):
        x = np.ascontiguousarray(np.atleast_2d(x), np.float32)
        diag = np.ascontiguousarray(diag, np.float32)
        out = np.empty((x.shape[0], len(diag)), np.float32)
        self.lib.ref_fs_rotate(x.shape[1], _ptr(diag), _ptr(x), x.shape[0], _ptr(out))
        return out

    def query_prepare(self, q, diag, deg=32):
        q = np.ascontiguousarray(q, np.float32)
        diag = np.ascontiguousarray(diag, np.float32)
        lut = np.empty(len(diag) * 4, np.uint8)
        w, lo, sq = C.c_float(), C.c_float(), C.c_int32()
        self.lib.ref_fs_query_prepare(len(q), deg, _ptr(diag), _ptr(q), _ptr(lut), C.byref(w),
                                      C.byref(lo), C.byref(sq))
        return lut, w.value, lo.value, sq.value

    def rabitq(self, rot_nb, rot_c):
        rot_nb = np.ascontiguousarray(rot_nb, np.float32)
        rot_c = np.ascontiguousarray(rot_c, np.float32)
        deg, P = rot_nb.shape
        packed = np.empty(deg * P // 8, np.uint8)
        fac = np.empty((3, deg), np.float32)
        self.lib.ref_fs_rabitq(P, deg, _ptr(rot_nb), _ptr(rot_c), _ptr(packed), _ptr(fac))
        return packed, fac

    def scan(self, lut, sqr_y, lower, width, sumq, packed, factors, deg):
        lut = np.ascontiguousarray(lut, np.uint8)
        packed = np.ascontiguousarray(packed, np.uint8)
        factors = np.ascontiguousarray(factors, np.float32)
        out = np.empty(deg, np.float32)
        self.lib.ref_fs_scan(len(lut) // 4, deg, _ptr(lut), sqr_y, lower, width, sumq,
                             _ptr(packed), _ptr(factors), _ptr(out))
        return out

    def open(self, n, dim, deg, entry, vectors, nbrs, packed, factors, diag):
        """The reference's QuantizedGraph with upstream's row layout, filled from
        arrays (packed codes in the FastScan block layout)."""
        return _RefFsIndex(self, n, dim, deg, entry, vectors, nbrs, packed, factors, diag)

    def search(self, fs: FsArrays, q, k, ef, nthreads=0):
        o = FsOracle()
        packed = np.stack([o.pack(fs.codes[i]) for i in range(fs.n)])
        h = self.open(fs.n, fs.dim, fs.deg, fs.entry, fs.vectors, fs.nbrs, packed, fs.factors,
                      fs.diag)
        try:
            return h.search(q, k, ef, nthreads)
        finally:
            h.close()


class _RefFsIndex:
    def __init__(self, r: RefFastScan, n, dim, deg, entry, vectors, nbrs, packed, factors, diag):
        self.r, self.dim = r, dim
        keep = (np.ascontiguousarray(vectors, np.float32), np.ascontiguousarray(nbrs, np.uint32),
                np.ascontiguousarray(packed, np.uint8), np.ascontiguousarray(factors, np.float32),
                np.ascontiguousarray(diag, np.float32))
        self.handle = r.lib.ref_fs_open(n, dim, deg, entry, *[_ptr(a) for a in keep])

    def search(self, q, k, ef, nthreads=0):
        """The reference's search() with search_qg, per query, on nthreads threads."""
        q = np.ascontiguousarray(np.atleast_2d(q), np.float32)
        out = np.zeros((q.shape[0], k), np.uint32)
        self.r.lib.ref_fs_search(self.handle, _ptr(q), q.shape[0], k, ef, _ptr(out), nthreads)
        return out

    def close(self):
        if self.handle:
            self.r.lib.ref_fs_close(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
