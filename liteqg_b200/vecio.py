"""Vector-file I/O for real datasets (the formats the reference's tools read).

* ``.fvecs`` / ``.ivecs``: every row is an int32 dimension d followed by d
  float32 / int32 values (symqglib/utils/io.hpp:20-49 ``load_vecs``;
  reproduce/utils/io.py:3-27 ``ivecs_read``/``fvecs_read``/``*_write``).
* ``.fbin`` / ``.ibin`` (big-ann-benchmarks): an int32 row count n and an
  int32 dimension d, then n*d float32 / int32 values (io.hpp:51-76
  ``load_bin``; reproduce/utils/io.py ``read_fbin``/``read_ibin``, which can
  read a row range).

Readers validate what the reference's readers assume: every row of a
``*vecs`` file carries the same d, and the file holds whole rows (the C++
loader silently drops a partial last row; here that is an error). Large files
are read through ``np.memmap`` when ``mmap=True``.
"""
from __future__ import annotations

import os

import numpy as np

_DT = {"f": np.float32, "i": np.int32}


def _vecs(path: str, kind: str, mmap: bool) -> np.ndarray:
    raw = np.memmap(path, dtype=np.int32, mode="r") if mmap else np.fromfile(path, dtype=np.int32)
    if raw.size == 0:
        return np.empty((0, 0), _DT[kind])
    d = int(raw[0])
    if d <= 0:
        raise ValueError(f"{path}: bad dimension {d} in the first row")
    if raw.size % (d + 1):
        raise ValueError(f"{path}: {raw.size * 4} bytes is not a whole number of {d}-dim rows")
    rows = raw.reshape(-1, d + 1)
    if not (rows[:, 0] == d).all():
        bad = int(np.argmax(rows[:, 0] != d))
        raise ValueError(f"{path}: row {bad} has dimension {int(rows[bad, 0])}, expected {d}")
    out = rows[:, 1:]
    return out.view(_DT[kind]) if mmap else np.ascontiguousarray(out).view(_DT[kind])


def read_fvecs(path: str, mmap: bool = False) -> np.ndarray:
    """float32 [n, d] from an .fvecs file."""
    return _vecs(path, "f", mmap)


def read_ivecs(path: str, mmap: bool = False) -> np.ndarray:
    """int32 [n, d] from an .ivecs file (e.g. ground-truth neighbour ids)."""
    return _vecs(path, "i", mmap)


def _write_vecs(path: str, m, kind: str) -> None:
    a = np.ascontiguousarray(m, dtype=_DT[kind])
    if a.ndim != 2:
        raise ValueError("expected a 2-D array")
    n, d = a.shape
    out = np.empty((n, d + 1), dtype=np.int32)
    out[:, 0] = d
    out[:, 1:] = a.view(np.int32)
    out.tofile(path)


def write_fvecs(path: str, m) -> None:
    _write_vecs(path, m, "f")


def write_ivecs(path: str, m) -> None:
    _write_vecs(path, m, "i")


def _bin(path: str, kind: str, start: int, count: int | None, mmap: bool) -> np.ndarray:
    with open(path, "rb") as f:
        hdr = np.fromfile(f, dtype=np.int32, count=2)
    if hdr.size != 2:
        raise ValueError(f"{path}: missing the (n, d) header")
    n, d = int(hdr[0]), int(hdr[1])
    if n < 0 or d <= 0:
        raise ValueError(f"{path}: bad header n={n} d={d}")
    want = 8 + 4 * n * d
    size = os.path.getsize(path)
    if size != want:
        raise ValueError(f"{path}: {size} bytes, the header says {want}")
    if start < 0 or start > n:
        raise ValueError(f"start {start} outside [0, {n}]")
    cnt = n - start if count is None else int(count)
    if cnt < 0 or start + cnt > n:
        raise ValueError(f"rows [{start}, {start + cnt}) outside [0, {n})")
    off = 8 + 4 * start * d
    if mmap:
        return np.memmap(path, dtype=_DT[kind], mode="r", offset=off, shape=(cnt, d))
    with open(path, "rb") as f:
        f.seek(off)
        return np.fromfile(f, dtype=_DT[kind], count=cnt * d).reshape(cnt, d)


def read_fbin(path: str, start: int = 0, count: int | None = None, mmap: bool = False) -> np.ndarray:
    """float32 rows [start, start + count) of an .fbin file (all by default)."""
    return _bin(path, "f", start, count, mmap)


def read_ibin(path: str, start: int = 0, count: int | None = None, mmap: bool = False) -> np.ndarray:
    """int32 rows [start, start + count) of an .ibin file (all by default)."""
    return _bin(path, "i", start, count, mmap)


def _write_bin(path: str, m, kind: str) -> None:
    a = np.ascontiguousarray(m, dtype=_DT[kind])
    if a.ndim != 2:
        raise ValueError("expected a 2-D array")
    with open(path, "wb") as f:
        np.asarray(a.shape, dtype=np.int32).tofile(f)
        a.tofile(f)


def write_fbin(path: str, m) -> None:
    _write_bin(path, m, "f")


def write_ibin(path: str, m) -> None:
    _write_bin(path, m, "i")
