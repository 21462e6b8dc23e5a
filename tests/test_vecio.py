"""Vector-file I/O (.fvecs/.ivecs/.fbin/.ibin) against the reference's layouts."""
import numpy as np
import pytest

from liteqg_b200 import vecio


def test_fvecs_layout_and_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    x = rng.random((7, 5), dtype=np.float32)
    p = str(tmp_path / "a.fvecs")
    vecio.write_fvecs(p, x)
    raw = np.fromfile(p, dtype=np.int32).reshape(7, 6)
    assert (raw[:, 0] == 5).all()  # every row: int32 d, then d values
    assert np.array_equal(raw[:, 1:].view(np.float32), x)
    assert np.array_equal(vecio.read_fvecs(p), x)
    assert np.array_equal(np.asarray(vecio.read_fvecs(p, mmap=True)), x)


def test_ivecs_roundtrip(tmp_path):
    gt = np.arange(30, dtype=np.int32).reshape(3, 10)
    p = str(tmp_path / "gt.ivecs")
    vecio.write_ivecs(p, gt)
    assert np.array_equal(vecio.read_ivecs(p), gt)


def test_vecs_rejects_inconsistent_rows(tmp_path):
    p = str(tmp_path / "bad.fvecs")
    rows = np.array([[3, 0, 0, 0], [4, 0, 0, 0]], dtype=np.int32)
    rows.tofile(p)
    with pytest.raises(ValueError, match="row 1 has dimension 4"):
        vecio.read_fvecs(p)
    np.array([3, 1, 2, 3, 3, 1], dtype=np.int32).tofile(p)  # a partial second row
    with pytest.raises(ValueError, match="whole number"):
        vecio.read_fvecs(p)


def test_fbin_header_ranges_and_errors(tmp_path):
    rng = np.random.default_rng(1)
    x = rng.random((11, 4), dtype=np.float32)
    p = str(tmp_path / "b.fbin")
    vecio.write_fbin(p, x)
    hdr = np.fromfile(p, dtype=np.int32, count=2)
    assert hdr.tolist() == [11, 4]
    assert np.array_equal(vecio.read_fbin(p), x)
    assert np.array_equal(vecio.read_fbin(p, start=3, count=5), x[3:8])
    assert np.array_equal(np.asarray(vecio.read_fbin(p, start=9, mmap=True)), x[9:])
    with pytest.raises(ValueError, match="outside"):
        vecio.read_fbin(p, start=8, count=5)
    with open(p, "ab") as f:
        f.write(b"\0\0\0\0")
    with pytest.raises(ValueError, match="header says"):
        vecio.read_fbin(p)
    q = str(tmp_path / "ids.ibin")
    vecio.write_ibin(q, np.arange(12, dtype=np.int32).reshape(3, 4))
    assert vecio.read_ibin(q, start=1).tolist() == [[4, 5, 6, 7], [8, 9, 10, 11]]
