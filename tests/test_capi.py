"""The C-ABI library: loads, exports every declared symbol, validates input (no GPU)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from liteqg_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "lqg.h")).read()
    return sorted(set(re.findall(r"^LQG_API[^(]*?\b(lqg_\w+)\s*\(", hdr, flags=re.M)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 15
    lib = _capi.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.library_path()],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (lqg_\w+)", out))
    for s in syms:
        assert s in exported, s
        assert hasattr(lib, s), s
        assert s in _capi.SIGNATURES, s
    assert set(_capi.SIGNATURES) == set(syms)


def test_library_is_sm100a_only():
    out = subprocess.run(["cuobjdump", "--list-elf", _capi.library_path()],
                         capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    arches = set(re.findall(r"sm_(\d+a?)", out.stdout))
    assert arches == {"100a"}, arches


def _create(t="QG", m="L2", n=1000, d=64, g=32):
    h = C.c_void_p()
    st = _capi.lib().lqg_create(t.encode(), m.encode(), n, d, g, 0, C.byref(h))
    return st, h


@pytest.mark.parametrize("args,frag", [
    (dict(m="IP"), "Only L2"),
    (dict(g=48), "multiple of 32"),
    (dict(g=0), "multiple of 32"),
    (dict(t="HNSW"), "not supported"),
    (dict(d=32), "dimension"),
    (dict(d=4096), "dimension"),
    (dict(g=256), "above 128"),
])
def test_create_rejects_like_the_reference(args, frag):
    st, h = _create(**args)
    assert st == 1
    assert frag in _capi.lib().lqg_last_error().decode()
    assert not h.value


def test_python_index_raises_value_error():
    from liteqg_b200 import Index
    with pytest.raises(ValueError, match="Only L2"):
        Index("QG", "IP", 100, 64)
