import gzip
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ("u48", "bin40", "mix128d64")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    so = os.path.join(ROOT, "oracle", "_lib", "liblqg_oracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


@pytest.fixture(scope="session")
def golden(tmp_path_factory):
    """name -> dict(path, n, dim, deg, queries, expected {(ef, k): ids})."""
    d = tmp_path_factory.mktemp("golden")
    out = {}
    for name in GOLDEN_CASES:
        path = str(d / f"{name}.idx")
        with gzip.open(os.path.join(GOLDEN, f"{name}.idx.gz"), "rb") as f, open(path, "wb") as g:
            shutil.copyfileobj(f, g)
        z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
        exp = {}
        for key in z.files:
            if key.startswith("ids_ef"):
                ef, k = key[6:].split("_k")
                exp[(int(ef), int(k))] = z[key]
        out[name] = dict(path=path, n=int(z["n"]), dim=int(z["dim"]), deg=int(z["deg"]),
                         queries=z["queries"], expected=exp)
    return out
