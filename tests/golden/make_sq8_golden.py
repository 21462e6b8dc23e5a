"""Generates tests/golden/sq8_signed_zero.npz: the reference's SQ8 encoder
(quantization/sq8.hpp:11-25, compiled from its sources with its own -Ofast
flags into oracle/_ref) on rounded integer data that holds both -0.0 and 0.0
in every column, so the minimum's sign - and with it the index file's bytes -
depends on which of the equal values the compiled std::min keeps.

usage: python tests/golden/make_sq8_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import RefHarness  # noqa: E402


def signed_zero_data(seed=8, n=400, dim=48):
    """Rounded N(0, 3) clipped at 0 (np.rint keeps the sign of small negative
    values, np.clip keeps -0.0); the first and the last rows set so that the
    first and the last zero of a column differ in sign for every column."""
    rng = np.random.default_rng(seed)
    x = np.clip(np.rint(rng.normal(0.0, 3.0, (n, dim))), 0, 255).astype(np.float32)
    h = dim // 2
    x[0, :h], x[0, h:] = 0.0, -0.0
    x[-1, :h], x[-1, h:] = -0.0, 0.0
    return x


def main():
    x = signed_zero_data()
    codes, params = RefHarness().sq8_quantize(x)
    np.savez_compressed(os.path.join(HERE, "sq8_signed_zero.npz"), x=x, codes=codes, params=params)
    print("min sign bits:", np.signbit(params[:, 0]).astype(int))


if __name__ == "__main__":
    main()
