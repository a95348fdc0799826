"""Generate the golden 1D FFT vectors from the reference's own FFT code.

Runs the reference's fft_real (src/fft/fft_real_scalar.cpp) and fft_complex
(src/fft/fft_complex_vector.cpp), compiled from the reference tree into
oracle/_ref by `make -C oracle ref`, on seeded inputs, the way its own test
program does (src/fft/fft_test.cpp:81-159: scramble, then transform), and
stores inputs and outputs in fft1d_golden.npz.

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from oracle import oracle as O  # noqa: E402


def main():
    assert O.ref_fft_lib() is not None, "build oracle/_ref first (make -C oracle ref)"
    rng = np.random.Generator(np.random.PCG64(2023))
    out = {}
    for lg in range(3, 13):
        N = 1 << lg
        x = rng.uniform(0.0, 1.0, N)
        out["real_in_%d" % N] = x
        out["real_out_%d" % N] = O.ref_fft_real(x)
    for lg in range(3, 11):
        N = 1 << lg
        z = rng.uniform(0.0, 1.0, N) + 1j * rng.uniform(0.0, 1.0, N)
        out["cplx_in_%d" % N] = z
        out["cplx_out_%d" % N] = O.ref_fft_complex(z)
    np.savez_compressed(os.path.join(HERE, "fft1d_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
