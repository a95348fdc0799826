"""Generate the golden 1D FFT vectors from the reference's own FFT code.

Runs the reference's fft_real (src/fft/fft_real_scalar.cpp, and the 4-lane
src/fft/fft_real_vector.cpp) and fft_complex (src/fft/fft_complex_vector.cpp),
compiled from the reference tree into oracle/_ref by `make -C oracle ref`, on
seeded inputs, the way its own test program does (src/fft/fft_test.cpp:81-159:
scramble, then transform), plus its scramble, transpose_r2c and twiddle
tables (scramble.cpp, transpose.cpp, twiddles.cpp), and stores inputs and
outputs in fft1d_golden.npz.

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
    L = O.ref_fft_lib()
    for lg in (3, 6, 10):
        N = 1 << lg
        x = rng.uniform(0.0, 1.0, (N, 4))
        X = np.ascontiguousarray(x.copy().reshape(-1))
        L.ref_scramble(X, 1, N, 4)
        L.ref_fft_real4(X, N, 1)
        out["real4_in_%d" % N] = x
        out["real4_out_%d" % N] = X.reshape(N, 4)
    x = rng.uniform(0.0, 1.0, 3 * 16 * 5)
    X = x.copy()
    L.ref_scramble(X, 3, 16, 5)
    out["scramble_in"], out["scramble_out"] = x, X
    for N in (8, 16):
        x = rng.uniform(0.0, 1.0, N ** 3)
        Y = np.zeros(2 * N * N * (N // 2 + 1))
        L.ref_transpose_r2c(np.ascontiguousarray(x), Y, N)
        out["r2c_in_%d" % N], out["r2c_out_%d" % N] = x, Y
    for which, nm in enumerate(("cos", "sin", "inv_sin")):
        w = np.zeros(64)
        L.ref_twiddles(which, 64, w)
        out["twiddle_%s_64" % nm] = w
    np.savez_compressed(os.path.join(HERE, "fft1d_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
