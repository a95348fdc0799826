"""The reference's 1D FFT surface (cosmictiger/fft.hpp:18-27) on the GPU,
through the C ABI, against golden vectors the reference's own code produced
(tests/golden/fft1d_golden.npz, tests/golden/make_golden.py): fft_real in
its scalar and 4-lane forms, fft_complex, scramble, transpose_r2c and the
twiddle tables.  FP64 throughout; tolerance 1e-12 relative to the largest
output value (the golden values themselves carry the reference's FP64
rounding).  The parts where the reference does not compute what its callers
need (dir = -1, transpose_yz, transpose_c2r) are checked against their
definitions with numpy.
"""
import os

import numpy as np
import pytest

from ct2_b200.gravity import Gravity

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "fft1d_golden.npz"))
TOL = 1e-12


@pytest.fixture(scope="module")
def g():
    ctx = Gravity(mesh=8, order=1, bwidth=1.0, hsoft=0.01)
    yield ctx
    ctx.close()


def _bitrev_perm(N):
    b = int(np.log2(N))
    return np.array([int(format(i, "0%db" % b)[::-1], 2) if b else 0 for i in range(N)])


def _close(a, b):
    return np.abs(a - b).max() <= TOL * max(1.0, np.abs(b).max())


@pytest.mark.parametrize("lg", range(3, 13))
def test_fft_real_matches_reference(g, lg):
    N = 1 << lg
    x = GOLD["real_in_%d" % N]
    X = np.ascontiguousarray(x.copy())
    g.scramble(X, 1, N, 1)
    assert np.array_equal(X, x[_bitrev_perm(N)])
    g.fft1d_real(X, N, 1, 1)
    assert _close(X, GOLD["real_out_%d" % N])


@pytest.mark.parametrize("lg", (3, 6, 10))
def test_fft_real_four_lanes_matches_reference(g, lg):
    N = 1 << lg
    X = np.ascontiguousarray(GOLD["real4_in_%d" % N].copy().reshape(-1))
    g.scramble(X, 1, N, 4)
    g.fft1d_real(X, N, 4, 1)
    assert _close(X.reshape(N, 4), GOLD["real4_out_%d" % N])


@pytest.mark.parametrize("lg", range(3, 11))
def test_fft_complex_matches_reference(g, lg):
    N = 1 << lg
    z = GOLD["cplx_in_%d" % N]
    # complex<fft_simd>: four real lanes then four imaginary lanes per element
    X = np.zeros((N, 2, 4))
    X[:, 0, :] = z.real[:, None]
    X[:, 1, :] = z.imag[:, None]
    X = np.ascontiguousarray(X.reshape(-1))
    g.scramble(X, 1, N, 8)
    g.fft1d_complex(X, N, 4, 1)
    X = X.reshape(N, 2, 4)
    got = X[:, 0, :] + 1j * X[:, 1, :]
    for lane in range(4):
        assert _close(got[:, lane], GOLD["cplx_out_%d" % N])


@pytest.mark.parametrize("N", (2, 16, 4096, 8192))
def test_fft_dir_minus_one_is_the_opposite_sign(g, N):
    rng = np.random.Generator(np.random.PCG64(N))
    z = rng.normal(size=N) + 1j * rng.normal(size=N)
    X = np.ascontiguousarray(np.stack([z.real, z.imag], 1).reshape(-1))
    g.scramble(X, 1, N, 2)
    g.fft1d_complex(X, N, 1, -1)
    got = X[0::2] + 1j * X[1::2]
    want = np.fft.ifft(z) * N
    assert np.abs(got - want).max() <= TOL * np.abs(want).max()
    x = rng.normal(size=N)
    R = np.ascontiguousarray(x[_bitrev_perm(N)])
    g.fft1d_real(R, N, 1, -1)
    w = np.fft.ifft(x) * N
    assert np.allclose(R[: N // 2 + 1], w.real[: N // 2 + 1], rtol=0, atol=TOL * np.abs(w).max())
    k = np.arange(1, N // 2)
    assert np.allclose(R[N - k], w.imag[k], rtol=0, atol=TOL * np.abs(w).max())


def test_scramble_matches_reference(g):
    X = GOLD["scramble_in"].copy()
    g.scramble(X, 3, 16, 5)
    assert np.array_equal(X, GOLD["scramble_out"])


@pytest.mark.parametrize("N", (8, 16))
def test_transpose_r2c_matches_reference_and_c2r_inverts_it(g, N):
    x = GOLD["r2c_in_%d" % N]
    Y = np.zeros(2 * N * N * (N // 2 + 1))
    g.transpose_r2c(x, Y, N)
    assert np.array_equal(Y, GOLD["r2c_out_%d" % N])
    # transpose_c2r undoes it on every value transpose_r2c keeps: the rows
    # iy in [0, N/2] and the imaginary rows N - iy
    back = np.zeros(N ** 3)
    g.transpose_c2r(Y, back, N)
    xr = x.reshape(N, N, N)
    br = back.reshape(N, N, N)
    assert np.array_equal(br[:, : N // 2 + 1, :], xr[:, : N // 2 + 1, :])
    assert np.array_equal(br[:, N // 2 + 1:, :], xr[:, N // 2 + 1:, :])


def test_transpose_yz(g):
    N = 16
    x = np.arange(N ** 3, dtype=np.float64)
    X = x.copy()
    g.transpose_yz(X, N)
    assert np.array_equal(X.reshape(N, N, N), x.reshape(N, N, N).transpose(0, 2, 1))


def test_twiddles_match_reference(g):
    for which, nm in enumerate(("cos", "sin", "inv_sin")):
        w = g.twiddles(which, 64)
        # the reference takes libm cos/sin of the rounded argument -2 pi n/N;
        # the library takes cospi/sinpi of the exact 2n/N: a few ulp apart
        assert np.abs(w - GOLD["twiddle_%s_64" % nm]).max() <= 1.2e-15


def test_bad_sizes_are_refused(g):
    X = np.zeros(48)
    for call in (lambda: g.fft1d_real(X, 12, 1, 1), lambda: g.fft1d_real(X, 16, 1, 0),
                 lambda: g.scramble(X, 1, 12, 4)):
        with pytest.raises(Exception):
            call()
