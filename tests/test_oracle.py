"""CPU tests of the oracle itself: pins against the reference's own FFT
golden vectors, known physics answers, and the restated bisection."""
import numpy as np
import pytest

from oracle import oracle as O
from ct2_b200 import ics

GOLD = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                          "fft1d_golden.npz"))


@pytest.mark.parametrize("N", [8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096])
def test_numpy_fft_matches_reference_real_fft(N):
    # src/fft/fft_test.cpp:132-159 compares fft_real with FFTW; FFTW is absent,
    # numpy's pocketfft stands in and is pinned here against the reference's output
    x = GOLD["real_in_%d" % N]
    hc = O.halfcomplex_to_complex(GOLD["real_out_%d" % N])
    ref = np.fft.rfft(x)
    assert np.abs(ref - hc).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("N", [8, 16, 32, 64, 128, 256, 512, 1024])
def test_numpy_fft_matches_reference_complex_fft(N):
    z = GOLD["cplx_in_%d" % N]
    Z = GOLD["cplx_out_%d" % N]
    assert np.abs(np.fft.fft(z) - Z).max() <= 1e-13 * np.abs(Z).max()


def test_reference_fft_compiled_matches_golden():
    if O.ref_fft_lib() is None:
        pytest.skip("oracle/_ref not built on this host")
    for N in (8, 64, 1024):
        assert np.array_equal(O.ref_fft_real(GOLD["real_in_%d" % N]), GOLD["real_out_%d" % N])


def _rand_fixed(rng, n):
    return [rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(3)]


def test_ewald_madelung_constant():
    # a single particle in its periodic lattice with a neutralising background:
    # potential of the images = -GM * zeta, zeta = -2.8372974794806 (simple cubic)
    x = np.array([123456789], np.uint32)
    y = np.array([987654321], np.uint32)
    z = np.array([5555555], np.uint32)
    h = 1e-3
    f, pot = O.ewald_direct(x, y, z, x, y, z, O.KERNEL_PLUMMER, h, 1.0, with_pot=True)
    assert np.abs(f).max() < 1e-12
    assert abs((pot[0] + 1.0 / h) - 2.8372974794806) < 1e-9


def test_ewald_split_independence_and_momentum():
    rng = np.random.Generator(np.random.PCG64(1))
    x, y, z = _rand_fixed(rng, 64)
    fa = O.ewald_direct(x, y, z, x, y, z, 0, 1e-4, 1.0)
    fb = O.ewald_direct(x, y, z, x, y, z, 0, 1e-4, 1.0, alpha=13.0, kmax=26)
    assert np.abs(fa - fb).max() < 1e-9 * np.abs(fa).max()
    assert np.abs(fa.sum(0)).max() < 1e-10 * np.abs(fa).max()


def test_ewald_two_body_short_range_is_newton():
    # two particles 1e-3 apart: force ~ 1/r^2 with periodic correction O(r)
    x = np.array([0, 4294967], np.uint32)
    y = np.zeros(2, np.uint32)
    z = np.zeros(2, np.uint32)
    f = O.ewald_direct(x, y, z, x, y, z, O.KERNEL_SPHERE, 1e-6, 1.0)
    r = 4294967 * 2.0 ** -32
    assert abs(f[0, 0] - 1.0 / r ** 2) < 1e-5 / r ** 2
    assert abs(f[0, 0] + f[1, 0]) < 1e-9 / r ** 2


@pytest.mark.parametrize("mbits", [3, 4, 5])
def test_bisection_leaves_equal_cell_keys(mbits):
    rng = np.random.Generator(np.random.PCG64(mbits))
    x, y, z = _rand_fixed(rng, 5000)
    ids, cb, ce = O.bin_bisect(x, y, z, mbits)
    perm, cs = O.bin_stable(x, y, z, mbits)
    # identical cell ranges: the bisection lays cells out in Morton order
    b2, e2 = O.cell_ranges_rowmajor(cs, mbits)
    assert np.array_equal(cb, b2) and np.array_equal(ce, e2)
    # identical particle sets per cell
    for c in np.nonzero(ce - cb)[0][:300]:
        assert np.array_equal(np.sort(ids[cb[c]:ce[c]]), np.sort(perm[cb[c]:ce[c]]))
    keys = O.cell_keys(x, y, z, mbits)
    assert np.all(np.diff(keys[perm].astype(np.int64)) >= 0)
    # and every particle's key is the Morton key of its top position bits
    sh = 32 - mbits
    assert np.array_equal(keys, O.morton(x >> sh, y >> sh, z >> sh).astype(np.uint32))


def test_greens_derivative_formula_vs_finite_differences():
    # G_n(R) from the radial-derivative expansion equals finite differences of G_0
    mbits, p = 4, 3
    G = O.greens_real(mbits, p, O.KERNEL_PLUMMER, 1e-3, 1.0)
    M = 1 << mbits
    # finite differences are only meaningful on the smooth (near-zone) part:
    # near-zone offsets carry -erf(alpha r)/r; check d/dx at offset (1,0,0)
    # against a direct evaluation of the radial formula
    import math
    alpha = O.GREENS_ALPHA

    def phi(x):
        r = math.sqrt(x[0] ** 2 + x[1] ** 2 + x[2] ** 2)
        return -math.erf(alpha * r) / r

    R = np.array([1.0 / M, 0.0, 0.0])
    eps = 1e-5
    d = (phi(R + [eps, 0, 0]) - phi(R - [eps, 0, 0])) / (2 * eps)
    k = O.mi_index(1, 0, 0)
    assert abs(G[k, 1, 0, 0] - d) < 1e-6 * abs(d)


def test_method_error_decreases_with_order():
    P = ics.plummer_spheres(4096, seed=1, nspheres=4, a=0.04)
    x, y, z = P["x"], P["y"], P["z"]
    n = len(x)
    truth = O.ewald_direct(x, y, z, x, y, z, 0, 1.0 / 800, 1.0 / n)
    errs = []
    for p in (1, 3, 5):
        r = O.method_forces(x, y, z, 4, p, 0, 1.0 / 800, 2.0, 1.0 / n)
        f = np.empty((n, 3))
        f[r["perm"]] = r["ffar"] + r["fnear"]
        errs.append(O.force_errors(f, truth)["rms_norm"])
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 2e-3


def test_drift_wraps_and_truncates():
    x = np.array([0xFFFFFFF0, 5, 100], np.uint32)
    v = np.array([1.0, -1.0, 0.25], np.float32)
    z0 = np.zeros(3, np.uint32)
    zv = np.zeros(3, np.float32)
    nx, _, _ = O.drift(x, z0, z0, v, zv, zv, 2.0 ** -30, 1.0)
    # displacement = v * 2^-30 * 2^32 = 4 v
    assert list(nx) == [(0xFFFFFFF0 + 4) & 0xFFFFFFFF, 1, 101]


def test_kick_update_rung_rule():
    # rung rises by at most one per kick (src/kick.cpp:92), falls by at most one
    n = 4
    v = np.zeros(n, np.float32)
    rung = np.array([0, 3, 0, 0], np.int8)
    f = np.array([1e6, 0.0, 1e-12, 10.0], np.float32)
    z = np.zeros(n, np.float32)
    vx, vy, vz, r, mr = O.kick_update(v, v, v, rung, f, z, z, ascending=1, descending=1, top=1,
                                      first=0, prung=0, t0=1e-2, eta=0.15, max_dt=1.0,
                                      scale=1.0, hsoft=1e-3)
    assert r[0] == 1 and r[1] == 2 and r[2] == 0
    assert mr == 2
    assert np.allclose(vx, f * 1e-2, rtol=1e-6)
