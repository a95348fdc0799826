"""The oracle pinned to the reference's own code (CPU).

The reference's particle_to_grid, rung bookkeeping and kick_step
(src/particle.cpp, src/main.cpp) and its cosmology (src/cosmology.cpp) are
compiled from its sources into oracle/_ref (oracle/Makefile target `ref`).
Where that library is present the oracle is checked against it directly;
everywhere, the oracle is checked against the golden fixtures it produced
(tests/golden/make_ref_fixtures.py).
"""
import json
import os

import numpy as np
import pytest

from ct2_b200 import ics
from oracle import kick_step as KS
from oracle import oracle as O
from oracle import ref_particle as R

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")

import sys  # noqa: E402
sys.path.insert(0, GOLD)
import make_ref_fixtures as MF  # noqa: E402

needs_ref = pytest.mark.skipif(R.lib() is None, reason="oracle/_ref not built here")


@pytest.mark.parametrize("n,ppcell", MF.BIN_CASES)
def test_oracle_bisection_is_the_reference_order(n, ppcell):
    """oracle.bin_bisect (restating particle.cpp:69-114) leaves the particles
    in exactly the order the reference's own bisection does, id for id; the
    stable Morton order (the GPU's) has the same cells with the same ranges."""
    g = np.load(os.path.join(GOLD, "ref_binning.npz"))
    order = g["order_%d_%d" % (n, ppcell)].astype(np.int64)
    mesh = int(g["ncell_%d_%d" % (n, ppcell)])
    mbits = mesh.bit_length() - 1
    assert 1 << mbits == mesh
    P = ics.plummer_spheres(n, seed=3, nspheres=4, a=0.02)
    ids, cb, ce = O.bin_bisect(P["x"], P["y"], P["z"], mbits)
    assert np.array_equal(ids, order)
    perm, cs = O.bin_stable(P["x"], P["y"], P["z"], mbits)
    keys = O.cell_keys(P["x"], P["y"], P["z"], mbits).astype(np.int64)
    # the reference's order walks the cells in Morton order ...
    assert np.all(np.diff(keys[order]) >= 0)
    # ... with the same ranges as the stable sort, and the same particles in each
    assert np.array_equal(keys[order], keys[perm])
    for c in np.flatnonzero(np.diff(cs)):
        b, e = cs[c], cs[c + 1]
        assert np.array_equal(np.sort(order[b:e]), np.sort(perm[b:e]))


@needs_ref
@pytest.mark.parametrize("n,ppcell", MF.BIN_CASES)
def test_fixture_is_the_reference_binning(n, ppcell):
    g = np.load(os.path.join(GOLD, "ref_binning.npz"))
    P = ics.plummer_spheres(n, seed=3, nspheres=4, a=0.02)
    x, y, z, vx, nc = R.particle_to_grid(P["x"], P["y"], P["z"], ppcell,
                                         vx=np.arange(n, dtype=np.float32))
    assert nc == int(g["ncell_%d_%d" % (n, ppcell)])
    assert np.array_equal(vx.astype(np.uint32), g["order_%d_%d" % (n, ppcell)])
    o = vx.astype(np.int64)
    assert np.array_equal(x, P["x"][o]) and np.array_equal(z, P["z"][o])


def _cmp_trace(a, b):
    assert len(a) == len(b)
    for ea, eb in zip(a, b):
        assert ea == eb, (ea, eb)


@pytest.mark.parametrize("case", [c[0] for c in MF.STEP_CASES])
def test_oracle_kick_step_matches_reference_fixture(case):
    """The restated driver makes the same kick() and drift() calls, with the
    same parameters and ranges, returns the same values and leaves the same
    particle state as the reference's kick_step over three steps."""
    fx = json.load(open(os.path.join(GOLD, "ref_kick_step.json")))[case]
    trace, vals, dig = MF.run_steps("oracle", fx["nocrop"], tuple(fx["amp"]), fx["tau0"])
    _cmp_trace(MF.trace_json(trace), fx["trace"])
    assert [list(v) for v in vals] == fx["returns"]
    assert dig == fx["digest"]
    # the reference returns its max_rung argument, not the last kick's rung
    assert [v for _, v in vals][0] == 0


@needs_ref
@pytest.mark.parametrize("case", [c[0] for c in MF.STEP_CASES])
def test_fixture_is_the_reference_kick_step(case):
    fx = json.load(open(os.path.join(GOLD, "ref_kick_step.json")))[case]
    trace, vals, dig = MF.run_steps("reference", fx["nocrop"], tuple(fx["amp"]), fx["tau0"])
    _cmp_trace(MF.trace_json(trace), fx["trace"])
    assert [list(v) for v in vals] == fx["returns"]
    assert dig == fx["digest"]


def test_fixture_cases_cover_the_level_rules():
    fx = json.load(open(os.path.join(GOLD, "ref_kick_step.json")))
    # clip_top taken (minrung rises) without nocrop, never with it
    assert fx["clip"]["returns"][-1][0] == 1
    assert all(m == 0 for m, _ in fx["nocrop"]["returns"])
    # first (tau == 0) kicks, ascending levels and several depths occur
    kicks = [e[1] for c in fx.values() for e in c["trace"] if e[0] == "kick"]
    assert any(k["first"] for k in kicks) and any(not k["first"] for k in kicks)
    assert any(k["ascending"] and not k["descending"] for k in kicks)
    assert max(k["rung"] for k in kicks) >= 4


@needs_ref
def test_reference_rung_partition_and_stack():
    """particle_sort_by_rung / push / pop / set_minrung / rung_counts of the
    reference against the Store restatement: same ranges and counts; the
    partition's two sides hold the same particles."""
    P = ics.plummer_spheres(3000, seed=5, nspheres=3, a=0.02)
    rng = np.random.Generator(np.random.PCG64(1))
    rung = rng.integers(0, 5, 3000).astype(np.int8)
    a = KS.Store(P["x"], P["y"], P["z"], np.arange(3000, dtype=np.float32), P["vy"], P["vz"],
                 rung)
    b = KS.Store(P["x"], P["y"], P["z"], np.arange(3000, dtype=np.float32), P["vy"], P["vz"],
                 rung)
    R.reset(b)
    L = R.lib()
    for lev in (1, 2, 4, 0, 3):
        if lev:
            a.push_rungs()
            L.ref_push_rungs()
        a.sort_by_rung(lev)
        L.ref_sort_by_rung(lev)
        import ctypes
        rb, re_ = ctypes.c_size_t(), ctypes.c_size_t()
        L.ref_current_range(ctypes.byref(rb), ctypes.byref(re_))
        assert (rb.value, re_.value) == a.current_range()
        ra, rbv = a.current_range()[0], rb.value
        assert np.array_equal(np.sort(a.vx[ra:]), np.sort(b.vx[rbv:]))
    for _ in range(4):
        a.pop_rungs()
        L.ref_pop_rungs()
    assert R.stack_depth() == len(a.stack) == 0
    a.set_minrung(2)
    L.ref_set_minrung(2)
    import ctypes
    counts = (ctypes.c_size_t * 16)()
    m = L.ref_rung_counts(counts, 16)
    assert list(counts[:m]) == [int(c) for c in a.rung_counts()]


@pytest.mark.skipif(O.ref_fft_lib() is None, reason="oracle/_ref not built here")
def test_reference_transposes_as_compiled():
    """What the reference's layout helpers compute (src/fft/transpose.cpp),
    next to what the library implements: transpose_r2c is the documented
    gather; transpose_yz swaps every pair twice and leaves X unchanged;
    transpose_c2r does not invert transpose_r2c (row stride N instead of
    N/2+1 on its input, z loop started at the block's y)."""
    L = O.ref_fft_lib()
    N = 8
    rng = np.random.Generator(np.random.PCG64(9))
    x = rng.uniform(size=N ** 3)
    X = x.copy()
    L.ref_transpose_yz(X, N)
    assert np.array_equal(X, x)
    Y = np.zeros(2 * N * N * (N // 2 + 1))
    L.ref_transpose_r2c(np.ascontiguousarray(x), Y, N)
    h = N // 2 + 1
    xr = x.reshape(N, N, N)
    re = Y[: N * N * h].reshape(N, N, h)
    im = Y[N * N * h:].reshape(N, N, h)
    for iy in range(h):
        assert np.array_equal(re[:, :, iy], xr[:, iy, :])
        want = 0.0 if iy in (0, N // 2) else xr[:, N - iy, :]
        assert np.array_equal(im[:, :, iy], np.broadcast_to(want, (N, N)))
    back = np.zeros(N ** 3)
    L.ref_transpose_c2r(Y, back, N)
    assert not np.array_equal(back, x)
