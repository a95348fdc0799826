"""The headline configuration at its full size (128^3 = 2,097,152 particles in
512 Plummer spheres plus a uniform background, 256^3 mesh), checked through
properties that do not need an O(N^2) oracle:

  * binning: the order and every cell range equal the oracle's stable
    counting sort (C, linear time) id for id;
  * drift is exactly reversible: drift(+dt) then drift(-dt) gives back the
    positions bit for bit (the displacement is truncated toward zero, so
    fixed32(-v dt) = -fixed32(v dt));
  * momentum: with equal particle masses the pairwise forces are equal and
    opposite (the near-field stencil is symmetric, the Green's tensor has
    the parity of its order), so sum_i F_i vanishes up to rounding and the
    multipole truncation (checked against sum_i |F_i|);
  * the whole step's forces match the FP64 Ewald sum on 1024 sinks within
    rms 1e-4.
"""
import numpy as np
import pytest

from ct2_b200 import ics
from ct2_b200.gravity import Gravity, kick_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N_SIDE, MESH = 128, 256


@pytest.fixture(scope="module")
def full():
    n = N_SIDE ** 3
    P = ics.plummer_spheres(n, seed=0, nspheres=512, a=0.005)
    g = Gravity(mesh=MESH, order=4, bwidth=4.0, hsoft=1.0 / (50 * N_SIDE), GM=1.0 / n,
                max_particles=n)
    g.upload_dict(P)
    yield P, n, g
    g.close()


def test_fullsize_binning_bit_exact(gpu, full):
    P, n, g = full
    g.upload_dict(P)
    g.particle_to_grid()
    d = g.download()
    perm, cs = O.bin_stable(P["x"], P["y"], P["z"], 8)
    assert np.array_equal(d["id"].astype(np.int64), perm)
    b, e = g.cells()
    ob, oe = O.cell_ranges_rowmajor(cs, 8)
    assert np.array_equal(b, ob) and np.array_equal(e, oe)


def test_fullsize_drift_is_reversible(gpu, full):
    P, n, g = full
    rng = np.random.Generator(np.random.PCG64(1))
    Q = dict(P)
    for k in ("vx", "vy", "vz"):
        Q[k] = rng.normal(0.0, 0.5, n).astype(np.float32)
    g.upload_dict(Q)
    g.drift(1e-3, 1.0)
    moved = g.download()
    g.drift(-1e-3, 1.0)
    back = g.download()
    assert not np.array_equal(moved["x"], Q["x"])
    assert np.array_equal(back["x"], Q["x"]) and np.array_equal(back["y"], Q["y"])
    assert np.array_equal(back["z"], Q["z"])


def test_fullsize_forces_momentum_and_accuracy(gpu, full):
    P, n, g = full
    g.upload_dict(P)
    g.particle_to_grid()
    g.compute_forces()
    f, _ = g.forces()
    ids = g.download()["id"]
    inter = g.interaction_count()
    assert inter > 4e9
    inv = np.empty(n, np.int64)
    inv[ids.astype(np.int64)] = np.arange(n)
    rng = np.random.Generator(np.random.PCG64(123))
    sel = np.sort(rng.choice(n, size=1024, replace=False))
    truth = g.ewald_direct(P["x"][sel], P["y"][sel], P["z"][sel])
    err = O.force_errors(f[inv[sel]].astype(np.float64), truth)
    print("128^3 step forces vs FP64 Ewald:", err)
    assert err["rms_rel"] < 1e-4
    tot = f.astype(np.float64).sum(0)
    scale = np.abs(f).astype(np.float64).sum()
    print("sum F / sum |F| =", tot / scale)
    assert np.all(np.abs(tot) < 1e-4 * scale)


def test_binning_at_the_largest_mesh(gpu):
    """mesh 512 (the largest the context takes: 134 M cells, 27-bit keys) on
    the same 2.1 M particles: order and cell ranges bit-exact."""
    n = N_SIDE ** 3
    P = ics.plummer_spheres(n, seed=2, nspheres=512, a=0.005)
    g = Gravity(mesh=512, order=1, bwidth=1.0, hsoft=1.0 / (50 * N_SIDE), GM=1.0 / n,
                max_particles=n)
    g.upload_dict(P)
    g.particle_to_grid()
    ids = g.download()["id"].astype(np.int64)
    perm, cs = O.bin_stable(P["x"], P["y"], P["z"], 9)
    assert np.array_equal(ids, perm)
    b, e = g.cells()
    ob, oe = O.cell_ranges_rowmajor(cs, 9)
    assert np.array_equal(b, ob) and np.array_equal(e, oe)
    g.close()
