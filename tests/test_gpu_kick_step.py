"""The rung-hierarchical step on the GPU (ct2g_kick_step, src/main.cpp:8-92)
against the restated driver in oracle/kick_step.py, whose level bookkeeping
is checked against the reference's own compiled kick_step in
tests/test_ref_pinned.py.

The oracle's driver does its own rung partition, push/pop, set_minrung,
binning (stable Morton sort), velocity + rung update (the restatement of
kick.cpp:75-99) and drift (drift.cpp:4-18).  Only the forces of each level
come from the GPU: a scratch context holding exactly the level's range, in
the order the driver binned it, runs the library's kick and hands its force
buffer back.  The two paths therefore agree bit for bit: ids (the order),
positions, velocities, rungs, the current range, minrung and the return
value, after every call of a sequence.
"""
import numpy as np
import pytest

from ct2_b200 import ics
from ct2_b200.gravity import Gravity, kick_params
from oracle import kick_step as KS

pytestmark = pytest.mark.gpu

MBITS, ORDER, BW = 4, 3, 2.0


def _gpu_forces(soft, GM):
    g = Gravity(mesh=1 << MBITS, order=ORDER, bwidth=BW, hsoft=soft, GM=GM)

    def fn(store, b):
        g.upload(store.x[b:], store.y[b:], store.z[b:], store.vx[b:], store.vy[b:],
                 store.vz[b:], store.rung[b:])
        g.particle_to_grid()
        d = g.download()
        # the driver binned the range already: binning again is the identity
        assert np.array_equal(d["id"], np.arange(store.n - b, dtype=np.uint32))
        g.kick(kick_params(t0=1e-3))
        f, _ = g.forces()
        return f
    return g, fn


def _state(d):
    return {k: d[k] for k in ("id", "x", "y", "z", "vx", "vy", "vz", "rung")}


@pytest.mark.parametrize("case,t0,nocrop,tau0", [
    ("clustered", 1e-2, False, 0.0),  # deep hierarchy, clip_top taken (3 fast > slow), first kick
    ("clustered", 1e-2, True, 1.0),   # the same with nocrop: minrung stays
    ("lattice", 2e-3, False, 1.0),    # quiet lattice: most particles at rung 0, no clip_top
])
def test_kick_step_sequence_matches_oracle_bitwise(gpu, case, t0, nocrop, tau0):
    n = 4096
    if case == "clustered":
        P = ics.plummer_spheres(n, seed=11, nspheres=6, a=0.01)
    else:
        P = ics.lattice(16, seed=11, sigma_cells=0.3)
    soft = 1.0 / 800.0
    GM = float(np.float32(1.0 / n))
    g = Gravity(mesh=1 << MBITS, order=ORDER, bwidth=BW, hsoft=soft, GM=GM)
    g.upload_dict(P)
    scratch, fn = _gpu_forces(soft, GM)
    s = KS.Store(P["x"], P["y"], P["z"], P["vx"], P["vy"], P["vz"], P["rung"])
    kick = KS.kick_with_forces(fn, float(np.float32(soft)))
    to_grid = KS.oracle_to_grid(MBITS)
    minrung_g = minrung_o = 0
    max_rung = 0
    tau = tau0
    clipped = False
    depths = []
    for step in range(3):
        val_g, minrung_g = g.kick_step(minrung_g, max_rung, 1.0, 1.0, tau, t0, 0, nocrop)
        minrung_o, val_o, _ = KS.kick_step(s, minrung_o, max_rung, 1.0, 1.0, tau, t0, 0, nocrop,
                                           eta=0.15, to_grid=to_grid, kick=kick,
                                           drift=KS.oracle_drift)
        assert val_g == val_o == max_rung  # the reference returns its max_rung argument
        assert minrung_g == minrung_o
        d = _state(g.download())
        o = s.arrays()
        for k in d:
            assert np.array_equal(d[k], o[k]), (step, k)
        assert g.current_range() == s.current_range()
        counts = g.rung_counts()
        assert list(counts) == [int(c) for c in s.rung_counts()]
        max_rung = len(counts) - 1
        depths.append(max_rung)
        clipped |= minrung_o > 0
        tau += t0
    print(case, t0, nocrop, "rung depths", depths, "clipped", clipped)
    if case == "clustered":
        assert max(depths) >= 2  # the hierarchy was exercised
        assert clipped == (not nocrop)
    else:
        assert not clipped
    scratch.close()
    g.close()


def test_kick_step_unbalanced_stack_is_an_error(gpu):
    # a first call with max_rung above minrung pops levels no earlier call
    # pushed: the reference reads an empty std::stack there; here it is
    # CT2G_ESTATE and nothing is left half done on the device
    P = ics.plummer_spheres(2048, seed=3, nspheres=2, a=0.02)
    g = Gravity(mesh=16, order=2, bwidth=1.0, hsoft=1e-3, GM=1.0 / 2048)
    g.upload_dict(P)
    with pytest.raises(Exception) as e:
        g.kick_step(0, 2, 1.0, 1.0, 1.0, 1e-3, 0)
    assert "rung stack" in str(e.value)
    g.close()
