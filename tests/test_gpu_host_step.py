"""The host-state step (ct2g_kick_drift_host) against upload + kick_drift +
download on the same particles.

The host-state step uploads the velocities and rungs on a second stream
while binning and the force solve run, and gathers them into cell order just
before the update instead of inside binning.  That moves data, not
arithmetic, so every output array (positions, velocities, rungs, ids) and
the returned max rung must be bit-identical to the three separate calls, for
the recorded-graph and the eager step, over two steps in a row (the second
fed with the first's output).  A device-resident graph step after it must
also still match the eager calls (the velocity wait it records is a no-op
there).
"""
import numpy as np
import pytest

from ct2_b200 import ics
from ct2_b200.gravity import CT2GError, Gravity, kick_params

pytestmark = pytest.mark.gpu

KP = kick_params(ascending=True, descending=True, top=True, first=False, rung=0, t0=1e-3,
                 eta=0.15, max_dt=0.01, scale=1.0)
DT = 1e-3
KEYS = ("x", "y", "z", "vx", "vy", "vz", "rung")
TYPES = (np.uint32,) * 3 + (np.float32,) * 3 + (np.int8,)


def _state(P, n):
    s = {k: np.ascontiguousarray(P[k], t) for k, t in zip(KEYS[:6], TYPES[:6])}
    s["rung"] = np.ascontiguousarray(P.get("rung", np.zeros(n, np.int8)), np.int8)
    return s


def _pinned(s):
    import torch
    out = {}
    for k, a in s.items():
        v = a.view(np.int32) if a.dtype == np.uint32 else a
        p = torch.from_numpy(v).pin_memory().numpy()
        out[k] = p.view(np.uint32) if a.dtype == np.uint32 else p
    return out


def _empty(n):
    d = {k: np.empty(n, t) for k, t in zip(KEYS, TYPES)}
    d["id"] = np.empty(n, np.uint32)
    return d


@pytest.mark.parametrize("graph,pinned", [(True, True), (False, False)])
def test_host_step_matches_separate_calls(gpu, graph, pinned):
    n, mesh = 60000, 64
    P = ics.plummer_spheres(n, seed=7, nspheres=12, a=2.0 / mesh)
    rng = np.random.default_rng(3)
    P["vx"], P["vy"], P["vz"] = (rng.normal(0, 0.05, n).astype(np.float32) for _ in range(3))
    kw = dict(mesh=mesh, order=4, bwidth=2.0, hsoft=1.0 / (25 * mesh), GM=1.0 / n)
    ga, gb, gc = Gravity(**kw), Gravity(**kw), Gravity(**kw)
    state = _state(P, n)
    gb.upload_dict(state)
    for step in range(2):
        ga.upload_dict(state)
        mr_a = ga.kick_drift(KP, DT, 1.0, graph=graph, wait=True)
        ref = ga.download()
        # the reference's call sequence, whose binning gathers everything at once
        gc.upload_dict(state)
        gc.particle_to_grid()
        mr_c = gc.kick(KP)
        gc.drift(DT, 1.0)
        ref_c = gc.download()
        out = _empty(n)
        src = _pinned(state) if pinned else state
        mr_b = gb.kick_drift_host(KP, DT, src, out, graph=graph)
        assert mr_a == mr_b == mr_c, step
        for k in KEYS + ("id",):
            assert np.array_equal(out[k], ref[k]), (step, k)
            assert np.array_equal(out[k], ref_c[k]), (step, k)
        state = {k: out[k].copy() for k in KEYS}
    # a device-resident step on the same context after the host-state steps
    gb.upload_dict(state)
    ga.upload_dict(state)
    gb.kick_drift(KP, DT, 1.0, graph=True, wait=True)
    ga.kick_drift(KP, DT, 1.0, graph=False, wait=True)
    da, db = ga.download(), gb.download()
    for k in KEYS + ("id",):
        assert np.array_equal(da[k], db[k]), k
    ga.close()
    gb.close()
    gc.close()


def test_host_step_refuses_another_count(gpu):
    n, mesh = 4096, 32
    P = ics.plummer_spheres(n, seed=1, nspheres=2, a=2.0 / mesh)
    g = Gravity(mesh=mesh, order=3, bwidth=2.0, hsoft=1.0 / (25 * mesh), GM=1.0 / n)
    g.upload_dict(_state(P, n))
    small = {k: v[: n // 2].copy() for k, v in _state(P, n).items()}
    with pytest.raises(CT2GError):
        g.kick_drift_host(KP, DT, small, _empty(n // 2))
    # the context is still usable
    g.kick_drift_host(KP, DT, _state(P, n), _empty(n))
    g.close()
