"""Generate golden fixtures from the reference's own particle code.

Runs the reference's particle_to_grid (src/particle.cpp:69-114,349-362) and
kick_step (src/main.cpp:8-92), compiled from the reference tree into
oracle/_ref by `make -C oracle ref`, on seeded inputs, and stores:

  ref_binning.npz    per case: the order in which the reference's bisection
                     leaves the particles (their upload indices) and the Ncell
                     it chose; inputs are ics.plummer_spheres(n, seed=3,
                     nspheres=4, a=0.02)
  ref_kick_step.json per case: every kick() call (parameters and range) and
                     drift() call the reference's kick_step makes over a
                     sequence of three steps under the analytic force field of
                     oracle.kick_step.analytic_forces, the values it returns,
                     and a SHA-256 of the final particle state (sorted by
                     position, so independent of the store's order)

    make -C oracle ref && python tests/golden/make_ref_fixtures.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from ct2_b200 import ics  # noqa: E402
from oracle import kick_step as KS  # noqa: E402
from oracle import ref_particle as R  # noqa: E402

# (n, ppcell): the reference picks Ncell = int(cbrt(n // ppcell)) + 4
BIN_CASES = [(5000, 64), (32768, 16), (23000, 1)]

# (label, nocrop, force amplitudes, tau of the first step)
STEP_CASES = [("clip", False, (3.0, 40.0, 900.0), 0.0),
              ("nocrop", True, (3.0, 40.0, 900.0), 1.0),
              ("mild", False, (0.3, 2.0, 20.0), 1.0),
              ("shallow", False, (0.01, 0.1, 2.0), 0.0)]
STEP_N, STEP_T0, STEP_HSOFT, STEP_MBITS = 4096, 1e-2, 0.002, 3


def step_inputs():
    return ics.plummer_spheres(STEP_N, seed=3, nspheres=4, a=0.02)


def state_digest(s):
    k = np.lexsort((s.z, s.y, s.x))
    h = hashlib.sha256()
    for f in ("x", "y", "z", "vx", "vy", "vz", "rung"):
        h.update(np.ascontiguousarray(getattr(s, f)[k]).tobytes())
    return h.hexdigest()


def run_steps(driver, nocrop, amp, tau0, nsteps=3):
    """A sequence of kick_step calls; driver 'oracle' or 'reference'.
    Returns (trace, [(minrung, value)], digest)."""
    P = step_inputs()
    s = KS.Store(P["x"], P["y"], P["z"], P["vx"], P["vy"], P["vz"])
    kick = KS.kick_with_forces(KS.analytic_forces(amp), STEP_HSOFT)
    trace, out = [], []
    minrung, max_rung, tau = 0, 0, tau0
    if driver == "reference":
        R.reset(s)
    for _ in range(nsteps):
        if driver == "reference":
            minrung, val = R.kick_step(s, minrung, max_rung, 1.0, 1.0, tau, STEP_T0, 0, nocrop,
                                       eta=0.15, kick=kick, drift=KS.oracle_drift, trace=trace)
        else:
            minrung, val, _ = KS.kick_step(s, minrung, max_rung, 1.0, 1.0, tau, STEP_T0, 0,
                                           nocrop, eta=0.15,
                                           to_grid=KS.oracle_to_grid(STEP_MBITS), kick=kick,
                                           drift=KS.oracle_drift, trace=trace)
        out.append((int(minrung), int(val)))
        max_rung = int(s.rung.max())
        tau += STEP_T0
    return trace, out, state_digest(s)


def trace_json(trace):
    return [[e[0], e[1], int(e[2]), int(e[3])] if e[0] == "kick" else list(e) for e in trace]


def main():
    assert R.lib() is not None, "build oracle/_ref first (make -C oracle ref)"
    out = {}
    for n, ppcell in BIN_CASES:
        P = ics.plummer_spheres(n, seed=3, nspheres=4, a=0.02)
        _, _, _, vx, nc = R.particle_to_grid(P["x"], P["y"], P["z"], ppcell,
                                            vx=np.arange(n, dtype=np.float32))
        out["order_%d_%d" % (n, ppcell)] = vx.astype(np.uint32)
        out["ncell_%d_%d" % (n, ppcell)] = np.int64(nc)
    np.savez_compressed(os.path.join(HERE, "ref_binning.npz"), **out)
    steps = {}
    for label, nocrop, amp, tau0 in STEP_CASES:
        trace, vals, dig = run_steps("reference", nocrop, amp, tau0)
        steps[label] = dict(nocrop=nocrop, amp=list(amp), tau0=tau0, returns=vals,
                            trace=trace_json(trace), digest=dig)
    with open(os.path.join(HERE, "ref_kick_step.json"), "w") as f:
        json.dump(steps, f, separators=(",", ":"))
    print("wrote", len(out), "binning arrays and", len(steps), "kick_step cases")


if __name__ == "__main__":
    main()
