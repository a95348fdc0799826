"""Run the force computation of the gravity step on a seeded synthetic box.

    python -m ct2_b200.run_step [--mesh 256] [--order 4] [--bwidth 4] [--n 2097152] [--reps 3]
                                [--split-mg2l 0|1]

Plummer spheres (one per 4096 particles, scale radius two cells) on a periodic
unit box, softening one 25th of a cell, G x mass = 1/n; each repetition bins
the particles (particle_to_grid) and computes the forces (P2M, FFT, Green's
multiply, inverse FFT + L2P, direct sum) through the eager entry points.  A
minimal end-to-end use of the library, and the command the kernel profiles
are taken on; it prints the device time of each stage of the last repetition.
"""
from __future__ import annotations

import argparse

import numpy as np

from . import ics
from .gravity import Gravity


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--mesh", type=int, default=256)
    ap.add_argument("--order", type=int, default=4)
    ap.add_argument("--bwidth", type=float, default=4.0)
    ap.add_argument("--n", type=int, default=1 << 21)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--split-mg2l", type=int, default=0,
                    help="1: x passes and MG2L as three launches instead of one")
    a = ap.parse_args(argv)
    P = ics.plummer_spheres(a.n, seed=a.seed, nspheres=max(1, a.n // 4096), a=2.0 / a.mesh)
    g = Gravity(mesh=a.mesh, order=a.order, bwidth=a.bwidth, hsoft=1.0 / (25 * a.mesh),
                GM=1.0 / a.n)
    g.set_tuning(**{**g.tuning(), "split_mg2l": a.split_mg2l})
    g.upload_dict(P)
    for _ in range(a.reps):
        g.particle_to_grid()
        g.compute_forces()
    f, _ = g.forces()
    print("n %d mesh %d order %d: sum |f| = %.6e, interactions %d"
          % (a.n, a.mesh, a.order, float(np.abs(f).sum()), g.interaction_count()))
    names = ("bin", "p2m", "fft_fwd", "mg2l", "fft_inv", "forces")
    print("last repetition, ms: " + ", ".join("%s %.3f" % (k, v)
                                              for k, v in zip(names, g.stage_times())))
    g.close()


if __name__ == "__main__":
    main()
