"""The z and y passes run as one plane pipeline per direction (tuning
plane_pipe = 1; 2 also drops the inverse pass's read L2 lines) give the same
forces, potentials, velocities and positions bit for bit as the separate
passes (plane_pipe = 0): every value is computed by the same arithmetic in
the same order, only the kernels that run it and the order of the planes
differ.  Covered: meshes 64-256, orders 2-6, box contexts, eager calls and
recorded graphs, with the near field overlapped."""
import numpy as np
import pytest

from ct2_b200 import ics
from ct2_b200.gravity import Gravity, kick_params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mesh,order,nbox,overlap", [
    (64, 2, 1, 0), (128, 4, 1, 1), (64, 6, 2, 0), (256, 4, 1, 0), (128, 5, 1, 0)])
def test_plane_pipe_is_bitwise_the_separate_passes(gpu, mesh, order, nbox, overlap):
    n = 40000
    P = ics.plummer_spheres(n * nbox, seed=mesh + order, nspheres=8, a=0.02)
    g = Gravity(mesh=mesh, order=order, bwidth=2.0, hsoft=1.0 / (25 * mesh), GM=1.0 / n,
                nbox=nbox)

    def upload():
        g.upload_dict(P)
        if nbox > 1:  # box b: the next n particles
            g.set_boxes([n] * nbox, [1.0 / n] * nbox)

    out = {}
    for pipe in (0, 1, 2):
        g.set_tuning(**{**g.tuning(), "plane_pipe": pipe, "overlap": overlap})
        upload()
        g.particle_to_grid()
        g.compute_forces()  # with the potential
        f, pot = g.forces()
        upload()
        for _ in range(2):
            g.kick_drift(kick_params(t0=1e-3), 1e-3, 1.0, graph=True)
        assert g.synchronize_status() == 0
        out[pipe] = (f, pot, g.download())
    f0, p0, d0 = out[0]
    assert np.isfinite(f0).all() and np.abs(f0).max() > 0
    for pipe in (1, 2):
        f, p, d = out[pipe]
        assert np.array_equal(f0, f) and np.array_equal(p0, p), pipe
        for k in ("id", "x", "y", "z", "vx", "vy", "vz", "rung"):
            assert np.array_equal(d0[k], d[k]), (pipe, k)
    g.close()
