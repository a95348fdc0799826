"""The near field overlapped with the mesh solve (tuning overlap = 1: its own
stream and buffers, added to the far field afterwards) gives the same forces,
velocities and positions bit for bit as the serial form, eagerly and as a
recorded graph, with the potential, and for every sparse-sink path."""
import numpy as np
import pytest

from ct2_b200 import ics
from ct2_b200.gravity import Gravity, kick_params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("sparse_path,blocks", [(1, 0), (1, 2), (0, 1), (2, 0)])
def test_overlap_is_bitwise_the_serial_form(gpu, sparse_path, blocks):
    n = 60000
    P = ics.plummer_spheres(n, seed=8, nspheres=12, a=0.01)
    g = Gravity(mesh=64, order=4, bwidth=3.0, hsoft=1.0 / 3200, GM=1.0 / n)
    out = {}
    for overlap in (0, 1):
        g.set_tuning(**{**g.tuning(), "overlap": overlap, "sparse_path": sparse_path,
                        "near_blocks_per_sm": blocks})
        g.upload_dict(P)
        g.particle_to_grid()
        g.compute_forces()  # with the potential
        f, pot = g.forces()
        inter = g.interaction_count()
        g.upload_dict(P)
        for _ in range(2):
            g.kick_drift(kick_params(t0=1e-3), 1e-3, 1.0, graph=True)
        d = g.download()
        out[overlap] = (f, pot, inter, d)
    (f0, p0, i0, d0), (f1, p1, i1, d1) = out[0], out[1]
    assert np.array_equal(f0, f1) and np.array_equal(p0, p1) and i0 == i1 > 0
    for k in ("id", "x", "y", "z", "vx", "vy", "vz", "rung"):
        assert np.array_equal(d0[k], d1[k]), k
    g.close()
