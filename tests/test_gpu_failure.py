"""Failure detection without a GPU fault: a bounded device-side wait that
runs out reports CT2G_ETIMEOUT through the context's device error word, the
kernel returns, and the context keeps working.

ct2g_wait_selftest queues a kernel that waits on an mbarrier nothing arrives
at (a flag that nothing sets) with a poll limit of a few thousand, the same
bounded wait and error report the tensor-core FFT passes use for their MMA
completions.  Nothing traps, faults or hangs.
"""
import numpy as np
import pytest

from ct2_b200 import ics
from ct2_b200.gravity import Gravity

pytestmark = pytest.mark.gpu

CT2G_ETIMEOUT = 5


def test_bounded_wait_reports_timeout_and_context_survives(gpu):
    P = ics.plummer_spheres(5000, seed=2, nspheres=3, a=0.02)
    g = Gravity(mesh=16, order=3, bwidth=2.0, hsoft=2e-3, GM=1.0 / 5000)
    g.upload_dict(P)
    g.particle_to_grid()
    g.compute_forces()
    f0, _ = g.forces()
    assert g.synchronize_status() == 0
    g.wait_selftest(4096)
    assert g.synchronize_status() == CT2G_ETIMEOUT
    assert g.synchronize_status() == 0  # reported once, then cleared
    # the context is intact: the same forces again, bit for bit
    g.compute_forces()
    f1, _ = g.forces()
    assert np.array_equal(f0, f1)
    # and a step still runs
    g.kick_step(0, 0, 1.0, 1.0, 1.0, 1e-3, 0)
    assert g.synchronize_status() == 0
    with pytest.raises(Exception):
        g.wait_selftest(0)
    g.close()
