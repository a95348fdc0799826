"""The fused X pass + MG2L kernel against the split path (X pass, MG2L, inverse
X pass as three launches) on the same particles.

The fused kernel reads the Green's table in column order ([qj][qk][c][qi]),
value for value the table the split MG2L reads, transforms each line with
the same arithmetic and contracts the same terms in the same order, so the
two paths agree to FP32 rounding (tolerance 1e-5 max, 1e-6 rms relative;
in practice they are bit-identical).

The table is NOT folded by its mirror symmetry in qi or qj: the reference's
real-space tensor is sampled with the image sum centred on the minimum image,
so on the plane x = N/2 an odd-in-x component does not vanish, and its
transform carries an even part of a few 1e-6 of the component's scale
(test_greens_not_exactly_odd pins that), which a folded table would flip on
half of the spectrum.
"""
import numpy as np
import pytest

from ct2_b200 import ics
from ct2_b200.gravity import Gravity
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_greens_not_exactly_odd(gpu):
    N, p = 16, 4
    g = Gravity(mesh=N, order=p, bwidth=2.0, hsoft=0.3 / N)
    G = g.greens()
    mi = O.mi_table(p)
    rev = (-np.arange(N)) % N
    worst = 0.0
    for k in range(G.shape[0]):
        sx = -1.0 if mi[k][0] % 2 else 1.0
        d = np.abs(G[k][rev] - sx * G[k]).max() / np.abs(G[k]).max()
        worst = max(worst, d)
        assert d < 1e-4, k  # odd or even up to the x = N/2 plane's share
    assert worst > 1e-6  # ... which a folded table would lose


def _forces(mesh, p, bw, P, split, pot=False):
    g = Gravity(mesh=mesh, order=p, bwidth=bw, hsoft=1.0 / (25 * mesh), GM=1.0 / len(P["x"]))
    g.set_tuning(**{**g.tuning(), "split_mg2l": split})
    g.upload_dict(P)
    g.particle_to_grid()
    g.compute_forces()
    f, ph = g.forces()
    g.compute_expansions()
    L = g.expansions()
    g.close()
    return f, ph, L


@pytest.mark.parametrize("mesh,p,bw,n", [(64, 4, 2.0, 60000), (256, 4, 4.0, 300000),
                                         (32, 6, 2.0, 20000), (128, 5, 3.0, 100000)])
def test_fused_matches_split(gpu, mesh, p, bw, n):
    P = ics.plummer_spheres(n, seed=mesh + p, nspheres=max(1, n // 3000), a=2.0 / mesh)
    f0, p0, L0 = _forces(mesh, p, bw, P, 0)
    f1, p1, L1 = _forces(mesh, p, bw, P, 1)
    rel = np.linalg.norm(f0 - f1, axis=1) / np.linalg.norm(f1, axis=1)
    print("fused vs split: max %.2e rms %.2e" % (rel.max(), np.sqrt(np.mean(rel ** 2))))
    print("bit-identical forces:", np.array_equal(f0, f1))
    assert rel.max() < 1e-5 and np.sqrt(np.mean(rel ** 2)) < 1e-6
    for k in range(L0.shape[0]):
        s = np.abs(L1[k]).max()
        assert np.abs(L0[k] - L1[k]).max() <= 1e-5 * s, k


def test_split_flag_in_tuning(gpu):
    g = Gravity(mesh=32, order=3, bwidth=2.0, hsoft=1e-3)
    assert g.tuning()["split_mg2l"] == 0
    g.set_tuning(**{**g.tuning(), "split_mg2l": 1})
    assert g.tuning()["split_mg2l"] == 1
    with pytest.raises(RuntimeError):
        g.set_tuning(**{**g.tuning(), "split_mg2l": 2})
