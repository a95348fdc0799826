"""Cloud-in-cell deposit and the complex-to-complex 3D FFT on device grids
(the precision form's configuration: a batch of four complex grids), against
numpy FP64.  Tolerances: the deposit 2e-6 relative to the largest value
(FP32 weights, atomic sums in any order); the FP32 transform 2e-6 rms
relative to the FP64 spectrum; the tensor-core passes (BF16 hi+lo operands,
FP32 accumulation) 3e-5.
"""
import numpy as np
import pytest
import torch

from ct2_b200 import ics
from ct2_b200.gravity import Gravity
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_cic_deposit_matches_oracle(gpu):
    N = 16
    P = ics.plummer_spheres(6000, seed=4, nspheres=3, a=0.05)
    g = Gravity(mesh=16, order=1, bwidth=1.0, hsoft=1e-3)
    g.upload_dict(P)
    grid = torch.empty(4 * N ** 3 * 2, dtype=torch.float32, device="cuda")
    g.cic_deposit(N, grid.data_ptr())
    g.synchronize()
    got = grid.cpu().numpy().reshape(4, N, N, N, 2)
    want = O.cic_deposit(P["x"], P["y"], P["z"], N)
    assert np.all(got[..., 1] == 0.0)
    assert np.abs(got[..., 0] - want).max() <= 2e-6 * np.abs(want).max()
    assert abs(got[0, ..., 0].sum() - 6000) < 1e-2  # the weights of a particle add to 1
    g.close()


@pytest.mark.parametrize("N,batch", [(8, 3), (32, 2), (64, 1)])
def test_c2c_fft_fp32_matches_numpy(gpu, N, batch):
    rng = np.random.Generator(np.random.PCG64(N))
    z = (rng.normal(size=(batch, N, N, N)) + 1j * rng.normal(size=(batch, N, N, N)))
    a = np.stack([z.real, z.imag], -1).astype(np.float32)
    g = Gravity(mesh=8, order=1, bwidth=1.0, hsoft=1e-3)
    t = torch.from_numpy(a.copy()).cuda()
    g.fft3d_c2c_dev(t.data_ptr(), N, batch, 1)
    g.synchronize()
    got = t.cpu().numpy()
    got = got[..., 0] + 1j * got[..., 1]
    want = np.fft.fftn(z, axes=(1, 2, 3))
    assert _rel(got, want) < 2e-6
    g.fft3d_c2c_dev(t.data_ptr(), N, batch, -1)
    g.synchronize()
    back = t.cpu().numpy()
    back = (back[..., 0] + 1j * back[..., 1]) / N ** 3
    assert _rel(back, z) < 2e-6
    g.close()


def test_c2c_fft_tensor_cores_at_256(gpu):
    N = 256
    P = ics.plummer_spheres(200000, seed=5, nspheres=16, a=0.01)
    g = Gravity(mesh=N, order=1, bwidth=1.0, hsoft=1e-4)
    g.upload_dict(P)
    grid = torch.empty(4 * N ** 3 * 2, dtype=torch.float32, device="cuda")
    g.cic_deposit(N, grid.data_ptr())
    g.synchronize()
    x0 = grid.view(4, N, N, N, 2)[0, ..., 0].double().cpu().numpy()
    want = np.fft.fftn(x0)
    errs = {}
    for mode in ("fp32", "tc"):
        g.set_fft_mode(mode)
        t = grid.clone()
        g.fft3d_c2c_dev(t.data_ptr(), N, 4, 1)
        g.synchronize()
        got = t.view(4, N, N, N, 2)[0].double().cpu().numpy()
        errs[mode] = _rel(got[..., 0] + 1j * got[..., 1], want)
        # and back: the inverse of the transform, unnormalised
        g.fft3d_c2c_dev(t.data_ptr(), N, 4, -1)
        g.synchronize()
        back = t.view(4, N, N, N, 2)[0, ..., 0].double().cpu().numpy() / N ** 3
        assert _rel(back, x0) < (3e-5 if mode == "tc" else 2e-6)
    print("c2c 256^3 spectrum rms rel error vs FP64:", errs)
    assert errs["fp32"] < 2e-6 and errs["tc"] < 3e-5
    g.close()
