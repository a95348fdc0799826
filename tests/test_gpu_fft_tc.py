"""Precision form: the y/x FFT passes as tensor-core DFT matrix products with
BF16 hi + lo operands (CT2G_FFT_TC_BF16X3).

Tolerances: the split keeps ~16 significant bits per operand, so a 3D
transform carries a relative error near 1e-5 of the spectrum's scale (the
FP32 CUDA-core passes: ~1e-7); forces through the mesh move by far less than
the method's own 1e-4 error budget."""
import ctypes

import numpy as np
import pytest

from ct2_b200 import _lib, ics
from ct2_b200.gravity import Gravity

pytestmark = pytest.mark.gpu


def _fft_dev(g, x, batch):
    import torch
    N = x.shape[-1]
    xin = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    out = torch.empty((batch, N, N, N // 2 + 1), dtype=torch.complex64, device="cuda")
    lib = _lib.load()
    torch.cuda.synchronize()
    rc = lib.ct2g_fft3d_f32_dev(g.handle, 1, ctypes.c_void_p(xin.data_ptr()),
                               ctypes.c_void_p(out.data_ptr()), N, batch)
    assert rc == 0, lib.ct2g_last_error(g.handle).decode()
    g.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("N", [256])
def test_tc_fft_matches_fp64(gpu, N):
    rng = np.random.Generator(np.random.PCG64(3))
    x = rng.normal(0, 1, (2, N, N, N)).astype(np.float32)
    ref = np.fft.rfftn(x.astype(np.float64), axes=(1, 2, 3))
    scale = np.sqrt(np.mean(np.abs(ref) ** 2))
    g = Gravity(mesh=N, order=1, bwidth=1.0, hsoft=1e-3)
    y32 = _fft_dev(g, x, 2)
    g.set_fft_mode("tc")
    ytc = _fft_dev(g, x, 2)
    e32 = np.sqrt(np.mean(np.abs(y32 - ref) ** 2)) / scale
    etc = np.sqrt(np.mean(np.abs(ytc - ref) ** 2)) / scale
    print("rms rel spectrum error: fp32 %.2e  tensor-core bf16x3 %.2e" % (e32, etc))
    assert e32 < 1e-6
    assert etc < 3e-5
    assert np.abs(ytc - ref).max() < 3e-4 * np.abs(ref).max()


def test_tc_mesh_forces(gpu):
    n = 64 ** 3
    P = ics.plummer_spheres(n, seed=5, nspheres=64, a=0.005)
    soft = 1.0 / (25 * 256)
    out = {}
    for mode in ("fp32", "tc"):
        g = Gravity(mesh=256, order=3, bwidth=3.0, hsoft=soft, GM=1.0 / n)
        g.set_fft_mode(mode)
        g.upload_dict(P)
        g.particle_to_grid()
        g.compute_forces()
        f, _ = g.forces()
        d = g.download()
        inv = np.empty_like(d["id"])
        inv[d["id"]] = np.arange(n, dtype=inv.dtype)
        out[mode] = f[inv]
        if mode == "fp32":
            rng = np.random.Generator(np.random.PCG64(8))
            sel = np.sort(rng.choice(n, 2048, replace=False))
            truth = g.ewald_direct(P["x"][sel], P["y"][sel], P["z"][sel])
        g.close()

    def rel(f, t):
        return np.sqrt(np.mean((np.linalg.norm(f - t, axis=1) / np.linalg.norm(t, axis=1)) ** 2))

    d = rel(out["tc"], out["fp32"])
    e32, etc = rel(out["fp32"][sel], truth), rel(out["tc"][sel], truth)
    print("tc vs fp32 forces %.2e; vs Ewald: fp32 %.3e tc %.3e" % (d, e32, etc))
    assert d < 2e-5
    assert etc < e32 * 1.05 + 1e-6
