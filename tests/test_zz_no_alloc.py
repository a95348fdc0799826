"""The allocation-free Ewald entry point, checked against the allocating one.

ct2g_ewald_direct_noalloc is for callers that cannot call cudaMalloc (a host
framework that owns every device buffer, or a loop where allocation is not
allowed): it takes device pointers for all inputs and outputs and keeps its
scratch in a static device array of the library.  Here the buffers come from
torch, as such a caller's own allocator would provide them; the result must
match ct2g_ewald_direct (which allocates its own scratch) to the same
tolerance the GPU-vs-CPU Ewald test uses, on two calls in a row (the second
call must clear what the first left in the shared scratch), for both
softening kernels, up to the largest kmax the scratch holds, and on a
caller's side stream.  This file runs
last so that a failure here leaves every other test's result in place.
"""
import ctypes

import numpy as np
import pytest

from ct2_b200 import _lib, ics
from ct2_b200.gravity import Gravity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel,kmax,side_stream", [
    (_lib.SOFT_PLUMMER, 20, False),
    (_lib.SOFT_SPHERE, 20, True),
    (_lib.SOFT_PLUMMER, 24, True),  # the largest kmax the static scratch holds
])
def test_noalloc_ewald_matches_allocating_entry_point(gpu, kernel, kmax, side_stream):
    import torch
    n = 6000
    P = ics.plummer_spheres(n, seed=4, nspheres=4, a=0.05)
    soft = float(np.float32(1e-3))
    GM = float(np.float32(1.0 / n))  # the context keeps GM as float
    g = Gravity(mesh=16, order=2, bwidth=1.0, hsoft=soft, GM=GM, kernel=kernel)
    g.upload_dict(P)
    sel = np.arange(0, n, 23)
    ref_f, ref_p = g.ewald_direct(P["x"][sel], P["y"][sel], P["z"][sel], alpha=10.5, rcut=0.5,
                                  kmax=kmax, with_pot=True)
    lib = _lib.load()
    stream = torch.cuda.Stream() if side_stream else None
    sp = ctypes.c_void_p(stream.cuda_stream) if side_stream else None
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()  # noqa: E731
    qx, qy, qz = dev(P["x"]), dev(P["y"]), dev(P["z"])
    sx, sy, sz = dev(P["x"][sel]), dev(P["y"][sel]), dev(P["z"][sel])
    ns = len(sel)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    for call in range(2):
        f = torch.full((ns, 3), float("nan"), dtype=torch.float64, device="cuda")
        pot = torch.full((ns,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.ct2g_ewald_direct_noalloc(0, vp(qx), vp(qy), vp(qz), n, vp(sx), vp(sy), vp(sz),
                                           ns, kernel, soft, GM, 10.5, 0.5, kmax, vp(f),
                                           vp(pot), sp)
        assert rc == 0, call
        assert torch.cuda.current_device() == 0  # the caller's device is kept
        torch.cuda.synchronize()
        got_f, got_p = f.cpu().numpy(), pot.cpu().numpy()
        assert np.abs(got_f - ref_f).max() <= 1e-10 * np.abs(ref_f).max(), call
        assert np.abs(got_p - ref_p).max() <= 1e-10 * np.abs(ref_p).max(), call
    # sizes beyond the static scratch are refused, not run
    rc = lib.ct2g_ewald_direct_noalloc(0, vp(qx), vp(qy), vp(qz), n, vp(sx), vp(sy), vp(sz), ns,
                                       kernel, soft, GM, 10.5, 0.5, 25, vp(f), vp(pot), sp)
    assert rc == 1  # CT2G_EINVAL
    g.close()
