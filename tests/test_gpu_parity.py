"""GPU parity tests: every stage of the CUDA path through the C ABI against
the CPU oracle on the same seeded particles.

Tolerances (written per test): binning, kick update and drift are integer or
exactly-rounded work and must be bit-exact; the mesh stages run in FP32
(moments accumulated in FP64, stored FP32) against an FP64 oracle.
"""
import numpy as np
import pytest

from ct2_b200 import ics
from ct2_b200.gravity import Gravity, kick_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _plummer(n, seed, mbits):
    return ics.plummer_spheres(n, seed=seed, nspheres=4, a=2.0 / (1 << mbits))


def _ctx(mbits, p, bw, soft, kernel=0, **kw):
    return Gravity(mesh=1 << mbits, order=p, bwidth=bw, hsoft=soft, kernel=kernel, **kw)


@pytest.mark.parametrize("mbits,n", [(3, 1000), (4, 20000), (5, 5000), (6, 70000)])
def test_binning_bit_exact(gpu, mbits, n):
    P = _plummer(n, 7 + mbits, mbits)
    g = _ctx(mbits, 2, 1.0, 1e-3)
    g.upload_dict(P)
    g.particle_to_grid()
    d = g.download()
    perm, cs = O.bin_stable(P["x"], P["y"], P["z"], mbits)
    # the sorted order is the oracle's stable order, id for id
    assert np.array_equal(d["id"].astype(np.int64), perm)
    for k in ("x", "y", "z", "vx", "vy", "vz", "rung"):
        assert np.array_equal(d[k], P[k][perm])
    b, e = g.cells()
    ob, oe = O.cell_ranges_rowmajor(cs, mbits)
    assert np.array_equal(b, ob) and np.array_equal(e, oe)
    # and the reference's bisection reaches the same leaves with the same ranges
    ids, cb, ce = O.bin_bisect(P["x"], P["y"], P["z"], mbits)
    assert np.array_equal(cb, b) and np.array_equal(ce, e)
    # re-binning an already sorted store is the identity (stability)
    g.particle_to_grid()
    assert np.array_equal(g.download()["id"], d["id"])


@pytest.mark.parametrize("n,ppcell", [(5000, 64), (32768, 16), (23000, 1)])
def test_binning_matches_reference_fixture(gpu, n, ppcell):
    """Against the reference's own compiled bisection (tests/golden/
    ref_binning.npz): the same cells, in the same order, with the same
    particles in each; only the order inside a cell (arbitrary in the
    reference's Hoare partition) is the stable one."""
    import os
    g0 = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_binning.npz"))
    order = g0["order_%d_%d" % (n, ppcell)].astype(np.int64)
    mesh = int(g0["ncell_%d_%d" % (n, ppcell)])
    mbits = mesh.bit_length() - 1
    P = ics.plummer_spheres(n, seed=3, nspheres=4, a=0.02)
    g = _ctx(mbits, 2, 1.0, 1e-3)
    g.upload_dict(P)
    g.particle_to_grid()
    ids = g.download()["id"].astype(np.int64)
    keys = O.cell_keys(P["x"], P["y"], P["z"], mbits).astype(np.int64)
    assert np.array_equal(keys[ids], keys[order])
    b, e = g.cells()
    for c in np.flatnonzero(e > b):
        assert np.array_equal(np.sort(ids[b[c]:e[c]]), np.sort(order[b[c]:e[c]]))


def test_binning_empty_and_single(gpu):
    g = _ctx(3, 1, 1.0, 1e-3)
    one = ics.lattice(1, seed=0)
    g.upload_dict(one)
    g.particle_to_grid()
    b, e = g.cells()
    assert (e - b).sum() == 1
    z = np.zeros(0, np.uint32)
    zf = np.zeros(0, np.float32)
    g.upload(z, z, z, zf, zf, zf)
    g.particle_to_grid()
    b, e = g.cells()
    assert (e - b).sum() == 0


@pytest.mark.parametrize("p", [1, 3, 5])
def test_p2m_matches_oracle(gpu, p):
    mbits = 4
    P = _plummer(20000, 3, mbits)
    g = _ctx(mbits, p, 1.0, 1e-3)
    g.upload_dict(P)
    g.particle_to_grid()
    g.compute_multipoles()
    got = g.multipoles()
    perm, cs = O.bin_stable(P["x"], P["y"], P["z"], mbits)
    ref = O.p2m(P["x"][perm], P["y"][perm], P["z"][perm], cs, mbits, p)
    # FP64 accumulation stored as FP32: per-component relative 1e-6 of the scale
    for k in range(ref.shape[0]):
        s = np.abs(ref[k]).max()
        assert np.abs(got[k] - ref[k]).max() <= 1e-6 * s + 1e-30, k


@pytest.mark.parametrize("mbits,p,bw,kernel", [(3, 2, 1.0, 0), (4, 4, 2.0, 0), (5, 3, 3.0, 1),
                                               (4, 6, 1.0, 0)])
def test_greens_matches_oracle(gpu, mbits, p, bw, kernel):
    soft = 0.5 / (1 << mbits)
    g = _ctx(mbits, p, bw, soft, kernel)
    got = g.greens()
    ref = O.greens_k(mbits, p, kernel, soft, bw)
    # FP64 build stored FP32: relative to each component's largest value
    for k in range(ref.shape[0]):
        s = np.abs(ref[k]).max()
        assert np.abs(got[k] - ref[k]).max() <= 2e-6 * s, k


@pytest.mark.parametrize("N", [4, 8, 16, 32, 64])
def test_fft_r2c_c2r_fp64(gpu, N):
    rng = np.random.Generator(np.random.PCG64(N))
    x = rng.uniform(-1, 1, (2, N, N, N))
    g = _ctx(3, 1, 1.0, 1e-3)
    y = g.fft_r2c_3d(x)
    nk = N * N * (N // 2 + 1)
    ref = np.fft.rfftn(x, axes=(1, 2, 3)).reshape(2, -1)
    got = y[:, :nk] + 1j * y[:, nk:]
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    back = g.fft_c2r_3d(y, N)
    assert np.abs(back - x * N ** 3).max() <= 1e-11 * N ** 3


GOLD = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                          "fft1d_golden.npz"))


@pytest.mark.parametrize("N", [8, 16, 32, 64, 128, 256])
def test_fft_axis_lines_match_reference_golden(gpu, N):
    # a grid varying along one axis only: its 3D transform is N^2 times the 1D
    # transform, compared with the reference's own fft_real output
    x1 = GOLD["real_in_%d" % N]
    X1 = O.halfcomplex_to_complex(GOLD["real_out_%d" % N])
    g = _ctx(3, 1, 1.0, 1e-3)
    nk = N * N * (N // 2 + 1)
    grid = np.broadcast_to(x1[None, None, :], (N, N, N)).copy()
    y = g.fft_r2c_3d(grid)
    spec = (y[:nk] + 1j * y[nk:]).reshape(N, N, N // 2 + 1)
    assert np.abs(spec[0, 0, :] / N ** 2 - X1).max() <= 1e-12 * np.abs(X1).max()
    # along the first axis (full complex range): conj-symmetric extension
    grid = np.broadcast_to(x1[:, None, None], (N, N, N)).copy()
    y = g.fft_r2c_3d(grid)
    spec = (y[:nk] + 1j * y[nk:]).reshape(N, N, N // 2 + 1)
    full = np.concatenate([X1, np.conj(X1[1:N // 2][::-1])])
    assert np.abs(spec[:, 0, 0] / N ** 2 - full).max() <= 1e-12 * np.abs(X1).max()


def _oracle_pipeline(P, mbits, p, bw, soft, kernel, GM):
    return O.method_forces(P["x"], P["y"], P["z"], mbits, p, kernel, soft, bw, GM)


@pytest.mark.parametrize("mbits,p,bw,kernel,n", [(4, 3, 2.0, 0, 20000), (5, 4, 2.0, 0, 30000),
                                                 (4, 5, 3.0, 1, 8000), (5, 2, 1.0, 0, 30000)])
def test_expansions_and_forces_match_oracle(gpu, mbits, p, bw, kernel, n):
    P = _plummer(n, 11 + p, mbits)
    soft = 0.02 / (1 << mbits)
    GM = 1.0 / n
    g = _ctx(mbits, p, bw, soft, kernel, GM=GM)
    g.upload_dict(P)
    g.particle_to_grid()
    g.compute_expansions()
    L = g.expansions()
    r = _oracle_pipeline(P, mbits, p, bw, soft, kernel, GM)
    # FP32 FFTs of FP32-stored moments: relative to each component's scale
    for k in range(L.shape[0]):
        s = np.abs(r["L"][k]).max()
        assert np.abs(L[k] - r["L"][k]).max() <= 2e-5 * s, k
    g.compute_forces()
    f, pot = g.forces()
    d = g.download()
    assert np.array_equal(d["id"].astype(np.int64), r["perm"])
    fref = r["ffar"] + r["fnear"]
    err = np.linalg.norm(f - fref, axis=1) / np.maximum(np.linalg.norm(fref, axis=1), 1e-30)
    # FP32 near field + FP32 mesh against FP64: rms 1e-5, max 1e-3 relative
    assert np.sqrt(np.mean(err ** 2)) < 1e-5
    assert err.max() < 1e-3
    # the potential sums the self term -GM/eps and the far-field constant in
    # FP32, so it carries more cancellation than the force: rms 1e-3
    prel = np.abs(pot - r["pot"]) / np.abs(r["pot"])
    assert np.sqrt(np.mean(prel ** 2)) < 1e-3
    # the exact interaction count: sum over cells of n_c * sum_nbr n_nbr
    assert g.interaction_count() > 0


def test_kick_update_bit_exact(gpu):
    rng = np.random.Generator(np.random.PCG64(5))
    n = 50000
    P = ics.lattice(1, seed=0)
    x = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    v = rng.normal(0, 1, (3, n)).astype(np.float32)
    rung = rng.integers(0, 5, n).astype(np.int8)
    f = (rng.normal(0, 1, (n, 3)) * 10.0 ** rng.uniform(-6, 6, (n, 1))).astype(np.float32)
    g = _ctx(3, 1, 1.0, 1e-3)
    g.upload(x, x, x, v[0], v[1], v[2], rung)
    for params in (kick_params(True, True, True, False, 0, 1e-2, 0.15, 0.01, 1.0),
                   kick_params(True, False, False, False, 2, 3e-3, 0.2, 1e-3, 0.5),
                   kick_params(False, True, True, True, 1, 1e-2, 0.15, 0.02, 2.0)):
        g.upload(x, x, x, v[0], v[1], v[2], rung)
        g.upload_forces(f)
        mr = g.kick_update(params)
        d = g.download()
        ovx, ovy, ovz, orung, omr = O.kick_update(
            v[0], v[1], v[2], rung, f[:, 0], f[:, 1], f[:, 2], ascending=params.ascending,
            descending=params.descending, top=params.top, first=params.first, prung=params.rung,
            t0=params.t0, eta=params.eta, max_dt=params.max_dt, scale=params.scale, hsoft=1e-3)
        assert np.array_equal(d["vx"], ovx) and np.array_equal(d["vy"], ovy)
        assert np.array_equal(d["vz"], ovz) and np.array_equal(d["rung"], orung)
        assert mr == omr


def test_drift_bit_exact(gpu):
    rng = np.random.Generator(np.random.PCG64(9))
    n = 100000
    x, y, z = (rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(3))
    v = (rng.normal(0, 1, (3, n)) * 10.0 ** rng.uniform(-4, 2, (1, n))).astype(np.float32)
    g = _ctx(3, 1, 1.0, 1e-3)
    g.upload(x, y, z, v[0], v[1], v[2])
    g.drift(1e-3, 0.7)
    d = g.download()
    ox, oy, oz = O.drift(x, y, z, v[0], v[1], v[2], 1e-3, 0.7)
    assert np.array_equal(d["x"], ox) and np.array_equal(d["y"], oy) and np.array_equal(d["z"], oz)


def test_ewald_gpu_matches_cpu(gpu):
    P = _plummer(4000, 2, 4)
    n = 4000
    g = _ctx(4, 2, 1.0, 1e-3, GM=1.0 / n)
    g.upload_dict(P)
    sel = np.arange(0, n, 37)
    fg, pg = g.ewald_direct(P["x"][sel], P["y"][sel], P["z"][sel], with_pot=True)
    # the context keeps GM (and hsoft) as float, like the reference's options
    fc, pc = O.ewald_direct(P["x"][sel], P["y"][sel], P["z"][sel], P["x"], P["y"], P["z"], 0,
                            float(np.float32(1e-3)), float(np.float32(1.0 / n)), with_pot=True)
    assert np.abs(fg - fc).max() <= 1e-10 * np.abs(fc).max()
    assert np.abs(pg - pc).max() <= 1e-10 * np.abs(pc).max()


def test_one_kick_drift_step_matches_oracle(gpu):
    # config-1 shape at reduced N: lattice + noise, one kick+drift at rung 0
    ng, mbits, p, bw = 16, 5, 4, 3.0
    P = ics.lattice(ng, seed=0)
    n = ng ** 3
    soft = 1.0 / (50 * ng)
    g = _ctx(mbits, p, bw, soft, GM=1.0 / n)
    g.upload_dict(P)
    t0 = 1e-3
    mr, minrung = g.kick_step(0, 0, 1.0, 1.0, 1.0, t0, 0)
    d = g.download()
    r = _oracle_pipeline(P, mbits, p, bw, soft, 0, 1.0 / n)
    f = (r["ffar"] + r["fnear"]).astype(np.float32)
    perm = r["perm"]
    ovx, ovy, ovz, orung, omr = O.kick_update(
        P["vx"][perm], P["vy"][perm], P["vz"][perm], P["rung"][perm], f[:, 0], f[:, 1], f[:, 2],
        ascending=1, descending=1, top=1, first=0, prung=0, t0=t0, eta=0.15, max_dt=0.01,
        scale=1.0, hsoft=soft)
    assert np.array_equal(d["id"].astype(np.int64), perm)
    vref = np.stack([ovx, ovy, ovz], 1)
    vgot = np.stack([d["vx"], d["vy"], d["vz"]], 1)
    err = np.linalg.norm(vgot - vref, axis=1) / np.maximum(np.linalg.norm(vref, axis=1), 1e-30)
    assert np.sqrt(np.mean(err ** 2)) < 1e-5
    ox, oy, oz = O.drift(P["x"][perm], P["y"][perm], P["z"][perm], d["vx"], d["vy"], d["vz"],
                         t0, 1.0)
    assert np.array_equal(d["x"], ox) and np.array_equal(d["y"], oy) and np.array_equal(d["z"], oz)


def test_method_accuracy_vs_ewald(gpu):
    # clustered set at the config-2 density (1/8 particle per cell), 3-cell
    # stencil, order 5: rms relative force error against FP64 Ewald <= 1e-4
    mbits = 6
    n = 32768
    P = ics.plummer_spheres(n, seed=0, nspheres=8, a=0.005 * 4)
    soft = 1.0 / 1600
    g = _ctx(mbits, 5, 3.0, soft, GM=1.0 / n)
    g.upload_dict(P)
    g.particle_to_grid()
    g.compute_forces()
    f, _ = g.forces()
    d = g.download()
    truth = np.empty((n, 3))
    sel = np.arange(n)
    tr = g.ewald_direct(d["x"], d["y"], d["z"])
    e = O.force_errors(f.astype(np.float64), tr)
    assert e["rms_rel"] < 1e-4, e


@pytest.mark.parametrize("N", [4, 8, 16, 32, 64, 128, 256])
def test_fft_fp32_device_roundtrip(gpu, N):
    # the FP32 mesh transform (device pointers on the context stream) against
    # numpy's FP64 rfftn: FP32 rounding, relative 2e-6 of the largest mode
    import ctypes

    import torch
    from ct2_b200 import _lib
    rng = np.random.Generator(np.random.PCG64(N + 1))
    x = rng.uniform(-1, 1, (3, N, N, N)).astype(np.float32)
    g = _ctx(3, 1, 1.0, 1e-3)
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty((3, N, N, N // 2 + 1), dtype=torch.complex64, device="cuda")
    lib = _lib.load()
    torch.cuda.synchronize()
    assert lib.ct2g_fft3d_f32_dev(g.handle, 1, ctypes.c_void_p(dx.data_ptr()),
                                  ctypes.c_void_p(dy.data_ptr()), N, 3) == 0
    g.synchronize()
    ref = np.fft.rfftn(x.astype(np.float64), axes=(1, 2, 3))
    got = dy.cpu().numpy()
    assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max()
    back = torch.empty_like(dx)
    assert lib.ct2g_fft3d_f32_dev(g.handle, -1, ctypes.c_void_p(back.data_ptr()),
                                  ctypes.c_void_p(dy.data_ptr()), N, 3) == 0
    g.synchronize()
    assert np.abs(back.cpu().numpy() / N ** 3 - x).max() <= 2e-6
