"""Python host layer over the ct2g C ABI, mirroring the reference's
operator interface for the gravity step (dmarce1/ct2):

  particle store   particle_allocate / SoA accessors (src/particle.cpp:273-288,
                   cosmictiger/particle.hpp:22-56)  -> Gravity.upload / download
  particle_to_grid (src/particle.cpp:349-362)      -> Gravity.particle_to_grid
  particle_compute_multipoles / _expansions         -> compute_multipoles /
                   (src/particle.cpp:180-271)          compute_expansions
  kick(const kick_params&) (src/kick.cpp:105-125)   -> Gravity.kick
  drift(float dt, float scale) (src/drift.cpp:4-18) -> Gravity.drift
  kick_step(...) (src/main.cpp:8-92)                -> Gravity.kick_step
  fft_r2c_3d / fft_c2r_3d (cosmictiger/fft.hpp:28-29) -> fft_r2c_3d / fft_c2r_3d

Beyond the reference: Gravity.kick_drift (one kick + drift, optionally as a
replayed CUDA graph), box contexts (nbox independent periodic boxes sharing
one mesh), Batch (several contexts stepped by one graph launch) and the
launch-shape tuning / autotuner.

Arrays are numpy; every call goes to libct2g.so on the GPU.  Errors raise
CT2GError with the library's message (the reference aborts or has none).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import CT2GError, KickParams, Options, Tuning


def ncomp(p: int) -> int:
    return (p + 1) * (p + 2) * (p + 3) // 6


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class kick_params:
    """Field for field cosmictiger/kick.hpp:10-20."""
    ascending: bool = True
    descending: bool = True
    top: bool = True
    first: bool = False
    rung: int = 0
    t0: float = 1e-3
    eta: float = 0.15
    max_dt: float = 0.01
    scale: float = 1.0

    def _c(self):
        return KickParams(int(self.ascending), int(self.descending), int(self.top),
                          int(self.first), int(self.rung), self.t0, self.eta, self.max_dt,
                          self.scale)


class Gravity:
    """One GPU context: particle store, mesh, Green's tensor, stream."""

    def __init__(self, mesh=64, order=4, bwidth=3.0, hsoft=1.0 / 50.0, eta=0.15, GM=0.0,
                 kernel=_lib.SOFT_PLUMMER, device=0, max_particles=0, nbox=1):
        self._l = _lib.load()
        o = Options()
        self._l.ct2g_default_options(ctypes.byref(o))
        o.mesh, o.order, o.bwidth, o.hsoft, o.eta, o.GM = mesh, order, bwidth, hsoft, eta, GM
        o.kernel, o.device, o.max_particles = kernel, device, max_particles
        h = ctypes.c_void_p()
        rc = self._l.ct2g_create_boxes(ctypes.byref(o), int(nbox), ctypes.byref(h))
        if rc != 0:
            raise CT2GError(rc, "ct2g_create_boxes(mesh=%d, order=%d, bwidth=%g, nbox=%d)"
                            % (mesh, order, bwidth, nbox))
        self._h = h
        self.device = int(device)
        self.mesh, self.order, self.bwidth, self.kernel = mesh, order, bwidth, kernel
        self.nbox = int(nbox)
        self.nc = ncomp(order)

    # -- plumbing -----------------------------------------------------------
    def _chk(self, rc):
        if rc != 0:
            raise CT2GError(rc, self._l.ct2g_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._l.ct2g_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def options(self):
        o = Options()
        self._chk(self._l.ct2g_get_options(self._h, ctypes.byref(o)))
        return o

    def set_params(self, hsoft, eta, GM=0.0):
        self._chk(self._l.ct2g_set_params(self._h, hsoft, eta, GM))

    # -- particle store -----------------------------------------------------
    def upload(self, x, y, z, vx, vy, vz, rung=None):
        arrs = [np.ascontiguousarray(a, t) for a, t in
                ((x, np.uint32), (y, np.uint32), (z, np.uint32), (vx, np.float32),
                 (vy, np.float32), (vz, np.float32))]
        r = None if rung is None else np.ascontiguousarray(rung, np.int8)
        n = len(arrs[0])
        self._chk(self._l.ct2g_upload_particles(self._h, *[_ptr(a) for a in arrs], _ptr(r), n))

    def upload_dict(self, d):
        self.upload(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d.get("rung"))

    def set_boxes(self, counts, GM):
        """Box b holds the next counts[b] uploaded particles; GM[b] = G x mass."""
        c = np.ascontiguousarray(counts, np.uint64)
        g = np.ascontiguousarray(GM, np.float32)
        if len(c) != self.nbox or len(g) != self.nbox:
            raise ValueError("need %d box counts and GM values" % self.nbox)
        self._chk(self._l.ct2g_set_boxes(self._h, _ptr(c), _ptr(g)))

    def count(self):
        return int(self._l.ct2g_particle_count(self._h))

    def download(self):
        n = self.count()
        out = dict(x=np.empty(n, np.uint32), y=np.empty(n, np.uint32), z=np.empty(n, np.uint32),
                   vx=np.empty(n, np.float32), vy=np.empty(n, np.float32),
                   vz=np.empty(n, np.float32), rung=np.empty(n, np.int8),
                   id=np.empty(n, np.uint32))
        self._chk(self._l.ct2g_download_particles(
            self._h, *[_ptr(out[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "rung", "id")]))
        return out

    # -- stages -------------------------------------------------------------
    def particle_to_grid(self):
        self._chk(self._l.ct2g_particle_to_grid(self._h))

    def cells(self):
        """(begin, end) per row-major cell box*mesh^3 + (i*mesh+j)*mesh+k."""
        b = np.empty(self.nbox * self.mesh ** 3, np.int64)
        e = np.empty(self.nbox * self.mesh ** 3, np.int64)
        self._chk(self._l.ct2g_download_cells(self._h, _ptr(b), _ptr(e)))
        return b, e

    def compute_multipoles(self):
        self._chk(self._l.ct2g_compute_multipoles(self._h))

    def _grid_shape(self):
        m = self.mesh
        return (self.nc, m, m, m) if self.nbox == 1 else (self.nc, self.nbox, m, m, m)

    def multipoles(self):
        out = np.empty(self._grid_shape(), np.float32)
        self._chk(self._l.ct2g_download_multipoles(self._h, _ptr(out)))
        return out

    def compute_expansions(self):
        self._chk(self._l.ct2g_compute_expansions(self._h))

    def expansions(self):
        out = np.empty(self._grid_shape(), np.float32)
        self._chk(self._l.ct2g_download_expansions(self._h, _ptr(out)))
        return out

    def greens(self):
        m = self.mesh
        out = np.empty((self.nc, m, m, m // 2 + 1), np.float32)
        self._chk(self._l.ct2g_download_greens(self._h, _ptr(out)))
        return out

    def compute_forces(self):
        self._chk(self._l.ct2g_compute_forces(self._h))

    def forces(self):
        n = self.count()
        f = [np.empty(n, np.float32) for _ in range(4)]
        self._chk(self._l.ct2g_download_forces(self._h, *[_ptr(a) for a in f]))
        return np.stack(f[:3], 1), f[3]

    def upload_forces(self, f):
        f = np.asarray(f, np.float32)
        cols = [np.ascontiguousarray(f[:, k]) for k in range(3)]
        self._chk(self._l.ct2g_upload_forces(self._h, *[_ptr(c) for c in cols]))

    def kick_update(self, params: kick_params) -> int:
        mr = ctypes.c_int(0)
        self._chk(self._l.ct2g_kick_update(self._h, ctypes.byref(params._c()), ctypes.byref(mr)))
        return mr.value

    def kick(self, params: kick_params) -> int:
        """int kick(const kick_params&): returns the max rung."""
        mr = ctypes.c_int(0)
        self._chk(self._l.ct2g_kick(self._h, ctypes.byref(params._c()), ctypes.byref(mr)))
        return mr.value

    def drift(self, dt: float, scale: float):
        self._chk(self._l.ct2g_drift(self._h, dt, scale))

    def kick_drift(self, params: kick_params, dt: float, scale: float = 1.0, graph=True,
                   wait=True):
        """particle_to_grid + kick + drift; graph=True records the sequence
        once into a CUDA graph and replays it.  Returns the max rung (None
        with wait=False: the call only queues the work)."""
        mr = ctypes.c_int(0)
        self._chk(self._l.ct2g_kick_drift(self._h, ctypes.byref(params._c()), dt, scale,
                                          _lib.STEP_GRAPH if graph else 0,
                                          ctypes.byref(mr) if wait else None))
        return mr.value if wait else None

    def kick_drift_host(self, params: kick_params, dt: float, state, out, scale: float = 1.0,
                        graph=True):
        """One kick+drift from host arrays to host arrays (ct2g_kick_drift_host):
        `state` holds x, y, z (uint32), vx, vy, vz (float32) and optionally
        rung (int8) of the uploaded particle count; `out` the preallocated
        arrays to fill (any key may be missing; "id" maps the new order back
        to input order).  Pinned arrays give the copies their full rate.
        Returns the max rung."""
        n = len(state["x"])
        ins = [state[k] for k in ("x", "y", "z", "vx", "vy", "vz")] + [state.get("rung")]
        for a, t in zip(ins, (np.uint32,) * 3 + (np.float32,) * 3 + (np.int8,)):
            if a is not None and (a.dtype != t or len(a) != n or not a.flags["C_CONTIGUOUS"]):
                raise ValueError("state arrays: %d contiguous values of %s" % (n, np.dtype(t)))
        outs = [out.get(k) for k in ("x", "y", "z", "vx", "vy", "vz", "rung", "id")]
        for a, t in zip(outs, (np.uint32,) * 3 + (np.float32,) * 3 + (np.int8, np.uint32)):
            if a is not None and (a.dtype != t or len(a) != n or not a.flags["C_CONTIGUOUS"]):
                raise ValueError("output arrays: %d contiguous values of %s" % (n, np.dtype(t)))
        mr = ctypes.c_int(0)
        self._chk(self._l.ct2g_kick_drift_host(
            self._h, ctypes.byref(params._c()), dt, scale, _lib.STEP_GRAPH if graph else 0,
            *[_ptr(a) for a in ins], n, *[_ptr(a) for a in outs], ctypes.byref(mr)))
        return mr.value

    # -- learned near-field correction ---------------------------------------
    def learned_enable(self, bwidth_ext):
        self._chk(self._l.ct2g_learned_enable(self._h, float(bwidth_ext)))

    def learned_select(self, mode, threshold=0.0):
        """mode: 'none', 'fixed', 'mlp' or 'all' (or the CT2G_SELECT_* value)."""
        m = {"none": 0, "fixed": 1, "mlp": 2, "all": 3}.get(mode, mode)
        self._chk(self._l.ct2g_learned_select(self._h, int(m), float(threshold)))

    def learned_collect(self):
        n = ctypes.c_size_t(0)
        self._chk(self._l.ct2g_learned_collect(self._h, ctypes.byref(n)))
        return n.value

    def learned_dataset(self):
        n = ctypes.c_size_t(0)
        self._chk(self._l.ct2g_learned_dataset(self._h, None, None, 0, ctypes.byref(n)))
        X = np.empty((n.value, _lib.MLP_NIN), np.float32)
        T = np.empty(n.value, np.float32)
        self._chk(self._l.ct2g_learned_dataset(self._h, _ptr(X), _ptr(T), n.value, None))
        return X, T

    def learned_clear(self):
        self._chk(self._l.ct2g_learned_clear(self._h))

    def learned_cells(self):
        """Cells of the last selection pass: dict of keys, X, score, pred, selected."""
        n, s = ctypes.c_size_t(0), ctypes.c_size_t(0)
        self._chk(self._l.ct2g_learned_cells(self._h, None, None, None, None, None, 0,
                                             ctypes.byref(n), ctypes.byref(s)))
        m = n.value
        out = dict(keys=np.empty(m, np.uint32), X=np.empty((m, _lib.MLP_NIN), np.float32),
                   score=np.empty(m, np.float32), pred=np.empty(m, np.float32),
                   selected=np.empty(m, np.uint8))
        self._chk(self._l.ct2g_learned_cells(self._h, _ptr(out["keys"]), _ptr(out["X"]),
                                             _ptr(out["score"]), _ptr(out["pred"]),
                                             _ptr(out["selected"]), m, None, None))
        out["nselected"] = s.value
        return out

    def mlp_init(self, seed=0):
        self._chk(self._l.ct2g_mlp_init(self._h, int(seed)))

    def mlp_set(self, params, fmean, fstd):
        p = np.ascontiguousarray(params, np.float32)
        m = np.ascontiguousarray(fmean, np.float32)
        sd = np.ascontiguousarray(fstd, np.float32)
        self._chk(self._l.ct2g_mlp_set(self._h, _ptr(p), _ptr(m), _ptr(sd)))

    def mlp_get(self):
        p = np.empty(_lib.MLP_NPARAM, np.float32)
        m = np.empty(_lib.MLP_NIN, np.float32)
        sd = np.empty(_lib.MLP_NIN, np.float32)
        self._chk(self._l.ct2g_mlp_get(self._h, _ptr(p), _ptr(m), _ptr(sd)))
        return p, m, sd

    def mlp_train(self, epochs=20, batch=4096, lr=1e-3, seed=0, normalize=True):
        loss = ctypes.c_float(0)
        self._chk(self._l.ct2g_mlp_train(self._h, int(epochs), int(batch), float(lr), int(seed),
                                         int(bool(normalize)), ctypes.byref(loss)))
        return loss.value

    def mlp_gradients(self, X, T):
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        g = np.empty(_lib.MLP_NPARAM, np.float32)
        loss = ctypes.c_float(0)
        self._chk(self._l.ct2g_mlp_gradients(self._h, _ptr(X), _ptr(T), len(T), _ptr(g),
                                             ctypes.byref(loss)))
        return g, loss.value

    def set_fft_mode(self, mode):
        """'fp32' (CUDA cores) or 'tc' (tensor-core DFT passes, BF16 hi+lo)."""
        m = {"fp32": _lib.FFT_FP32, "tc": _lib.FFT_TC_BF16X3}.get(mode, mode)
        self._chk(self._l.ct2g_set_fft_mode(self._h, int(m)))

    # -- launch shapes ------------------------------------------------------
    def tuning(self):
        t = Tuning()
        self._chk(self._l.ct2g_get_tuning(self._h, ctypes.byref(t)))
        return dict(dense_cell=t.dense_cell, near_blocks_per_sm=t.near_blocks_per_sm,
                    fft_tile=t.fft_tile, split_mg2l=t.split_mg2l, sparse_path=t.sparse_path,
                    overlap=t.overlap, mg2l_greens_direct=t.mg2l_greens_direct,
                    near_chunks_per_warp=t.near_chunks_per_warp, plane_pipe=t.plane_pipe,
                    cols_tma=t.cols_tma, x_tma=t.x_tma, p2m_compact=t.p2m_compact)

    def set_tuning(self, dense_cell=16, near_blocks_per_sm=0, fft_tile=0, split_mg2l=0,
                   sparse_path=2, overlap=0, mg2l_greens_direct=0, near_chunks_per_warp=0,
                   plane_pipe=0, cols_tma=1, x_tma=2, p2m_compact=0):
        t = Tuning(dense_cell, near_blocks_per_sm, fft_tile, split_mg2l, sparse_path, overlap,
                   mg2l_greens_direct, near_chunks_per_warp, plane_pipe, cols_tma, x_tma,
                   p2m_compact)
        self._chk(self._l.ct2g_set_tuning(self._h, ctypes.byref(t)))

    def autotune(self, params: kick_params, dt: float, scale: float = 1.0, cache_path=None):
        t = Tuning()
        cp = None if cache_path is None else str(cache_path).encode()
        self._chk(self._l.ct2g_autotune(self._h, ctypes.byref(params._c()), dt, scale, cp,
                                        ctypes.byref(t)))
        return dict(dense_cell=t.dense_cell, near_blocks_per_sm=t.near_blocks_per_sm,
                    fft_tile=t.fft_tile, split_mg2l=t.split_mg2l, sparse_path=t.sparse_path,
                    overlap=t.overlap, mg2l_greens_direct=t.mg2l_greens_direct,
                    near_chunks_per_warp=t.near_chunks_per_warp, plane_pipe=t.plane_pipe,
                    cols_tma=t.cols_tma, x_tma=t.x_tma, p2m_compact=t.p2m_compact)

    def kick_step(self, minrung, max_rung, scale, adot, tau, t0, minrung0, nocrop=False):
        """Returns (value, minrung): the reference's return value, which is its
        max_rung argument (main.cpp:68 shadows it, :90 returns the parameter),
        and minrung as updated through its reference argument.  The highest
        rung after the step is len(rung_counts()) - 1."""
        mr = ctypes.c_int(minrung)
        out = ctypes.c_int(0)
        self._chk(self._l.ct2g_kick_step(self._h, ctypes.byref(mr), max_rung, scale, adot, tau,
                                         t0, minrung0, int(nocrop), ctypes.byref(out)))
        return out.value, mr.value

    # rung bookkeeping
    def sort_by_rung(self, minrung):
        self._chk(self._l.ct2g_sort_by_rung(self._h, minrung))

    def push_rungs(self):
        self._chk(self._l.ct2g_push_rungs(self._h))

    def pop_rungs(self):
        self._chk(self._l.ct2g_pop_rungs(self._h))

    def set_minrung(self, minrung):
        self._chk(self._l.ct2g_set_minrung(self._h, minrung))

    def current_range(self):
        b, e = ctypes.c_size_t(), ctypes.c_size_t()
        self._chk(self._l.ct2g_current_range(self._h, ctypes.byref(b), ctypes.byref(e)))
        return b.value, e.value

    def rung_counts(self):
        c = np.zeros(128, np.uint64)
        nr = ctypes.c_int(0)
        self._chk(self._l.ct2g_rung_counts(self._h, _ptr(c), 128, ctypes.byref(nr)))
        return c[:nr.value].astype(np.int64)

    # -- FFT ----------------------------------------------------------------
    def _on_torch_order(self, call):
        """Run `call` (work on device buffers that torch owns) on the context's
        stream, ordered after the work already queued on torch's current
        stream, and make torch's current stream wait for it: the buffers are
        written by torch and read back by torch, and the context's stream is
        a non-blocking stream of its own, so without the two waits the
        kernels could read a buffer before torch's copy into it has finished
        (the context's stream also runs at a higher priority)."""
        import sys
        torch = sys.modules.get("torch")
        if torch is None or not torch.cuda.is_initialized():
            return call()
        ext = torch.cuda.ExternalStream(self.stream(), device=self.device)
        cur = torch.cuda.current_stream(self.device)
        ext.wait_stream(cur)
        r = call()
        cur.wait_stream(ext)
        return r

    def fft3d_c2c_dev(self, ptr, N, batch, dir=1):
        """In-place complex 3D FFT of `batch` device grids (a device pointer,
        e.g. a torch tensor's data_ptr()) on the context's stream, ordered
        with torch's current stream both ways."""
        self._on_torch_order(lambda: self._chk(self._l.ct2g_fft3d_c2c_f32_dev(
            self._h, dir, ctypes.c_void_p(ptr), N, batch)))

    def fft3d_r2c_dev(self, real_ptr, cplx_ptr, N, batch, dir=1):
        """The real <-> half-spectrum 3D FFT on device pointers (dir +1 r2c,
        -1 c2r), FP32, ordered with torch's current stream both ways."""
        self._on_torch_order(lambda: self._chk(self._l.ct2g_fft3d_f32_dev(
            self._h, dir, ctypes.c_void_p(real_ptr), ctypes.c_void_p(cplx_ptr), N, batch)))

    def cic_deposit(self, N, ptr):
        """CIC mass and first moments of the particles onto four complex
        device grids float2[4][N][N][N] at `ptr`, ordered with torch's current
        stream both ways."""
        self._on_torch_order(lambda: self._chk(self._l.ct2g_cic_deposit(
            self._h, N, ctypes.c_void_p(ptr))))

    def fft1d_real(self, X, N, lanes=1, dir=1):
        """fft_real (fft.hpp:25-26) in place on a float64 array: input in
        bit-reversed order, output halfcomplex; lanes interleaved."""
        assert X.dtype == np.float64 and X.flags.c_contiguous and X.size >= N * lanes
        self._chk(self._l.ct2g_fft1d_real(self._h, _ptr(X), N, lanes, dir))

    def fft1d_complex(self, X, N, lanes=1, dir=1):
        """fft_complex (fft.hpp:27) in place: element n of lane l at
        X[(2n)*lanes + l] (real) and X[(2n+1)*lanes + l] (imaginary)."""
        assert X.dtype == np.float64 and X.flags.c_contiguous and X.size >= 2 * N * lanes
        self._chk(self._l.ct2g_fft1d_complex(self._h, _ptr(X), N, lanes, dir))

    def scramble(self, X, N1, N2, N3):
        assert X.dtype == np.float64 and X.flags.c_contiguous and X.size >= N1 * N2 * N3
        self._chk(self._l.ct2g_scramble(self._h, _ptr(X), N1, N2, N3))

    def transpose_yz(self, X, N):
        assert X.dtype == np.float64 and X.flags.c_contiguous and X.size >= N ** 3
        self._chk(self._l.ct2g_transpose_yz(self._h, _ptr(X), N))

    def transpose_r2c(self, xin, xout, N):
        xin = np.ascontiguousarray(xin, np.float64)
        assert xout.dtype == np.float64 and xout.size >= 2 * N * N * (N // 2 + 1)
        self._chk(self._l.ct2g_transpose_r2c(self._h, _ptr(xin), _ptr(xout), N))

    def transpose_c2r(self, xin, xout, N):
        xin = np.ascontiguousarray(xin, np.float64)
        assert xout.dtype == np.float64 and xout.size >= N ** 3
        self._chk(self._l.ct2g_transpose_c2r(self._h, _ptr(xin), _ptr(xout), N))

    def twiddles(self, which, N):
        out = np.zeros(N, np.float64)
        self._chk(self._l.ct2g_twiddles(self._h, which, N, _ptr(out)))
        return out

    def fft_r2c_3d(self, x):
        """x: float64 [batch,]N,N,N -> split planes float64 [batch,] 2*N*N*(N/2+1)."""
        x = np.ascontiguousarray(x, np.float64)
        N = x.shape[-1]
        b = 1 if x.ndim == 3 else x.shape[0]
        out = np.empty((b, 2 * N * N * (N // 2 + 1)), np.float64)
        self._chk(self._l.ct2g_fft_r2c_3d(self._h, _ptr(x), _ptr(out), N, b))
        return out[0] if x.ndim == 3 else out

    def fft_c2r_3d(self, y, N):
        y = np.ascontiguousarray(y, np.float64)
        b = 1 if y.ndim == 1 else y.shape[0]
        out = np.empty((b, N, N, N), np.float64)
        self._chk(self._l.ct2g_fft_c2r_3d(self._h, _ptr(y), _ptr(out), N, b))
        return out[0] if y.ndim == 1 else out

    # -- diagnostics --------------------------------------------------------
    def ewald_direct(self, sx, sy, sz, alpha=10.5, rcut=0.5, kmax=20, with_pot=False):
        sx, sy, sz = (np.ascontiguousarray(a, np.uint32) for a in (sx, sy, sz))
        ns = len(sx)
        f = np.empty((ns, 3), np.float64)
        pot = np.empty(ns, np.float64) if with_pot else None
        self._chk(self._l.ct2g_ewald_direct(self._h, _ptr(sx), _ptr(sy), _ptr(sz), ns, alpha,
                                            rcut, kmax, _ptr(f), _ptr(pot)))
        return (f, pot) if with_pot else f

    def stage_times(self):
        t = np.zeros(7, np.float32)
        self._chk(self._l.ct2g_stage_times(self._h, _ptr(t), 7))
        return t

    def synchronize(self):
        self._chk(self._l.ct2g_synchronize(self._h))

    def wait_selftest(self, polls):
        """Queue the failure-path self-test (a bounded wait that runs out)."""
        self._chk(self._l.ct2g_wait_selftest(self._h, int(polls)))

    def synchronize_status(self):
        """ct2g_synchronize's status code (no exception)."""
        return int(self._l.ct2g_synchronize(self._h))

    def stream(self):
        return self._l.ct2g_stream(self._h)

    def launch_count(self):
        return int(self._l.ct2g_launch_count(self._h))

    def interaction_count(self):
        return int(self._l.ct2g_interaction_count(self._h))


class Batch:
    """Several contexts on one device stepped by one CUDA graph launch (on the
    first context's stream); each context runs on its own stream inside it."""

    def __init__(self, contexts):
        self._l = _lib.load()
        self.contexts = list(contexts)
        arr = (ctypes.c_void_p * len(self.contexts))(*[g.handle for g in self.contexts])
        h = ctypes.c_void_p()
        rc = self._l.ct2g_batch_create(arr, len(self.contexts), ctypes.byref(h))
        if rc != 0:
            raise CT2GError(rc, self._l.ct2g_last_error(self.contexts[0].handle).decode())
        self._h = h

    def _chk(self, rc):
        if rc != 0:
            raise CT2GError(rc, self._l.ct2g_last_error(self.contexts[0].handle).decode())

    def kick_drift(self, params: kick_params, dt: float, scale: float = 1.0, wait=True):
        mr = ctypes.c_int(0)
        self._chk(self._l.ct2g_batch_kick_drift(self._h, ctypes.byref(params._c()), dt, scale,
                                                ctypes.byref(mr) if wait else None))
        return mr.value if wait else None

    def last_ms(self):
        ms = ctypes.c_float(0)
        self._chk(self._l.ct2g_batch_last_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "_h", None):
            self._l.ct2g_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
