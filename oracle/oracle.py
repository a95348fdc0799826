"""CPU oracle for the ct2 gravity step -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
this module, and only as the checker.  The product (ct2_b200) never calls it.

It wraps the C restatement in ct2_oracle.c (binning, P2M, real-space Green's
tensor, L2P + direct sum, kick update, drift, FP64 Ewald direct sum) and adds
the Fourier-space stages in numpy (pocketfft, FP64):

  forward r2c 3D FFT of every moment grid  -- particle.cpp:221-242
  Green's tensor to k-space (+ Ewald part) -- particle.cpp:116-178
  MG2L contraction per k-point             -- particle.cpp:244-250
  inverse c2r 3D FFT of every expansion    -- particle.cpp:251-270

Parity status: binning, kick update and drift are bit-exact restatements of
src/particle.cpp, src/kick.cpp and src/drift.cpp.  The multipole basis of the
un-vendored sfmm library (P2M/MG2L/L2P/greens/greens_ewald, no version pin)
cannot be reproduced, so the multipole stages are parity UNPINNED against sfmm;
the forces are pinned instead by the FP64 Ewald direct sum, which is itself
pinned by the simple-cubic-lattice Madelung constant.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

KERNEL_PLUMMER = 0
KERNEL_SPHERE = 1

# Green's-table Ewald split (box units): real-space images beyond the nearest
# are below 1e-16 for alpha*0.5 = 6; the k-space sum is cut at |k| <= 36.
GREENS_ALPHA = 12.0
GREENS_KMAX = 36
# FP64 Ewald direct sum: min-image real space cut at r=0.5 (erfc(5.25)~1e-13).
EWALD_ALPHA = 10.5
EWALD_RCUT = 0.5
EWALD_KMAX = 20

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64 = ctypes.c_int64
_int = ctypes.c_int
_dbl = ctypes.c_double
_flt = ctypes.c_float


def lib():
    """Load (building if needed) the C restatement."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "libct2oracle.so")
    src = os.path.join(_HERE, "ct2_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "libct2oracle.so"])
    L = ctypes.CDLL(path)
    L.ct2o_ncomp.argtypes = [_int]
    L.ct2o_ncomp.restype = _int
    L.ct2o_mi_table.argtypes = [_int, _i32p]
    L.ct2o_cell_keys.argtypes = [_u32p, _u32p, _u32p, _i64, _int, _u32p]
    L.ct2o_bin_stable.argtypes = [_u32p, _i64, _i64, _i64p, _i64p]
    L.ct2o_bin_bisect.argtypes = [_u32p, _u32p, _u32p, _i64, _int, _i64p, _i64p, _i64p]
    L.ct2o_p2m.argtypes = [_u32p, _u32p, _u32p, _i64p, _int, _int, _f64p]
    L.ct2o_greens_real.argtypes = [_int, _int, _int, _dbl, _dbl, _dbl, _f64p]
    L.ct2o_greens_kfold.argtypes = [_int, _int, _dbl, _int, _f64p]
    L.ct2o_forces.argtypes = [_u32p, _u32p, _u32p, _i64p, _int, _int, ctypes.c_void_p,
                              _int, _dbl, _dbl, _dbl, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_void_p]
    L.ct2o_kick_update.argtypes = [_f32p, _f32p, _f32p, _i8p, _f32p, _f32p, _f32p, _i64,
                                   _int, _int, _int, _int, _int, _flt, _flt, _flt, _flt, _flt]
    L.ct2o_kick_update.restype = _int
    L.ct2o_drift.argtypes = [_u32p, _u32p, _u32p, _f32p, _f32p, _f32p, _i64, _flt, _flt]
    L.ct2o_ewald_direct.argtypes = [_u32p, _u32p, _u32p, _i64, _u32p, _u32p, _u32p, _i64,
                                    _int, _dbl, _dbl, _dbl, _dbl, _int, _f64p, _f64p, _f64p,
                                    ctypes.c_void_p]
    _LIB = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


# --------------------------------------------------------------------------
# multi-indices
# --------------------------------------------------------------------------
def ncomp(p: int) -> int:
    return (p + 1) * (p + 2) * (p + 3) // 6


def mi_table(p: int) -> np.ndarray:
    t = np.zeros((ncomp(p), 3), np.int32)
    lib().ct2o_mi_table(p, t)
    return t


def mi_index(nx, ny, nz):
    d = nx + ny + nz
    return d * (d + 1) * (d + 2) // 6 + (d - nx) * (d - nx + 1) // 2 + nz


def mg2l_pairs(p: int):
    """(a, b, a+b) index triples with |a|+|b| <= p (the MG2L contraction)."""
    mi = mi_table(p)
    out = []
    for ia, a in enumerate(mi):
        for ib, b in enumerate(mi):
            if a.sum() + b.sum() <= p:
                out.append((ia, ib, mi_index(*(a + b))))
    return np.array(out, np.int64)


# --------------------------------------------------------------------------
# binning
# --------------------------------------------------------------------------
def cell_keys(x, y, z, mbits):
    k = np.empty(len(x), np.uint32)
    lib().ct2o_cell_keys(x, y, z, len(x), mbits, k)
    return k


def bin_stable(x, y, z, mbits):
    """Stable counting sort by cell (Morton order): (perm, cell_start[ncells+1])
    with cell_start indexed by the Morton key."""
    keys = cell_keys(x, y, z, mbits)
    nc = 1 << (3 * mbits)
    perm = np.empty(len(x), np.int64)
    cs = np.empty(nc + 1, np.int64)
    lib().ct2o_bin_stable(keys, len(x), nc, perm, cs)
    return perm, cs


def morton(i, j, k):
    i, j, k = (np.asarray(a, np.uint64) for a in (i, j, k))
    out = np.zeros(np.broadcast(i, j, k).shape, np.uint64)
    for b in range(10):
        out |= ((i >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + 2)
        out |= ((j >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + 1)
        out |= ((k >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b)
    return out


def cell_ranges_rowmajor(cell_start, mbits):
    """(begin, end) per row-major cell (i*M+j)*M+k from a Morton-indexed
    cell_start: the reference's cells[i][j][k] (particle.cpp:23,92)."""
    M = 1 << mbits
    i, j, k = np.meshgrid(np.arange(M), np.arange(M), np.arange(M), indexing="ij")
    key = morton(i.ravel(), j.ravel(), k.ravel()).astype(np.int64)
    return cell_start[key], cell_start[key + 1]


def bin_bisect(x, y, z, mbits):
    """Restated reference bisection: (ids order, cell_begin, cell_end)."""
    nc = 1 << (3 * mbits)
    ids = np.empty(len(x), np.int64)
    cb = np.zeros(nc, np.int64)
    ce = np.zeros(nc, np.int64)
    lib().ct2o_bin_bisect(x, y, z, len(x), mbits, ids, cb, ce)
    return ids, cb, ce


# --------------------------------------------------------------------------
# mesh stages
# --------------------------------------------------------------------------
def p2m(xs, ys, zs, cell_start, mbits, p):
    M = 1 << mbits
    out = np.empty((ncomp(p), M, M, M), np.float64)
    lib().ct2o_p2m(xs, ys, zs, cell_start, mbits, p, out)
    return out


def greens_real(mbits, p, kernel, soft, bwidth, alpha=GREENS_ALPHA):
    M = 1 << mbits
    out = np.empty((ncomp(p), M, M, M), np.float64)
    lib().ct2o_greens_real(mbits, p, kernel, soft, bwidth, alpha, out)
    return out


def greens_kfold(mbits, p, alpha=GREENS_ALPHA, kmax=GREENS_KMAX):
    M = 1 << mbits
    out = np.empty((ncomp(p), M, M, M // 2 + 1), np.float64)
    lib().ct2o_greens_kfold(mbits, p, alpha, kmax, out)
    return out


def greens_k(mbits, p, kernel, soft, bwidth, alpha=GREENS_ALPHA, kmax=GREENS_KMAX):
    """k-space Green's tensor, normalised by 1/M^3, one real number per
    component and k-point: the real part for even |n| and the imaginary part
    for odd |n| (the other part vanishes by parity)."""
    M = 1 << mbits
    gr = greens_real(mbits, p, kernel, soft, bwidth, alpha)
    gk = np.fft.rfftn(gr, axes=(1, 2, 3)) / float(M) ** 3
    deg = mi_table(p).sum(1)
    out = np.where((deg % 2 == 0)[:, None, None, None], gk.real, gk.imag)
    return out + greens_kfold(mbits, p, alpha, kmax)


def mg2l(Mk, Gk, p):
    """L_a(k) = sum_b G_{a+b}(k) M_b(k); G stored as real (even) / imag (odd)."""
    deg = mi_table(p).sum(1)
    Lk = np.zeros_like(Mk)
    for ia, ib, iab in mg2l_pairs(p):
        g = Gk[iab] if deg[iab] % 2 == 0 else 1j * Gk[iab]
        Lk[ia] += g * Mk[ib]
    return Lk


def forces(xs, ys, zs, cell_start, mbits, p, L, kernel, soft, bwidth, GM):
    """Far (L2P) and near (direct sum) accelerations, potential; sorted order."""
    n = len(xs)
    ffar = np.zeros((n, 3), np.float64)
    fnear = np.zeros((n, 3), np.float64)
    pot = np.zeros(n, np.float64)
    Lc = None if L is None else np.ascontiguousarray(L, np.float64)
    lib().ct2o_forces(xs, ys, zs, cell_start, mbits, p, _ptr(Lc), kernel, soft, bwidth, GM,
                      _ptr(ffar), _ptr(fnear), _ptr(pot))
    return ffar, fnear, pot


def method_forces(x, y, z, mbits, p, kernel, soft, bwidth, GM, Gk=None):
    """The whole force pipeline in FP64.  Returns dict with perm (sorted ->
    original index), cell_start, ffar, fnear, pot (sorted order), moments and
    expansions."""
    M = 1 << mbits
    perm, cs = bin_stable(x, y, z, mbits)
    xs, ys, zs = (np.ascontiguousarray(a[perm]) for a in (x, y, z))
    Mg = p2m(xs, ys, zs, cs, mbits, p)
    Mk = np.fft.rfftn(Mg, axes=(1, 2, 3))
    if Gk is None:
        Gk = greens_k(mbits, p, kernel, soft, bwidth)
    Lk = mg2l(Mk, Gk, p)
    L = np.fft.irfftn(Lk, s=(M, M, M), axes=(1, 2, 3)) * float(M) ** 3
    ffar, fnear, pot = forces(xs, ys, zs, cs, mbits, p, L, kernel, soft, bwidth, GM)
    return dict(perm=perm, cell_start=cs, xs=xs, ys=ys, zs=zs, moments=Mg, L=L,
                ffar=ffar, fnear=fnear, pot=pot, Gk=Gk)


# --------------------------------------------------------------------------
# kick / drift
# --------------------------------------------------------------------------
def kick_update(vx, vy, vz, rung, fx, fy, fz, *, ascending, descending, top, first, prung,
                t0, eta, max_dt, scale, hsoft):
    vx, vy, vz = (np.array(a, np.float32) for a in (vx, vy, vz))
    rung = np.array(rung, np.int8)
    fx, fy, fz = (np.ascontiguousarray(a, np.float32) for a in (fx, fy, fz))
    mr = lib().ct2o_kick_update(vx, vy, vz, rung, fx, fy, fz, len(vx), int(ascending),
                                int(descending), int(top), int(first), prung, t0, eta,
                                max_dt, scale, hsoft)
    return vx, vy, vz, rung, mr


def drift(x, y, z, vx, vy, vz, dt, scale):
    x, y, z = (np.array(a, np.uint32) for a in (x, y, z))
    vx, vy, vz = (np.ascontiguousarray(a, np.float32) for a in (vx, vy, vz))
    lib().ct2o_drift(x, y, z, vx, vy, vz, len(x), dt, scale)
    return x, y, z


# --------------------------------------------------------------------------
# FP64 Ewald direct sum (the force truth)
# --------------------------------------------------------------------------
def ewald_direct(sx, sy, sz, qx, qy, qz, kernel, soft, GM, alpha=EWALD_ALPHA,
                 rcut=EWALD_RCUT, kmax=EWALD_KMAX, with_pot=False):
    ns = len(sx)
    fx = np.empty(ns)
    fy = np.empty(ns)
    fz = np.empty(ns)
    pot = np.empty(ns) if with_pot else None
    lib().ct2o_ewald_direct(sx, sy, sz, ns, qx, qy, qz, len(qx), kernel, soft, GM, alpha,
                            rcut, kmax, fx, fy, fz, _ptr(pot))
    f = np.stack([fx, fy, fz], 1)
    return (f, pot) if with_pot else f


def force_errors(f, ftrue):
    """rms and max of |F-F_true|/|F_true|, and rms|F-F_true| / rms|F_true|."""
    d = np.linalg.norm(f - ftrue, axis=1)
    t = np.linalg.norm(ftrue, axis=1)
    rel = d / np.maximum(t, 1e-300)
    return dict(rms_rel=float(np.sqrt(np.mean(rel ** 2))), max_rel=float(rel.max()),
                rms_norm=float(np.sqrt(np.mean(d ** 2)) / np.sqrt(np.mean(t ** 2))))


# --------------------------------------------------------------------------
# The reference's own 1D FFT (oracle/_ref, compiled from the reference's
# src/fft/{fft_real_scalar,fft_complex_vector,twiddles,scramble}.cpp)
# --------------------------------------------------------------------------
_REF = None


def ref_fft_lib():
    """The compiled reference FFT, or None when oracle/_ref was not built
    (it is built from the reference tree, which only the build host has)."""
    global _REF
    if _REF is not None:
        return _REF
    path = os.path.join(_HERE, "_ref", "libct2ref_fft.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    L.ref_fft_real.argtypes = [_f64p, _int, _int]
    L.ref_scramble.argtypes = [_f64p, _int, _int, _int]
    L.ref_fft_complex4.argtypes = [_f64p, _int, _int]
    L.ref_fft_real4.argtypes = [_f64p, _int, _int]
    L.ref_transpose_yz.argtypes = [_f64p, _int]
    L.ref_transpose_r2c.argtypes = [_f64p, _f64p, _int]
    L.ref_transpose_c2r.argtypes = [_f64p, _f64p, _int]
    L.ref_twiddles.argtypes = [_int, _int, _f64p]
    _REF = L
    return L


def ref_fft_real(x):
    """Reference fft_real on a copy of x (scrambled first, as fft_test.cpp
    does): returns the halfcomplex result X[k]=Re, X[N-k]=Im."""
    L = ref_fft_lib()
    X = np.array(x, np.float64)
    L.ref_scramble(X, 1, len(X), 1)
    L.ref_fft_real(X, len(X), 1)
    return X


def ref_fft_complex(z):
    """Reference fft_complex (lane 0 of its 4-lane SIMD form) on complex z."""
    L = ref_fft_lib()
    N = len(z)
    X = np.zeros((N, 8), np.float64)
    X[:, 0:4] = np.real(z)[:, None]
    X[:, 4:8] = np.imag(z)[:, None]
    X = np.ascontiguousarray(X.reshape(-1))
    L.ref_scramble(X, 1, N, 8)
    L.ref_fft_complex4(X, N, 1)
    X = X.reshape(N, 8)
    return X[:, 0] + 1j * X[:, 4]


def halfcomplex_to_complex(X):
    """halfcomplex [X0, Re1.., Re(N/2), Im(N/2-1)..Im1] -> N/2+1 complex."""
    N = len(X)
    out = np.zeros(N // 2 + 1, np.complex128)
    out.real[: N // 2 + 1] = X[: N // 2 + 1]
    k = np.arange(1, N // 2)
    out.imag[k] = X[N - k]
    return out


# --------------------------------------------------------------------------
# Cloud-in-cell deposit (no counterpart in the reference; the published CIC
# scheme, as ct2g_cic_deposit states it): four grids, the CIC mass and the
# first moments about each mesh point, in FP64
# --------------------------------------------------------------------------
def cic_deposit(x, y, z, N):
    pos = np.stack([x, y, z], 1).astype(np.float64) * 2.0 ** -32
    u = pos * N - 0.5
    m = np.floor(u).astype(np.int64)
    f = u - m
    out = np.zeros((4, N, N, N), np.float64)
    for corner in range(8):
        b = np.array([(corner >> 2) & 1, (corner >> 1) & 1, corner & 1])
        w = np.prod(np.where(b[None, :] == 1, f, 1.0 - f), axis=1)
        s = np.where(b[None, :] == 1, f - 1.0, f)
        idx = (m + b[None, :]) & (N - 1)
        flat = (idx[:, 0] * N + idx[:, 1]) * N + idx[:, 2]
        np.add.at(out[0].reshape(-1), flat, w)
        for d in range(3):
            np.add.at(out[1 + d].reshape(-1), flat, w * s[:, d])
    return out
