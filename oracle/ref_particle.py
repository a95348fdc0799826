"""The reference's own particle store, binning, rung bookkeeping, step driver
and cosmology, compiled from its sources into oracle/_ref/libct2ref_particle.so
by `make -C oracle ref` -- TEST INFRASTRUCTURE ONLY.

The library exists only where the reference tree was present at build time;
every loader here returns None otherwise and the tests that need it skip.
Committed golden fixtures (tests/golden/) carry its outputs to machines
without it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from oracle import kick_step as KS

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
_szp = ctypes.POINTER(ctypes.c_size_t)
_dp = ctypes.POINTER(ctypes.c_double)

KICK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                           ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                           ctypes.c_float, ctypes.c_size_t, ctypes.c_size_t)
DRIFT_FN = ctypes.CFUNCTYPE(None, ctypes.c_float, ctypes.c_float)


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "_ref", "libct2ref_particle.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    L.ref_set_options.argtypes = [ctypes.c_float, ctypes.c_int, ctypes.c_size_t, ctypes.c_float,
                                  ctypes.c_float]
    L.ref_set_cosmology.argtypes = [ctypes.c_float] * 5
    L.ref_set_store.argtypes = [_u32p, _u32p, _u32p, _f32p, _f32p, _f32p, _i8p, ctypes.c_size_t]
    L.ref_set_arrays.argtypes = L.ref_set_store.argtypes
    L.ref_stack_depth.restype = ctypes.c_size_t
    L.ref_particle_to_grid.restype = ctypes.c_int
    L.ref_sort_by_rung.argtypes = [ctypes.c_int]
    L.ref_set_minrung.argtypes = [ctypes.c_int]
    L.ref_current_range.argtypes = [_szp, _szp]
    L.ref_rung_counts.argtypes = [_szp, ctypes.c_int]
    L.ref_rung_counts.restype = ctypes.c_int
    L.ref_kick_step.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_double,
                                ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                ctypes.c_int, KICK_FN, DRIFT_FN]
    L.ref_kick_step.restype = ctypes.c_int
    L.ref_cosmos_dadt.argtypes = [ctypes.c_double]
    L.ref_cosmos_dadt.restype = ctypes.c_double
    L.ref_cosmos_time.argtypes = [ctypes.c_double, ctypes.c_double]
    L.ref_cosmos_time.restype = ctypes.c_double
    L.ref_cosmos_conformal_time.argtypes = [ctypes.c_double, ctypes.c_double]
    L.ref_cosmos_conformal_time.restype = ctypes.c_double
    L.ref_cosmos_update.argtypes = [_dp, _dp, _dp, ctypes.c_double]
    _LIB = L
    return L


class RefStore(KS.Store):
    """A Store whose arrays the reference's code works on in place."""

    def attach(self):
        L = lib()
        L.ref_set_arrays(self.x, self.y, self.z, self.vx, self.vy, self.vz, self.rung, self.n)


def reset(store):
    """Start a sequence of reference kick_step calls on `store`: its arrays
    become the reference's store, with range [0, n) and an empty rung stack
    (the stack then carries over from call to call, as in the reference)."""
    lib().ref_set_store(store.x, store.y, store.z, store.vx, store.vy, store.vz, store.rung,
                        store.n)


def stack_depth():
    return int(lib().ref_stack_depth())


def particle_to_grid(x, y, z, ppcell, vx=None):
    """The reference's particle_to_grid() (particle.cpp:349-362, bisection of
    :69-114) on copies of the arrays.  vx (optional, float32) rides along with
    the particles, so an id stored in it shows the permutation.  Returns
    (x, y, z, vx, Ncell)."""
    L = lib()
    n = len(x)
    s = KS.Store(x, y, z, np.zeros(n, np.float32) if vx is None else vx,
                 np.zeros(n, np.float32), np.zeros(n, np.float32))
    L.ref_set_options(0.15, int(ppcell), 32, 3.0, 0.02)
    L.ref_set_store(s.x, s.y, s.z, s.vx, s.vy, s.vz, s.rung, n)
    nc = L.ref_particle_to_grid()
    return s.x, s.y, s.z, s.vx, nc


def kick_step(store, minrung, max_rung, scale, adot, tau, t0, minrung0, nocrop, *, eta,
              kick, drift, trace=None):
    """The reference's kick_step (main.cpp:8-92) over `store`'s arrays, with
    its own particle_to_grid, rung sort, push/pop and set_minrung.  kick and
    drift are the same callables oracle.kick_step.kick_step takes; the store
    must have been given to reset() before the first call of a sequence and
    keep its arrays (they are updated in place).  ppcell is
    set above any range size, so the reference's Ncell = cbrt(count/ppcell)+4
    (particle.cpp:355) is 4 at every level.  Returns (minrung, value)."""
    L = lib()
    L.ref_set_options(float(eta), 1 << 30, 32, 3.0, 0.02)
    rs = RefStore.__new__(RefStore)
    rs.__dict__.update(store.__dict__)
    rs.attach()

    def _kick(asc, desc, top, first, rung, t0_, eta_, max_dt, scale_, b, e):
        p = KS.kick_params(ascending=asc, descending=desc, top=top, first=first, rung=rung,
                           t0=t0_, eta=eta_, max_dt=max_dt, scale=scale_)
        rs.rung_begin = b
        if trace is not None:
            trace.append(("kick", p, b, e))
        return int(kick(rs, p))

    def _drift(dt, scale_):
        if trace is not None:
            trace.append(("drift", float(np.float32(dt)), float(np.float32(scale_))))
        x, y, z = rs.x.copy(), rs.y.copy(), rs.z.copy()
        tmp = KS.Store(x, y, z, rs.vx, rs.vy, rs.vz, rs.rung)
        drift(tmp, dt, scale_)
        rs.x[:], rs.y[:], rs.z[:] = tmp.x, tmp.y, tmp.z

    kf, df = KICK_FN(_kick), DRIFT_FN(_drift)
    mr = ctypes.c_int(minrung)
    val = L.ref_kick_step(ctypes.byref(mr), max_rung, scale, adot, tau, t0, minrung0,
                          1 if nocrop else 0, kf, df)
    return mr.value, val


def cosmology(omega_m, omega_r, omega_lam, hubble, code_to_s):
    """Set the options the reference's cosmology reads; returns the library."""
    L = lib()
    L.ref_set_cosmology(omega_m, omega_r, omega_lam, hubble, code_to_s)
    return L
