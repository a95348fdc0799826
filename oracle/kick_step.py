"""CPU restatement of the reference's rung-hierarchical step -- TEST
INFRASTRUCTURE ONLY (tests/ and the bench's CPU legs; the product never
imports it).

Restates, over a numpy particle store:
  kick_step                 src/main.cpp:8-92 (level list, clip_top rule,
                            push/pop order, kick parameters, drift per level)
  particle_sort_by_rung     src/particle.cpp:320-340
  particle_push/pop_rungs   src/particle.cpp:31-38
  particle_set_minrung      src/particle.cpp:342-347
  particle_rung_counts      src/particle.cpp:40-50
  particle_current_range    src/particle.cpp:52-57

The store's order follows the GPU's conventions, which the reference leaves
open: the rung partition is stable (the reference's Hoare-style partition
leaves the order inside each side arbitrary) and binning is the stable Morton
sort of oracle.bin_stable.  Per-particle results do not depend on these
orders; the level bookkeeping, ranges and parameters are checked against the
reference's own kick_step (compiled from its source into oracle/_ref) in
tests/test_ref_pinned.py.

kick(), drift() and particle_to_grid() are passed in as callables, so the
same driver runs with the oracle's forces, an analytic force field, or forces
computed elsewhere.
"""
from __future__ import annotations

import numpy as np

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "rung", "id")


class Store:
    """The reference's process-global particle arrays (src/particle.cpp:17-25)
    plus the current-range bookkeeping."""

    def __init__(self, x, y, z, vx, vy, vz, rung=None, ids=None):
        n = len(x)
        self.x = np.array(x, np.uint32)
        self.y = np.array(y, np.uint32)
        self.z = np.array(z, np.uint32)
        self.vx = np.array(vx, np.float32)
        self.vy = np.array(vy, np.float32)
        self.vz = np.array(vz, np.float32)
        self.rung = np.zeros(n, np.int8) if rung is None else np.array(rung, np.int8)
        self.id = np.arange(n, dtype=np.uint32) if ids is None else np.array(ids, np.uint32)
        self.rung_begin = 0
        self.stack = []

    @property
    def n(self):
        return len(self.x)

    def permute_range(self, b, perm):
        """Reorder [b, n) by perm (indices relative to b)."""
        for f in FIELDS:
            a = getattr(self, f)
            a[b:] = a[b:][perm]

    # particle.cpp:52-57
    def current_range(self):
        return self.rung_begin, self.n

    # particle.cpp:31-38
    def push_rungs(self):
        self.stack.append(self.rung_begin)

    def pop_rungs(self):
        self.rung_begin = self.stack.pop()

    # particle.cpp:320-340: [rung_begin, n) split so that rungs >= minrung
    # come last; rung_begin moves to the first of them.  minrung 0 resets the
    # range to the whole store.
    def sort_by_rung(self, minrung):
        if minrung == 0:
            self.rung_begin = 0
            return
        b = self.rung_begin
        r = self.rung[b:]
        low = np.flatnonzero(r < minrung)
        high = np.flatnonzero(r >= minrung)
        self.permute_range(b, np.concatenate([low, high]))
        self.rung_begin = b + len(low)

    # particle.cpp:342-347
    def set_minrung(self, minrung):
        np.maximum(self.rung, np.int8(minrung), out=self.rung)

    # particle.cpp:40-50: counts[r] for r up to the highest rung present
    def rung_counts(self):
        if self.n == 0:
            return []
        return list(np.bincount(self.rung.astype(np.int64), minlength=0))

    def arrays(self):
        return {f: getattr(self, f).copy() for f in FIELDS}


def kick_params(*, ascending, descending, top, first, rung, t0, eta, max_dt, scale):
    """kick_params (cosmictiger/kick.hpp:10-20); the float fields carry the
    float32 values the reference stores."""
    return dict(ascending=bool(ascending), descending=bool(descending), top=bool(top),
                first=bool(first), rung=int(rung), t0=float(np.float32(t0)),
                eta=float(np.float32(eta)), max_dt=float(np.float32(max_dt)),
                scale=float(np.float32(scale)))


def kick_step(store, minrung, max_rung, scale, adot, tau, t0, minrung0, nocrop, *, eta,
              to_grid, kick, drift, trace=None):
    """src/main.cpp:8-92.  Returns (minrung, value, last_kick_max):
    minrung as updated through the reference's reference argument, the value
    the reference returns (its max_rung argument: the max_rung the loop body
    declares at main.cpp:68 shadows it and goes out of scope before the return
    at :90) and the value the last kick() returned.

    to_grid(store): bin the current range.  kick(store, params) -> int: kick
    the current range.  drift(store, dt, scale): drift every particle.  trace
    (a list, optional) receives ("kick", params, begin, end) and
    ("drift", dt, scale) events in call order."""
    levels = [0] * (max(max_rung - minrung, 0) + 1)
    k = 0
    for i in range(max_rung, minrung, -1):
        levels[k] = i
        k += 1
    levels[k] = minrung
    ascending = True
    clip_top = False
    top = False
    mr = 0
    li = 0
    while li < len(levels):
        if levels[li] == minrung:
            ascending = False
            top = True
        else:
            top = False
        if not ascending and not top:
            store.push_rungs()
        if not ascending:
            store.sort_by_rung(levels[li])
        if top and minrung == minrung0:
            counts = store.rung_counts()
            if len(counts) > minrung0 + 1:
                fast = int(sum(counts[minrung0 + 1:]))
                slow = int(counts[minrung0])
                if 3 * fast > slow:
                    clip_top = not nocrop
        to_grid(store)
        p = kick_params(
            top=True if (clip_top and levels[li] == minrung0 + 1) else top,
            ascending=ascending or top,
            descending=False if (clip_top and top) else ((not ascending) or top),
            eta=eta, scale=scale, first=(tau == 0.0), rung=levels[li], t0=t0,
            # 0.01f / adot: the float literal promoted to double, stored as float
            max_dt=np.float64(np.float32(0.01)) / np.float64(adot))
        b, e = store.current_range()
        if trace is not None:
            trace.append(("kick", p, b, e))
        mr = int(kick(store, p))
        if clip_top and top:
            store.set_minrung(minrung0 + 1)
        if clip_top and top:
            levels.append(minrung0 + 1)
        elif (not ascending) or top:
            if mr > levels[li]:
                levels.append(levels[li] + 1)
        if ((not ascending) or top) and not (clip_top and top):
            dt = float(np.float32(t0 / float(1 << levels[li])))
            if trace is not None:
                trace.append(("drift", dt, float(np.float32(scale))))
            drift(store, dt, float(np.float32(scale)))
        if ascending and not top:
            store.pop_rungs()
        li += 1
    if clip_top:
        minrung += 1
    return minrung, max_rung, mr


# --------------------------------------------------------------------------
# stage callables built from the oracle's own restatements
# --------------------------------------------------------------------------
def oracle_to_grid(mbits):
    """Binning of the current range by the oracle's stable Morton sort."""
    from oracle import oracle as O

    def to_grid(store):
        b = store.rung_begin
        if store.n - b == 0:
            return
        perm, _ = O.bin_stable(np.ascontiguousarray(store.x[b:]),
                               np.ascontiguousarray(store.y[b:]),
                               np.ascontiguousarray(store.z[b:]), mbits)
        store.permute_range(b, perm)
    return to_grid


def kick_with_forces(force_fn, hsoft):
    """kick(): forces of the current range from force_fn(store, b) (float32
    [n-b, 3] in store order), then the restated velocity + rung update
    (kick.cpp:75-99) on that range."""
    from oracle import oracle as O

    def kick(store, p):
        b = store.rung_begin
        if store.n - b == 0:
            return 0
        f = np.asarray(force_fn(store, b), np.float32)
        vx, vy, vz, rung, mr = O.kick_update(
            store.vx[b:], store.vy[b:], store.vz[b:], store.rung[b:], f[:, 0], f[:, 1], f[:, 2],
            ascending=p["ascending"], descending=p["descending"], top=p["top"],
            first=p["first"], prung=p["rung"], t0=p["t0"], eta=p["eta"], max_dt=p["max_dt"],
            scale=p["scale"], hsoft=hsoft)
        store.vx[b:], store.vy[b:], store.vz[b:], store.rung[b:] = vx, vy, vz, rung
        return mr
    return kick


def oracle_drift(store, dt, scale):
    """drift (drift.cpp:4-18) of every particle."""
    from oracle import oracle as O
    store.x, store.y, store.z = O.drift(store.x, store.y, store.z, store.vx, store.vy,
                                        store.vz, dt, scale)


def analytic_forces(amp=(3.0, 40.0, 900.0)):
    """A smooth force field of the particle's own position only (so its
    values do not depend on the store's order): components
    -A_d sin(2 pi k_d x_d) with a few wavenumbers, spanning several rungs."""
    amp = np.asarray(amp, np.float64)

    def fn(store, b):
        x = np.stack([store.x[b:], store.y[b:], store.z[b:]], 1).astype(np.float64) * 2.0 ** -32
        k = np.array([1.0, 3.0, 7.0])
        f = -(amp[None, :] * np.sin(2.0 * np.pi * k[None, :] * x)
              * (1.0 + 0.5 * np.cos(2.0 * np.pi * x[:, ::-1])))
        return f.astype(np.float32)
    return fn
