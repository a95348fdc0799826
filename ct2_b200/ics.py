"""Seeded synthetic particle sets for the gravity-step workloads.

The reference initialises particles with libc rand() (src/particle.cpp:364-374,
src/util.cpp:3-5); the workloads here use numpy PCG64 generators instead so
that every run, test and benchmark sees the same particles.

Positions are returned as 32-bit fixed point (x * 2^32, periodic unit box),
the reference's pos_fixed SoA (cosmictiger/cosmictiger.hpp:22); velocities as
float32; rungs as int8.  All particles have equal mass 1/N (GM = 1/N with
G = 1), as in the reference's options (src/options.cpp:88).
"""
from __future__ import annotations

import numpy as np


def to_fixed32(pos: np.ndarray) -> np.ndarray:
    """Periodic positions in box units -> fixed32, going through float32 as the
    reference's FP32 particle inputs do."""
    p = np.mod(pos, 1.0).astype(np.float32).astype(np.float64)
    u = np.floor(p * 4294967296.0).astype(np.uint64) & np.uint64(0xFFFFFFFF)
    return u.astype(np.uint32)


def _pack(pos, n):
    x = to_fixed32(pos[:, 0])
    y = to_fixed32(pos[:, 1])
    z = to_fixed32(pos[:, 2])
    v = np.zeros(n, np.float32)
    return dict(x=x, y=y, z=z, vx=v.copy(), vy=v.copy(), vz=v.copy(),
                rung=np.zeros(n, np.int8))


def lattice(ngrid: int, seed: int = 0, sigma_cells: float = 0.1):
    """ngrid^3 particles on the lattice (i+1/2)/ngrid displaced by Gaussian
    noise of sigma_cells lattice spacings per coordinate, wrapped."""
    rng = np.random.Generator(np.random.PCG64(seed))
    i = (np.arange(ngrid) + 0.5) / ngrid
    g = np.stack(np.meshgrid(i, i, i, indexing="ij"), -1).reshape(-1, 3)
    g = g + rng.normal(0.0, sigma_cells / ngrid, size=g.shape)
    return _pack(g, len(g))


def _plummer_radii(rng, n, a, rmax_over_a=20.0):
    umax = rmax_over_a ** 3 / (1.0 + rmax_over_a ** 2) ** 1.5
    u = rng.uniform(0.0, umax, n)
    u = np.maximum(u, 1e-300)
    return a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)


def _unit_vectors(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _split_counts(weights, total):
    w = np.asarray(weights, np.float64)
    raw = w / w.sum() * total
    cnt = np.floor(raw).astype(np.int64)
    rem = total - cnt.sum()
    cnt[np.argsort(-(raw - cnt), kind="stable")[:rem]] += 1
    return cnt


def plummer_spheres(n: int, seed: int = 0, nspheres: int = 512, a: float = 0.005,
                    frac_clustered: float = 0.7, mass_range: float = 10.0):
    """n particles: frac_clustered of them in nspheres Plummer spheres (scale
    radius a, centres uniform, sphere masses log-uniform over [1, mass_range],
    radii from the Plummer CDF truncated at 20a), the rest uniform.  Equal
    particle masses, so a sphere's mass sets its particle count."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n_cl = int(round(frac_clustered * n))
    masses = mass_range ** rng.uniform(0.0, 1.0, nspheres)
    counts = _split_counts(masses, n_cl)
    centres = rng.uniform(0.0, 1.0, (nspheres, 3))
    parts = []
    for s in range(nspheres):
        r = _plummer_radii(rng, counts[s], a)
        parts.append(centres[s] + r[:, None] * _unit_vectors(rng, counts[s]))
    parts.append(rng.uniform(0.0, 1.0, (n - n_cl, 3)))
    pos = np.concatenate(parts, 0)
    pos = pos[rng.permutation(n)]
    return _pack(pos, n)


def nfw_halos(n: int, seed: int = 0, nhalos: int = 2000, c_range=(5.0, 15.0),
              slope: float = 1.9, decades: float = 2.0, rvir_max: float = 0.02):
    """n particles in nhalos NFW halos: concentration c ~ U(c_range), halo
    masses from dN/dM ~ M^-slope over `decades` decades, r_vir ~ M^(1/3) with
    the heaviest at rvir_max; radii by numerically inverting the NFW enclosed
    mass m(x) = ln(1+x) - x/(1+x) up to x = c."""
    rng = np.random.Generator(np.random.PCG64(seed))
    # inverse-CDF sampling of the power-law mass function over [1, 10^decades]
    u = rng.uniform(0.0, 1.0, nhalos)
    lo, hi = 1.0, 10.0 ** decades
    e = 1.0 - slope
    masses = (lo ** e + u * (hi ** e - lo ** e)) ** (1.0 / e)
    counts = _split_counts(masses, n)
    rvir = rvir_max * (masses / masses.max()) ** (1.0 / 3.0)
    conc = rng.uniform(c_range[0], c_range[1], nhalos)
    centres = rng.uniform(0.0, 1.0, (nhalos, 3))
    xs = np.linspace(0.0, 1.0, 4097)
    parts = []
    for h in range(nhalos):
        c = conc[h]
        xg = xs * c
        mg = np.log1p(xg) - xg / (1.0 + xg)
        q = rng.uniform(0.0, mg[-1], counts[h])
        x = np.interp(q, mg, xg)
        r = x / c * rvir[h]
        parts.append(centres[h] + r[:, None] * _unit_vectors(rng, counts[h]))
    pos = np.concatenate(parts, 0)
    pos = pos[rng.permutation(n)]
    return _pack(pos, n)


def batch_boxes(nboxes: int = 96, seed: int = 0, log2_min: float = 12.0,
                log2_max: float = 21.0, mesh_min: int = 32, mesh_max: int = 256):
    """Independent periodic boxes: N_b = round(2^U[log2_min, log2_max]) with the
    Plummer + background generator seeded seed+b; mesh = the power of two
    nearest to 2 N_b^(1/3), clipped to [mesh_min, mesh_max]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for b in range(nboxes):
        nb = int(round(2.0 ** rng.uniform(log2_min, log2_max)))
        mesh = int(2 ** round(np.log2(2.0 * nb ** (1.0 / 3.0))))
        mesh = int(min(max(mesh, mesh_min), mesh_max))
        box = plummer_spheres(nb, seed=seed + b, nspheres=max(1, int(round(512 * nb / 2 ** 21))))
        box["mesh"] = mesh
        out.append(box)
    return out


SOA_MAGIC = b"CT2SOA1\x00"


def save_soa(path, d):
    """Write particles as the raw SoA file the C++ layer's particles_save /
    particles_load use: magic, uint64 count, x y z (uint32), vx vy vz
    (float32), rung (int8)."""
    n = len(d["x"])
    with open(path, "wb") as f:
        f.write(SOA_MAGIC)
        f.write(np.uint64(n).tobytes())
        for k, t in (("x", np.uint32), ("y", np.uint32), ("z", np.uint32), ("vx", np.float32),
                     ("vy", np.float32), ("vz", np.float32)):
            f.write(np.ascontiguousarray(d[k], t).tobytes())
        f.write(np.ascontiguousarray(d.get("rung", np.zeros(n, np.int8)), np.int8).tobytes())


def load_soa(path):
    with open(path, "rb") as f:
        if f.read(8) != SOA_MAGIC:
            raise ValueError("not a particle file: %s" % path)
        n = int(np.frombuffer(f.read(8), np.uint64)[0])
        out = {}
        for k, t in (("x", np.uint32), ("y", np.uint32), ("z", np.uint32), ("vx", np.float32),
                     ("vy", np.float32), ("vz", np.float32), ("rung", np.int8)):
            b = f.read(n * np.dtype(t).itemsize)
            if len(b) != n * np.dtype(t).itemsize:
                raise ValueError("file too short: %s" % path)
            out[k] = np.frombuffer(b, t).copy()
    return out
