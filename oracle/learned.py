"""CPU restatement of the learned near-field correction -- TEST INFRASTRUCTURE ONLY.

Only tests/ may import this module, as the checker.  The reference
(dmarce1/ct2) has no learned part, so there is nothing of it to pin against:
this file restates, in FP64 numpy, the definitions the library implements --

  * the shell of a cell: offsets bwidth^2 < |o|^2 <= bwidth_ext^2 in the loop
    order i, j, k = -B..B, stably sorted by |o|^2, cut into three distance
    bins of equal size;
  * the 24 per-cell features and the fixed criterion's score, from the cell
    ranges, the moment grid and the plain forces;
  * the MLP 24 -> 64 -> 64 -> 1 (ReLU) on BF16-rounded weights, its mean
    squared error and the gradient of that error (what the training kernels
    compute).

The correction itself is checked against the wider-stencil method of
oracle.method_forces (bwidth_ext), which it must reproduce.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O

NIN, NH = 24, 64
OW1 = 0
OB1 = OW1 + NH * NIN
OW2 = OB1 + NH
OB2 = OW2 + NH * NH
OW3 = OB2 + NH
OB3 = OW3 + NH
NP = OB3 + 1


def bf16_round(a):
    """float32 -> nearest bfloat16 (ties to even) -> float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def unpack(params):
    w = np.asarray(params, np.float64)
    return (w[OW1:OB1].reshape(NH, NIN), w[OB1:OW2], w[OW2:OB2].reshape(NH, NH), w[OB2:OW3],
            w[OW3:OB3], w[OB3])


def mlp_forward(params, fmean, fstd, X):
    W1, b1, W2, b2, W3, b3 = unpack(bf16_round(params))
    x = (np.asarray(X, np.float64) - np.asarray(fmean, np.float64)) / np.asarray(fstd, np.float64)
    h1 = np.maximum(x @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ W3 + b3


def mlp_loss_grad(params, fmean, fstd, X, T):
    """Mean squared error of the prediction and its gradient with respect to
    the (BF16-rounded) parameters, FP64."""
    W1, b1, W2, b2, W3, b3 = unpack(bf16_round(params))
    x = (np.asarray(X, np.float64) - np.asarray(fmean, np.float64)) / np.asarray(fstd, np.float64)
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    y = h2 @ W3 + b3
    e = y - np.asarray(T, np.float64)
    n = len(e)
    dy = 2.0 * e / n
    dz2 = dy[:, None] * W3[None, :] * (z2 > 0)
    dz1 = (dz2 @ W2) * (z1 > 0)
    g = np.concatenate([(dz1.T @ x).ravel(), dz1.sum(0), (dz2.T @ h1).ravel(), dz2.sum(0),
                        h2.T @ dy, [dy.sum()]])
    return float(np.mean(e ** 2)), g


def morton_decode(keys):
    """Morton key -> (i, j, k), the inverse of oracle.morton (x bits highest)."""
    keys = np.asarray(keys, np.uint64)
    out = np.zeros((len(keys), 3), np.int64)
    for b in range(10):
        for d in range(3):
            out[:, d] |= (((keys >> np.uint64(3 * b + 2 - d)) & np.uint64(1)).astype(np.int64)) << b
    return out


def shell_offsets(bwidth, bwidth_ext):
    B = int(np.floor(bwidth_ext))
    b2, x2 = float(bwidth) ** 2, float(bwidth_ext) ** 2
    offs = [(i, j, k) for i in range(-B, B + 1) for j in range(-B, B + 1) for k in range(-B, B + 1)
            if b2 < i * i + j * j + k * k <= x2]
    offs.sort(key=lambda o: o[0] ** 2 + o[1] ** 2 + o[2] ** 2)
    ns = len(offs)
    bins = [min(2, 3 * s // max(ns, 1)) for s in range(ns)]
    return np.array(offs, np.int64).reshape(-1, 3), np.array(bins, np.int64)


def features(cells, cell_start, moments, f, box_off, box_gm, mbits, p, bwidth, bwidth_ext):
    """24 features and the fixed-criterion score per occupied cell.

    cells: Morton keys (box above the key); cell_start: Morton-indexed
    absolute ranges [nbox*C + 1]; moments: [nc, nbox*C] row-major per box
    (unit mass); f: [n, 3] plain forces in cell order."""
    M = 1 << mbits
    C = M ** 3
    h = 1.0 / M
    cells = np.asarray(cells, np.int64)
    cs = np.asarray(cell_start, np.int64)
    Mg = np.asarray(moments, np.float64)
    i200, i020, i002 = O.mi_index(2, 0, 0), O.mi_index(0, 2, 0), O.mi_index(0, 0, 2)
    i100, i010, i001 = O.mi_index(1, 0, 0), O.mi_index(0, 1, 0), O.mi_index(0, 0, 1)
    box = cells >> (3 * mbits)
    m = cells & (C - 1)
    ijk = morton_decode(m)
    c0, c1 = cs[cells], cs[cells + 1]
    nc = (c1 - c0).astype(np.float64)
    fn = np.linalg.norm(np.asarray(f, np.float64), axis=1)
    s1 = np.add.reduceat(fn, c0) if len(c0) else np.zeros(0)
    s2 = np.add.reduceat(fn ** 2, c0) if len(c0) else np.zeros(0)
    # reduceat over consecutive occupied cells (cells are in key order and
    # every particle of the range belongs to one of them)
    fmean = np.maximum(s1 / nc, 1e-30)
    fstd = np.sqrt(np.maximum(s2 / nc - fmean ** 2, 0.0))
    GM = np.asarray(box_gm, np.float64)[box]
    bo = np.asarray(box_off, np.float64)
    nbox = bo[box + 1] - bo[box]

    def rowmajor(b, i, j, k):
        return b * C + ((i % M) * M + (j % M)) * M + (k % M)

    rc = rowmajor(box, ijk[:, 0], ijk[:, 1], ijk[:, 2])
    sig_c = np.sqrt(np.maximum(2.0 * (Mg[i200, rc] + Mg[i020, rc] + Mg[i002, rc]) / nc, 0.0))
    dip = np.sqrt(Mg[i100, rc] ** 2 + Mg[i010, rc] ** 2 + Mg[i001, rc] ** 2) / nc
    offs, bins = shell_offsets(bwidth, bwidth_ext)
    ncell = len(cells)
    cntb = np.zeros((3, ncell))
    mono = np.zeros((3, ncell))
    quad = np.zeros((3, ncell))
    trunc = np.zeros((3, ncell))
    monop = np.zeros(ncell)
    maxn = np.zeros(ncell)
    pull = np.zeros((3, ncell))
    for (ox, oy, oz), b in zip(offs, bins):
        ii, jj, kk = (ijk[:, 0] + ox) % M, (ijk[:, 1] + oy) % M, (ijk[:, 2] + oz) % M
        k2 = (box << (3 * mbits)) | O.morton(ii, jj, kk).astype(np.int64)
        ns = (cs[k2 + 1] - cs[k2]).astype(np.float64)
        on = ns > 0
        r2c = rowmajor(box, ii, jj, kk)
        sig2 = np.where(on, np.maximum(2.0 * (Mg[i200, r2c] + Mg[i020, r2c] + Mg[i002, r2c])
                                       / np.where(on, ns, 1.0), 0.0), 0.0)
        R2 = float(ox * ox + oy * oy + oz * oz) * h * h
        R = np.sqrt(R2)
        mm = ns / R2
        cntb[b] += ns
        mono[b] += mm
        quad[b] += mm * sig2 / R2
        trunc[b] += mm * (np.sqrt(sig2) / R) ** (p + 1)
        monop += ns / R2 / R ** (p + 1)
        maxn = np.maximum(maxn, ns)
        w = mm * h / R
        pull += w[None, :] * np.array([ox, oy, oz], np.float64)[:, None]
    inv = GM / fmean
    mono_all = mono.sum(0)
    cnt_all = cntb.sum(0)
    X = np.zeros((ncell, NIN))
    X[:, 0] = np.log2(1 + nc)
    X[:, 1] = np.log10(fmean / (GM * nbox * M * M) + 1e-30)
    X[:, 2] = fstd / fmean
    X[:, 3] = sig_c / h
    X[:, 4] = dip / h
    for b in range(3):
        X[:, 5 + b] = np.log2(1 + cntb[b])
        X[:, 8 + b] = np.log10(inv * mono[b] + 1e-12)
        X[:, 11 + b] = np.log10(inv * quad[b] + 1e-14)
        X[:, 14 + b] = np.log10(inv * trunc[b] + 1e-16)
    X[:, 17] = np.log10(inv * sig_c ** (p + 1) * monop + 1e-16)
    X[:, 18] = np.log2(1 + maxn)
    X[:, 19] = np.where(mono_all > 0, np.minimum(np.linalg.norm(pull, axis=0)
                                                 / np.where(mono_all > 0, mono_all, 1.0), 1.0), 0.0)
    X[:, 20] = np.log10(inv * mono_all + 1e-12)
    X[:, 21] = mbits / 10.0
    X[:, 22] = (c1 - c0 == 1).astype(np.float64)
    X[:, 23] = cntb[0] / (cnt_all + 1)
    return X, inv * mono_all
