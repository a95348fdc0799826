"""The recorded-graph step, box contexts, batches and launch-shape tuning.

All of these reorganise the same arithmetic, so their results must be
bit-identical to the eager single-box path on the same particles:
  * a replayed graph runs the same kernels as the eager call;
  * a box context sorts each box's particles exactly as a one-box context
    does (the box index sits above the Morton key of a stable sort), runs the
    same per-grid FFT and the same per-sink near-field sequence;
  * FFT tile widths, the y and x passes' transport (TMA or per-thread
    copies), where the cells' moments are summed (a cell-parallel pass into
    compact records, or inside the z pass) and the near-field grid size
    change which block does the work, not its arithmetic.  The sink chunking (dense_cell) moves a sink
    between the dense path (sources shifted into the sink cell's frame) and
    the sparse path (the sink shifted into each source cell's frame), and
    the streamed sparse path (sparse_path 2) evaluates its sinks and sources
    in the chunk block's frame: the same sums with different FP32 rounding,
    checked to 1e-5 relative, with the same interaction count.
"""
import numpy as np
import pytest

from ct2_b200 import ics
from ct2_b200.gravity import Batch, Gravity, kick_params

pytestmark = pytest.mark.gpu

KP = kick_params(ascending=True, descending=True, top=True, first=False, rung=0, t0=1e-3,
                 eta=0.15, max_dt=0.01, scale=1.0)
DT = 1e-3


def _box(n, seed, mesh):
    return ics.plummer_spheres(n, seed=seed, nspheres=max(1, n // 4000), a=2.0 / mesh)


def _state(g):
    d = g.download()
    o = np.argsort(d["id"], kind="stable")
    return {k: d[k][o] for k in ("x", "y", "z", "vx", "vy", "vz", "rung")}


def _same(a, b):
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def _mk(mesh, nbox=1, order=3, bw=2.0):
    return Gravity(mesh=mesh, order=order, bwidth=bw, hsoft=1.0 / (25 * mesh), nbox=nbox)


def test_graph_step_matches_eager(gpu):
    P = _box(30000, 3, 64)
    a, b = _mk(64), _mk(64)
    a.upload_dict(P)
    b.upload_dict(P)
    for step in range(3):
        ra = a.kick_drift(KP, DT, graph=False)
        rb = b.kick_drift(KP, DT, graph=True)
        assert ra == rb
        _same(_state(a), _state(b))
    # a parameter change records the graph again
    kp2 = kick_params(**{**KP.__dict__, "t0": 2e-3})
    assert a.kick_drift(kp2, DT, graph=False) == b.kick_drift(kp2, DT, graph=True)
    _same(_state(a), _state(b))
    # replays without waiting, then one wait
    for _ in range(2):
        a.kick_drift(KP, DT, graph=False, wait=False)
        b.kick_drift(KP, DT, graph=True, wait=False)
    _same(_state(a), _state(b))
    # the recorded graph counts its kernels on every replay
    l0 = b.launch_count()
    b.kick_drift(KP, DT, graph=True)
    assert b.launch_count() > l0


def test_box_context_matches_single_boxes(gpu):
    mesh = 32
    sizes = [5000, 12000, 800]
    boxes = [_box(n, 10 + i, mesh) for i, n in enumerate(sizes)]
    gms = np.array([1.0 / n for n in sizes], np.float32)
    multi = _mk(mesh, nbox=len(sizes))
    cat = {k: np.concatenate([b[k] for b in boxes]) for k in ("x", "y", "z", "vx", "vy", "vz")}
    multi.upload_dict(cat)
    multi.set_boxes(sizes, gms)
    singles = []
    for b, gm in zip(boxes, gms):
        g = _mk(mesh)
        g.upload_dict(b)
        g.set_params(1.0 / (25 * mesh), 0.15, float(gm))
        singles.append(g)
    # forces and potentials, box by box, bit for bit
    multi.particle_to_grid()
    multi.compute_forces()
    fm, pm = multi.forces()
    dm = multi.download()
    off = 0
    for g, n in zip(singles, sizes):
        g.particle_to_grid()
        g.compute_forces()
        f, p = g.forces()
        d = g.download()
        # same cell order inside the box; ids restart at the box offset
        assert np.array_equal(dm["id"][off:off + n] - off, d["id"])
        assert np.array_equal(fm[off:off + n], f)
        assert np.array_equal(pm[off:off + n], p)
        off += n
    # a graph-recorded kick + drift of all boxes == each box's own
    for _ in range(2):
        multi.kick_drift(KP, DT, graph=True)
        for g in singles:
            g.kick_drift(KP, DT, graph=False)
    sm = _state(multi)
    off = 0
    for g, n in zip(singles, sizes):
        s = _state(g)
        for k in s:
            assert np.array_equal(sm[k][off:off + n], s[k]), k
        off += n


def test_box_context_rejects_bad_tables(gpu):
    g = _mk(32, nbox=2)
    P = _box(2000, 1, 32)
    g.upload_dict(P)
    with pytest.raises(RuntimeError):
        g.particle_to_grid()  # boxes not described yet
    with pytest.raises(RuntimeError):
        g.set_boxes([1000, 999], [1e-3, 1e-3])  # does not add up
    with pytest.raises(RuntimeError):
        g.set_boxes([1000, 1000], [1e-3, 0.0])  # GM must be > 0
    g.set_boxes([1000, 1000], [1e-3, 1e-3])
    g.particle_to_grid()
    with pytest.raises(RuntimeError):
        g.sort_by_rung(1)  # rung levels need one box
    with pytest.raises(RuntimeError):
        Gravity(mesh=512, order=2, bwidth=2.0, hsoft=1e-4, nbox=64)  # 27 + 6 key bits


def test_batch_of_meshes_matches_eager(gpu):
    specs = [(32, 3000, 1), (64, 20000, 2), (32, 6000, 3)]
    ctxs, refs = [], []
    for mesh, n, seed in specs:
        P = _box(n, seed, mesh)
        for lst in (ctxs, refs):
            g = _mk(mesh)
            g.upload_dict(P)
            lst.append(g)
    batch = Batch(ctxs)
    for _ in range(3):
        mr = batch.kick_drift(KP, DT)
        mrs = [g.kick_drift(KP, DT, graph=False) for g in refs]
        assert mr == max(mrs)
        assert batch.last_ms() > 0
    for g, r in zip(ctxs, refs):
        _same(_state(g), _state(r))
    batch.close()


@pytest.mark.parametrize("tuning", [dict(dense_cell=8), dict(dense_cell=48),
                                    dict(sparse_path=2), dict(sparse_path=2, dense_cell=48),
                                    dict(near_blocks_per_sm=1), dict(fft_tile=32),
                                    dict(fft_tile=128), dict(cols_tma=0),
                                    dict(cols_tma=1, fft_tile=16), dict(x_tma=0),
                                    dict(x_tma=0, mg2l_greens_direct=1),
                                    dict(mg2l_greens_direct=1), dict(x_tma=2),
                                    dict(x_tma=2, mg2l_greens_direct=1), dict(p2m_compact=1)])
def test_tuning_keeps_results(gpu, tuning):
    P = _box(40000, 5, 64)
    a, b = _mk(64, order=4), _mk(64, order=4)
    b.set_tuning(**{**a.tuning(), **tuning})
    for g in (a, b):
        g.upload_dict(P)
        g.particle_to_grid()
        g.compute_forces()
    fa, pa = a.forces()
    fb, pb = b.forces()
    if "dense_cell" in tuning or "sparse_path" in tuning:
        rel = np.linalg.norm(fa - fb, axis=1) / np.linalg.norm(fa, axis=1)
        assert rel.max() < 1e-5 and np.sqrt(np.mean(rel ** 2)) < 1e-6
        assert a.interaction_count() == b.interaction_count() > 0
        return
    assert np.array_equal(fa, fb) and np.array_equal(pa, pb)
    a.kick_drift(KP, DT, graph=True)
    b.kick_drift(KP, DT, graph=True)
    _same(_state(a), _state(b))


def test_autotune_restores_particles_and_caches(gpu, tmp_path):
    P = _box(30000, 8, 64)
    g = _mk(64)
    g.upload_dict(P)
    before = _state(g)
    cache = tmp_path / "tune.txt"
    t = g.autotune(KP, DT, cache_path=cache)
    assert t == g.tuning()
    assert t["dense_cell"] >= 1
    _same(before, _state(g))
    line = cache.read_text().strip().split()
    assert line[0].startswith("m64_p3_") and [int(v) for v in line[1:4]] == \
        [t["dense_cell"], t["near_blocks_per_sm"], t["fft_tile"]]
    # a cache hit applies the stored choice without timing
    h = _mk(64)
    h.upload_dict(P)
    assert h.autotune(KP, DT, cache_path=cache) == t
