"""Benchmark of the ct2 gravity step on B200: particles/s per kick+drift.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one kick+drift at rung 0 through the reference-facing entry points
particle_to_grid -> kick -> drift (the first level of kick_step,
src/main.cpp:49-82): bin -> P2M -> FFT -> Green's multiply -> IFFT -> L2P +
direct sum -> kick -> drift, on seeded synthetic particles resident in HBM.  Default
workload: 128^3 = 2,097,152 particles, 70% in 512 Plummer spheres (a = 0.005,
log-uniform masses over 10x) plus 30% uniform, 256^3 mesh, Plummer softening
eps = 1/(50*128), dt = 1e-3.

Two forms of the same step are timed on the same particles:
  plain   the eager calls particle_to_grid, kick, drift (one host call per
          stage, the reference's call sequence);
  graph   ct2g_kick_drift with CT2G_STEP_GRAPH after ct2g_autotune: the whole
          step recorded once as a CUDA graph (device-held work-list sizes,
          persistent near-field grid) with autotuned launch shapes, one graph
          launch per step.
`value` is the graph form's whole-job particles/s (device time, CUDA events,
max over ranks); `forms` holds both.  `e2e` is the same metric through the
public API's host-state step (ct2g_kick_drift_host: the particle state copied
host->device, the step, the state copied device->host, every step; the
velocity and rung upload overlaps binning and the force solve).  `roofline` is for the
kernel with the largest share of the step; `cpu_baseline` is the CPU oracle
timed on a bounded sample.  Under torchrun (N>1) every rank runs an
independent box (replicas; the step has no exchange), value = all particles /
max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particles/s per kick+drift at 128^3 (rms force err <=1e-4 vs FP64 direct sum)"
UNIT = "particles/s"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return dict(hbm=float(d["hbm_gbs"]), sm_max_mhz=float(d.get("sm_max_mhz", 1965.0)),
                    source="measured")
    return dict(hbm=6650.0, sm_max_mhz=1965.0, source="fallback")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        # the raw samples: CT2G_CLOCKS_DIR when set (to keep them), else a
        # temporary directory
        out = os.environ.get("CT2G_CLOCKS_DIR") or tempfile.mkdtemp(prefix="ct2g_clocks_")
        self.path = os.path.join(out, "clocks_rank%d.csv" % device)

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device),
                                          "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                c = [s.strip() for s in line.split(",")]
                if len(c) >= 9:
                    rows.append(c)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        loaded = [s for s in sm if s > 0.5 * (max(sm) if sm else 1)]
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def workload(args, rank):
    from ct2_b200 import ics
    n = args.ngrid ** 3
    P = ics.plummer_spheres(n, seed=args.seed + rank, nspheres=args.nspheres, a=args.a)
    return P, n


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def _oracle_step_seconds(P, mbits, order, soft, bwidth, dt, reps=2):
    """Best-of-reps wall time of one CPU-oracle kick+drift (forces, update,
    drift) on particles P; the Green's table is built first and not timed (it
    is cached per mesh in the reference's design and here)."""
    from oracle import oracle as O
    n = len(P["x"])
    Gk = O.greens_k(mbits, order, 0, soft, bwidth)
    times = []
    for _ in range(reps):
        t = time.perf_counter()
        r = O.method_forces(P["x"], P["y"], P["z"], mbits, order, 0, soft, bwidth, 1.0 / n, Gk=Gk)
        f = (r["ffar"] + r["fnear"]).astype(np.float32)
        perm = r["perm"]
        vx, vy, vz, rung, mr = O.kick_update(P["vx"][perm], P["vy"][perm], P["vz"][perm],
                                             P["rung"][perm], f[:, 0], f[:, 1], f[:, 2],
                                             ascending=1, descending=1, top=1, first=0, prung=0,
                                             t0=dt, eta=0.15, max_dt=0.01, scale=1.0,
                                             hsoft=soft)
        O.drift(r["xs"], r["ys"], r["zs"], vx, vy, vz, dt, 1.0)
        times.append(time.perf_counter() - t)
    return min(times)


def _sample_shape(args):
    """The bounded CPU sample of the workload: the same generator scaled to
    1/64 of the particles and mesh cells (same particles per cell, sphere
    size in cells and softening in cells)."""
    ng, mesh = args.ngrid // 4, args.mesh // 4
    return ng, mesh, max(1, args.nspheres // 64)


def cpu_baseline(args, config1=True):
    """CPU oracle (C + numpy, all host threads) on a bounded sample of the
    workload (_sample_shape), and on the CPU parity configuration (32^3
    lattice + 0.1-spacing noise, 64^3 mesh, bwidth 3, order 4, eps = 1/1600)."""
    from ct2_b200 import ics
    ng, mesh, nsph = _sample_shape(args)
    P = ics.plummer_spheres(ng ** 3, seed=args.seed, nspheres=nsph, a=args.a * 4)
    n = ng ** 3
    soft = 1.0 / (50 * args.ngrid) * 4
    sec = _oracle_step_seconds(P, int(np.log2(mesh)), args.order, soft, args.bwidth, args.dt)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
    out = {"value": n / sec, "unit": UNIT, "cores": cores, "kind": "port",
           "cpu_model": cpu_model(),
           "sample": "CPU oracle, one full kick+drift (best of 2) on the workload generator "
                     "scaled to %d^3 particles, %d spheres, %d^3 mesh, order %d, bwidth %g (1/64 "
                     "of the particles and cells; particles/s extrapolates per particle); "
                     "Green's table excluded (cached per mesh)"
                     % (ng, nsph, mesh, args.order, args.bwidth)}
    if config1:
        L = ics.lattice(32, seed=0, sigma_cells=0.1)
        s1 = _oracle_step_seconds(L, 6, 4, float(np.float32(1.0 / 1600)), 3.0, 1e-3)
        out["config1"] = {"workload": "lattice_32cubed_mesh64 (32^3 lattice + 0.1-spacing noise, "
                                      "64^3 mesh, bwidth 3, order 4, eps 1/1600, dt 1e-3)",
                          "particles_per_s": 32768 / s1, "seconds_per_step": s1}
    return out


def run_reference(args, rank, world):
    """--impl reference: the reference path's CPU restatement (the reference
    itself does not build: HPX/sfmm absent, 3D FFT drivers empty), all host
    threads, a bounded sample per step."""
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    for _ in range(args.warmup):
        cpu_baseline(args, config1=False)
    vals = []
    for _ in range(args.steps):
        vals.append(cpu_baseline(args, config1=False))
    v = min(x["value"] for x in vals)
    cb = dict(vals[0])
    cb["value"] = v
    ng, mesh, nsph = _sample_shape(args)
    cfg = dict(_config(args, world))
    cfg.update({"workload": "plummer_spheres_%dcubed_mesh%d" % (ng, mesh),
                "particles_per_gpu": ng ** 3, "mesh": mesh, "spheres": nsph,
                "softening": "plummer eps=1/(50*%d) (the same in cells)" % ng,
                "sample_of": _config(args, world)["workload"],
                "sample": "1/64 of the particles and mesh cells of the GPU workload (same "
                          "particles per cell, sphere size and softening in cells); value is "
                          "particles/s of this sample"})
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg, "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _config(args, world):
    return {"workload": "plummer_spheres_128cubed_mesh256" if args.ngrid == 128 else
            "plummer_spheres_%dcubed_mesh%d" % (args.ngrid, args.mesh),
            "particles_per_gpu": args.ngrid ** 3, "mesh": args.mesh, "order": args.order,
            "bwidth": args.bwidth, "softening": "plummer eps=1/(50*%d)" % args.ngrid,
            "dt": args.dt, "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (particle store + mesh grids >> 126 MB)"}


def precision_form(args, g, P, n, local, kp, accuracy, stream):
    """Precision form: the same context with its y/x FFT passes on the tensor
    cores (BF16 hi+lo DFT matrix products), graph replays, own accuracy; the
    forward / inverse FFT stage times of both modes from one eager step."""
    import torch

    from ct2_b200 import replicas
    stages = {}
    for mode in ("fp32", "tc"):
        g.set_fft_mode(mode)
        g.upload_dict(P)
        g.particle_to_grid()
        g.kick(kp)
        st = g.stage_times()
        stages[mode] = {"fft_fwd_ms": float(st[2]), "mg2l_ms": float(st[3]),
                        "fft_inv_l2p_ms": float(st[4])}
    acc = accuracy(g)
    g.upload_dict(P)
    for _ in range(args.warmup):
        g.kick_drift(kp, args.dt, 1.0, graph=True, wait=False)
    g.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        g.kick_drift(kp, args.dt, 1.0, graph=True, wait=False)
    e1.record(stream)
    e1.synchronize()
    g.synchronize()
    value, ms = replicas.job_throughput(n, e0.elapsed_time(e1) / args.steps, device="cuda")
    g.set_fft_mode("fp32")
    return {"value": value, "ms_per_step": ms, "accuracy": acc, "stages": stages,
            "fft": "y/x passes: tcgen05 DFT products, BF16 hi+lo operands, FP32 accumulation"}


CAL_THRESHOLDS = tuple(round(-4.5 + 0.1 * k, 1) for k in range(16))  # -4.5 .. -3.0
CAL_TARGET = 0.95e-4  # rms relative force error the calibration aims under


def calibrate_threshold(gl, Pt, n, nsample, seed):
    """The MLP threshold for the learned form, picked on the TRAINING state
    (never on the state the form is judged on): the largest of CAL_THRESHOLDS
    whose rms relative force error, against the FP64 Ewald sum on a seeded
    sample of the training state's particles, is within CAL_TARGET (the
    smallest threshold when none is).  Returns (threshold, table)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sel = np.sort(rng.choice(n, size=min(n, nsample), replace=False))
    truth = gl.ewald_direct(Pt["x"][sel], Pt["y"][sel], Pt["z"][sel])
    tn = np.linalg.norm(truth, axis=1)
    gl.upload_dict(Pt)
    gl.particle_to_grid()
    ids = gl.download()["id"]
    inv = np.empty_like(ids)
    inv[ids] = np.arange(len(ids), dtype=ids.dtype)
    best, table = CAL_THRESHOLDS[0], []
    for t in CAL_THRESHOLDS:
        gl.learned_select("mlp", t)
        gl.compute_forces()
        f, _ = gl.forces()
        rms = float(np.sqrt(np.mean((np.linalg.norm(f[inv[sel]] - truth, axis=1) / tn) ** 2)))
        table.append({"threshold_log10": t, "rms_rel": rms,
                      "cells_selected": int(gl.learned_cells()["nselected"])})
        if rms <= CAL_TARGET:
            best = t
    return best, table


def learned_form(args, P, n, soft, local, kp, accuracy):
    """Learned form: the plain stencil narrowed to --learned-base, and the
    cells an MLP selects widened back to --bwidth.  The MLP is trained first
    on a state of the same generator with another seed (time reported, not
    part of the step); the step is then timed as graph replays."""
    import torch

    from ct2_b200 import ics, replicas
    from ct2_b200.gravity import Gravity
    gl = Gravity(mesh=args.mesh, order=args.order, bwidth=args.learned_base, hsoft=soft,
                 GM=1.0 / n, device=local, max_particles=n)
    gl.learned_enable(args.bwidth)
    Pt = ics.plummer_spheres(n, seed=args.seed + 100, nspheres=args.nspheres, a=args.a)
    t = time.perf_counter()
    gl.upload_dict(Pt)
    gl.particle_to_grid()
    ncell = gl.learned_collect()
    gl.mlp_init(seed=1)
    loss = gl.mlp_train(epochs=args.learned_epochs, batch=4096, lr=2e-3, seed=2)
    gl.synchronize()
    train_s = time.perf_counter() - t
    thr, cal = args.learned_threshold, None
    if thr is None:
        thr, cal = calibrate_threshold(gl, Pt, n, 4096, args.seed + 101)
    gl.upload_dict(P)
    gl.learned_select("mlp", thr)
    acc = accuracy(gl)
    nsel = gl.learned_cells()["nselected"]
    tune = gl.autotune(kp, args.dt, 1.0, cache_path=args.tune_cache)
    gl.upload_dict(P)
    stream = torch.cuda.ExternalStream(gl.stream(), device=local)
    for _ in range(args.warmup):
        gl.kick_drift(kp, args.dt, 1.0, graph=True, wait=False)
    gl.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        gl.kick_drift(kp, args.dt, 1.0, graph=True, wait=False)
    e1.record(stream)
    e1.synchronize()
    value, ms = replicas.job_throughput(n, e0.elapsed_time(e1) / args.steps, device="cuda")
    # the same context with the correction off: the narrow base step alone,
    # so that the correction's own cost (learned - base) is on the line
    gl.learned_select("none")
    gl.upload_dict(P)
    base_acc = accuracy(gl)
    gl.upload_dict(P)
    for _ in range(args.warmup):
        gl.kick_drift(kp, args.dt, 1.0, graph=True, wait=False)
    gl.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        gl.kick_drift(kp, args.dt, 1.0, graph=True, wait=False)
    e1.record(stream)
    e1.synchronize()
    base_ms = e0.elapsed_time(e1) / args.steps
    out = {"value": value, "ms_per_step": ms, "accuracy": acc, "tuning": tune,
           "base_narrow": {"bwidth": args.learned_base, "ms_per_step": base_ms,
                           "accuracy": base_acc},
           "correction_ms": ms - base_ms,
           "base_bwidth": args.learned_base, "widened_to": args.bwidth,
           "threshold_log10": thr, "calibration": cal, "cells_selected": int(nsel),
           "training": {"cells": int(ncell), "epochs": args.learned_epochs, "mse": loss,
                        "seconds": train_s, "state": "same generator, seed + 100"}}
    gl.close()
    return out


FFT_METRIC = "complex 3D FFT of 4 x 512^3 CIC grids (grid points/s, forward)"
NFW_METRIC = "particles/s per kick+drift, 256^3 NFW halos on a 512^3 mesh"


def run_nfw(args, rank, world, local, emit=True):
    """--workload nfw256: the learned form's configuration.  256^3 particles in
    2000 NFW halos (c ~ U[5,15], dN/dM ~ M^-1.9 over two decades, r_vir ~
    M^(1/3)), 512^3 mesh, Plummer eps = cell/25, order --order.  plain: the
    graph step at bwidth --bwidth.  learned: bwidth --learned-base, the cells
    an MLP (trained first on the same generator with another seed) selects
    widened to --bwidth.  Both judged on a seeded 1% particle sample against
    the FP64 Ewald direct sum."""
    import torch

    from ct2_b200 import ics, replicas
    from ct2_b200.gravity import Gravity, kick_params
    ng = 256
    n = ng ** 3
    M = 512
    soft = 1.0 / (25 * M)
    t = time.perf_counter()
    P = ics.nfw_halos(n, seed=args.seed + rank)
    gen_s = time.perf_counter() - t
    kp = kick_params(ascending=True, descending=True, top=True, first=False, rung=0,
                     t0=args.dt, eta=0.15, max_dt=0.01, scale=1.0)
    rng = np.random.Generator(np.random.PCG64(321))
    sel = np.sort(rng.choice(n, size=max(1, int(round(args.nfw_sample * n))), replace=False))

    def timed(g):
        st = torch.cuda.ExternalStream(g.stream(), device=local)
        g.upload_dict(P)
        for _ in range(args.warmup):
            g.kick_drift(kp, args.dt, 1.0, graph=True, wait=False)
        g.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            g.kick_drift(kp, args.dt, 1.0, graph=True, wait=False)
        e1.record(st)
        e1.synchronize()
        g.synchronize()
        return e0.elapsed_time(e1) / args.steps

    def errors(g, truth):
        g.upload_dict(P)
        g.particle_to_grid()
        g.compute_forces()
        f, _ = g.forces()
        ids = g.download()["id"]
        inv = np.empty_like(ids)
        inv[ids] = np.arange(n, dtype=ids.dtype)
        d = np.linalg.norm(f[inv[sel]] - truth, axis=1)
        tn = np.linalg.norm(truth, axis=1)
        return {"rms_rel": float(np.sqrt(np.mean((d / tn) ** 2))), "max_rel": float((d / tn).max()),
                "sinks": int(len(sel))}

    g = Gravity(mesh=M, order=args.order, bwidth=args.bwidth, hsoft=soft, GM=1.0 / n,
                device=local, max_particles=n)
    g.upload_dict(P)
    t = time.perf_counter()
    truth = g.ewald_direct(P["x"][sel], P["y"][sel], P["z"][sel])
    truth_s = time.perf_counter() - t
    plain_acc = errors(g, truth)
    inter = g.interaction_count()
    plain_ms = timed(g)
    g.close()
    del g
    gl = Gravity(mesh=M, order=args.order, bwidth=args.learned_base, hsoft=soft, GM=1.0 / n,
                 device=local, max_particles=n)
    gl.learned_enable(args.bwidth)
    t = time.perf_counter()
    Pt = ics.nfw_halos(n, seed=args.seed + 100 + rank)
    gl.upload_dict(Pt)
    gl.particle_to_grid()
    ncell = gl.learned_collect()
    gl.mlp_init(seed=1)
    loss = gl.mlp_train(epochs=args.learned_epochs, batch=4096, lr=2e-3, seed=2)
    gl.synchronize()
    train_s = time.perf_counter() - t
    thr, cal = args.learned_threshold, None
    if thr is None:
        thr, cal = calibrate_threshold(gl, Pt, n, max(1, int(round(0.2 * args.nfw_sample * n))),
                                       args.seed + 101 + rank)
    del Pt
    gl.learned_select("none")
    base_acc = errors(gl, truth)
    base_ms = timed(gl)
    gl.learned_select("mlp", thr)
    learned_acc = errors(gl, truth)
    nsel = gl.learned_cells()["nselected"]
    learned_ms = timed(gl)
    gl.close()
    value, ms = replicas.job_throughput(n, plain_ms, device="cuda")
    if rank == 0:
        line = {"metric": NFW_METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic: seeded NFW halos",
                "config": {"workload": "nfw256_mesh512", "particles_per_gpu": n, "mesh": M,
                           "order": args.order, "bwidth": args.bwidth,
                           "softening": "plummer eps=cell/25", "halos": 2000,
                           "l2": "inputs larger than L2"},
                "accuracy": plain_acc, "interactions_per_step": inter,
                "forms": {"plain": {"value": n / (plain_ms * 1e-3), "ms_per_step": plain_ms,
                                    "accuracy": plain_acc},
                          "base_narrow": {"bwidth": args.learned_base,
                                          "value": n / (base_ms * 1e-3), "ms_per_step": base_ms,
                                          "accuracy": base_acc},
                          "learned": {"value": n / (learned_ms * 1e-3), "ms_per_step": learned_ms,
                                      "accuracy": learned_acc, "cells_selected": int(nsel),
                                      "threshold_log10": thr, "calibration": cal,
                                      "training": {"cells": int(ncell), "mse": loss,
                                                   "seconds": train_s,
                                                   "state": "same generator, seed + 100"}}},
                "timings_s": {"generate": gen_s, "ewald_truth": truth_s},
                "e2e": None, "gpu_launches": None, "roofline": None, "cpu_baseline": None}
        if emit:
            print(json.dumps(line), flush=True)
        return line
    return None



def fft512_form(args, P, n, local, with_forces=True):
    """The precision form's configuration: the 128^3 Plummer particles'
    cloud-in-cell deposit on a 512^3 mesh as four complex grids (the CIC mass
    and its three first moments about the mesh points, imaginary parts zero),
    transformed forward and back as one batch of complex 3D FFTs -- FP32
    CUDA-core passes against tensor-core y/x passes (radix-16/32 DFT products,
    BF16 hi+lo operands, FP32 accumulation); times by CUDA events on the
    context's stream, each spectrum checked against the FP64 transform of the
    mass grid; and the end force error of a mesh-512 solve with the
    tensor-core passes against the FP64 Ewald sum."""
    import torch

    from ct2_b200.gravity import Gravity
    M = 512
    peaks = _peaks()
    g = Gravity(mesh=M, order=1, bwidth=args.bwidth, hsoft=1.0 / (50 * args.ngrid),
                GM=1.0 / n, device=local, max_particles=n)
    g.upload_dict(P)
    stream = torch.cuda.ExternalStream(g.stream(), device=local)
    grid = torch.empty(4 * M ** 3 * 2, dtype=torch.float32, device="cuda")
    work = torch.empty_like(grid)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    g.cic_deposit(M, grid.data_ptr())
    e1.record(stream)
    e1.synchronize()
    deposit_ms = e0.elapsed_time(e1)
    # FP64 reference: the r2c transform of the mass grid on the GPU in FP64
    m0 = grid.view(4, M, M, M, 2)[0, ..., 0].double().cpu().numpy()
    ref = g.fft_r2c_3d(np.ascontiguousarray(m0))
    dim = M * M * (M // 2 + 1)
    ref = (ref[:dim] + 1j * ref[dim:]).reshape(M, M, M // 2 + 1)
    del m0
    res = {}
    for mode in ("fp32", "tc"):
        g.set_fft_mode(mode)
        fw, iv = [], []
        for it in range(args.warmup + args.steps):
            work.copy_(grid)
            torch.cuda.synchronize()
            e0.record(stream)
            g.fft3d_c2c_dev(work.data_ptr(), M, 4, 1)
            e1.record(stream)
            g.fft3d_c2c_dev(work.data_ptr(), M, 4, -1)
            e2.record(stream)
            e2.synchronize()
            if it >= args.warmup:
                fw.append(e0.elapsed_time(e1))
                iv.append(e1.elapsed_time(e2))
        work.copy_(grid)
        g.fft3d_c2c_dev(work.data_ptr(), M, 4, 1)
        g.synchronize()
        z = work.view(4, M, M, M, 2)[0, :, :, : M // 2 + 1, :].cpu().numpy()
        z = z[..., 0].astype(np.float64) + 1j * z[..., 1]
        err = float(np.linalg.norm(z - ref) / np.linalg.norm(ref))
        del z
        f_ms, i_ms = float(np.median(fw)), float(np.median(iv))
        # algorithmic bytes: one read and one write of the batch per 3D
        # transform (4 x 16 x 512^3); the three passes move three times that
        algo = 4 * 16.0 * M ** 3
        res[mode] = {"fft_fwd_ms": f_ms, "fft_inv_ms": i_ms, "spectrum_rms_rel_err": err,
                     "algorithmic_bytes_per_transform": algo,
                     "passes_bytes_per_transform": 3 * algo,
                     "achieved_gbs_passes": 3 * algo / (f_ms * 1e-3) / 1e9,
                     "frac_of_measured_hbm": 3 * algo / (f_ms * 1e-3) / 1e9 / peaks["hbm"]}
    g.set_fft_mode("fp32")
    g.close()
    del grid, work
    torch.cuda.empty_cache()
    out = {"deposit_ms": deposit_ms, "grids": 4, "mesh": M, "forms": res,
           "fft": "batch of 4 complex 512^3 grids; tc: y/x passes as tcgen05 DFT products, "
                  "BF16 hi+lo operands, FP32 accumulation"}
    if with_forces:
        # the end force error of the tensor-core passes on a 512^3 mesh solve
        gf = Gravity(mesh=M, order=args.order, bwidth=args.bwidth, hsoft=1.0 / (50 * args.ngrid),
                     GM=1.0 / n, device=local, max_particles=n)
        gf.upload_dict(P)
        rng = np.random.Generator(np.random.PCG64(123))
        sel = np.sort(rng.choice(n, size=min(args.accuracy_sinks, n), replace=False))
        truth = gf.ewald_direct(P["x"][sel], P["y"][sel], P["z"][sel])
        acc = {}
        for mode in ("fp32", "tc"):
            gf.set_fft_mode(mode)
            gf.upload_dict(P)
            gf.particle_to_grid()
            gf.compute_forces()
            f, _ = gf.forces()
            ids = gf.download()["id"]
            inv = np.empty_like(ids)
            inv[ids] = np.arange(n, dtype=ids.dtype)
            d = np.linalg.norm(f[inv[sel]] - truth, axis=1)
            tn = np.linalg.norm(truth, axis=1)
            acc[mode] = {"rms_rel": float(np.sqrt(np.mean((d / tn) ** 2))),
                         "max_rel": float((d / tn).max()), "sinks": int(len(sel))}
        gf.close()
        out["force_accuracy_mesh512"] = {"order": args.order, "bwidth": args.bwidth,
                                         "vs": "FP64 Ewald direct sum", **acc}
    return out


def run_fft512(args, rank, world, local):
    """--workload fft512: the precision form's configuration on its own line
    (fft512_form)."""
    P, n = workload(args, rank)
    out = fft512_form(args, P, n, local)
    best = out["forms"]["tc"]
    ms = best["fft_fwd_ms"]
    points = 4.0 * 512 ** 3
    if rank == 0:
        line = {"metric": FFT_METRIC, "value": points / (ms * 1e-3), "unit": "grid points/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "bf16x3 (tensor cores) / f32",
                "data": "synthetic: CIC deposit of the seeded 128^3 Plummer workload",
                "config": {"workload": "cic512x4_c2c", "mesh": 512, "grids": 4,
                           "particles": n, "l2": "inputs larger than L2 (4.3 GB)"},
                "result": out, "gpu_launches": None, "roofline": {
                    "kernel": "tensor-core y/x passes + z pass, forward batch", "bound": "hbm",
                    "achieved": best["achieved_gbs_passes"], "peak": _peaks()["hbm"],
                    "unit": "GB/s", "frac": best["frac_of_measured_hbm"], "traffic": None},
                "cpu_baseline": None, "e2e": None}
        print(json.dumps(line), flush=True)


BOX_METRIC = ("particles/s per kick+drift over 96 independent periodic boxes "
              "(16^3..128^3 particles, meshes 32^3..256^3)")


def run_boxes(args, rank, world, local, emit=True):
    """--workload boxes96: 96 independent boxes (particle counts 2^U[12,21],
    mesh = nearest power of two to 2 N^(1/3) clipped to [32, 256], Plummer +
    background generator seeded per box, softening = cell/25, GM = 1/N per
    box).  plain: the boxes one after another, each through the eager calls
    on a context of its mesh (data resident, uploads untimed).  batched: one
    box context per mesh holding all of that mesh's boxes, autotuned, and one
    Batch graph launch per step for all 96 boxes."""
    import torch

    from ct2_b200 import ics, replicas
    from ct2_b200.gravity import Batch, Gravity, kick_params
    boxes = ics.batch_boxes(96, seed=args.seed + 1000 * rank)
    meshes = sorted({b["mesh"] for b in boxes})
    groups = {m: [b for b in boxes if b["mesh"] == m] for m in meshes}
    ntot = sum(len(b["x"]) for b in boxes)
    kp = kick_params(ascending=True, descending=True, top=True, first=False, rung=0,
                     t0=args.dt, eta=0.15, max_dt=0.01, scale=1.0)
    keys = ("x", "y", "z", "vx", "vy", "vz")

    def order_for(mesh):
        # the sparse boxes of the small meshes need one more order for rms
        # 1e-4 (measured 1.0e-4 and 1.1e-4 at order 4); they hold ~3% of the
        # particles
        return args.order + 1 if mesh <= 64 else args.order

    def mk(mesh, nbox=1, nmax=0):
        return Gravity(mesh=mesh, order=order_for(mesh), bwidth=args.bwidth,
                       hsoft=1.0 / (25 * mesh), device=local, nbox=nbox, max_particles=nmax)

    # plain: box after box, eager calls, device time per box
    plain_ms = 0.0
    acc = []
    rng = np.random.Generator(np.random.PCG64(7))
    for m in meshes:
        g = mk(m, nmax=max(len(b["x"]) for b in groups[m]))
        st = torch.cuda.ExternalStream(g.stream(), device=local)
        for bi, b in enumerate(groups[m]):
            n = len(b["x"])
            g.upload_dict(b)
            g.set_params(1.0 / (25 * m), 0.15, 1.0 / n)
            if bi == 0:  # accuracy on the first box of each mesh
                g.particle_to_grid()
                g.compute_forces()
                f, _ = g.forces()
                d = g.download()
                sel = np.sort(rng.choice(n, size=min(1024, n), replace=False))
                t = g.ewald_direct(d["x"][sel], d["y"][sel], d["z"][sel])
                diff = np.linalg.norm(f[sel] - t, axis=1) / np.linalg.norm(t, axis=1)
                acc.append({"mesh": m, "particles": n, "rms_rel": float(np.sqrt(np.mean(diff ** 2))),
                            "max_rel": float(diff.max())})
                g.upload_dict(b)
            for _ in range(args.warmup):
                g.particle_to_grid()
                g.kick(kp)
                g.drift(args.dt, 1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(args.steps):
                g.particle_to_grid()
                g.kick(kp)
                g.drift(args.dt, 1.0)
            e1.record(st)
            e1.synchronize()
            plain_ms += e0.elapsed_time(e1) / args.steps
        g.close()
        del g
    plain_value = ntot / (plain_ms * 1e-3)

    # batched: a box context per mesh, autotuned, one graph launch per step
    ctxs = []
    tunings = {}
    for m in meshes:
        bs = groups[m]
        g = mk(m, nbox=len(bs), nmax=sum(len(b["x"]) for b in bs))
        cat = {k: np.concatenate([b[k] for b in bs]) for k in keys}
        g.upload_dict(cat)
        counts = [len(b["x"]) for b in bs]
        g.set_boxes(counts, [1.0 / c for c in counts])
        tunings[m] = g.autotune(kp, args.dt, 1.0, cache_path=args.tune_cache)
        g.upload_dict(cat)
        g.set_boxes(counts, [1.0 / c for c in counts])
        ctxs.append((g, cat, counts))
    batch = Batch([c[0] for c in ctxs])
    st = torch.cuda.ExternalStream(ctxs[0][0].stream(), device=local)
    for _ in range(args.warmup):
        batch.kick_drift(kp, args.dt, 1.0, wait=False)
    torch.cuda.synchronize()
    l0 = sum(c[0].launch_count() for c in ctxs)
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        batch.kick_drift(kp, args.dt, 1.0, wait=False)
    e1.record(st)
    e1.synchronize()
    torch.cuda.synchronize()
    ck = clocks.stop()
    launches = sum(c[0].launch_count() for c in ctxs) - l0
    value, ms = replicas.job_throughput(ntot, e0.elapsed_time(e1) / args.steps, device="cuda")

    # end to end: every box's state host->device, one batch step, device->host
    e2e = None
    if not args.no_e2e:
        def e2e_step():
            for g, cat, counts in ctxs:
                g.upload_dict(cat)
                g.set_boxes(counts, [1.0 / c for c in counts])
            batch.kick_drift(kp, args.dt, 1.0, wait=True)
            for g, _, _ in ctxs:
                g.download()
        e2e_step()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(max(1, args.steps // 2)):
            e2e_step()
        torch.cuda.synchronize()
        ems = (time.perf_counter() - t) * 1e3 / max(1, args.steps // 2)
        ev, _ = replicas.job_throughput(ntot, ems, device="cuda")
        e2e = {"value": ev, "unit": UNIT, "h2d_bytes_per_step": int(ntot * 25),
               "d2h_bytes_per_step": int(ntot * 29), "timing": "host wall clock (pageable copies)"}
    batch.close()
    if rank == 0:
        line = {"metric": BOX_METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic: 96 seeded Plummer+background boxes",
                "config": {"workload": "boxes96", "particles_per_gpu": ntot,
                           "boxes_per_mesh": {str(m): len(groups[m]) for m in meshes},
                           "particles_per_mesh": {str(m): int(sum(len(b["x"]) for b in groups[m]))
                                                  for m in meshes},
                           "order": {str(m): order_for(m) for m in meshes},
                           "bwidth": args.bwidth,
                           "softening": "plummer eps = cell/25", "dt": args.dt,
                           "parallelism": "replicas" if world > 1 else "single",
                           "l2": "inputs larger than L2"},
                "e2e": e2e, "gpu_launches": int(launches), "roofline": None,
                "cpu_baseline": None, "clocks": ck, "accuracy": acc,
                "forms": {"plain_box_by_box": {"value": plain_value, "ms_per_step": plain_ms},
                          "batched_graph": {"value": value, "ms_per_step": ms,
                                            "tuning": {str(k): v for k, v in tunings.items()}}}}
        if emit:
            print(json.dumps(line), flush=True)
    for g, _, _ in ctxs:
        g.close()
    return line if rank == 0 else None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ngrid", type=int, default=128)
    ap.add_argument("--mesh", type=int, default=256)
    ap.add_argument("--order", type=int, default=4)
    ap.add_argument("--bwidth", type=float, default=4.0)
    ap.add_argument("--nspheres", type=int, default=512)
    ap.add_argument("--a", type=float, default=0.005)
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--accuracy-sinks", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="plummer128",
                    choices=["plummer128", "boxes96", "fft512", "nfw256"])
    ap.add_argument("--nfw-sample", type=float, default=0.01,
                    help="nfw256: fraction of particles judged against FP64 Ewald")
    ap.add_argument("--learned-base", type=float, default=3.0,
                    help="learned form: plain stencil of the base step (0: skip the form)")
    ap.add_argument("--learned-threshold", type=float, default=None,
                    help="learned form: widen cells whose predicted log10 residual exceeds "
                         "this (default: calibrated on the training state)")
    ap.add_argument("--learned-epochs", type=int, default=30)
    ap.add_argument("--no-precision-form", dest="precision_form", action="store_false",
                    help="skip the tensor-core FFT form")
    ap.add_argument("--no-extra-forms", action="store_true",
                    help="skip the fft512, boxes96 and nfw256 forms of the default run")
    ap.add_argument("--form-steps", type=int, default=5,
                    help="timed steps of the extra forms in the default run")
    ap.add_argument("--tune-cache", default=None,
                    help="autotuner cache file (default: tune on every run)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)

    if args.workload in ("boxes96", "fft512", "nfw256"):
        {"boxes96": run_boxes, "fft512": run_fft512, "nfw256": run_nfw}[args.workload](
            args, rank, world, local)
        if dist:
            dist.destroy_process_group()
        return

    from ct2_b200 import replicas
    from ct2_b200.gravity import Gravity

    P, n = workload(args, rank)
    soft = 1.0 / (50 * args.ngrid)
    g = Gravity(mesh=args.mesh, order=args.order, bwidth=args.bwidth, hsoft=soft,
                GM=1.0 / n, device=local, max_particles=n)
    g.upload_dict(P)
    stream = torch.cuda.ExternalStream(g.stream(), device=local)

    from ct2_b200.gravity import kick_params
    kp = kick_params(ascending=True, descending=True, top=True, first=False, rung=0,
                     t0=args.dt, eta=0.15, max_dt=0.01, scale=1.0)

    def step():
        # one kick+drift at rung 0: the first level of kick_step
        # (src/main.cpp:49-82): particle_to_grid, kick, drift
        g.particle_to_grid()
        g.kick(kp)
        g.drift(args.dt, 1.0)

    # accuracy on the initial state: forces vs the FP64 Ewald direct sum at
    # a seeded sample of particles (by upload index)
    rng = np.random.Generator(np.random.PCG64(123))
    sel = np.sort(rng.choice(n, size=min(args.accuracy_sinks, n), replace=False))
    truth = g.ewald_direct(P["x"][sel], P["y"][sel], P["z"][sel])

    def accuracy(ctx):
        ctx.particle_to_grid()
        ctx.compute_forces()
        f, _ = ctx.forces()
        ids = ctx.download()["id"]
        inv = np.empty_like(ids)
        inv[ids] = np.arange(len(ids), dtype=ids.dtype)
        diff = np.linalg.norm(f[inv[sel]] - truth, axis=1)
        tn = np.linalg.norm(truth, axis=1)
        return {"rms_rel": float(np.sqrt(np.mean((diff / tn) ** 2))),
                "max_rel": float((diff / tn).max()),
                "rms_norm": float(np.sqrt(np.mean(diff ** 2) / np.mean(tn ** 2))),
                "sinks": int(len(sel))}

    acc = accuracy(g)
    g.upload_dict(P)

    # plain form: eager calls, per-stage events
    for _ in range(args.warmup):
        step()
    g.synchronize()
    stage_sum = np.zeros(7)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    inter = 0
    for _ in range(args.steps):
        step()
        stage_sum += g.stage_times()
        inter += g.interaction_count()
    e1.record(stream)
    e1.synchronize()
    plain_value, plain_ms = replicas.job_throughput(n, e0.elapsed_time(e1) / args.steps,
                                                    device="cuda")

    # graph form: autotuned launch shapes, one recorded graph per step
    tune = g.autotune(kp, args.dt, 1.0, cache_path=args.tune_cache)
    g.upload_dict(P)
    for _ in range(args.warmup):
        g.kick_drift(kp, args.dt, 1.0, graph=True, wait=False)
    g.synchronize()
    l0 = g.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0.record(stream)
    for _ in range(args.steps):
        g.kick_drift(kp, args.dt, 1.0, graph=True, wait=False)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    ck = clocks.stop()
    launches = g.launch_count() - l0
    ms_local = e0.elapsed_time(e1) / args.steps
    value, ms = replicas.job_throughput(n, ms_local, device="cuda")
    forms = {"plain": {"value": plain_value, "ms_per_step": plain_ms, "accuracy": acc},
             "graph_autotuned": {"value": value, "ms_per_step": ms, "tuning": tune,
                                 "accuracy": acc}}
    if args.precision_form and args.mesh in (256, 512):
        forms["precision"] = precision_form(args, g, P, n, local, kp, accuracy, stream)
        g.upload_dict(P)
    if args.learned_base > 0:
        forms["learned"] = learned_form(args, P, n, soft, local, kp, accuracy)
    if dist:
        dist.barrier()

    # end to end through the public API: host state in, step, host state out
    e2e = None
    if not args.no_e2e:
        def pinned(a):
            v = np.ascontiguousarray(a)
            view = v.view(np.int32) if v.dtype == np.uint32 else v
            return torch.from_numpy(view).pin_memory().numpy().view(v.dtype)
        pin = {k: pinned(P[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "rung")}
        outb = {k: torch.empty(n, dtype={"x": torch.int32, "y": torch.int32, "z": torch.int32,
                                         "vx": torch.float32, "vy": torch.float32,
                                         "vz": torch.float32, "rung": torch.int8}[k]).pin_memory()
                for k in pin}
        outn = {k: v.numpy() for k, v in outb.items()}
        for k in ("x", "y", "z"):
            outn[k] = outn[k].view(np.uint32)

        def e2e_step():
            # ct2g_kick_drift_host: positions in, the step (its velocity and
            # rung upload beside binning and the force solve), state out
            g.kick_drift_host(kp, args.dt, pin, outn, graph=True)
        for _ in range(2):
            e2e_step()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        e1.record(stream)
        e1.synchronize()
        evalue, ems = replicas.job_throughput(n, e0.elapsed_time(e1) / args.steps, device="cuda")
        e2e = {"value": evalue, "unit": UNIT,
               "h2d_bytes_per_step": int(n * 25), "d2h_bytes_per_step": int(n * 25)}

    # roofline of the dominant stage
    st = stage_sum / args.steps
    names = ["bin", "p2m", "fft_fwd", "mg2l", "fft_inv", "forces", "update_drift"]
    peaks = _peaks()
    M, nc = args.mesh, (args.order + 1) * (args.order + 2) * (args.order + 3) // 6
    CK = M * M * (M // 2 + 1)
    # algorithmic HBM bytes per stage of the step as it runs here: fft_fwd =
    # P2M inside the z pass (particles in, spectrum out) + the y pass (one
    # read, one write); mg2l = the fused x pass + Green's multiply + inverse x
    # pass (spectrum and Green's table in, spectrum out); fft_inv = the y pass
    # + the z pass with L2P (spectrum in; particle offsets in, forces out)
    algo_bytes = {"bin": 66.0 * n, "p2m": 0.0,
                  "fft_fwd": 24.0 * nc * CK + 12.0 * n, "mg2l": 20.0 * nc * CK,
                  "fft_inv": 24.0 * nc * CK + 28.0 * n, "update_drift": 61.0 * n}
    k = int(np.argmax(st))
    dom = names[k]
    if dom == "forces":
        flops = 20.0 * inter / args.steps
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        peak = sms * 128 * 2 * peaks["sm_max_mhz"] * 1e6 / 1e12
        ach = flops / (st[k] * 1e-3) / 1e12
        # DRAM traffic is not measured inside this run (no profiler here):
        # null, with the ncu figures kept beside the kernel's profile
        roof = {"kernel": "forces (direct sum)", "bound": "fp32", "achieved": ach, "peak": peak,
                "unit": "TFLOP/s", "frac": ach / peak, "traffic": None,
                "peak_source": "derived: SMs x 128 x 2 x max SM clock (no measured FP32 peak)"}
    else:
        ach = algo_bytes[dom] / (st[k] * 1e-3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": peaks["hbm"],
                "unit": "GB/s", "frac": ach / peaks["hbm"], "traffic": None,
                "peak_source": peaks["source"]}
    stages = {nm: float(t) for nm, t in zip(names, st)}
    # the HBM-bound stages against the measured copy bandwidth
    stage_roof = {nm: {"algorithmic_bytes": algo_bytes[nm],
                       "achieved_gbs": algo_bytes[nm] / (st[i] * 1e-3) / 1e9,
                       "frac": algo_bytes[nm] / (st[i] * 1e-3) / 1e9 / peaks["hbm"]}
                  for i, nm in enumerate(names) if nm in ("fft_fwd", "mg2l", "fft_inv") and st[i] > 0}

    # the configurations of the precision, batching and learned forms, each on
    # its own workload, with fewer timed steps (their own lines come from
    # --workload fft512 / boxes96 / nfw256)
    if not args.no_extra_forms:
        import copy
        a2 = copy.copy(args)
        a2.steps, a2.warmup = min(args.steps, args.form_steps), min(args.warmup, 3)
        forms["precision_fft512"] = fft512_form(a2, P, n, local)
        bl = run_boxes(a2, rank, world, local, emit=False)
        if bl is not None:
            forms["batched_boxes96"] = {k: bl[k] for k in ("metric", "value", "unit", "ms_per_step",
                                                          "config", "accuracy", "forms", "e2e",
                                                          "gpu_launches")}
        nl = run_nfw(a2, rank, world, local, emit=False)
        if nl is not None:
            forms["learned_nfw256"] = {k: nl[k] for k in ("metric", "value", "unit", "ms_per_step",
                                                         "config", "accuracy", "forms",
                                                         "interactions_per_step", "timings_s")}

    cb = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            cb = cpu_baseline(args)
        except Exception as ex:  # reported, not fatal
            cb = {"value": None, "error": repr(ex)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic: seeded Plummer spheres + uniform background",
                "config": _config(args, world), "e2e": e2e, "gpu_launches": int(launches),
                "roofline": roof, "cpu_baseline": cb, "clocks": ck, "accuracy": acc,
                "forms": forms, "stage_ms": stages, "stage_roofline": stage_roof,
                "interactions_per_step": inter / args.steps}
        print(json.dumps(line), flush=True)
    g.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
