#!/usr/bin/env python3
"""Benchmark of the PRT-LB hot path on B200: D3Q19 TRT flow + ADR transport.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one complete solve of the plain 3D case):
  64^3 periodic pack of solid spheres, radius U[4, 7], porosity 0.45, seed 0
  (synthetic stand-in for the reference's rock images);
  D3Q19 TRT Stokes from rest, float32 populations (f - w) collided in
  float32, float64 residual and integrals, force 2e-6, tau 0.8, run to a
  relative change of
  mean |u_x| <= 1e-6 per 50 iterations;
  then transport of one Monod solute (Ks = 0.5) at Pe = 10, Da = 1 until the
  reference's stop rule is met (tol 2e-3), 5 snapshots.

value  whole-job GLUPS with inputs resident in HBM: (flow iterations + transport
       steps) x 64^3 voxels per second, every voxel counted as the reference
       iterates every voxel; device-timed with CUDA events on the solver's
       stream, one event pair per step, L2 flushed between steps.
e2e    the same through the public drop-in API (stokes_d3q19 + solve_adr on
       host numpy arrays), host<->device copies inside the timed region.
roofline  the dominant kernel (the D3Q19 stream-collide) against the measured
       HBM copy bandwidth: algorithmic bytes = 152 B per pore voxel (19
       float32 read + written) + 1 B mask per voxel, per iteration.
cpu_baseline  the NumPy oracle (a restatement of the reference's algorithm)
       on a bounded sample of the same workload, one core.

--impl reference times the reference's CPU algorithm (the oracle port, since
the reference is Python that does not travel to the GPU host) with one
process per host core, on the same metric.

Multi-GPU: replicas only (the path does not shard; one independent solve per
rank), value = all ranks' updates / max-over-ranks time.
"""

import os

# concurrent solves need more than the default 8 hardware work queues; read
# when the CUDA context is created, so before torch touches the device
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import argparse  # noqa: E402
import contextlib  # noqa: E402
import ctypes
import io
import json
import multiprocessing as mp
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "prt-deeponet-gui_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

EDGE = 64
POROSITY = 0.45
SEED = 0
FORCE, TAU, FLOW_TOL, FLOW_NIT = 2e-6, 0.8, 1e-6, 30000
ADR_STEPS = None  # None: run to the reference's stop rule
# DRAM bytes (read + write) of one lb_step_kernel launch from an ncu capture
# (cache flushed before the launch), by grid edge.  At 64^3 they include the
# upstream-slot table (72 B per pore voxel, 8.4 MB), which the solve reads
# instead of the voxel map because its working set fits in L2.
TRAFFIC_PER_LAUNCH = {64: 25157632, 128: 176652032}
PE, DA, KS, N_T = 10.0, 1.0, 0.5, 5
# float32 populations collided in float32 (the "fp32" mode keeps the
# momentum in float64); float64 only for the residual and the integrals
PRECISION = "fp32f"
METRIC = "D3Q19 TRT+ADR GLUPS"
UNIT = "GLUPS"
LB_BYTES_PER_FLUID = 19 * 4 * 2  # float32 populations read + written
# one solute: C read and written, three face velocities, flags, list index
ADR_BYTES_PER_SOLUTE = 4 + 4 + 12 + 4 + 4
WORKLOAD = ("plain-3d: 64^3 sphere pack (r U[4,7], porosity 0.45, seed 0), D3Q19 TRT fp32 "
            "to tol 1e-6 + Monod ADR (Ks 0.5) Pe 10 Da 1 to the stop rule")


def geometry():
    from prtlb_gpu.geometry import sphere_pack_3d
    return sphere_pack_3d(EDGE, POROSITY, SEED)


def host_geometry():
    """The same pack from the NumPy placement loop of prtlb_gpu/geometry.py,
    loaded as a plain module by its path: neither the package nor its
    library enters the process (the CPU arms use this)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "prt_host_geometry", os.path.join(PKG, "prtlb_gpu", "geometry.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.random_pack((EDGE,) * 3, POROSITY, 4.0, 7.0, seed=SEED, native=False)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks(object):
    """nvidia-smi sampled every 200 ms while the timed region runs; the raw
    samples go to bench_clocks_<pid>.csv in $PRT_CLOCKS_DIR (default: the
    system's temporary directory)."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        where = os.environ.get("PRT_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(where, "bench_clocks_%d.csv" % os.getpid())

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 7:
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def flush_l2(torch, dev):
    buf = flush_l2.buf
    if buf is None:
        buf = flush_l2.buf = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    buf.fill_(1)


flush_l2.buf = None


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def device_solve(ctx, L, d_mat, d_vel, d_out, shape, chem):
    """One complete solve on device-resident buffers; returns (iters, steps)."""
    from prtlb_gpu import _lib
    from prtlb_gpu.adr import prepare, stats_dict, _run_device
    p = _lib.FlowParams()
    p.nd = 3
    for i in range(3):
        p.dims[i] = shape[i]
    p.nit, p.force, p.tau, p.magic, p.tol = FLOW_NIT, FORCE, TAU, 3.0 / 16.0, FLOW_TOL
    p.every, p.precision = 50, _lib.PRT_FP32_F32
    fi = _lib.FlowInfo()
    ctx.check(L.prt_flow_dev(ctx.handle, ctypes.c_void_p(d_mat), ctypes.byref(p),
                             ctypes.c_void_p(d_vel), ctypes.byref(fi)))
    geom = _lib.AdrGeom()
    geom.nd = 3
    for i in range(3):
        geom.dims[i] = shape[i]
    geom.pore_code, geom.biofilm_code = 2, -1
    st = _lib.AdrStats()
    ctx.check(L.prt_adr_stage_dev(ctx.handle, ctypes.c_void_p(d_mat), ctypes.c_void_p(d_vel),
                                  ctypes.byref(geom), ctypes.byref(st)))
    S = prepare(shape, stats_dict(st), PE, DA, n_species=1, chem=chem)
    steps = _run_device(ctx, S, N_T, d_out, steps=ADR_STEPS)
    return int(fi.iters), int(steps)


def max_over_ranks(torch, dist, ms, device):
    """The slowest rank's time: every rank's figure is all-reduced with MAX."""
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(updates_per_rank, world, max_ms):
    """Whole-job GLUPS of `world` independent replicas, each doing
    updates_per_rank, timed by the slowest rank."""
    return updates_per_rank * world / (max_ms * 1e-3) / 1e9


def run_ours(args, rank, world, torch, dist):
    from prtlb_gpu import _lib, solve_adr, stokes_d3q19
    from prtlb_gpu.chemistry import monod_chemistry
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    g = geometry()
    shape = g.shape
    ncell = int(np.prod(shape))
    nfluid = int((g == 2).sum())
    chem = monod_chemistry(KS)
    ctx = _lib.Context(dev)
    L = _lib.lib()
    t_mat = torch.from_numpy(g.copy()).to(f"cuda:{dev}")
    t_vel = torch.empty((3,) + shape, dtype=torch.float32, device=f"cuda:{dev}")
    t_out = torch.empty((N_T, 1) + shape, dtype=torch.float32, device=f"cuda:{dev}")
    stream = torch.cuda.ExternalStream(ctx.stream(), device=f"cuda:{dev}")

    def step():
        return device_solve(ctx, L, t_mat.data_ptr(), t_vel.data_ptr(), t_out.data_ptr(), shape,
                            chem)

    quiet = contextlib.redirect_stdout(io.StringIO())
    with quiet:
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches()
    ms_steps, flow_ms, adr_ms, iters, nsteps = [], [], [], [], []
    with Clocks(dev) as clk, contextlib.redirect_stdout(io.StringIO()):
        for _ in range(args.steps):
            flush_l2(torch, f"cuda:{dev}")
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            it, ns = step()
            e1.record(stream)
            e1.synchronize()
            ms_steps.append(e0.elapsed_time(e1))
            tm = ctx.timing()
            flow_ms.append(tm[0])
            adr_ms.append(tm[2])
            iters.append(it)
            nsteps.append(ns)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    launches = ctx.launches() - launches0
    total_ms = float(sum(ms_steps))
    updates = float(sum(iters) + sum(nsteps)) * ncell
    if dist is not None:
        total_ms = max_over_ranks(torch, dist, total_ms, f"cuda:{dev}")
    value = replicas_value(updates, world, total_ms)

    # e2e: the drop-in API on host arrays
    e2e_ms, e2e_split = [], []
    h2d = d2h = 0
    with contextlib.redirect_stdout(io.StringIO()):
        for k in range(max(1, min(args.steps, 3))):
            flush_l2(torch, f"cuda:{dev}")
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            w0 = time.perf_counter()
            v = stokes_d3q19(g, nit=FLOW_NIT, force=FORCE, tau_lb=TAU, tol=FLOW_TOL,
                             precision=PRECISION, ctx=ctx)
            w1 = time.perf_counter()
            tf = ctx.timing()
            out, tn = solve_adr(g, v, pe=PE, da=DA, n_t=N_T, n_species=1, chem=chem, ctx=ctx,
                                steps=ADR_STEPS)
            w2 = time.perf_counter()
            ta = ctx.timing()
            e1.record(stream)
            e1.synchronize()
            e2e_ms.append(e0.elapsed_time(e1))
            # host seconds of each call next to its device loop
            e2e_split.append({"flow_call_ms": (w1 - w0) * 1e3, "flow_loop_ms": tf[0],
                              "adr_call_ms": (w2 - w1) * 1e3, "adr_loop_ms": ta[2]})
    h2d = g.nbytes + g.nbytes + v.nbytes           # flow: mat; transport: mat + vel
    d2h = v.nbytes + out.nbytes                    # flow: vel; transport: snapshots
    e2e_updates = float(iters[0] + nsteps[0]) * ncell
    e2e_value = e2e_updates * world / (statistics.median(e2e_ms) * 1e-3) / 1e9

    # roofline of the dominant kernel from this run's own events
    fl_ms = statistics.mean(flow_ms)
    ad_ms = statistics.mean(adr_ms)
    per_launch_ms = fl_ms / max(iters[0], 1)
    lb_bytes = nfluid * LB_BYTES_PER_FLUID + 4 * ncell
    achieved = lb_bytes / (per_launch_ms * 1e-3) / 1e9
    peak, kind = peaks()
    roof = {"kernel": "lb_step_kernel<D3Q19,ModeF32>", "bound": "hbm",
            "regime": "L2-resident (two lattices + slot table = 26 MB < 126 MB L2): "
                      "latency-bound, not DRAM-bound; see side.dram_128 for the "
                      "DRAM-resident figures",
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": kind,
            "bytes_per_iteration": lb_bytes, "traffic": TRAFFIC_PER_LAUNCH.get(EDGE),
            "note": "algorithmic bytes = 152 B per pore voxel (19 float32 read + written) + "
                    "4 B voxel map per voxel, per iteration; time per iteration = flow loop "
                    "events / iterations (one launch per iteration, graph node gaps "
                    "included); traffic = DRAM bytes of one cold-cache iteration (the slot "
                    "table read instead of the map)"}
    res = {"ms_per_step": total_ms / args.steps, "value": value, "e2e": e2e_value,
           "h2d": h2d, "d2h": d2h, "launches": launches, "roof": roof, "clocks": clk.summary(),
           "flow_ms": fl_ms, "adr_ms": ad_ms, "iters": iters[0], "adr_steps": nsteps[0],
           "ncell": ncell, "nfluid": nfluid, "e2e_ms": e2e_ms, "e2e_split": e2e_split}
    if rank == 0 and not args.no_side:
        res["side"] = side_measurements(ctx, peak, kind)
        if world == 1:
            # figures beside the line: a failure there is recorded, not fatal
            for key, fn in (("batched_small_mix", batched_side), ("served_short", served_side)):
                try:
                    res["side"][key] = fn(args, torch)
                except Exception as e:  # noqa: BLE001
                    res["side"][key] = {"error": "%s: %s" % (type(e).__name__, e)}
    ctx.close()
    return res


def served_side(args, torch):
    """The served loop on a short stream (the first 16 requests of the served
    set, edges 32-160, Poisson 20 /s, concurrent solves) against the same
    stream one at a time, as `--mode served --requests 16` measures it."""
    ns = argparse.Namespace(**vars(args))
    ns.requests, ns.rate, ns.serve_mode, ns.warmup = 16, 20.0, "streams", 1
    d = run_served(ns, torch)
    keep = ("value", "unit", "latency_p50_s", "latency_p99_s", "queue_p50_s", "completed",
            "failed", "speedup_vs_plain", "identical_to_plain", "clocks")
    out = {k: d.get(k) for k in keep}
    out["plain"] = d.get("plain")
    out["workload"] = d["config"]["workload"]
    return out


def batched_side(args, torch):
    """The batch engine on 48 small solves (edges 24-48, the batched set's
    draws) against the same solves one at a time, as `--mode batched
    --edge-lo 24 --edge-hi 48` measures it (without its concurrent-solve arm)."""
    ns = argparse.Namespace(**vars(args))
    ns.edge_lo, ns.edge_hi, ns.requests, ns.warmup, ns.graph_steps = 24, 48, 48, 1, 20
    d = run_batched(ns, torch, streams=False)
    return {"metric": d["metric"], "unit": d["unit"], "value": round(d["value"], 1),
            "plain_solves_per_hour": round(d["plain"]["solves_per_hour"], 1),
            "speedup_vs_plain": round(d["speedup_vs_plain"], 3),
            "identical_to_plain": d["identical_to_plain"], "failed": d["failed"],
            "workload": d["config"]["workload"], "batch_seconds": round(d["ms_per_step"] / 1e3, 3),
            "plain_seconds": round(d["plain"]["seconds"], 3), "tiling": d["tiling"],
            "clocks": d["clocks"]}


def side_measurements(ctx, peak, kind):
    """Figures beside the bench line, each from its own loop's CUDA events:
    the flow and transport kernels on a DRAM-resident 128^3 pack (porosity
    0.45, seed 0: 2000 float32 flow iterations, 3000 Monod steps), and the
    whole plain 2D configuration (128^2 disks, porosity 0.6, D2Q9 to tol 1e-7
    at force 1e-6, then 4000 first-order steps at Pe 10, Da 1)."""
    from prtlb_gpu import solve_adr, stokes_d2q9, stokes_d3q19
    from prtlb_gpu.chemistry import default_chemistry, monod_chemistry
    from prtlb_gpu.geometry import disk_pack_2d, sphere_pack_3d
    quiet = contextlib.redirect_stdout(io.StringIO())
    g = sphere_pack_3d(128, POROSITY, SEED)
    n = int(g.size)
    nf = int((g == 2).sum())
    with quiet:
        v = stokes_d3q19(g, nit=2000, tol=0.0, precision=PRECISION, ctx=ctx)
        tf = ctx.timing()
        solve_adr(g, v, pe=PE, da=DA, n_t=3, n_species=1, chem=monod_chemistry(KS), steps=3000,
                  ctx=ctx)
        ta = ctx.timing()
    fl_us = tf[0] / tf[1] * 1e3
    fl_bytes = nf * LB_BYTES_PER_FLUID + 4 * n
    ad_us = ta[2] / ta[3] * 1e3
    ad_bytes = nf * ADR_BYTES_PER_SOLUTE
    dram = {
        "workload": "128^3 sphere pack (r U[4,7], porosity 0.45, seed 0), %d pore voxels" % nf,
        "flow": {"kernel": "lb_step_kernel<D3Q19,ModeF32>", "bound": "hbm",
                 "us_per_iteration": round(fl_us, 3),
                 "achieved": round(fl_bytes / fl_us / 1e3, 1), "peak": peak, "unit": "GB/s",
                 "frac": round(fl_bytes / fl_us / 1e3 / peak, 4), "peak_kind": kind,
                 "bytes_per_launch": fl_bytes, "traffic": TRAFFIC_PER_LAUNCH.get(128),
                 "glups_all_voxels": round(n / fl_us / 1e3, 3),
                 "glups_pore_voxels": round(nf / fl_us / 1e3, 3)},
        "transport": {"kernel": "adr_step_kernel<3,1,no biofilm>", "bound": "hbm",
                      "us_per_step": round(ad_us, 3),
                      "achieved": round(ad_bytes / ad_us / 1e3, 1), "peak": peak, "unit": "GB/s",
                      "frac": round(ad_bytes / ad_us / 1e3 / peak, 4), "peak_kind": kind,
                      "bytes_per_launch": ad_bytes,
                      "note": "algorithmic bytes = 28 B per solute voxel (C read + written, "
                              "3 faces, flags, index); the kernel is bounded by instruction "
                              "issue, not DRAM"},
    }
    g2 = disk_pack_2d(128, 0.6, SEED)
    n2 = int(g2.size)
    with quiet:
        w0 = time.perf_counter()
        v2 = stokes_d2q9(g2, nit=30000, force=1e-6, tau_lb=0.8, tol=1e-7, precision=PRECISION,
                         ctx=ctx)
        t2f = ctx.timing()
        solve_adr(g2, v2, pe=PE, da=DA, n_t=5, n_species=1, chem=default_chemistry(1),
                  steps=4000, ctx=ctx)
        w1 = time.perf_counter()
        t2a = ctx.timing()
    dev_ms = t2f[0] + t2a[2]
    ups = (t2f[1] + t2a[3]) * n2
    plain2d = {"workload": "plain 2D: 128^2 disks (r U[4,8], porosity 0.6, seed 0), D2Q9 TRT "
                           "fp32 force 1e-6 tau 0.8 to tol 1e-7, then one first-order solute "
                           "Pe 10 Da 1, 4000 steps, 5 snapshots",
               "flow_iters": int(t2f[1]), "transport_steps": int(t2a[3]),
               "device_ms": round(dev_ms, 3), "glups": round(ups / (dev_ms * 1e6), 3),
               "e2e_ms": round((w1 - w0) * 1e3, 3),
               "e2e_glups": round(ups / ((w1 - w0) * 1e9), 3)}
    return {"dram_128": dram, "plain2d": plain2d}


# ---------------------------------------------------------------------------
# batched and served modes (solves per hour; not the default bench line)
# ---------------------------------------------------------------------------
def plain_solve(req, ctx):
    """One request through the drop-in single-solve API, one after another:
    the plain per-geometry GPU path the batched and served forms are
    compared with.  Returns (out, t_norm) or the exception that ended it."""
    from prtlb_gpu import solve_adr, stokes_d3q19
    f = dict(req.flow)
    prec = f.pop("precision")
    a = dict(req.adr)
    try:
        with contextlib.redirect_stdout(io.StringIO()):
            v = stokes_d3q19(req.mat, precision=prec, ctx=ctx, **f)
            return solve_adr(req.mat, v, a.pop("pe"), a.pop("da"), a.pop("n_t"), ctx=ctx, **a)
    except (Exception, SystemExit) as e:
        return e


def _same(res, ref):
    if isinstance(ref, BaseException) or res.error is not None:
        return isinstance(ref, BaseException) and res.error is not None
    return bool(np.array_equal(res.out, ref[0]) and np.array_equal(res.t_norm, ref[1]))


def profile_batched(args, torch):
    """A short batch for kernel profiles: the batched set's solves capped at
    --profile-nit flow iterations and --profile-steps transport steps, one
    fixed tiling, the batch alone (no plain or concurrent arms), graphs as
    PRT_GRAPHS says.  Prints what ran; it is not a measurement."""
    from prtlb_gpu.batch import Batch
    from prtlb_gpu.workloads import request_set
    lo, hi = args.edge_lo or 24, args.edge_hi or 96
    reqs, _ = request_set(args.requests, lo, hi, seed=SEED, nit=args.profile_nit,
                          max_steps=args.profile_steps)
    tb, gm = (int(x) for x in args.profile_tiling.split(","))
    b = Batch(device=0, graph_steps=args.graph_steps, quiet=True)
    try:
        b.tune(tb, gm)
        res = [b.submit(r) for r in reqs]
        b.run()
        st = b.stats()
    finally:
        b.close()
    torch.cuda.synchronize()
    return {"profile": "batched", "requests": len(reqs), "edges": [lo, hi],
            "flow_nit": args.profile_nit, "transport_steps": args.profile_steps,
            "tiling": [tb, gm], "failed": sum(r.error is not None for r in res),
            "launches": int(st["launches"]), "steps": int(st["steps"])}


def run_batched(args, torch, streams=True):
    """48 uneven geometries (edges 24-96): the batch engine against the same
    solves one at a time."""
    from prtlb_gpu import _lib
    from prtlb_gpu.batch import solve_batch
    from prtlb_gpu.workloads import batched_set
    from prtlb_gpu.workloads import request_set
    t = time.perf_counter()
    if args.edge_lo or args.edge_hi:
        lo, hi = args.edge_lo or 24, args.edge_hi or 96
        reqs, draws = request_set(args.requests, lo, hi, seed=SEED)
    else:
        lo, hi = 24, 96
        reqs, draws = batched_set(args.requests, seed=SEED)
    gen_s = time.perf_counter() - t
    # warm-up: the same solves cut to 200 iterations and steps, so every
    # kernel variant, graph shape and allocation of the timed runs is met first
    small, _ = request_set(args.requests, lo, hi, seed=SEED, nit=200, max_steps=200)
    ctx = _lib.Context(0)
    for _ in range(args.warmup):
        [plain_solve(r, ctx) for r in small]
        solve_batch(small, quiet=True)
        if streams:
            solve_batch(small, quiet=True, mode="streams")
    torch.cuda.synchronize()
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        bstats = {}
        res = solve_batch(reqs, quiet=True, mode="tiles", graph_steps=args.graph_steps,
                          stats=bstats)
        torch.cuda.synchronize()
        t_batch = time.perf_counter() - t0
        t0 = time.perf_counter()
        res_streams = solve_batch(reqs, quiet=True, mode="streams") if streams else None
        torch.cuda.synchronize()
        t_streams = time.perf_counter() - t0
        t0 = time.perf_counter()
        ref, loops = [], []
        for r in reqs:
            ref.append(plain_solve(r, ctx))
            loops.append(ctx.timing())
        torch.cuda.synchronize()
        t_plain = time.perf_counter() - t0
    ctx.close()
    n = len(reqs)
    same = all(_same(a, b) for a, b in zip(res, ref))
    cells = sum(int(r.mat.size) for r in reqs)
    ceiling = batching_ceiling(reqs, loops, t_plain)
    return {"metric": "batched solves/h", "value": n / t_batch * 3600.0, "unit": "solves/h",
            "n_gpus": 1, "steps": 1, "warmup": args.warmup, "ms_per_step": t_batch * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "batched: %d sphere packs, edge U{%d..%d}, porosity "
                                   "U[0.35,0.6], Pe logU[0.1,100], Da logU[0.01,10], kinetics "
                                   "Monod / first order / reversible sorption, D3Q19 fp32 to tol "
                                   "1e-6 (cap 30000) + ADR to the stop rule (cap 100000)" % (
                                       n, lo, hi),
                       "voxels": cells, "seed": SEED, "geometry_s": round(gen_s, 2)},
            "mode": "tiles: one persistent launch per class of solves per step over a work "
                    "list of 256-voxel tiles, %d steps per CUDA graph, autotuned tiling"
                    % args.graph_steps,
            "plain": {"solves_per_hour": n / t_plain * 3600.0, "seconds": t_plain},
            "streams": ({"solves_per_hour": n / t_streams * 3600.0, "seconds": t_streams,
                         "identical_to_plain": all(_same(a, b) for a, b in zip(res_streams, ref))}
                        if streams else None),
            "speedup_vs_plain": t_plain / t_batch, "identical_to_plain": same,
            "tiling": {"tile_blocks": int(bstats["tile_blocks"]),
                       "grid_mult": int(bstats["grid_mult"]),
                       "launches": int(bstats["launches"]), "steps": int(bstats["steps"])},
            "ceiling": ceiling,
            "failed": sum(1 for r in res if r.error is not None), "clocks": clk.summary()}


def batching_ceiling(reqs, loops, t_plain):
    """What any batching of these solves can gain at most: the plain solves'
    wall time against the time their algorithmic bytes take at the HBM peak
    (flow: 2 x 19 float32 populations per pore voxel and iteration plus the
    4-byte voxel map; transport: (8 ns + 20) bytes per solute voxel and
    step), and against the sum of their device loops alone."""
    peak, kind = peaks()
    es = {"fp64": 8, "fp32": 4, "fp32f": 4, "fp16": 2}
    t_bytes = t_loops = 0.0
    for r, tm in zip(reqs, loops):
        nf = int((np.asarray(r.mat) == 2).sum())
        nv = int(np.asarray(r.mat).size)
        ns = int(r.adr["n_species"])
        fb = tm[1] * (2 * 19 * es[r.flow["precision"]] * nf + 4 * nv)
        ab = tm[3] * (8 * ns + 20) * nf
        t_bytes += (fb + ab) / (peak * 1e9)
        t_loops += (tm[0] + tm[2]) * 1e-3
    return {"plain_wall_s": t_plain, "plain_device_loops_s": t_loops,
            "bytes_at_peak_s": t_bytes, "peak_gbs": peak, "peak_kind": kind,
            "max_speedup_bytes": t_plain / max(t_bytes, 1e-12),
            "max_speedup_host_overhead": t_plain / max(t_loops, 1e-12),
            "note": "a batch can at most remove the host and launch time between loops "
                    "(max_speedup_host_overhead) and, beyond that, make every loop run at "
                    "the HBM peak on algorithmic bytes (max_speedup_bytes)"}


def run_served(args, torch):
    """A Poisson stream of requests (edges 32-160) through the served loop,
    against the same stream through the plain path one at a time (first
    come, first served)."""
    from prtlb_gpu import _lib
    from prtlb_gpu.batch import solve_batch
    from prtlb_gpu.serve import poisson_arrivals, serve
    from prtlb_gpu.workloads import batched_set, served_set
    t = time.perf_counter()
    reqs, draws = served_set(args.requests, seed=SEED)
    gen_s = time.perf_counter() - t
    arrivals = poisson_arrivals(len(reqs), args.rate, seed=SEED)
    small, _ = batched_set(2, seed=SEED + 1, nit=200, max_steps=200)
    ctx = _lib.Context(0)
    for _ in range(args.warmup):
        [plain_solve(r, ctx) for r in small]
        solve_batch(small, quiet=True)
    torch.cuda.synchronize()
    with Clocks(0) as clk:
        srv = serve(reqs, arrivals, mode=args.serve_mode, flow_cap=args.flow_cap)
        torch.cuda.synchronize()
        # plain: one server, first come first served, same arrival times
        t0 = time.perf_counter()
        lat, ref = [], [None] * len(reqs)
        for i in np.argsort(arrivals, kind="stable"):
            now = time.perf_counter() - t0
            if now < arrivals[i]:
                time.sleep(arrivals[i] - now)
            ref[i] = plain_solve(reqs[i], ctx)
            lat.append(time.perf_counter() - t0 - arrivals[i])
        t_plain = time.perf_counter() - t0
    ctx.close()
    byreq = {r.tag: r for r in srv.results}
    same = all(_same(byreq[i], ref[i]) for i in range(len(reqs)))
    S = srv.summary
    n = len(reqs)
    return {"metric": "served solves/h", "value": S["solves_per_hour"], "unit": "solves/h",
            "n_gpus": 1, "steps": 1, "warmup": args.warmup, "ms_per_step": S["makespan_s"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "served: %d requests, Poisson %.3g req/s, edge U{32..160}, "
                                   "draws as the batched set, 80%% HBM admission, flow phase "
                                   "capped at %d pore voxels, %s" % (
                                       n, args.rate, args.flow_cap, args.serve_mode),
                       "seed": SEED, "geometry_s": round(gen_s, 2)},
            "latency_p50_s": S["latency_p50_s"], "latency_p99_s": S["latency_p99_s"],
            "queue_p50_s": S["queue_p50_s"], "completed": S["completed"], "failed": S["failed"],
            "plain": {"solves_per_hour": n / t_plain * 3600.0, "seconds": t_plain,
                      "latency_p50_s": float(np.percentile(lat, 50)),
                      "latency_p99_s": float(np.percentile(lat, 99))},
            "speedup_vs_plain": (S["solves_per_hour"] * t_plain) / (n * 3600.0),
            "identical_to_plain": same, "clocks": clk.summary()}


def _err(a, b, mask=None):
    """(relative L2, max abs error / max |reference|) of a against b."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is not None:
        a, b = a[..., mask], b[..., mask]
    nb = float(np.sqrt((b ** 2).sum()))
    mb = float(np.abs(b).max())
    return (float(np.sqrt(((a - b) ** 2).sum())) / nb if nb else 0.0,
            float(np.abs(a - b).max()) / mb if mb else 0.0)


def run_precision(args, torch):
    """The precision sweep: flow stored in fp32 / fp32f / fp16 against the
    fp64 solve (the reference's arithmetic) on sphere packs at 128^3 and
    192^3 -- velocity, permeability -- and the float32 transport (reversible
    sorption, K_d 0.5) driven by each field at Pe 1 / 10 / 100 against the
    transport driven by the fp64 field.  (The float32 transport against its
    float64 twin is a test: tests/test_sorption.py.)"""
    from prtlb_gpu import _lib, solve_adr, stokes_d3q19
    from prtlb_gpu.chemistry import reversible_sorption_chemistry
    from prtlb_gpu.geometry import sphere_pack_3d
    ctx = _lib.Context(0)
    rows = []
    q = contextlib.redirect_stdout(io.StringIO())
    cases = [(128, 0.35), (128, 0.45), (128, 0.55), (192, 0.45)]
    with Clocks(0) as clk, q:
        for edge, phi in cases:
            g = sphere_pack_3d(edge, phi, SEED)
            m = g == 2
            v, info = {}, {}
            for prec in ("fp64", "fp32", "fp32f", "fp16"):
                info[prec] = {}
                v[prec] = stokes_d3q19(g, nit=FLOW_NIT, force=FORCE, tau_lb=TAU, tol=FLOW_TOL,
                                       precision=prec, info=info[prec], ctx=ctx)
            for prec in ("fp32", "fp32f", "fp16"):
                l2, mx = _err(v[prec], v["fp64"], m)
                k, k64 = info[prec]["permeability"], info["fp64"]["permeability"]
                row = {"edge": edge, "porosity": phi, "precision": prec, "field": "velocity",
                       "rel_l2": l2, "max_err": mx, "permeability_rel_err": abs(k - k64) / abs(k64),
                       "flow_iters": info[prec]["flow_iters"],
                       "flow_iters_fp64": info["fp64"]["flow_iters"]}
                rows.append(row)
            if edge == 128 and phi == 0.45:
                chem = reversible_sorption_chemistry(0.5, 1.0)
                for pe in (1.0, 10.0, 100.0):
                    c = {}
                    for prec in ("fp64", "fp32", "fp16"):
                        c[prec], _ = solve_adr(g, v[prec], pe=pe, da=1.0, n_t=3, n_species=2,
                                               chem=chem, steps=args.adr_sweep_steps, ctx=ctx)
                    for prec in ("fp32", "fp16"):
                        l2, mx = _err(c[prec][-1], c["fp64"][-1])
                        rows.append({"edge": edge, "porosity": phi, "precision": prec,
                                     "field": "concentration (sorption, Pe %g, %d steps)" % (
                                         pe, args.adr_sweep_steps), "rel_l2": l2, "max_err": mx})
    ctx.close()
    worst = max(r["rel_l2"] for r in rows if r["precision"] == "fp32" and r["field"] == "velocity")
    return {"metric": "fp32 velocity rel L2 vs fp64 (worst case)", "value": worst,
            "unit": "relative L2", "n_gpus": 1, "steps": 1, "warmup": 0,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "precision sweep: sphere packs 128^3 (porosity 0.35/0.45/0.55) "
                                   "and 192^3 (0.45), r U[4,7], seed 0; flow to tol 1e-6 "
                                   "(cap 30000)", "seed": SEED},
            "rows": rows, "clocks": clk.summary()}


# ---------------------------------------------------------------------------
# CPU: the oracle (a restatement of the reference's NumPy algorithm)
# ---------------------------------------------------------------------------
def cpu_sample(args_tuple):
    """Time a bounded sample of the workload with the NumPy oracle:
    `its` flow iterations and `steps` transport steps on the 64^3 pack."""
    its, steps = args_tuple
    sys.path[:0] = [ROOT]
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle import prtlb_oracle as O
    g = host_geometry()
    t0 = time.perf_counter()
    v = O.stokes(g, nit=its, force=FORCE, tau_lb=TAU, tol=0.0)
    t1 = time.perf_counter()
    v[0] += 1e-4 * (g == 2)  # a moving field for the transport sample
    with contextlib.redirect_stdout(io.StringIO()):
        O.solve_adr(g, v, pe=PE, da=DA, n_t=2, n_species=1, steps=steps,
                    chem=O.monod_chemistry(KS))
    t2 = time.perf_counter()
    n = g.size
    return {"flow_s": t1 - t0, "adr_s": t2 - t1, "updates": float(its + steps) * n,
            "its": its, "steps": steps}


def cpu_baseline_line(procs, its, steps):
    ctxm = mp.get_context("spawn")
    t0 = time.perf_counter()
    if procs == 1:
        res = [cpu_sample((its, steps))]
    else:
        with ctxm.Pool(procs) as pool:
            res = pool.map(cpu_sample, [(its, steps)] * procs)
    wall = time.perf_counter() - t0
    per = [r["updates"] / (r["flow_s"] + r["adr_s"]) for r in res]
    value = sum(per) / 1e9
    return value, res, wall


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-its", type=int, default=20)
    ap.add_argument("--cpu-steps", type=int, default=100)
    # smaller cases of the same kernels, for profiling runs only (the bench
    # line is always taken with the defaults)
    ap.add_argument("--edge", type=int, default=64)
    ap.add_argument("--flow-nit", type=int, default=30000)
    ap.add_argument("--adr-steps", type=int, default=None)
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the CPU baseline sample (profiling runs)")
    ap.add_argument("--no-side", action="store_true",
                    help="skip the 128^3 kernel rooflines and the plain 2D figures")
    # solves-per-hour modes (each prints its own line; the default is the
    # plain 3D bench line)
    ap.add_argument("--mode", default="plain",
                    choices=["plain", "batched", "served", "precision"])
    ap.add_argument("--adr-sweep-steps", type=int, default=3000)
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--profile-nit", type=int, default=0,
                    help="batched mode: a short batch for kernel profiles, solves capped at "
                         "this many flow iterations")
    ap.add_argument("--profile-steps", type=int, default=600,
                    help="with --profile-nit: transport steps per solve")
    ap.add_argument("--profile-tiling", default="4,0",
                    help="with --profile-nit: tile blocks, grid multiple")
    ap.add_argument("--graph-steps", type=int, default=20,
                    help="batched mode: batch steps per graph replay between host checks")
    ap.add_argument("--edge-lo", type=int, default=0,
                    help="batched mode: smallest cubic edge (default: the batched set's 24)")
    ap.add_argument("--edge-hi", type=int, default=0,
                    help="batched mode: largest cubic edge (default: the batched set's 96)")
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--serve-mode", default="streams", choices=["streams", "tiles"])
    ap.add_argument("--flow-cap", type=int, default=2000000)
    args = ap.parse_args()
    if args.mode != "plain" and args.impl == "ours":
        import torch
        fn = {"batched": run_batched, "served": run_served, "precision": run_precision}[args.mode]
        if args.mode == "batched" and args.profile_nit:
            fn = profile_batched
        print(json.dumps(fn(args, torch)))
        return
    globals().update(EDGE=args.edge, FLOW_NIT=args.flow_nit, ADR_STEPS=args.adr_steps)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    config = {"workload": WORKLOAD, "edge": EDGE, "voxels": EDGE ** 3, "porosity": POROSITY,
              "seed": SEED, "flow": "D3Q19 TRT: f-w stored and collided in float32, "
                                    "float64 residual, mass and permeability sums",
              "transport": "Monod Ks 0.5, Pe 10, Da 1, n_t 5, stop rule tol 2e-3",
              "l2": "flushed (256 MB write) before every timed step",
              "parallelism": "replicas" if world > 1 else "single"}

    if args.impl == "reference":
        if rank != 0:
            return
        procs = os.cpu_count() or 1
        vals = []
        for _ in range(args.warmup + args.steps):
            v, res, wall = cpu_baseline_line(procs, 4, 20)
            vals.append(v)
        value = statistics.median(vals[args.warmup:]) if args.steps else vals[-1]
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                                 "sample": "per process: 4 D3Q19 iterations + 20 transport "
                                           "steps of the 64^3 workload (NumPy oracle)"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_mod
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod
    r = run_ours(args, rank, world, torch, dist)
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            v, res, wall = cpu_baseline_line(1, args.cpu_its, args.cpu_steps)
            cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": "%d D3Q19 iterations + %d Monod transport steps of the 64^3 "
                             "workload, NumPy oracle, %.1f s" % (args.cpu_its, args.cpu_steps,
                                                                 wall)}
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": config,
                "e2e": {"value": r["e2e"], "unit": UNIT, "h2d_bytes_per_step": r["h2d"],
                        "d2h_bytes_per_step": r["d2h"]},
                "gpu_launches": r["launches"], "roofline": r["roof"], "clocks": r["clocks"],
                "cpu_baseline": cpu,
                "detail": {"flow_ms": r["flow_ms"], "transport_ms": r["adr_ms"],
                           "flow_iters": r["iters"], "transport_steps": r["adr_steps"],
                           "voxels": r["ncell"], "pore_voxels": r["nfluid"],
                           "e2e_ms": r["e2e_ms"], "e2e_split": r["e2e_split"],
                           "solves_per_hour": 3.6e6 / r["ms_per_step"] * world,
                           # the same updates counted over the pore voxels only
                           "glups_pore_voxels": r["value"] * r["nfluid"] / r["ncell"],
                           # each loop on its own, over all voxels (one chemical)
                           "flow_glups": r["iters"] * r["ncell"] / max(r["flow_ms"] * 1e6, 1e-9),
                           "transport_gcell_species_per_s":
                               r["adr_steps"] * r["ncell"] / max(r["adr_ms"] * 1e6, 1e-9)},
                "side": r.get("side")}
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
