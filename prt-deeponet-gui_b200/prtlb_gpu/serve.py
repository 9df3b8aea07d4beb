"""Served solves: a request loop over the batch engine.

Requests arrive at given times (a Poisson stream in the benchmarks).  A
request is admitted when its estimated device footprint fits in a fraction
(80 % by default) of the GPU's memory next to the solves already admitted;
admitted requests join the running batch at its next launch (continuous
batching), keep their state resident on the device through the flow and
transport phases, and retire when their own loop finishes.  Host work of
finished phases and new admissions overlaps the next batch launch.

The reference has no serving layer; this exists to run many solves per GPU
hour.  Each result is bit-identical to the single-solve calls.
"""

import collections
import ctypes
import math
import time

import numpy as np

from . import _lib
from .batch import Batch, Result, StreamBatch


def ladder_slots(limit, ratio):
    """Snapshot slots a transport run keeps: step 0, the ladder steps up to
    `limit` (n -> max(n + 1, ceil(n ratio))) and a final record."""
    k, n = 0, 1
    while n <= limit:
        k += 1
        n = max(n + 1, int(math.ceil(n * ratio)))
    return k + 2


def footprint(req):
    """Estimated peak device bytes of one request: the flow phase (two
    lattices, maps) or the transport phase (state, faces, snapshot ladder),
    whichever is larger, plus the material grid and field kept by both."""
    mat = req.mat
    n = int(mat.size)
    nf = int(np.count_nonzero(mat == 2))
    nd = mat.ndim
    q = 19 if nd == 3 else 9
    es = {"fp64": 8, "fp32": 4, "fp32f": 4, "fp16": 2}[req.flow["precision"]]
    common = n * (1 + 12)
    flow = 2 * q * nf * es + 4 * nf + 4 * n + n + 5 * 8 * (nf // 256 + 1)
    # the upstream-slot table of solves that fit in half the L2 cache,
    # counted up to an L2 of 256 MiB (an upper bound of the devices run on)
    table = 4 * (q - 1) * nf
    if 2 * q * nf * es + table <= (128 << 20):
        flow += table
    adr = 0
    if req.adr is not None:
        a = req.adr
        ns = int(a["n_species"])
        limit = int(a["steps"]) if a["steps"] is not None else int(a["max_steps"])
        slots = ladder_slots(limit, float(a["ratio"]))
        adr = n * (4 + 1 + 4 + 12 + 8 * ns) + 4 * nf * 2 + 4 * n * ns * slots + 4 * (limit + 1)
    return common + max(flow, adr) + (1 << 20)


def device_memory(device=0):
    """(free, total) bytes of the device."""
    fr, to = ctypes.c_uint64(), ctypes.c_uint64()
    rc = _lib.lib().prt_mem_info(int(device), ctypes.byref(fr), ctypes.byref(to))
    if rc != _lib.PRT_OK:
        msg = _lib.lib().prt_last_error(None)
        raise _lib.PrtError(rc, msg.decode() if msg else "prt_mem_info failed")
    return int(fr.value), int(to.value)


def poisson_arrivals(n, rate, seed=0):
    """n arrival times of a Poisson stream of `rate` per second, from 0."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / float(rate), int(n))) - 0.0


class Served(object):
    """Outcome of a served run: per-request Results (arrival, admission and
    completion host times attached) and the summary statistics."""

    def __init__(self, results, t0, t_end, launches):
        self.results = results
        lat = np.array([r.t_done - r.t_arrive for r in results if r.t_done is not None])
        wait = np.array([r.t_admit - r.t_arrive for r in results if r.t_admit is not None])
        ok = [r for r in results if r.error is None]
        span = max(t_end - t0, 1e-9)
        self.summary = {
            "requests": len(results),
            "completed": len(ok),
            "failed": len(results) - len(ok),
            "makespan_s": span,
            "solves_per_hour": len(ok) / span * 3600.0,
            "latency_p50_s": float(np.percentile(lat, 50)) if lat.size else None,
            "latency_p99_s": float(np.percentile(lat, 99)) if lat.size else None,
            "queue_p50_s": float(np.percentile(wait, 50)) if wait.size else None,
            "batch_launches": launches,
        }


def pore_voxels(req):
    """Pore voxels of a request (the flow solve's work per iteration)."""
    n = getattr(req, "_pores", None)
    if n is None:
        n = req._pores = int(np.count_nonzero(req.mat == 2))
    return n


def serve(requests, arrivals, device=0, hbm_fraction=0.8, graph_steps=20, quiet=True,
          budget_bytes=None, mode="streams", flow_cap=2000000):
    """Serve `requests` arriving at host times `arrivals` (seconds after the
    start).  Admission is first-come first-served while the summed
    footprints stay within hbm_fraction of the device memory (or
    `budget_bytes`) and the pore voxels of the solves in their flow phase
    stay within `flow_cap` (enough flow work to keep the GPU's memory system
    busy; a solve's transport phase is light and does not count, so new
    flows start as soon as older ones reach their transport).  An arrival
    that alone exceeds the cap is admitted when no flow is running.  Under
    overload this keeps the GPU full while finishing requests nearly in
    arrival order, instead of sharing the GPU among every queued request.
    mode "streams" runs the admitted solves as concurrent single-solve loops
    (StreamBatch), "tiles" through the batch engine's tile-list kernels
    (Batch).  Returns a Served."""
    order = np.argsort(np.asarray(arrivals, np.float64), kind="stable")
    pending = collections.deque((float(arrivals[i]), requests[i]) for i in order)
    if budget_bytes is None:
        _, total = device_memory(device)
        budget_bytes = int(hbm_fraction * total)
    b = (StreamBatch(device=device, quiet=quiet) if mode == "streams"
         else Batch(device=device, graph_steps=graph_steps, quiet=quiet))
    waiting = collections.deque()
    reserved = {}
    used = 0
    results = []
    t0 = time.perf_counter()
    try:
        while pending or waiting or len(b):
            now = time.perf_counter() - t0
            while pending and pending[0][0] <= now:
                waiting.append(pending.popleft())
            if len(b) == 0 and not waiting:
                time.sleep(max(0.0, pending[0][0] - now))
                continue
            if len(b):
                b.launch()
            # host work overlapping the launch: finished phases, admissions
            for res in b.process():
                used -= reserved.pop(id(res), 0)
            flow_load = sum(pore_voxels(j.req) for j in b._jobs.values() if j.phase == "flow")
            while waiting:
                t_arr, req = waiting[0]
                need = footprint(req)
                if used + need > budget_bytes and used > 0:
                    break
                if flow_cap and flow_load + pore_voxels(req) > flow_cap and flow_load > 0:
                    break
                flow_load += pore_voxels(req)
                waiting.popleft()
                try:
                    res = b.submit(req)
                except (_lib.PrtError, ValueError) as e:  # refused or out of memory
                    res = Result(req.tag)
                    res.error = e
                    res.t_submit = res.t_done = time.perf_counter()
                else:
                    reserved[id(res)] = need
                    used += need
                res.t_arrive = t0 + t_arr
                res.t_admit = time.perf_counter()
                results.append(res)
            if b._in_flight:
                b.wait(process=False)
        t_end = time.perf_counter()
        launches = b.stats()["launches"]
    finally:
        b.close()
    return Served(results, t0, t_end, launches)
