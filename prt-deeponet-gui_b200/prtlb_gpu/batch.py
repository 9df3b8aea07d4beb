"""Batched solves: many flow + transport solves through one time loop.

The reference solves one rock at a time (build_dataset_3d.py calls
stokes_d3q19 and then solve_adr per rock).  Here a ``Batch`` holds any
number of solves, each in its own libprtlb context; the library's batch
engine advances all of them together, one persistent launch per class of
jobs per step inside a CUDA graph, and a solve leaves the batch when its
own loop has finished.  A solve's results are bit-identical to
``stokes_d3q19`` / ``stokes_d2q9`` followed by ``solve_adr`` on the same
arguments, whatever else shares the batch.

A ``Request`` carries the arguments of both calls.  ``Batch.submit`` sets
up its flow solve; ``Batch.advance`` runs batch steps, then moves finished
flow solves on to their transport run (the host set-up of solve_adr, with
the velocity field staying on the device) and finished transport runs to
their ``Result``.
"""

import atexit
import contextlib
import ctypes
import io
import threading
import time

import numpy as np

from . import _lib
from . import adr as _adr
from . import flow as _flow

FLOW_DEFAULTS = dict(nit=30000, force=2e-6, tau_lb=0.8, magic=3.0 / 16.0, tol=1e-6,
                     precision="fp64")
ADR_DEFAULTS = dict(n_species=2, steps=None, tol=2e-3, max_steps=100000, ratio=1.12, chem=None,
                    da_abio=0.0)


# Idle contexts kept for the next solves on a device (at most _POOL_CAP):
# a solve that takes one reuses its device buffers instead of allocating
# them, and a finished solve's context costs no cudaFree.  What a kept
# context holds: the material grid and velocity field of its last solve and
# the transport buffers up to the keep size of prt_adr_end (256 MiB each).
_POOL_CAP = 64
_pool = {}
_pool_lock = threading.Lock()


def _take_context(device):
    with _pool_lock:
        kept = _pool.get(device)
        if kept:
            return kept.pop()
    return _lib.Context(device)


def _return_context(ctx, device):
    """A finished solve's context, with the device idle: kept, or closed
    when it failed or the pool is full."""
    if not ctx.handle:
        return
    if not getattr(ctx, "broken", False):
        _lib.lib().prt_adr_end(ctx.handle)  # frees transport buffers above the keep size
        with _pool_lock:
            kept = _pool.setdefault(device, [])
            if len(kept) < _POOL_CAP:
                kept.append(ctx)
                return
    ctx.close()


def release_contexts():
    """Close the idle contexts kept for reuse (and free their memory)."""
    with _pool_lock:
        kept = [c for lst in _pool.values() for c in lst]
        _pool.clear()
    for c in kept:
        c.close()


atexit.register(release_contexts)


class Request(object):
    """One solve: ``flow`` holds stokes_d3q19 / stokes_d2q9 keyword arguments
    (nit, force, tau_lb, magic, tol, precision); ``adr`` holds solve_adr's
    (pe, da, n_t and the optional n_species, steps, tol, max_steps, ratio,
    chem, da_abio), or None for a flow-only solve.  ``keep_velocity`` copies
    the velocity field to the host; ``fetch`` copies the snapshots."""

    def __init__(self, mat, flow=None, adr=None, tag=None, keep_velocity=False, fetch=True):
        self.mat = np.asarray(mat)
        self.flow = dict(FLOW_DEFAULTS)
        self.flow.update(flow or {})
        if adr is not None:
            missing = [k for k in ("pe", "da", "n_t") if k not in adr]
            if missing:
                raise ValueError("the transport solve needs %s" % ", ".join(missing))
            a = dict(ADR_DEFAULTS)
            a.update(adr)
            adr = a
        self.adr = adr
        self.tag = tag
        self.keep_velocity = bool(keep_velocity)
        self.fetch = bool(fetch)


class Result(object):
    """What one solve returns: ``vel`` (host copy or None), ``flow_info`` (the
    info dict of stokes_*), ``out`` / ``t_norm`` / ``adr_info`` (solve_adr's),
    ``error`` (the exception that ended the solve, or None) and host clock
    times ``t_submit``, ``t_flow`` (flow loop finished), ``t_done``; a
    served request also has ``t_arrive`` and ``t_admit``."""

    def __init__(self, tag):
        self.tag = tag
        self.vel = None
        self.flow_info = {}
        self.out = None
        self.t_norm = None
        self.adr_info = None
        self.steps = 0
        self.error = None
        self.t_submit = None
        self.t_flow = None
        self.t_done = None
        self.t_arrive = None
        self.t_admit = None

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_submit


class _Job(object):
    def __init__(self, req, ctx, res):
        self.req = req
        self.ctx = ctx
        self.res = res
        self.phase = "flow"
        self.S = None


class Batch(object):
    """A set of solves advanced together on one GPU.

    ``graph_steps`` steps form one CUDA graph replay; ``advance(steps)``
    enqueues whole replays.  ``quiet`` keeps the per-solve warnings of the
    reference (iteration cap, Mach, grid Peclet) out of stdout; they are
    kept in ``Result.flow_info['messages']`` instead."""

    def __init__(self, device=0, graph_steps=20, quiet=False):
        L = _lib.lib()
        h = ctypes.c_void_p()
        rc = L.prt_batch_create(int(device), int(graph_steps), ctypes.byref(h))
        if rc != _lib.PRT_OK:
            msg = L.prt_last_error(None)
            raise _lib.PrtError(rc, msg.decode() if msg else "prt_batch_create failed")
        self.handle = h
        self.device = int(device)
        self.graph_steps = int(graph_steps) or 20
        self.quiet = bool(quiet)
        self._jobs = {}
        self._ready = []      # collected solves waiting for their host work
        self._graveyard = []  # finished contexts, freed when the device is idle
        self._unlattice = []  # contexts past their flow loop: lattices freed then too
        self._in_flight = False
        self.finished = []

    # -- library plumbing -------------------------------------------------
    def _check(self, rc):
        if rc != _lib.PRT_OK:
            msg = _lib.lib().prt_batch_last_error(self.handle)
            raise _lib.PrtError(rc, msg.decode() if msg else "")

    def close(self):
        if self.handle:
            for job in list(self._jobs.values()):
                job.ctx.close()
            self._jobs.clear()
            self._ready = []
            self._bury()
            _lib.lib().prt_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        """Solves not finished yet (in the batch or waiting for host work)."""
        return len(self._jobs)

    def stats(self):
        """Kernel launches, graph builds, tile blocks, grid multiple, steps
        run, last launch ms, tiles of the last launch, and 1 while the
        tiling candidates are still being timed."""
        out = (ctypes.c_double * 8)()
        self._check(_lib.lib().prt_batch_stats(self.handle, out))
        keys = ("launches", "graph_builds", "tile_blocks", "grid_mult", "steps", "last_ms",
                "tiles", "tuning")
        return {k: float(out[i]) for i, k in enumerate(keys)}

    def tune(self, tile_blocks=0, grid_mult=0):
        """Fix the tiling (tile_blocks 1/2/4; grid_mult 1/2 resident waves of
        persistent blocks, or 0 for one block per tile) or, with
        tile_blocks 0, let the next launches time the candidates and keep
        the fastest."""
        self._check(_lib.lib().prt_batch_tune(self.handle, int(tile_blocks), int(grid_mult)))

    def _quiet(self):
        return contextlib.redirect_stdout(io.StringIO()) if self.quiet else contextlib.nullcontext()

    # -- solves -----------------------------------------------------------
    def submit(self, req):
        """Set up the flow solve of `req` and add it to the batch."""
        if not isinstance(req, Request):
            raise TypeError("submit() takes a Request")
        res = Result(req.tag)
        res.t_submit = time.perf_counter()
        nd = req.mat.ndim
        name = "3D flow" if nd == 3 else "2D flow"
        f = req.flow
        g, p = _flow.flow_params(req.mat, nd, name, f["nit"], f["force"], f["tau_lb"],
                                 f["magic"], f["tol"], f["precision"])
        ctx = _take_context(self.device)
        try:
            L = _lib.lib()
            ctx.check(L.prt_flow_start(ctx.handle, g.ctypes.data_as(ctypes.c_void_p),
                                       ctypes.byref(p)))
            self._enqueue(ctx, "flow")
        except BaseException:
            ctx.close()
            raise
        job = _Job(req, ctx, res)
        self._jobs[ctx.handle.value] = job
        return res

    def _enqueue(self, ctx, phase):
        """A started solve (its flow or its transport loop) joins the batch."""
        self._check(_lib.lib().prt_batch_add(self.handle, ctx.handle))

    def launch(self, steps=None):
        """Enqueue `steps` batch steps (default: one graph replay)."""
        steps = self.graph_steps if steps is None else int(steps)
        self._check(_lib.lib().prt_batch_launch(self.handle, steps))
        self._in_flight = True

    def wait(self, process=True):
        """Wait for the enqueued steps and collect the solves whose loop
        finished in them.  With process=True (default) their host work is
        done at once (see process()) and the Results completed now are
        returned; with process=False it is left for process(), so a caller
        can overlap it with the next launch."""
        L = _lib.lib()
        nd = ctypes.c_int32()
        self._check(L.prt_batch_wait(self.handle, ctypes.byref(nd)))
        self._in_flight = False
        self._bury()  # the device is idle: freeing memory costs no stall now
        if nd.value:
            handles = (ctypes.c_void_p * nd.value)()
            cnt = ctypes.c_int32()
            self._check(L.prt_batch_collect(self.handle, handles, nd.value, ctypes.byref(cnt)))
            for i in range(cnt.value):
                job = self._jobs.get(handles[i])
                if job is not None:
                    self._ready.append(job)
        return self.process() if process else []

    def process(self):
        """Host work of the collected solves: a finished flow solve gets its
        field and report and starts its transport run (which joins the
        batch); a finished transport run gets its snapshots.  Returns the
        Results completed."""
        done = []
        ready, self._ready = self._ready, []
        for job in ready:
            try:
                if job.phase == "flow":
                    self._flow_done(job)
                else:
                    self._adr_done(job)
            except (Exception, SystemExit) as e:  # SystemExit: a dead flow
                job.res.error = e
                job.phase = "done"
                job.ctx.broken = True  # closed, not kept for another solve
            if job.phase == "done":
                job.res.t_done = time.perf_counter()
                del self._jobs[job.ctx.handle.value]
                self._graveyard.append(job.ctx)
                done.append(job.res)
        if not self._in_flight:
            self._bury()
        self.finished.extend(done)
        return done

    def _bury(self):
        L = _lib.lib()
        for ctx in self._unlattice:
            if ctx.handle:
                ctx.check(L.prt_flow_release(ctx.handle))
        self._unlattice = []
        for ctx in self._graveyard:
            _return_context(ctx, self.device)
        self._graveyard = []

    def advance(self, steps=None):
        """launch() then wait()."""
        self.launch(steps)
        return self.wait()

    def run(self, max_steps=None):
        """Advance until every solve has finished (or `max_steps` steps).
        The host work of the solves collected by one wait (a finished flow
        solve's field and transport set-up, a finished run's snapshots) is
        done while the next graph replay runs, as in the served loop.
        One launch runs up to 8 graph replays (1, 2, 4, then 8), so the
        host's per-launch work is paid less often and the host work of the
        solves that finished has a long launch to hide behind; a solve that
        finishes is seen at most 8 replays late (its place in the batch
        costs nothing meanwhile), which for the longest solve of a batch
        adds at most two such delays (its flow end, its transport end)."""
        out = []
        n = 0
        reps = 1
        while self._jobs and (max_steps is None or n < max_steps):
            steps = self.graph_steps * reps
            if max_steps is not None:
                steps = min(steps, max_steps - n)
            self.launch(steps)
            out.extend(self.process())
            self.wait(process=False)
            reps = min(reps * 2, 8)
            n += steps
        out.extend(self.process())
        return out

    # -- phase changes ----------------------------------------------------
    def _flow_done(self, job):
        L = _lib.lib()
        req, ctx, res = job.req, job.ctx, job.res
        res.t_flow = time.perf_counter()
        fi = _lib.FlowInfo()
        vel = None
        if req.keep_velocity or (req.adr is not None and _needs_host_stage(req)):
            vel = np.empty((3,) + req.mat.shape, np.float32)
        ctx.check(L.prt_flow_finish(ctx.handle,
                                    vel.ctypes.data_as(ctypes.c_void_p) if vel is not None else None,
                                    ctypes.byref(fi)))
        f = req.flow
        name = "3D flow" if req.mat.ndim == 3 else "2D flow"
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf) if self.quiet else contextlib.nullcontext():
            _flow.flow_report(name, fi, f["force"], f["tau_lb"], f["tol"], res.flow_info,
                              f["precision"])
        if self.quiet:
            res.flow_info["messages"] = buf.getvalue()
        if req.keep_velocity:
            res.vel = vel
        if req.adr is None:
            job.phase = "done"
            return
        a = req.adr
        st = _lib.AdrStats()
        mat8, geom = _adr.stage_geom(req.mat, a["chem"])
        if _needs_host_stage(req):
            vel32 = np.ascontiguousarray(vel)
            ctx.check(L.prt_adr_stage(ctx.handle, mat8.ctypes.data_as(ctypes.c_void_p),
                                      vel32.ctypes.data_as(ctypes.c_void_p), ctypes.byref(geom),
                                      ctypes.byref(st)))
        else:
            ctx.check(L.prt_adr_stage_flow(ctx.handle, ctypes.byref(geom), ctypes.byref(st)))
        with self._quiet():
            S = _adr.prepare(req.mat.shape, _adr.stats_dict(st), a["pe"], a["da"],
                             n_species=a["n_species"], chem=a["chem"], da_abio=a["da_abio"],
                             mat=req.mat)
        job.S = S
        ctx.check(L.prt_adr_begin(ctx.handle, ctypes.byref(S.params)))
        # the lattices are freed once the device is idle (a free now would
        # wait for the launch in flight)
        self._unlattice.append(ctx)
        R = _adr.run_params(S, a["steps"], a["tol"], a["max_steps"], a["ratio"])
        ctx.check(L.prt_adr_start(ctx.handle, ctypes.byref(R)))
        self._enqueue(ctx, "adr")
        job.phase = "adr"

    def _adr_done(self, job):
        L = _lib.lib()
        req, ctx, res, S = job.req, job.ctx, job.res, job.S
        a = req.adr
        r = _lib.AdrResult()
        ctx.check(L.prt_adr_finish(ctx.handle, ctypes.byref(r)))
        n = int(r.steps)
        ks = _adr.ladder_steps(ctx)
        picked = _adr.pick(ks, n, int(a["n_t"]))
        res.steps = n
        res.adr_info = {}
        # the context is destroyed once the device is idle, which frees the
        # transport state (ending it here would wait for the launch in flight)
        if req.fetch:
            res.out, res.t_norm = _adr.outputs(ctx, S, int(a["n_t"]), n, ks, picked, a["steps"],
                                               a["max_steps"], res.adr_info, a["da"],
                                               a["da_abio"], end=False)
        else:
            total = int(max(n, 1))
            res.t_norm = (ks[picked].astype(np.float32) / total).astype(np.float32)
        job.phase = "done"


class StreamBatch(Batch):
    """The same interface over concurrent single-solve loops: every solve
    runs its own flow loop, then its own transport loop, each as one CUDA
    graph launched on the solve's own stream (prt_flow_launch /
    prt_adr_launch), so many solves share the GPU at once and each keeps the
    single-solve kernels.  wait() returns when at least one solve finished
    its current loop (or after `poll_s` with nothing finished)."""

    def __init__(self, device=0, quiet=False, poll_s=0.002):
        self.handle = None
        self.device = int(device)
        self.graph_steps = 0
        self.quiet = bool(quiet)
        self.poll_s = float(poll_s)
        self._jobs = {}
        self._ready = []
        self._graveyard = []
        self._unlattice = []
        self._in_flight = False
        self.finished = []
        self._launches = 0

    def _check(self, rc):
        if rc != _lib.PRT_OK:
            raise _lib.PrtError(rc, "stream batch call failed")

    def close(self):
        for job in list(self._jobs.values()):
            job.ctx.close()
        self._jobs.clear()
        self._ready = []
        self._bury()

    def stats(self):
        return {"launches": float(self._launches), "graph_builds": 0.0, "tile_blocks": 0.0,
                "grid_mult": 0.0, "steps": 0.0, "last_ms": 0.0, "tiles": 0.0}

    def tune(self, tile_blocks=0, grid_mult=0):
        pass

    def _enqueue(self, ctx, phase):
        L = _lib.lib()
        launch = L.prt_flow_launch if phase == "flow" else L.prt_adr_launch
        ctx.check(launch(ctx.handle))
        self._launches += 1

    def launch(self, steps=None):
        self._in_flight = True

    def wait(self, process=True):
        L = _lib.lib()
        busy = ctypes.c_int32()
        t0 = time.perf_counter()
        while True:
            found = False
            for key, job in list(self._jobs.items()):
                if job in self._ready or job.phase == "done":
                    continue
                job.ctx.check(L.prt_ctx_busy(job.ctx.handle, ctypes.byref(busy)))
                if not busy.value:
                    self._ready.append(job)
                    found = True
            if found or not self._jobs or time.perf_counter() - t0 >= self.poll_s:
                break
            time.sleep(0.0002)
        self._in_flight = False
        self._bury()
        return self.process() if process else []

    def run(self, max_steps=None):
        out = []
        while self._jobs:
            out.extend(self.advance())
        return out


def _needs_host_stage(req):
    """A biofilm material code makes the transport grid differ from the
    flow's pore/solid grid, so the transport is staged from the host."""
    chem = req.adr.get("chem") if req.adr else None
    return chem is not None and getattr(chem, "biofilm_code", None) is not None


def solve_batch(requests, device=0, graph_steps=20, quiet=False, mode="tiles", stats=None):
    """Solve every Request in one batch; Results in request order.  mode
    "tiles": the batch engine's persistent tile-list kernels; "streams":
    concurrent single-solve loops (StreamBatch).  A dict given as `stats`
    receives the batch's final statistics."""
    b = (StreamBatch(device=device, quiet=quiet) if mode == "streams"
         else Batch(device=device, graph_steps=graph_steps, quiet=quiet))
    try:
        results = [b.submit(r) for r in requests]
        b.run()
        if stats is not None:
            stats.update(b.stats())
        return results
    finally:
        b.close()
