"""Batched solves on the GPU: every solve of a batch must give exactly what
the single-solve calls (stokes_d3q19 / stokes_d2q9, then solve_adr) give on
the same arguments -- the same velocity field bit for bit, the same flow
iteration count and convergence record, the same transport steps,
snapshots and t_norm -- alone in a batch, mixed with other solves, joining
a batch that is already running, and under every tiling of the work list."""

import contextlib
import io

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pack3(shape, phi, seed):
    from prtlb_gpu import random_pack
    return random_pack(shape, phi, 2.0, 3.5, seed=seed)


def _pack2(shape, phi, seed):
    from prtlb_gpu import random_pack
    return random_pack(shape, phi, 2.0, 4.0, seed=seed)


def _requests():
    """Mixed lattices, precisions, kinetics, fixed-step and stop-rule runs."""
    from prtlb_gpu import (first_order_chemistry, monod_chemistry,
                           reversible_sorption_chemistry)
    from prtlb_gpu.batch import Request
    R = []
    R.append(Request(_pack3((20, 14, 14), 0.5, 1),
                     flow=dict(nit=700, tol=1e-6, precision="fp32"),
                     adr=dict(pe=10.0, da=1.0, n_t=4, n_species=1, chem=monod_chemistry(0.5),
                              max_steps=2500), tag="monod3"))
    R.append(Request(_pack3((16, 12, 18), 0.45, 2),
                     flow=dict(nit=550, tol=1e-6, precision="fp64"),
                     adr=dict(pe=3.0, da=0.3, n_t=3, n_species=1, chem=first_order_chemistry(),
                              steps=420), tag="first3"))
    # the same class as monod3 with other constants: its flow launches read
    # them per job instead of as one shared parameter
    R.append(Request(_pack3((24, 10, 12), 0.55, 3),
                     flow=dict(nit=800, tol=0.0, precision="fp32", tau_lb=0.9),
                     adr=dict(pe=30.0, da=2.0, n_t=5, n_species=2,
                              chem=reversible_sorption_chemistry(0.5, 2.0), max_steps=1800),
                     tag="sorb3"))
    R.append(Request(_pack2((48, 32), 0.6, 4),
                     flow=dict(nit=1000, tol=1e-7, precision="fp32"),
                     adr=dict(pe=10.0, da=1.0, n_t=4, n_species=4, max_steps=2000),
                     tag="dual2"))
    R.append(Request(_pack3((18, 16, 16), 0.5, 5),
                     flow=dict(nit=333, tol=1e-6, precision="fp16"), tag="flowonly3",
                     keep_velocity=True))
    return R


def _single(req):
    """The same solve through the drop-in single-solve API."""
    from prtlb_gpu import solve_adr, stokes_d2q9, stokes_d3q19
    f = dict(req.flow)
    prec = f.pop("precision")
    fn = stokes_d3q19 if req.mat.ndim == 3 else stokes_d2q9
    finfo = {}
    with contextlib.redirect_stdout(io.StringIO()):
        vel = fn(req.mat, info=finfo, precision=prec, **f)
    out = tn = ainfo = None
    if req.adr is not None:
        a = dict(req.adr)
        ainfo = {}
        with contextlib.redirect_stdout(io.StringIO()):
            out, tn = solve_adr(req.mat, vel, a.pop("pe"), a.pop("da"), a.pop("n_t"),
                                info=ainfo, **a)
    return vel, finfo, out, tn, ainfo


def _same(res, ref, req):
    vel, finfo, out, tn, ainfo = ref
    assert res.error is None, res.error
    for k in ("flow_iters", "flow_converged", "flow_change", "permeability", "flow_mass"):
        assert res.flow_info[k] == finfo[k], (req.tag, k, res.flow_info[k], finfo[k])
    if req.keep_velocity:
        assert np.array_equal(res.vel, vel), req.tag
    if req.adr is not None:
        assert res.adr_info["steps"] == ainfo["steps"], req.tag
        assert res.adr_info["dt"] == ainfo["dt"]
        assert res.adr_info["ladder"] == ainfo["ladder"]
        assert res.adr_info["converged"] == ainfo["converged"]
        assert np.array_equal(res.t_norm, tn), req.tag
        assert np.array_equal(res.out, out), (req.tag, float(np.abs(res.out - out).max()))


@pytest.fixture(scope="module")
def singles():
    reqs = _requests()
    for r in reqs:
        r.keep_velocity = True
    return reqs, [_single(r) for r in reqs]


def _batch(reqs, graph_steps=20, tiling=None, stagger=0, mode="tiles"):
    from prtlb_gpu.batch import Batch, StreamBatch
    b = StreamBatch(quiet=True) if mode == "streams" else Batch(graph_steps=graph_steps, quiet=True)
    try:
        if tiling:
            b.tune(*tiling)
        res = []
        for i, r in enumerate(reqs):
            res.append(b.submit(r))
            if stagger:
                b.advance(stagger)  # later solves join a running batch
        b.run()
        return res, b.stats()
    finally:
        b.close()


def test_batch_equals_single_solves(singles):
    reqs, refs = singles
    res, st = _batch(reqs)
    for r, q, ref in zip(res, reqs, refs):
        _same(r, ref, q)
    assert st["launches"] > 0


@pytest.mark.parametrize("tiling", [(1, 0), (1, 1), (2, 1), (4, 0), (1, 2)])
def test_every_tiling_gives_the_same_results(singles, tiling):
    reqs, refs = singles
    res, st = _batch(reqs, tiling=tiling)
    assert (st["tile_blocks"], st["grid_mult"]) == tiling
    for r, q, ref in zip(res, reqs, refs):
        _same(r, ref, q)


def test_alone_and_in_the_mix_are_identical(singles):
    reqs, refs = singles
    # each solve alone in a batch
    for q, ref in zip(reqs, refs):
        res, _ = _batch([q], graph_steps=7)
        _same(res[0], ref, q)
    # all of them, joining one by one while the batch runs (continuous batching)
    res, _ = _batch(list(reversed(reqs)), graph_steps=13, stagger=40)
    for r, q, ref in zip(res, list(reversed(reqs)), list(reversed(refs))):
        _same(r, ref, q)


def test_dead_flow_fails_alone():
    """A solve whose pore space is empty ends with the reference's SystemExit
    and leaves the other solves untouched."""
    from prtlb_gpu.batch import Request
    reqs, _ = _requests(), None
    good = reqs[1]
    good.keep_velocity = True
    dead = Request(np.zeros((12, 10, 10), np.uint8), flow=dict(nit=200), tag="dead",
                   adr=dict(pe=1.0, da=1.0, n_t=2))
    res, _ = _batch([dead, good])
    assert isinstance(res[0].error, SystemExit)
    _same(res[1], _single(good), good)


def test_graphs_off_matches(singles, monkeypatch):
    reqs, refs = singles
    monkeypatch.setenv("PRT_GRAPHS", "0")
    res, _ = _batch(reqs[:2])
    for r, q, ref in zip(res, reqs[:2], refs[:2]):
        _same(r, ref, q)


def test_concurrent_streams_equal_single_solves(singles):
    """The same solves as concurrent single-solve loops, one stream each,
    some joining while others run."""
    reqs, refs = singles
    res, st = _batch(reqs, mode="streams", stagger=1)
    for r, q, ref in zip(res, reqs, refs):
        _same(r, ref, q)
    assert st["launches"] >= 2 * sum(1 for q in reqs if q.adr is not None)


def test_moving_between_batches_keeps_the_counts(singles):
    """Solves that leave a batch part-way (prt_batch_remove) and finish in
    another: one in its flow loop, one in its transport loop.  The batch
    keeps step counts on the device and writes a job's count to its control
    block only on check steps, so leaving writes the count back; the results
    must still equal the single solves."""
    from prtlb_gpu import _lib
    from prtlb_gpu.batch import Batch
    reqs, refs = singles
    moved = [(reqs[0], refs[0]), (reqs[2], refs[2])]
    L = _lib.lib()
    a = Batch(graph_steps=7, quiet=True)
    b = Batch(graph_steps=11, quiet=True)
    try:
        res = [a.submit(q) for q, _ in moved]
        jobs = list(a._jobs.values())

        def move(job):
            assert L.prt_batch_remove(a.handle, job.ctx.handle) == _lib.PRT_OK
            del a._jobs[job.ctx.handle.value]
            b._jobs[job.ctx.handle.value] = job
            assert L.prt_batch_add(b.handle, job.ctx.handle) == _lib.PRT_OK

        # the first leaves during its flow loop (cap 700 iterations)
        a.advance(70)
        assert jobs[0].phase == "flow"
        move(jobs[0])
        # the second once its transport loop has run a while
        while jobs[1].phase == "flow":
            a.advance()
        a.advance(30)
        assert jobs[1].phase == "adr"
        move(jobs[1])
        b.run()
        for r, (q, ref) in zip(res, moved):
            _same(r, ref, q)
    finally:
        a.close()
        b.close()
