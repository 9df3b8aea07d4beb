"""The served loop: admission arithmetic on the host (CPU) and, on the GPU,
a small Poisson stream whose every result must equal the same solve run
alone through the single-solve calls (continuous batching changes when a
solve runs, never what it computes)."""

import contextlib
import io

import numpy as np
import pytest


def test_ladder_slots_follow_the_ratio_schedule():
    from prtlb_gpu.serve import ladder_slots
    assert ladder_slots(0, 1.12) == 2
    assert ladder_slots(1, 1.12) == 3
    # n = 1, 2, ..., 9 then ceil(1.12 n) grows faster than n + 1
    sched, n = [], 1
    while n <= 100000:
        sched.append(n)
        n = max(n + 1, int(np.ceil(n * 1.12)))
    assert ladder_slots(100000, 1.12) == len(sched) + 2


def test_footprint_grows_with_size_and_ladder():
    from prtlb_gpu.batch import Request
    from prtlb_gpu.serve import footprint
    g1 = np.full((16, 16, 16), 2, np.uint8)
    g2 = np.full((32, 32, 32), 2, np.uint8)
    a = dict(pe=1.0, da=1.0, n_t=3, n_species=1)
    r1 = Request(g1, adr=dict(a, max_steps=1000))
    r2 = Request(g2, adr=dict(a, max_steps=1000))
    r3 = Request(g2, adr=dict(a, max_steps=100000))
    assert footprint(r1) < footprint(r2) < footprint(r3)
    # the transport ladder dominates a long run: ~4 bytes x voxels x slots
    assert footprint(r3) > 4 * g2.size * 100


def test_poisson_arrivals_are_seeded_and_increasing():
    from prtlb_gpu.serve import poisson_arrivals
    a = poisson_arrivals(50, 20.0, seed=3)
    assert np.all(np.diff(a) > 0) and np.array_equal(a, poisson_arrivals(50, 20.0, seed=3))
    assert 1.0 < a[-1] < 6.0  # about 50 / 20 s


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["streams", "tiles"])
def test_served_results_equal_single_solves(mode):
    from prtlb_gpu import solve_adr, stokes_d3q19
    from prtlb_gpu.serve import poisson_arrivals, serve
    from prtlb_gpu.workloads import request_set
    reqs, draws = request_set(6, 14, 26, seed=5, nit=400, max_steps=1500, n_t=3)
    arrivals = poisson_arrivals(len(reqs), 40.0, seed=5)
    srv = serve(reqs, arrivals, graph_steps=9, mode=mode)
    assert srv.summary["completed"] == len(reqs)
    assert srv.summary["latency_p99_s"] >= srv.summary["latency_p50_s"] > 0
    by = {r.tag: r for r in srv.results}
    for i, q in enumerate(reqs):
        f = dict(q.flow)
        prec = f.pop("precision")
        a = dict(q.adr)
        with contextlib.redirect_stdout(io.StringIO()):
            v = stokes_d3q19(q.mat, precision=prec, **f)
            out, tn = solve_adr(q.mat, v, a.pop("pe"), a.pop("da"), a.pop("n_t"), **a)
        assert by[i].error is None
        assert np.array_equal(by[i].out, out), i
        assert np.array_equal(by[i].t_norm, tn), i


@pytest.mark.gpu
def test_admission_budget_serialises_when_tight():
    """With a budget that holds one request at a time, the loop still
    finishes everything, one solve after the other."""
    from prtlb_gpu.serve import footprint, poisson_arrivals, serve
    from prtlb_gpu.workloads import request_set
    reqs, _ = request_set(3, 12, 16, seed=9, nit=200, max_steps=300, n_t=2)
    budget = max(footprint(r) for r in reqs) + 1
    srv = serve(reqs, poisson_arrivals(3, 100.0, seed=1), budget_bytes=budget, graph_steps=5)
    assert srv.summary["completed"] == 3
    adm = sorted(r.t_admit for r in srv.results)
    done = sorted(r.t_done for r in srv.results)
    assert adm[1] >= done[0] - 1e-6 and adm[2] >= done[1] - 1e-6


@pytest.mark.gpu
def test_flow_cap_admits_the_next_flow_after_the_previous_one():
    """With a flow cap of one voxel, a request is admitted only once the
    previous request's flow phase has finished (its transport may still run)."""
    from prtlb_gpu.serve import poisson_arrivals, serve
    from prtlb_gpu.workloads import request_set
    reqs, _ = request_set(3, 14, 18, seed=11, nit=300, max_steps=400, n_t=2)
    srv = serve(reqs, poisson_arrivals(3, 200.0, seed=2), graph_steps=7, flow_cap=1)
    assert srv.summary["completed"] == 3
    rs = sorted(srv.results, key=lambda r: r.t_admit)
    assert rs[1].t_admit >= rs[0].t_flow - 1e-6
    assert rs[2].t_admit >= rs[1].t_flow - 1e-6
