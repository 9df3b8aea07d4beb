"""Transport parity on the GPU: solve_adr through libprtlb.so against the
reference's golden runs.  The bar is bit-identity: the reference integrates
in float32 with numpy and the CUDA step replays its operation order with no
fused multiply-add, and the stop rule's float32 means replay numpy's
pairwise summation, so steps, snapshots, t_norm and the on_progress records
must all be equal."""

import contextlib
import glob
import io
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from test_oracle_golden import adr_kwargs

pytestmark = pytest.mark.gpu

ADR32 = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "adr_*.npz")))


def run(z, name, **extra):
    from prtlb_gpu import solve_adr
    kw = adr_kwargs(z, name)
    kw.update(extra)
    info = {}
    prog = []
    with contextlib.redirect_stdout(io.StringIO()):
        out, tn = solve_adr(z["mat"], z["vel"], info=info,
                            on_progress=lambda *a: prog.append(a), **kw)
    return out, tn, info, np.asarray(prog, np.float64).reshape(-1, 4)


@pytest.mark.parametrize("name", ADR32)
def test_bit_identical_to_reference(name):
    z = load_golden(name)
    out, tn, info, prog = run(z, name)
    assert info["steps"] == int(z["info_steps"])
    assert info["ladder"] == int(z["info_ladder"])
    assert info["dt"] == float(z["info_dt"])
    assert info["converged"] == bool(z["info_converged"])
    assert info["repeated_snapshots"] == int(z["info_repeated_snapshots"])
    assert np.array_equal(tn, z["t_norm"])
    assert np.array_equal(prog, z["progress"])
    assert out.shape == z["out"].shape
    assert np.array_equal(out, z["out"]), float(np.abs(out - z["out"]).max())


def test_plug_flow_is_exp_minus_da():
    from prtlb_gpu import solve_adr
    for da in (0.5, 1.0, 2.0):
        g = np.full((80, 8), 2, np.uint8)
        v = np.zeros((3, 80, 8), np.float32)
        v[0] = 1.0
        with contextlib.redirect_stdout(io.StringIO()):
            out, _ = solve_adr(g, v, pe=4000.0, da=da, n_t=3, n_species=1)
        got = float(out[-1, 0, -1].mean())
        assert abs(got - np.exp(-da)) < 0.05, (da, got)
        assert out[-1].max() <= 1.0 + 1e-4
    g3 = np.full((40, 6, 6), 2, np.uint8)
    v3 = np.zeros((3, 40, 6, 6), np.float32)
    v3[0] = 1.0
    with contextlib.redirect_stdout(io.StringIO()):
        out3, _ = solve_adr(g3, v3, pe=4000.0, da=1.0, n_t=3, n_species=1)
    assert abs(float(out3[-1, 0, -1].mean()) - np.exp(-1.0)) < 0.06
    assert out3.max() <= 1.0 + 1e-4


def test_progress_callback_exception_propagates():
    from prtlb_gpu import solve_adr
    g = np.full((40, 8), 2, np.uint8)
    v = np.zeros((3, 40, 8), np.float32)
    v[0] = 1.0

    class Stop(Exception):
        pass

    def cb(*a):
        raise Stop()

    with pytest.raises(Stop):
        with contextlib.redirect_stdout(io.StringIO()):
            solve_adr(g, v, pe=30.0, da=1.0, n_t=3, n_species=1, on_progress=cb)
    # the context is usable afterwards
    with contextlib.redirect_stdout(io.StringIO()):
        out, _ = solve_adr(g, v, pe=30.0, da=1.0, n_t=3, n_species=1, steps=50)
    assert np.isfinite(out).all()


def test_buffers_kept_between_runs_hold_no_stale_values():
    """prt_adr_end keeps the transport buffers on the context for its next
    run.  Runs on one context, largest grid first, then smaller 3D and 2D
    grids with other porosities, match their golden runs bit for bit: every
    run initialises what it reads, so nothing of an earlier run leaks in
    (rock voxels included).  prt_adr_release then frees them and the
    context still works."""
    from prtlb_gpu import _lib, solve_adr
    names = sorted(ADR32, key=lambda n: -load_golden(n)["mat"].size)
    ctx = _lib.Context(0)
    try:
        for name in names[:4] + names[-2:]:
            z = load_golden(name)
            kw = adr_kwargs(z, name)
            with contextlib.redirect_stdout(io.StringIO()):
                out, tn = solve_adr(z["mat"], z["vel"], ctx=ctx, **kw)
            assert np.array_equal(out, z["out"]), name
            assert np.array_equal(tn, z["t_norm"]), name
        ctx.check(_lib.lib().prt_adr_release(ctx.handle))
        z = load_golden(names[0])
        with contextlib.redirect_stdout(io.StringIO()):
            out, _ = solve_adr(z["mat"], z["vel"], ctx=ctx, **adr_kwargs(z, names[0]))
        assert np.array_equal(out, z["out"])
    finally:
        ctx.close()


@pytest.mark.parametrize("pdl,late", [("0", ""), ("1", ""), ("1", "all"), ("1", "none")])
def test_transport_with_and_without_programmatic_launch(monkeypatch, pdl, late):
    """The transport step goes out with programmatic dependent launch by
    default (its voxel index, flags and face velocities are read while the
    previous step drains) or plainly (PRT_PDL=0), letting the next step in at
    its start or after its stores (PRT_PDL_LATE=none / all; by default after
    the stores when its grid is one wave); every way matches the reference's
    golden runs bit for bit."""
    monkeypatch.setenv("PRT_PDL", pdl)
    monkeypatch.setenv("PRT_PDL_LATE", late)
    for name in ("adr_spheres3d_biofilm", "adr_spheres3d_ns4", "adr_disks2d_first",
                 "adr_chan2d_capped"):
        z = load_golden(name)
        out, tn, info, prog = run(z, name)
        assert np.array_equal(tn, z["t_norm"]), name
        assert np.array_equal(prog, z["progress"]), name
        assert np.array_equal(out, z["out"]), (name, float(np.abs(out - z["out"]).max()))


def test_cached_loop_graph_follows_every_change():
    """A transport solve replays the previous solve's loop graph when nothing
    the graph holds has changed.  Alternating solves on one context that
    differ in grid, chemistry, Peclet number, step count and chemicals --
    A, B, C, A, B, C, then A again after a PRT_PDL flip -- each match their
    golden runs bit for bit."""
    import os
    from prtlb_gpu import _lib, solve_adr
    names = ["adr_spheres3d_monod", "adr_spheres3d_ns4", "adr_disks2d_first"]
    ctx = _lib.Context(0)
    try:
        for rep in range(2):
            for name in names:
                z = load_golden(name)
                with contextlib.redirect_stdout(io.StringIO()):
                    out, tn = solve_adr(z["mat"], z["vel"], ctx=ctx, **adr_kwargs(z, name))
                assert np.array_equal(out, z["out"]) and np.array_equal(tn, z["t_norm"]), name
        z = load_golden(names[0])
        kw = adr_kwargs(z, names[0])
        for pdl in ("0", "1"):
            os.environ["PRT_PDL"] = pdl
            try:
                with contextlib.redirect_stdout(io.StringIO()):
                    out, tn = solve_adr(z["mat"], z["vel"], ctx=ctx, **kw)
            finally:
                os.environ.pop("PRT_PDL", None)
            assert np.array_equal(out, z["out"])
        kw2 = dict(kw, steps=kw["steps"] // 2)
        with contextlib.redirect_stdout(io.StringIO()):
            half, _ = solve_adr(z["mat"], z["vel"], ctx=ctx, **kw2)
            full, _ = solve_adr(z["mat"], z["vel"], ctx=ctx, **kw)
        assert np.array_equal(full, z["out"]) and not np.array_equal(half, full)
    finally:
        ctx.close()
