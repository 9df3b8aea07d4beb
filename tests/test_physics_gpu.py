"""check_physics with its statistics reduced on the GPU (on_gpu=True) must
give the host's complaints, word for word, and the exact extremes, counts and
plane maxima numpy finds, on randomised results (non-finite values, negative
and runaway values, vanished chemicals, rescaled copies, wrap-around
signatures, empty pore) and on a real transport solve."""

import contextlib
import ctypes
import io
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases(n):
    from prtlb_gpu.chemistry import default_chemistry
    rng = np.random.default_rng(1)
    for trial in range(n):
        shape = ((int(rng.integers(4, 30)), int(rng.integers(1, 9)), int(rng.integers(2, 9)))
                 if trial % 2 else (int(rng.integers(4, 40)), int(rng.integers(2, 12))))
        g = np.where(rng.random(shape) < 0.7, 2, 0).astype(np.uint8)
        if trial % 7 == 0:
            g[:] = 0
        chem = default_chemistry() if trial % 3 == 0 else None
        ns = len(chem.names) if chem is not None else int(rng.integers(1, 5))
        nt = int(rng.integers(1, 6))
        out = (rng.random((nt, ns) + shape) * rng.choice([0.5, 1.0, 3.0, 2000.0])).astype(np.float32)
        if trial % 5 == 0:
            out[..., ::2] *= -0.1
        if trial % 9 == 0:
            out[0, 0].flat[0] = np.nan
        if trial % 11 == 0:
            out[-1, -1].flat[-1] = np.inf
        if trial % 4 == 0 and ns > 1:
            out[:, 1] = 2.0 * out[:, 0]
        if trial % 6 == 0:
            out[:, :, shape[0] // 2] = 0
        if trial % 8 == 0:
            out[-1] = 0
        if trial % 10 == 0:  # a checkerboard along x
            out[-1, 0] = np.where(np.arange(shape[0]) % 2 == 0, 1.0, 0.2).reshape(
                (-1,) + (1,) * (len(shape) - 1)) * np.ones(shape, np.float32)
        yield g, out, chem


def test_device_statistics_give_the_host_complaints():
    from prtlb_gpu.physics import check_physics
    n = 0
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        for g, out, chem in _cases(80):
            host = check_physics(out, g, chem=chem, da=1.0, da_abio=0.5)
            dev = check_physics(out, g, chem=chem, da=1.0, da_abio=0.5, on_gpu=True)
            assert dev == host, (host, dev)
            n += bool(host)
    assert n > 40  # most cases carry complaints, of every kind


def test_device_extremes_and_counts_are_exact():
    from prtlb_gpu import _lib
    from prtlb_gpu.physics import _DeviceStats
    ctx = _lib.default_context()
    for g, out, _ in _cases(30):
        m = g == 2
        st = _DeviceStats(out, g, ctx)
        assert st.n_nan == int(np.isnan(out).sum()) and st.n_inf == int(np.isinf(out).sum())
        if not st.finite or not m.any():
            continue
        for j in range(out.shape[1]):
            assert st.hi[j] == float(out[:, j][:, m].max())
            assert st.lo[j] == float(out[:, j][:, m].min())
            assert st.final_absmax[j] == float(np.abs(out[-1, j][m]).max())
        nx = g.shape[0]
        assert np.array_equal(st.mid, out[:, 0, nx // 2].reshape(out.shape[0], -1).max(1))
        assert np.array_equal(st.end, out[:, 0, nx - 1].reshape(out.shape[0], -1).max(1))


def test_on_a_transport_solve():
    from prtlb_gpu import sphere_pack_3d, stokes_d3q19, solve_adr, default_chemistry
    from prtlb_gpu.physics import check_physics
    g = sphere_pack_3d(24, 0.45, 2)
    chem = default_chemistry()
    with contextlib.redirect_stdout(io.StringIO()):
        v = stokes_d3q19(g, nit=400, tol=0.0)
        out, _ = solve_adr(g, v, pe=10.0, da=1.0, n_t=5, n_species=len(chem.names), chem=chem,
                           steps=1500)
    assert check_physics(out, g, chem=chem, da=1.0, on_gpu=True) == \
        check_physics(out, g, chem=chem, da=1.0)


def test_nothing_staged_is_refused():
    from prtlb_gpu import _lib
    ctx = _lib.Context(0)
    try:
        st = _lib.PhysicsStats()
        dims = (ctypes.c_int32 * 3)(4, 4, 4)
        rc = _lib.lib().prt_physics_stats_dev(ctx.handle, None, None, 3, dims, 1, 1, 2,
                                              ctypes.byref(st))
        assert rc == _lib.PRT_E_STATE
    finally:
        ctx.close()
