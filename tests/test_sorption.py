"""Reversible sorption (no counterpart in the reference, so no golden run):
pinned by its own known answers, first on the oracle (CPU), then the GPU
path against the oracle.

  (i)   a closed, well-mixed batch relaxes to S / C = K_d
  (ii)  C + S is conserved in a closed box (float32: to rounding)
  (iii) with fast exchange a plug-flow front is retarded by R = 1 + K_d
"""

import contextlib
import io

import numpy as np
import pytest

from oracle import prtlb_oracle as O

KD = 0.5


def _closed_chem(kd=KD, da=2.0):
    from prtlb_gpu.chemistry import Chemistry, Sorption
    return Chemistry(names=["C", "S"], inlet=[np.nan, np.nan], c_init=[1.0, 0.0],
                     d_rel=[1.0, 0.0], immobile=[False, True], biotic_on=False,
                     source="closed batch", sorption=Sorption(0, 1, kd=kd, da=da))


def _front_chem(sorbing, kd=KD, da=400.0):
    from prtlb_gpu.chemistry import Chemistry, Sorption
    return Chemistry(names=["C", "S"], inlet=[1.0, np.nan], c_init=[0.0, 0.0],
                     d_rel=[1.0, 0.0], immobile=[False, True], biotic_on=False,
                     source="front",
                     sorption=Sorption(0, 1, kd=kd, da=da) if sorbing else None)


def _closed_box():
    from prtlb_gpu import random_pack
    g = random_pack((28, 20), 0.6, 2.0, 4.0, seed=3)
    v = np.zeros((3,) + g.shape, np.float32)
    return g, v


def _channel():
    g = np.full((160, 6), 2, np.uint8)
    v = np.zeros((3,) + g.shape, np.float32)
    v[0] = 1.0
    return g, v


def _run(fn, g, v, chem, steps, pe):
    info = {}
    with contextlib.redirect_stdout(io.StringIO()):
        out, tn = fn(g, v, pe=pe, da=1.0, n_t=2, n_species=2, steps=steps, chem=chem, info=info)
    return out, tn, info


def _oracle(dtype):
    def fn(*a, **k):
        return O.solve_adr(*a, dtype=dtype, **k)
    return fn


def _front_speed(out, info, steps):
    c = out[-1, 0].astype(np.float64).mean(axis=1)  # mean over the channel width
    x = int(np.argmax(c < 0.5))  # first cell below one half
    # linear interpolation of the 0.5 crossing between x-1 and x
    xf = (x - 1) + (c[x - 1] - 0.5) / (c[x - 1] - c[x])
    return xf / (steps * info["dt"])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_oracle_closed_batch_reaches_kd_and_conserves(dtype):
    g, v = _closed_box()
    out, tn, info = _run(_oracle(dtype), g, v, _closed_chem(), 200, 1000.0)
    m = g == 2
    C, S = out[-1, 0][m].astype(np.float64), out[-1, 1][m].astype(np.float64)
    tol = 2e-6 if dtype == np.float32 else 1e-12
    assert np.abs(C + S - 1.0).max() < tol
    assert np.abs(S / C - KD).max() < 1e-4
    assert abs(C.mean() - 1.0 / (1.0 + KD)) < 1e-4


def _retardation(fn):
    """Front speed without sorption / with it, both fronts mid-channel: the
    sorbing run takes 900 steps, the tracer run as many of its (larger)
    steps as cover the same time."""
    g, v = _channel()
    o2, _, i2 = _run(fn, g, v, _front_chem(True), 900, 2000.0)
    _, _, i0 = _run(fn, g, v, _front_chem(False), 1, 2000.0)
    n1 = int(round(900 * i2["dt"] / i0["dt"]))
    o1, _, i1 = _run(fn, g, v, _front_chem(False), n1, 2000.0)
    return _front_speed(o1, i1, n1) / _front_speed(o2, i2, 900), o2


def test_oracle_front_is_retarded_by_one_plus_kd():
    r, _ = _retardation(_oracle(np.float32))
    assert abs(r - (1.0 + KD)) < 0.06 * (1.0 + KD), r


@pytest.mark.gpu
def test_gpu_closed_batch_matches_oracle_and_known_answers():
    from prtlb_gpu import solve_adr
    g, v = _closed_box()
    out, tn, info = _run(solve_adr, g, v, _closed_chem(), 200, 1000.0)
    ref, rtn, rinfo = _run(_oracle(np.float32), g, v, _closed_chem(), 200, 1000.0)
    assert info["dt"] == rinfo["dt"]
    assert np.array_equal(tn, rtn)
    assert np.array_equal(out, ref), float(np.abs(out - ref).max())
    m = g == 2
    C, S = out[-1, 0][m].astype(np.float64), out[-1, 1][m].astype(np.float64)
    assert np.abs(C + S - 1.0).max() < 2e-6
    assert np.abs(S / C - KD).max() < 1e-4


@pytest.mark.gpu
def test_gpu_front_matches_oracle_and_is_retarded():
    from prtlb_gpu import solve_adr
    g, v = _channel()
    r, o2 = _retardation(solve_adr)
    r2, _, _ = _run(_oracle(np.float32), g, v, _front_chem(True), 900, 2000.0)
    assert np.array_equal(o2, r2), float(np.abs(o2 - r2).max())
    assert abs(r - (1.0 + KD)) < 0.06 * (1.0 + KD), r


@pytest.mark.gpu
def test_gpu_sorption_in_a_porous_flow_matches_oracle():
    """Sorption with flow, inlet feed and a porous geometry: bit-identical to
    the oracle, steps and snapshots included."""
    from prtlb_gpu import random_pack, solve_adr, stokes_d2q9
    from prtlb_gpu.chemistry import reversible_sorption_chemistry
    g = random_pack((48, 24), 0.6, 2.0, 4.0, seed=8)
    with contextlib.redirect_stdout(io.StringIO()):
        v = stokes_d2q9(g, nit=1500, force=1e-6, tol=0.0, precision="fp32")
    chem = reversible_sorption_chemistry(KD, 3.0)
    out, tn, info = _run(solve_adr, g, v, chem, 700, 10.0)
    ref, rtn, rinfo = _run(_oracle(np.float32), g, v, chem, 700, 10.0)
    assert info["dt"] == rinfo["dt"]
    assert np.array_equal(tn, rtn)
    assert np.array_equal(out, ref), float(np.abs(out - ref).max())


@pytest.mark.gpu
def test_gpu_float32_transport_against_float64_twin():
    """The transport is float32 like the reference; its distance from the
    same algorithm in float64 (the oracle's twin) on a 3D pack with flow and
    sorption stays at float32 rounding level."""
    from prtlb_gpu import solve_adr, sphere_pack_3d, stokes_d3q19
    from prtlb_gpu.chemistry import reversible_sorption_chemistry
    g = sphere_pack_3d(24, 0.45, 0)
    with contextlib.redirect_stdout(io.StringIO()):
        v = stokes_d3q19(g, nit=2000, tol=0.0, precision="fp64")
    chem = reversible_sorption_chemistry(KD, 1.0)
    c32, _, _ = _run(solve_adr, g, v, chem, 600, 10.0)
    c64, _, _ = _run(_oracle(np.float64), g, v, chem, 600, 10.0)
    d = c32.astype(np.float64) - c64
    rel = float(np.sqrt((d ** 2).sum() / (c64 ** 2).sum()))
    assert rel < 1e-5, rel
