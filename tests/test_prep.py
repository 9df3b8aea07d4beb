"""The geometry-preparation walk: keep_inlet_connected, geodesic_steps,
distance_column and the practice-dataset geodesic.

The oracle (oracle/prep_oracle.py) is pinned bit for bit to golden runs of the
reference itself (tests/golden/make_golden_prep.py); the GPU walk
(prt_inlet_walk through prtlb_gpu.prep) must then equal both, bit for bit,
on the golden grids, on larger seeded grids near the percolation threshold
(many components, long tortuous paths, walks of hundreds of levels), on
every inlet axis, and on the edge cases (no pore, no pore on the inlet face,
a cut channel)."""

import glob
import os
import warnings

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

PREP = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "prep_*.npz")))
CONVENTIONS = ("ours", "published", "published_pore")


def _same(a, b):
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("name", PREP)
def test_oracle_matches_reference(name):
    from oracle import prep_oracle as O
    z = load_golden(name)
    g = z["mat"]
    kept, n = O.keep_inlet_connected(g.copy())
    assert np.array_equal(kept, z["kept"]) and n == int(z["n_removed"])
    for ax in range(g.ndim):
        for seed in (0.0, 0.5):
            assert _same(O.geodesic_steps(g == 2, ax, seed), z["steps_a%d_s%g" % (ax, seed)])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        for c in CONVENTIONS:
            assert _same(O.distance_column(g, c, 0), z["column_" + c]), c
    if "geodesic" in z:
        assert _same(O.geodesic_relaxed(kept), z["geodesic"])
    if "geodesic_2d" in z:
        assert _same(O.geodesic_relaxed(kept), z["geodesic_2d"])
    assert O.percolates(g) == bool(z["percolates"])
    for k, (xi, xo) in enumerate(_planes(g)):
        assert O.percolates_between(g == 2, xi, xo) == bool(z["perc_between_%d" % k])
        ks, r = O.keep_percolating_cluster(g != 2, xi, xo)
        assert np.array_equal(ks, z["keep_perc_%d" % k]) and r == int(z["keep_perc_removed_%d" % k])


def _planes(g):
    """The plane pairs the golden runs use (3D grids only)."""
    if g.ndim != 3:
        return []
    nx = g.shape[0]
    return [(0, nx - 1), (2, nx - 3), (nx // 2, nx // 2)]


@pytest.mark.gpu
@pytest.mark.parametrize("name", PREP)
def test_gpu_walk_matches_reference(name):
    from prtlb_gpu import prep
    z = load_golden(name)
    g = z["mat"]
    kept, n = prep.keep_inlet_connected(g.copy())
    assert np.array_equal(kept, z["kept"]) and n == int(z["n_removed"])
    for ax in range(g.ndim):
        for seed in (0.0, 0.5):
            assert _same(prep.geodesic_steps(g == 2, ax, seed), z["steps_a%d_s%g" % (ax, seed)])
    for c in CONVENTIONS:
        assert _same(prep.distance_column(g, c, 0), z["column_" + c]), c
    if "geodesic" in z:
        assert _same(prep.geodesic(kept), z["geodesic"])
    if "geodesic_2d" in z:
        assert _same(prep.geodesic_2d(kept), z["geodesic_2d"])
    assert prep.percolates(g) == bool(z["percolates"])
    for k, (xi, xo) in enumerate(_planes(g)):
        assert prep.percolates_between(g == 2, xi, xo) == bool(z["perc_between_%d" % k])
        ks, r = prep.keep_percolating_cluster(g != 2, xi, xo)
        assert np.array_equal(ks, z["keep_perc_%d" % k]) and r == int(z["keep_perc_removed_%d" % k])


def _site(shape, p, seed):
    rng = np.random.default_rng(seed)
    g = np.where(rng.random(shape) < p, 2, 0).astype(np.uint8)
    g[rng.random(shape) < 0.02] = 1
    return g


def _serpentine(n, width=1):
    """A 2D channel that sweeps the whole grid: a walk of about n^2 / 2 steps."""
    g = np.zeros((n, n), np.uint8)
    for x in range(0, n, 2 * (width + 1)):
        g[x:x + width, 1:n - 1] = 2
        if x + width < n:
            end = n - 2 if (x // (2 * (width + 1))) % 2 == 0 else 1
            g[x:min(x + 2 * (width + 1), n), end] = 2
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["site3d", "site2d", "pack3d", "serpentine2d", "slab3d"])
def test_gpu_walk_matches_oracle(case):
    from oracle import prep_oracle as O
    from prtlb_gpu import prep
    from prtlb_gpu.geometry import sphere_pack_3d
    if case == "site3d":
        g = _site((40, 32, 28), 0.34, 1)
    elif case == "site2d":
        g = _site((200, 150), 0.62, 2)
    elif case == "pack3d":
        g = sphere_pack_3d(48, 0.45, 3)
    elif case == "serpentine2d":
        g = _serpentine(64)
    else:  # thin slab: one pore layer in the middle of y
        g = np.zeros((30, 7, 20), np.uint8)
        g[:, 3, :] = 2
        g[10, 3, 5:] = 0
    pore = g == 2
    steps, n_reached, n_pore = prep.inlet_walk(g)
    ref = O.geodesic_steps(pore, 0, 0.0)
    assert n_pore == int(pore.sum())
    assert n_reached == int(np.isfinite(ref).sum())
    assert np.array_equal(np.where(np.isfinite(ref), ref, -2).astype(np.int64)[pore],
                          steps[pore].astype(np.int64))
    assert (steps[~pore] == -1).all()
    for ax in range(g.ndim):
        assert _same(prep.geodesic_steps(pore, ax, 0.5), O.geodesic_steps(pore, ax, 0.5))
    kept, n = prep.keep_inlet_connected(g)
    kept_o, n_o = O.keep_inlet_connected(g)
    assert np.array_equal(kept, kept_o) and n == n_o
    assert prep.percolates(g) == O.percolates(g)
    nx = g.shape[0]
    for xi, xo in ((0, nx - 1), (1, -2), (nx // 3, 2 * nx // 3), (nx - 1, 0)):
        assert prep.percolates_between(pore, xi, xo) == O.percolates_between(pore, xi, xo)
        ks, r = prep.keep_percolating_cluster(~pore, xi, xo)
        ks_o, r_o = O.keep_percolating_cluster(~pore, xi, xo)
        assert np.array_equal(ks, ks_o) and r == r_o
    if case == "serpentine2d":
        assert np.nanmax(ref) > 900  # about 30 chunks of levels


@pytest.mark.gpu
def test_gpu_walk_edges_and_refusals():
    from prtlb_gpu import prep, PrtError
    one = np.full((1, 1, 1), 2, np.uint8)
    steps, nr, npore = prep.inlet_walk(one)
    assert steps.tolist() == [[[0]]] and nr == 1 and npore == 1
    solid = np.zeros((5, 4, 3), np.uint8)
    assert prep.keep_inlet_connected(solid)[1] == 0
    assert np.isnan(prep.geodesic_steps(solid == 2)).all()
    with pytest.raises(ValueError):
        prep.inlet_walk(np.zeros((4, 4, 4, 4), np.uint8))
    with pytest.raises(ValueError):
        prep.inlet_walk(solid, inlet_axis=3)
    with pytest.raises(ValueError):
        prep.distance_column(solid, "backwards")
    from prtlb_gpu import _lib
    import ctypes
    ctx = _lib.default_context()
    dims = (ctypes.c_int32 * 3)(4, 0, 4)
    out = np.empty(16, np.int32)
    rc = _lib.lib().prt_inlet_walk(ctx.handle, solid.ctypes.data_as(ctypes.c_void_p), 3, dims, 2,
                                   0, out.ctypes.data_as(ctypes.c_void_p), None, None)
    assert rc == _lib.PRT_E_INVALID
    assert PrtError  # the module's error type is what ctx.check raises


def test_argument_checks_need_no_gpu():
    """The wrappers refuse bad shapes, axes, planes and conventions before
    any device call, with the reference's error types."""
    from prtlb_gpu import prep
    g = np.zeros((4, 3, 2), np.uint8)
    with pytest.raises(ValueError):
        prep.inlet_walk(np.zeros((2, 2, 2, 2), np.uint8))
    with pytest.raises(ValueError):
        prep.inlet_walk(g, inlet_axis=3)
    with pytest.raises(IndexError):
        prep.walk_from_plane(g, 2, 0, 4)
    with pytest.raises(ValueError):
        prep.distance_column(g, "reversed")
    with pytest.raises(ValueError):
        prep.geodesic(np.zeros((4, 4), np.uint8))
    with pytest.raises(ValueError):
        prep.geodesic_2d(g)
    assert prep.pore_mask(np.array([[0, 1]], np.uint8)).tolist() == [[False, True]]
    assert prep.pore_mask(np.array([[0, 2, 1]], np.uint8)).tolist() == [[False, True, False]]
    s = prep._seeded(0.1, 3)
    assert s.dtype == np.float32 and s[3] == ((np.float32(0.1) + np.float32(1)) + np.float32(1)) + \
        np.float32(1)


LABEL = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "label_*.npz")))


@pytest.mark.parametrize("name", LABEL)
def test_label_materials_oracle_matches_reference(name):
    from oracle import prep_oracle as O
    z = load_golden(name)
    assert _same(O.label_materials(z["solid"]), z["materials"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", LABEL)
def test_label_materials_gpu_matches_reference(name):
    from prtlb_gpu import prep
    z = load_golden(name)
    assert _same(prep.label_materials(z["solid"]), z["materials"])


@pytest.mark.gpu
def test_label_materials_gpu_matches_oracle_on_larger_grids():
    """2D and 3D, sparse and dense solids, odd sizes (block tails)."""
    from oracle import prep_oracle as O
    from prtlb_gpu import prep
    rng = np.random.default_rng(5)
    for shape, p in (((97, 64, 33), 0.5), ((64, 64, 64), 0.85), ((130, 77), 0.4),
                     ((1, 1, 5), 0.5), ((3, 200), 0.7)):
        solid = rng.random(shape) < p
        assert _same(prep.label_materials(solid), O.label_materials(solid)), shape
