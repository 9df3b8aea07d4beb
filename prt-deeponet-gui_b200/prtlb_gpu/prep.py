"""Geometry preparation on the GPU: the walk from the inlet face.

One breadth-first walk through the pore space (libprtlb's prt_inlet_walk)
serves the reference's per-rock preparation routines, with their names,
arguments and outputs:

  keep_inlet_connected   prtlb_3d.py:530-563 (the pore the walk never reaches
                         is what it turns into solid)
  geodesic_steps         prt_core/conventions.py:72-115 (the step counts)
  distance_column        prt_core/conventions.py:119-158 (the three scalings
                         of the trunk's distance column, on those counts)
  geodesic, geodesic_2d  build_practice_dataset.py:53-73, build_dataset_2d.py:
                         297-319 (the value their relaxation sweeps converge to)
  percolates             build_dataset_3d.py:281-286 (percolates_3d),
                         build_dataset_2d.py:290-294
  percolates_between,    build_geometry_3d.py:201-221 (_percolates and
  keep_percolating_cluster  keep_percolating_cluster: two walks, one from each
                         plane; a component touches both when both reach it)
  label_materials        build_geometry_3d.py:224-239 (a face-neighbour
                         stencil, no walk)

The reference labels components with scipy and walks with a Python queue,
one voxel at a time; here each level of the walk is one kernel launch over
the grid.  Results are bit-identical to the reference's (tests/test_prep.py).
"""

import ctypes

import numpy as np

from . import _lib

SOLID, WALL, PORE = 0, 1, 2


def inlet_walk(mat, pore_code=PORE, inlet_axis=0, *, device=None, ctx=None):
    """Steps from the inlet face to every voxel of `mat` (2D or 3D): int32,
    the count for reached pore voxels (material pore_code), -1 for other
    materials, -2 for pore the walk never reaches.  Returns
    (steps, n_reached, n_pore)."""
    return walk_from_plane(mat, pore_code, inlet_axis, 0, device=device, ctx=ctx)


def walk_from_plane(mat, pore_code=PORE, axis=0, plane=0, *, device=None, ctx=None):
    """inlet_walk seeded on the plane where `axis` equals `plane` (negative
    planes count from the far face, as numpy indices do)."""
    mat = np.asarray(mat)
    if mat.ndim not in (2, 3):
        raise ValueError("grid must be 2D or 3D, got %dD" % mat.ndim)
    if not 0 <= int(axis) < mat.ndim:
        raise ValueError("axis %r is not an axis of a %dD grid" % (axis, mat.ndim))
    n = mat.shape[int(axis)]
    if not -n <= int(plane) < n:
        raise IndexError("plane %r is outside an axis of %d voxels" % (plane, n))
    plane = int(plane) % n
    if mat.dtype != np.uint8:
        hit = mat == pore_code
        mat8 = hit.astype(np.uint8)
        code = 1
    else:
        mat8 = np.ascontiguousarray(mat)
        code = int(pore_code)
    ctx = ctx or _lib.default_context(device)
    dims = (ctypes.c_int32 * 3)(*(list(mat.shape) + [1] * (3 - mat.ndim)))
    steps = np.empty(mat.shape, np.int32)
    nr, npore = ctypes.c_int64(), ctypes.c_int64()
    with ctx.lock:
        ctx.check(_lib.lib().prt_walk_from_plane(
            ctx.handle, mat8.ctypes.data_as(ctypes.c_void_p), mat.ndim, dims, code, int(axis),
            plane, steps.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nr),
            ctypes.byref(npore)))
    return steps, int(nr.value), int(npore.value)


def keep_inlet_connected(g, *, device=None, ctx=None):
    """Pore voxels the inlet face cannot reach become SOLID; returns
    (g, n_removed).  The components touching the face are kept, not the
    largest one.  With pore but none of it on the x = 0 face the grid comes
    back unchanged with n_removed = the pore count, as the reference's does
    (prtlb_3d.py:530-563)."""
    g = np.asarray(g)
    if g.ndim not in (2, 3):
        raise ValueError("grid must be 2D or 3D, got %dD" % g.ndim)
    steps, n_reached, n_pore = inlet_walk(g, PORE, 0, device=device, ctx=ctx)
    if n_pore == 0:
        return g, 0
    if n_reached == 0:
        return g, n_pore
    if n_reached == n_pore:
        return g, 0
    out = g.copy()
    out[steps == -2] = SOLID
    return out, n_pore - n_reached


def _seeded(seed_value, top):
    """seed, seed + 1, ... as float32 sums one step at a time, as a walk
    that adds 1.0 per step forms them."""
    s = np.empty(top + 1, np.float32)
    s[0] = np.float32(seed_value)
    for k in range(1, top + 1):
        s[k] = s[k - 1] + np.float32(1.0)
    return s


def geodesic_steps(pore, inlet_axis=0, seed_value=0.0, *, device=None, ctx=None):
    """Steps through the pore space from the face inlet_axis = 0 (face
    neighbours, not periodic): seed_value on the face, one more per step,
    float32; NaN in the solid and in pore the walk does not reach
    (prt_core/conventions.py:72-115)."""
    pore = np.asarray(pore, bool)
    steps, _, _ = inlet_walk(pore.view(np.uint8), 1, inlet_axis, device=device, ctx=ctx)
    d = np.full(pore.shape, np.nan, np.float32)
    hit = steps >= 0
    if hit.any():
        d[hit] = _seeded(seed_value, int(steps[hit].max()))[steps[hit]]
    return d


def pore_mask(material):
    """Where a chemical can be: boolean arrays as they are, 0/1 grids with 1
    as pore, material codes as PORE (prt_core/conventions.py:60-68)."""
    m = np.asarray(material)
    if m.dtype == bool:
        return m
    if set(np.unique(m).tolist()) <= {0, 1}:
        return m == 1
    return m == PORE


DISTANCE_CONVENTIONS = ("ours", "published", "published_pore")


def distance_column(material, convention="ours", inlet_axis=0, *, device=None, ctx=None):
    """The trunk's distance column under a named convention, float32, zero
    in the solid (prt_core/conventions.py:119-158):
      ours            steps from the inlet / (n - 1) along the inlet axis;
      published       seed 0.5, the solid set one past the furthest pore,
                      negated and scaled onto [0, 1] over the whole grid;
      published_pore  the same scaled over the pore only."""
    if convention not in DISTANCE_CONVENTIONS:
        raise ValueError("no distance convention called %r; the three are %s (not "
                         "interchangeable: 'ours' is 0 at the inlet, 'published' is 1 there)"
                         % (convention, ", ".join(DISTANCE_CONVENTIONS)))
    material = np.asarray(material)
    pore = pore_mask(material)
    if convention == "ours":
        d = geodesic_steps(pore, inlet_axis, 0.0, device=device, ctx=ctx)
        span = max(material.shape[inlet_axis] - 1, 1)
        col = np.where(np.isnan(d), np.float32(0.0), d) / float(span)
        col[~pore] = 0.0
        return col.astype(np.float32)
    d = geodesic_steps(pore, inlet_axis, 0.5, device=device, ctx=ctx)
    if not pore.any():
        far = 0.0
    elif np.isnan(d[pore]).all():
        far = float("nan")
    else:
        far = float(np.nanmax(d[pore]))
    neg = -np.where(pore, d, far + 1.0)
    col = np.zeros(neg.shape, np.float32)
    ok = np.isfinite(neg) if convention == "published" else (pore & np.isfinite(neg))
    if ok.any():
        lo, hi = float(neg[ok].min()), float(neg[ok].max())
        if hi > lo:
            col[ok] = (neg[ok] - lo) / (hi - lo)
        else:
            col[ok] = 1.0 if convention == "published_pore" else 0.0
    col[~pore] = 0.0
    return col.astype(np.float32)


def geodesic(g, *, device=None, ctx=None):
    """The practice dataset's distance from the inlet (build_practice_dataset.py:53-73):
    steps from the x = 0 face through the pore, 1e9 in pore that is not
    reached, 0 in the solid, float32.  The reference relaxes d = min(d,
    neighbour + 1) until a sweep changes nothing (at most 4 nx sweeps); this
    is the value those sweeps converge to."""
    g = np.asarray(g)
    if g.ndim != 3:
        raise ValueError("geodesic takes a 3D grid, got %dD" % g.ndim)
    return _relaxed(g, device, ctx)


def geodesic_2d(g, *, device=None, ctx=None):
    """geodesic on a 2D grid (build_dataset_2d.py:297-319)."""
    g = np.asarray(g)
    if g.ndim != 2:
        raise ValueError("geodesic_2d takes a 2D grid, got %dD" % g.ndim)
    return _relaxed(g, device, ctx)


def _relaxed(g, device, ctx):
    steps, _, _ = inlet_walk(g, PORE, 0, device=device, ctx=ctx)
    d = np.zeros(g.shape, np.float32)
    d[steps >= 0] = steps[steps >= 0].astype(np.float32)
    d[steps == -2] = np.float32(1e9)
    return d


def percolates(g, *, device=None, ctx=None):
    """Whether one pore component touches both x faces, i.e. the walk from
    the x = 0 face reaches the last x plane (percolates_3d,
    build_dataset_3d.py:281-286; the 2D builder's percolates,
    build_dataset_2d.py:290-294)."""
    g = np.asarray(g)
    steps, n_reached, _ = inlet_walk(g, PORE, 0, device=device, ctx=ctx)
    return bool(n_reached) and bool((steps[-1] >= 0).any())


def percolates_between(pore, x_in, x_out, *, device=None, ctx=None):
    """Whether one component of the boolean `pore` touches both planes
    x = x_in and x = x_out (build_geometry_3d.py:201-205, `_percolates`)."""
    pore = np.asarray(pore, bool)
    steps, n_reached, _ = walk_from_plane(pore.view(np.uint8), 1, 0, x_in, device=device, ctx=ctx)
    return bool(n_reached) and bool((steps[x_out] >= 0).any())


def keep_percolating_cluster(solid, x_in, x_out, *, device=None, ctx=None):
    """Pore outside every component that touches both planes x = x_in and
    x = x_out becomes solid: returns (solid, n_removed), or the input and -1
    when there is no pore or no such component (build_geometry_3d.py:208-221).
    A voxel is kept when the walks from both planes reach it."""
    solid = np.asarray(solid, bool)
    pore = (~solid).view(np.uint8)
    s_in, r_in, n_pore = walk_from_plane(pore, 1, 0, x_in, device=device, ctx=ctx)
    if n_pore == 0 or r_in == 0:
        return solid, -1
    s_out, _, _ = walk_from_plane(pore, 1, 0, x_out, device=device, ctx=ctx)
    keep = (s_in >= 0) & (s_out >= 0)
    if not keep.any():
        return solid, -1
    return ~keep, int(n_pore - np.count_nonzero(keep))


def label_materials(solid, *, device=None, ctx=None):
    """Material codes of a boolean solid grid on the GPU: pore 2, solid with a
    pore face neighbour 1 (the bounce-back wall), other solid 0; beyond the
    grid's faces counts as solid, nothing wraps (label_materials,
    build_geometry_3d.py:224-239).  2D and 3D grids."""
    solid = np.ascontiguousarray(np.asarray(solid, bool).view(np.uint8))
    if solid.ndim not in (2, 3):
        raise ValueError("label_materials expects a 2D or 3D grid, got %dD" % solid.ndim)
    ctx = ctx or _lib.default_context(device)
    dims = (ctypes.c_int32 * 3)(*(list(solid.shape) + [1] * (3 - solid.ndim)))
    out = np.empty(solid.shape, np.uint8)
    with ctx.lock:
        ctx.check(_lib.lib().prt_label_materials(ctx.handle, solid.ctypes.data_as(ctypes.c_void_p),
                                                 solid.ndim, dims,
                                                 out.ctypes.data_as(ctypes.c_void_p)))
    return out
