"""NumPy restatement of the geometry-preparation walk (TEST ORACLE).

Test infrastructure only (see oracle/__init__.py): the GPU walk in
libprtlb.so is checked against these functions, which are checked against
golden runs of the reference (tests/golden/make_golden_prep.py).  Each
function cites the reference lines it restates.
"""

from collections import deque

import numpy as np

SOLID, WALL, PORE = 0, 1, 2


def keep_inlet_connected(g):
    """Pore voxels outside every 6- (4-) connected pore component that
    touches the x = 0 face become SOLID; returns (g, n_removed).  With pore
    but none on the face the grid comes back unchanged and n_removed is the
    pore count (prtlb_3d.py:530-563)."""
    from scipy import ndimage
    g = np.asarray(g)
    pore = g == PORE
    if not pore.any():
        return g, 0
    lab, _ = ndimage.label(pore)
    seeds = np.setdiff1d(np.unique(lab[0][pore[0]]), [0])
    if seeds.size == 0:
        return g, int(pore.sum())
    drop = pore & ~np.isin(lab, seeds)
    if not drop.any():
        return g, 0
    out = g.copy()
    out[drop] = SOLID
    return out, int(drop.sum())


def geodesic_steps(pore, inlet_axis=0, seed_value=0.0):
    """Breadth-first walk through `pore` from its voxels on the face
    inlet_axis = 0: seed_value there, one more per face-neighbour step, not
    periodic; NaN in the solid and in pore the walk never reaches, float32
    (prt_core/conventions.py:72-115)."""
    pore = np.asarray(pore, bool)
    d = np.full(pore.shape, np.nan, np.float32)
    todo = deque()
    for idx in np.argwhere(np.take(pore, 0, axis=inlet_axis)):
        p = tuple(int(i) for i in np.insert(idx, inlet_axis, 0))
        d[p] = np.float32(seed_value)
        todo.append(p)
    steps = []
    for ax in range(pore.ndim):
        for s in (1, -1):
            o = [0] * pore.ndim
            o[ax] = s
            steps.append(o)
    while todo:
        p = todo.popleft()
        nxt = d[p] + np.float32(1.0)
        for o in steps:
            q = tuple(a + b for a, b in zip(p, o))
            if not all(0 <= a < n for a, n in zip(q, pore.shape)) or not pore[q]:
                continue
            if np.isnan(d[q]) or d[q] > nxt:
                d[q] = nxt
                todo.append(q)
    return d


def pore_mask(material):
    """Boolean arrays as they are, 0/1 grids as 1 = pore, material codes as
    PORE (prt_core/conventions.py:60-68)."""
    m = np.asarray(material)
    if m.dtype == bool:
        return m
    if set(np.unique(m).tolist()) <= {0, 1}:
        return m == 1
    return m == PORE


def distance_column(material, convention="ours", inlet_axis=0):
    """The walk scaled one of three ways, zero in the solid
    (prt_core/conventions.py:119-158): "ours" = steps / (n_axis - 1);
    "published" / "published_pore" = seed 0.5, solid set one past the
    furthest pore, negated, min-max scaled over the whole grid / the pore."""
    pore = pore_mask(material)
    if convention == "ours":
        d = geodesic_steps(pore, inlet_axis, 0.0)
        n = max(np.asarray(material).shape[inlet_axis] - 1, 1)
        col = np.where(np.isnan(d), np.float32(0), d) / float(n)
        col[~pore] = 0.0
        return col.astype(np.float32)
    d = geodesic_steps(pore, inlet_axis, 0.5)
    with np.errstate(all="ignore"):
        far = float(np.nanmax(d[pore])) if pore.any() and np.isfinite(d[pore]).any() else \
            (float("nan") if pore.any() else 0.0)
    d = -np.where(pore, d, far + 1.0)
    col = np.zeros(d.shape, np.float32)
    ok = np.isfinite(d) if convention == "published" else (pore & np.isfinite(d))
    if ok.any():
        lo, hi = float(d[ok].min()), float(d[ok].max())
        if hi > lo:
            col[ok] = (d[ok] - lo) / (hi - lo)
        else:
            col[ok] = 1.0 if convention == "published_pore" else 0.0
    col[~pore] = 0.0
    return col.astype(np.float32)


def geodesic_relaxed(g, sweeps=None):
    """The practice-dataset distance (build_practice_dataset.py:53-73; in 2D
    geodesic_2d, build_dataset_2d.py:297-319): 1e9 in pore, 0 on the pore of
    the x = 0 face, then sweeps of d = min(d, neighbour + 1) over the face
    neighbours in turn (no wrap), until a sweep changes nothing or 4 nx
    sweeps ran; solid 0."""
    g = np.asarray(g)
    pore = g == PORE
    big = np.float32(1e9)
    d = np.where(pore, big, np.nan).astype(np.float32)
    d[0][pore[0]] = 0.0
    for _ in range(4 * g.shape[0] if sweeps is None else sweeps):
        before = d.copy()
        for ax in range(g.ndim):
            for s in (1, -1):
                nb = np.roll(d, s, axis=ax)
                edge = [slice(None)] * g.ndim
                edge[ax] = 0 if s > 0 else -1
                nb[tuple(edge)] = big
                d = np.where(pore, np.fmin(d, np.where(np.isnan(nb), big, nb) + 1.0), np.nan)
        if np.nanmax(np.abs(np.where(np.isnan(d - before), 0.0, d - before)), initial=0.0) < 1e-6:
            break
    return np.where(np.isnan(d), np.float32(0), d).astype(np.float32)


def percolates(g):
    """Whether one pore component touches both x faces
    (build_dataset_3d.py:281-286, build_dataset_2d.py:290-294)."""
    from scipy import ndimage
    g = np.asarray(g)
    lab, _ = ndimage.label(g == PORE)
    first = set(np.unique(lab[0][g[0] == PORE]).tolist()) - {0}
    last = set(np.unique(lab[-1][g[-1] == PORE]).tolist()) - {0}
    return bool(first & last)


def percolates_between(pore, x_in, x_out):
    """Whether one component of `pore` touches both planes x = x_in and
    x = x_out (build_geometry_3d.py:201-205)."""
    from scipy import ndimage
    lab, n = ndimage.label(pore)
    if n == 0:
        return False
    return bool((set(np.unique(lab[x_in]).tolist()) - {0}) &
                (set(np.unique(lab[x_out]).tolist()) - {0}))


def keep_percolating_cluster(solid, x_in, x_out):
    """Pore outside every component touching both planes becomes solid;
    returns (solid, n_removed), or (solid unchanged, -1) without pore or
    without such a component (build_geometry_3d.py:208-221)."""
    from scipy import ndimage
    solid = np.asarray(solid, bool)
    pore = ~solid
    lab, n = ndimage.label(pore)
    if n == 0:
        return solid, -1
    good = (set(np.unique(lab[x_in]).tolist()) - {0}) & (set(np.unique(lab[x_out]).tolist()) - {0})
    if not good:
        return solid, -1
    keep = np.isin(lab, sorted(good))
    return ~keep, int((pore & ~keep).sum())


def label_materials(solid):
    """Material codes of a boolean solid grid: pore 2, solid with a pore face
    neighbour 1 (the bounce-back wall), other solid 0.  Neighbours beyond the
    grid's faces count as solid: nothing wraps (build_geometry_3d.py:224-239,
    a padded dilation over the three axes)."""
    solid = np.asarray(solid, bool)
    pore = ~solid
    touch = np.zeros_like(pore)
    for ax in range(pore.ndim):
        n = pore.shape[ax]
        lo = [slice(None)] * pore.ndim
        hi = [slice(None)] * pore.ndim
        lo[ax], hi[ax] = slice(0, n - 1), slice(1, n)
        touch[tuple(hi)] |= pore[tuple(lo)]  # the neighbour below is pore
        touch[tuple(lo)] |= pore[tuple(hi)]  # the neighbour above is pore
    g = np.full(pore.shape, SOLID, np.uint8)
    g[solid & touch] = WALL
    g[pore] = PORE
    return g
