"""Host-side geometry: the reference's mask helpers and seeded synthetic packs.

keep_inlet_connected, coat_with_biofilm and assert_finite_distance restate
3D/tools/prtlb_3d.py:530-612 (same inputs, outputs and messages).  The
random disk / sphere packs are this project's own generators for the
benchmark workloads; the reference's build_spheres (build_geometry_3d.py:129)
makes a different, walled geometry and is not reused.
"""

import numpy as np

SOLID, WALL, PORE = 0, 1, 2


def keep_inlet_connected(g):
    """Pore voxels not connected to the x = 0 face become solid.

    Returns (g, n_removed); the inlet-touching components are kept, not the
    largest one (prtlb_3d.py:530-563)."""
    from scipy import ndimage
    g = np.asarray(g)
    pore = (g == PORE)
    if not pore.any():
        return g, 0
    lab, _ = ndimage.label(pore)
    seeds = np.unique(lab[0][pore[0]])
    seeds = seeds[seeds != 0]
    if seeds.size == 0:
        return g, int(pore.sum())
    drop = pore & ~np.isin(lab, seeds)
    if not drop.any():
        return g, 0
    g = g.copy()
    g[drop] = SOLID
    return g, int(drop.sum())


def coat_with_biofilm(g, code, layers=1):
    """Pore voxels within `layers` dilation steps of the rock get material
    `code`.  Returns (g, n_marked) (prtlb_3d.py:566-592)."""
    from scipy import ndimage
    g = np.asarray(g).copy()
    if code is None or layers <= 0:
        return g, 0
    grown = (g != PORE)
    for _ in range(int(layers)):
        grown = ndimage.binary_dilation(grown)
    lining = grown & (g == PORE)
    g[lining] = code
    return g, int(lining.sum())


def assert_finite_distance(d, g, name="geodesic"):
    """None when `d` is finite (and < 1e6) on every pore voxel, else the
    complaint (prtlb_3d.py:595-612)."""
    d = np.asarray(d)
    m = (np.asarray(g) == PORE)
    if not m.any():
        return None
    v = d[m]
    if np.isfinite(v).all() and float(v.max()) < 1e6:
        return None
    n = int((~np.isfinite(v)).sum() + (v >= 1e6).sum())
    return ("%s is not finite on %d of %d pore voxels (max %.4g). Those voxels cannot be "
            "reached from the inlet; run keep_inlet_connected first."
            % (name, n, m.sum(), float(v.max())))


def _stamp(solid, centre, r, periodic=True):
    """Mark a ball (disk) of radius r at `centre` solid; periodic wrap."""
    nd = solid.ndim
    rr = int(np.ceil(r))
    offs = np.arange(-rr, rr + 1)
    grids = np.meshgrid(*([offs] * nd), indexing="ij")
    d2 = sum(o.astype(np.float64) ** 2 for o in grids)
    inside = d2 <= r * r
    idx = []
    for a in range(nd):
        c = int(np.floor(centre[a]))
        pos = (c + grids[a][inside])
        idx.append(pos % solid.shape[a] if periodic else np.clip(pos, 0, solid.shape[a] - 1))
    solid[tuple(idx)] = True


def random_pack(shape, porosity, rmin, rmax, seed=0, max_tries=200000, overlap_after=5000):
    """Seeded pack of solid balls (disks in 2D) with radius U[rmin, rmax].

    Balls are placed at uniform random centres without overlap (periodic
    distance) until the pore fraction is <= `porosity`.  Random sequential
    placement jams before dense packs (about 0.55 covered in 2D, 0.38 in 3D),
    so after `overlap_after` consecutive rejections overlaps are accepted.
    The result is uint8 with PORE / SOLID, cut to the pore component that
    touches the x = 0 face."""
    rng = np.random.default_rng(seed)
    shape = tuple(int(s) for s in shape)
    nd = len(shape)
    solid = np.zeros(shape, bool)
    centres, radii = [], []
    L = np.array(shape, np.float64)
    rejects = 0
    tries = 0
    frac = 0.0
    while frac < 1.0 - porosity and tries < max_tries:
        tries += 1
        c = rng.random(nd) * L
        r = rmin + (rmax - rmin) * rng.random()
        ok = True
        if rejects < overlap_after and centres:
            d = np.abs(np.asarray(centres) - c)
            d = np.minimum(d, L - d)
            ok = bool((np.sqrt((d ** 2).sum(1)) >= np.asarray(radii) + r).all())
        if not ok:
            rejects += 1
            continue
        rejects = 0 if rejects < overlap_after else rejects
        centres.append(c)
        radii.append(r)
        _stamp(solid, c, r)
        frac = float(solid.mean())
    g = np.where(solid, SOLID, PORE).astype(np.uint8)
    g, _ = keep_inlet_connected(g)
    return g


def disk_pack_2d(n=128, porosity=0.6, seed=0):
    """The plain 2D workload: 128 x 128 periodic, disks r ~ U[4, 8]."""
    return random_pack((n, n), porosity, 4.0, 8.0, seed=seed)


def sphere_pack_3d(n=64, porosity=0.45, seed=0, rmin=4.0, rmax=7.0):
    """The plain 3D workload: n^3 periodic, spheres r ~ U[4, 7]."""
    return random_pack((n, n, n), porosity, rmin, rmax, seed=seed)
