"""Host-side geometry: seeded synthetic packs and the mask helpers they need.

The random disk / sphere packs are this project's own generators for the
benchmark workloads; the reference's build_spheres (build_geometry_3d.py:129)
makes a different, walled geometry and is not reused.  The helpers below keep
the outputs and messages of the reference's (prtlb_3d.py:530-612) for callers
without a GPU, such as the pack generators; with a device,
prtlb_gpu.keep_inlet_connected is the GPU walk (prtlb_gpu.prep), which gives
the same grid bit for bit.
"""

import numpy as np

SOLID, WALL, PORE = 0, 1, 2


def keep_inlet_connected_host(g):
    """Pore voxels outside every face-connected pore component that touches
    the x = 0 face become SOLID; returns (g, n_removed).  A grid with pore
    but none of it on that face comes back unchanged with n_removed = the
    pore count (the reference's behaviour, prtlb_3d.py:530-563)."""
    from scipy import ndimage
    g = np.asarray(g)
    pore = g == PORE
    if not pore.any():
        return g, 0
    labels, n = ndimage.label(pore)
    on_face = np.zeros(n + 1, bool)  # component id -> touches x = 0
    on_face[labels[0][pore[0]]] = True
    on_face[0] = False
    if not on_face.any():
        return g, int(pore.sum())
    cut = pore & ~on_face[labels]
    n_cut = int(np.count_nonzero(cut))
    if n_cut == 0:
        return g, 0
    out = g.copy()
    out[cut] = SOLID
    return out, n_cut


def coat_with_biofilm(g, code, layers=1):
    """Pore voxels within `layers` face-neighbour steps of non-pore become
    material `code`; returns (g, n_marked) (prtlb_3d.py:566-592)."""
    from scipy import ndimage
    g = np.asarray(g).copy()
    if code is None or layers <= 0:
        return g, 0
    near = ndimage.binary_dilation(g != PORE, iterations=int(layers))
    lining = near & (g == PORE)
    g[lining] = code
    return g, int(np.count_nonzero(lining))


def assert_finite_distance(d, g, name="geodesic"):
    """None when the distance field `d` is finite and below 1e6 on every pore
    voxel of `g`, else the reference's complaint (prtlb_3d.py:595-612); its
    count adds the non-finite values and those >= 1e6, so an infinity counts
    twice, as there."""
    pore = np.asarray(g) == PORE
    if not pore.any():
        return None
    vals = np.asarray(d)[pore]
    nonfinite = ~np.isfinite(vals)
    huge = vals >= 1e6
    if not (nonfinite.any() or huge.any()):
        return None
    n = int(np.count_nonzero(nonfinite) + np.count_nonzero(huge))
    return ("%s is not finite on %d of %d pore voxels (max %.4g). Those voxels cannot be "
            "reached from the inlet; run keep_inlet_connected first."
            % (name, n, pore.sum(), float(vals.max())))


def _stamp(solid, centre, r, periodic=True):
    """Mark a ball (disk) of radius r at `centre` solid; periodic wrap.
    Returns how many voxels turned solid."""
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
    lin = np.ravel_multi_index(tuple(idx), solid.shape)
    if 2 * rr + 1 > min(solid.shape) or not periodic:
        lin = np.unique(lin)  # a ball wider than the box wraps onto itself
    flat = solid.reshape(-1)
    new = int(np.count_nonzero(~flat[lin]))
    flat[lin] = True
    return new


class _CellList(object):
    """Ball centres hashed into periodic cells at least 2 rmax wide, so the
    overlap test only visits the 3^nd cells around a candidate."""

    def __init__(self, L, rmax):
        self.L = L
        self.n = np.maximum(1, np.floor(L / max(2.0 * rmax, 1e-9))).astype(int)
        self.size = L / self.n
        self.cells = {}

    def _key(self, c):
        return tuple(int(v) % int(m) for v, m in zip(np.floor(c / self.size), self.n))

    def add(self, c, r):
        self.cells.setdefault(self._key(c), []).append((c, r))

    def near(self, c):
        k = self._key(c)
        keys = set()
        for off in np.ndindex(*([3] * len(k))):
            keys.add(tuple((k[a] + off[a] - 1) % int(self.n[a]) for a in range(len(k))))
        out = []
        for kk in keys:
            out.extend(self.cells.get(kk, ()))
        return out


def random_pack(shape, porosity, rmin, rmax, seed=0, max_tries=None, overlap_after=5000,
                native=True):
    """Seeded pack of solid balls (disks in 2D) with radius U[rmin, rmax].

    Balls are placed at uniform random centres without overlap (periodic
    distance) until the pore fraction is <= `porosity`.  Random sequential
    placement jams before dense packs (about 0.55 covered in 2D, 0.38 in 3D),
    so after `overlap_after` consecutive rejections overlaps are accepted.
    `max_tries` (default 200000 per 64^3 voxels) bounds the placements.
    The result is uint8 with PORE / SOLID, cut to the pore component that
    touches the x = 0 face.  The placement loop runs in libprtlb's host
    helper prt_pack_balls (native=True) or in NumPy; both give the same
    pack."""
    shape = tuple(int(s) for s in shape)
    ntot = int(np.prod(shape))
    if max_tries is None:
        max_tries = 200000 * max(1, -(-ntot // 262144))
    loop = _pack_loop_native if native else _pack_loop_numpy
    solid = loop(shape, porosity, rmin, rmax, seed, max_tries, overlap_after)
    g = np.where(solid, SOLID, PORE).astype(np.uint8)
    g, _ = keep_inlet_connected_host(g)
    return g


def _pack_loop_numpy(shape, porosity, rmin, rmax, seed, max_tries, overlap_after):
    rng = np.random.default_rng(seed)
    nd = len(shape)
    ntot = int(np.prod(shape))
    solid = np.zeros(shape, bool)
    L = np.array(shape, np.float64)
    grid = _CellList(L, rmax)
    nballs = 0
    rejects = 0
    tries = 0
    nsolid = 0
    frac = 0.0
    while frac < 1.0 - porosity and tries < max_tries:
        tries += 1
        c = rng.random(nd) * L
        r = rmin + (rmax - rmin) * rng.random()
        ok = True
        if rejects < overlap_after and nballs:
            near = grid.near(c)
            if near:
                cs = np.asarray([q[0] for q in near])
                rs = np.asarray([q[1] for q in near])
                d = np.abs(cs - c)
                d = np.minimum(d, L - d)
                ok = bool((np.sqrt((d ** 2).sum(1)) >= rs + r).all())
        if not ok:
            rejects += 1
            continue
        rejects = 0 if rejects < overlap_after else rejects
        grid.add(c, r)
        nballs += 1
        nsolid += _stamp(solid, c, r)
        frac = nsolid / ntot
    return solid


def _pack_loop_native(shape, porosity, rmin, rmax, seed, max_tries, overlap_after):
    """The same loop in prt_pack_balls: the uniform numbers are drawn here in
    chunks, in the order the NumPy loop draws them (nd for the centre, one
    for the radius, per try)."""
    import ctypes
    from . import _lib
    L = _lib.lib()
    rng = np.random.default_rng(seed)
    nd = len(shape)
    ntot = int(np.prod(shape))
    solid = np.zeros(shape, np.uint8)
    shp = (ctypes.c_int32 * nd)(*shape)
    vball = (4.0 / 3.0 * np.pi * rmin ** 3) if nd == 3 else (np.pi * rmin ** 2)
    cap = int(4 * ntot / max(vball, 1.0)) + 64
    centres = np.zeros((cap, nd), np.float64)
    radii = np.zeros(cap, np.float64)
    state = (ctypes.c_int64 * 4)(0, 0, 0, 0)
    target = 1.0 - porosity
    chunk = 65536
    while state[3] / ntot < target and state[2] < max_tries:
        cand = rng.random((chunk, nd + 1))
        pos = 0
        while pos < chunk:
            used = L.prt_pack_balls(solid.ctypes.data_as(ctypes.c_void_p), nd, shp,
                                    ctypes.c_void_p(cand.ctypes.data + pos * (nd + 1) * 8),
                                    chunk - pos, float(rmin), float(rmax), target,
                                    int(overlap_after), int(max_tries),
                                    centres.ctypes.data_as(ctypes.c_void_p),
                                    radii.ctypes.data_as(ctypes.c_void_p), cap, state)
            if used < 0:
                raise ValueError("prt_pack_balls refused its arguments (%d)" % used)
            pos += used
            if state[0] >= cap:  # more balls than room: grow and go on
                cap *= 2
                centres = np.concatenate([centres, np.zeros_like(centres)])
                radii = np.concatenate([radii, np.zeros_like(radii)])
                continue
            if state[3] / ntot >= target or state[2] >= max_tries or used == 0:
                break
        if state[3] / ntot >= target or state[2] >= max_tries:
            break
    return solid.astype(bool)


def disk_pack_2d(n=128, porosity=0.6, seed=0):
    """The plain 2D workload: 128 x 128 periodic, disks r ~ U[4, 8]."""
    return random_pack((n, n), porosity, 4.0, 8.0, seed=seed)


def sphere_pack_3d(n=64, porosity=0.45, seed=0, rmin=4.0, rmax=7.0):
    """The plain 3D workload: n^3 periodic, spheres r ~ U[4, 7]."""
    return random_pack((n, n, n), porosity, rmin, rmax, seed=seed)
