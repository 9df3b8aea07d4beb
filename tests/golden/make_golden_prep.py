#!/usr/bin/env python3
"""Golden vectors of the geometry-preparation walk, made by running the REFERENCE.

Runs the reference's own helpers (shahram444/PRT-DeepONet-GUI, imported
read-only from the reference checkout) on small seeded grids and saves inputs
and outputs as compressed .npz files next to this script:

  keep_inlet_connected   3D/tools/prtlb_3d.py:530-563 (scipy 6-connected
                         labels, the components touching the x = 0 face)
  geodesic_steps         prt_core/conventions.py:72-115 (breadth-first walk
                         from the inlet face, seeds 0 and 0.5, every axis)
  distance_column        prt_core/conventions.py:119-158 (the three scalings)
  geodesic               3D/tools/build_practice_dataset.py:53-73 (repeated
                         relaxation, 1e9 in unreached pore, 0 in the solid)
  geodesic_2d            3D/tools/build_dataset_2d.py:297-319 (the same in 2D)
  percolates_3d          3D/tools/build_dataset_3d.py:281-286 (a pore component
  percolates (2D)        3D/tools/build_dataset_2d.py:290-294  touches both x faces)
  _percolates,           3D/tools/build_geometry_3d.py:201-221 (components
  keep_percolating_cluster                            touching two x planes)

Needs the reference checkout, so it runs in the development container only;
the fixtures are committed and are all the tests read.

    python tests/golden/make_golden_prep.py --ref /path/to/reference
"""

import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(ref):
    sys.path.insert(0, ref)
    sys.path.insert(0, os.path.join(ref, "3D", "tools"))
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    import prtlb_3d
    from prt_core import conventions
    import build_practice_dataset
    import build_dataset_2d
    import build_dataset_3d
    import build_geometry_3d
    return prtlb_3d, conventions, build_practice_dataset, build_dataset_2d, build_dataset_3d, \
        build_geometry_3d


def grids():
    """Seeded site-percolation grids near the threshold (many clusters, some
    of them larger than the inlet-connected one), with wall voxels, plus the
    edge cases: no pore on the inlet face, no pore at all, a single column."""
    rng = np.random.default_rng(7)
    out = {}

    def site(shape, p):
        g = np.where(rng.random(shape) < p, 2, 0).astype(np.uint8)
        g[rng.random(shape) < 0.03] = 1  # walls: neither pore nor solid code
        return g

    out["prep_site3d"] = site((24, 18, 14), 0.36)
    out["prep_site3d_dense"] = site((20, 16, 12), 0.55)
    out["prep_site2d"] = site((48, 36), 0.61)
    g = site((16, 12, 10), 0.5)
    g[0] = 0
    out["prep_noinlet3d"] = g
    out["prep_solid3d"] = np.zeros((8, 6, 5), np.uint8)
    g = np.zeros((12, 5, 5), np.uint8)
    g[:, 2, 2] = 2
    g[7, 2, 2] = 0  # the column is cut: the far part is unreachable
    out["prep_column3d"] = g
    g = site((30, 40), 0.66)
    g[:, 0] = g[:, -1] = 1  # transverse walls, as the 2D builder makes them
    out["prep_site2d_walls"] = g
    return out


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print("wrote %-28s %6.1f KB" % (name, os.path.getsize(path) / 1024.0), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True,
                    help="path of the reference checkout")
    args = ap.parse_args()
    p3, conv, bpd, bd2, bd3, bg3 = load_reference(args.ref)
    for name, g in grids().items():
        kept, n_removed = p3.keep_inlet_connected(g.copy())
        arrays = {"mat": g, "kept": np.asarray(kept, np.uint8), "n_removed": np.asarray(n_removed)}
        pore = g == p3.PORE
        for axis in range(g.ndim):
            for seed in (0.0, 0.5):
                d = conv.geodesic_steps(pore, inlet_axis=axis, seed_value=seed)
                arrays["steps_a%d_s%g" % (axis, seed)] = np.asarray(d, np.float32)
        for c in conv.DISTANCE_CONVENTIONS:
            arrays["column_" + c] = np.asarray(conv.distance_column(g, c, 0), np.float32)
        if g.ndim == 3:
            arrays["geodesic"] = np.asarray(bpd.geodesic(np.asarray(kept)), np.float32)
            arrays["percolates"] = np.asarray(bd3.percolates_3d(g))
            solid = g != p3.PORE
            nx = g.shape[0]
            for k, (xi, xo) in enumerate(((0, nx - 1), (2, nx - 3), (nx // 2, nx // 2))):
                arrays["perc_between_%d" % k] = np.asarray(bg3._percolates(~solid, xi, xo))
                kept_s, removed = bg3.keep_percolating_cluster(solid.copy(), xi, xo)
                arrays["keep_perc_%d" % k] = np.asarray(kept_s, bool)
                arrays["keep_perc_removed_%d" % k] = np.asarray(removed)
        else:
            arrays["geodesic_2d"] = np.asarray(bd2.geodesic_2d(np.asarray(kept)), np.float32)
            arrays["percolates"] = np.asarray(bd2.percolates(g))
        save(name, **arrays)
    # label_materials (build_geometry_3d.py:224-239): the 3D grids above as
    # solids, plus seeded solids whose pore touches every face of the box
    rng = np.random.default_rng(11)
    solids = {"label_site3d": grids()["prep_site3d"] != p3.PORE,
              "label_dense3d": grids()["prep_site3d_dense"] != p3.PORE,
              "label_rand3d": rng.random((17, 13, 9)) < 0.5,
              "label_sparse3d": rng.random((9, 11, 16)) < 0.15,
              "label_allsolid3d": np.ones((5, 4, 3), bool)}
    for name, solid in solids.items():
        save(name, solid=np.asarray(solid, bool),
             materials=np.asarray(bg3.label_materials(np.asarray(solid, bool)), np.uint8))


if __name__ == "__main__":
    main()
