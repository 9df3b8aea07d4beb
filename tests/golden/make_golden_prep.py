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

Needs the reference checkout, so it runs in the development container only;
the fixtures are committed and are all the tests read.

    python tests/golden/make_golden_prep.py [--ref /path/to/reference]
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
    return prtlb_3d, conventions, build_practice_dataset


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
    return out


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print("wrote %-28s %6.1f KB" % (name, os.path.getsize(path) / 1024.0), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    p3, conv, bpd = load_reference(args.ref)
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
        save(name, **arrays)


if __name__ == "__main__":
    main()
