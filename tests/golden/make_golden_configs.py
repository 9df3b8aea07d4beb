#!/usr/bin/env python3
"""Golden vectors at the benchmark configurations' sizes, made by running
the REFERENCE (shahram444/PRT-DeepONet-GUI, 3D/tools/prtlb_2d.py and
prtlb_3d.py, imported read-only from the reference checkout).

    python tests/golden/make_golden_configs.py --ref /path/to/reference [--only NAME ...]

Cases (written as cfg_*.npz next to this script):
  cfg_plain2d       the plain 2D configuration in full: 128 x 128 periodic
                    disks (r U[4, 8], porosity 0.6, seed 0), stokes_d2q9 at
                    force 1e-6, tau 0.8, magic 3/16, run to tol 1e-7; then
                    solve_adr of one first-order solute (the built-in
                    chemistry with one chemical) at Pe 10, Da 1, 4000 steps,
                    5 snapshots, on the reference's own velocity field
  cfg_plain3d64     the plain 3D pack (64^3 spheres r U[4, 7], porosity 0.45,
                    seed 0) at fixed counts: 300 stokes_d3q19 iterations
                    (tol 0), then 200 Monod steps (Ks 0.5, Pe 10, Da 1) on
                    that field; plus the same transport in float64 (the
                    reference with float32 replaced by float64 in its module
                    namespace, kept as its relative L2 and max difference from
                    the float32 run) and 200 steps of the four-chemical
                    dual-Monod chemistry with Ks 0.5; transport results are
                    kept as sha256, sums and a subsample of 4000 pore voxels
  cfg_sphere128     a 128^3 pack (r U[4, 7], porosity 0.45, seed 0): 100
                    stokes_d3q19 iterations (subsample of 8000 pore voxels
                    and whole-field statistics), and 50 steps of the
                    four-chemical chemistry (Ks 0.5) on integer_velocity(g)
                    (hash, statistics, subsample)

Large grids are regenerated by the tests from the seeded generator and
checked against the stored sha256, instead of being committed.
"""

import argparse
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "prt-deeponet-gui_b200"))
sys.path.insert(0, HERE)

from fields import digest, field_stats, integer_velocity, subsample  # noqa: E402
from prtlb_gpu.geometry import random_pack  # noqa: E402  (host-only)


def load_reference(ref):
    tools = os.path.join(ref, "3D", "tools")
    sys.path.insert(0, tools)
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    import prtlb_2d
    import prtlb_3d
    import settings_and_units
    return prtlb_2d, prtlb_3d, settings_and_units


def float64_twin(ref):
    """A second copy of the reference's prtlb_3d with np.float32 meaning
    float64 in its module namespace (its own code, float64 arithmetic)."""
    import importlib.util
    path = os.path.join(ref, "3D", "tools", "prtlb_3d.py")
    spec = importlib.util.spec_from_file_location("prtlb_3d_f64", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    shim = types.ModuleType("numpy_f64")
    shim.__dict__.update(np.__dict__)
    shim.float32 = np.float64
    mod.np = shim
    return mod


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print("wrote %-28s %8.1f KB" % (name, os.path.getsize(path) / 1024.0), flush=True)


def info_arrays(info, prefix):
    out = {}
    for k, v in info.items():
        if isinstance(v, (bool, int, float, str, np.floating, np.integer)):
            out[prefix + k] = np.asarray(v)
    return out


def run_adr(mod, mat, vel, kw):
    info, prog = {}, []
    t = time.time()
    out, tn = mod.solve_adr(mat, vel, info=info, on_progress=lambda *a: prog.append(a), **kw)
    print("  solve_adr %s: %.1f s, %d steps" % (kw, time.time() - t, info["steps"]), flush=True)
    return out, tn, info, np.asarray(prog, np.float64).reshape(-1, 4)


def adr_args(kw, prefix):
    return {prefix + k: np.asarray(v) for k, v in kw.items()
            if k != "chem" and v is not None}


def summary(out, m, prefix):
    """Hash, per (snapshot, chemical) float64 sums over the pore and a
    subsample of 4000 pore voxels of a transport result too large to commit."""
    out = np.asarray(out)
    flat = out.reshape(out.shape[0], out.shape[1], -1)
    idx = subsample(int(m.sum()), 4000, seed=1)
    pore = np.flatnonzero(m.reshape(-1))[idx]
    return {prefix + "sha256": np.asarray(digest(out)),
            prefix + "shape": np.asarray(out.shape),
            prefix + "sums": flat[:, :, m.reshape(-1)].astype(np.float64).sum(-1),
            prefix + "sub_index": pore, prefix + "sub": flat[:, :, pore]}


def case_plain2d(p2, p3, su):
    g = random_pack((128, 128), 0.6, 4.0, 8.0, seed=0, native=False)
    info = {}
    t = time.time()
    v = p2.stokes_d2q9(g, nit=30000, force=1e-6, tau_lb=0.8, magic=3.0 / 16.0, tol=1e-7,
                       info=info)
    print("  stokes_d2q9 128^2: %.1f s, %d iterations" % (time.time() - t, info["flow_iters"]),
          flush=True)
    kw = dict(pe=10.0, da=1.0, n_t=5, n_species=1, steps=4000)
    out, tn, ainfo, prog = run_adr(p2, g, v, kw)
    save("cfg_plain2d", g=g, v=v, nit=30000, force=1e-6, tau=0.8, tol=1e-7,
         **info_arrays(info, "info_"), out=out, t_norm=tn, progress=prog,
         **adr_args(kw, "arg_"), **info_arrays(ainfo, "ainfo_"))


def monod(su, ks=0.5):
    return su.Chemistry(names=["C"], inlet=[1.0], c_init=[0.0], d_rel=[1.0],
                        immobile=[False], ks_donor=ks)


def dual_monod(su, ks=0.5):
    c = su.default_chemistry(4)
    c.ks_donor = ks
    return c


def case_plain3d64(ref, p2, p3, su):
    g = random_pack((64, 64, 64), 0.45, 4.0, 7.0, seed=0, native=False)
    info = {}
    t = time.time()
    v = p3.stokes_d3q19(g, nit=300, force=2e-6, tau_lb=0.8, magic=3.0 / 16.0, tol=0.0,
                        info=info)
    print("  stokes_d3q19 64^3: %.1f s" % (time.time() - t), flush=True)
    m = g == 2
    kw = dict(pe=10.0, da=1.0, n_t=5, n_species=1, steps=200)
    out, tn, ainfo, prog = run_adr(p3, g, v, dict(kw, chem=monod(su)))
    f64 = float64_twin(ref)
    out64, tn64, _, _ = run_adr(f64, g, v, dict(kw, chem=monod(su)))
    kw4 = dict(pe=10.0, da=1.0, n_t=5, n_species=4, steps=200)
    out4, tn4, ainfo4, prog4 = run_adr(p3, g, v, dict(kw4, chem=dual_monod(su)))
    # the reference's float32 transport against its float64 twin: the GPU
    # run must equal the float32 one bit for bit, so these are its errors too
    d = out.astype(np.float64) - out64
    twin = np.asarray([np.linalg.norm(d) / np.linalg.norm(out64),
                       np.abs(d).max() / np.abs(out64).max()])
    save("cfg_plain3d64", g=g, v=v, nit=300, force=2e-6, tau=0.8, tol=0.0,
         **info_arrays(info, "info_"),
         t_norm=tn, progress=prog, **adr_args(kw, "arg_"), **info_arrays(ainfo, "ainfo_"),
         **summary(out, m, "out_"), t_norm64=tn64, twin_rel_l2_max=twin,
         t_norm4=tn4, progress4=prog4, **adr_args(kw4, "arg4_"),
         **info_arrays(ainfo4, "ainfo4_"), **summary(out4, m, "out4_"))


def case_sphere128(p2, p3, su):
    g = random_pack((128, 128, 128), 0.45, 4.0, 7.0, seed=0, native=False)
    m = g == 2
    info = {}
    t = time.time()
    v = p3.stokes_d3q19(g, nit=100, force=2e-6, tau_lb=0.8, magic=3.0 / 16.0, tol=0.0,
                        info=info)
    print("  stokes_d3q19 128^3: %.1f s" % (time.time() - t), flush=True)
    idx = subsample(int(m.sum()), 8000, seed=0)
    pore = np.flatnonzero(m.reshape(-1))[idx]
    vflat = v.reshape(3, -1)
    vel = integer_velocity(g)
    kw = dict(pe=10.0, da=1.0, n_t=5, n_species=4, steps=50)
    out, tn, ainfo, prog = run_adr(p3, g, vel, dict(kw, chem=dual_monod(su)))
    save("cfg_sphere128", g_sha256=np.asarray(digest(g)), g_shape=np.asarray(g.shape),
         nit=100, force=2e-6, tau=0.8, tol=0.0, **info_arrays(info, "info_"),
         v_sub_index=pore, v_sub=vflat[:, pore], v_stats=field_stats(v, m),
         vel_sha256=np.asarray(digest(vel)), t_norm=tn, progress=prog,
         **adr_args(kw, "arg_"), **info_arrays(ainfo, "ainfo_"), **summary(out, m, "out_"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path of the reference checkout")
    ap.add_argument("--only", nargs="*", default=None)
    args = ap.parse_args()
    p2, p3, su = load_reference(args.ref)
    cases = {"cfg_plain2d": lambda: case_plain2d(p2, p3, su),
             "cfg_plain3d64": lambda: case_plain3d64(args.ref, p2, p3, su),
             "cfg_sphere128": lambda: case_sphere128(p2, p3, su)}
    for name in (args.only or list(cases)):
        print(name, flush=True)
        cases[name]()


if __name__ == "__main__":
    main()
