#!/usr/bin/env python3
"""Generate the golden vectors of the test suite by running the REFERENCE.

Runs the reference's own solver (shahram444/PRT-DeepONet-GUI,
3D/tools/prtlb_2d.py and prtlb_3d.py, imported read-only from the reference
checkout) on small seeded cases and saves inputs and outputs as compressed
.npz files next to this script.  Needs the reference checkout, so it runs in
the development container only; the fixtures it writes are committed and are
all the tests read.

    python tests/golden/make_golden.py --ref /path/to/reference

Cases (every one small enough for the reference to finish in seconds):
  flow_*   stokes_d2q9 / stokes_d3q19: slits (fixed iteration counts and
           converged), a porous 2D disk pack, a 3D sphere pack, tau sweeps
  adr_*    solve_adr in float32: plug flow, porous 2D/3D with first-order and
           Monod kinetics, the 4-chemical default chemistry run to
           convergence, biofilm + abiotic + coupled biomass, n_t variants,
           a sealed half, on_progress records
  adr64_*  the same solve with the reference's float32 replaced by float64
           in its module namespace (the float64 twin used for error bars)
"""

import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "prt-deeponet-gui_b200"))

from prtlb_gpu.geometry import random_pack, coat_with_biofilm  # noqa: E402  (host-only)


def load_reference(ref):
    tools = os.path.join(ref, "3D", "tools")
    sys.path.insert(0, tools)
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    import prtlb_2d
    import prtlb_3d
    import settings_and_units
    return prtlb_2d, prtlb_3d, settings_and_units


def float64_twin(mod):
    """The reference module with np.float32 meaning float64 (its own code)."""
    shim = types.ModuleType("numpy_f64")
    shim.__dict__.update(np.__dict__)
    shim.float32 = np.float64
    mod.np = shim
    return mod


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print("wrote %-32s %7.1f KB" % (name, os.path.getsize(path) / 1024.0), flush=True)


def info_arrays(info, prefix="info_"):
    out = {}
    for k, v in info.items():
        if isinstance(v, (bool, int, float, np.floating, np.integer)):
            out[prefix + k] = np.asarray(v)
        elif isinstance(v, str):
            out[prefix + k] = np.asarray(v)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True,
                    help="path of the reference checkout")
    args = ap.parse_args()
    p2, p3, su = load_reference(args.ref)
    PORE, SOLID = p3.PORE, p3.SOLID

    # ---------------- flow ----------------
    g = np.full((12, 22), PORE, np.uint8)
    g[:, 0] = SOLID
    g[:, -1] = SOLID
    for nit, tag in ((1000, "fixed1000"), (1001, "fixed1001")):
        info = {}
        v = p2.stokes_d2q9(g, nit=nit, force=2e-6, tau_lb=0.8, tol=0.0, info=info)
        save("flow_slit2d_" + tag, g=g, v=v, nit=nit, force=2e-6, tau=0.8, tol=0.0,
             **info_arrays(info))
    for tau in (0.55, 1.2):
        info = {}
        gg = np.full((8, 10), PORE, np.uint8)
        gg[:, 0] = SOLID
        gg[:, -1] = SOLID
        v = p2.stokes_d2q9(gg, nit=20000, force=2e-6, tau_lb=tau, tol=1e-6, info=info)
        save("flow_slit2d_tau%g" % tau, g=gg, v=v, nit=20000, force=2e-6, tau=tau, tol=1e-6,
             **info_arrays(info))
    gd = random_pack((48, 32), 0.6, 3.0, 5.0, seed=3)
    info = {}
    v = p2.stokes_d2q9(gd, nit=30000, force=1e-6, tau_lb=0.8, tol=1e-7, info=info)
    save("flow_disks2d", g=gd, v=v, nit=30000, force=1e-6, tau=0.8, tol=1e-7, **info_arrays(info))
    v2d_disks = v

    g3 = np.full((8, 12, 6), PORE, np.uint8)
    g3[:, 0, :] = SOLID
    g3[:, -1, :] = SOLID
    info = {}
    v = p3.stokes_d3q19(g3, nit=601, force=2e-6, tau_lb=0.8, tol=0.0, info=info)
    save("flow_slit3d_fixed601", g=g3, v=v, nit=601, force=2e-6, tau=0.8, tol=0.0,
         **info_arrays(info))
    gs = random_pack((20, 20, 20), 0.45, 3.0, 5.0, seed=1)
    info = {}
    v = p3.stokes_d3q19(gs, nit=6000, force=2e-6, tau_lb=0.8, tol=1e-6, info=info)
    save("flow_spheres3d", g=gs, v=v, nit=6000, force=2e-6, tau=0.8, tol=1e-6,
         **info_arrays(info))
    v3d_spheres = v
    info = {}
    v = p3.stokes_d3q19(gs, nit=200, force=3e-3, tau_lb=0.8, tol=1e-6, info=info)
    save("flow_spheres3d_fast", g=gs, v=v, nit=200, force=3e-3, tau=0.8, tol=1e-6,
         **info_arrays(info))

    # ---------------- transport ----------------
    def adr(name, mod, mat, vel, kw, fp64=False):
        info = {}
        prog = []
        kw = dict(kw)
        kw["on_progress"] = lambda *a: prog.append(a)
        out, tn = mod.solve_adr(mat, vel, info=info, **kw)
        extra = {}
        for key in ("pe", "da", "n_t", "n_species", "steps", "tol", "max_steps", "da_abio"):
            if key in kw and kw[key] is not None:
                extra["arg_" + key] = np.asarray(kw[key])
        save(name, mat=np.asarray(mat), vel=np.asarray(vel, np.float32), out=out, t_norm=tn,
             progress=np.asarray(prog, np.float64).reshape(-1, 4), **extra,
             **info_arrays(info))
        return out

    g = np.full((40, 8), PORE, np.uint8)
    v = np.zeros((3, 40, 8), np.float32)
    v[0] = 1.0
    adr("adr_plug2d", p2, g, v, dict(pe=4000.0, da=1.0, n_t=3, n_species=1))
    adr("adr_chan2d_ns4", p2, g, v, dict(pe=30.0, da=1.0, n_t=4, n_species=4))
    g = np.full((60, 8), PORE, np.uint8)
    g[30:] = SOLID
    v = np.zeros((3, 60, 8), np.float32)
    v[0, :30] = 1.0
    adr("adr_sealed2d", p2, g, v, dict(pe=50.0, da=0.1, n_t=5, n_species=1))
    g = np.full((40, 6), PORE, np.uint8)
    v = np.zeros((3, 40, 6), np.float32)
    v[0] = 1.0
    adr("adr_nt11_2d", p2, g, v, dict(pe=100.0, da=1.0, n_t=11, n_species=1, steps=200))
    adr("adr_nt2_2d", p2, g, v, dict(pe=100.0, da=1.0, n_t=2, n_species=1))
    adr("adr_nt1_2d", p2, g, v, dict(pe=100.0, da=1.0, n_t=1, n_species=1, steps=150))

    adr("adr_disks2d_first", p2, gd, v2d_disks, dict(pe=10.0, da=1.0, n_t=5, n_species=1,
                                                     steps=600))
    monod = su.Chemistry(names=["C"], inlet=[1.0], c_init=[0.0], d_rel=[1.0],
                         immobile=[False], ks_donor=0.5)
    adr("adr_spheres3d_monod", p3, gs, v3d_spheres, dict(pe=10.0, da=1.0, n_t=5, n_species=1,
                                                         steps=300, chem=monod))
    adr("adr_spheres3d_ns4", p3, gs, v3d_spheres, dict(pe=10.0, da=2.0, n_t=4, n_species=4,
                                                       steps=250, da_abio=0.5))
    # biofilm + per-chemical diffusivities + abiotic surface reaction making a product
    gb, nb = coat_with_biofilm(gs, 3, 1)
    chem_bf = su.Chemistry(names=["Ac", "A", "P", "Bio"], inlet=[1.0, 0.8, 0.0, np.nan],
                           c_init=[0.0, 0.05, 0.0, 0.1], d_rel=[1.0, 1.3, 0.7, 0.0],
                           immobile=[False, False, False, True], ks_donor=0.2,
                           ks_acceptor=0.15, alpha=0.4, yield_=0.04, decay_lattice=0.006,
                           biomass_coupled=True, abiotic_surface_only=True,
                           d_biofilm_rel=[0.5, 0.6, 0.4, 0.0], biofilm_code=3,
                           seed_in_biofilm=True, abiotic_index=2, abiotic_product_index=1,
                           source="golden biofilm")
    adr("adr_spheres3d_biofilm", p3, gb, v3d_spheres, dict(pe=20.0, da=3.0, n_t=5, n_species=4,
                                                           steps=300, chem=chem_bf,
                                                           da_abio=2.0))
    # run to convergence with the stop rule (2D channel, ns=4), and capped
    g = np.full((40, 8), PORE, np.uint8)
    v = np.zeros((3, 40, 8), np.float32)
    v[0] = 1.0
    adr("adr_chan2d_capped", p2, g, v, dict(pe=30.0, da=1.0, n_t=6, n_species=4, max_steps=1500))
    # float64 twin on two cases
    f64 = float64_twin(p3)
    adr("adr64_spheres3d_monod", f64, gs, v3d_spheres, dict(pe=10.0, da=1.0, n_t=5, n_species=1,
                                                            steps=300, chem=monod))
    adr("adr64_spheres3d_ns4", f64, gs, v3d_spheres, dict(pe=10.0, da=2.0, n_t=4, n_species=4,
                                                          steps=250, da_abio=0.5))


if __name__ == "__main__":
    main()
