"""The oracle against the reference's own outputs (golden vectors).

Pins the CPU restatement in oracle/ before any CUDA result is compared with
it: the float32 transport must be bit-identical to the reference (same steps,
same snapshots, same t_norm), the float64 twin likewise, and the float64 flow
equal to the reference's float32-cast field within a few float32 ulps.
"""

import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from oracle import prtlb_oracle as O
from oracle.pairwise import pairwise_mean, pairwise_sum, tree

FLOW = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "flow_*.npz")))
ADR32 = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "adr_*.npz")))
ADR64 = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "adr64_*.npz")))


def golden_chem(name, ns):
    """Chemistry objects the fixtures were made with (see make_golden.py)."""
    from prtlb_gpu.chemistry import Chemistry
    if "monod" in name:
        return Chemistry(names=["C"], inlet=[1.0], c_init=[0.0], d_rel=[1.0], immobile=[False],
                         ks_donor=0.5)
    if "biofilm" in name:
        return Chemistry(names=["Ac", "A", "P", "Bio"], inlet=[1.0, 0.8, 0.0, np.nan],
                         c_init=[0.0, 0.05, 0.0, 0.1], d_rel=[1.0, 1.3, 0.7, 0.0],
                         immobile=[False, False, False, True], ks_donor=0.2, ks_acceptor=0.15,
                         alpha=0.4, yield_=0.04, decay_lattice=0.006, biomass_coupled=True,
                         abiotic_surface_only=True, d_biofilm_rel=[0.5, 0.6, 0.4, 0.0],
                         biofilm_code=3, seed_in_biofilm=True, abiotic_index=2,
                         abiotic_product_index=1, source="golden biofilm")
    return None


def adr_kwargs(z, name):
    kw = dict(pe=float(z["arg_pe"]), da=float(z["arg_da"]), n_t=int(z["arg_n_t"]),
              n_species=int(z["arg_n_species"]))
    if "arg_steps" in z:
        kw["steps"] = int(z["arg_steps"])
    if "arg_max_steps" in z:
        kw["max_steps"] = int(z["arg_max_steps"])
    if "arg_da_abio" in z:
        kw["da_abio"] = float(z["arg_da_abio"])
    kw["chem"] = golden_chem(name, kw["n_species"])
    return kw


@pytest.mark.parametrize("name", FLOW)
def test_flow_oracle_matches_reference(name):
    z = load_golden(name)
    info = {}
    v = O.stokes(z["g"], nit=int(z["nit"]), force=float(z["force"]), tau_lb=float(z["tau"]),
                 tol=float(z["tol"]), info=info)
    assert info["flow_iters"] == int(z["info_flow_iters"])
    assert info["flow_converged"] == bool(z["info_flow_converged"])
    ref = z["v"].astype(np.float64)
    err = np.abs(v - ref).max() / np.abs(ref).max()
    assert err < 1e-6, err


@pytest.mark.parametrize("name", ADR32)
def test_adr_oracle_bit_identical_to_reference(name):
    z = load_golden(name)
    kw = adr_kwargs(z, name)
    info = {}
    prog = []
    out, tn = O.solve_adr(z["mat"], z["vel"], info=info, on_progress=lambda *a: prog.append(a),
                          **kw)
    assert info["steps"] == int(z["info_steps"])
    assert info["ladder"] == int(z["info_ladder"])
    assert info["dt"] == float(z["info_dt"])
    assert np.array_equal(tn, z["t_norm"])
    assert np.array_equal(out, z["out"]), np.abs(out - z["out"]).max()
    assert np.array_equal(np.asarray(prog, np.float64).reshape(-1, 4), z["progress"])


@pytest.mark.parametrize("name", ADR64)
def test_adr_oracle_float64_twin(name):
    z = load_golden(name)
    kw = adr_kwargs(z, name)
    info = {}
    out, tn = O.solve_adr(z["mat"], z["vel"], info=info, dtype=np.float64, **kw)
    assert info["steps"] == int(z["info_steps"])
    assert np.array_equal(tn, z["t_norm"])
    assert np.array_equal(out, z["out"]), np.abs(out - z["out"]).max()


@pytest.mark.parametrize("n", [0, 1, 7, 8, 9, 127, 128, 129, 1000, 4097, 65536, 123457])
def test_pairwise_order_is_numpys(n):
    rng = np.random.default_rng(n)
    a = (rng.random(n) * rng.random(n) ** 3).astype(np.float32)
    assert pairwise_sum(a) == np.add.reduce(a)
    if n:
        assert pairwise_mean(a) == np.float32(a.mean())
    assert sum(k for _, k in tree(n)) == n
