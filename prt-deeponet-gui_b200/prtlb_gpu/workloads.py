"""Seeded synthetic request sets for the batched and served benchmarks.

Each request is a random periodic sphere pack (cubic edge and porosity
drawn per request, radius U[4, 7]) with a D3Q19 TRT fp32 flow solve run to
the reference's defaults (30000-iteration cap, tol 1e-6) and a transport
solve to the reference's stop rule, with Pe log-uniform in [0.1, 100], Da
log-uniform in [0.01, 10] and kinetics drawn from Monod (Ks 0.5), first-order
irreversible uptake and reversible sorption (Kd 0.5, one sorbed species).
"""

import numpy as np

from .batch import Request
from .chemistry import first_order_chemistry, monod_chemistry, reversible_sorption_chemistry
from .geometry import random_pack

KINETICS = ("monod", "first_order", "sorption")


def draw(rng, edge_lo, edge_hi):
    """One request's parameters."""
    return dict(edge=int(rng.integers(edge_lo, edge_hi + 1)),
                porosity=float(rng.uniform(0.35, 0.6)),
                pe=float(10.0 ** rng.uniform(-1.0, 2.0)),
                da=float(10.0 ** rng.uniform(-2.0, 1.0)),
                kinetics=KINETICS[int(rng.integers(0, 3))],
                seed=int(rng.integers(0, 2 ** 31 - 1)))


def make_request(d, nit=30000, flow_tol=1e-6, max_steps=100000, n_t=5, precision="fp32",
                 fetch=True, tag=None):
    """The Request of a parameter draw."""
    e = d["edge"]
    g = random_pack((e, e, e), d["porosity"], 4.0, 7.0, seed=d["seed"])
    if d["kinetics"] == "monod":
        chem, ns = monod_chemistry(0.5), 1
    elif d["kinetics"] == "first_order":
        chem, ns = first_order_chemistry(), 1
    else:
        chem, ns = reversible_sorption_chemistry(0.5, d["da"]), 2
    return Request(g, flow=dict(nit=nit, tol=flow_tol, precision=precision),
                   adr=dict(pe=d["pe"], da=d["da"], n_t=n_t, n_species=ns, chem=chem,
                            max_steps=max_steps),
                   tag=tag, fetch=fetch)


def request_set(n, edge_lo, edge_hi, seed=0, **kw):
    """n requests with edges uniform in [edge_lo, edge_hi] and the draws
    above; returns (requests, draws)."""
    rng = np.random.default_rng(seed)
    draws = [draw(rng, edge_lo, edge_hi) for _ in range(int(n))]
    return [make_request(d, tag=i, **kw) for i, d in enumerate(draws)], draws


def batched_set(n=48, seed=0, **kw):
    """The batched configuration: edges 24-96."""
    return request_set(n, 24, 96, seed=seed, **kw)


def served_set(n=48, seed=0, **kw):
    """The served configuration's requests: edges 32-160 (arrivals come from
    prtlb_gpu.serve.poisson_arrivals)."""
    return request_set(n, 32, 160, seed=seed, **kw)
