"""The dimensionless chemistry that solve_adr consumes.

solve_adr accepts the reference's own ``settings_and_units.Chemistry``
(3D/tools/settings_and_units.py:1834-1929) by duck typing: only attributes
are read.  This module provides an equivalent class for callers that do not
have the reference installed, with the same attribute names and meaning, the
same ``truncate`` / ``decay_for`` behaviour, and the same built-in fallback
(``default_chemistry``, settings_and_units.py:1934-1947).

One extension has no reference counterpart: ``sorption``, a reversible
sorption exchange between a dissolved chemical and an immobile sorbed one
(see ``Sorption``).
"""

import numpy as np


class Sorption(object):
    """Reversible linear sorption: S <-> C with r = k_a (C - S / K_d).

    dissolved   index of the dissolved chemical C (transported)
    sorbed      index of the sorbed chemical S (must be immobile)
    kd          the linear partition coefficient K_d (S/C at equilibrium)
    da          Damkohler number of the exchange; the lattice rate is da / l_ref

    Not part of the reference: PRT-LB names sorption only as a DeepONet
    parameter label (prt_core/reactions.py:190-212) and has no sorption
    kinetics, so this term is pinned by its own known answers (closed batch
    reaches S/C = K_d, C + S is conserved, retardation 1 + K_d).
    """

    def __init__(self, dissolved=0, sorbed=1, kd=0.5, da=1.0):
        self.dissolved = int(dissolved)
        self.sorbed = int(sorbed)
        self.kd = float(kd)
        self.da = float(da)


class Chemistry(object):
    """Per-chemical feed, start value, diffusivity ratio and mobility, plus the
    reaction constants; attribute for attribute what solve_adr reads."""

    def __init__(self, names, inlet, c_init, d_rel, immobile,
                 ks_donor=0.0, ks_acceptor=0.15, alpha=0.4, yield_=0.04,
                 da_decay=None, decay_lattice=None, source="built in",
                 biomass_coupled=False, abiotic_surface_only=False,
                 d_biofilm_rel=None, biofilm_code=None, seed_in_biofilm=False,
                 abiotic_index=2, biotic_on=True, l_ref_voxels=None,
                 abiotic_product_index=None, sorption=None):
        self.names = [str(n) for n in names]
        n = len(self.names)
        self.inlet = np.asarray(inlet, np.float32)
        self.c_init = np.asarray(c_init, np.float32)
        self.d_rel = np.asarray(d_rel, np.float32)
        self.immobile = np.asarray(immobile, bool)
        for arr, label in ((self.inlet, "inlet"), (self.c_init, "c_init"),
                           (self.d_rel, "d_rel"), (self.immobile, "immobile")):
            if arr.shape != (n,):
                raise ValueError("chemistry: %s has %d entries but there are %d chemicals"
                                 % (label, arr.size, n))
        self.ks_donor = float(ks_donor)
        self.ks_acceptor = float(ks_acceptor)
        self.alpha = float(alpha)
        self.yield_ = float(yield_)
        self.da_decay = None if da_decay is None else float(da_decay)
        self.decay_lattice = None if decay_lattice is None else float(decay_lattice)
        self.biomass_coupled = bool(biomass_coupled)
        self.abiotic_surface_only = bool(abiotic_surface_only)
        self.d_biofilm_rel = (self.d_rel.copy() if d_biofilm_rel is None
                              else np.asarray(d_biofilm_rel, np.float32))
        self.biofilm_code = None if biofilm_code is None else int(biofilm_code)
        self.seed_in_biofilm = bool(seed_in_biofilm)
        self.abiotic_index = int(abiotic_index)
        self.abiotic_product_index = (None if abiotic_product_index is None
                                      else int(abiotic_product_index))
        self.biotic_on = bool(biotic_on)
        self.l_ref_voxels = None if l_ref_voxels is None else float(l_ref_voxels)
        self.source = source
        self.sorption = sorption

    def decay_for(self, nx):
        """Biomass decay in lattice units: given directly, or a Damkohler / nx."""
        if self.decay_lattice is not None:
            return float(self.decay_lattice)
        return float((self.da_decay or 0.0) / max(nx, 1))

    def truncate(self, ns):
        """The first ns chemicals (at least 1, at most all of them)."""
        ns = max(1, min(int(ns), len(self.names)))
        return Chemistry(self.names[:ns], self.inlet[:ns], self.c_init[:ns],
                         self.d_rel[:ns], self.immobile[:ns],
                         ks_donor=self.ks_donor, ks_acceptor=self.ks_acceptor,
                         alpha=self.alpha, yield_=self.yield_, da_decay=self.da_decay,
                         decay_lattice=self.decay_lattice, source=self.source,
                         biomass_coupled=self.biomass_coupled,
                         abiotic_surface_only=self.abiotic_surface_only,
                         d_biofilm_rel=self.d_biofilm_rel[:ns],
                         biofilm_code=self.biofilm_code,
                         seed_in_biofilm=self.seed_in_biofilm,
                         abiotic_index=self.abiotic_index, biotic_on=self.biotic_on,
                         l_ref_voxels=self.l_ref_voxels,
                         abiotic_product_index=self.abiotic_product_index,
                         sorption=self.sorption)

    def describe(self):
        """One line per chemical: its name, feed, start value, diffusivity
        ratio and whether it is transported."""
        out = []
        for i, nm in enumerate(self.names):
            feed = "unfed" if self.inlet[i] != self.inlet[i] else "feed=%g" % self.inlet[i]
            out.append("%s: %s, c0=%g, D/D_ref=%g, %s"
                       % (nm, feed, self.c_init[i], self.d_rel[i],
                          "immobile" if self.immobile[i] else "mobile"))
        return "; ".join(out)


def default_chemistry(n_species=2):
    """The built-in chemistry: donor, acceptor, product, attached biomass.

    Feeds 1, 1, 0 and none; biomass 0.1 at the start; one shared diffusivity
    for the three solutes; acceptor half-saturation 0.15; stoichiometry 0.4;
    yield 0.04; decay 0.006 per lattice time (settings_and_units.py:1934-1947,
    the constants prtlb_3d.py BLOCK 5 documents)."""
    ns = max(1, min(int(n_species), 4))
    nan = np.float32(np.nan)
    return Chemistry(
        names=["Ac", "A", "P", "Bio"][:ns],
        inlet=np.array([1.0, 1.0, 0.0, nan], np.float32)[:ns],
        c_init=np.array([0.0, 0.0, 0.0, 0.1], np.float32)[:ns],
        d_rel=np.array([1.0, 1.0, 1.0, 0.0], np.float32)[:ns],
        d_biofilm_rel=np.array([1.0, 1.0, 1.0, 0.0], np.float32)[:ns],
        immobile=np.array([False, False, False, True])[:ns],
        ks_donor=0.0, ks_acceptor=0.15, alpha=0.4, yield_=0.04,
        decay_lattice=0.006, source="built in")


def monod_chemistry(ks=0.5):
    """Single-substrate Monod: one fed, mobile solute consumed at
    k C / (Ks + C) (the published 'monod' species ['C'])."""
    return Chemistry(names=["C"], inlet=[1.0], c_init=[0.0], d_rel=[1.0],
                     immobile=[False], ks_donor=float(ks), source="monod")


def first_order_chemistry():
    """First-order irreversible uptake: R = k C (ks_donor = 0, one chemical)."""
    return Chemistry(names=["C"], inlet=[1.0], c_init=[0.0], d_rel=[1.0],
                     immobile=[False], ks_donor=0.0, source="first order")


def reversible_sorption_chemistry(kd=0.5, da=1.0):
    """Dissolved C (fed, mobile) exchanging with sorbed S (immobile), no
    biotic reaction: r = k_a (C - S/K_d)."""
    return Chemistry(names=["C", "S"], inlet=[1.0, np.nan], c_init=[0.0, 0.0],
                     d_rel=[1.0, 0.0], immobile=[False, True], biotic_on=False,
                     source="reversible sorption",
                     sorption=Sorption(dissolved=0, sorbed=1, kd=kd, da=da))
