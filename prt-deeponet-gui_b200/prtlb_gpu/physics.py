"""check_physics: the post-run sanity rules of the reference, on the host.

Restates 3D/tools/prtlb_3d.py:1632-1843 (BLOCK 10): finite, per-chemical
upper bounds, non-negative, not silently zero, reactant present when a rate
was asked for, no checkerboard along the flow, no wrap-around, no chemical
that is a rescaled copy of the donor.  Returns the list of complaints, empty
for a sound run.  It runs on the arrays solve_adr returned.
"""

import numpy as np

PORE = 2


def _name(chem, j):
    try:
        return str(chem.names[j])
    except Exception:
        return ("the donor", "the acceptor", "the product", "the biomass")[j] if j < 4 \
            else "chemical %d" % j


def _seen(chem, j):
    """Largest of the feed and the start value of chemical j (NaN ignored)."""
    if chem is None:
        return 1.0
    vals = [float(v) for v in (chem.inlet[j], chem.c_init[j]) if v == v]
    return max(vals) if vals else 0.0


def check_physics(out, mat, verbose=False, chem=None, da=None, da_abio=None):
    """Complaints about a solve_adr result `out` (n_t, ns, *grid) on `mat`."""
    mat = np.asarray(mat)
    m = (mat == PORE)
    out = np.asarray(out)
    ns = out.shape[1]
    bad = []

    def done():
        if verbose:
            for s in bad:
                print("     PHYSICS: " + s, flush=True)
        return bad

    if not np.isfinite(out).all():
        bad.append("the field is not finite: %d NaN and %d infinite values -- the "
                   "integration diverged" % (int(np.isnan(out).sum()), int(np.isinf(out).sum())))
        return done()

    # upper bounds: what each chemical could at most have been made from
    caps = [None] * ns
    if chem is not None:
        donor_cap = _seen(chem, 0)
        caps[0] = donor_cap
        if ns > 1:
            caps[1] = _seen(chem, 1)
        if ns > 2:
            y = 0.0
            if ns > 3 and getattr(chem, "biotic_on", True):
                y = float(getattr(chem, "yield_", 0.0))
            caps[2] = _seen(chem, 2) + max(donor_cap * (1.0 - y), 0.0)
    else:
        for j in range(min(ns, 3)):
            caps[j] = 1.0
    if m.any():
        for j in range(ns):
            fj = out[:, j][:, m]
            hi = float(fj.max())
            if caps[j] is not None and hi > 1.02 * max(caps[j], 1e-6):
                bad.append("%s reaches %.3f, above the %.3f it could be made from -- the "
                           "time step is unstable" % (_name(chem, j), hi, caps[j]))
            elif caps[j] is None and hi > 1e3 * max(_seen(chem, j), 1e-3):
                bad.append("%s reaches %.4g, a thousand times what it started from -- this "
                           "is runaway growth, not a solution" % (_name(chem, j), hi))
            lo = float(fj.min())
            if lo < -1e-6:
                bad.append("%s reaches %.3g, which is negative" % (_name(chem, j), lo))

        # a chemical that was fed or present must not vanish everywhere
        for j in range(ns):
            expect = 1.0
            if chem is not None:
                fed_j = float(chem.inlet[j]) if chem.inlet[j] == chem.inlet[j] else 0.0
                expect = max(fed_j, float(chem.c_init[j]))
                if j > 1 and expect <= 0:
                    continue
            if expect > 0 and float(np.abs(out[-1, j][m]).max()) <= 0.0:
                bad.append("%s is exactly zero in every voxel at the end of the run, though "
                           "%.3g of it was fed in or present at the start -- it has not been "
                           "solved, it has been lost" % (_name(chem, j), expect))

        # a rate was requested: its reactant must exist somewhere, some time
        if chem is not None:
            for rate, jr, what in ((da, 0, "biotic"),
                                   (da_abio, getattr(chem, "abiotic_index", 2), "abiotic")):
                if rate is None or float(rate) <= 0 or not (0 <= jr < ns):
                    continue
                if float(np.abs(out[:, jr][:, m]).max()) <= 0.0:
                    bad.append("the %s reaction was given a Damkohler number of %.3g but the "
                               "chemical it consumes, %s, is zero in every voxel at every "
                               "time -- the reaction never happened, and that Damkohler "
                               "number is recorded against a run it had no effect on"
                               % (what, float(rate), _name(chem, jr)))

    # checkerboard: neighbouring differences along x alternating in sign
    f = out[-1, 0]
    d = np.where(m[1:] & m[:-1], f[1:] - f[:-1], 0.0)
    trip = (m[2:] & m[1:-1] & m[:-2])
    if trip.sum() > 100:
        flips = float(((np.sign(d[1:]) * np.sign(d[:-1]) < 0) & trip).sum()) / float(trip.sum())
        if flips > 0.45:
            bad.append("%.0f%% of neighbouring pore voxels along the flow disagree in sign -- "
                       "this is a checkerboard, not a concentration field" % (100 * flips))

    # causality: solute at the outlet while the mid-plane is still empty
    nx = m.shape[0]
    donor = out[:, 0]
    mid = donor[:, nx // 2].reshape(donor.shape[0], -1).max(1)
    end = donor[:, nx - 1].reshape(donor.shape[0], -1).max(1)
    early = np.where((end > 1e-3) & (mid < 1e-6))[0]
    if chem is not None and chem.c_init[0] > 0:
        early = np.array([], int)
    if early.size:
        bad.append("solute is at the outlet while the mid-plane is still empty at snapshot "
                   "%d -- something is wrapping around" % early[0])

    # a second chemical that is only a rescaled copy of the first
    if ns > 1:
        a0 = out[:, 0][:, m].ravel()
        for j in range(1, ns):
            aj = out[:, j][:, m].ravel()
            if a0.std() < 1e-9 or aj.std() < 1e-9:
                continue
            r = float(np.corrcoef(a0, aj)[0, 1])
            scale = aj.std() / max(a0.std(), 1e-12)
            if r > 0.9999 and float(np.abs(aj - scale * a0).max()) < 1e-4:
                bad.append("species %d is a rescaled copy of species 0 (correlation %.5f) -- "
                           "it is not a second chemical" % (j, r))
    return done()
