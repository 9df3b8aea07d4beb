"""check_physics: the post-run sanity rules of the reference.

Restates 3D/tools/prtlb_3d.py:1632-1843 (BLOCK 10): finite, per-chemical
upper bounds, non-negative, not silently zero, reactant present when a rate
was asked for, no checkerboard along the flow, no wrap-around, no chemical
that is a rescaled copy of the donor.  Returns the list of complaints, empty
for a sound run.  It runs on the arrays solve_adr returned.

The statistics the rules read come from NumPy on the host, or with
on_gpu=True from reductions in libprtlb (prt_physics_*: extremes and counts
exactly, the donor correlations in float64), so a long run is judged
without a pass of NumPy over every snapshot.  The rules and messages are
the same code either way.
"""

import ctypes
import math

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


class _HostStats(object):
    """What the rules read, from NumPy on the result `out` and pore mask m."""

    def __init__(self, out, m):
        self.out, self.m = out, m
        self.ns = out.shape[1]
        self.finite = bool(np.isfinite(out).all())
        if not self.finite:
            self.n_nan, self.n_inf = int(np.isnan(out).sum()), int(np.isinf(out).sum())
            return
        self.any_pore = bool(m.any())
        if self.any_pore:
            self.hi = [float(out[:, j][:, m].max()) for j in range(self.ns)]
            self.lo = [float(out[:, j][:, m].min()) for j in range(self.ns)]
            self.final_absmax = [float(np.abs(out[-1, j][m]).max()) for j in range(self.ns)]
            self.all_absmax = [float(np.abs(out[:, j][:, m]).max()) for j in range(self.ns)]
        # checkerboard: neighbouring differences along x alternating in sign
        f = out[-1, 0]
        d = np.where(m[1:] & m[:-1], f[1:] - f[:-1], 0.0)
        trip = (m[2:] & m[1:-1] & m[:-2])
        self.n_triples = int(trip.sum())
        self.n_flips = int(((np.sign(d[1:]) * np.sign(d[:-1]) < 0) & trip).sum())
        # causality: the donor on the mid-plane and the outlet plane
        nx = m.shape[0]
        donor = out[:, 0]
        self.mid = donor[:, nx // 2].reshape(donor.shape[0], -1).max(1)
        self.end = donor[:, nx - 1].reshape(donor.shape[0], -1).max(1)

    def copy_test(self, j):
        """Whether chemical j is a rescaled copy of the donor over the pore of
        every snapshot: (correlation, it is), or None when either is flat."""
        a0 = self.out[:, 0][:, self.m].ravel()
        aj = self.out[:, j][:, self.m].ravel()
        if a0.std() < 1e-9 or aj.std() < 1e-9:
            return None
        r = float(np.corrcoef(a0, aj)[0, 1])
        scale = aj.std() / max(a0.std(), 1e-12)
        return r, r > 0.9999 and float(np.abs(aj - scale * a0).max()) < 1e-4


class _DeviceStats(object):
    """The same statistics from libprtlb's reductions."""

    def __init__(self, out, mat, ctx):
        from . import _lib
        self.L, self.ctx = _lib.lib(), ctx
        self.ns, n_t = out.shape[1], out.shape[0]
        if n_t > 256:
            raise ValueError("on_gpu judges at most 256 snapshots")
        mat8 = np.ascontiguousarray(mat, np.uint8)
        out32 = np.ascontiguousarray(out, np.float32)
        self.dims = (ctypes.c_int32 * 3)(*(list(mat.shape) + [1] * (3 - mat.ndim)))
        self.args = (mat.ndim, self.dims, n_t, self.ns)
        st = _lib.PhysicsStats()
        with ctx.lock:
            ctx.check(self.L.prt_physics_stage(ctx.handle, out32.ctypes.data_as(ctypes.c_void_p),
                                               mat8.ctypes.data_as(ctypes.c_void_p), *self.args))
            ctx.check(self.L.prt_physics_stats_dev(ctx.handle, None, None, *self.args, PORE,
                                                   ctypes.byref(st)))
        self.finite = st.n_nan == 0 and st.n_inf == 0
        self.n_nan, self.n_inf = int(st.n_nan), int(st.n_inf)
        if not self.finite:
            return
        self.any_pore = bool(st.has_pore[0])
        ns = self.ns
        self.hi = [float(st.pore_max[j]) for j in range(ns)]
        self.lo = [float(st.pore_min[j]) for j in range(ns)]
        self.final_absmax = [float(st.final_absmax[j]) for j in range(ns)]
        self.all_absmax = [max(abs(self.hi[j]), abs(self.lo[j])) for j in range(ns)]
        self.n_triples, self.n_flips = int(st.n_triples), int(st.n_flips)
        self.mid = np.array(st.mid_max[:n_t], np.float32)
        self.end = np.array(st.end_max[:n_t], np.float32)

    def copy_test(self, j):
        mom = (ctypes.c_double * 6)()
        with self.ctx.lock:
            self.ctx.check(self.L.prt_physics_moments_dev(self.ctx.handle, None, None, *self.args,
                                                          PORE, int(j), mom))
        s0 = np.float32(math.sqrt(max(mom[3], 0.0)))
        sj = np.float32(math.sqrt(max(mom[4], 0.0)))
        if s0 < 1e-9 or sj < 1e-9:
            return None
        r = float(np.clip(mom[5] / math.sqrt(mom[3] * mom[4]), -1.0, 1.0))
        if not r > 0.9999:
            return r, False
        scale = sj / max(s0, 1e-12)
        dev = ctypes.c_float()
        with self.ctx.lock:
            self.ctx.check(self.L.prt_physics_maxdev_dev(self.ctx.handle, None, None, *self.args,
                                                         PORE, int(j), float(np.float32(scale)),
                                                         ctypes.byref(dev)))
        return r, float(dev.value) < 1e-4


def check_physics(out, mat, verbose=False, chem=None, da=None, da_abio=None, *,
                  on_gpu=False, device=None, ctx=None):
    """Complaints about a solve_adr result `out` (n_t, ns, *grid) on `mat`.
    on_gpu: compute the statistics with libprtlb's reductions."""
    mat = np.asarray(mat)
    m = (mat == PORE)
    out = np.asarray(out)
    ns = out.shape[1]
    if on_gpu:
        from . import _lib
        st = _DeviceStats(out, mat, ctx or _lib.default_context(device))
    else:
        st = _HostStats(out, m)
    bad = []

    def done():
        if verbose:
            for s in bad:
                print("     PHYSICS: " + s, flush=True)
        return bad

    if not st.finite:
        bad.append("the field is not finite: %d NaN and %d infinite values -- the "
                   "integration diverged" % (st.n_nan, st.n_inf))
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
    if st.any_pore:
        for j in range(ns):
            hi = st.hi[j]
            if caps[j] is not None and hi > 1.02 * max(caps[j], 1e-6):
                bad.append("%s reaches %.3f, above the %.3f it could be made from -- the "
                           "time step is unstable" % (_name(chem, j), hi, caps[j]))
            elif caps[j] is None and hi > 1e3 * max(_seen(chem, j), 1e-3):
                bad.append("%s reaches %.4g, a thousand times what it started from -- this "
                           "is runaway growth, not a solution" % (_name(chem, j), hi))
            lo = st.lo[j]
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
            if expect > 0 and st.final_absmax[j] <= 0.0:
                bad.append("%s is exactly zero in every voxel at the end of the run, though "
                           "%.3g of it was fed in or present at the start -- it has not been "
                           "solved, it has been lost" % (_name(chem, j), expect))

        # a rate was requested: its reactant must exist somewhere, some time
        if chem is not None:
            for rate, jr, what in ((da, 0, "biotic"),
                                   (da_abio, getattr(chem, "abiotic_index", 2), "abiotic")):
                if rate is None or float(rate) <= 0 or not (0 <= jr < ns):
                    continue
                if st.all_absmax[jr] <= 0.0:
                    bad.append("the %s reaction was given a Damkohler number of %.3g but the "
                               "chemical it consumes, %s, is zero in every voxel at every "
                               "time -- the reaction never happened, and that Damkohler "
                               "number is recorded against a run it had no effect on"
                               % (what, float(rate), _name(chem, jr)))

    # checkerboard: neighbouring differences along x alternating in sign
    if st.n_triples > 100:
        flips = float(st.n_flips) / float(st.n_triples)
        if flips > 0.45:
            bad.append("%.0f%% of neighbouring pore voxels along the flow disagree in sign -- "
                       "this is a checkerboard, not a concentration field" % (100 * flips))

    # causality: solute at the outlet while the mid-plane is still empty
    early = np.where((st.end > 1e-3) & (st.mid < 1e-6))[0]
    if chem is not None and chem.c_init[0] > 0:
        early = np.array([], int)
    if early.size:
        bad.append("solute is at the outlet while the mid-plane is still empty at snapshot "
                   "%d -- something is wrapping around" % early[0])

    # a second chemical that is only a rescaled copy of the first
    if ns > 1:
        for j in range(1, ns):
            res = st.copy_test(j)
            if res is None:
                continue
            r, copy = res
            if copy:
                bad.append("species %d is a rescaled copy of species 0 (correlation %.5f) -- "
                           "it is not a second chemical" % (j, r))
    return done()
