"""Transport on the GPU: drop-in ``solve_adr``.

The set-up (solve_adr 9.1-9.3, prtlb_3d.py:831-993) turns Pe, Da and the
chemistry into float32 lattice numbers on the host, with the same numpy
scalar types and promotion the reference uses, so the time step, check
interval and every coefficient are the reference's to the last bit.  The
per-voxel work -- face tables, the fused transport + reaction step, the
snapshot ladder and the convergence means -- runs in libprtlb.so as one CUDA
graph with a device-side while condition.  Snapshot picking and the ``info``
dict (prtlb_3d.py:1550-1595) are host logic over the step numbers.

Keyword-only additions: ``device`` and ``ctx``.
"""

import ctypes

import numpy as np

from . import _lib
from .chemistry import default_chemistry

SOLID, WALL, PORE = 0, 1, 2
ATTACHED = 3


def _nearest_unused(i, used, n):
    """The ladder index closest to i not taken yet (prtlb_3d.py:716-722)."""
    for d in range(n):
        for j in (i - d, i + d):
            if 0 <= j < n and j not in used:
                return j
    return i


def _wanted_steps(total, n_t):
    """Log-spaced snapshot steps from 0 to total (prtlb_3d.py:725-737):
    one snapshot is the end, two are the ends, more are 0 plus a geometric
    ladder from total // 400 to total."""
    if n_t <= 1:
        return np.array([total], int)
    if n_t == 2:
        return np.array([0, total], int)
    tail = np.geomspace(max(total // 400, 1), max(total, 1), n_t - 1)
    return np.round(np.concatenate([[0.0], tail])).astype(int)


def _name(ch, j):
    try:
        return str(ch.names[j])
    except Exception:
        return ("the donor", "the acceptor", "the product", "the biomass")[j] if j < 4 \
            else "chemical %d" % j


def _harmonic(a1, a2):
    """Face diffusivity 2 a1 a2 / (a1 + a2), 0 unless both positive, float32."""
    a1 = np.float32(a1)
    a2 = np.float32(a2)
    if not (a1 > 0 and a2 > 0):
        return np.float32(0.0)
    return np.float32(2 * a1 * a2 / (a1 + a2))


class AdrSetup(object):
    """Everything solve_adr derives before its time loop."""


def solute_mask(mat, chem):
    """(m, biofilm): voxels that hold solute (pore, plus biofilm when the
    chemistry names a biofilm code) and the biofilm voxels (9.1)."""
    mat = np.asarray(mat)
    bf_code = getattr(chem, "biofilm_code", None) if chem is not None else None
    m = (mat == PORE)
    biofilm = np.zeros(m.shape, bool)
    if bf_code is not None:
        biofilm = (mat == bf_code)
        m = m | biofilm
    return m, biofilm


def velocity_stats_host(mat, vel, chem=None):
    """The velocity statistics of prt_adr_stage, computed with numpy on the
    host (float32 means in numpy's order, per-axis max |v| over the solute)."""
    m, biofilm = solute_mask(mat, chem)
    nd = m.ndim
    vel = np.asarray(vel, np.float32)
    sp = np.sqrt((vel[:nd] ** 2).sum(0))
    st = {"solute_voxels": int(m.sum()), "biofilm_voxels": int(biofilm.sum()),
          "mean_axial": np.float32(vel[0][m].mean()) if m.any() else np.float32(0.0),
          "mean_speed": np.float32(sp[m].mean()) if m.any() else np.float32(0.0),
          "vmax": [np.float32(np.abs(vel[a][m]).max()) if m.any() else np.float32(0.0)
                   for a in range(nd)] + [np.float32(0.0)] * (3 - nd)}
    return st


def stats_dict(st):
    """A prt_adr_stats struct as the dict velocity_stats_host returns."""
    return {"solute_voxels": int(st.solute_voxels), "biofilm_voxels": int(st.biofilm_voxels),
            "mean_axial": np.float32(st.mean_axial), "mean_speed": np.float32(st.mean_speed),
            "vmax": [np.float32(st.vmax[a]) for a in range(3)]}


def prepare(shape, stats, pe, da, n_species=2, chem=None, da_abio=0.0, mat=None):
    """solve_adr's set-up: velocity scale, lattice numbers, time step.

    `shape` is the grid shape and `stats` the velocity statistics
    (prt_adr_stage on the device, or velocity_stats_host).  `mat` is only
    needed for the surface weights of a surface-only abiotic reaction.
    Returns an AdrSetup with the C parameter block ``params`` and the host
    quantities the info dict reports."""
    S = AdrSetup()
    shape = tuple(int(n) for n in shape)
    bf_code = getattr(chem, "biofilm_code", None) if chem is not None else None
    nd = len(shape)
    if nd not in (2, 3):
        raise ValueError("grid must be 2D or 3D, got %dD" % nd)
    nx = shape[0]
    any_m = stats["solute_voxels"] > 0
    # velocity scale: mean axial pore velocity, or mean speed when the axial
    # mean is not meaningful (float32 numpy means, as the reference takes them)
    mean_axial = float(stats["mean_axial"]) if any_m else 0.0
    mean_speed = float(stats["mean_speed"]) if any_m else 0.0
    u_scale = mean_axial if mean_axial > 0.1 * mean_speed else mean_speed
    us = max(u_scale, 1e-30)
    us32 = np.float32(us)

    ns = int(n_species)
    ch = default_chemistry(ns) if chem is None else chem.truncate(ns)
    if len(ch.names) != ns:
        raise ValueError("the chemistry describes %d chemicals but %d were asked for"
                         % (len(ch.names), ns))
    if ns > _lib.PRT_MAX_SPECIES:
        raise ValueError("at most %d chemicals are supported" % _lib.PRT_MAX_SPECIES)
    l_ref = float(getattr(ch, "l_ref_voxels", None) or nx)
    D = np.float32(l_ref / max(pe, 1e-6))
    pe_grid = float(pe) / l_ref
    if pe_grid > 2.0:
        print("     WARNING: Peclet %.4g on %d voxels is a grid Peclet number of %.1f.\n"
              "              The front is thinner than the mesh; the sample will behave\n"
              "              as though its Peclet number were lower than %.4g. Use a\n"
              "              longer domain, or a lower Peclet number."
              % (pe, int(l_ref), pe_grid, pe), flush=True)
    k = np.float32(da / l_ref)
    ka = np.float32(max(da_abio, 0.0) / l_ref)
    j_ab = getattr(ch, "abiotic_index", 2)
    if ka > 0 and j_ab >= ns:
        raise ValueError(
            "an abiotic Damkohler number of %g was given, but it consumes chemical %d (%s) "
            "and this run has only %d chemicals, so the reaction cannot happen. Ask for at "
            "least %d chemicals, or set the abiotic reactant to one that is in the run, or "
            "set the abiotic Damkohler number to zero."
            % (da_abio, j_ab, _name(ch, j_ab), ns, j_ab + 1))
    kd = np.float32(ch.decay_for(l_ref))
    immobile = np.asarray(ch.immobile, bool)
    d_rel = np.asarray(ch.d_rel, np.float32).copy()
    d_rel[immobile] = 0.0
    has_bf = stats["biofilm_voxels"] > 0
    if has_bf:
        d_bf = np.asarray(ch.d_biofilm_rel, np.float32).copy()
        d_bf[immobile] = 0.0
        d_worst = float(max(d_rel.max(), d_bf.max()))
    else:
        d_bf = d_rel.copy()
        d_worst = float(d_rel.max())
    dmax = float(D) * float(max(d_worst, 1.0))
    # largest |u| per axis after normalisation: division by a positive
    # float32 is monotone, so max(|v|)/s equals max(|v|/s) bit for bit.  The
    # per-axis maxima are numpy float32 scalars summed from the integer 0, so
    # the sum is a float32 sum, as in the reference.
    umax32 = 0
    for ax in range(nd):
        top = np.float32(np.float32(stats["vmax"][ax]) / us32)
        umax32 = umax32 + max(top, np.float32(0.0))
    umax = float(umax32)
    k_lin = float(k)
    if ch.ks_donor > 0:
        k_lin = max(k_lin, float(k) / float(ch.ks_donor))
    if ns > 1 and ch.ks_acceptor > 0:
        k_lin = max(k_lin, float(k) / float(ch.ks_acceptor))
    sorp = getattr(ch, "sorption", None)
    k_sorp = np.float32(0.0)
    if sorp is not None:
        if not (0 <= sorp.dissolved < ns and 0 <= sorp.sorbed < ns):
            raise ValueError("sorption refers to a chemical outside this run")
        if not immobile[sorp.sorbed]:
            raise ValueError("the sorbed chemical must be immobile")
        if not sorp.kd > 0:
            raise ValueError("the sorption partition coefficient K_d must be positive")
        k_sorp = np.float32(max(sorp.da, 0.0) / l_ref)
        k_lin = k_lin + float(k_sorp) * (1.0 + 1.0 / sorp.kd)
    # same operand types as the reference: the trailing float32 terms make
    # the whole denominator a float32 sum
    dt = np.float32(0.4 / (umax + 2.0 * nd * dmax + k_lin + ka + kd + 1e-30))

    fed = np.asarray(ch.inlet, np.float32)
    moving = [j for j in range(ns) if not immobile[j]]
    surf_sum = 0.0
    if ka > 0 and getattr(ch, "abiotic_surface_only", False) and mat is not None:
        surf_sum = float(_surface_weights(solute_mask(mat, chem)[0]).sum())

    P = _lib.AdrParams()
    P.nd = nd
    for i, n in enumerate(shape):
        P.dims[i] = int(n)
    P.ns = ns
    P.moving_mask = sum(1 << j for j in moving)
    P.pinned_mask = sum(1 << j for j in moving if fed[j] == fed[j])
    P.pore_code = PORE
    P.biofilm_code = -1 if bf_code is None else int(bf_code)
    P.u_scale = float(us32)
    P.dt = float(dt)
    c_init = np.asarray(ch.c_init, np.float32)
    seed_bf = bool(getattr(ch, "seed_in_biofilm", False))
    for j in range(ns):
        P.feed[j] = float(fed[j]) if fed[j] == fed[j] else 0.0
        if not c_init[j]:
            P.init_mode[j] = 0
        elif j == ATTACHED and seed_bf and has_bf and immobile[j]:
            P.init_mode[j] = 2
        else:
            P.init_mode[j] = 1
        P.init_value[j] = float(c_init[j])
        dp = np.float32(d_rel[j] * D)
        db = np.float32(d_bf[j] * D) if has_bf else dp
        P.dface[j][0] = float(_harmonic(dp, dp))
        P.dface[j][1] = float(_harmonic(dp, db))
        P.dface[j][2] = float(_harmonic(db, db))
    biotic_on = bool(getattr(ch, "biotic_on", True))
    P.biotic_on = 1 if biotic_on else 0
    P.k = float(k)
    P.ks_donor_pos = 1 if ch.ks_donor > 0 else 0
    P.ks_donor = float(np.float32(ch.ks_donor))
    P.ks_acceptor_pos = 1 if ch.ks_acceptor > 0 else 0
    P.ks_acceptor = float(np.float32(ch.ks_acceptor))
    P.coupled = 1 if (getattr(ch, "biomass_coupled", False) and ns > 3 and c_init[3] > 0) else 0
    P.c3_init = float(np.float32(c_init[3])) if ns > 3 else 1.0
    P.neg_alpha = float(np.float32(-ch.alpha))
    P.alpha_cap = 1 if (ns > 1 and ch.alpha > 0) else 0
    P.alpha_dt = float(np.float32(float(ch.alpha) * dt))
    P.prod_coef = float(np.float32(1.0 - (ch.yield_ if ns > 3 else 0.0)))
    P.yield_ = float(np.float32(ch.yield_))
    P.kd = float(kd)
    P.abio_on = 1 if (ka > 0 and j_ab < ns) else 0
    P.j_ab = int(j_ab)
    j_mk = getattr(ch, "abiotic_product_index", None)
    P.j_mk = int(j_mk) if (j_mk is not None and j_mk < ns) else -1
    P.ka = float(ka)
    P.surface_only = 1 if getattr(ch, "abiotic_surface_only", False) else 0
    if sorp is not None:
        P.sorp_on = 1
        P.j_c = sorp.dissolved
        P.j_s = sorp.sorbed
        P.k_sorp = float(k_sorp)
        P.inv_kd_sorp = float(np.float32(1.0 / sorp.kd))
    else:
        P.sorp_on = 0
        P.j_c = P.j_s = -1

    S.params = P
    S.shape = shape
    S.nbiofilm = int(stats["biofilm_voxels"])
    S.nd = nd
    S.ns = ns
    S.ch = ch
    S.dt = dt
    S.check = max(int(1.0 / float(dt)), 100)
    S.umax = umax
    S.dmax = dmax
    S.pe_grid = pe_grid
    S.l_ref = l_ref
    S.surf_sum = surf_sum
    S.u_scale = u_scale
    return S


def _surface_weights(m):
    """Closed faces per solute voxel / (2 nd), edge-replicated neighbours."""
    nd = m.ndim
    P = np.pad(m, [(1, 1)] * nd, mode="edge")
    nface = np.zeros(m.shape, np.float32)
    for ax in range(nd):
        lo = tuple(slice(0, -2) if j == ax else slice(1, -1) for j in range(nd))
        hi = tuple(slice(2, None) if j == ax else slice(1, -1) for j in range(nd))
        nface += (~P[lo]).astype(np.float32)
        nface += (~P[hi]).astype(np.float32)
    return np.where(m, nface / float(2 * nd), 0.0).astype(np.float32)


def stage_inputs(mat, vel, chem=None):
    """The uint8 material grid (pore and biofilm kept, the rest solid), the
    float32 (3,) + grid velocity and the AdrGeom that solve_adr stages."""
    mat8, geom = stage_geom(mat, chem)
    vel32 = np.asarray(vel, np.float32)
    if vel32.shape[0] < 3:
        pad = np.zeros((3,) + vel32.shape[1:], np.float32)
        pad[:vel32.shape[0]] = vel32
        vel32 = pad
    vel32 = np.ascontiguousarray(vel32[:3])
    return mat8, vel32, geom


def stage_geom(mat, chem=None):
    """The uint8 material grid and the AdrGeom of solve_adr's staging."""
    mat = np.asarray(mat)
    nd = mat.ndim
    bf_code = getattr(chem, "biofilm_code", None) if chem is not None else None
    if mat.dtype == np.uint8:
        mat8 = np.ascontiguousarray(mat)
    else:
        if bf_code is not None and not 0 <= int(bf_code) < 256:
            raise ValueError("the biofilm material code must fit in 0..255")
        keep = (mat == PORE) | ((mat == bf_code) if bf_code is not None else False)
        mat8 = np.where(keep, mat, SOLID).astype(np.uint8)
    geom = _lib.AdrGeom()
    geom.nd = nd
    for i, n in enumerate(mat.shape):
        geom.dims[i] = int(n)
    geom.pore_code = PORE
    geom.biofilm_code = -1 if bf_code is None else int(bf_code)
    return mat8, geom


def solve_adr(mat, vel, pe, da, n_t, n_species=2, steps=None, tol=2e-3, max_steps=100000,
              info=None, ratio=1.12, chem=None, da_abio=0.0, on_progress=None,
              *, device=None, ctx=None):
    """Advection, dispersion and reaction on the flow field ``vel`` through
    ``mat``.  Returns (out, t_norm): out (n_t, n_species) + grid float32,
    zero off the pore space; t_norm the true normalised time of each
    snapshot.  Arguments and ``info`` keys are those of the reference's
    solve_adr (prtlb_3d.py:781)."""
    mat = np.asarray(mat)
    nd = mat.ndim
    if nd not in (2, 3):
        raise ValueError("grid must be 2D or 3D, got %dD" % nd)
    ctx = ctx or _lib.default_context(device)
    L = _lib.lib()
    mat8, vel32, geom = stage_inputs(mat, vel, chem)
    st = _lib.AdrStats()
    ctx.lock.acquire()
    try:
        ctx.check(L.prt_adr_stage(ctx.handle, mat8.ctypes.data_as(ctypes.c_void_p),
                                  vel32.ctypes.data_as(ctypes.c_void_p), ctypes.byref(geom),
                                  ctypes.byref(st)))
        S = prepare(mat.shape, stats_dict(st), pe, da, n_species=n_species, chem=chem,
                    da_abio=da_abio, mat=mat)
        return _run(ctx, S, n_t, steps, tol, max_steps, info, ratio, da, da_abio, on_progress)
    finally:
        ctx.lock.release()


def run_params(S, steps, tol, max_steps, ratio):
    """The run block of solve_adr's loop: a fixed step count, or the stop
    rule with the `max_steps` cap (prtlb_3d.py:1460-1548)."""
    R = _lib.AdrRunParams()
    R.limit = int(steps) if steps is not None else int(max_steps)
    R.until_conv = 1 if steps is None else 0
    R.check = S.check
    R.tol = float(tol)
    R.ratio = float(ratio)
    return R


def ladder_steps(ctx):
    """Step numbers of the kept snapshots of a finished run."""
    L = _lib.lib()
    nkeep = ctypes.c_int32()
    ctx.check(L.prt_adr_ladder(ctx.handle, None, 0, ctypes.byref(nkeep)))
    ks = np.zeros(nkeep.value, np.int64)
    ctx.check(L.prt_adr_ladder(ctx.handle, ks.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                               nkeep.value, ctypes.byref(nkeep)))
    return ks


def pick(ks, n, n_t):
    """Ladder indices of the n_t output snapshots (prtlb_3d.py:1550-1568)."""
    total = int(max(n, 1))
    used, picked = set(), []
    for w in _wanted_steps(total, n_t):
        i = int(np.abs(ks - w).argmin())
        if i in used:
            i = _nearest_unused(i, used, len(ks))
        used.add(i)
        picked.append(i)
    return picked


def _loop(ctx, S, n_t, steps, tol, max_steps, ratio, on_progress):
    """Begin + run on a staged context, then pick the snapshots.  Returns
    (steps run, keep_steps, picked)."""
    L = _lib.lib()
    R = run_params(S, steps, tol, max_steps, ratio)
    res = _lib.AdrResult()
    err = []

    def _cb(_user, n, lim, mean0, change):
        try:
            on_progress(int(n), int(lim), float(mean0), float(change))
            return 0
        except BaseException as e:  # re-raised after the run unwinds
            err.append(e)
            return 1

    cb = _lib.PROGRESS_CB(_cb) if on_progress is not None else _lib.PROGRESS_CB()
    ctx.check(L.prt_adr_begin(ctx.handle, ctypes.byref(S.params)))
    rc = L.prt_adr_run(ctx.handle, ctypes.byref(R), cb, None, ctypes.byref(res))
    if rc == _lib.PRT_E_CANCELLED and err:
        L.prt_adr_end(ctx.handle)
        raise err[0]
    ctx.check(rc)
    n = int(res.steps)
    ks = ladder_steps(ctx)
    return n, ks, pick(ks, n, n_t)


def _run(ctx, S, n_t, steps, tol, max_steps, info, ratio, da, da_abio, on_progress):
    """solve_adr's loop and outputs on a staged context (lock held)."""
    n, ks, picked = _loop(ctx, S, n_t, steps, tol, max_steps, ratio, on_progress)
    return outputs(ctx, S, n_t, n, ks, picked, steps, max_steps, info, da, da_abio)


def outputs(ctx, S, n_t, n, ks, picked, steps, max_steps, info, da, da_abio, end=True):
    """(out, t_norm) and the info keys of a finished run (prtlb_3d.py:1565-1595);
    ends the transport state of the context unless `end` is false."""
    L = _lib.lib()
    total = int(max(n, 1))
    repeated = n_t - len(set(picked))
    out = np.zeros((n_t, S.ns) + S.shape, np.float32)
    cache = {}
    for j, i in enumerate(picked):
        if i not in cache:
            buf = np.empty((S.ns,) + S.shape, np.float32)
            ctx.check(L.prt_adr_fetch(ctx.handle, int(i), buf.ctypes.data_as(ctypes.c_void_p)))
            cache[i] = buf
        out[j] = cache[i]
    if end:
        L.prt_adr_end(ctx.handle)
    t_norm = (ks[picked].astype(np.float32) / total).astype(np.float32)
    hit_cap = steps is None and n >= max_steps
    if info is not None:
        info["converged"] = not (hit_cap or steps is not None)
        info["steps"] = total
        info["dt"] = float(S.dt)
        info["ladder"] = len(ks)
        info["chemistry"] = getattr(S.ch, "source", "")
        info["da_bio"] = float(da)
        info["da_abio"] = float(da_abio)
        info["dt_limited_by"] = ("advection" if S.umax > 2.0 * S.nd * S.dmax else "diffusion")
        info["biofilm_voxels"] = int(S.nbiofilm)
        info["grid_peclet"] = float(S.pe_grid)
        info["l_ref_voxels"] = float(S.l_ref)
        info["surface_voxels"] = float(S.surf_sum)
        info["repeated_snapshots"] = int(max(repeated, 0))
    return out, t_norm


def _run_device(ctx, S, n_t, d_out, steps=None, tol=2e-3, max_steps=100000, ratio=1.12):
    """The loop on a staged context with the snapshots copied into the device
    buffer `d_out` ((n_t, ns) + grid float32).  Returns the steps run."""
    L = _lib.lib()
    n, ks, picked = _loop(ctx, S, n_t, steps, tol, max_steps, ratio, None)
    nbytes = S.ns * int(np.prod(S.shape)) * 4
    for j, i in enumerate(picked):
        ctx.check(L.prt_adr_fetch_dev(ctx.handle, int(i), ctypes.c_void_p(int(d_out) + j * nbytes)))
    return n
