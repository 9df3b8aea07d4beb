"""NumPy restatement of PRT-LB's flow and transport solves (TEST ORACLE).

Test infrastructure only (see oracle/__init__.py).  Each function cites the
reference lines it restates; the arithmetic is the reference's, operation for
operation where that fixes the float32 result (transport), and to float64
round-off for the flow.
"""

import numpy as np

SOLID, WALL, PORE = 0, 1, 2
ATTACHED = 3

# ---------------------------------------------------------------------------
# lattices (prtlb_3d.py:370-375, prtlb_2d.py:391-394)
# ---------------------------------------------------------------------------
E3 = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
               [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1],
               [1, 0, -1], [-1, 0, 1], [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1]])
W3 = np.array([1 / 3.] + [1 / 18.] * 6 + [1 / 36.] * 12)
E2 = np.array([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, 1], [-1, -1], [1, -1]])
W2 = np.array([4 / 9.] + [1 / 9.] * 4 + [1 / 36.] * 4)


def _opposites(E):
    return np.array([int(np.where((E == -e).all(1))[0][0]) for e in E])


def trt_minus(om_p, magic=3.0 / 16.0):
    """omega- from the magic parameter (prtlb_3d.py:130-139)."""
    lam = 1.0 / float(om_p) - 0.5
    if lam <= 0:
        raise ValueError("tau must exceed 0.5")
    return 1.0 / (float(magic) / lam + 0.5)


def stokes(g, nit=30000, force=2e-6, tau_lb=0.8, magic=3.0 / 16.0, tol=1e-6, info=None,
           every=50, return_f=False):
    """TRT Stokes flow on a 2D or 3D material grid, float64.

    Restates stokes_d2q9 (prtlb_2d.py:348-486) and stokes_d3q19
    (prtlb_3d.py:348-456) with FlowConvergence (prtlb_3d.py:168-252):
    moments with +g/2 on u_x, u masked to the pore; TRT relaxation of the
    symmetric and antisymmetric parts; Guo term w_i (1 - om-/2) 3 g e_ix;
    solid voxels take the reversed ARRIVED populations; periodic streaming;
    stop when mean |u_x| over the pore changes by <= tol per `every` steps.
    Returns float32 (3, *grid), zero in solid (and info like the reference)."""
    g = np.asarray(g)
    nd = g.ndim
    E, W = (E3, W3) if nd == 3 else (E2, W2)
    opp = _opposites(E)
    Q = len(W)
    solid = g != PORE
    fluid = ~solid
    om_p = 1.0 / float(tau_lb)
    om_m = trt_minus(om_p, magic)
    gf = float(force)
    shape = g.shape
    f = np.ones((Q,) + shape) * W.reshape((Q,) + (1,) * nd)
    Ef = E.astype(np.float64)
    guo = W * (1 - 0.5 * om_m) * 3.0 * gf * Ef[:, 0]
    prev, iters, converged, change = None, 0, False, float("inf")
    for it in range(int(nit)):
        rho = f.sum(0)
        j = np.tensordot(Ef.T, f, axes=(1, 0))      # (nd, *grid)
        u = j / rho
        u[0] = (j[0] + 0.5 * gf) / rho
        u = u * fluid
        usq = (u * u).sum(0)
        eu = np.tensordot(Ef, u, axes=(1, 0))        # (Q, *grid)
        feq = W.reshape((Q,) + (1,) * nd) * rho * (1 + 3 * eu + 4.5 * eu * eu - 1.5 * usq)
        fo, feo = f[opp], feq[opp]
        post = (f - om_p * (0.5 * (f + fo) - 0.5 * (feq + feo))
                - om_m * (0.5 * (f - fo) - 0.5 * (feq - feo)))
        post += guo.reshape((Q,) + (1,) * nd)
        post[:, solid] = fo[:, solid]
        for i in range(Q):
            f[i] = np.roll(post[i], shift=tuple(int(s) for s in E[i]), axis=tuple(range(nd)))
        iters = it + 1
        if tol > 0 and iters % every == 0:
            um = float(np.abs(u[0][fluid]).mean()) if fluid.any() else 0.0
            if prev is not None:
                change = abs(um - prev) / max(abs(um), 1e-30)
                if change <= tol:
                    converged = True
                    prev = um
                    break
            prev = um
    if info is not None:
        info["flow_iters"] = iters
        info["flow_converged"] = bool(converged)
        info["flow_change"] = change
    rho = f.sum(0)
    j = np.tensordot(Ef.T, f, axes=(1, 0))
    v = np.zeros((3,) + shape)
    v[0] = (j[0] + 0.5 * gf) / rho
    for a in range(1, nd):
        v[a] = j[a] / rho
    v[:, solid] = 0.0
    if return_f:
        return v.astype(np.float32), v, f
    return v.astype(np.float32)


# ---------------------------------------------------------------------------
# transport (prtlb_3d.py:781-1595)
# ---------------------------------------------------------------------------
def _take(a, axis, off):
    """a shifted by `off` along `axis` with edge replication (no wrap)."""
    n = a.shape[axis]
    return np.take(a, np.clip(np.arange(n) + off, 0, n - 1), axis=axis)


def _muscl(up, upup, down):
    """Minmod-limited face value (prtlb_3d.py:650-705), division-free."""
    d1 = down - up
    d2 = up - upup
    return up + 0.5 * ((0.5 * (np.sign(d1) + np.sign(d2))) * np.minimum(np.abs(d1), np.abs(d2)))


def wanted_steps(total, n_t):
    """prtlb_3d.py:725-737."""
    if n_t <= 1:
        return np.array([total], int)
    if n_t == 2:
        return np.array([0, total], int)
    tail = np.geomspace(max(total // 400, 1), max(total, 1), n_t - 1)
    return np.round(np.concatenate([[0.0], tail])).astype(int)


def nearest_unused(i, used, n):
    """prtlb_3d.py:716-722."""
    for d in range(n):
        for j in (i - d, i + d):
            if 0 <= j < n and j not in used:
                return j
    return i


def default_chemistry(n_species=2):
    """The built-in chemistry numbers (settings_and_units.py:1934-1947), as a
    plain namespace for the oracle."""
    class C(object):
        pass
    ns = max(1, min(int(n_species), 4))
    c = C()
    c.names = ["Ac", "A", "P", "Bio"][:ns]
    c.inlet = np.array([1.0, 1.0, 0.0, np.nan], np.float32)[:ns]
    c.c_init = np.array([0.0, 0.0, 0.0, 0.1], np.float32)[:ns]
    c.d_rel = np.array([1.0, 1.0, 1.0, 0.0], np.float32)[:ns]
    c.d_biofilm_rel = np.array([1.0, 1.0, 1.0, 0.0], np.float32)[:ns]
    c.immobile = np.array([False, False, False, True])[:ns]
    c.ks_donor, c.ks_acceptor, c.alpha, c.yield_ = 0.0, 0.15, 0.4, 0.04
    c.biomass_coupled = False
    c.abiotic_surface_only = False
    c.biofilm_code = None
    c.seed_in_biofilm = False
    c.abiotic_index = 2
    c.abiotic_product_index = None
    c.biotic_on = True
    c.l_ref_voxels = None
    c.source = "built in"
    c.decay_for = lambda nx: 0.006
    c.truncate = lambda n: default_chemistry(min(n, ns))
    return c


def monod_chemistry(ks=0.5):
    """Single-substrate Monod as the reference's Chemistry(names=["C"],
    inlet=[1], c_init=[0], d_rel=[1], immobile=[False], ks_donor=ks) holds it
    (settings_and_units.py:1834-1929: no decay given, so decay_for is 0), as
    a plain namespace for the oracle."""
    c = default_chemistry(1)
    c.names = ["C"]
    c.ks_donor = float(ks)
    c.source = "monod"
    c.decay_for = lambda nx: 0.0
    c.truncate = lambda n: c
    return c


def solve_adr(mat, vel, pe, da, n_t, n_species=2, steps=None, tol=2e-3, max_steps=100000,
              info=None, ratio=1.12, chem=None, da_abio=0.0, on_progress=None,
              dtype=np.float32, record_means=None):
    """The transport solve in `dtype` (float32 = the reference; float64 its twin).

    Restates solve_adr (prtlb_3d.py:781-1595): pore/biofilm mask, velocity
    normalised by the mean axial pore velocity, D = l_ref/Pe, k = Da/l_ref,
    the one combined explicit time step, face tables in flux form, MUSCL
    advection, harmonic diffusion, C div u, inlet pin, reactions with their
    caps, Euler + clip, the log-spaced snapshot ladder and the geometric-tail
    stop rule.  Optional `record_means` list receives (n, means) per check."""
    T = np.dtype(dtype).type
    mat = np.asarray(mat)
    bf_code = getattr(chem, "biofilm_code", None) if chem is not None else None
    m = mat == PORE
    biofilm = np.zeros(m.shape, bool)
    if bf_code is not None:
        biofilm = mat == bf_code
        m = m | biofilm
    nd = m.ndim
    nx = m.shape[0]
    vel = np.asarray(vel, T)
    sp = np.sqrt((vel[:nd] ** 2).sum(0))
    mean_axial = float(vel[0][m].mean()) if m.any() else 0.0
    mean_speed = float(sp[m].mean()) if m.any() else 0.0
    u_scale = mean_axial if mean_axial > 0.1 * mean_speed else mean_speed
    u = vel[:nd] / max(u_scale, 1e-30)
    u = np.where(m[None], u, 0.0)
    ns = int(n_species)
    ch = default_chemistry(ns) if chem is None else chem.truncate(ns)
    l_ref = float(getattr(ch, "l_ref_voxels", None) or nx)
    D = T(l_ref / max(pe, 1e-6))
    k = T(da / l_ref)
    ka = T(max(da_abio, 0.0) / l_ref)
    j_ab = getattr(ch, "abiotic_index", 2)
    kd = T(ch.decay_for(l_ref))
    immobile = np.asarray(ch.immobile, bool)
    d_rel = np.asarray(ch.d_rel, T).copy()
    d_rel[immobile] = 0.0
    shp = (ns,) + (1,) * nd
    if biofilm.any():
        d_bf = np.asarray(ch.d_biofilm_rel, T).copy()
        d_bf[immobile] = 0.0
        dfield = np.where(biofilm[None], d_bf.reshape(shp), d_rel.reshape(shp)).astype(T) * float(D)
        d_worst = float(max(d_rel.max(), d_bf.max()))
    else:
        dfield = np.ones((ns,) + m.shape, T) * d_rel.reshape(shp) * float(D)
        d_worst = float(d_rel.max())
    dmax = float(D) * float(max(d_worst, 1.0))
    umax = float(sum(np.abs(u[a]).max() for a in range(nd)))
    k_lin = float(k)
    if ch.ks_donor > 0:
        k_lin = max(k_lin, float(k) / float(ch.ks_donor))
    if ns > 1 and ch.ks_acceptor > 0:
        k_lin = max(k_lin, float(k) / float(ch.ks_acceptor))
    sorp = getattr(ch, "sorption", None)
    k_s = T(0.0)
    if sorp is not None:
        k_s = T(max(sorp.da, 0.0) / l_ref)
        k_lin = k_lin + float(k_s) * (1.0 + 1.0 / sorp.kd)
    dt = T(0.4 / (umax + 2.0 * nd * dmax + k_lin + ka + kd + 1e-30))

    surf = np.zeros(m.shape, T)
    if ka > 0 and getattr(ch, "abiotic_surface_only", False):
        nface = np.zeros(m.shape, T)
        for a in range(nd):
            nface += (~_take(m, a, -1)).astype(T)
            nface += (~_take(m, a, 1)).astype(T)
        surf = np.where(m, nface / float(2 * nd), 0.0).astype(T)
    inlet = m[0]
    fed = np.asarray(ch.inlet, T)
    moving = [j for j in range(ns) if not immobile[j]]
    js = list(range(ns)) if len(moving) == ns else moving

    faces = []
    for a in range(nd):
        o_lo = m & _take(m, a, -1)
        o_hi = m & _take(m, a, 1)
        f_lo = o_lo & _take(m, a, -2)
        f_hi = o_hi & _take(m, a, 2)
        u_lo = np.where(o_lo, 0.5 * (u[a] + _take(u[a], a, -1)), 0.0)
        u_hi = np.where(o_hi, 0.5 * (u[a] + _take(u[a], a, 1)), 0.0)
        dl, dh = [], []
        for j in js:
            a1 = dfield[j]
            a2 = _take(a1, a, -1)
            b2 = _take(a1, a, 1)
            with np.errstate(divide="ignore", invalid="ignore"):
                hl = np.where((a1 > 0) & (a2 > 0), 2 * a1 * a2 / (a1 + a2), 0.0)
                hh = np.where((a1 > 0) & (b2 > 0), 2 * a1 * b2 / (a1 + b2), 0.0)
            dl.append(np.where(o_lo, hl, 0.0))
            dh.append(np.where(o_hi, hh, 0.0))
        faces.append((o_lo, o_hi, f_lo, f_hi, u_lo, u_hi,
                      np.stack(dl).astype(T), np.stack(dh).astype(T)))
    divu = np.zeros(m.shape, T)
    for a in range(nd):
        divu += faces[a][5] - faces[a][4]

    def transport(C):
        out = np.zeros_like(C)
        for a in range(nd):
            o_lo, o_hi, f_lo, f_hi, u_lo, u_hi, D_lo, D_hi = faces[a]
            ax = a + 1
            Cm1 = np.where(o_lo, _take(C, ax, -1), C)
            Cp1 = np.where(o_hi, _take(C, ax, 1), C)
            Cm2 = np.where(f_lo, _take(C, ax, -2), Cm1)
            Cp2 = np.where(f_hi, _take(C, ax, 2), Cp1)
            out += D_hi * (Cp1 - C) + D_lo * (Cm1 - C)
            fh = np.where(u_hi >= 0, _muscl(C, Cm1, Cp1), _muscl(Cp1, Cp2, C))
            fl = np.where(u_lo >= 0, _muscl(Cm1, Cm2, C), _muscl(C, Cp1, Cm1))
            out -= u_hi * fh - u_lo * fl
        out += C * divu
        return out

    def reaction(C):
        biotic = getattr(ch, "biotic_on", True)
        if biotic:
            R = k * C[0] / (ch.ks_donor + C[0]) if ch.ks_donor > 0 else k * C[0]
            if ns > 1:
                R = R * (C[1] if ch.ks_acceptor <= 0 else C[1] / (ch.ks_acceptor + C[1]))
            if getattr(ch, "biomass_coupled", False) and ns > 3 and ch.c_init[3] > 0:
                R = R * C[3] / T(ch.c_init[3])
            lim = C[0] / dt
            if ns > 1 and ch.alpha > 0:
                lim = np.minimum(lim, C[1] / (float(ch.alpha) * dt))
            R = np.minimum(R, 0.5 * lim)
        else:
            R = T(0.0)
        Ra = T(0.0)
        if ka > 0 and ns > j_ab:
            Ra = ka * C[j_ab] * surf if ch.abiotic_surface_only else ka * C[j_ab]
            Ra = np.minimum(Ra, 0.5 * C[j_ab] / dt)
        out = np.zeros_like(C)
        out[0] = -R
        if ns > 1:
            out[1] = -ch.alpha * R
        if ns > 2:
            out[2] = (1.0 - (ch.yield_ if ns > 3 else 0.0)) * R
        if ns > 3:
            out[3] = (ch.yield_ * R - kd * C[3]) if biotic else 0.0
        if j_ab < ns:
            out[j_ab] = out[j_ab] - Ra
            j_mk = getattr(ch, "abiotic_product_index", None)
            if j_mk is not None and j_mk < ns and j_mk != j_ab:
                out[j_mk] = out[j_mk] + Ra
        if sorp is not None:
            c, s = C[sorp.dissolved], C[sorp.sorbed]
            r = k_s * (c - s * T(1.0 / sorp.kd))
            r = np.minimum(r, 0.5 * c / dt)
            r = np.maximum(r, -(0.5 * s / dt))
            out[sorp.dissolved] = out[sorp.dissolved] - r
            out[sorp.sorbed] = out[sorp.sorbed] + r
        return out

    def step(C):
        for j in moving:
            if fed[j] == fed[j]:
                C[j, 0][inlet] = fed[j]
        if len(moving) == ns:
            trans = transport(C)
        else:
            trans = np.zeros_like(C)
            trans[moving] = transport(C[moving])
        C = C + dt * (trans + reaction(C))
        return np.where(m, np.maximum(C, 0.0), 0.0)

    C = np.zeros((ns,) + m.shape, T)
    for j in range(ns):
        if not ch.c_init[j]:
            continue
        if (j == ATTACHED and getattr(ch, "seed_in_biofilm", False) and biofilm.any()
                and immobile[j]):
            C[j] = np.where(biofilm, ch.c_init[j], 0.0)
        else:
            C[j] = np.where(m, ch.c_init[j], 0.0)
    keep_steps, keep = [0], [np.where(m, C, 0.0).astype(T)]
    check = max(int(1.0 / float(dt)), 100)
    prev = np.zeros(ns)
    scale = np.full(ns, 1e-6)
    prev_change = np.zeros(ns)
    n = 0
    nxt = 1
    limit = int(steps) if steps is not None else max_steps
    while n < limit:
        n += 1
        C = step(C)
        if n >= nxt:
            keep_steps.append(n)
            keep.append(np.where(m, C, 0.0).astype(T))
            nxt = max(n + 1, int(np.ceil(n * ratio)))
        if n % check == 0:
            cur = np.array([float(C[j][m].mean()) for j in range(ns)])
            if record_means is not None:
                record_means.append((n, cur.copy()))
            scale = np.maximum(scale, np.abs(cur))
            step_ch = np.abs(cur - prev) / scale
            change = float(step_ch.max())
            with np.errstate(divide="ignore", invalid="ignore"):
                r = np.where(prev_change > 0, step_ch / prev_change, 0.0)
            rest = np.where(r < 1.0, step_ch * r / np.maximum(1.0 - r, 1e-12), np.inf)
            rest = float(np.nanmax(np.where(np.isfinite(rest), rest, np.inf)))
            if on_progress is not None:
                on_progress(n, limit, float(cur[0]), rest if np.isfinite(rest) else change)
            if steps is None and n >= 10 * check and rest <= tol:
                break
            prev, prev_change = cur, step_ch
    hit_cap = steps is None and n >= max_steps
    if keep_steps[-1] != n:
        keep_steps.append(n)
        keep.append(np.where(m, C, 0.0).astype(T))
    total = int(max(n, 1))
    ks = np.asarray(keep_steps)
    used, picked = set(), []
    for w in wanted_steps(total, n_t):
        i = int(np.abs(ks - w).argmin())
        if i in used:
            i = nearest_unused(i, used, len(ks))
        used.add(i)
        picked.append(i)
    out = np.zeros((n_t, ns) + m.shape, T)
    for jj, i in enumerate(picked):
        out[jj] = keep[i]
    t_norm = (ks[picked].astype(T) / total).astype(T)
    if info is not None:
        info["converged"] = not (hit_cap or steps is not None)
        info["steps"] = total
        info["dt"] = float(dt)
        info["ladder"] = len(ks)
        info["check"] = check
        info["repeated_snapshots"] = int(max(n_t - len(set(picked)), 0))
        info["keep_steps"] = list(keep_steps)
    return out, t_norm
