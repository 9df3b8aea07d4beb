"""The reference's own known answers, on the GPU path.

Restated from the reference's self-tests (3D/tools/prtlb_3d.py transport
self-test 16a-16j, 3D/tools/test_flow_solvers.py): answers that do not depend
on the implementation, so they check the physics rather than agreement with
one code.  Each case runs through prtlb_gpu; the same functions run on the
oracle (run(..., oracle=True)) to confirm the thresholds hold for the
reference's algorithm itself.
"""

import contextlib
import io

import numpy as np
import pytest

PORE, SOLID = 2, 0


def _adr(oracle):
    if oracle:
        from oracle import prtlb_oracle as O
        return O.solve_adr
    from prtlb_gpu import solve_adr
    return solve_adr


def _chem(**kw):
    from prtlb_gpu.chemistry import Chemistry
    return Chemistry(**kw)


def _tracer():
    return _chem(names=["Ac"], inlet=[1.0], c_init=[0.0], d_rel=[1.0], immobile=[False],
                 biotic_on=False)


def _channel(nx, ny):
    g = np.full((nx, ny), PORE, np.uint8)
    v = np.zeros((3, nx, ny), np.float32)
    v[0] = 1.0
    return g, v


def front_widths(oracle=False):
    """16a (prtlb_3d.py:2270-2296): a step fed into an empty channel spreads
    as erfc; its 90 %-10 % width against 2 erfcinv(0.2) sqrt(4 D t)."""
    from scipy.special import erfcinv
    solve_adr = _adr(oracle)
    out = []
    for pe, tol in ((20.0, 0.10), (50.0, 0.08), (100.0, 0.08)):
        g, v = _channel(64, 8)
        info = {}
        with contextlib.redirect_stdout(io.StringIO()):
            solve_adr(g, v, pe=pe, da=0.0, n_t=2, n_species=1, steps=1, chem=_tracer(), info=info)
            n = int(round(32 / info["dt"]))
            o, _ = solve_adr(g, v, pe=pe, da=0.0, n_t=2, n_species=1, steps=n, chem=_tracer())
        prof = o[-1, 0].mean(1).astype(float)
        xs = np.arange(64) + 0.5
        x90, x10 = np.interp([0.9, 0.1], prof[::-1], xs[::-1])
        exact = 2 * erfcinv(0.2) * np.sqrt(4 * (64 / pe) * n * info["dt"])
        out.append((abs(abs(x10 - x90) - exact) / exact, tol))
    return out


def monotone_rise(oracle=False):
    """16b (:2298-2318): a fed front never grows a bump along x."""
    g, v = _channel(80, 8)
    with contextlib.redirect_stdout(io.StringIO()):
        o, _ = _adr(oracle)(g, v, pe=150.0, da=0.0, n_t=6, n_species=1, steps=400,
                            chem=_tracer())
    return max(float(np.diff(o[i, 0].mean(1)).max()) for i in range(o.shape[0]))


def mass_at_high_da(oracle=False):
    """16d (:2335-2355): with no yield and a non-limiting acceptor, donor plus
    product never exceeds the feed, even nearly zero order at Da 400."""
    worst = []
    for da in (20.0, 100.0, 400.0):
        ch = _chem(names=["Ac", "A", "P"], inlet=[1.0, 1.0, 0.0], c_init=[0.0, 1.0, 0.0],
                   d_rel=[1.0, 1.0, 1.0], immobile=[False, False, False], ks_donor=1e-3,
                   alpha=0.0)
        g, v = _channel(40, 8)
        with contextlib.redirect_stdout(io.StringIO()):
            o, _ = _adr(oracle)(g, v, pe=30.0, da=da, n_t=3, n_species=3, chem=ch)
        worst.append(float((o[-1, 0] + o[-1, 2]).max()))
    return worst


def zero_ks_is_finite(oracle=False):
    """16e (:2357-2366): a zero acceptor half-saturation is first order, not 0/0."""
    from prtlb_gpu.chemistry import default_chemistry
    ch = default_chemistry(4)
    ch.ks_acceptor = 0.0
    g = np.full((30, 8), PORE, np.uint8)
    v = np.stack([np.ones((30, 8), np.float32)] * 3)
    with contextlib.redirect_stdout(io.StringIO()):
        o, _ = _adr(oracle)(g, v, pe=30.0, da=2.0, n_t=3, n_species=4, chem=ch)
    return bool(np.isfinite(o).all())


def divergent_field_peak(oracle=False, steps=40000):
    """16i (:2436-2454): a 10 % compressible field makes no solute from nothing."""
    g = np.full((24, 16), PORE, np.uint8)
    g[:, 0] = g[:, -1] = SOLID
    xs = np.arange(24)[:, None] * np.ones((1, 16))
    v = np.zeros((3, 24, 16), np.float32)
    v[0] = 1.0 + 0.10 * np.sin(2 * np.pi * xs / 24.0)
    ch = _chem(names=["Ac", "A"], inlet=[1.0, 1.0], c_init=[0.0, 1.0], d_rel=[1.0, 1.0],
               immobile=[False, False], biotic_on=False)
    with contextlib.redirect_stdout(io.StringIO()):
        o, _ = _adr(oracle)(g, v, pe=2.0, da=0.0, n_t=3, n_species=2, steps=steps, chem=ch)
    p = g == PORE
    return max(float(o[:, 0][:, p].max()), float(o[:, 1][:, p].max()))


def abiotic_conversion(oracle=False):
    """16j (:2495-2516): abiotic only, the donor becomes the product; more of
    it at higher Da_abio, and the two sum to the feed."""
    g = np.full((60, 16), PORE, np.uint8)
    g[:, 0] = g[:, -1] = SOLID
    v = np.zeros((3, 60, 16), np.float32)
    v[0] = 1.0
    m = g == PORE
    res = []
    for da_a in (0.5, 5.0):
        ch = _chem(names=["Ac", "A", "P"], inlet=[1.0, 1.0, 0.0], c_init=[0.0, 0.0, 0.0],
                   d_rel=[1.0, 1.0, 1.0], immobile=[False, False, False], biotic_on=False,
                   abiotic_index=0, abiotic_product_index=2)
        with contextlib.redirect_stdout(io.StringIO()):
            o, _ = _adr(oracle)(g, v, pe=10.0, da=0.0, n_t=3, n_species=3, chem=ch,
                                da_abio=da_a)
        res.append((float(o[-1, 0][m].mean()), float(o[-1, 2][m].mean()), o, ch, da_a))
    return g, res


def _sound_run(oracle=False):
    """The four-chemical run of 16f (prtlb_3d.py:2368-2373): a walled channel,
    the default chemistry, Pe 30, Da 1, to the stop rule."""
    from prtlb_gpu.chemistry import default_chemistry
    g = np.full((40, 8), PORE, np.uint8)
    g[:, 0] = g[:, -1] = SOLID
    v = np.zeros((3, 40, 8), np.float32)
    v[0] = 1.0
    ch = default_chemistry(4)
    info = {}
    with contextlib.redirect_stdout(io.StringIO()):
        o, _ = _adr(oracle)(g, v, pe=30.0, da=1.0, n_t=4, n_species=4, chem=ch, info=info)
    return g, v, ch, o, info


def planted_complaints(on_gpu=False, oracle=False):
    """16f (:2368-2397): check_physics is quiet on a sound run and names each
    planted fault: product above its bound, a negative chemical, a vanished
    one, runaway biomass, a checkerboard along the flow (but not across it)."""
    from prtlb_gpu.physics import check_physics
    g, _, ch, o, _ = _sound_run(oracle)
    cp = lambda x: check_physics(x, g, chem=ch, on_gpu=on_gpu)  # noqa: E731
    got = {"sound": cp(o)}
    b = o.copy(); b[:, 2] = 5.0
    got["product"] = cp(b)
    b = o.copy(); b[:, 1] = -0.5 * (g == PORE)
    got["negative"] = cp(b)
    b = o.copy(); b[:, 0] = 0.0
    got["zero"] = cp(b)
    b = o.copy(); b[:, 3] = 500.0
    got["runaway"] = cp(b)
    xs = np.arange(40)[:, None] * np.ones((1, 8))
    b = o.copy(); b[-1, 0] = np.where(g == PORE, 0.5 + 0.4 * ((-1.0) ** xs), 0.0)
    got["along"] = cp(b)
    zs = np.arange(8)[None, :] * np.ones((40, 1))
    b = o.copy(); b[-1, 0] = np.where(g == PORE, 0.5 + 0.4 * ((-1.0) ** zs), 0.0)
    got["across"] = cp(b)
    return got


def _check_planted(got):
    assert got["sound"] == []
    assert any("P reaches" in c for c in got["product"])
    assert any("negative" in c for c in got["negative"])
    assert any("exactly zero" in c for c in got["zero"])
    assert any("runaway" in c for c in got["runaway"])
    assert any("checkerboard" in c for c in got["along"])
    assert not any("checkerboard" in c for c in got["across"])


def stop_point_gap(oracle=False):
    """16g (:2399-2421): when the stop rule fires, the slowest chemicals
    (product, biomass) are within 1 % of a run 16 times longer."""
    g, v, ch, stopped, info = _sound_run(oracle)
    with contextlib.redirect_stdout(io.StringIO()):
        long_run, _ = _adr(oracle)(g, v, pe=30.0, da=1.0, n_t=4, n_species=4, chem=ch,
                                   steps=info["steps"] * 16)
    p = g == PORE
    return [abs(float(stopped[-1, j][p].mean()) - float(long_run[-1, j][p].mean())) /
            max(abs(float(long_run[-1, j][p].mean())), 1e-9) for j in (2, 3)]


def axial_peclet_fronts(oracle=False):
    """16h (:2423-2434): the Peclet number is taken against the axial
    velocity, so a transverse component does not move the front."""
    g = np.full((40, 16), PORE, np.uint8)
    v_ax = np.zeros((3, 40, 16), np.float32)
    v_ax[0] = 1.0
    v_tt = v_ax.copy()
    v_tt[1] = 0.6
    fronts = []
    for v in (v_ax, v_tt):
        with contextlib.redirect_stdout(io.StringIO()):
            o, _ = _adr(oracle)(g, v, pe=30.0, da=0.0, n_t=2, n_species=1, steps=200,
                                chem=_tracer())
        fronts.append(float(np.argmax(o[-1, 0].mean(1) < 0.5)))
    return fronts


def grid_peclet_warnings():
    from prtlb_gpu import solve_adr
    g, v = _channel(80, 8)
    said = []
    for pe in (5000.0, 50.0):
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            solve_adr(g, v, pe=pe, da=0.0, n_t=2, n_species=1, steps=5, chem=_tracer())
        said.append("grid Peclet" in buf.getvalue())
    return said


# --------------------------------------------------------------------- tests
gpu = pytest.mark.gpu


@gpu
def test_front_width_matches_erfc():
    for err, tol in front_widths():
        assert err < tol, (err, tol)


@gpu
def test_monotone_front_stays_monotone():
    assert monotone_rise() < 1e-6


@gpu
def test_grid_peclet_is_warned_about_only_when_unresolved():
    assert grid_peclet_warnings() == [True, False]


@gpu
def test_donor_plus_product_never_exceeds_the_feed():
    assert max(mass_at_high_da()) <= 1.02


@gpu
def test_zero_acceptor_half_saturation_is_first_order():
    assert zero_ks_is_finite()


@gpu
def test_divergent_field_makes_no_solute():
    assert divergent_field_peak() <= 1.0005


@gpu
def test_abiotic_donor_becomes_product():
    from prtlb_gpu.physics import check_physics
    g, res = abiotic_conversion()
    prev = -1.0
    for ac, p, o, ch, da_a in res:
        assert p > prev and p > 0.05, (ac, p)
        assert abs(ac + p - 1.0) < 0.01, (ac, p)
        assert not check_physics(o, g, chem=ch, da_abio=da_a)
        prev = p


@gpu
@pytest.mark.parametrize("on_gpu", [False, True])
def test_check_physics_names_each_planted_fault(on_gpu):
    _check_planted(planted_complaints(on_gpu=on_gpu))


@gpu
def test_stop_point_is_within_one_percent_of_settled():
    assert max(stop_point_gap()) < 0.01


@gpu
def test_peclet_is_taken_against_the_axial_velocity():
    a, b = axial_peclet_fronts()
    assert abs(a - b) <= 1


def _poiseuille_peak(nd, H):
    from prtlb_gpu import stokes_d2q9, stokes_d3q19
    with contextlib.redirect_stdout(io.StringIO()):
        if nd == 2:
            g = np.full((12, H + 2), PORE, np.uint8)
            g[:, 0] = g[:, -1] = SOLID
            return float(stokes_d2q9(g, nit=20000, force=2e-6, precision="fp64")[0].max())
        g = np.full((8, H + 2, 8), PORE, np.uint8)
        g[:, 0, :] = g[:, -1, :] = SOLID
        return float(stokes_d3q19(g, nit=20000, force=2e-6, precision="fp64")[0].max())


@gpu
def test_d2q9_and_d3q19_agree_on_the_same_channel():
    """test_flow_solvers.py:326-340: a 2D and a 3D slit of the same aperture."""
    for H in (4, 8):
        u2, u3 = _poiseuille_peak(2, H), _poiseuille_peak(3, H)
        assert abs(u2 - u3) / u2 < 1e-3, (H, u2, u3)


@gpu
def test_flux_is_the_same_through_every_plane():
    """test_flow_solvers.py:342-350: a duct walled in y and z, open along x."""
    from prtlb_gpu import stokes_d3q19
    g = np.full((16, 16, 16), PORE, np.uint8)
    g[:, 0, :] = g[:, -1, :] = SOLID
    g[:, :, 0] = g[:, :, -1] = SOLID
    with contextlib.redirect_stdout(io.StringIO()):
        v = stokes_d3q19(g, nit=400, force=2e-6)
    p = g == PORE
    flux = [float(v[0, i][p[i]].sum()) for i in range(2, g.shape[0] - 2)]
    assert (max(flux) - min(flux)) / abs(np.mean(flux)) < 0.01
