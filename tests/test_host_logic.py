"""Host-side logic that needs no GPU: solve_adr's set-up (time step, check
interval, coefficients) from host statistics against the reference's golden
runs, the snapshot ladder and picking, chemistry, geometry helpers,
check_physics, and the flow wrapper's refusals."""

import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from test_oracle_golden import adr_kwargs

from prtlb_gpu import adr as A
from prtlb_gpu import chemistry as C
from prtlb_gpu import geometry as G
from prtlb_gpu.physics import check_physics

ADR32 = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "adr_*.npz")))


@pytest.mark.parametrize("name", ADR32)
def test_prepare_reproduces_reference_time_step(name):
    z = load_golden(name)
    kw = adr_kwargs(z, name)
    st = A.velocity_stats_host(z["mat"], z["vel"], kw["chem"])
    S = A.prepare(z["mat"].shape, st, kw["pe"], kw["da"], n_species=kw["n_species"],
                  chem=kw["chem"], da_abio=kw.get("da_abio", 0.0), mat=z["mat"])
    assert float(S.dt) == float(z["info_dt"])
    assert S.l_ref == float(z["info_l_ref_voxels"])
    assert S.pe_grid == float(z["info_grid_peclet"])
    assert S.nbiofilm == int(z["info_biofilm_voxels"])
    assert S.surf_sum == float(z["info_surface_voxels"])
    lim = "advection" if S.umax > 2.0 * S.nd * S.dmax else "diffusion"
    assert lim == str(z["info_dt_limited_by"])


def test_wanted_steps_and_nearest_unused():
    assert list(A._wanted_steps(200, 1)) == [200]
    assert list(A._wanted_steps(200, 2)) == [0, 200]
    w = A._wanted_steps(10000, 5)
    assert w[0] == 0 and w[-1] == 10000 and list(w) == sorted(w)
    assert A._nearest_unused(3, {3, 2}, 6) == 4
    assert A._nearest_unused(0, {0}, 1) == 0


def test_chemistry_truncate_and_default():
    d = C.default_chemistry(4)
    assert d.names == ["Ac", "A", "P", "Bio"]
    assert d.inlet[3] != d.inlet[3] and list(d.d_rel[:3]) == [1.0, 1.0, 1.0]
    assert list(np.where(d.immobile)[0]) == [3]
    t = d.truncate(2)
    assert t.names == ["Ac", "A"] and t.inlet.shape == (2,)
    assert abs(d.decay_for(40) - 0.006) < 1e-12
    with pytest.raises(ValueError):
        C.Chemistry(names=["a", "b"], inlet=[1.0], c_init=[0, 0], d_rel=[1, 1],
                    immobile=[False, False])


def test_abiotic_without_reactant_is_refused():
    g = np.full((20, 6), 2, np.uint8)
    v = np.zeros((3, 20, 6), np.float32)
    v[0] = 1.0
    st = A.velocity_stats_host(g, v)
    with pytest.raises(ValueError):
        A.prepare(g.shape, st, 10.0, 1.0, n_species=2, da_abio=1.0)


def test_geometry_helpers():
    g = np.full((10, 6, 6), 2, np.uint8)
    g[4] = 0
    g2, n = G.keep_inlet_connected_host(g)
    assert n == 5 * 36 and (g2[5:] == 0).all()
    gb, nb = G.coat_with_biofilm(np.pad(np.full((6, 6), 2, np.uint8), 1), 3, 1)
    assert nb > 0 and (gb == 3).sum() == nb
    d = np.zeros((4, 4))
    d[0, 0] = np.inf
    assert G.assert_finite_distance(d, np.full((4, 4), 2)) is not None
    assert G.assert_finite_distance(np.zeros((4, 4)), np.full((4, 4), 2)) is None
    pack = G.sphere_pack_3d(24, 0.45, seed=3)
    assert abs((pack == 2).mean() - 0.45) < 0.05


def test_check_physics_rules():
    g = np.full((20, 8), 2, np.uint8)
    nan_field = np.full((3, 1, 20, 8), np.nan, np.float32)
    assert any("not finite" in s for s in check_physics(nan_field, g))
    good = np.linspace(1, 0, 20, dtype=np.float32)[None, None, :, None].repeat(8, 3)
    good = np.concatenate([good * 0.5, good], 0)
    assert check_physics(good, g) == []
    neg = good.copy()
    neg[-1, 0, 3, 3] = -0.5
    assert any("negative" in s for s in check_physics(neg, g))


def test_native_pack_loop_matches_numpy_loop():
    """prt_pack_balls places exactly the balls of the NumPy loop (jammed
    packs included, where overlaps are accepted)."""
    import numpy as np
    from prtlb_gpu.geometry import random_pack
    for shp, phi, a, b, sd in (((24, 20, 18), 0.45, 2.0, 4.0, 0), ((40, 40), 0.5, 2.0, 5.0, 3),
                               ((16, 16, 16), 0.3, 1.5, 3.0, 7), ((9, 30), 0.6, 1.0, 5.5, 1)):
        g1 = random_pack(shp, phi, a, b, seed=sd, overlap_after=300)
        g2 = random_pack(shp, phi, a, b, seed=sd, overlap_after=300, native=False)
        assert np.array_equal(g1, g2), shp


def _fastdiv(d):
    """make_fastdiv of csrc/prt_internal.h, restated: s = ceil(log2 d),
    m = floor(2^32 (2^s - d) / d) + 1."""
    s = 0
    while s < 31 and (1 << s) < d:
        s += 1
    m = ((1 << 32) * ((1 << s) - d)) // d + 1
    assert 0 < m < (1 << 32)
    return m, s


def test_multiply_shift_division_is_exact_below_2_pow_31():
    """The transport step finds voxel coordinates with fast_div (high
    multiply, add, shift).  Checked here against integer division for every
    divisor up to 4096 and the powers of two and their neighbours above it,
    on numerators spread over [0, 2^31) with the multiples of d and their
    neighbours, and the ends of the range."""
    rng = np.random.default_rng(0)
    divisors = list(range(1, 4097)) + [x + o for k in range(12, 31)
                                        for x in (1 << k,) for o in (-1, 0, 1)]
    top = (1 << 31) - 1
    for d in divisors:
        m, s = _fastdiv(d)
        ks = np.concatenate([np.arange(0, 4), [top // d - 1, top // d],
                             rng.integers(0, top // d + 1, 200)]).astype(np.int64)
        near = (ks[:, None] * d + np.arange(-1, 2)[None, :]).ravel()
        t = np.concatenate([rng.integers(0, top, 4000, dtype=np.int64), near,
                            np.arange(0, min(3 * d + 3, 20000), dtype=np.int64),
                            np.array([top, top - 1], np.int64)])
        t = t[(t >= 0) & (t <= top)].astype(np.uint64)
        q = (((t * np.uint64(m)) >> np.uint64(32)) + t) >> np.uint64(s)
        assert np.array_equal(q, t // np.uint64(d)), d
