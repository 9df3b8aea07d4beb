"""Parity at the benchmark configurations' sizes, against golden runs of the
reference itself (tests/golden/make_golden_configs.py).

  plain 2D   128 x 128 disks (porosity 0.6), D2Q9 to tol 1e-7, then one
             first-order solute at Pe 10, Da 1 for 4000 steps, 5 snapshots
  plain 3D   the 64^3 sphere pack of the bench: 300 D3Q19 iterations, then
             200 Monod steps (Ks 0.5) and 200 four-chemical dual-Monod steps
  128^3      a 128^3 sphere pack: 100 D3Q19 iterations, 50 four-chemical
             steps on a velocity field made of integer arithmetic

Bars: the float64 flow within 1e-6 (relative to the largest speed) of the
reference's field with the same iteration count; float32 storage ("fp32",
float64 momentum) and the all-float32 collision ("fp32f") within 1e-5
relative L2 of the reference's float64 field; the transport bit-identical
(snapshots, t_norm, progress records, step count), and within 1e-5 relative
L2 of the reference's float64 twin.  At 128^3 the stored flow field is a
subsample of 8000 pore voxels plus whole-field float64 statistics; 3D
transport results are kept as a sha256 and a subsample.  The measured
errors are printed (pytest -s).
"""

import contextlib
import io
import sys

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

sys.path.insert(0, GOLDEN)
from fields import digest, field_stats, integer_velocity  # noqa: E402

pytestmark = pytest.mark.gpu

FLOW_BAR_FP64 = 1e-6   # max |v - v_ref| / max |v_ref|
FLOW_BAR_FP32 = 1e-5   # relative L2 against the reference's float64 field
ADR_BAR_TWIN = 1e-5    # float32 transport against the float64 twin, relative L2


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rel_max(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def report(config, what, **vals):
    print("CONFIG %-9s %-34s %s" % (config, what,
                                    " ".join("%s=%.3g" % kv for kv in vals.items())))


def flow(g, nit, force, tau, tol, precision, info):
    from prtlb_gpu import stokes_d2q9, stokes_d3q19
    fn = stokes_d3q19 if g.ndim == 3 else stokes_d2q9
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(g, nit=nit, force=force, tau_lb=tau, tol=tol, info=info, precision=precision)


def transport(g, v, z, prefix, chem):
    from prtlb_gpu import solve_adr
    kw = dict(pe=float(z[prefix + "pe"]), da=float(z[prefix + "da"]),
              n_t=int(z[prefix + "n_t"]), n_species=int(z[prefix + "n_species"]),
              steps=int(z[prefix + "steps"]))
    info, prog = {}, []
    with contextlib.redirect_stdout(io.StringIO()):
        out, tn = solve_adr(g, v, info=info, chem=chem, on_progress=lambda *a: prog.append(a),
                            **kw)
    return out, tn, info, np.asarray(prog, np.float64).reshape(-1, 4)


def monod():
    from prtlb_gpu.chemistry import monod_chemistry
    return monod_chemistry(0.5)


def dual_monod():
    from prtlb_gpu.chemistry import default_chemistry
    c = default_chemistry(4)
    c.ks_donor = 0.5
    return c


def flow_case(z):
    return dict(nit=int(z["nit"]), force=float(z["force"]), tau=float(z["tau"]),
                tol=float(z["tol"]))


def check_summary(out, z, prefix):
    """A transport result against a fixture kept as sha256, shape and a
    subsample (the subsample first, so a failure shows the size of the
    difference)."""
    assert tuple(out.shape) == tuple(z[prefix + "shape"])
    flat = out.reshape(out.shape[0], out.shape[1], -1)
    sub = flat[:, :, z[prefix + "sub_index"]]
    ref = z[prefix + "sub"]
    assert np.array_equal(sub, ref), float(np.abs(sub - ref).max())
    assert digest(out) == str(z[prefix + "sha256"])


# ---------------------------------------------------------------------------
# plain 2D: the whole configuration
# ---------------------------------------------------------------------------
def test_plain2d_flow_fp64_matches_reference():
    z = load_golden("cfg_plain2d")
    info = {}
    v = flow(z["g"], precision="fp64", info=info, **flow_case(z))
    assert info["flow_iters"] == int(z["info_flow_iters"])
    assert info["flow_converged"] == bool(z["info_flow_converged"])
    err = rel_max(v, z["v"])
    report("plain-2d", "flow fp64 vs reference", rel_max=err, l2=rel_l2(v, z["v"]),
           k=info["permeability"], iters=info["flow_iters"])
    assert err < FLOW_BAR_FP64, err
    assert info["permeability"] > 0 and np.isfinite(info["permeability"])


@pytest.mark.parametrize("precision", ["fp32", "fp32f"])
def test_plain2d_flow_fp32_within_1e5(precision):
    z = load_golden("cfg_plain2d")
    info, info64 = {}, {}
    v = flow(z["g"], precision=precision, info=info, **flow_case(z))
    flow(z["g"], precision="fp64", info=info64, **flow_case(z))
    l2 = rel_l2(v, z["v"])
    dk = abs(info["permeability"] / info64["permeability"] - 1)
    report("plain-2d", "flow %s vs reference fp64" % precision, rel_l2=l2,
           rel_max=rel_max(v, z["v"]), k_rel_err=dk, iters=info["flow_iters"])
    assert l2 <= FLOW_BAR_FP32, l2
    assert dk <= FLOW_BAR_FP32, dk


def test_plain2d_transport_bit_identical():
    from prtlb_gpu.chemistry import default_chemistry
    z = load_golden("cfg_plain2d")
    out, tn, info, prog = transport(z["g"], z["v"], z, "arg_", default_chemistry(1))
    assert info["steps"] == int(z["ainfo_steps"])
    assert info["dt"] == float(z["ainfo_dt"])
    assert np.array_equal(tn, z["t_norm"])
    assert np.array_equal(prog, z["progress"])
    assert np.array_equal(out, z["out"]), float(np.abs(out - z["out"]).max())
    report("plain-2d", "transport (first order, 4000 steps)", max_abs_diff=0.0,
           steps=info["steps"])


# ---------------------------------------------------------------------------
# plain 3D: the bench's 64^3 pack at fixed counts
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32f"])
def test_plain3d64_flow(precision):
    z = load_golden("cfg_plain3d64")
    info = {}
    v = flow(z["g"], precision=precision, info=info, **flow_case(z))
    assert info["flow_iters"] == int(z["info_flow_iters"])
    l2, mx = rel_l2(v, z["v"]), rel_max(v, z["v"])
    report("plain-3d", "flow %s vs reference fp64 (300 its)" % precision, rel_l2=l2,
           rel_max=mx, k=info["permeability"])
    if precision == "fp64":
        assert mx < FLOW_BAR_FP64, mx
    else:
        assert l2 <= FLOW_BAR_FP32, l2


def test_plain3d64_monod_bit_identical_and_near_float64_twin():
    z = load_golden("cfg_plain3d64")
    out, tn, info, prog = transport(z["g"], z["v"], z, "arg_", monod())
    assert info["steps"] == int(z["ainfo_steps"])
    assert np.array_equal(tn, z["t_norm"])
    assert np.array_equal(prog, z["progress"])
    check_summary(out, z, "out_")
    # bit-identical to the reference's float32 run, so its distance from the
    # reference's float64 twin is the one the generator measured
    assert np.array_equal(tn, z["t_norm64"].astype(np.float32))
    l2, mx = (float(x) for x in z["twin_rel_l2_max"])
    report("plain-3d", "Monod transport vs float64 twin", rel_l2=l2, rel_max=mx)
    assert l2 <= ADR_BAR_TWIN, l2


def test_plain3d64_dual_monod_bit_identical():
    z = load_golden("cfg_plain3d64")
    out, tn, info, prog = transport(z["g"], z["v"], z, "arg4_", dual_monod())
    assert info["steps"] == int(z["ainfo4_steps"])
    assert np.array_equal(tn, z["t_norm4"])
    assert np.array_equal(prog, z["progress4"])
    check_summary(out, z, "out4_")


# ---------------------------------------------------------------------------
# 128^3
# ---------------------------------------------------------------------------
def pack128(z):
    from prtlb_gpu.geometry import sphere_pack_3d
    g = sphere_pack_3d(128, 0.45, 0)
    assert digest(g) == str(z["g_sha256"]), "the seeded 128^3 pack differs from the fixture's"
    return g


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32f"])
def test_sphere128_flow(precision):
    z = load_golden("cfg_sphere128")
    g = pack128(z)
    info = {}
    v = flow(g, precision=precision, info=info, **flow_case(z))
    assert info["flow_iters"] == int(z["info_flow_iters"])
    sub = v.reshape(3, -1)[:, z["v_sub_index"]]
    ref = z["v_sub"]
    stats = field_stats(v, g == 2)
    ref_stats = z["v_stats"]
    l2, mx = rel_l2(sub, ref), rel_max(sub, ref)
    # whole-field sums and norms of each component against the reference's
    sums = float(np.abs(stats[:, 0] - ref_stats[:, 0]).max() / np.abs(ref_stats[:, 0]).max())
    norm = float(np.abs(np.sqrt(stats[:, 1]) - np.sqrt(ref_stats[:, 1])).max()
                 / np.sqrt(ref_stats[:, 1]).max())
    report("128^3", "flow %s vs reference fp64 (100 its)" % precision, sub_rel_l2=l2,
           sub_rel_max=mx, sums=sums, norms=norm)
    bar = FLOW_BAR_FP64 if precision == "fp64" else FLOW_BAR_FP32
    assert (mx if precision == "fp64" else l2) < bar
    assert sums < bar and norm < bar


def test_sphere128_transport_bit_identical():
    z = load_golden("cfg_sphere128")
    g = pack128(z)
    vel = integer_velocity(g)
    assert digest(vel) == str(z["vel_sha256"])
    out, tn, info, prog = transport(g, vel, z, "arg_", dual_monod())
    assert info["steps"] == int(z["ainfo_steps"])
    assert np.array_equal(tn, z["t_norm"])
    assert np.array_equal(prog, z["progress"])
    check_summary(out, z, "out_")
    report("128^3", "four-chemical transport (50 steps)", max_abs_diff=0.0)


def test_sphere128_fp32_to_convergence_within_1e5_of_fp64():
    """The precision-sweep bar on the GPU alone: both runs to tol 1e-6 (cap
    30 000), float32 storage against float64 storage."""
    z = load_golden("cfg_sphere128")
    g = pack128(z)
    m = g == 2
    i64 = {}
    v64 = flow(g, nit=30000, force=2e-6, tau=0.8, tol=1e-6, precision="fp64", info=i64)
    for precision in ("fp32", "fp32f"):
        info = {}
        v = flow(g, nit=30000, force=2e-6, tau=0.8, tol=1e-6, precision=precision, info=info)
        l2 = rel_l2(v[:, m], v64[:, m])
        dk = abs(info["permeability"] / i64["permeability"] - 1)
        report("128^3", "flow %s vs fp64, converged" % precision, rel_l2=l2,
               rel_max=rel_max(v[:, m], v64[:, m]), k_rel_err=dk, iters=info["flow_iters"],
               iters64=i64["flow_iters"])
        assert l2 <= FLOW_BAR_FP32, (precision, l2)
        assert dk <= FLOW_BAR_FP32, (precision, dk)
