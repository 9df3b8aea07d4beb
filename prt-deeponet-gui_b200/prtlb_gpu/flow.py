"""Stokes flow on the GPU: drop-in ``stokes_d2q9`` / ``stokes_d3q19``.

Signatures, defaults, returned array, ``info`` keys, refusals and warnings
follow the reference (3D/tools/prtlb_2d.py:348-486, prtlb_3d.py:348-456,
FlowConvergence prtlb_3d.py:168-252, _checked_flow prtlb_3d.py:267-316).
The solve itself runs in libprtlb.so: one CUDA graph per solve whose body is
50 fused stream-collide iterations plus the convergence check.

Keyword-only additions: ``precision`` ("fp64" default = the reference's
arithmetic; "fp32" stores f_i - w_i in float32 and forms the momentum and
the antisymmetric non-equilibrium part in float64, the rest in float32;
"fp32f" does all of the collision in float32; "fp16" stores f_i - w_i scaled
by 2^k in float16 and collides in float32), ``device`` (CUDA ordinal) and
``ctx`` (an explicit ``prtlb_gpu.Context``).
"""

import ctypes

import numpy as np

from . import _lib

SOLID, WALL, PORE = 0, 1, 2
CHECK_EVERY = 50


def trt_minus(om_p, magic=3.0 / 16.0):
    """omega- from Lambda = (1/omega+ - 1/2)(1/omega- - 1/2) (prtlb_3d.py:130-139)."""
    lam_p = 1.0 / float(om_p) - 0.5
    if lam_p <= 0:
        raise ValueError("tau must exceed 0.5; the viscosity (tau-1/2)/3 is negative below it "
                         "and the solver cannot run.")
    return 1.0 / (float(magic) / lam_p + 0.5)


def _material_u8(g):
    g = np.asarray(g)
    if g.dtype == np.uint8:
        return np.ascontiguousarray(g)
    # only "is it pore" matters to the flow solve
    return np.where(g == PORE, PORE, SOLID).astype(np.uint8)


def _report(name, every, tol, fi, info):
    """FlowConvergence.report: fill info, warn when the cap was hit."""
    iters = int(fi.iters)
    conv = bool(fi.converged)
    change = float(fi.change)
    if info is not None:
        info["flow_iters"] = iters
        info["flow_converged"] = conv
        info["flow_change"] = change
    if not conv and tol > 0:
        print("     WARNING: the %s solve stopped at its %d iteration cap with the mean\n"
              "              speed still changing by %.3g per %d steps, against a\n"
              "              tolerance of %.3g. The field is not settled and the\n"
              "              permeability read from it will be too low. Raise\n"
              "              ns_max_iT." % (name, iters, change, every, tol), flush=True)


def _checked(name, fi, force, tau_lb):
    """The refusals of _checked_flow, from the device reductions of the
    float32 field: non-finite, no pore space, zero flow; Mach warning."""
    if int(fi.nonfinite) > 0:
        raise SystemExit(
            "the %s solver produced %d non-finite values. The driving force of %g is too "
            "large for tau = %g: lower it, or raise tau. Nothing downstream can use this "
            "field." % (name, int(fi.nonfinite), force, tau_lb))
    if int(fi.fluid_cells) == 0:
        raise SystemExit("the %s solver was given a geometry with no pore space at all." % name)
    if not float(fi.speed_sum) > 0:
        raise SystemExit(
            "the %s solver produced a field that is zero everywhere. Either the driving "
            "force (%g) is too small to survive rounding, or the pore space does not "
            "connect inlet to outlet." % (name, force))
    umax = float(fi.umax)
    ma = umax / np.sqrt(1.0 / 3.0)
    if ma > 0.05:
        print("     WARNING: peak lattice speed %.4g gives a Mach number of %.3f.\n"
              "              Lattice Boltzmann is a low-Mach expansion and is only\n"
              "              reliable below about 0.05. Halve the pressure drop and the\n"
              "              flow halves with it, so nothing is lost but time."
              % (umax, ma), flush=True)


def flow_params(g, nd, name, nit, force, tau_lb, magic, tol, precision):
    """The uint8 grid and the prt_flow_params of one solve, with the
    reference's refusals (tau, grid rank) raised before any work."""
    g = _material_u8(g)
    if g.ndim != nd:
        raise ValueError("%s expects a %dD material grid, got %dD" % (name, nd, g.ndim))
    trt_minus(1.0 / float(tau_lb), magic)  # the reference's tau refusal, before any work
    if precision not in _lib.PRECISIONS:
        raise ValueError("precision must be one of %s" % sorted(_lib.PRECISIONS))
    p = _lib.FlowParams()
    p.nd = nd
    for i, n in enumerate(g.shape):
        p.dims[i] = int(n)
    p.nit = int(nit)
    p.force = float(force)
    p.tau = float(tau_lb)
    p.magic = float(magic)
    p.tol = float(tol)
    p.every = CHECK_EVERY
    p.precision = _lib.PRECISIONS[precision]
    return g, p


def flow_report(name, fi, force, tau_lb, tol, info, precision):
    """What a finished solve reports: FlowConvergence.report, the extra info
    keys, and _checked_flow's refusals and warning."""
    _report(name, CHECK_EVERY, float(tol), fi, info)
    if info is not None:
        info["permeability"] = float(fi.permeability)
        info["flow_mass"] = float(fi.mass)
        info["flow_precision"] = precision
    _checked("flow", fi, force, tau_lb)


def _solve(g, nd, name, nit, force, tau_lb, magic, tol, info, precision, device, ctx):
    g, p = flow_params(g, nd, name, nit, force, tau_lb, magic, tol, precision)
    ctx = ctx or _lib.default_context(device)
    vel = np.empty((3,) + g.shape, np.float32)
    fi = _lib.FlowInfo()
    with ctx.lock:
        ctx.check(_lib.lib().prt_flow(ctx.handle, g.ctypes.data_as(ctypes.c_void_p),
                                      ctypes.byref(p), vel.ctypes.data_as(ctypes.c_void_p),
                                      ctypes.byref(fi)))
    flow_report(name, fi, force, tau_lb, tol, info, precision)
    return vel


def stokes_d3q19(g, nit=30000, force=2e-6, tau_lb=0.8, magic=3.0 / 16.0, tol=1e-6, info=None,
                 *, precision="fp64", device=None, ctx=None):
    """D3Q19 TRT Stokes flow through ``g`` (0 solid, 1 wall, 2 pore).

    Returns float32 (3, nx, ny, nz), zero in the rock.  ``nit`` is a cap; the
    solve stops when mean |u_x| over the pore changes by <= ``tol`` (relative)
    per 50 iterations.  ``info`` gets flow_iters / flow_converged /
    flow_change as in the reference, plus ``permeability`` (nu <u_x>_V / g,
    voxel^2, averaged over all voxels) and ``flow_mass``."""
    return _solve(g, 3, "3D flow", nit, force, tau_lb, magic, tol, info, precision, device, ctx)


def stokes_d2q9(g, nit=30000, force=2e-6, tau_lb=0.8, magic=3.0 / 16.0, tol=1e-6, info=None,
                *, precision="fp64", device=None, ctx=None):
    """D2Q9 TRT Stokes flow through ``g`` (nx, ny).  Returns float32
    (3, nx, ny) with the third component zero; otherwise as stokes_d3q19."""
    return _solve(g, 2, "2D flow", nit, force, tau_lb, magic, tol, info, precision, device, ctx)


def permeability(vel, force, tau_lb=0.8):
    """Darcy permeability nu <u_x>_V / g in voxel^2 from a returned field
    (float64 mean over every voxel; solid voxels hold 0)."""
    nu = (float(tau_lb) - 0.5) / 3.0
    return nu * float(np.asarray(vel)[0].astype(np.float64).mean()) / float(force)
