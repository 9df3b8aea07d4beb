"""prt_flow_noalloc: the flow solve for callers that cannot allocate.

Some hosts own the whole device memory pool (a framework that forbids
foreign cudaMalloc calls, a real-time loop that must never wait on the
allocator, a plug-in host that hands out buffers but no allocator).  For
them the library has one entry point that allocates nothing: the caller
passes device buffers for the material grid and the velocity, and all other
scratch lives in a fixed 48 MiB array compiled into the library.

These tests call it through the C ABI and compare each result with the
ordinary entry point (prt_flow) on the same inputs.  Both run the same step
kernels on the same pore-only layout, so the fields, iteration counts and
permeabilities must be equal bit for bit.  One test calls it twice in a row
on each case; another walks from a large grid to smaller ones of another
dimension and precision, so stale scratch left by a bigger call would show.
They also check that a grid too large for the array is refused with a clear
message and that a later success clears that message.  The file is named to
be collected last, so a run that stops at the first failure has run
everything else first.
"""

import ctypes

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def params(g, precision, nit, tol, force=2e-6, tau=0.8):
    from prtlb_gpu import _lib
    p = _lib.FlowParams()
    p.nd = g.ndim
    for i, n in enumerate(g.shape):
        p.dims[i] = int(n)
    p.nit = nit
    p.force = force
    p.tau = tau
    p.magic = 3.0 / 16.0
    p.tol = tol
    p.every = 50
    p.precision = _lib.PRECISIONS[precision]
    return p


def via_prt_flow(g, p):
    from prtlb_gpu import _lib
    ctx = _lib.default_context(0)
    vel = np.empty((3,) + g.shape, np.float32)
    info = _lib.FlowInfo()
    g8 = np.ascontiguousarray(g.astype(np.uint8))
    with ctx.lock:
        ctx.check(_lib.lib().prt_flow(ctx.handle, g8.ctypes.data_as(ctypes.c_void_p),
                                      ctypes.byref(p), vel.ctypes.data_as(ctypes.c_void_p),
                                      ctypes.byref(info)))
    return vel, info


def via_noalloc(g, p, torch, stream):
    from prtlb_gpu import _lib
    L = _lib.lib()
    d_mat = torch.from_numpy(np.ascontiguousarray(g.astype(np.uint8))).cuda()
    d_vel = torch.full((3,) + g.shape, float("nan"), dtype=torch.float32, device="cuda")
    info = _lib.FlowInfo()
    torch.cuda.synchronize()
    rc = L.prt_flow_noalloc(ctypes.c_void_p(d_mat.data_ptr()), ctypes.byref(p),
                            ctypes.c_void_p(d_vel.data_ptr()), ctypes.byref(info),
                            ctypes.c_void_p(stream.cuda_stream))
    msg = L.prt_last_error(None)
    assert rc == 0, msg.decode() if msg else rc
    torch.cuda.synchronize()
    return d_vel.cpu().numpy(), info


def assert_same(v, info, ref, rinfo):
    assert np.isfinite(v).all()
    assert info.iters == rinfo.iters and info.converged == rinfo.converged
    assert info.fluid_cells == rinfo.fluid_cells
    assert np.array_equal(v, ref), float(np.abs(v - ref).max())
    assert info.permeability == rinfo.permeability


def case(name, precision):
    z = load_golden(name)
    g = z["g"]
    p = params(g, precision, int(z["nit"]), float(z["tol"]), force=float(z["force"]),
               tau=float(z["tau"]))
    return g, p


@pytest.mark.parametrize("name,precision", [("flow_spheres3d", "fp64"),
                                            ("flow_spheres3d", "fp32"),
                                            ("flow_disks2d", "fp32"),
                                            ("flow_slit3d_fixed601", "fp64")])
def test_noalloc_matches_prt_flow_twice(name, precision):
    torch = pytest.importorskip("torch")
    g, p = case(name, precision)
    ref, rinfo = via_prt_flow(g, p)
    stream = torch.cuda.Stream()
    for _ in range(2):  # the shared array keeps the previous call's contents
        v, info = via_noalloc(g, p, torch, stream)
        assert_same(v, info, ref, rinfo)


def test_noalloc_large_then_smaller_grids():
    """A big 3D float32 solve leaves its lattices in the array; smaller
    solves of another dimension and precision that follow must not see them."""
    from prtlb_gpu.geometry import random_pack
    torch = pytest.importorskip("torch")
    big = random_pack((40, 36, 32), 0.45, 3.0, 5.0, seed=11)
    seq = [(big, params(big, "fp32", 400, 0.0))]
    for name, precision in (("flow_disks2d", "fp32"), ("flow_slit3d_fixed601", "fp64"),
                            ("flow_spheres3d", "fp32f")):
        seq.append(case(name, precision))
    stream = torch.cuda.Stream()
    for g, p in seq:
        ref, rinfo = via_prt_flow(g, p)
        v, info = via_noalloc(g, p, torch, stream)
        assert_same(v, info, ref, rinfo)


def test_noalloc_refuses_grids_larger_than_its_scratch():
    from prtlb_gpu import _lib
    torch = pytest.importorskip("torch")
    g = np.full((96, 96, 96), 2, np.uint8)  # 96^3 D3Q19 float32 needs ~137 MB
    p = params(g, "fp32", 100, 1e-6)
    d_mat = torch.zeros(16, dtype=torch.uint8, device="cuda")   # never read: refused first
    d_vel = torch.zeros(16, dtype=torch.float32, device="cuda")
    L = _lib.lib()
    rc = L.prt_flow_noalloc(ctypes.c_void_p(d_mat.data_ptr()), ctypes.byref(p),
                            ctypes.c_void_p(d_vel.data_ptr()), None, None)
    assert rc == _lib.PRT_E_INVALID
    msg = L.prt_last_error(None).decode()
    assert "bytes of scratch" in msg and str(48 << 20) in msg
    # a successful call afterwards leaves no message behind
    g, p = case("flow_slit3d_fixed601", "fp64")
    via_noalloc(g, p, torch, torch.cuda.Stream())
    assert L.prt_last_error(None).decode() == ""
