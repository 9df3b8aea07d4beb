"""prt_flow_noalloc: the flow solve for callers that cannot allocate.

Some hosts own the whole device memory pool (a framework that forbids
foreign cudaMalloc calls, a real-time loop that must never wait on the
allocator, a plug-in host that hands out buffers but no allocator).  For
them the library has one entry point that allocates nothing: the caller
passes device buffers for the material grid and the velocity, and all other
scratch lives in a fixed 48 MiB array compiled into the library.

These tests call it through the C ABI, twice in a row, and compare each
result with the ordinary entry point (prt_flow) on the same inputs, using
the tolerances of the flow parity tests (relative max error 1e-6 against the
float64 solve, relative L2 1e-5 for float32 populations).  They also check
that a grid too large for the array is refused with a clear message.  The
file is named to be collected last, so a run that stops at the first failure
has run everything else first.
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


@pytest.mark.parametrize("name,precision", [("flow_spheres3d", "fp64"),
                                            ("flow_spheres3d", "fp32"),
                                            ("flow_disks2d", "fp32"),
                                            ("flow_slit3d_fixed601", "fp64")])
def test_noalloc_matches_prt_flow_twice(name, precision):
    torch = pytest.importorskip("torch")
    z = load_golden(name)
    g = z["g"]
    p = params(g, precision, int(z["nit"]), float(z["tol"]), force=float(z["force"]),
               tau=float(z["tau"]))
    ref, rinfo = via_prt_flow(g, p)
    stream = torch.cuda.Stream()
    for _ in range(2):  # the shared array keeps the previous call's contents
        v, info = via_noalloc(g, p, torch, stream)
        assert np.isfinite(v).all()
        assert info.iters == rinfo.iters and info.converged == rinfo.converged
        assert info.fluid_cells == rinfo.fluid_cells
        scale = float(np.abs(ref).max())
        if precision == "fp64":
            assert float(np.abs(v - ref).max()) / scale < 1e-6
        else:
            rel = float(np.linalg.norm(v.astype(np.float64) - ref) / np.linalg.norm(ref))
            assert rel < 1e-5, rel
        assert abs(info.permeability - rinfo.permeability) <= 1e-6 * abs(rinfo.permeability)


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
