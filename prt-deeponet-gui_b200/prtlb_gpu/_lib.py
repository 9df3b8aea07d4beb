"""ctypes binding of libprtlb.so (the C ABI declared in include/prtlb.h).

The library is built in-tree (``make -C prt-deeponet-gui_b200/csrc``) and sits
next to this file.  There is no CPU fallback: if the library or a CUDA device
is missing, the first solve raises.
"""

import ctypes
import os
import threading

# concurrent solves (one stream each) need more than the default 8 hardware
# work queues; read when the process creates its CUDA context
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libprtlb.so")

PRT_MAX_SPECIES = 8

PRT_OK = 0
PRT_E_INVALID = -1
PRT_E_CUDA = -2
PRT_E_OOM = -3
PRT_E_STATE = -4
PRT_E_CANCELLED = -5
PRT_E_NODEV = -6

PRT_FP64 = 0
PRT_FP32 = 1
PRT_FP16 = 2
PRT_FP32_F32 = 3

PRECISIONS = {"fp64": PRT_FP64, "fp32": PRT_FP32, "fp16": PRT_FP16, "fp32f": PRT_FP32_F32}

c_i32, c_u32, c_i64, c_f32, c_f64 = (ctypes.c_int32, ctypes.c_uint32, ctypes.c_int64,
                                     ctypes.c_float, ctypes.c_double)


class FlowParams(ctypes.Structure):
    _fields_ = [("nd", c_i32), ("dims", c_i32 * 3), ("nit", c_i64), ("force", c_f64),
                ("tau", c_f64), ("magic", c_f64), ("tol", c_f64), ("every", c_i32),
                ("precision", c_i32)]


class FlowInfo(ctypes.Structure):
    _fields_ = [("iters", c_i64), ("converged", c_i32), ("pad0", c_i32), ("change", c_f64),
                ("fluid_cells", c_i64), ("nonfinite", c_i64), ("umax", c_f64),
                ("speed_sum", c_f64), ("ux_sum", c_f64), ("mass", c_f64),
                ("permeability", c_f64), ("fp16_scale", c_f64)]


class AdrParams(ctypes.Structure):
    _fields_ = [("nd", c_i32), ("dims", c_i32 * 3), ("ns", c_i32), ("moving_mask", c_u32),
                ("pinned_mask", c_u32), ("pore_code", c_i32), ("biofilm_code", c_i32),
                ("u_scale", c_f32), ("dt", c_f32), ("feed", c_f32 * PRT_MAX_SPECIES),
                ("init_mode", c_i32 * PRT_MAX_SPECIES), ("init_value", c_f32 * PRT_MAX_SPECIES),
                ("dface", (c_f32 * 3) * PRT_MAX_SPECIES),
                ("biotic_on", c_i32), ("k", c_f32), ("ks_donor_pos", c_i32), ("ks_donor", c_f32),
                ("ks_acceptor_pos", c_i32), ("ks_acceptor", c_f32), ("coupled", c_i32),
                ("c3_init", c_f32), ("neg_alpha", c_f32), ("alpha_cap", c_i32),
                ("alpha_dt", c_f32), ("prod_coef", c_f32), ("yield_", c_f32), ("kd", c_f32),
                ("abio_on", c_i32), ("j_ab", c_i32), ("j_mk", c_i32), ("ka", c_f32),
                ("surface_only", c_i32), ("sorp_on", c_i32), ("j_c", c_i32), ("j_s", c_i32),
                ("k_sorp", c_f32), ("inv_kd_sorp", c_f32), ("pad1", c_i32)]


class AdrGeom(ctypes.Structure):
    _fields_ = [("nd", c_i32), ("dims", c_i32 * 3), ("pore_code", c_i32), ("biofilm_code", c_i32)]


class AdrStats(ctypes.Structure):
    _fields_ = [("solute_voxels", c_i64), ("biofilm_voxels", c_i64), ("mean_axial", c_f32),
                ("mean_speed", c_f32), ("vmax", c_f32 * 3), ("pad", c_f32)]


class AdrRunParams(ctypes.Structure):
    _fields_ = [("limit", c_i64), ("until_conv", c_i32), ("check", c_i32), ("tol", c_f64),
                ("ratio", c_f64)]


class AdrResult(ctypes.Structure):
    _fields_ = [("steps", c_i64), ("hit_cap", c_i32), ("ladder", c_i32), ("checks", c_i64),
                ("last_rest", c_f64)]


PROGRESS_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, c_i64, c_i64, c_f64, c_f64)

# every entry point of include/prtlb.h with its ctypes prototype
_PROTOS = {
    "prt_abi_version": (ctypes.c_int, []),
    "prt_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "prt_destroy": (None, [ctypes.c_void_p]),
    "prt_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "prt_kernel_launches": (c_i64, [ctypes.c_void_p]),
    "prt_sizeof": (ctypes.c_size_t, [ctypes.c_int]),
    "prt_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "prt_last_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(c_f64)]),
    "prt_flow": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(FlowParams),
                                ctypes.c_void_p, ctypes.POINTER(FlowInfo)]),
    "prt_flow_dev": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(FlowParams),
                                    ctypes.c_void_p, ctypes.POINTER(FlowInfo)]),
    "prt_flow_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(FlowParams),
                                        ctypes.c_void_p, ctypes.POINTER(FlowInfo),
                                        ctypes.c_void_p]),
    "prt_adr_stage": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.POINTER(AdrGeom), ctypes.POINTER(AdrStats)]),
    "prt_adr_stage_dev": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.POINTER(AdrGeom), ctypes.POINTER(AdrStats)]),
    "prt_adr_begin": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AdrParams)]),
    "prt_adr_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AdrRunParams), PROGRESS_CB,
                                   ctypes.c_void_p, ctypes.POINTER(AdrResult)]),
    "prt_adr_ladder": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(c_i64), c_i32,
                                      ctypes.POINTER(c_i32)]),
    "prt_adr_fetch": (ctypes.c_int, [ctypes.c_void_p, c_i32, ctypes.c_void_p]),
    "prt_adr_fetch_dev": (ctypes.c_int, [ctypes.c_void_p, c_i32, ctypes.c_void_p]),
    "prt_adr_means": (ctypes.c_int, [ctypes.c_void_p, c_i32, ctypes.POINTER(c_f32)]),
    "prt_adr_end": (ctypes.c_int, [ctypes.c_void_p]),
    "prt_adr_release": (ctypes.c_int, [ctypes.c_void_p]),
    "prt_physics_stage": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                         ctypes.c_int32, ctypes.c_int32]),
    "prt_physics_stats_dev": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                             ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_void_p]),
    "prt_physics_moments_dev": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                               ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                               ctypes.c_int32, ctypes.POINTER(c_f64)]),
    "prt_physics_maxdev_dev": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                              ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                              ctypes.c_int32, ctypes.c_float,
                                              ctypes.POINTER(ctypes.c_float)]),
    "prt_label_materials": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                           ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p]),
    "prt_walk_from_plane": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                           ctypes.POINTER(ctypes.c_int32), ctypes.c_int32,
                                           ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                           ctypes.POINTER(ctypes.c_int64),
                                           ctypes.POINTER(ctypes.c_int64)]),
    "prt_inlet_walk": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                      ctypes.POINTER(ctypes.c_int32), ctypes.c_int32,
                                      ctypes.c_int32, ctypes.c_void_p,
                                      ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(ctypes.c_int64)]),
    # split solves and the batch engine
    "prt_flow_start": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(FlowParams)]),
    "prt_flow_finish": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(FlowInfo)]),
    "prt_adr_stage_flow": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AdrGeom),
                                          ctypes.POINTER(AdrStats)]),
    "prt_flow_release": (ctypes.c_int, [ctypes.c_void_p]),
    "prt_adr_start": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AdrRunParams)]),
    "prt_adr_finish": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AdrResult)]),
    "prt_flow_launch": (ctypes.c_int, [ctypes.c_void_p]),
    "prt_adr_launch": (ctypes.c_int, [ctypes.c_void_p]),
    "prt_ctx_busy": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(c_i32)]),
    "prt_batch_create": (ctypes.c_int, [ctypes.c_int, c_i32, ctypes.POINTER(ctypes.c_void_p)]),
    "prt_batch_destroy": (None, [ctypes.c_void_p]),
    "prt_batch_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "prt_batch_add": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "prt_batch_remove": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "prt_batch_launch": (ctypes.c_int, [ctypes.c_void_p, c_i32]),
    "prt_batch_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(c_i32)]),
    "prt_batch_run": (ctypes.c_int, [ctypes.c_void_p, c_i32, ctypes.POINTER(c_i32)]),
    "prt_batch_collect": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), c_i32,
                                         ctypes.POINTER(c_i32)]),
    "prt_batch_size": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(c_i32),
                                      ctypes.POINTER(c_i32)]),
    "prt_batch_tune": (ctypes.c_int, [ctypes.c_void_p, c_i32, c_i32]),
    "prt_batch_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(c_f64)]),
    "prt_mem_info": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_uint64),
                                    ctypes.POINTER(ctypes.c_uint64)]),
    "prt_pack_balls": (c_i64, [ctypes.c_void_p, c_i32, ctypes.POINTER(c_i32), ctypes.c_void_p,
                               c_i64, c_f64, c_f64, c_f64, c_i64, c_i64, ctypes.c_void_p,
                               ctypes.c_void_p, c_i64, ctypes.POINTER(c_i64)]),
}

class PhysicsStats(ctypes.Structure):
    """prt_physics_stats of include/prtlb.h."""
    _fields_ = [("n_nan", ctypes.c_int64), ("n_inf", ctypes.c_int64),
                ("n_triples", ctypes.c_int64), ("n_flips", ctypes.c_int64),
                ("has_pore", ctypes.c_int32 * 8), ("pore_max", ctypes.c_float * 8),
                ("pore_min", ctypes.c_float * 8), ("final_absmax", ctypes.c_float * 8),
                ("mid_max", ctypes.c_float * 256), ("end_max", ctypes.c_float * 256)]


SIZEOF_ORDER = [FlowParams, FlowInfo, AdrParams, AdrRunParams, AdrResult, AdrGeom, AdrStats,
                PhysicsStats]

_lib = None
_lib_lock = threading.Lock()


class PrtError(RuntimeError):
    """A failed libprtlb call (status code and the library's message)."""

    def __init__(self, code, msg):
        super().__init__("libprtlb error %d: %s" % (code, msg))
        self.code = code
        self.msg = msg


def lib():
    """The loaded library, prototypes set.  Raises if it is not built."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    "libprtlb.so is not built (expected at %s); run "
                    "`make -C prt-deeponet-gui_b200/csrc`.  There is no CPU fallback."
                    % LIB_PATH)
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in _PROTOS.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
        return _lib


class Context(object):
    """One libprtlb context: a CUDA device and a stream.  Calls are serialised."""

    def __init__(self, device=0):
        L = lib()
        h = ctypes.c_void_p()
        rc = L.prt_create(int(device), ctypes.byref(h))
        if rc != PRT_OK:
            msg = L.prt_last_error(None)
            raise PrtError(rc, msg.decode() if msg else "prt_create failed")
        self.handle = h
        self.device = int(device)
        self.lock = threading.RLock()

    def check(self, rc):
        if rc != PRT_OK:
            msg = lib().prt_last_error(self.handle)
            raise PrtError(rc, msg.decode() if msg else "")

    def launches(self):
        return int(lib().prt_kernel_launches(self.handle))

    def stream(self):
        """The context's cudaStream_t as an integer."""
        return int(lib().prt_stream(self.handle) or 0)

    def timing(self):
        """(flow loop ms, flow iterations, transport loop ms, transport steps)
        of the last solves, from CUDA events on the context's stream."""
        out = (c_f64 * 4)()
        self.check(lib().prt_last_timing(self.handle, out))
        return tuple(float(x) for x in out)

    def close(self):
        if self.handle:
            lib().prt_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts = {}
_ctx_lock = threading.Lock()


def default_context(device=None):
    """The process-wide context of `device` (default: 0), created on first use."""
    dev = 0 if device is None else int(device)
    with _ctx_lock:
        c = _contexts.get(dev)
        if c is None or c.handle is None:
            c = Context(dev)
            _contexts[dev] = c
        return c


def close_all():
    with _ctx_lock:
        for c in _contexts.values():
            c.close()
        _contexts.clear()


import atexit  # noqa: E402

atexit.register(close_all)
