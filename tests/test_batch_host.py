"""Host side of the batch API (no GPU needed): request validation, the
library entry points, and a clear error when no device is present."""

import pytest


def test_request_defaults_and_validation():
    import numpy as np
    from prtlb_gpu.batch import Request
    g = np.full((8, 6, 6), 2, np.uint8)
    r = Request(g, flow=dict(nit=10), adr=dict(pe=1.0, da=1.0, n_t=2))
    assert r.flow["nit"] == 10 and r.flow["tau_lb"] == 0.8 and r.flow["precision"] == "fp64"
    assert r.adr["max_steps"] == 100000 and r.adr["steps"] is None and r.adr["n_species"] == 2
    with pytest.raises(ValueError):
        Request(g, adr=dict(pe=1.0, da=1.0))
    assert Request(g).adr is None


def test_batch_entry_points_are_bound():
    from prtlb_gpu import _lib
    L = _lib.lib()
    for name in ("prt_flow_start", "prt_flow_finish", "prt_adr_stage_flow", "prt_flow_release",
                 "prt_adr_start", "prt_adr_finish", "prt_batch_create", "prt_batch_destroy",
                 "prt_batch_add", "prt_batch_remove", "prt_batch_launch", "prt_batch_wait",
                 "prt_batch_run", "prt_batch_collect", "prt_batch_size", "prt_batch_tune",
                 "prt_batch_stats", "prt_batch_last_error", "prt_mem_info"):
        assert getattr(L, name).argtypes is not None, name


def test_null_arguments_are_refused():
    from prtlb_gpu import _lib
    L = _lib.lib()
    assert L.prt_batch_create(0, 0, None) == _lib.PRT_E_INVALID
    assert L.prt_batch_launch(None, 1) == _lib.PRT_E_INVALID
    assert L.prt_batch_wait(None, None) == _lib.PRT_E_INVALID
    assert L.prt_batch_add(None, None) == _lib.PRT_E_INVALID
    assert L.prt_flow_start(None, None, None) == _lib.PRT_E_INVALID
    assert L.prt_adr_finish(None, None) == _lib.PRT_E_INVALID


def test_batch_without_a_gpu_raises():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from prtlb_gpu import _lib
    from prtlb_gpu.batch import Batch
    with pytest.raises(_lib.PrtError) as e:
        Batch()
    assert e.value.code == _lib.PRT_E_NODEV
