"""Allocation-free speckle removal (elas_b200_speckle_noalloc) through the
C ABI.  Callers that cannot call cudaMalloc -- inside a stream capture, in
plugin hosts or real-time loops that forbid allocation -- use it; its
scratch is a fixed array inside the library.  Its output must equal the
speckle stage of the regular entry point, call after call (the scratch is
shared and keeps the previous call's contents).
"""
import ctypes

import numpy as np
import pytest

import elas_b200 as eb

pytestmark = pytest.mark.gpu


def _entry():
    lib = eb.library()
    fn = lib.elas_b200_speckle_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                   ctypes.c_int32, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def test_speckle_noalloc_matches_regular_entry_point():
    import torch

    fn = _entry()
    p = eb.params_reference()
    p.speckle_size = 200
    e = eb.Elas(p)
    stream = torch.cuda.current_stream()
    try:
        for seed in (1, 2):          # two calls in a row on different maps
            L, R, _, _ = eb.synth_pair(1, seed)
            H, W = L.shape
            D1, _ = e.process(L, R)
            lr = e.stage("lr_left").view(np.float32).reshape(H, W)
            d_in = torch.from_numpy(lr.copy()).cuda()
            d_out = torch.full_like(d_in, 12345.0)
            torch.cuda.synchronize()
            rc = fn(d_in.data_ptr(), d_out.data_ptr(), W, H, p.speckle_sim_threshold, p.speckle_size,
                    stream.cuda_stream)
            assert rc == eb.ELAS_OK
            torch.cuda.synchronize()
            np.testing.assert_allclose(d_out.cpu().numpy(), D1, atol=1e-4, rtol=0)
    finally:
        e.close()


def test_speckle_noalloc_rejects_oversized_input():
    import torch

    fn = _entry()
    buf = torch.zeros(16, device="cuda")
    assert fn(buf.data_ptr(), buf.data_ptr(), 2048, 1024, 1.0, 200, None) == 8   # ELAS_ERR_TOO_LARGE
