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



def _oracle_speckle(D, sim, size):
    """The oracle's post-filter with speckle removal as its only pass (the
    regular entry point's speckle stage equals it; see the parity tests)."""
    import oracle

    p = eb.params_reference()
    p.speckle_sim_threshold = sim
    p.speckle_size = size
    return oracle.postprocess(D, p)


def _blocky(rng, h, w):
    """Piecewise-constant segments of varied size, +0.5 jitter, 10 % holes."""
    base = rng.integers(0, 40, (h // 4 + 1, w // 4 + 1)).astype(np.float32)
    D = np.kron(base, np.ones((4, 4), np.float32))[:h, :w].copy()
    D += rng.integers(0, 2, (h, w)).astype(np.float32) * 0.5
    D[rng.random((h, w)) < 0.1] = -1.0
    return np.ascontiguousarray(D)


def test_speckle_noalloc_in_place_small_after_large_and_no_op():
    """In place (d_in == d_out); a small map right after a large one (the
    shared scratch still holds the large map's labels); a one-column map
    taller than the 65535-row limit of a grid's y dimension; min_size = 0
    (output equals input).  Each against the oracle's speckle pass."""
    import torch

    fn = _entry()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(5)
    for h, w, size in [(700, 740, 12), (33, 47, 5), (70000, 1, 3), (600, 800, 0)]:
        D = _blocky(rng, h, w)
        d = torch.from_numpy(D.copy()).cuda()
        torch.cuda.synchronize()
        rc = fn(d.data_ptr(), d.data_ptr(), w, h, 1.0, size, stream)
        assert rc == eb.ELAS_OK, (h, w, rc)
        torch.cuda.synchronize()
        got = d.cpu().numpy()
        if size == 0:
            assert np.array_equal(got, D)
        else:
            np.testing.assert_allclose(got, _oracle_speckle(D, 1.0, size), atol=1e-4, rtol=0)
