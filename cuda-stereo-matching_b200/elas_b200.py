"""Python binding of the ELAS B200 library (ctypes over include/elas_b200.h).

Mirrors the reference's interface (src/Elas.h): an ``Elas`` object built
from an ``Elas.parameters``-compatible block whose ``process(left, right)``
returns the left and right disparity maps (float32, -1 = invalid).  All work
runs in ``libelas_b200.so``; there is no CPU fallback: if the library or a
B200 is missing the calls raise.
"""
import ctypes
import os
from ctypes import POINTER, c_bool, c_float, c_int, c_int32, c_int64, c_size_t, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# ELAS_B200_LIB may name another build of the library (for side-by-side measurements)
LIB_PATH = os.environ.get("ELAS_B200_LIB") or os.path.join(HERE, "libelas_b200.so")

ELAS_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "unsupported", 3: "CUDA error", 4: "out of memory",
          5: "internal consistency check failed", 6: "no usable sm_100 device", 7: "bounded device loop hit its limit",
          8: "input exceeds the fixed scratch capacity of the allocation-free entry point"}

STAGES = {
    "desc_left": 0, "desc_right": 1, "can_lr": 2, "can": 3, "support": 4, "grid_left": 5, "grid_right": 6,
    "tri_left": 7, "tri_right": 8, "prior_left": 9, "prior_right": 10, "disp_left": 11, "disp_right": 12,
    "lr_left": 13, "lr_right": 14, "pn_features": 15, "pn_output": 16, "pn_bins": 17, "del_counters": 18,
}

PN_PARAMS = 36992
PN_WEIGHTS = os.path.join(HERE, "weights", "proposal.f32")


def bf16_to_f32(raw):
    """bf16 values (raw uint16 / bytes) -> float32."""
    u = np.frombuffer(np.ascontiguousarray(raw).tobytes(), np.uint16).astype(np.uint32) << 16
    return u.view(np.float32)


def load_proposal(path=PN_WEIGHTS):
    """Trained proposal parameters (ELAS_PN_PARAMS little-endian float32)."""
    w = np.fromfile(path, np.float32)
    if w.size != PN_PARAMS:
        raise ElasError(1, f"{path}: {w.size} values, expected {PN_PARAMS}")
    return w


class ElasParams(ctypes.Structure):
    """Byte-compatible with Elas::parameters (reference src/Elas.h:14-40)."""

    _fields_ = [
        ("disp_min", c_int32), ("disp_max", c_int32), ("support_threshold", c_float),
        ("support_texture", c_int32), ("candidate_stepsize", c_int32), ("incon_window_size", c_int32),
        ("incon_threshold", c_int32), ("incon_min_support", c_int32), ("add_corners", c_bool),
        ("grid_size", c_int32), ("beta", c_float), ("gamma", c_float), ("sigma", c_float), ("sradius", c_float),
        ("match_texture", c_int32), ("lr_threshold", c_int32), ("speckle_sim_threshold", c_float),
        ("speckle_size", c_int32), ("ipol_gap_width", c_int32), ("filter_median", c_bool),
        ("filter_adaptive_mean", c_bool), ("postprocess_only_left", c_bool), ("subsampling", c_bool),
    ]

    def copy(self):
        p = ElasParams()
        ctypes.pointer(p)[0] = self
        return p

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class ElasError(RuntimeError):
    def __init__(self, status, msg=""):
        super().__init__(f"{STATUS.get(status, status)} ({status}){': ' + msg if msg else ''}")
        self.status = status


_lib = None


def library():
    """Load libelas_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ElasError(1, f"{LIB_PATH} is missing; run __graft_entry__.build()")
        lib = ctypes.CDLL(LIB_PATH)
        pp = POINTER(ElasParams)
        lib.elas_params_default.argtypes = [pp]
        lib.elas_params_reference.argtypes = [pp]
        lib.elas_b200_status_string.restype = ctypes.c_char_p
        lib.elas_b200_status_string.argtypes = [c_int]
        lib.elas_b200_create.argtypes = [pp, c_int, POINTER(c_void_p)]
        lib.elas_b200_destroy.argtypes = [c_void_p]
        lib.elas_b200_set_params.argtypes = [c_void_p, pp]
        lib.elas_b200_get_params.argtypes = [c_void_p, pp]
        lib.elas_b200_last_error.restype = ctypes.c_char_p
        lib.elas_b200_last_error.argtypes = [c_void_p]
        lib.elas_b200_process.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
        lib.elas_b200_process_device.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                                 c_void_p]
        lib.elas_b200_process_batch.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                                c_void_p, c_void_p]
        lib.elas_b200_process_batch_device.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                                       c_void_p, c_void_p, c_void_p]
        lib.elas_b200_set_graphs.argtypes = [c_void_p, c_int]
        lib.elas_b200_set_test_mode.argtypes = [c_void_p, c_int32, c_int32]
        lib.elas_b200_group_create.argtypes = [pp, c_void_p, c_int, POINTER(c_void_p)]
        lib.elas_b200_group_destroy.argtypes = [c_void_p]
        lib.elas_b200_group_set_params.argtypes = [c_void_p, pp]
        lib.elas_b200_group_last_error.restype = ctypes.c_char_p
        lib.elas_b200_group_last_error.argtypes = [c_void_p]
        lib.elas_b200_group_plan.argtypes = [c_int, c_void_p, c_void_p, c_int32, c_int, c_void_p]
        lib.elas_b200_group_process_batch.argtypes = [c_void_p, c_int] + [c_void_p] * 7
        lib.elas_b200_batch_latency.argtypes = [c_void_p, c_void_p, c_int]
        lib.elas_b200_dense_shape.argtypes = [c_void_p, c_int32, c_int32]
        lib.elas_b200_set_proposal.argtypes = [c_void_p, c_void_p, c_int32]
        lib.elas_b200_proposal_stats.argtypes = [c_void_p, c_void_p, c_int32]
        lib.elas_b200_pn_infer.argtypes = [c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p]
        lib.elas_b200_pn_features.argtypes = [c_void_p, c_void_p, c_void_p]
        lib.elas_b200_pn_bf16_to_f32.argtypes = [c_void_p, c_void_p, c_size_t, c_void_p]
        lib.elas_b200_pn_conv_forward.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32,
                                                  c_int32, c_void_p]
        lib.elas_b200_pn_conv_backward.argtypes = [c_void_p] * 8 + [c_int32] * 4 + [c_void_p]
        lib.elas_b200_pn_corr_loss.argtypes = [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32, c_void_p,
                                               c_void_p, c_void_p, c_void_p]
        lib.elas_b200_pn_adam.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_float, c_float, c_float,
                                          c_float, c_int32, c_void_p]
        lib.elas_b200_get_stage.argtypes = [c_void_p, c_int, c_void_p, c_size_t, POINTER(c_size_t)]
        lib.elas_b200_set_timing.argtypes = [c_void_p, c_int]
        lib.elas_b200_get_timing.argtypes = [c_void_p, c_void_p, c_int]
        lib.elas_b200_launch_count.restype = c_int64
        lib.elas_b200_launch_count.argtypes = [c_void_p]
        lib.elas_b200_synth_pair.argtypes = [c_int, c_uint64, c_int32, c_int32, c_int32, c_void_p, c_void_p,
                                             c_void_p, c_void_p]
        lib.elas_b200_synth_dims.argtypes = [c_int, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32)]
        _lib = lib
    return _lib


def params_default():
    """Elas::parameters() defaults (reference src/Elas.h:42-66)."""
    p = ElasParams()
    library().elas_params_default(ctypes.byref(p))
    return p


def params_reference():
    """The values the reference kernels are compiled with, post-filters off."""
    p = ElasParams()
    library().elas_params_reference(ctypes.byref(p))
    return p


def params_config(disp_max, post=True):
    """Parameters of the benchmark configurations: the reference kernel
    constants with the configured disparity range; post-filters (speckle 200,
    gap width 3, median and adaptive mean) on unless ``post`` is False."""
    p = params_reference()
    p.disp_max = int(disp_max)
    if post:
        p.speckle_size = 200
        p.ipol_gap_width = 3
        p.filter_median = True
        p.filter_adaptive_mean = True
    return p


def _ptr(a):
    return a.ctypes.data_as(c_void_p)


def synth_dims(preset):
    w, h, d = c_int32(), c_int32(), c_int32()
    rc = library().elas_b200_synth_dims(preset, ctypes.byref(w), ctypes.byref(h), ctypes.byref(d))
    if rc:
        raise ElasError(rc)
    return w.value, h.value, d.value


def synth_pair(preset, seed, width=0, height=0, disp_max=0, gt=True):
    """Seeded synthetic pair: (left, right, gt_left, gt_right) (gt None if not asked)."""
    W, H, D = synth_dims(preset)
    W = width or W
    H = height or H
    left = np.empty((H, W), np.uint8)
    right = np.empty((H, W), np.uint8)
    gl = np.empty((H, W), np.float32) if gt else None
    gr = np.empty((H, W), np.float32) if gt else None
    rc = library().elas_b200_synth_pair(preset, seed, W, H, disp_max, _ptr(left), _ptr(right),
                                        _ptr(gl) if gt else None, _ptr(gr) if gt else None)
    if rc:
        raise ElasError(rc)
    return left, right, gl, gr


class Elas:
    """Drop-in for the reference's ``Elas`` class (src/Elas.h:11-83)."""

    def __init__(self, params=None, device=0):
        self._lib = library()
        self._h = c_void_p()
        self.params = (params or params_default()).copy()
        rc = self._lib.elas_b200_create(ctypes.byref(self.params), device, ctypes.byref(self._h))
        if rc != ELAS_OK:
            raise ElasError(rc)

    def close(self):
        if self._h:
            self._lib.elas_b200_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != ELAS_OK:
            msg = self._lib.elas_b200_last_error(self._h)
            raise ElasError(rc, msg.decode() if msg else "")

    def set_params(self, params):
        self._check(self._lib.elas_b200_set_params(self._h, ctypes.byref(params)))
        self.params = params.copy()

    def process(self, left, right, stream=None):
        """left, right: uint8 (H, W) arrays.  Returns (D1, D2) float32."""
        left = np.ascontiguousarray(left, np.uint8)
        right = np.ascontiguousarray(right, np.uint8)
        if left.shape != right.shape or left.ndim != 2:
            raise ElasError(1, "images must be 2-D and of the same size")
        H, W = left.shape
        shape = self.out_shape(W, H)
        d1 = np.empty(shape, np.float32)
        d2 = np.empty(shape, np.float32)
        dims = np.array([W, H, W], np.int32)
        self._check(self._lib.elas_b200_process(self._h, _ptr(left), _ptr(right), _ptr(d1), _ptr(d2), _ptr(dims),
                                                stream))
        return d1, d2

    def out_shape(self, width, height):
        """(rows, columns) of the output maps: (H, W), or (H / 2, W / 2) when
        the parameters ask for subsampling."""
        return (height // 2, width // 2) if self.params.subsampling else (height, width)

    def process_device(self, left_ptr, right_ptr, d1_ptr, d2_ptr, width, height, stream=None):
        """Device-pointer form (ints); asynchronous on `stream` (a cudaStream_t int)."""
        dims = np.array([width, height, width], np.int32)
        self._dims_keepalive = dims
        self._check(self._lib.elas_b200_process_device(self._h, c_void_p(left_ptr), c_void_p(right_ptr),
                                                       c_void_p(d1_ptr), c_void_p(d2_ptr), _ptr(dims),
                                                       c_void_p(stream) if stream else None))

    def process_batch(self, lefts, rights, disp_max=None):
        n = len(lefts)
        outs1, outs2 = [], []
        dims = np.zeros(2 * n, np.int32)
        keep = []
        for i, (l, r) in enumerate(zip(lefts, rights)):
            l = np.ascontiguousarray(l, np.uint8)
            r = np.ascontiguousarray(r, np.uint8)
            keep += [l, r]
            dims[2 * i] = l.shape[1]
            dims[2 * i + 1] = l.shape[0]
            outs1.append(np.empty(self.out_shape(l.shape[1], l.shape[0]), np.float32))
            outs2.append(np.empty(self.out_shape(l.shape[1], l.shape[0]), np.float32))
        arr = lambda xs: (c_void_p * n)(*[x.ctypes.data for x in xs])
        dm = np.asarray(disp_max, np.int32) if disp_max is not None else None
        self._check(self._lib.elas_b200_process_batch(self._h, n, arr(keep[0::2]), arr(keep[1::2]), arr(outs1),
                                                      arr(outs2), _ptr(dims), _ptr(dm) if dm is not None else None,
                                                      None))
        return outs1, outs2

    def process_batch_device(self, lefts, rights, outs1, outs2, dims, disp_max=None, stream=None):
        """Batch on device pointers (ints); dims is a sequence of (width, height).
        Replays a cached CUDA graph when sizes, buffers, parameters and stream
        repeat."""
        n = len(lefts)
        d = np.asarray(dims, np.int32).reshape(-1)
        arr = lambda xs: (c_void_p * n)(*[int(x) for x in xs])
        dm = np.asarray(disp_max, np.int32) if disp_max is not None else None
        self._check(self._lib.elas_b200_process_batch_device(self._h, n, arr(lefts), arr(rights), arr(outs1),
                                                             arr(outs2), _ptr(d), _ptr(dm) if dm is not None else None,
                                                             c_void_p(stream) if stream else None))

    def set_graphs(self, enable=True):
        self._check(self._lib.elas_b200_set_graphs(self._h, int(bool(enable))))

    TEST_FLIP_GLOBAL = 1      # every triangulation on the global-memory flip kernel
    TEST_DENSE_BITSET = 2     # every dense candidate list walked as a bitset
    TEST_PRIOR_TILED = 4      # plane prior painted tile by tile at every size
    TEST_PRIOR_DIRECT = 8     # plane prior painted with global atomics at every size
    TEST_DELAUNAY_FLIPS = 16  # triangulations from row strips and edge flips at every size
    TEST_DELAUNAY_STARS = 32  # triangulations found star by star at every size
    TEST_PRIOR_SMALL_BINS = 256  # tiled prior paint with 2-entry tile bins (the overflow list used)

    def set_test_mode(self, flags=0, flip_round_limit=0):
        """Force fallback paths (results unchanged) and/or cap the flip rounds
        (a triangulation that needs more raises ElasError with status 7)."""
        self._check(self._lib.elas_b200_set_test_mode(self._h, int(flags), int(flip_round_limit)))

    def batch_latency(self, n):
        """Milliseconds from the last batch's start to each pair's completion."""
        out = np.zeros(max(n, 1), np.float32)
        rc = self._lib.elas_b200_batch_latency(self._h, _ptr(out), n)
        if rc < 0:
            self._check(-rc)
        return out[:rc]

    def dense_shape(self, width, disp_max):
        return self._lib.elas_b200_dense_shape(self._h, width, disp_max)

    def stage(self, name):
        """Copy an intermediate stage of the last single-pair call."""
        sid = STAGES[name]
        need = c_size_t()
        self._check(self._lib.elas_b200_get_stage(self._h, sid, None, 0, ctypes.byref(need)))
        buf = np.empty(need.value, np.uint8)
        self._check(self._lib.elas_b200_get_stage(self._h, sid, _ptr(buf), need.value, ctypes.byref(need)))
        return buf

    def set_proposal(self, params):
        """Enable the learned support-point proposal with these parameters
        (ELAS_PN_PARAMS float32), or disable it with None."""
        if params is None:
            self._check(self._lib.elas_b200_set_proposal(self._h, None, 0))
            return
        w = np.ascontiguousarray(params, np.float32)
        self._check(self._lib.elas_b200_set_proposal(self._h, _ptr(w), w.size))

    def proposal_stats(self):
        """(settled by the proposal, sent to the full sweep) for the last call."""
        out = np.zeros(2, np.int32)
        self._check(self._lib.elas_b200_proposal_stats(self._h, _ptr(out), 2))
        return int(out[0]), int(out[1])

    def pn_infer(self, in_ptr, out_ptr, hd, wd, stream=None):
        self._check(self._lib.elas_b200_pn_infer(self._h, c_void_p(in_ptr), c_void_p(out_ptr), hd, wd,
                                                 c_void_p(stream) if stream else None))

    def pn_features(self, out_ptr, stream=None):
        self._check(self._lib.elas_b200_pn_features(self._h, c_void_p(out_ptr), c_void_p(stream) if stream else None))

    TIME_STAGES = ["descriptor", "support", "compact", "grid", "delaunay", "prior", "dense", "lr", "post"]

    def set_timing(self, enable=True):
        self._check(self._lib.elas_b200_set_timing(self._h, int(enable)))

    def timing(self):
        """Per-stage device times (ms) of the last call, as a dict."""
        out = np.zeros(len(self.TIME_STAGES), np.float32)
        self._check(self._lib.elas_b200_get_timing(self._h, _ptr(out), len(out)))
        return dict(zip(self.TIME_STAGES, out.tolist()))

    @property
    def launch_count(self):
        return int(self._lib.elas_b200_launch_count(self._h))


# ---- training kernels of the proposal network (device pointers as ints) ----

def _pn_check(rc):
    if rc != ELAS_OK:
        raise ElasError(rc)


def pn_bf16_to_f32(src, dst, n, stream=None):
    _pn_check(library().elas_b200_pn_bf16_to_f32(c_void_p(src), c_void_p(dst), n, c_void_p(stream) if stream else None))


def pn_conv_forward(x, w, b, y, nimg, hd, wd, relu, stream=None):
    _pn_check(library().elas_b200_pn_conv_forward(c_void_p(x), c_void_p(w), c_void_p(b) if b else None, c_void_p(y),
                                                  nimg, hd, wd, int(relu), c_void_p(stream) if stream else None))


def pn_conv_backward(x, y, w, dy, dx, dw, db, w_scratch, nimg, hd, wd, relu, stream=None):
    _pn_check(library().elas_b200_pn_conv_backward(c_void_p(x), c_void_p(y), c_void_p(w), c_void_p(dy),
                                                   c_void_p(dx) if dx else None, c_void_p(dw), c_void_p(db),
                                                   c_void_p(w_scratch), nimg, hd, wd, int(relu),
                                                   c_void_p(stream) if stream else None))


def pn_corr_loss(f, labels, nlab, hd, wd, disp_max, df, loss_sum, correct, stream=None):
    _pn_check(library().elas_b200_pn_corr_loss(c_void_p(f), c_void_p(labels), nlab, hd, wd, disp_max, c_void_p(df),
                                               c_void_p(loss_sum), c_void_p(correct),
                                               c_void_p(stream) if stream else None))


def pn_adam(p, g, m, v, n, lr, beta1, beta2, eps, step, stream=None):
    _pn_check(library().elas_b200_pn_adam(c_void_p(p), c_void_p(g), c_void_p(m), c_void_p(v), n, lr, beta1, beta2,
                                          eps, step, c_void_p(stream) if stream else None))


# ---- pair-parallel batches over several GPUs ----

def group_plan(dims, ndev, disp_max=None, default_disp_max=255):
    """Device entry of each pair under the group's plan (host only)."""
    d = np.ascontiguousarray(np.asarray(dims, np.int32).reshape(-1))
    n = d.size // 2
    dm = np.ascontiguousarray(np.asarray(disp_max, np.int32)) if disp_max is not None else None
    out = np.zeros(max(n, 1), np.int32)
    rc = library().elas_b200_group_plan(n, _ptr(d), _ptr(dm) if dm is not None else None, int(default_disp_max),
                                        int(ndev), _ptr(out))
    if rc != ELAS_OK:
        raise ElasError(rc)
    return out[:n]


class ElasGroup:
    """One matcher per device entry; batches are dealt to the devices with no
    exchange between them (elas_b200_group_*)."""

    def __init__(self, params, devices):
        self._lib = library()
        self._g = c_void_p()
        self.params = params.copy()
        devs = np.ascontiguousarray(np.asarray(devices, np.int32))
        rc = self._lib.elas_b200_group_create(ctypes.byref(self.params), _ptr(devs), devs.size, ctypes.byref(self._g))
        if rc != ELAS_OK:
            raise ElasError(rc)

    def close(self):
        if self._g:
            self._lib.elas_b200_group_destroy(self._g)
            self._g = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != ELAS_OK:
            msg = self._lib.elas_b200_group_last_error(self._g)
            raise ElasError(rc, msg.decode() if msg else "")

    def set_params(self, params):
        self._check(self._lib.elas_b200_group_set_params(self._g, ctypes.byref(params)))
        self.params = params.copy()

    def process_batch(self, lefts, rights, disp_max=None):
        """Returns (D1 list, D2 list, plan)."""
        n = len(lefts)
        keep, outs1, outs2 = [], [], []
        dims = np.zeros(2 * n, np.int32)
        sub = self.params.subsampling
        for i, (l, r) in enumerate(zip(lefts, rights)):
            l = np.ascontiguousarray(l, np.uint8)
            r = np.ascontiguousarray(r, np.uint8)
            keep += [l, r]
            H, W = l.shape
            dims[2 * i], dims[2 * i + 1] = W, H
            shape = (H // 2, W // 2) if sub else (H, W)
            outs1.append(np.empty(shape, np.float32))
            outs2.append(np.empty(shape, np.float32))
        arr = lambda xs: (c_void_p * n)(*[x.ctypes.data for x in xs])
        dm = np.asarray(disp_max, np.int32) if disp_max is not None else None
        plan = np.zeros(n, np.int32)
        self._check(self._lib.elas_b200_group_process_batch(self._g, n, arr(keep[0::2]), arr(keep[1::2]),
                                                            arr(outs1), arr(outs2), _ptr(dims),
                                                            _ptr(dm) if dm is not None else None, _ptr(plan)))
        return outs1, outs2, plan
