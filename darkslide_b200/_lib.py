"""ctypes binding of libdsgpu.so (the C ABI in include/dsgpu.h).

The library is built in-tree (``python -m darkslide_b200.build``). There is no
CPU fallback: if the library or a CUDA device is missing, calls raise.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdsgpu.so")

DSGPU_OK = 0
DSGPU_ERR_ARG = -1
DSGPU_ERR_CFA = -2
DSGPU_ERR_SIZE = -3
DSGPU_ERR_NOMEM = -4
DSGPU_ERR_CUDA = -5
DSGPU_ERR_NODEV = -6
DSGPU_ERR_TIMEOUT = -7
DSGPU_ERR_UNSUPPORTED = -8
DSGPU_HOST = 1
DSGPU_ASYNC = 2
DSGPU_FP16_STAGING = 4
DSGPU_HIGHLIGHTS = 8
DSGPU_QUALITY_DRAFT = 0
DSGPU_QUALITY_FULL = 1
DSGPU_STAGE_DEMOSAIC = 0
DSGPU_STAGE_NLM = 1
DSGPU_STAGE_COPY = 2
DSGPU_STAGE_CNN = 3
DSGPU_STAGE_CNN_HIDDEN = 4
DSGPU_NOALLOC_MAX_PIXELS = 1 << 20

# every symbol include/dsgpu.h and include/dsgpu_scene.h declare
EXPORTS = [
    "dsgpu_strerror", "dsgpu_abi_version", "dsgpu_create", "dsgpu_destroy", "dsgpu_set_stream",
    "dsgpu_get_stream", "dsgpu_synchronize", "dsgpu_trim", "dsgpu_last_error", "dsgpu_set_black_pattern",
    "dsgpu_selftest_batch_timeout",
    "dsgpu_normalize_u16",
    "dsgpu_clip_plane", "dsgpu_mhc", "dsgpu_rcd", "dsgpu_demosaic", "dsgpu_box_blur", "dsgpu_nlm",
    "dsgpu_develop_u16", "dsgpu_develop_u16_noalloc", "dsgpu_estimate_noise", "dsgpu_guided_filter",
    "dsgpu_oklab_matrices", "dsgpu_denoise", "dsgpu_cnn_param_count", "dsgpu_cnn_create", "dsgpu_cnn_destroy",
    "dsgpu_cnn_state", "dsgpu_cnn_gradients", "dsgpu_cnn_train_step", "dsgpu_cnn_infer", "dsgpu_cnn_denoise",
    "dsgpu_develop_u16_cnn", "dsgpu_cnn_set_engine", "dsgpu_cnn_set_clip", "dsgpu_cnn_set_loss",
    "dsgpu_cnn_set_judge", "dsgpu_cnn_judge_stats", "dsgpu_cnn_judge_tile", "dsgpu_profile", "dsgpu_stage_ms", "dsgpu_launch_count", "dsgpu_measure_peaks",
    "dsgpu_measure_mma_sync",
    "dsgpu_scene_render_host", "dsgpu_scene_truth_host", "dsgpu_scene_render", "dsgpu_scene_render_window",
    "dsgpu_cfa_clip_levels", "dsgpu_reconstruct_highlights", "dsgpu_apply_orientation", "dsgpu_rcd_nlm_batch", "dsgpu_batch_frame_ms", "dsgpu_autotune", "dsgpu_autotune_get", "dsgpu_autotune_set",
]


class DsgpuError(RuntimeError):
    def __init__(self, status: int, where: str = "", detail: str = ""):
        self.status = status
        msg = f"{where}: {strerror(status)} ({status})"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


class Frame(ctypes.Structure):
    """dsgpu_frame: one frame of a batched develop (device pointers)."""
    _fields_ = [
        ("raw", ctypes.c_void_p),
        ("pitch_elems", ctypes.c_size_t),
        ("w", ctypes.c_int),
        ("h", ctypes.c_int),
        ("cfa", ctypes.c_uint8 * 4),
        ("black", ctypes.c_float),
        ("white", ctypes.c_float * 3),
        ("mul", ctypes.c_float * 3),
        ("h_param", ctypes.c_float),
        ("out_rgb", ctypes.c_void_p),
        ("out_clip", ctypes.c_void_p),
        ("black_pattern", ctypes.c_void_p),
        ("black_w", ctypes.c_int),
        ("black_h", ctypes.c_int),
        ("black_x0", ctypes.c_int),
        ("black_y0", ctypes.c_int),
    ]


class SceneDesc(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("w", ctypes.c_int),
        ("h", ctypes.c_int),
        ("cfa", ctypes.c_uint8 * 4),
        ("black", ctypes.c_int),
        ("white", ctypes.c_int),
        ("gain_e_per_dn", ctypes.c_float),
        ("read_sigma_dn", ctypes.c_float),
    ]


_lib = None
_lock = threading.Lock()


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m darkslide_b200.build`")
            L = ctypes.CDLL(LIB_PATH)
            vp, i, f, u, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_uint, ctypes.c_size_t
            L.dsgpu_strerror.restype = ctypes.c_char_p
            L.dsgpu_strerror.argtypes = [i]
            L.dsgpu_abi_version.restype = i
            L.dsgpu_create.argtypes = [i, ctypes.POINTER(vp)]
            L.dsgpu_destroy.argtypes = [vp]
            L.dsgpu_set_stream.argtypes = [vp, vp]
            L.dsgpu_get_stream.argtypes = [vp]
            L.dsgpu_get_stream.restype = vp
            L.dsgpu_synchronize.argtypes = [vp]
            L.dsgpu_trim.argtypes = [vp]
            L.dsgpu_last_error.argtypes = [vp]
            L.dsgpu_last_error.restype = ctypes.c_char_p
            L.dsgpu_normalize_u16.argtypes = [vp, vp, i, i, sz, vp, f, vp, vp, u]
            L.dsgpu_set_black_pattern.argtypes = [vp, vp, i, i, i, i]
            L.dsgpu_selftest_batch_timeout.argtypes = [vp]
            L.dsgpu_clip_plane.argtypes = [vp, vp, i, i, vp, u]
            L.dsgpu_mhc.argtypes = [vp, vp, i, i, vp, vp, vp, u]
            L.dsgpu_rcd.argtypes = [vp, vp, i, i, vp, vp, vp, u]
            L.dsgpu_demosaic.argtypes = [vp, vp, i, i, vp, vp, i, vp, vp, u]
            L.dsgpu_box_blur.argtypes = [vp, vp, i, i, i, vp, u]
            L.dsgpu_nlm.argtypes = [vp, vp, i, i, i, f, i, i, vp, u]
            L.dsgpu_develop_u16.argtypes = [vp, vp, i, i, sz, vp, f, vp, vp, f, i, i, vp, vp, u]
            L.dsgpu_develop_u16_noalloc.argtypes = [vp, vp, i, i, sz, vp, f, vp, vp, f, i, i, vp, vp, u]
            L.dsgpu_estimate_noise.argtypes = [vp, vp, i, i, ctypes.POINTER(f), u]
            L.dsgpu_guided_filter.argtypes = [vp, vp, vp, i, i, i, f, vp, u]
            L.dsgpu_oklab_matrices.argtypes = [vp]
            L.dsgpu_denoise.argtypes = [vp, vp, i, i, f, vp, u]
            L.dsgpu_cnn_param_count.argtypes = []
            L.dsgpu_cnn_create.argtypes = [vp, i, i, ctypes.POINTER(vp)]
            L.dsgpu_cnn_destroy.argtypes = [vp, vp]
            L.dsgpu_cnn_state.argtypes = [vp, vp, i, vp, i, ctypes.POINTER(ctypes.c_longlong), u]
            L.dsgpu_cnn_gradients.argtypes = [vp, vp, vp, vp, f, vp, i, vp, ctypes.POINTER(f), u]
            L.dsgpu_cnn_train_step.argtypes = [vp, vp, vp, vp, f, vp, i, f, ctypes.POINTER(f)]
            L.dsgpu_cnn_infer.argtypes = [vp, vp, vp, i, i, f, vp, u]
            L.dsgpu_cnn_denoise.argtypes = [vp, vp, vp, i, i, f, i, i, f, vp, ctypes.POINTER(i), u]
            L.dsgpu_develop_u16_cnn.argtypes = [vp, vp, vp, i, i, sz, vp, f, vp, vp, f, i, i, f, vp, vp, u]
            L.dsgpu_measure_mma_sync.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
            L.dsgpu_cnn_set_engine.argtypes = [vp, vp, i]
            L.dsgpu_cnn_set_judge.argtypes = [vp, vp, f, f, u]
            L.dsgpu_cnn_judge_stats.argtypes = [vp, vp, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(f),
                                                ctypes.POINTER(f)]
            L.dsgpu_cnn_judge_tile.argtypes = [u, f, i]
            L.dsgpu_cnn_set_clip.argtypes = [vp, vp, f]
            L.dsgpu_cnn_set_loss.argtypes = [vp, vp, i]
            L.dsgpu_profile.argtypes = [vp, i]
            L.dsgpu_stage_ms.argtypes = [vp, i, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(i)]
            L.dsgpu_launch_count.argtypes = [vp]
            L.dsgpu_measure_peaks.argtypes = [vp] + [ctypes.POINTER(ctypes.c_double)] * 3
            L.dsgpu_scene_render_host.argtypes = [ctypes.POINTER(SceneDesc), i, i, i, i, vp]
            L.dsgpu_scene_truth_host.argtypes = [ctypes.POINTER(SceneDesc), i, i, i, i, vp]
            L.dsgpu_scene_render.argtypes = [vp, ctypes.POINTER(SceneDesc), vp, u]
            L.dsgpu_scene_render_window.argtypes = [vp, ctypes.POINTER(SceneDesc), i, i, i, i, vp, u]
            L.dsgpu_apply_orientation.argtypes = [vp, vp, i, i, i, vp, u]
            L.dsgpu_cfa_clip_levels.argtypes = [vp, vp, i, i, vp, ctypes.POINTER(f), u]
            L.dsgpu_reconstruct_highlights.argtypes = [vp, vp, vp, i, i, vp, vp, u]
            L.dsgpu_rcd_nlm_batch.argtypes = [vp, ctypes.POINTER(Frame), i, i, i, u]
            L.dsgpu_batch_frame_ms.argtypes = [vp, ctypes.POINTER(ctypes.c_double), i]
            L.dsgpu_autotune.argtypes = [vp, ctypes.POINTER(i), i, i, i]
            L.dsgpu_autotune_get.argtypes = [vp, i, i, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(i),
                                             ctypes.POINTER(ctypes.c_double)]
            L.dsgpu_autotune_set.argtypes = [vp, i, i, i, i, i]
            for name in EXPORTS:
                if name not in ("dsgpu_strerror", "dsgpu_get_stream", "dsgpu_last_error", "dsgpu_launch_count"):
                    getattr(L, name).restype = i
            L.dsgpu_launch_count.restype = ctypes.c_ulonglong
            _lib = L
    return _lib


def strerror(status: int) -> str:
    return lib().dsgpu_strerror(int(status)).decode()


class Context:
    """One dsgpu context: a device, a stream and cached scratch (dsgpu_create)."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        st = lib().dsgpu_create(int(device), ctypes.byref(h))
        if st != DSGPU_OK:
            raise DsgpuError(st, "dsgpu_create")
        self.handle = h
        self.device = int(device)

    def check(self, status: int, where: str) -> None:
        if status != DSGPU_OK:
            detail = lib().dsgpu_last_error(self.handle)
            raise DsgpuError(status, where, detail.decode() if detail else "")

    def set_stream(self, stream_ptr: int | None) -> None:
        """Order the context's work on a CUDA stream handle: None = the
        context's own stream; 0 (torch's default stream) = CUDA's legacy
        default stream (handle 1), which orders with torch's work on it."""
        handle = 0 if stream_ptr is None else (1 if stream_ptr == 0 else stream_ptr)
        self.check(lib().dsgpu_set_stream(self.handle, ctypes.c_void_p(handle)), "dsgpu_set_stream")

    def synchronize(self) -> None:
        self.check(lib().dsgpu_synchronize(self.handle), "dsgpu_synchronize")

    def set_black_pattern(self, levels=None, origin=(0, 0)) -> None:
        """Per-site black levels for this context's u16 calls (load_raw's
        black_at, decode.rs:266-270): ``levels`` a (bh, bw) array of up to
        4 x 4, indexed at uncropped sensor coordinates; ``origin`` the crop
        origin (x, y) of the frames passed. None clears it (the scalar black
        arguments apply again)."""
        import numpy as np

        if levels is None:
            self.check(lib().dsgpu_set_black_pattern(self.handle, None, 0, 0, 0, 0), "dsgpu_set_black_pattern")
            return
        a = np.ascontiguousarray(np.asarray(levels, np.float32))
        if a.ndim != 2:
            raise DsgpuError(DSGPU_ERR_ARG, "set_black_pattern", "levels must be a (bh, bw) array")
        bh, bw = a.shape
        self.check(lib().dsgpu_set_black_pattern(self.handle, ctypes.c_void_p(a.ctypes.data), int(bw), int(bh),
                                                 int(origin[0]), int(origin[1])), "dsgpu_set_black_pattern")

    def profile(self, enable: bool) -> None:
        self.check(lib().dsgpu_profile(self.handle, int(bool(enable))), "dsgpu_profile")

    def stage_ms(self, stage: int) -> tuple[float, int]:
        t, n = ctypes.c_double(), ctypes.c_int()
        self.check(lib().dsgpu_stage_ms(self.handle, int(stage), ctypes.byref(t), ctypes.byref(n)), "dsgpu_stage_ms")
        return t.value, n.value

    def launch_count(self) -> int:
        return int(lib().dsgpu_launch_count(self.handle))

    def measure_peaks(self) -> tuple[float, float, float]:
        """(FP32 FMA FLOP/s, ex2/s, packed f32x2 FMA FLOP/s) on this device."""
        f, e, f2 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self.check(lib().dsgpu_measure_peaks(self.handle, ctypes.byref(f), ctypes.byref(e), ctypes.byref(f2)),
                   "dsgpu_measure_peaks")
        return f.value, e.value, f2.value

    def measure_mma_sync(self) -> float:
        f = ctypes.c_double()
        self.check(lib().dsgpu_measure_mma_sync(self.handle, ctypes.byref(f)), "dsgpu_measure_mma_sync")
        return f.value

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and _lib is not None:
            lib().dsgpu_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


_default: dict[int, Context] = {}


def default_context(device: int = 0) -> Context:
    ctx = _default.get(device)
    if ctx is None:
        ctx = _default[device] = Context(device)
    return ctx
