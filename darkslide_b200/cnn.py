"""The learned stand-in for NLM (include/dsgpu.h, "learned path").

A residual CNN of 8 conv3x3 layers (7 -> 48 x 7 -> 3, ReLU; dilations
1, 2, 3, 4, 3, 2, 1, 1, a 35 x 35 receptive field): input the demosaiced
RGB split into its 3x3 local mean and the remainder (so that BF16 keeps the
remainder's precision) plus a constant channel STRENGTH_SCALE * h (h = the NLM
strength of enhance.rs:36), output input + network. It is trained on the GPU,
by the library's own BF16 tensor-core forward/backward kernels and Adam, to
reproduce plain NLM; `infer` runs it and falls back to NLM on tiles whose
removed component fails a residual check.

Checkpoints are a small versioned binary: magic b"DSCNN1\\0\\0", u32 version
(3: the dilated network on the local-mean split input; versions 1-2 held
earlier networks and are refused),
u32 parameter count, i64 Adam step, u64 data seed, then parameters, Adam m and
Adam v as little-endian float32.
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from . import _lib
from ._lib import Context, DsgpuError, default_context, lib

STRENGTH_SCALE = 50.0
LAYERS = [(7, 48)] + [(48, 48)] * 6 + [(48, 3)]  # (cin, cout)
DILATIONS = [1, 2, 3, 4, 3, 2, 1, 1]
MAGIC = b"DSCNN1\0\0"
VERSION = 3


def param_count() -> int:
    return int(lib().dsgpu_cnn_param_count())


def layer_slices():
    """(weights slice, bias slice, (cin, cout)) of each layer in the flat array."""
    out, o = [], 0
    for cin, cout in LAYERS:
        nw = 9 * cout * cin
        out.append((slice(o, o + nw), slice(o + nw, o + nw + cout), (cin, cout)))
        o += nw + cout
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal conv weights, zero biases; the last layer starts at zero, so
    the initial network is the identity (out = in)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(param_count(), np.float32)
    for i, (ws, bs, (cin, cout)) in enumerate(layer_slices()):
        if i == len(LAYERS) - 1:
            continue
        p[ws] = rng.normal(0, np.sqrt(2.0 / (9 * cin)), ws.stop - ws.start).astype(np.float32)
    return p


class ResidualCNN:
    def __init__(self, ctx: Context | None = None, max_batch: int = 0, crop: int = 0, params=None, seed: int = 0):
        self.ctx = ctx or default_context(0)
        h = ctypes.c_void_p()
        self.ctx.check(lib().dsgpu_cnn_create(self.ctx.handle, int(max_batch), int(crop), ctypes.byref(h)),
                       "dsgpu_cnn_create")
        self.handle = h
        self.max_batch, self.crop = max_batch, crop
        self.seed = seed
        self.set_params(init_params(seed) if params is None else params)

    # ---- state
    def _state(self, which: int, buf: np.ndarray | None, set_: bool, step: int | None = None) -> int:
        st = ctypes.c_longlong(step or 0)
        p = buf.ctypes.data_as(ctypes.c_void_p) if buf is not None else ctypes.c_void_p(0)
        self.ctx.check(lib().dsgpu_cnn_state(self.ctx.handle, self.handle, which, p, int(set_),
                                             ctypes.byref(st) if (step is not None or not set_) else None,
                                             _lib.DSGPU_HOST), "dsgpu_cnn_state")
        return int(st.value)

    def get_params(self) -> np.ndarray:
        out = np.empty(param_count(), np.float32)
        self._state(0, out, False)
        return out

    def set_params(self, p) -> None:
        a = np.ascontiguousarray(p, np.float32)
        if a.size != param_count():
            raise DsgpuError(_lib.DSGPU_ERR_ARG, "set_params", f"expected {param_count()} floats")
        self._state(0, a, True)

    @property
    def step(self) -> int:
        return self._state(0, None, False)

    def snapshot(self):
        """(params, m, v, step) on the host: the full training state."""
        m = np.empty(param_count(), np.float32)
        v = np.empty(param_count(), np.float32)
        self._state(1, m, False)
        self._state(2, v, False)
        return self.get_params(), m, v, self.step

    def restore(self, snap) -> None:
        p, m, v, step = snap
        self.set_params(p)
        self._state(1, np.ascontiguousarray(m), True)
        self._state(2, np.ascontiguousarray(v), True, step)

    def save(self, path: str) -> None:
        m = np.empty(param_count(), np.float32)
        v = np.empty(param_count(), np.float32)
        self._state(1, m, False)
        self._state(2, v, False)
        with open(path, "wb") as f:
            f.write(MAGIC + struct.pack("<IIqQ", VERSION, param_count(), self.step, self.seed))
            f.write(self.get_params().astype("<f4").tobytes())
            f.write(m.astype("<f4").tobytes())
            f.write(v.astype("<f4").tobytes())

    def load(self, path: str) -> None:
        with open(path, "rb") as f:
            head = f.read(8 + 24)
            if head[:8] != MAGIC:
                raise DsgpuError(_lib.DSGPU_ERR_ARG, "load", "not a dsgpu CNN checkpoint")
            ver, n, step, seed = struct.unpack("<IIqQ", head[8:])
            if ver != VERSION or n != param_count():
                raise DsgpuError(_lib.DSGPU_ERR_ARG, "load", f"version {ver} / {n} parameters not supported")
            arrs = [np.frombuffer(f.read(4 * n), "<f4").astype(np.float32) for _ in range(3)]
        self.set_params(arrs[0])
        self._state(1, np.ascontiguousarray(arrs[1]), True)
        self._state(2, np.ascontiguousarray(arrs[2]), True, step)
        self.seed = seed

    # ---- compute (device tensors)
    def _ptr(self, t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)

    def gradients(self, rgb, strength, target, strength_map=None):
        """(grads, loss_sum) for a device batch rgb/target [B, crop, crop, 3]."""
        import torch

        g = torch.empty(param_count(), dtype=torch.float32, device=rgb.device)
        loss = ctypes.c_float()
        self.ctx.set_stream(torch.cuda.current_stream(rgb.device).cuda_stream)
        self.ctx.check(lib().dsgpu_cnn_gradients(self.ctx.handle, self.handle, self._ptr(rgb), self._ptr(strength_map),
                                                 float(strength), self._ptr(target), rgb.shape[0], self._ptr(g),
                                                 ctypes.byref(loss), 0), "dsgpu_cnn_gradients")
        return g, float(loss.value)

    def train_step(self, rgb, strength, target, lr: float, strength_map=None, want_loss=True):
        import torch

        loss = ctypes.c_float()
        self.ctx.set_stream(torch.cuda.current_stream(rgb.device).cuda_stream)
        self.ctx.check(lib().dsgpu_cnn_train_step(self.ctx.handle, self.handle, self._ptr(rgb),
                                                  self._ptr(strength_map), float(strength), self._ptr(target),
                                                  rgb.shape[0], float(lr),
                                                  ctypes.byref(loss) if want_loss else None),
                       "dsgpu_cnn_train_step")
        return float(loss.value) if want_loss else None

    def infer(self, img, h_param: float):
        """out = img + network(img, STRENGTH_SCALE * h) on an Image3 (numpy or
        CUDA tensor data)."""
        from . import Image3, _Call

        c = _Call(img.data, self.ctx)
        _, pi = c.inp(img.data, np.float32)
        out, po = c.out((img.h, img.w, 3))
        c.ctx.check(lib().dsgpu_cnn_infer(c.ctx.handle, self.handle, pi, img.w, img.h,
                                          float(h_param * STRENGTH_SCALE), po, c.flags), "dsgpu_cnn_infer")
        return Image3(img.w, img.h, out)

    def denoise(self, img, h_param: float, search: int = 10, patch: int = 3, tau: float = 3.0):
        """Learned NLM with per-tile fallback: (Image3, number of NLM tiles recomputed)."""
        from . import Image3, _Call

        c = _Call(img.data, self.ctx)
        _, pi = c.inp(img.data, np.float32)
        out, po = c.out((img.h, img.w, 3))
        nf = ctypes.c_int()
        c.ctx.check(lib().dsgpu_cnn_denoise(c.ctx.handle, self.handle, pi, img.w, img.h, float(h_param), int(search),
                                            int(patch), float(tau), po, ctypes.byref(nf), c.flags),
                    "dsgpu_cnn_denoise")
        return Image3(img.w, img.h, out), int(nf.value)

    def develop_u16(self, raw, pattern, black: float, white, mul, h_param: float, search: int = 10, patch: int = 3,
                    tau: float = 3.0, with_clip: bool = False):
        """u16 raw -> normalise -> RCD -> the network, with NLM recomputing the
        tiles that fail the residual check (dsgpu_develop_u16_cnn). A numpy raw
        runs as the host-buffer band pipeline, a CUDA tensor on the device.
        Returns the Image3 (and the clip Plane when ``with_clip``)."""
        from . import Image3, Plane, _Call, _f3, _vp

        c = _Call(raw, self.ctx)
        h, w = raw.shape
        _, p = c.inp(raw, np.uint16)
        rgb, pr = c.out((h, w, 3))
        clip, pc = c.out((h, w)) if with_clip else (None, ctypes.c_void_p(0))
        pat, wh, m = pattern.codes(), _f3(white), _f3(mul)
        c.ctx.check(lib().dsgpu_develop_u16_cnn(c.ctx.handle, self.handle, p, w, h, w, _vp(pat), float(black), _vp(wh),
                                                _vp(m), float(h_param), int(search), int(patch), float(tau), pr, pc,
                                                c.flags), "dsgpu_develop_u16_cnn")
        img = Image3(w, h, rgb)
        return (img, Plane(w, h, clip)) if with_clip else img

    def set_judge(self, fraction: float, limit: float = 0.5, seed: int = 0) -> None:
        """Judge mode (dsgpu_cnn_set_judge): plain NLM recomputes a seeded
        `fraction` of the NLM tiles and a sampled tile keeps NLM's result when
        the network's RMS error against it exceeds `limit` x sigma. 0: off."""
        self.ctx.check(lib().dsgpu_cnn_set_judge(self.ctx.handle, self.handle, float(fraction), float(limit),
                                                 int(seed) & 0xFFFFFFFF), "dsgpu_cnn_set_judge")

    def judge_stats(self) -> dict:
        """The judge's record of the last call: sampled tiles, tiles that kept
        NLM, max and RMS error of the network against NLM (over sigma)."""
        j, f = ctypes.c_int(), ctypes.c_int()
        mx, rms = ctypes.c_float(), ctypes.c_float()
        self.ctx.check(lib().dsgpu_cnn_judge_stats(self.ctx.handle, self.handle, ctypes.byref(j), ctypes.byref(f),
                                                   ctypes.byref(mx), ctypes.byref(rms)), "dsgpu_cnn_judge_stats")
        return {"judged": j.value, "failed": f.value, "max_rms_over_sigma": mx.value, "rms_over_sigma": rms.value}

    def set_clip(self, max_norm: float) -> None:
        """Clip the global gradient norm to max_norm in train_step (0: off)."""
        self.ctx.check(lib().dsgpu_cnn_set_clip(self.ctx.handle, self.handle, float(max_norm)), "dsgpu_cnn_set_clip")

    def set_loss(self, relative: bool) -> None:
        """Training loss: plain MSE, or (relative) squared errors weighted by
        1 / strength^2, the error relative to the frame's noise level."""
        self.ctx.check(lib().dsgpu_cnn_set_loss(self.ctx.handle, self.handle, int(bool(relative))),
                       "dsgpu_cnn_set_loss")

    def set_engine(self, tensor_core_gen5: bool) -> None:
        """Inference and training on tcgen05 (default; training runs its
        forward pass, data, weight and bias gradients there) or on the
        mma.sync kernels."""
        self.ctx.check(lib().dsgpu_cnn_set_engine(self.ctx.handle, self.handle, int(bool(tensor_core_gen5))),
                       "dsgpu_cnn_set_engine")

    def close(self):
        if getattr(self, "handle", None) is not None:
            lib().dsgpu_cnn_destroy(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
