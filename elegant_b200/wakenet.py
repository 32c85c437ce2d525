"""Python binding of the wake network (include/elegant_b200.h, b2e_wakenet_*).

The network runs entirely in the engine library's tcgen05 kernels; this class
only owns the handle and passes device pointers (torch tensors are used as
device buffers and for the training driver's plumbing).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat

DILATIONS = (1, 3, 9, 27, 81, 243)
LAYERS, CH, TAPS = 6, 64, 5
IN_CH = 4  # density, derivative, slippage code, density shifted by the slippage
WSIZE = TAPS * CH * CH


def init_params(seed: int, out_scale: float = 0.1) -> np.ndarray:
    """He-style initialisation of the flat parameter array: weights
    N(0, 2/fan_in) with fan_in counted over live input channels (3 for the
    first layer: IN_CH); only output channel 0 of the last layer live, scaled by
    out_scale; biases zero."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = np.zeros((LAYERS, TAPS, CH, CH))
    for l in range(LAYERS):
        std = np.sqrt(2.0 / (TAPS * (IN_CH if l == 0 else CH)))
        if l == 0:
            w[l, :, :, :IN_CH] = rng.normal(0, std, (TAPS, CH, IN_CH))
        elif l == LAYERS - 1:
            w[l, :, 0, :] = rng.normal(0, std * out_scale, (TAPS, CH))
        else:
            w[l] = rng.normal(0, std, (TAPS, CH, CH))
    return np.concatenate([w.ravel(), np.zeros(LAYERS * CH)]).astype(np.float32)


def _bind(lib):
    if getattr(lib, "_wakenet_bound", False):
        return lib
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    sig = {
        "b2e_wakenet_create": (ctypes.c_int, [ctypes.POINTER(vp), i32, i32, ctypes.POINTER(i32), i32]),
        "b2e_wakenet_destroy": (ctypes.c_int, [vp]),
        "b2e_wakenet_last_error": (ctypes.c_char_p, [vp]),
        "b2e_wakenet_param_count": (i64, []),
        "b2e_wakenet_set_params": (ctypes.c_int, [vp, vp]),
        "b2e_wakenet_get_params": (ctypes.c_int, [vp, vp, vp]),
        "b2e_wakenet_forward": (ctypes.c_int, [vp, vp, i32, vp, vp]),
        "b2e_wakenet_gradients": (ctypes.c_int, [vp, vp, vp, i32, ctypes.POINTER(ctypes.c_double), vp]),
        "b2e_wakenet_train_step": (ctypes.c_int, [vp, vp, vp, i32, ctypes.c_float, ctypes.POINTER(ctypes.c_double),
                                                  vp]),
        "b2e_csr_wake_batch": (ctypes.c_int, [vp, vp, i32, i32, i32, i32, i32, i32, i32, i32, vp, vp, vp, vp]),
        "b2e_wake_features": (ctypes.c_int, [vp, vp, vp, i32, i32, ctypes.c_double, ctypes.c_double, i32, vp, vp,
                                             vp]),
        "b2e_wake_t1_from_output": (ctypes.c_int, [vp, vp, vp, i32, i32, ctypes.c_double, vp, vp]),
        "b2e_umma_selftest": (ctypes.c_int, [ctypes.c_int, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    lib._wakenet_bound = True
    return lib


def library():
    return _bind(nat.load_library())


class WakeNet:
    """Handle to a device-resident wake network of fixed bin count and maximum batch."""

    def __init__(self, bins: int = 1024, max_batch: int = 256, dilations=DILATIONS, device: int = 0):
        self.lib = library()
        self.bins, self.max_batch, self.dilations = bins, max_batch, tuple(dilations)
        self._h = ctypes.c_void_p()
        d = (ctypes.c_int32 * LAYERS)(*self.dilations)
        rc = self.lib.b2e_wakenet_create(ctypes.byref(self._h), bins, max_batch, d, device)
        if rc != nat.B2E_OK:
            raise nat.EngineError(rc, "b2e_wakenet_create failed")
        self.n_params = int(self.lib.b2e_wakenet_param_count())

    def _check(self, rc):
        if rc != nat.B2E_OK:
            raise nat.EngineError(rc, self.lib.b2e_wakenet_last_error(self._h).decode())

    def close(self):
        if self._h:
            self.lib.b2e_wakenet_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- parameters ----------------------------------------------------------
    def set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == self.n_params
        self._check(self.lib.b2e_wakenet_set_params(self._h, p.ctypes.data))

    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, dtype=np.float32)
        self._check(self.lib.b2e_wakenet_get_params(self._h, p.ctypes.data, None))
        return p

    def grads(self) -> np.ndarray:
        g = np.empty(self.n_params, dtype=np.float32)
        self._check(self.lib.b2e_wakenet_get_params(self._h, None, g.ctypes.data))
        return g

    # -- compute (torch CUDA tensors as device buffers) ------------------------
    @staticmethod
    def _stream(stream):
        import torch
        return (stream or torch.cuda.current_stream()).cuda_stream

    def forward(self, inputs, out=None, stream=None):
        """inputs: float32 CUDA tensor [n][IN_CH][bins] -> [n][bins]."""
        import torch
        n = inputs.shape[0]
        assert inputs.is_contiguous() and inputs.dtype == torch.float32 and inputs.shape[1:] == (IN_CH, self.bins)
        if out is None:
            out = torch.empty((n, self.bins), dtype=torch.float32, device=inputs.device)
        for s in range(0, n, self.max_batch):
            e = min(n, s + self.max_batch)
            self._check(self.lib.b2e_wakenet_forward(self._h, inputs[s:e].data_ptr(), e - s, out[s:e].data_ptr(),
                                                     self._stream(stream)))
        return out

    def gradients(self, inputs, targets, stream=None) -> float:
        loss = ctypes.c_double()
        self._check(self.lib.b2e_wakenet_gradients(self._h, inputs.data_ptr(), targets.data_ptr(), inputs.shape[0],
                                                   ctypes.byref(loss), self._stream(stream)))
        return loss.value

    def train_step(self, inputs, targets, lr: float, want_loss: bool = False, stream=None):
        loss = ctypes.c_double()
        self._check(self.lib.b2e_wakenet_train_step(self._h, inputs.data_ptr(), targets.data_ptr(), inputs.shape[0],
                                                    lr, ctypes.byref(loss) if want_loss else None,
                                                    self._stream(stream)))
        return loss.value if want_loss else None
