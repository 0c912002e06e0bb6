"""The learned warm start's network over libvrad_cuda (vrad_mlp_*).

A 32 -> 128 -> 128 -> 3 network (ReLU, BF16 weights and activations, FP32
accumulation) trained and run on the device by the library's own tensor-core
kernels.  Inputs are (n, 32) torch.bfloat16 CUDA tensors, targets and
outputs (n, 3) float32 CUDA tensors; torch is only the allocator.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import tracer as T

INPUTS, HIDDEN, OUTPUTS = 32, 128, 3
PARAMS = INPUTS * HIDDEN + HIDDEN + HIDDEN * HIDDEN + HIDDEN + HIDDEN * OUTPUTS + OUTPUTS
# Offsets of each block in the flat parameter vector.
OFFSETS = {"w1": 0, "b1": INPUTS * HIDDEN}
OFFSETS["w2"] = OFFSETS["b1"] + HIDDEN
OFFSETS["b2"] = OFFSETS["w2"] + HIDDEN * HIDDEN
OFFSETS["w3"] = OFFSETS["b2"] + HIDDEN
OFFSETS["b3"] = OFFSETS["w3"] + HIDDEN * OUTPUTS
SHAPES = {"w1": (INPUTS, HIDDEN), "b1": (HIDDEN,), "w2": (HIDDEN, HIDDEN), "b2": (HIDDEN,),
          "w3": (HIDDEN, OUTPUTS), "b3": (OUTPUTS,)}


def _lib():
    lib = T.load_library()
    if not getattr(lib, "_mlp_bound", False):
        P, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
        lib.vrad_mlp_create.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(P)]
        lib.vrad_mlp_destroy.argtypes = [P]
        lib.vrad_mlp_params.argtypes = [P, P, P]
        lib.vrad_mlp_forward_device.argtypes = [P, P, i64, P, P]
        lib.vrad_mlp_gradient_device.argtypes = [P, P, P, i64, P, P, P]
        lib.vrad_mlp_train_step_device.argtypes = [P, P, P, i64, f32, P]
        lib.vrad_mlp_loss.argtypes = [P, P]
        for n in ("vrad_mlp_create", "vrad_mlp_destroy", "vrad_mlp_params", "vrad_mlp_forward_device",
                  "vrad_mlp_gradient_device", "vrad_mlp_train_step_device", "vrad_mlp_loss"):
            getattr(lib, n).restype = i32
        lib._mlp_bound = True
    return lib


def split(flat: np.ndarray) -> dict:
    """The flat parameter vector as named arrays."""
    return {k: flat[OFFSETS[k]:OFFSETS[k] + int(np.prod(s))].reshape(s) for k, s in SHAPES.items()}


class Network:
    """One network on the device of `tracer` (a CudaRayTracer or anything
    with its context)."""

    def __init__(self, tracer, seed: int = 1):
        self._tracer = tracer
        h = ctypes.c_void_p()
        T._check(_lib().vrad_mlp_create(tracer._ctx, seed, ctypes.byref(h)), tracer._ctx)
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            _lib().vrad_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.zeros(PARAMS, np.float32)
        T._check(_lib().vrad_mlp_params(self._h, out.ctypes.data, None), None)
        return out

    def set_params(self, flat: np.ndarray) -> None:
        flat = np.ascontiguousarray(flat, np.float32)
        assert flat.size == PARAMS
        T._check(_lib().vrad_mlp_params(self._h, None, flat.ctypes.data), None)

    @staticmethod
    def _stream(stream):
        import torch
        return stream if stream is not None else torch.cuda.current_stream().cuda_stream

    def forward(self, x, out=None, stream=None):
        import torch
        assert x.dtype == torch.bfloat16 and x.is_contiguous() and x.shape[1] == INPUTS
        y = out if out is not None else torch.empty((x.shape[0], OUTPUTS), dtype=torch.float32, device=x.device)
        T._check(_lib().vrad_mlp_forward_device(self._h, x.data_ptr(), x.shape[0], y.data_ptr(),
                                                ctypes.c_void_p(self._stream(stream))), None)
        return y

    def gradient(self, x, target, stream=None):
        """(flat gradient, loss) of the mean squared error."""
        g = np.zeros(PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        T._check(_lib().vrad_mlp_gradient_device(self._h, x.data_ptr(), target.data_ptr(), x.shape[0], g.ctypes.data,
                                                 loss.ctypes.data, ctypes.c_void_p(self._stream(stream))), None)
        return g, float(loss[0])

    def train_step(self, x, target, lr: float, stream=None) -> None:
        T._check(_lib().vrad_mlp_train_step_device(self._h, x.data_ptr(), target.data_ptr(), x.shape[0], lr,
                                                   ctypes.c_void_p(self._stream(stream))), None)

    def loss(self) -> float:
        v = np.zeros(1, np.float32)
        T._check(_lib().vrad_mlp_loss(self._h, v.ctypes.data), None)
        return float(v[0])
