"""The learned warm start's network over libvrad_cuda (vrad_mlp_*).

A 32 -> 128 -> 128 -> 3 network (ReLU, BF16 weights and activations, FP32
accumulation) trained and run on the device by the library's own tensor-core
kernels: the forward on tcgen05 with TMEM accumulators, the training on
mma.sync.  Inputs are (n, 32) torch.bfloat16 CUDA tensors, targets and
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
        lib.vrad_mlp_status.argtypes = [P]
        for n in ("vrad_mlp_create", "vrad_mlp_destroy", "vrad_mlp_params", "vrad_mlp_forward_device",
                  "vrad_mlp_gradient_device", "vrad_mlp_train_step_device", "vrad_mlp_loss", "vrad_mlp_status"):
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

    def status(self) -> None:
        """Raises when a forward since the last call gave up on a bounded
        tensor-core wait (vrad_mlp_status)."""
        T._check(_lib().vrad_mlp_status(self._h), None)

    def loss(self) -> float:
        v = np.zeros(1, np.float32)
        T._check(_lib().vrad_mlp_loss(self._h, v.ctypes.data), None)
        return float(v[0])


def training_config(k: int, seed0: int = 100):
    """The k-th training map: an 8x8-style room grid (pillars, point and
    spot lights, sun and sky) of 2 to 8 rooms a side, one light per room."""
    import dataclasses
    from . import roomgrid as rg
    side = 2 + k % 7
    return dataclasses.replace(rg.config_8x8(seed0 + k), side=side, lights=side * side)


def collect(configs, threshold: float = 0.1, bounces: int = 100):
    """Plain light passes over the maps: the receivers' features and the
    log1p of their converged bounced light, concatenated (CUDA tensors)."""
    import torch
    from . import lighting as L, roomgrid as rg
    xs, ts = [], []
    for cfg in configs:
        w = rg.generate(cfg)
        with L.LightingStage(w) as st:
            off, lst = L.pvs_lists(w)
            st.upload_bounce(L.face_reflectivity(w), off, lst, bounces=bounces, threshold=threshold)
            st.light_pass()
            x, t = st.bounce_features()
            xs.append(x.clone())
            ts.append(t.clone())
    return torch.cat(xs), torch.cat(ts)


def train(net: Network, x, t, steps: int = 3000, batch: int = 32768, lr: float = 2e-3, seed: int = 0,
          log=None) -> float:
    """Adam on random minibatches (the rate drops 4x for the last third);
    returns the last step's loss."""
    import torch
    g = torch.Generator(device=x.device)
    g.manual_seed(seed)
    n = len(x)
    for step in range(steps):
        idx = torch.randint(0, n, (min(batch, n),), device=x.device, generator=g)
        net.train_step(x[idx].contiguous(), t[idx].contiguous(), lr if step < 2 * steps // 3 else lr / 4)
        if log is not None and step % 500 == 0:
            log(step, net.loss())
    return net.loss()


def within_one_lsb(a: np.ndarray, b: np.ndarray) -> float:
    """The fraction of RGBE words of two LIGHTING lumps whose three channels
    differ by at most one unit of the larger word's last place."""
    va = a.view(np.uint8).reshape(-1, 4).astype(np.int64)
    vb = b.view(np.uint8).reshape(-1, 4).astype(np.int64)
    ea = va[:, 3].astype(np.int8).astype(np.int64)
    eb = vb[:, 3].astype(np.int8).astype(np.int64)
    fa = va[:, :3] * np.exp2(ea)[:, None]
    fb = vb[:, :3] * np.exp2(eb)[:, None]
    lsb = np.exp2(np.maximum(ea, eb))[:, None]
    return float((np.abs(fa - fb) <= lsb).all(1).mean())


def heldout_config(k: int, seed0: int = 900):
    """The k-th held-out map: the training maps' kind, seeds no training map
    uses, sides 3, 5 and 7 rooms."""
    import dataclasses
    from . import roomgrid as rg
    side = (3, 5, 7)[k % 3]
    return dataclasses.replace(rg.config_8x8(seed0 + k), side=side, lights=side * side)


def evaluate(net: Network, configs, threshold: float = 0.1, bounces: int = 100) -> list:
    """Per map: the plain and the warm bounce counts, the guess's relative
    error eps (mean |G - T| over mean T, G the network's converged-light
    guess, T the plain bounce's converged light, per receiver and channel),
    the plain iteration's contraction rho (the geometric mean of the ratio
    between successive bounces' added light: (A_n / A_1)^(1 / (n - 1)),
    A_k the light bounce k adds), the savings the bound log(1/eps) /
    log(1/rho) predicts, and whether the warm lump is within 1 LSB of the
    plain one."""
    import math
    from . import lighting as L, roomgrid as rg
    out = []
    for cfg in configs:
        w = rg.generate(cfg)
        off, lst = L.pvs_lists(w)
        refl = L.face_reflectivity(w)
        with L.LightingStage(w) as st:
            st.upload_bounce(refl, off, lst, bounces=1, threshold=0.0)
            st.light_pass()
            a1 = sum(st.bounce_stats().added)
            st.upload_bounce(refl, off, lst, bounces=bounces, threshold=threshold)
            plain_lump, _, _ = st.light_pass()
            bp = st.bounce_stats()
            an = sum(bp.added)
            x, t = st.bounce_features()
            y = net.forward(x)
            g, tt = y.float().expm1().clamp_min(0), t.float().expm1()
            eps = float((g - tt).abs().mean() / tt.abs().mean().clamp_min(1e-30))
            st.set_bounce_model(net)
            warm_lump, _, _ = st.light_pass()
            bw = st.bounce_stats()
            st.set_bounce_model(None)
        n = int(bp.bounces)
        rho = (an / a1) ** (1.0 / (n - 1)) if n > 1 and a1 > 0 and an > 0 else float("nan")
        pred = math.log(1.0 / eps) / math.log(1.0 / rho) if 0 < eps < 1 and 0 < rho < 1 else float("nan")
        out.append({"side": cfg.side, "seed": cfg.seed, "receivers": int(len(x)), "plain_bounces": n,
                    "warm_bounces": int(bw.bounces), "eps": eps, "rho": rho, "bound_savings": pred,
                    "within_1_lsb": within_one_lsb(warm_lump, plain_lump)})
    return out
