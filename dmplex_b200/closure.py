"""The learned flux closure's network on the tensor cores (libtrisk_b200.so, closure.cu).

An edge-local MLP 24 -> 64 -> 64 -> 2 with GELU: BF16 weights and activations, FP32
accumulation, FP32 master weights updated by Adam. There is no closure in the reference;
the plain FP64 method stays the measure of its error and its fallback (workloads, bench).
Device arrays are CUDA torch tensors: features (n, 24) bfloat16, targets and outputs
(n, 2) float32.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib

NIN, NH, NOUT = 24, 64, 2
SHAPES = (("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NOUT, NH)), ("b3", (NOUT,)))


def he_init(seed: int = 0) -> np.ndarray:
    """Seeded initial parameters: normal weights scaled by sqrt(2 / fan_in), zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in SHAPES:
        if name.startswith("b"):
            parts.append(np.zeros(shape))
        else:
            gain = 1.0 if name == "W3" else 2.0
            parts.append(rng.standard_normal(shape) * np.sqrt(gain / shape[1]))
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)


def _check_tensor(x, dtype: str, cols: int):
    if not hasattr(x, "data_ptr") or not x.is_cuda or str(x.dtype) != dtype or not x.is_contiguous():
        raise TypeError(f"expected a contiguous CUDA {dtype} tensor")
    if x.dim() != 2 or x.shape[1] != cols:
        raise ValueError(f"expected shape (n, {cols})")


class ClosureMLP:
    def __init__(self, params: np.ndarray | None = None, device: int = 0, seed: int = 0):
        self.nparam = int(lib.trisk_closure_param_count())
        p = he_init(seed) if params is None else np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.nparam:
            raise ValueError(f"expected {self.nparam} parameters")
        h = C.c_void_p()
        check(lib.trisk_closure_create(int(device), p.ctypes.data, C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            lib.trisk_closure_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def params(self) -> np.ndarray:
        out = np.zeros(self.nparam, dtype=np.float32)
        check(lib.trisk_closure_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib.trisk_closure_set_params(self._h, p.ctypes.data))

    def forward(self, X, Y=None):
        import torch
        _check_tensor(X, "torch.bfloat16", NIN)
        if Y is None:
            Y = torch.empty((X.shape[0], NOUT), dtype=torch.float32, device=X.device)
        _check_tensor(Y, "torch.float32", NOUT)
        check(lib.trisk_closure_forward(self._h, X.data_ptr(), X.shape[0], Y.data_ptr()))
        return Y

    def gradients(self, X, T):
        """(gradients packed like the parameters, mean loss)."""
        _check_tensor(X, "torch.bfloat16", NIN)
        _check_tensor(T, "torch.float32", NOUT)
        g = np.zeros(self.nparam, dtype=np.float32)
        loss = C.c_float()
        check(lib.trisk_closure_gradients(self._h, X.data_ptr(), T.data_ptr(), X.shape[0], g.ctypes.data,
                                          C.byref(loss)))
        return g, loss.value

    def info(self) -> dict:
        """The inference kernel's launch shape: CTAs per SM of its persistent grid, and SMs."""
        per_sm, sms = C.c_int32(), C.c_int32()
        check(lib.trisk_closure_info(self._h, C.byref(per_sm), C.byref(sms)))
        return {"forward_ctas_per_sm": per_sm.value, "sms": sms.value}

    def expire_wait_once(self, tile: int) -> None:
        """Test of the bounded tensor-core wait: the next forward call leaves tile `tile`'s first
        tensor-core operation un-issued, so it returns TRISK_ERR_TIMEOUT (TriskError status 5)
        after half a second; the closure stays usable."""
        check(lib.trisk_closure_expire_wait_once(self._h, int(tile)))

    def train_step(self, X, T, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> float:
        """Gradients on the batch, then one Adam step; returns the batch loss."""
        _check_tensor(X, "torch.bfloat16", NIN)
        _check_tensor(T, "torch.float32", NOUT)
        loss = C.c_float()
        check(lib.trisk_closure_gradients(self._h, X.data_ptr(), T.data_ptr(), X.shape[0], None, C.byref(loss)))
        check(lib.trisk_closure_adam(self._h, float(lr), float(beta1), float(beta2), float(eps)))
        return loss.value
