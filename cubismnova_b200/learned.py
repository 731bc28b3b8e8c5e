"""Learned 3-D convolutional smoother for the multigrid solver
(csrc/learned.cu): training on device-resident patches with the library's own
forward/backward kernels and Adam, and use inside the V-cycle."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .grid import Cartesian, _stream_handle

_P, _I, _D = C.c_void_p, C.c_int, C.c_double
_lib.register({
    "cn_nn_create": (_I, [C.c_uint64, _D, _D, C.POINTER(_P)]),
    "cn_nn_destroy": (_I, [_P]),
    "cn_nn_get_weights": (_I, [_P, _P]),
    "cn_nn_set_weights": (_I, [_P, _P]),
    "cn_nn_weight_count": (_I, []),
    "cn_nn_loss_grad": (_I, [_P, _P, _P, _P, _I, _I, _D, C.POINTER(C.c_double), _P, _P]),
    "cn_nn_adam_step": (_I, [_P, _D, _P]),
    "cn_nn_train": (_I, [_P, _P, _P, _P, _I, _I, _D, _I, _I, _D, C.c_uint64, C.POINTER(C.c_double), _P]),
    "cn_mg_collect_patches": (_I, [_P, _P, _I, _I, C.c_uint64, _P, _P, _P, _I, C.POINTER(_I), _P]),
    "cn_mg_set_smoother": (_I, [_P, _P, C.c_uint]),
    "cn_mg_set_smoother_phases": (_I, [_P, _P, C.c_uint, C.c_uint, _I, _I]),
    "cn_nn_set_inference": (_I, [_P, _I]),
    "cn_nn_set_training": (_I, [_P, _I]),
    "cn_conv3_bf16": (_I, [_P, _P, C.POINTER(C.c_int), C.POINTER(C.c_int), _P, _I, _P]),
})

CI, CH = 2, 16
SHAPES = ((27, CI, CH), (27, CH, CH), (27, CH, 1))


class LearnedSmoother:
    """p <- p + omega * x0 + N(x0, x0 ln k) with x0 = -r/D the Jacobi correction
    (r = f - L p, D = -diag L), N a 3-layer 3^3 conv net."""

    def __init__(self, seed: int = 0, omega: float = 0.8, init_scale: float = 1e-3):
        h = C.c_void_p()
        _lib.check(_lib.lib().cn_nn_create(seed, omega, init_scale, C.byref(h)))
        self._h, self.omega = h, omega
        self.nweights = _lib.lib().cn_nn_weight_count()

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().cn_nn_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def weights(self):
        w = np.empty(self.nweights, dtype=np.float32)
        _lib.check(_lib.lib().cn_nn_get_weights(self._h, w.ctypes.data_as(C.c_void_p)))
        out, o = [], 0
        for s in SHAPES:
            n = int(np.prod(s))
            out.append(w[o:o + n].reshape(s))
            o += n
        return out

    def set_inference(self, mode: str):
        """Grid inference on "tensor" cores (BF16 activations and weights,
        tcgen05, FP32 accumulation; the default) or "fp32" CUDA cores."""
        _lib.check(_lib.lib().cn_nn_set_inference(self._h, {"fp32": 0, "tensor": 1}[mode]))

    def set_training(self, mode: str):
        """Training arithmetic: "tensor" (the default: the hidden layer's
        forward, data gradient and weight gradient on the tensor cores with
        BF16 operands and activations, FP32 accumulation) or "fp32" (CUDA
        cores throughout)."""
        _lib.check(_lib.lib().cn_nn_set_training(self._h, {"fp32": 0, "tensor": 1}[mode]))

    def set_weights(self, W1, W2, W3):
        w = np.concatenate([np.asarray(a, dtype=np.float32).ravel() for a in (W1, W2, W3)])
        assert w.size == self.nweights
        _lib.check(_lib.lib().cn_nn_set_weights(self._h, w.ctypes.data_as(C.c_void_p)))

    def loss_grad(self, x, k, r, P: int, ih2: float, stream=None):
        """x (B,2,(P+8)^3), k (B,(P+2)^3), r (B,P^3): contiguous float32 CUDA tensors."""
        B = x.shape[0]
        loss = C.c_double()
        g = np.empty(self.nweights, dtype=np.float32)
        _lib.check(_lib.lib().cn_nn_loss_grad(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(k.data_ptr()),
                                              C.c_void_p(r.data_ptr()), B, P, ih2, C.byref(loss),
                                              g.ctypes.data_as(C.c_void_p), _stream_handle(stream)))
        out, o = [], 0
        for s in SHAPES:
            n = int(np.prod(s))
            out.append(g[o:o + n].reshape(s))
            o += n
        return loss.value, out

    def train(self, x, k, r, P: int, ih2: float, epochs: int = 10, batch: int = 16, lr: float = 1e-3,
              seed: int = 0, stream=None) -> float:
        last = C.c_double()
        _lib.check(_lib.lib().cn_nn_train(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(k.data_ptr()),
                                          C.c_void_p(r.data_ptr()), x.shape[0], P, ih2, epochs, batch, lr, seed,
                                          C.byref(last), _stream_handle(stream)))
        return last.value


def collect_patches(mg, f: Cartesian, cycles: int, per_snapshot: int, max_patches: int, seed: int = 0,
                    stream=None):
    """Training samples from plain V-cycles (see cn_mg_collect_patches)."""
    import torch
    n = f.getBlockCells()
    P = n[0]
    x = torch.empty((max_patches, 2, (P + 8) ** 3), dtype=torch.float32, device="cuda")
    k = torch.empty((max_patches, (P + 2) ** 3), dtype=torch.float32, device="cuda")
    r = torch.empty((max_patches, P ** 3), dtype=torch.float32, device="cuda")
    cnt = C.c_int()
    _lib.check(_lib.lib().cn_mg_collect_patches(mg.handle, f.handle, cycles, per_snapshot, seed,
                                                C.c_void_p(x.data_ptr()), C.c_void_p(k.data_ptr()),
                                                C.c_void_p(r.data_ptr()), max_patches, C.byref(cnt),
                                                _stream_handle(stream)))
    m = cnt.value
    return x[:m].contiguous(), k[:m].contiguous(), r[:m].contiguous(), P


def conv3_bf16(x, nblocks, block_cells, weights, relu: bool = False, stream=None):
    """One 16 -> 16 channel 3x3x3 convolution on the tensor cores
    (cn_conv3_bf16): x is a CUDA tensor [nblocks*cells, 16] of bfloat16 in
    grid order, weights a CUDA float32 tensor [27, 16, 16]; returns a new
    bfloat16 tensor of x's shape."""
    import torch
    out = torch.empty_like(x)
    _lib.check(_lib.lib().cn_conv3_bf16(C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), _lib.ivec3(nblocks),
                                        _lib.ivec3(block_cells), C.c_void_p(weights.data_ptr()), 1 if relu else 0,
                                        _stream_handle(stream)))
    return out


def use_in(mg, smoother, level_mask: int = 0xFFFF, post_mask=None, pre_apps: int = -1, post_apps: int = -1):
    """Replace Jacobi by the learned smoother on the levels in level_mask
    (pre- and post-smoothing; with post_mask, level_mask selects the
    pre-smoothing levels and post_mask the post-smoothing ones), with
    pre_apps / post_apps applications (-1: the solver's nu1 / nu2); smoother
    None: back to Jacobi everywhere."""
    h = smoother.handle if smoother else None
    if post_mask is None and pre_apps < 0 and post_apps < 0:
        _lib.check(_lib.lib().cn_mg_set_smoother(mg.handle, h, level_mask))
    else:
        pm = level_mask if post_mask is None else post_mask
        _lib.check(_lib.lib().cn_mg_set_smoother_phases(mg.handle, h, level_mask, pm, pre_apps, post_apps))
