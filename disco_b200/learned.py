"""Learned far-image surrogate (north-star form 4): the network, its training
and its use in the displacement sum.

MLP wraps the C-ABI network (14 -> 128 -> 128 -> 128 -> 3, SiLU, BF16 tensor
cores, FP32 accumulation and master weights, Adam), trained and evaluated by
this library's own tcgen05 kernels.  Tensors are torch CUDA tensors (device
memory and streams only)."""
import ctypes

import numpy as np

from . import _capi as C


class MLP:
    IN, OUT, IN_REAL, OUT_REAL = 16, 16, 14, 3

    def __init__(self, seed=0):
        self._lib = C.cuda_lib()
        h = ctypes.c_void_p()
        C.check(self._lib.disco_b200_mlp_create(ctypes.c_uint64(seed), ctypes.byref(h)), self._lib)
        self._h = h
        self.nparams = self._lib.disco_b200_mlp_param_count()

    def params(self):
        out = np.empty(self.nparams, dtype=np.float32)
        C.check(self._lib.disco_b200_mlp_get_params(self._h, out.ctypes.data), self._lib)
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams
        C.check(self._lib.disco_b200_mlp_set_params(self._h, p.ctypes.data), self._lib)

    def grads(self):
        out = np.empty(self.nparams, dtype=np.float32)
        C.check(self._lib.disco_b200_mlp_get_grads(self._h, out.ctypes.data), self._lib)
        return out

    @staticmethod
    def _stream(stream):
        import torch
        return (stream or torch.cuda.current_stream()).cuda_stream

    def forward(self, X, stream=None):
        """X: (n, 16) float32 CUDA tensor -> (n, 16) float32 (first 3 used)."""
        import torch
        assert X.dtype == torch.float32 and X.is_cuda and X.is_contiguous() and X.shape[1] == self.IN
        Y = torch.empty((X.shape[0], self.OUT), dtype=torch.float32, device=X.device)
        C.check(self._lib.disco_b200_mlp_forward(self._h, X.data_ptr(), X.shape[0], Y.data_ptr(),
                                                 ctypes.c_void_p(self._stream(stream))), self._lib)
        return Y

    def grad(self, X, T, stream=None):
        """Accumulates the MSE gradient over the rows of X (n, 16) against
        T (n, 3); returns the loss."""
        loss = ctypes.c_float()
        C.check(self._lib.disco_b200_mlp_grad(self._h, X.data_ptr(), T.data_ptr(), X.shape[0],
                                              ctypes.byref(loss), ctypes.c_void_p(self._stream(stream))),
                self._lib)
        return loss.value

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0, stream=None):
        C.check(self._lib.disco_b200_mlp_adam(self._h, lr, beta1, beta2, eps, weight_decay,
                                              ctypes.c_void_p(self._stream(stream))), self._lib)

    def status(self):
        C.check(self._lib.disco_b200_mlp_status(self._h), self._lib)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.disco_b200_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
