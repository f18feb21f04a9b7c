"""The learned collision-probability predictor over the C ABI (gprm_mlp_*).

Network: sin/cos of the joint angles (12 inputs for 6 joints, padded to 16)
-> 256 -> 256 -> 256 -> 256 -> 1, GELU (tanh form) hidden activations, sigmoid output,
binary cross-entropy, Adam.  Forward, backward and Adam run in the
library's CUDA kernels (BF16 tensor-core GEMMs, FP32 accumulation).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi

HID = 256
IN_PAD = 16
LAYERS = 4


def param_shapes():
    """[(name, shape)] in the order of the flat parameter vector."""
    out = []
    for l in range(LAYERS + 1):
        nin = IN_PAD if l == 0 else HID
        nout = 1 if l == LAYERS else HID
        out.append((f"W{l + 1}", (nout, nin)))
        out.append((f"b{l + 1}", (nout,)))
    return out


def unpack(vec: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shp in param_shapes():
        n = int(np.prod(shp))
        out[name] = vec[o:o + n].reshape(shp)
        o += n
    return out


class CollisionMLP:
    def __init__(self, ndof: int = 6, seed: int = 0):
        self.lib = _abi.load_library()
        h = C.c_void_p()
        st = self.lib.gprm_mlp_create(ndof, seed, C.byref(h))
        if st != 0:
            raise RuntimeError(f"gprm_mlp_create failed ({st})")
        self.h = h
        self.ndof = ndof

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.gprm_mlp_destroy(self.h)
            self.h = None

    def _check(self, st):
        if st != 0:
            raise RuntimeError(f"gprm_mlp status {st}: {self.lib.gprm_mlp_last_error(self.h).decode()}")

    @property
    def num_params(self) -> int:
        return int(self.lib.gprm_mlp_num_params(self.h))

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.num_params, np.float32)
        self._check(self.lib.gprm_mlp_get_params(self.h, _abi.fptr(out)))
        return out

    def set_params(self, vec: np.ndarray) -> None:
        v = np.ascontiguousarray(vec, np.float32)
        assert v.size == self.num_params
        self._check(self.lib.gprm_mlp_set_params(self.h, _abi.fptr(v)))

    def predict(self, q_soa, out=None, stream=None):
        """q_soa: (ndof, n) float32 CUDA tensor -> (n,) P(collision)."""
        import torch
        n = int(q_soa.shape[1])
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device=q_soa.device)
        st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(self.lib.gprm_mlp_predict(self.h, C.c_void_p(q_soa.data_ptr()), n, n,
                                              C.c_void_p(out.data_ptr()), C.c_void_p(st)))
        return out

    def set_inference(self, path: str) -> None:
        """'tcgen05' (default): one fused tensor-core kernel for all layers
        (TMEM accumulators, activations in shared memory); 'tcgen05_layers':
        one tensor-core kernel per layer; 'training': the training GEMMs."""
        code = {"tcgen05": _abi.GPRM_MLP_INFER_TCGEN05, "training": _abi.GPRM_MLP_INFER_TRAINING_GEMM,
                "tcgen05_layers": _abi.GPRM_MLP_INFER_TCGEN05_LAYERS}[path]
        self._check(self.lib.gprm_mlp_set_inference(self.h, code))

    def set_training(self, path: str) -> None:
        """GEMMs of training: 'tcgen05' (default; tensor-core GEMMs with
        TMA-loaded operands) or 'mma_sync' (warp-level MMA)."""
        code = {"tcgen05": _abi.GPRM_MLP_TRAIN_TCGEN05, "mma_sync": _abi.GPRM_MLP_TRAIN_MMA_SYNC}[path]
        self._check(self.lib.gprm_mlp_set_training(self.h, code))

    def set_wait_budget(self, cycles: int = 0) -> None:
        """Test hook: clock budget of the tensor-core kernels' pipeline waits
        (0 = default, about a second); also clears the device status."""
        st = self.lib.gprm_mlp_set_wait_budget(self.h, int(cycles))
        if st != 0:
            raise RuntimeError(self.lib.gprm_mlp_last_error(self.h).decode())

    def device_status(self) -> int:
        """Synchronises; 0 unless a tensor-core layer gave up waiting for its MMAs."""
        f = C.c_uint(0)
        self.lib.gprm_mlp_device_status(self.h, C.byref(f))
        return int(f.value)

    def gradients(self, q_soa, y):
        import torch
        n = int(q_soa.shape[1])
        torch.cuda.synchronize()
        g = np.zeros(self.num_params, np.float32)
        loss = C.c_float(0)
        self._check(self.lib.gprm_mlp_gradients(self.h, C.c_void_p(q_soa.data_ptr()), C.c_void_p(y.data_ptr()),
                                                n, n, _abi.fptr(g), C.byref(loss)))
        return g, loss.value

    def adam_step(self, lr: float = 1e-3) -> None:
        self._check(self.lib.gprm_mlp_adam_step(self.h, lr))

    def train(self, q_soa, y, epochs: int = 10, batch: int = 4096, lr: float = 1e-3, seed: int = 0):
        """Trains on labelled configurations (q_soa (ndof, n) and y (n,) float
        CUDA tensors); returns the mean loss of each epoch."""
        import torch
        n = int(q_soa.shape[1])
        g = torch.Generator(device=q_soa.device)
        g.manual_seed(seed)
        perm = torch.stack([torch.randperm(n, device=q_soa.device, generator=g) for _ in range(epochs)])
        perm = perm.to(torch.int32).contiguous()
        torch.cuda.synchronize()
        losses = np.zeros(epochs, np.float32)
        self._check(self.lib.gprm_mlp_train(self.h, C.c_void_p(q_soa.data_ptr()), C.c_void_p(y.data_ptr()), n, n,
                                            C.c_void_p(perm.data_ptr()), epochs, batch, lr, _abi.fptr(losses)))
        return losses
