"""The MLP over libdtlg.so's own FP32 kernels (dtlg_mlp_* in include/dtlg.h).

Forward, backward and Adam run as this library's CUDA kernels (csrc/mlp.cu);
torch only holds the device buffers.  Parameters: for each layer W [in x out]
(row-major) then b [out], back to back.
"""
import ctypes as C

import numpy as np

from .. import _lib
from ._torch import torch_mod


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    torch = torch_mod()
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class MLP:
    def __init__(self, n_in, width=64, hidden_layers=3, n_out=1, max_batch=4096):
        h = C.c_void_p()
        _lib.check(_lib.lib().dtlg_mlp_create(n_in, width, hidden_layers, n_out, max_batch, C.byref(h)), "mlp_create")
        self._h = h
        self.dims = [n_in] + [width] * hidden_layers + [n_out]
        self.max_batch = max_batch

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                _lib.lib().dtlg_mlp_destroy(h)
            except Exception:
                pass

    @property
    def n_in(self):
        return self.dims[0]

    @property
    def n_out(self):
        return self.dims[-1]

    def param_count(self):
        return int(_lib.lib().dtlg_mlp_param_count(self._h))

    def layers(self, flat):
        """Views (W [in x out], b [out]) of a flat parameter vector."""
        out, off = [], 0
        for a, b in zip(self.dims[:-1], self.dims[1:]):
            W = flat[off:off + a * b].reshape(a, b)
            off += a * b
            out.append((W, flat[off:off + b]))
            off += b
        return out

    def init_params(self, seed=0):
        """He-uniform weights (bound sqrt(6 / fan_in)), zero biases."""
        rng = np.random.default_rng(seed)
        flat = np.zeros(self.param_count(), dtype=np.float32)
        for W, b in self.layers(flat):
            bound = np.sqrt(6.0 / W.shape[0])
            W[...] = rng.uniform(-bound, bound, W.shape)
        self.set_params(flat)
        return flat

    def set_params(self, flat):
        flat = np.ascontiguousarray(flat, dtype=np.float32)
        assert flat.size == self.param_count()
        _lib.check(_lib.lib().dtlg_mlp_set_params(self._h, C.c_void_p(flat.ctypes.data)), "mlp_set_params")

    def get_params(self):
        out = np.empty(self.param_count(), dtype=np.float32)
        _lib.check(_lib.lib().dtlg_mlp_get_params(self._h, C.c_void_p(out.ctypes.data)), "mlp_get_params")
        return out

    def get_grads(self):
        out = np.empty(self.param_count(), dtype=np.float32)
        _lib.check(_lib.lib().dtlg_mlp_get_grads(self._h, C.c_void_p(out.ctypes.data)), "mlp_get_grads")
        return out

    def _check_rows(self, t, width, name):
        torch = torch_mod()
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
                and t.dim() == 2 and t.shape[1] == width):
            raise ValueError(f"{name} must be a contiguous float32 CUDA tensor [rows x {width}]")

    def forward(self, x):
        torch = torch_mod()
        self._check_rows(x, self.n_in, "x")
        y = torch.empty((x.shape[0], self.n_out), dtype=torch.float32, device=x.device)
        _lib.check(_lib.lib().dtlg_mlp_forward(self._h, _p(x), x.shape[0], _p(y), _stream()), "mlp_forward")
        return y

    def loss_grad(self, x, t, w):
        """Loss of one batch (float) and its gradients (into the model)."""
        torch = torch_mod()
        self._check_rows(x, self.n_in, "x")
        self._check_rows(t, self.n_out, "t")
        self._check_rows(w, self.n_out, "w")
        loss = torch.zeros(1, dtype=torch.float32, device=x.device)
        _lib.check(_lib.lib().dtlg_mlp_loss_grad(self._h, _p(x), _p(t), _p(w), x.shape[0], _p(loss), _stream()),
                   "mlp_loss_grad")
        return float(loss.item())

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        _lib.check(_lib.lib().dtlg_mlp_adam_step(self._h, lr, beta1, beta2, eps, _stream()), "mlp_adam_step")

    def train(self, x, t, w, batch_rows, batch, lr_start, lr_end):
        """Adam steps over the batches listed in batch_rows [steps x batch]
        (int32 CUDA tensor of row indexes); returns the loss curve (CUDA)."""
        torch = torch_mod()
        self._check_rows(x, self.n_in, "x")
        self._check_rows(t, self.n_out, "t")
        self._check_rows(w, self.n_out, "w")
        assert batch_rows.is_cuda and batch_rows.dtype == torch.int32 and batch_rows.is_contiguous()
        steps = batch_rows.numel() // batch
        curve = torch.zeros(steps, dtype=torch.float32, device=x.device)
        _lib.check(_lib.lib().dtlg_mlp_train(self._h, _p(x), _p(t), _p(w), x.shape[0], _p(batch_rows), batch, steps,
                                             lr_start, lr_end, _p(curve), _stream()), "mlp_train")
        return curve

    def choose(self, x, n_cand):
        """Per row: argmin of the first n_cand outputs and output n_cand + argmin."""
        torch = torch_mod()
        self._check_rows(x, self.n_in, "x")
        n = x.shape[0]
        y = torch.empty((n, self.n_out), dtype=torch.float32, device=x.device)
        choice = torch.empty(n, dtype=torch.int32, device=x.device)
        aux = torch.empty(n, dtype=torch.float32, device=x.device)
        _lib.check(_lib.lib().dtlg_mlp_choose(self._h, _p(x), n, n_cand, _p(y), _p(choice), _p(aux), _stream()),
                   "mlp_choose")
        return choice, aux
