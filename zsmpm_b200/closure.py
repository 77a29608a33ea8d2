"""Learned return-mapping closure: an MLP 6 -> 64 -> 64 -> 64 -> 6 (SiLU) that replaces the
return-mapping branch of the Drucker-Prager (ConstitutiveModel_Vol_dP.hpp:241-325) or snow
(SnowPlasticity.hpp:24-32) update inside G2P.

Rows are raw features [n, 6]: the log singular values of the trial F (sorted as the SVD
returns them), then (friction angle in degrees, cohesion as a log-strain shift, logJp) for
Drucker-Prager or (theta_c, theta_s, log Jp) for snow.  Outputs are [n, 6]: projected minus
trial log strain (3) and principal Kirchhoff stress (3).  Device buffers are torch CUDA
tensors; the work runs in libzsmpm.so (training by its forward/backward/Adam kernels,
inference on BF16 tensor cores).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .scenes import MaterialSpec


def _stream(stream) -> C.c_void_p:
    if stream is None or stream == 0:
        return C.c_void_p(0)
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def _rows(t, name):
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.dim() == 2
            and t.shape[1] == 6 and t.is_contiguous()):
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor of shape [n, 6]")
    return C.c_void_p(t.data_ptr())


# A longer schedule than fit()'s default: five stages of falling learning rate, 76 epochs in
# all (the bench trains its closures with the same stages).
SCHEDULE_LONG = ((20, 4096, 2e-3), (20, 4096, 5e-4), (16, 8192, 1e-4), (12, 16384, 3e-5), (8, 32768, 1e-5))


class Closure:
    """Owns one zsmpm_closure handle (weights, Adam state, training set) on one GPU."""

    def __init__(self, material: MaterialSpec, volume: float, device: int = 0):
        from . import material_struct
        self._lib = _abi.lib()
        self._h = C.c_void_p()
        self.device = device
        self.material = material
        mat = material_struct(material, volume)
        _abi.check(self._lib.zsmpm_closure_create(C.byref(mat), device, C.byref(self._h)),
                   "closure_create")

    def close(self) -> None:
        if self._h:
            self._lib.zsmpm_closure_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # ---- data and training
    def build_dataset(self, n_random: int, seed: int = 0, logged=None, stream=None) -> None:
        """Random trial states plus optional logged rows (CUDA tensor [m, 6]); sets the input
        normalisation and the training hull."""
        if logged is not None and logged.shape[0] > 0:
            ptr, n_logged = _rows(logged, "logged"), int(logged.shape[0])
        else:
            ptr, n_logged = None, 0
        _abi.check(self._lib.zsmpm_closure_build_dataset(self._h, int(n_random), C.c_uint64(seed), ptr,
                                                         n_logged, _stream(stream)), "closure_build_dataset")

    def dataset_size(self) -> tuple:
        """(rows generated or logged, rows kept: those the plain return map projects)."""
        g, k = C.c_int64(), C.c_int64()
        _abi.check(self._lib.zsmpm_closure_dataset_size(self._h, C.byref(g), C.byref(k)), "closure_dataset_size")
        return int(g.value), int(k.value)

    def train(self, epochs: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0,
              stream=None) -> np.ndarray:
        """Adam epochs over the training set; returns the mean loss of each epoch."""
        losses = np.zeros(epochs, np.float32)
        _abi.check(self._lib.zsmpm_closure_train(self._h, int(epochs), int(batch), C.c_float(lr),
                                                 C.c_uint64(seed), losses.ctypes.data_as(C.c_void_p),
                                                 _stream(stream)), "closure_train")
        return losses

    def fit(self, schedule=((6, 4096, 2e-3), (6, 4096, 5e-4), (4, 8192, 1e-4)), seed: int = 1) -> np.ndarray:
        """Train through a list of (epochs, batch, learning rate) phases; returns all epoch losses."""
        return np.concatenate([self.train(e, batch=b, lr=lr, seed=seed + k)
                               for k, (e, b, lr) in enumerate(schedule)])

    def loss_grad(self, x, y, stream=None):
        """Loss and gradient (torch tensors) of the training kernels on raw rows x, y."""
        import torch
        grad = torch.empty(_abi.MLP_PARAMS, dtype=torch.float32, device=x.device)
        loss = torch.empty(1, dtype=torch.float32, device=x.device)
        _abi.check(self._lib.zsmpm_closure_loss_grad(self._h, _rows(x, "x"), _rows(y, "y"), int(x.shape[0]),
                                                     C.c_void_p(grad.data_ptr()), C.c_void_p(loss.data_ptr()),
                                                     _stream(stream)), "closure_loss_grad")
        return loss, grad

    def infer(self, x, bf16: bool = True, stream=None, path: str | None = None):
        """Network outputs (D, tau) of raw rows x.  path: "fp32", "mma_sync", "tcgen05" (BF16
        operands) or "tcgen05_split" (split-BF16 operands, the substep's path); by default
        "mma_sync" when bf16 else "fp32"."""
        import torch
        mode = {"fp32": 0, "mma_sync": 1, "tcgen05": 2, "tcgen05_split": 3}[path or ("mma_sync" if bf16 else "fp32")]
        y = torch.empty_like(x)
        _abi.check(self._lib.zsmpm_closure_infer(self._h, _rows(x, "x"), _rows(y, "y"), int(x.shape[0]),
                                                 mode, _stream(stream)), "closure_infer")
        return y

    def status(self) -> None:
        """Synchronises; raises if a bounded tensor-core wait of the tcgen05 path gave up."""
        _abi.check(self._lib.zsmpm_closure_status(self._h), "closure_status")

    def targets(self, x, stream=None):
        """The plain return map's (D, tau) for raw rows x."""
        import torch
        y = torch.empty_like(x)
        _abi.check(self._lib.zsmpm_closure_targets(self._h, _rows(x, "x"), _rows(y, "y"), int(x.shape[0]),
                                                   _stream(stream)), "closure_targets")
        return y

    # ---- state
    def get_state(self) -> _abi.ClosureState:
        st = _abi.ClosureState()
        _abi.check(self._lib.zsmpm_closure_get_state(self._h, C.byref(st)), "closure_get_state")
        return st

    def set_state(self, st: _abi.ClosureState) -> None:
        _abi.check(self._lib.zsmpm_closure_set_state(self._h, C.byref(st)), "closure_set_state")

    def state_arrays(self) -> dict:
        st = self.get_state()
        return {"model": int(st.model), "params": np.ctypeslib.as_array(st.params).copy(),
                **{k: np.ctypeslib.as_array(getattr(st, k)).copy()
                   for k in ("in_mean", "in_inv_std", "in_min", "in_max", "out_scale")}}


def attach(scene, closure: Closure | None, audit_period: int = 100) -> None:
    """Make G2P of `scene` use `closure` (None restores the plain return map); one particle in
    `audit_period` per substep is checked against the plain map."""
    h = closure.handle if closure is not None else None
    _abi.check(scene._lib.zsmpm_scene_set_closure(scene.handle, h, int(audit_period)), "scene_set_closure")


def audit(scene, reset: bool = False) -> dict:
    a = _abi.ClosureAudit()
    _abi.check(scene._lib.zsmpm_scene_closure_audit(scene.handle, C.byref(a), int(bool(reset))),
               "scene_closure_audit")
    return {"audited": int(a.audited), "mean_rel_error": a.mean_rel_error,
            "max_rel_error": a.max_rel_error, "agg_rel_error": a.agg_rel_error,
            "fallbacks": int(a.fallbacks), "network_updates": int(a.network_updates), "updates": int(a.updates),
            "network_share": (a.network_updates / a.updates) if a.updates else 0.0}


def set_state_log(scene, buffer, period: int) -> None:
    """Log one particle in `period` per substep (trial-state features) into `buffer`, a CUDA
    tensor [cap, 6]; period 0 stops logging."""
    if period > 0:
        ptr, cap = _rows(buffer, "buffer"), int(buffer.shape[0])
    else:
        ptr, cap = None, 0
    _abi.check(scene._lib.zsmpm_scene_set_state_log(scene.handle, ptr, cap, int(period)),
               "scene_set_state_log")


def state_log_count(scene) -> int:
    n = C.c_int64()
    _abi.check(scene._lib.zsmpm_scene_state_log_count(scene.handle, C.byref(n)), "scene_state_log_count")
    return int(n.value)
