"""Learned snow plasticity: the host side of libmpm's surrogate network.

The reference always runs the exact return map applyPlasticity
(src/lib/gpu/shaderPrelude/plasticityOps.wgsl:7-48).  This module drives the
library's replacement for it: a 12 -> 64 -> 64 -> 64 -> 11 SiLU network whose
forward and backward passes run as BF16 tensor-core kernels (FP32
accumulation) in libmpm.so, trained on the GPU on (trial state -> exact
result) pairs that the exact map itself produces during rollouts
(PLASTICITY_COLLECT), and used in a substep with an exact fallback and an
audited sample (PLASTICITY_LEARNED).  Device arrays are torch CUDA tensors
(float32, contiguous); torch is only the allocator here.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import MpmMlpTrainConfig, MpmPlasticityStats, check, load

PARAMS = _lib.MLP_PARAMS


def _ptr(t) -> C.c_void_p:
    if not (t.is_cuda and t.is_contiguous()):
        raise ValueError("expected a contiguous CUDA tensor")
    return C.c_void_p(t.data_ptr())


class PlasticityNet:
    """One network (parameters, Adam state) on one device."""

    def __init__(self, device: int = 0, seed: int = 0):
        self._lib = load()
        h = C.c_void_p()
        rc = self._lib.mpm_mlp_create(device, seed, C.byref(h))
        if rc != _lib.MPM_OK:
            msg = self._lib.mpm_mlp_last_error(h).decode() if h.value else "mpm_mlp_create failed"
            if h.value:
                self._lib.mpm_mlp_destroy(h)
            raise _lib.MpmError(rc, msg)
        self.handle = h
        self.device = device

    def _check(self, rc: int) -> None:
        if rc != _lib.MPM_OK:
            raise _lib.MpmError(rc, self._lib.mpm_mlp_last_error(self.handle).decode())

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.mpm_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream: int | None) -> None:
        """Orders the network's kernels on a CUDA stream handle (None: private)."""
        self._check(self._lib.mpm_mlp_set_stream(self.handle, C.c_void_p(stream) if stream else None))

    @staticmethod
    def init_params(seed: int) -> np.ndarray:
        out = np.zeros(PARAMS, np.float32)
        load().mpm_mlp_init_params(seed, out.ctypes.data)
        return out

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(PARAMS, np.float32)
        self._check(self._lib.mpm_mlp_get_params(self.handle, out.ctypes.data))
        return out

    @params.setter
    def params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == PARAMS
        self._check(self._lib.mpm_mlp_set_params(self.handle, p.ctypes.data))

    def forward(self, x):
        """Network outputs [n, 11] for inputs x [n, 12] (CUDA tensors)."""
        import torch

        n = x.shape[0]
        y = torch.empty((n, _lib.MLP_OUTPUTS), dtype=torch.float32, device=x.device)
        self._check(self._lib.mpm_mlp_forward(self.handle, _ptr(x), n, _ptr(y)))
        return y

    def gradient(self, x, t, unc_weight: float = 0.1):
        """(loss, gradient [PARAMS]) of the batch loss over pairs (x, t)."""
        g = np.zeros(PARAMS, np.float32)
        loss = C.c_float(0.0)
        self._check(self._lib.mpm_mlp_gradient(self.handle, _ptr(x), _ptr(t), x.shape[0], unc_weight,
                                               g.ctypes.data, C.byref(loss)))
        return float(loss.value), g

    def train(self, x, t, *, epochs: int = 10, batch: int = 8192, lr: float = 2e-3, lr_final: float = 5e-5,
              unc_weight: float = 0.1, seed: int = 0) -> np.ndarray:
        """Adam on the GPU; returns the mean batch loss of every epoch."""
        cfg = MpmMlpTrainConfig(epochs=epochs, batch=batch, lr=lr, lr_final=lr_final, unc_weight=unc_weight,
                                seed=seed)
        hist = np.zeros(epochs, np.float32)
        self._check(self._lib.mpm_mlp_train(self.handle, _ptr(x), _ptr(t), x.shape[0], C.byref(cfg),
                                            hist.ctypes.data))
        return hist


class PlasticityController:
    """Plasticity mode of one buffer manager's handle (inline exact map by
    default; see include/mpm.h for the modes)."""

    def __init__(self, mpm_manager):
        self.mpm = mpm_manager
        self._lib = load()
        self._pairs = None

    def set_mode(self, mode: int, net: PlasticityNet | None = None, *, unc_threshold: float = 0.05,
                 det_threshold: float = 1e-3, audit_fraction: float = 0.01) -> None:
        """audit_fraction: LEARNED, the audited share of the network's answers;
        COLLECT, the sampled share of listed particles that write a pair."""
        self.net = net
        check(self._lib.mpm_set_plasticity(self.mpm.handle, mode, net.handle if net else None, unc_threshold,
                                           det_threshold, audit_fraction), self.mpm.handle)

    def collect_into(self, capacity: int, device: int = 0):
        """Allocates and attaches a pair buffer of `capacity` pairs."""
        import torch

        x = torch.zeros((capacity, _lib.MLP_INPUTS), dtype=torch.float32, device=f"cuda:{device}")
        t = torch.zeros((capacity, _lib.MLP_TARGETS), dtype=torch.float32, device=f"cuda:{device}")
        check(self._lib.mpm_set_pair_buffer(self.mpm.handle, _ptr(x), _ptr(t), capacity), self.mpm.handle)
        self._pairs = (x, t)
        return x, t

    def detach_pairs(self) -> None:
        check(self._lib.mpm_set_pair_buffer(self.mpm.handle, None, None, 0), self.mpm.handle)
        self._pairs = None

    def stats(self, reset: bool = False) -> dict:
        s = MpmPlasticityStats()
        check(self._lib.mpm_get_plasticity_stats(self.mpm.handle, C.byref(s), 1 if reset else 0), self.mpm.handle)
        return s.as_dict()
