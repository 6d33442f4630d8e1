"""Learned cost model of the decode scheduler (Python front end of the
kernels in csrc/costmodel.cu, reached through the C ABI).

A chain's decode time is predicted from 16 features of its packets' TOC
bytes (mode, frame sizes, bandwidth, channels, sizes) by an FP32 MLP
16 -> 64 -> 64 -> 1 with ReLU, trained on the GPU on log cycle counts that the
decoder itself records per chain (res[c].time_us).  The queue schedule then
visits chains longest first by prediction.  The fallback, and the baseline the
model is measured against, is the packet-count order (packets x channels).

The model only orders the work; decoded samples never depend on it.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import cuopus_native as cn

NFEAT = 16
NPARAM = 16 * 64 + 64 + 64 * 64 + 64 + 64 + 1


def _lib():
    lib = cn.lib()
    if not getattr(lib, "_cm_bound", False):
        c_p = ctypes.c_void_p
        tail = [c_p, ctypes.c_char_p, ctypes.c_size_t]
        lib.cuopus_chain_features.argtypes = [ctypes.POINTER(cn.Batch), c_p] + tail
        lib.cuopus_mlp_init.argtypes = [c_p, ctypes.c_uint64] + tail
        lib.cuopus_mlp_predict.argtypes = [c_p, c_p, ctypes.c_int, c_p] + tail
        lib.cuopus_mlp_grad.argtypes = [c_p, c_p, c_p, ctypes.c_int, c_p, c_p] + tail
        lib.cuopus_mlp_train.argtypes = [c_p, c_p, c_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, c_p] + tail
        for f in ("cuopus_chain_features", "cuopus_mlp_init", "cuopus_mlp_predict", "cuopus_mlp_grad",
                  "cuopus_mlp_train"):
            getattr(lib, f).restype = ctypes.c_int
        lib._cm_bound = True
    return lib


def _call(fn, *args):
    err = ctypes.create_string_buffer(512)
    rc = fn(*args, err, 512)
    if rc:
        raise cn.CuopusError(rc, err.value.decode(errors="replace"))


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def chain_features(batch: cn.Batch):
    """Device float32 tensor [nchains, 16] from a device-resident batch."""
    import torch
    out = torch.empty((max(batch.nchains, 1), NFEAT), dtype=torch.float32, device="cuda")
    _call(_lib().cuopus_chain_features, ctypes.byref(batch), ctypes.c_void_p(out.data_ptr()), _stream())
    return out[:batch.nchains]


def packet_order(npkts, channels):
    """The fallback order: packets x channels, longest first (stable)."""
    cost = np.asarray(npkts, np.int64) * np.asarray(channels, np.int64)
    return np.argsort(-cost, kind="stable")


def makespan(cost, order, slots):
    """The scheduler's estimate of a batch's decode time: chains taken in
    `order` by the first of `slots` decoder groups to come free, each busy for
    its chain's cost (list scheduling, as the device queue hands them out)."""
    import heapq
    free = [0.0] * max(int(slots), 1)
    end = 0.0
    for c in order:
        t = heapq.heappop(free) + float(cost[c])
        end = max(end, t)
        heapq.heappush(free, t)
    return end


class CostModel:
    """FP32 MLP over chain features; targets are standardised log decode times."""

    def __init__(self, seed=0):
        import torch
        self.params = torch.empty(NPARAM, dtype=torch.float32, device="cuda")
        _call(_lib().cuopus_mlp_init, ctypes.c_void_p(self.params.data_ptr()), ctypes.c_uint64(seed), _stream())
        self.mu, self.sigma = 0.0, 1.0

    def grad(self, X, T):
        """(loss, gradient) of the mean squared error on device tensors."""
        import torch
        X = X.contiguous().float()
        T = T.contiguous().float()
        g = torch.empty(NPARAM, dtype=torch.float32, device="cuda")
        loss = torch.empty(1, dtype=torch.float32, device="cuda")
        _call(_lib().cuopus_mlp_grad, ctypes.c_void_p(self.params.data_ptr()), ctypes.c_void_p(X.data_ptr()),
              ctypes.c_void_p(T.data_ptr()), int(X.shape[0]), ctypes.c_void_p(g.data_ptr()),
              ctypes.c_void_p(loss.data_ptr()), _stream())
        return float(loss.item()), g

    def fit(self, X, cost, steps=2000, lr=3e-3):
        """Train on device features X [n, 16] and measured decode times (host or
        device, > 0).  Returns the per-step losses."""
        import torch
        y = np.log(np.maximum(np.asarray(torch.as_tensor(cost).cpu().numpy(), np.float64), 1.0))
        self.mu, self.sigma = float(y.mean()), float(y.std() or 1.0)
        T = torch.from_numpy(((y - self.mu) / self.sigma).astype(np.float32)).cuda()
        X = X.contiguous().float()
        losses = np.zeros(max(int(steps), 1), np.float32)
        _call(_lib().cuopus_mlp_train, ctypes.c_void_p(self.params.data_ptr()), ctypes.c_void_p(X.data_ptr()),
              ctypes.c_void_p(T.data_ptr()), int(X.shape[0]), int(steps), ctypes.c_float(lr),
              ctypes.c_void_p(losses.ctypes.data), _stream())
        return losses[:steps]

    def predict_raw(self, X):
        """Network outputs (standardised log decode times) as a device tensor."""
        import torch
        X = X.contiguous().float()
        y = torch.empty(max(int(X.shape[0]), 1), dtype=torch.float32, device="cuda")
        _call(_lib().cuopus_mlp_predict, ctypes.c_void_p(self.params.data_ptr()), ctypes.c_void_p(X.data_ptr()),
              int(X.shape[0]), ctypes.c_void_p(y.data_ptr()), _stream())
        return y[:X.shape[0]]

    def predict(self, X):
        """Predicted decode time per chain (host float64, the unit of the targets)."""
        y = self.predict_raw(X).cpu().numpy().astype(np.float64)
        return np.exp(y * self.sigma + self.mu)

    def order(self, X):
        """Longest-first visiting order by predicted decode time (stable)."""
        return np.argsort(-self.predict(X), kind="stable")

    def state(self):
        return dict(params=self.params.cpu().numpy(), mu=self.mu, sigma=self.sigma)

    def load(self, state):
        import torch
        self.params.copy_(torch.as_tensor(np.asarray(state["params"], np.float32)))
        self.mu, self.sigma = float(state["mu"]), float(state["sigma"])
        return self
