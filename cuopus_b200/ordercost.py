"""Visiting order of the file entry points: the additive chain cost of
csrc/ordercost.cpp, its features through the C ABI, and the fit of its weights.

The file entry points (cuopus_decode_f16k_multi and the rest) queue chains
longest first by

    cost(chain) = w0 + sum over the chain's packets of w . features(packet)

with non-negative weights, one set for 8 lanes per chain and one for 32.  The
weights are fitted by non-negative least squares to per-chain decode times
that the decoder records on the device (res[c].time_us) while it decodes a
training corpus; `write_coefficients` writes them as csrc/ordercost_coef.inc,
which the library compiles in.  `python bench.py --fit-order` measures the
times and runs the fit.  The order changes no decoded sample.
"""
from __future__ import annotations

import ctypes
import datetime
import json

import numpy as np

from . import cuopus_native as cn

NFEAT = 27
FEATURE_NAMES = (["chain", "packets", "bytes/100"] +
                 ["%s%s_%s" % (m, d, s) for m, ds in (("silk", ("10", "20", "40", "60")), ("hybrid", ("10", "20")),
                                                      ("celt", ("2.5", "5", "10", "20")))
                  for d in ds for s in ("mono", "stereo")] +
                 ["silk_ms_x_bw", "celt_ms_x_bw", "stereo_out_ms", "empty_packets"])
assert len(FEATURE_NAMES) == NFEAT


def _lib():
    lib = cn.lib()
    if not getattr(lib, "_oc_bound", False):
        c_p = ctypes.c_void_p
        lib.cuopus_order_features.argtypes = [c_p] * 6 + [ctypes.c_int32, c_p]
        lib.cuopus_order_costs.argtypes = [c_p] * 6 + [ctypes.c_int32, ctypes.c_int32, c_p]
        lib.cuopus_order_features.restype = ctypes.c_int
        lib.cuopus_order_costs.restype = ctypes.c_int
        lib.cuopus_order_model_fitted.restype = ctypes.c_int
        lib._oc_bound = True
    return lib


def _tables(host):
    """The host chain tables (dict of numpy arrays: blob, off, len, first,
    npkts, chans) in the C ABI's types."""
    t = dict(blob=np.ascontiguousarray(host["blob"], np.uint8), off=np.ascontiguousarray(host["off"], np.uint64),
             len=np.ascontiguousarray(host["len"], np.uint32), first=np.ascontiguousarray(host["first"], np.uint32),
             npkts=np.ascontiguousarray(host["npkts"], np.uint32),
             chans=np.ascontiguousarray(host["chans"], np.uint8))
    P = lambda a: ctypes.c_void_p(a.ctypes.data)
    return t, [P(t[k]) for k in ("blob", "off", "len", "first", "npkts", "chans")]


def features(host):
    """[nchains, 27] float64 features of every chain."""
    t, ptrs = _tables(host)
    n = len(t["first"])
    out = np.zeros((max(n, 1), NFEAT), np.float64)
    rc = _lib().cuopus_order_features(*ptrs, n, ctypes.c_void_p(out.ctypes.data))
    if rc:
        raise cn.CuopusError(rc, "cuopus_order_features")
    return out[:n]


def costs(host, width):
    """Per-chain cost under the compiled-in weights for `width` lanes."""
    t, ptrs = _tables(host)
    n = len(t["first"])
    out = np.zeros(max(n, 1), np.float64)
    rc = _lib().cuopus_order_costs(*ptrs, n, int(width), ctypes.c_void_p(out.ctypes.data))
    if rc:
        raise cn.CuopusError(rc, "cuopus_order_costs")
    return out[:n]


def fitted():
    return bool(_lib().cuopus_order_model_fitted())


def weights(width):
    """The compiled-in weights for `width` lanes per chain."""
    w = np.zeros(NFEAT, np.float64)
    lib = _lib()
    lib.cuopus_order_weights.argtypes = [ctypes.c_int32, ctypes.c_void_p]
    if lib.cuopus_order_weights(int(width), ctypes.c_void_p(w.ctypes.data)):
        raise cn.CuopusError(3, "cuopus_order_weights")
    return w


def fit(feats, times):
    """Non-negative least squares of per-chain times (us) on the features.
    Columns are scaled to unit norm for the solve.  Returns (weights, stats)."""
    from scipy.optimize import nnls
    X = np.asarray(feats, np.float64)
    y = np.asarray(times, np.float64)
    scale = np.linalg.norm(X, axis=0)
    scale[scale == 0] = 1.0
    w, _ = nnls(X / scale, y, maxiter=50 * X.shape[1])
    w = w / scale
    pred = X @ w
    r2 = 1.0 - float(np.sum((y - pred) ** 2) / np.sum((y - y.mean()) ** 2))
    return w, {"chains": int(len(y)), "r2_time": round(r2, 4),
               "mean_abs_error_pct": round(float(np.mean(np.abs(pred - y)) / np.mean(y) * 100.0), 2)}


def makespan(cost, order, slots):
    """List scheduling: chains in `order` go to the first free of `slots`
    groups; returns the finish time of the last one."""
    import heapq
    free = [0.0] * int(slots)
    heapq.heapify(free)
    end = 0.0
    for c in order:
        t = heapq.heappop(free) + float(cost[c])
        end = max(end, t)
        heapq.heappush(free, t)
    return end


def _fmt_row(w):
    return ", ".join("%.6g" % v for v in w)


def write_coefficients(path, w8, w32, info):
    """csrc/ordercost_coef.inc with the fitted weights (microseconds)."""
    lines = ["// Weights of the visiting-order cost (ordercost.cpp), in microseconds of",
             "// device time per unit of each feature: non-negative least squares on the",
             "// per-chain decode times of a training corpus, written by",
             "// cuopus_b200/ordercost.py (python bench.py --fit-order) on %s." % datetime.date.today().isoformat()]
    for k in sorted(info):
        lines.append("// %s: %s" % (k, json.dumps(info[k], sort_keys=True)))
    lines.append("#define CUO_ORDER_FITTED 1")
    for name, w in (("kOrderCoef8", w8), ("kOrderCoef32", w32)):
        lines.append("static const double %s[%d] = {" % (name, NFEAT))
        for i in range(0, NFEAT, 6):
            lines.append("    " + _fmt_row(w[i:i + 6]) + ("," if i + 6 < NFEAT else "};"))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
