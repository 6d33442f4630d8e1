"""CPU restatement of the scheduler's cost model, for the tests.

TEST INFRASTRUCTURE (oracle).  The reference has no cost model (its decode
kernel assigns chains to slots in index order, cuopus_kernels.cuh:41-69); this
module restates in numpy, in float64, what the product's kernels in
cuopus_b200/csrc/costmodel.cu compute, so that the GPU forward pass, gradients
and features can be checked against an independent implementation:

  features(packets, chains, channels)   16 features per chain from TOC bytes
  forward(params, X)                    16 -> 64 -> 64 -> 1 MLP with ReLU
  loss_and_grad(params, X, T)           mean squared error and its gradient in
                                        the flat parameter layout
                                        W1[16][64] | b1 | W2[64][64] | b2 | w3 | b3
"""
from __future__ import annotations

import numpy as np

F, H = 16, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + F * H
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAM = OFF_B3 + 1


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OFF_W1:OFF_B1].reshape(F, H), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def forward(params, X):
    W1, b1, W2, b2, w3, b3 = unpack(params)
    X = np.asarray(X, np.float64)
    h1 = np.maximum(X @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    return h2 @ w3 + b3


def loss_and_grad(params, X, T):
    W1, b1, W2, b2, w3, b3 = unpack(params)
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    n = X.shape[0]
    a1 = X @ W1 + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0.0)
    y = h2 @ w3 + b3
    e = y - T
    loss = float(np.mean(e * e))
    d = 2.0 * e / n
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = h2.T @ d
    g[OFF_B3] = d.sum()
    g2 = (d[:, None] * w3[None, :]) * (a2 > 0)
    g[OFF_W2:OFF_B2] = (h1.T @ g2).reshape(-1)
    g[OFF_B2:OFF_W3] = g2.sum(0)
    g1 = (g2 @ W2.T) * (a1 > 0)
    g[OFF_W1:OFF_B1] = (X.T @ g1).reshape(-1)
    g[OFF_B1:OFF_W2] = g1.sum(0)
    return loss, g


def _qms(cfg):
    if cfg < 12:
        return (40, 80, 160, 240)[cfg & 3]
    if cfg < 16:
        return 80 if cfg & 1 else 40
    return 10 << (cfg & 3)


def _bw(cfg):
    if cfg < 12:
        return cfg >> 2
    if cfg < 16:
        return 3 if cfg < 14 else 4
    b = (cfg - 16) >> 2
    return 0 if b == 0 else b + 1


def features(packets, chains, channels):
    """float32 [n_chains, 16]; chains: (first, npkts, ...) over packets."""
    out = np.zeros((len(chains), F), np.float32)
    for c, ch in enumerate(chains):
        first, n = int(ch[0]), int(ch[1])
        nbytes = frames = q = 0.0
        fm = [0.0, 0.0, 0.0]
        f25 = f5 = f10 = f20 = f40 = bw = stereo = 0.0
        for k in range(n):
            p = packets[first + k]
            nbytes += len(p)
            if not p:
                continue
            toc = p[0]
            cfg, code = toc >> 3, toc & 3
            nf = 1 if code == 0 else 2 if code < 3 else ((p[1] & 63) if len(p) > 1 else 0)
            qms = _qms(cfg)
            frames += nf
            q += nf * qms
            fm[0 if cfg < 12 else 1 if cfg < 16 else 2] += nf
            if qms == 10:
                f25 += nf
            elif qms == 20:
                f5 += nf
            elif qms == 40:
                f10 += nf
            elif qms == 80:
                f20 += nf
            else:
                f40 += nf
            bw += nf * _bw(cfg)
            stereo += (toc >> 2) & 1
        secs = q / 4000.0
        fr = 1.0 / frames if frames > 0 else 0.0
        chans = channels[c] if hasattr(channels, "__len__") else channels
        out[c] = [np.log1p(n), np.log1p(nbytes), np.log1p(frames), np.log1p(secs), chans - 1,
                  fm[0] * fr, fm[1] * fr, fm[2] * fr, f25 * fr, f5 * fr, f10 * fr, f20 * fr, f40 * fr,
                  bw * fr * 0.25, stereo / n if n else 0.0, np.log1p(nbytes / secs if secs > 0 else 0.0)]
    return out


def makespan(costs, order, slots):
    """Greedy list schedule: chains in `order` go to the earliest free of
    `slots` identical decoder slots; returns the finish time of the last."""
    import heapq
    free = [0.0] * max(int(slots), 1)
    heapq.heapify(free)
    end = 0.0
    for c in order:
        t = heapq.heappop(free) + float(costs[c])
        end = max(end, t)
        heapq.heappush(free, t)
    return end
