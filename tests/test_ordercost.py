"""The visiting order of the file entry points (csrc/ordercost.cpp), CPU only:
the chain features against a restatement from the TOC (RFC 6716 section 3.1),
costs as the weights' dot product with the features, and the non-negative
least-squares fit recovering planted weights."""
import json
import os
import re

import numpy as np
import pytest

from cuopus_b200 import cuopus_native as cn
from cuopus_b200 import ordercost

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
QMS = [40, 80, 160, 240] * 3 + [40, 80, 40, 80] + [10, 20, 40, 80] * 4


def _host_tables(names, seg=1.0):
    """Chain tables of golden streams cut in `seg` s chains with 250 ms preroll."""
    blobs, offs, lens, first, npk, chans = [], [], [], [], [], []
    bb = bp = 0
    for name in names:
        with open(os.path.join(GOLD, "streams", name + ".opus"), "rb") as f:
            ix = cn.index(f.read(), seg_s=seg, preroll_ms=250.0)
        blobs.append(ix.blob)
        offs.append(ix.pkt_off + bb)
        lens.append(ix.pkt_len)
        first.append(ix.first + bp)
        npk.append(ix.npkts)
        chans.append(np.full(len(ix.first), ix.channels, np.uint8))
        bb += len(ix.blob)
        bp += len(ix.pkt_len)
    cat = np.concatenate
    return dict(blob=cat(blobs + [np.zeros(16, np.uint8)]), off=cat(offs), len=cat(lens), first=cat(first),
                npkts=cat(npk), chans=cat(chans))


def _features_restated(h):
    n = len(h["first"])
    F = np.zeros((n, ordercost.NFEAT))
    for c in range(n):
        F[c, 0] = 1
        for q in range(int(h["first"][c]), int(h["first"][c]) + int(h["npkts"][c])):
            L = int(h["len"][q])
            F[c, 1] += 1
            F[c, 2] += L / 100.0
            if L == 0:
                F[c, 26] += 1
                continue
            p = h["blob"][int(h["off"][q]):int(h["off"][q]) + L]
            toc = int(p[0])
            cfg, code, s = toc >> 3, toc & 3, (toc >> 2) & 1
            nf = 1 if code == 0 else 2 if code < 3 else (int(p[1]) & 63 if L > 1 else 0)
            cls = (cfg & 3) if cfg < 12 else (4 + (cfg & 1)) if cfg < 16 else 6 + (cfg & 3)
            ms = nf * QMS[cfg] / 4.0
            F[c, 3 + 2 * cls + s] += nf
            if cfg < 12:
                F[c, 23] += ms * (cfg >> 2)
            elif cfg >= 16:
                F[c, 24] += ms * ((cfg - 16) >> 2)
            if int(h["chans"][c]) == 2:
                F[c, 25] += ms
    return F


@pytest.fixture(scope="module")
def tables():
    with open(os.path.join(GOLD, "index.json")) as f:
        names = sorted(json.load(f))
    return _host_tables(names)


def test_features_match_the_toc_restatement(tables):
    got = ordercost.features(tables)
    want = _features_restated(tables)
    assert got.shape == want.shape and len(got) > 20
    assert np.allclose(got, want, rtol=0, atol=1e-9)
    # every mode, mono and stereo, reaches some chain of the golden streams
    assert got[:, 3:11].sum() > 0 and got[:, 11:15].sum() > 0 and got[:, 15:23].sum() > 0
    assert got[:, 25].sum() > 0


@pytest.mark.parametrize("width", [1, 8, 32])
def test_costs_are_the_weights_dot_the_features(tables, width):
    w = ordercost.weights(width)
    assert np.all(w >= 0)
    got = ordercost.costs(tables, width)
    want = ordercost.features(tables) @ w
    assert np.allclose(got, want, rtol=1e-12, atol=1e-9)


def test_fitted_flag_matches_the_compiled_weights():
    with open(os.path.join(ROOT, "cuopus_b200", "csrc", "ordercost_coef.inc")) as f:
        m = re.search(r"#define CUO_ORDER_FITTED (\d)", f.read())
    assert ordercost.fitted() == (m.group(1) == "1")


def test_fit_recovers_planted_weights(tables):
    F = ordercost.features(tables)
    rng = np.random.default_rng(3)
    # more chains than features: random non-negative combinations of the real rows
    X = rng.gamma(1.0, 1.0, (400, len(F))) @ F
    w_true = np.zeros(ordercost.NFEAT)
    used = np.flatnonzero(X.sum(axis=0) > 0)
    w_true[used] = rng.uniform(0.5, 5.0, len(used))
    y = X @ w_true
    w, st = ordercost.fit(X, y)
    assert st["r2_time"] > 0.999999
    assert np.allclose(X @ w, y, rtol=1e-6)
    assert np.all(w >= 0)


def test_makespan_list_scheduling():
    cost = np.array([5.0, 4.0, 3.0, 3.0, 2.0, 2.0, 2.0])
    # longest first: {5, 2}, {4, 2, 2}, {3, 3} -> 8; shortest first ends with the 5 on a group at 5 -> 10
    assert ordercost.makespan(cost, np.arange(7), 3) == 8.0
    assert ordercost.makespan(cost, np.arange(7)[::-1], 3) == 10.0
