"""The lane discipline of the decoder, checked on the host (CPU only).

On the GPU a chain is decoded by a group of lanes that run the decoder's
serial code redundantly and split its independent loops; nothing keeps those
lanes in lockstep between two __syncwarp barriers.  The decoder is therefore
correct only if no stretch of code between two barriers depends on the order
in which the lanes' memory accesses interleave: serial stretches that update
group memory in place run on the group's first lane (lead stretches), and the
lane-split loops touch disjoint elements.

libcuopus_lanesim.so is the decoder built for the host with every lane a fiber
of its own (cuopus_b200/csrc/lanesim.cpp).  Two schedules:

* barrier-only: each lane runs a whole stretch before the next one starts,
  and a detector reports every byte of the decoder slot that a later lane
  rewrote after an earlier lane had already changed it (a lane computing from
  what another lane has overwritten);
* random: the running lane is switched out at random function entries (the
  fixed-point helpers included) after runs of 1..max_run entries.

Every chain must match libopus 1.5.2 fixed point (the golden fixtures made by
the reference's own decoder, or the oracle for fresh streams): per-packet
sample counts, final ranges, stop status and every int16 sample.  Before its
serial stretches were made lead stretches, the decoder (whose lanes then all
updated group memory in place, relying on lockstep execution) failed both
schedules at two lanes.
"""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import corpus, ogg_port, ref_decode

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "cuopus_b200", "lib", "libcuopus_lanesim.so")
GOLD = os.path.join(ROOT, "tests", "golden")
with open(os.path.join(GOLD, "decode.json")) as _f:
    DECODE = json.load(_f)
with open(os.path.join(GOLD, "index.json")) as _f:
    INDEX = json.load(_f)


@pytest.fixture(scope="module")
def ls():
    if not os.path.exists(LIB):
        pytest.fail("libcuopus_lanesim.so must be built (python -m cuopus_b200.build)")
    lib = ctypes.CDLL(LIB)
    lib.ls_decode_chains.restype = ctypes.c_longlong
    lib.ls_decode_chains.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int] + [ctypes.c_void_p] * 8 + \
        [ctypes.c_int] * 4 + [ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong)]
    return lib


def lane_decode(lib, packets, chains, ch, width, max_run, seed, fec=0, detect=0):
    """Decode chains with `width` fiber lanes; returns (per chain (pcm, nsamp,
    rng, stop), lane switches, hazards)."""
    blob, off, lens = ref_decode.flatten(packets)
    n = len(chains)
    first = np.array([c[0] for c in chains], np.uint32)
    npk = np.array([c[1] for c in chains], np.uint32)
    chans = np.full(n, ch, np.int32)
    cap = np.array([sum(ogg_port.decode_capacity48(packets[int(first[i]) + k]) for k in range(int(npk[i])))
                    for i in range(n)], np.uint64)
    pcm_off = np.zeros(n, np.uint64)
    pcm_off[1:] = np.cumsum(cap[:-1] * ch)
    pcm = np.zeros(int(cap.sum()) * ch + 1, np.int16)
    rec = np.zeros(n, np.uint64)
    rec[1:] = np.cumsum(npk[:-1])
    ns = np.zeros(int(npk.sum()) + 1, np.uint32)
    rg = np.zeros_like(ns)
    res = np.zeros(4 * n, np.uint32)
    hz = ctypes.c_ulonglong(0)
    P = lambda a: ctypes.c_void_p(a.ctypes.data)
    sw = lib.ls_decode_chains(P(blob), P(off), P(lens), P(first), P(npk), P(chans), n, P(pcm), P(pcm_off), None,
                              None, P(rec), P(ns), P(rg), P(res), 4, fec, width, max_run, seed, detect,
                              ctypes.byref(hz))
    assert sw >= 0
    res = res.reshape(-1, 4)
    out = []
    for i in range(n):
        r0, k = int(rec[i]), int(npk[i])
        p0 = int(pcm_off[i])
        out.append((pcm[p0:p0 + int(res[i, 1]) * ch], ns[r0:r0 + k], rg[r0:r0 + k], int(np.int32(res[i, 0]))))
    return out, sw, hz.value


def _golden(name):
    with open(os.path.join(GOLD, "streams", name + ".opus"), "rb") as f:
        ix = ogg_port.demux(f.read())
    return ix, [tuple(c) for c in INDEX[name]["chains_1_250"]]


def _check_golden(name, got):
    for i, g in enumerate(DECODE[name]):
        pcm, ns, rg, stop = got[i]
        assert stop == g["status"], (name, i)
        assert [int(v) for v in ns] == g["nsamp"], (name, i)
        assert [int(v) for v in rg] == g["rng"], (name, i)
        assert hashlib.sha256(pcm.astype("<i2").tobytes()).hexdigest() == g["pcm_sha256"], (name, i)


@pytest.mark.parametrize("name", sorted(DECODE))
def test_no_stretch_depends_on_lane_order(ls, name):
    """Barrier-only schedule, two lanes, the hazard detector on: no hazard and
    libopus's output, for every golden stream (SILK, hybrid, CELT, mono and
    stereo, redundancy and mode transitions, code-3 packets)."""
    ix, chains = _golden(name)
    for seed in (1,):
        got, sw, hz = lane_decode(ls, ix["packets"], chains, ix["channels"], 2, 0, seed, detect=1)
        assert hz == 0, "%s: %d stretches depend on the lanes' order" % (name, hz)
        _check_golden(name, got)


@pytest.mark.parametrize("width,max_run", [(4, 3), (32, 8)])
def test_random_lane_interleavings(ls, width, max_run):
    """Random switches between the lanes inside every stretch, on the golden
    streams: libopus's output at 4 and 32 lanes per chain."""
    names = ["mixed_stereo_a", "mixed_mono_a", "mixed_mono_b", "long_hybrid", "code3_120ms", "plain_a",
             "short_stereo_300ms"]
    if width == 32:
        names = names[:3]
    for name in names:
        ix, chains = _golden(name)
        got, sw, _ = lane_decode(ls, ix["packets"], chains, ix["channels"], width, max_run, 7 + width)
        assert sw > 1000
        _check_golden(name, got)


def _lossy(packets, seed, p_lost, p_dtx):
    rng = np.random.default_rng(seed)
    out = []
    for p in packets:
        u = rng.random()
        if u < p_lost:
            out.append(b"")
        elif u < p_lost + p_dtx and (p[0] & 3) == 0:
            out.append(p[:1])
        else:
            out.append(p)
    return out


def test_loss_paths_under_random_interleavings(ls):
    """Lost and DTX packets (SILK PLC / CNG, CELT concealment, the
    transitions around them), in-band FEC, and chains ending in random
    packets, decoded with four lanes under random switching, against the
    oracle."""
    try:
        corpus.ref_lib()
    except OSError as e:
        pytest.fail(str(e))
    for seed in range(4):
        spec = dict(kind="mixed", seed=83000 + seed, seconds=2.0, channels=1 + seed % 2)
        if seed % 2 == 0:
            spec.update(inband_fec=1, loss_perc=20, dtx=1)
        ix = ogg_port.demux(corpus.make_stream(spec))
        pk = _lossy(ix["packets"], seed, 0.1, 0.05)
        for fec in (0, 1):
            ref = ref_decode.decode_chains(pk, [(0, len(pk))], ix["channels"], fec=fec)
            got, _, _ = lane_decode(ls, pk, [(0, len(pk))], ix["channels"], 4, 3, 100 + seed, fec=fec)
            pcm, ns, rg, stop = got[0]
            assert stop == int(ref["status"][0])
            assert np.array_equal(ns, ref["nsamp"][0]) and np.array_equal(rg, ref["rng"][0]), (seed, fec)
            assert np.array_equal(pcm, ref["pcm"][0]), (seed, fec)
    rng = np.random.default_rng(84)
    good = ogg_port.demux(corpus.make_stream(dict(kind="mixed", seed=83100, seconds=1.0, channels=2)))["packets"]
    pk, chains = [], []
    for k in range(60):
        n_good = int(rng.integers(0, 4))
        chains.append((len(pk), n_good + 1))
        pk += good[:n_good]
        pk.append(rng.integers(0, 256, int(rng.integers(1, 400)), dtype=np.uint8).tobytes())
    ref = ref_decode.decode_chains(pk, chains, 2)
    got, _, _ = lane_decode(ls, pk, chains, 2, 4, 3, 5)
    for c, (pcm, ns, rg, stop) in enumerate(got):
        assert stop == int(ref["status"][c]), c
        assert np.array_equal(ns, ref["nsamp"][c]) and np.array_equal(rg, ref["rng"][c]), c
        assert np.array_equal(pcm, ref["pcm"][c]), c
