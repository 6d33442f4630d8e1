"""Two-phase decoding on the host build (CPU only): every packet decoded once on
its own from a fresh decoder, recording what the range decoder hands the
decoder (csrc/dec/rangedec.cuh, symbol log), then the chains decoded with the
range decoder replaying those records.  The chains must decode to libopus's
samples exactly: the golden streams (SILK, hybrid, CELT, mono and stereo,
redundancy and mode transitions, code-3 packets), spliced mode changes without
redundancy (the hybrid -> SILK silence frame, whose decode is never logged),
lost / DTX / FEC packets and damaged packets; a log too small for its packet
falls back to the normal decode of that packet.  The lane simulator replays
with 2, 4 and 32 lanes, where every lane keeps its own cursor over the log.
"""
import ctypes
import hashlib
import json
import os
import sys

import numpy as np
import pytest

from oracle import corpus, ogg_port, ref_decode

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from branches import spliced_chains  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOSTCHECK = os.path.join(ROOT, "cuopus_b200", "lib", "libcuopus_hostcheck.so")
LANESIM = os.path.join(ROOT, "cuopus_b200", "lib", "libcuopus_lanesim.so")
GOLD = os.path.join(ROOT, "tests", "golden")
with open(os.path.join(GOLD, "decode.json")) as _f:
    DECODE = json.load(_f)
with open(os.path.join(GOLD, "index.json")) as _f:
    INDEX = json.load(_f)
SYM_BAD = 0xFFFFFFFF
P = lambda a: ctypes.c_void_p(a.ctypes.data) if a is not None else None


@pytest.fixture(scope="module")
def hc():
    lib = ctypes.CDLL(HOSTCHECK)
    lib.hc_decode_chains_sym.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int] + [ctypes.c_void_p] * 8 + \
        [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    return lib


@pytest.fixture(scope="module")
def ls():
    lib = ctypes.CDLL(LANESIM)
    lib.ls_decode_chains_sym.restype = ctypes.c_longlong
    lib.ls_decode_chains_sym.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int] + [ctypes.c_void_p] * 8 + \
        [ctypes.c_int] * 4 + [ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong)] + \
        [ctypes.c_void_p] * 3 + [ctypes.c_int]
    return lib


class Tables:
    """Packets and chains in the decoder's table layout, with a symbol log of
    `per_packet` entries per packet."""

    def __init__(self, packets, chains, ch, per_packet=1 << 14):
        self.packets = packets
        self.blob, self.off, self.lens = ref_decode.flatten(packets)
        self.np = len(packets)
        self.ch = ch
        self.chains = chains
        self.sym_off = (np.arange(self.np + 1, dtype=np.uint64) * np.uint64(per_packet)).astype(np.uint64)
        self.sym = np.zeros(max(int(self.sym_off[-1]), 1), np.uint32)
        self.sym_len = np.zeros(max(self.np, 1), np.uint32)

    def record(self, hc):
        """Phase 1: each packet alone, from a fresh decoder, recording its log."""
        n = self.np
        first = np.arange(n, dtype=np.uint32)
        npk = np.ones(n, np.uint32)
        chans = np.full(n, self.ch, np.int32)
        res = np.zeros(4 * max(n, 1), np.uint32)
        hc.hc_decode_chains_sym(P(self.blob), P(self.off), P(self.lens), P(first), P(npk), P(chans), n, None, None,
                                None, None, None, None, None, P(res), 4, 0, P(self.sym), P(self.sym_off),
                                P(self.sym_len), 1)
        return res.reshape(-1, 4)

    def layout(self):
        n = len(self.chains)
        first = np.array([c[0] for c in self.chains], np.uint32)
        npk = np.array([c[1] for c in self.chains], np.uint32)
        cap = np.array([sum(ogg_port.decode_capacity48(self.packets[int(first[i]) + k]) for k in range(int(npk[i])))
                        for i in range(n)], np.uint64)
        pcm_off = np.zeros(n, np.uint64)
        pcm_off[1:] = np.cumsum(cap[:-1] * self.ch)
        rec = np.zeros(n, np.uint64)
        rec[1:] = np.cumsum(npk[:-1])
        return first, npk, cap, pcm_off, rec

    def _outputs(self, n, npk, pcm, pcm_off, rec, ns, rg, res):
        res = res.reshape(-1, 4)
        out = []
        for i in range(n):
            r0, k = int(rec[i]), int(npk[i])
            p0 = int(pcm_off[i])
            out.append((pcm[p0:p0 + int(res[i, 1]) * self.ch], ns[r0:r0 + k], rg[r0:r0 + k],
                        int(np.int32(res[i, 0]))))
        return out

    def replay(self, hc, fec=0, mode=2):
        """Phase 2 on the host build: the chains, replaying the logs."""
        first, npk, cap, pcm_off, rec = self.layout()
        n = len(self.chains)
        chans = np.full(n, self.ch, np.int32)
        pcm = np.zeros(int(cap.sum()) * self.ch + 1, np.int16)
        ns = np.zeros(int(npk.sum()) + 1, np.uint32)
        rg = np.zeros_like(ns)
        res = np.zeros(4 * n, np.uint32)
        hc.hc_decode_chains_sym(P(self.blob), P(self.off), P(self.lens), P(first), P(npk), P(chans), n, P(pcm),
                                P(pcm_off), None, None, P(rec), P(ns), P(rg), P(res), 4, fec, P(self.sym),
                                P(self.sym_off), P(self.sym_len), mode)
        return self._outputs(n, npk, pcm, pcm_off, rec, ns, rg, res)

    def replay_lanes(self, ls, width, max_run, seed, detect=0):
        """Phase 2 in the lane simulator (every lane a fiber)."""
        first, npk, cap, pcm_off, rec = self.layout()
        n = len(self.chains)
        chans = np.full(n, self.ch, np.int32)
        pcm = np.zeros(int(cap.sum()) * self.ch + 1, np.int16)
        ns = np.zeros(int(npk.sum()) + 1, np.uint32)
        rg = np.zeros_like(ns)
        res = np.zeros(4 * n, np.uint32)
        hz = ctypes.c_ulonglong(0)
        sw = ls.ls_decode_chains_sym(P(self.blob), P(self.off), P(self.lens), P(first), P(npk), P(chans), n, P(pcm),
                                     P(pcm_off), None, None, P(rec), P(ns), P(rg), P(res), 4, 0, width, max_run, seed,
                                     detect, ctypes.byref(hz), P(self.sym), P(self.sym_off), P(self.sym_len), 2)
        assert sw >= 0
        return self._outputs(n, npk, pcm, pcm_off, rec, ns, rg, res), hz.value


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


def _check_ref(got, ref):
    for c, (pcm, ns, rg, stop) in enumerate(got):
        assert stop == int(ref["status"][c]), c
        assert np.array_equal(ns, ref["nsamp"][c]) and np.array_equal(rg, ref["rng"][c]), c
        assert np.array_equal(pcm, ref["pcm"][c]), c


@pytest.mark.parametrize("name", sorted(DECODE))
def test_replayed_chains_match_golden(hc, name):
    """Every golden stream: the record pass logs every packet (none too large
    for its log, none failing) and the replayed chains decode to libopus's
    output."""
    ix, chains = _golden(name)
    t = Tables(ix["packets"], chains, ix["channels"])
    res = t.record(hc)
    used = t.sym_len[:t.np]
    assert np.all(used != SYM_BAD), name
    assert np.all(res[:, 0] == 0)
    assert used.max() < (1 << 14)
    _check_golden(name, t.replay(hc))


def test_replay_reads_the_log(hc):
    """Replaying a log whose entries were altered changes the decode: the
    chains really take the range decoder's values from the log."""
    ix, chains = _golden("mixed_mono_a")
    t = Tables(ix["packets"], chains, ix["channels"])
    t.record(hc)
    ok = t.replay(hc)
    for p in range(t.np):
        a = int(t.sym_off[p])
        t.sym[a:a + int(t.sym_len[p])] ^= 1
    bad = t.replay(hc)
    assert any(not np.array_equal(x[0], y[0]) or not np.array_equal(x[2], y[2]) for x, y in zip(ok, bad))


def test_overflowing_logs_fall_back_to_normal_decoding(hc):
    """With 150 entries per packet some logs overflow and are marked unusable;
    those packets decode normally, the rest replay, and the output stays
    libopus's."""
    ix, chains = _golden("mixed_stereo_a")
    t = Tables(ix["packets"], chains, ix["channels"], per_packet=150)
    t.record(hc)
    used = t.sym_len[:t.np]
    assert np.any(used == SYM_BAD) and np.any(used != SYM_BAD)
    _check_golden("mixed_stereo_a", t.replay(hc))


@pytest.mark.parametrize("channels", [1, 2])
def test_spliced_mode_changes_replay(hc, channels):
    """Mode changes without redundancy: CELT -> SILK / hybrid crossfades and
    the hybrid -> SILK silence frame, whose range decode depends on the
    previous packet and is never logged."""
    packets, chains = spliced_chains(channels)
    t = Tables(packets, chains, channels)
    t.record(hc)
    ref = ref_decode.decode_chains(packets, chains, channels)
    _check_ref(t.replay(hc), ref)


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


def test_loss_fec_and_damaged_packets_replay(hc):
    """Lost and DTX packets (nothing to log), in-band FEC (the FEC decode of
    the packet after a loss never uses the log; its normal decode does), and
    chains ending in random packets (a packet that fails to decode is marked
    unusable and fails again, normally, in its chain)."""
    try:
        corpus.ref_lib()
    except OSError as e:
        pytest.fail(str(e))
    for seed in range(4):
        spec = dict(kind="mixed", seed=87000 + seed, seconds=2.0, channels=1 + seed % 2)
        if seed % 2 == 0:
            spec.update(inband_fec=1, loss_perc=20, dtx=1)
        ix = ogg_port.demux(corpus.make_stream(spec))
        pk = _lossy(ix["packets"], seed, 0.1, 0.05)
        t = Tables(pk, [(0, len(pk))], ix["channels"])
        t.record(hc)
        for fec in (0, 1):
            ref = ref_decode.decode_chains(pk, [(0, len(pk))], ix["channels"], fec=fec)
            _check_ref(t.replay(hc, fec=fec), ref)
    rng = np.random.default_rng(88)
    good = ogg_port.demux(corpus.make_stream(dict(kind="mixed", seed=87100, seconds=1.0, channels=2)))["packets"]
    pk, chains = [], []
    for k in range(60):
        n_good = int(rng.integers(0, 4))
        chains.append((len(pk), n_good + 1))
        pk += good[:n_good]
        pk.append(rng.integers(0, 256, int(rng.integers(1, 400)), dtype=np.uint8).tobytes())
    t = Tables(pk, chains, 2)
    t.record(hc)
    assert np.any(t.sym_len[:t.np] == SYM_BAD)
    _check_ref(t.replay(hc), ref_decode.decode_chains(pk, chains, 2))


@pytest.mark.parametrize("name", ["mixed_stereo_a", "mixed_mono_b", "long_hybrid", "code3_120ms"])
def test_replay_lanes_barrier_only(hc, ls, name):
    """Two lanes, barrier-only schedule with the hazard detector: no stretch
    depends on the lanes' order and the replayed output is libopus's."""
    ix, chains = _golden(name)
    t = Tables(ix["packets"], chains, ix["channels"])
    t.record(hc)
    got, hz = t.replay_lanes(ls, 2, 0, 1, detect=1)
    assert hz == 0
    _check_golden(name, got)


@pytest.mark.parametrize("width,max_run", [(4, 3), (32, 8)])
def test_replay_lanes_random_interleavings(hc, ls, width, max_run):
    """Random switches between lanes inside every stretch: each lane's log
    cursor stays with the others' and the output is libopus's."""
    for name in ["mixed_stereo_a", "mixed_mono_a"]:
        ix, chains = _golden(name)
        t = Tables(ix["packets"], chains, ix["channels"])
        t.record(hc)
        got, _ = t.replay_lanes(ls, width, max_run, 11 + width)
        _check_golden(name, got)
