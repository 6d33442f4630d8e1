"""Host-side parity (CPU only): the product's host code and the decoder's
host same-source build against the golden fixtures and the oracle.

* the C++ demuxer and chain builder of libcuopus.so (cuopus_index,
  cuopus_probe, cuopus_probe_pcm) against the reference indexer's tables,
  including its error returns on damaged input;
* the decoder sources compiled for the host (libcuopus_hostcheck.so, one lane
  per chain) against libopus: the range-decoder gate schedules and whole
  chains (per-packet sample counts, final ranges, every int16 sample).  This
  is the reference's "host same-source gate" (harness_host.cpp): it separates
  "the restatement is right" from "the CUDA execution is right".
"""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import corpus, ogg_port, ref_decode

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
HOSTCHECK = os.path.join(ROOT, "cuopus_b200", "lib", "libcuopus_hostcheck.so")

with open(os.path.join(GOLD, "index.json")) as _f:
    INDEX = json.load(_f)
with open(os.path.join(GOLD, "decode.json")) as _f:
    DECODE = json.load(_f)


def _stream(name):
    with open(os.path.join(GOLD, "streams", name + ".opus"), "rb") as f:
        return f.read()


@pytest.fixture(scope="module")
def cn():
    from cuopus_b200 import cuopus_native
    try:
        cuopus_native.lib()
    except OSError as e:
        pytest.fail("libcuopus.so must be built (python -m cuopus_b200.build): %s" % e)
    return cuopus_native


@pytest.fixture(scope="module")
def hc():
    if not os.path.exists(HOSTCHECK):
        pytest.fail("libcuopus_hostcheck.so must be built (python -m cuopus_b200.build)")
    return ctypes.CDLL(HOSTCHECK)


# ------------------------------------------------------------------ demuxer

@pytest.mark.parametrize("name", sorted(INDEX))
def test_cxx_demuxer_matches_reference_indexer(cn, name):
    g = INDEX[name]
    data = _stream(name)
    for seg, pre, key in ((1.0, 250.0, "chains_1_250"), (0.5, 80.0, "chains_0.5_80")):
        ix = cn.index(data, seg_s=seg, preroll_ms=pre)
        assert ix.channels == g["channels"]
        assert ix.play48 == g["pcm_samples_48k"]
        assert [int(v) for v in ix.pkt_len] == g["packet_len"]
        assert hashlib.sha256(ix.blob.tobytes()).hexdigest() == g["packets_sha256"]
        chains = [[int(a), int(b), int(c), int(d)] for a, b, c, d in zip(ix.first, ix.npkts, ix.trim, ix.keep)]
        assert chains == g[key]


@pytest.mark.parametrize("name", sorted(INDEX))
def test_probe_lengths(cn, name):
    g = INDEX[name]
    data = _stream(name)
    play, ch = cn.probe_pcm(data)
    assert (play, ch) == (g["pcm_samples_48k"], g["channels"])
    if g["channels"] == 1:
        assert cn.probe(data) == max(0, (g["pcm_samples_48k"] - 48) // 3)
    else:
        with pytest.raises(cn.CuopusError) as e:
            cn.probe(data)
        assert e.value.rc == 1


def test_probe_errors(cn):
    data = _stream("plain_a")
    with pytest.raises(cn.CuopusError) as e:      # not Ogg at all
        cn.probe(b"\x00" * 100)
    assert e.value.rc == 1
    with pytest.raises(cn.CuopusError) as e:      # OpusHead page only
        cn.probe(data[:60])
    assert e.value.rc == 1
    bad = bytearray(data)                         # wrong magic in the header packet
    i = bad.find(b"OpusHead")
    bad[i:i + 8] = b"OpusHexd"
    with pytest.raises(cn.CuopusError) as e:
        cn.probe(bytes(bad))
    assert e.value.rc == 1
    lib = cn.lib()                                # NULL output pointer: caller error
    err = ctypes.create_string_buffer(64)
    assert lib.cuopus_probe(data, len(data), None, err, 64) == 3
    assert err.value
    n16 = ctypes.c_int64(0)                       # NULL errbuf is tolerated
    assert lib.cuopus_probe(data, len(data), ctypes.byref(n16), None, 0) == 0
    assert n16.value == (INDEX["plain_a"]["pcm_samples_48k"] - 48) // 3


def test_granule_mismatch_is_rejected(cn):
    """A page granule that disagrees with the TOC durations fails the
    cross-check (reference cuopus_demux.h:216-262)."""
    data = bytearray(_stream("mixed_mono_b"))
    pages = []
    p = data.find(b"OggS")
    while p >= 0:
        pages.append(p)
        p = data.find(b"OggS", p + 4)
    mid = pages[len(pages) // 2]
    g = int.from_bytes(data[mid + 6:mid + 14], "little")
    data[mid + 6:mid + 14] = (g + 480).to_bytes(8, "little")
    with pytest.raises(cn.CuopusError) as e:
        cn.probe_pcm(bytes(data))
    assert e.value.rc == 1


def test_granule_warn_policy_resyncs(cn, monkeypatch):
    """CUOPUS_GRANULE=warn accepts the damaged granule and keeps the playable
    length the packets and the (legal) final granule give."""
    data = bytearray(_stream("mixed_mono_b"))
    pages = []
    p = data.find(b"OggS")
    while p >= 0:
        pages.append(p)
        p = data.find(b"OggS", p + 4)
    mid = pages[len(pages) // 2]
    g = int.from_bytes(data[mid + 6:mid + 14], "little")
    data[mid + 6:mid + 14] = (g + 480).to_bytes(8, "little")
    monkeypatch.setenv("CUOPUS_GRANULE", "warn")
    play, ch = cn.probe_pcm(bytes(data))
    assert (play, ch) == (INDEX["mixed_mono_b"]["pcm_samples_48k"], 1)
    ix = cn.index(bytes(data))
    chains = [[int(a), int(b), int(c), int(d)] for a, b, c, d in zip(ix.first, ix.npkts, ix.trim, ix.keep)]
    assert chains == INDEX["mixed_mono_b"]["chains_1_250"]


def test_page_crc_check(cn, monkeypatch):
    """CUOPUS_OGG_CRC=1 verifies every page checksum (RFC 3533)."""
    data = _stream("plain_b")
    assert cn.probe_pcm(data)[0] == INDEX["plain_b"]["pcm_samples_48k"]
    monkeypatch.setenv("CUOPUS_OGG_CRC", "1")
    assert cn.probe_pcm(data)[0] == INDEX["plain_b"]["pcm_samples_48k"]   # the corpus muxer writes valid CRCs
    bad = bytearray(data)
    bad[len(bad) // 2] ^= 0x40                                             # one payload bit
    with pytest.raises(cn.CuopusError) as e:
        cn.probe_pcm(bytes(bad))
    assert e.value.rc == 1 and "CRC" in str(e.value)
    monkeypatch.delenv("CUOPUS_OGG_CRC")
    cn.probe_pcm(bytes(bad))                                               # not checked by default


# ------------------------------------------------------------------ host same-source decoder

def _mutate(rng, data):
    """One seeded damage of an Ogg stream: a truncation, byte flips, a page's
    granule, lacing value, segment count or presence changed, or the OpusHead
    channel / preskip bytes rewritten."""
    b = bytearray(data)
    pages = [i for i in range(len(b) - 3) if b[i:i + 4] == b"OggS"]
    pg = pages[int(rng.integers(0, len(pages)))]
    kind = int(rng.integers(0, 9))
    if kind == 0:
        return bytes(b[:int(rng.integers(0, len(b)))])
    if kind == 1:
        for i in rng.integers(0, len(b), int(rng.integers(1, 9))):
            b[i] ^= 1 << int(rng.integers(0, 8))
    elif kind == 2:
        g = int.from_bytes(b[pg + 6:pg + 14], "little", signed=True)
        g = int(rng.choice([-1, 0, g + int(rng.integers(-960, 961)), int(rng.integers(0, 1 << 40))]))
        b[pg + 6:pg + 14] = g.to_bytes(8, "little", signed=True)
    elif kind == 3 and b[pg + 26]:
        b[pg + 27 + int(rng.integers(0, b[pg + 26]))] = int(rng.choice([0, 255, int(rng.integers(0, 256))]))
    elif kind == 4:
        b[pg + 26] = int(rng.integers(0, 256))
    elif kind == 5:
        nxt = [p for p in pages if p > pg]
        end = nxt[0] if nxt else len(b)
        del b[pg:end]
    elif kind == 6:
        nxt = [p for p in pages if p > pg]
        end = nxt[0] if nxt else len(b)
        b[pg:pg] = b[pg:end]
    elif kind == 7:
        h = b.find(b"OpusHead")
        b[h + 9] = int(rng.integers(0, 4))
    else:
        h = b.find(b"OpusHead")
        b[h + 10:h + 12] = int(rng.integers(0, 65536)).to_bytes(2, "little")
    return bytes(b)


def _port_index(data, seg, pre):
    try:
        ix = ogg_port.demux(data)
        if ix["channels"] not in (1, 2) or ix["granule_match"] != ix["granule_checked"]:
            return None
        return ix, ogg_port.build_chains(ix, seg, pre)
    except ogg_port.DemuxError:
        return None


def test_demuxer_on_damaged_streams_agrees_with_the_port(cn, monkeypatch):
    """1,500 seeded damages of the golden streams (truncations, bit flips,
    granules, lacing values, segment counts, dropped and repeated pages,
    OpusHead channel / preskip bytes): the C++ demuxer and the oracle's port of
    the reference indexer (ogg_index.py:75-367) refuse the same streams, with
    rc 1 and nothing else, and give identical packets, lengths and chain tables
    for the rest."""
    monkeypatch.delenv("CUOPUS_OGG_CRC", raising=False)
    monkeypatch.delenv("CUOPUS_GRANULE", raising=False)
    rng = np.random.default_rng(67)
    names = sorted(INDEX)
    accepted = refused = 0
    for trial in range(1500):
        data = _mutate(rng, _stream(names[trial % len(names)]))
        seg, pre = (1.0, 250.0) if trial % 2 else (0.5, 80.0)
        want = _port_index(data, seg, pre)
        try:
            got = cn.index(data, seg_s=seg, preroll_ms=pre)
        except cn.CuopusError as e:
            assert e.rc == 1, (trial, e)
            got = None
        assert (want is None) == (got is None), (trial, want is None, str(got))
        if got is None:
            refused += 1
            continue
        accepted += 1
        ix, chains = want
        assert got.channels == ix["channels"] and got.play48 == ix["play48"], trial
        assert [int(v) for v in got.pkt_len] == [len(p) for p in ix["packets"]], trial
        assert got.blob.tobytes() == b"".join(ix["packets"]), trial
        assert [tuple(int(v) for v in c) for c in zip(got.first, got.npkts, got.trim, got.keep)] == chains, trial
    assert accepted > 200 and refused > 200, (accepted, refused)


def test_header_only_stream_with_a_granule_is_refused(cn):
    """Two header packets and no audio, the header page carrying a granule past
    the preskip: playable samples without packets.  Refused with rc 1 (the
    reference's chain builder reads past its prefix sums here)."""
    data = bytearray(_stream("plain_a"))
    pages = [i for i in range(len(data) - 3) if data[i:i + 4] == b"OggS"]
    head = data[:pages[2]]                       # OpusHead page + OpusTags page
    head[6:14] = (100000).to_bytes(8, "little")
    with pytest.raises(ogg_port.DemuxError):
        _ = ogg_port.build_chains(ogg_port.demux(bytes(head)), 1.0, 250.0)
    with pytest.raises(cn.CuopusError) as e:
        cn.index(bytes(head))
    assert e.value.rc == 1 and "no audio packets" in str(e.value)


def test_range_decoder_gate_schedules(hc):
    with open(os.path.join(GOLD, "rangedec.json")) as f:
        cases = json.load(f)
    for case in cases:
        b = bytes.fromhex(case["buf"])
        arr = np.frombuffer(b + b"\0", np.uint8)
        o1 = np.zeros(147, np.uint32)
        o2 = np.zeros(163, np.uint32)
        hc.hc_ec_schedule(ctypes.c_void_p(arr.ctypes.data), len(b), ctypes.c_void_p(o1.ctypes.data))
        hc.hc_ec_schedule2(ctypes.c_void_p(arr.ctypes.data), len(b), ctypes.c_void_p(o2.ctypes.data))
        assert [int(x) for x in o1] == case["gate"]
        assert [int(x) for x in o2] == case["wide"]


def host_decode(hc, packets, chains, ch, nthreads=4, fec=0):
    """Decode chains with the host build; returns per chain (pcm, nsamp, rng, stop, samples)."""
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
    P = lambda a: ctypes.c_void_p(a.ctypes.data)
    hc.hc_decode_chains_fec(P(blob), P(off), P(lens), P(first), P(npk), P(chans), n, P(pcm), P(pcm_off), None,
                            None, P(rec), P(ns), P(rg), P(res), nthreads, fec)
    res = res.reshape(-1, 4)
    out = []
    for i in range(n):
        r0, k = int(rec[i]), int(npk[i])
        p0 = int(pcm_off[i])
        out.append((pcm[p0:p0 + int(res[i, 1]) * ch], ns[r0:r0 + k], rg[r0:r0 + k], int(np.int32(res[i, 0])),
                    int(res[i, 1])))
    return out


@pytest.mark.parametrize("name", sorted(DECODE))
def test_host_decoder_matches_golden_libopus(hc, name):
    ix = ogg_port.demux(_stream(name))
    chains = [tuple(c) for c in INDEX[name]["chains_1_250"]]
    got = host_decode(hc, ix["packets"], chains, ix["channels"])
    for i, g in enumerate(DECODE[name]):
        pcm, ns, rg, stop, samples = got[i]
        assert stop == g["status"] and samples == g["samples"], (name, i)
        assert [int(v) for v in ns] == g["nsamp"], (name, i)
        assert [int(v) for v in rg] == g["rng"], (name, i)
        assert hashlib.sha256(pcm.astype("<i2").tobytes()).hexdigest() == g["pcm_sha256"], (name, i)


@pytest.mark.parametrize("name", sorted(DECODE))
def test_lane_loops_are_order_independent(name):
    """The decoder built with every lane-split loop running backwards still
    matches libopus: no iteration of such a loop reads what another writes,
    which is what lets the GPU lanes run them in any order."""
    rev = os.path.join(ROOT, "cuopus_b200", "lib", "libcuopus_hostcheck_rev.so")
    if not os.path.exists(rev):
        pytest.fail("libcuopus_hostcheck_rev.so must be built (python -m cuopus_b200.build)")
    lib = ctypes.CDLL(rev)
    ix = ogg_port.demux(_stream(name))
    chains = [tuple(c) for c in INDEX[name]["chains_1_250"]]
    got = host_decode(lib, ix["packets"], chains, ix["channels"])
    for i, g in enumerate(DECODE[name]):
        pcm, ns, rg, stop, samples = got[i]
        assert [int(v) for v in rg] == g["rng"], (name, i)
        assert hashlib.sha256(pcm.astype("<i2").tobytes()).hexdigest() == g["pcm_sha256"], (name, i)


@pytest.mark.parametrize("seed", [11, 12, 13, 14])
def test_host_decoder_matches_libopus_mixed(hc, seed):
    """Fresh seeded streams (SILK/hybrid/CELT, 2.5-60 ms, mono/stereo),
    compared sample by sample with libopus."""
    try:
        corpus.ref_lib()
    except OSError as e:
        pytest.skip(str(e))
    d = corpus.make_stream(dict(kind="mixed", seed=seed, seconds=3.0, channels=1 + seed % 2))
    ix = ogg_port.demux(d)
    chains = ogg_port.build_chains(ix, 1.0, 250.0)
    ref = ref_decode.decode_chains(ix["packets"], chains, ix["channels"])
    got = host_decode(hc, ix["packets"], chains, ix["channels"])
    for i in range(len(chains)):
        pcm, ns, rg, stop, _ = got[i]
        assert stop == int(ref["status"][i]) == 0
        assert np.array_equal(ns, ref["nsamp"][i]) and np.array_equal(rg, ref["rng"][i])
        assert np.array_equal(pcm, ref["pcm"][i])


def test_host_decoder_damaged_packets_match_libopus(hc):
    """Truncated and bit-flipped packets: the decoder returns the same status,
    sample counts and samples as libopus (errors stop the chain)."""
    try:
        corpus.ref_lib()
    except OSError as e:
        pytest.skip(str(e))
    rng = np.random.default_rng(5)
    ix = ogg_port.demux(_stream("mixed_stereo_a"))
    pk = list(ix["packets"])
    for i in range(0, len(pk), 7):
        p = bytearray(pk[i])
        if i % 3 == 0 and len(p) > 3:
            p = p[: len(p) // 2]
        elif len(p) > 2:
            j = int(rng.integers(1, len(p)))
            p[j] ^= 1 << int(rng.integers(0, 8))
        pk[i] = bytes(p)
    chains = [(0, len(pk))]
    ref = ref_decode.decode_chains(pk, chains, ix["channels"])
    got = host_decode(hc, pk, chains, ix["channels"])
    pcm, ns, rg, stop, samples = got[0]
    assert stop == int(ref["status"][0])
    assert np.array_equal(ns, ref["nsamp"][0]) and np.array_equal(rg, ref["rng"][0])
    assert np.array_equal(pcm, ref["pcm"][0])


def _lossy(packets, seed, p_lost, p_dtx):
    """Packets with some replaced by an empty packet (lost: concealment) and
    some cut to their TOC byte (a DTX frame)."""
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


@pytest.mark.parametrize("seed", [21, 22, 23, 24])
def test_host_decoder_concealment_matches_libopus(hc, seed):
    """Lost and DTX packets in SILK, hybrid and CELT streams, mono and stereo:
    SILK PLC / CNG, CELT PLC (pitch search, LPC, IIR) and the transition
    frames around them match libopus sample for sample."""
    try:
        corpus.ref_lib()
    except OSError as e:
        pytest.skip(str(e))
    d = corpus.make_stream(dict(kind="mixed", seed=seed, seconds=4.0, channels=1 + seed % 2))
    ix = ogg_port.demux(d)
    pk = _lossy(ix["packets"], seed, 0.12, 0.08)
    assert any(len(p) == 0 for p in pk) and any(len(p) == 1 for p in pk)
    chains = [(0, len(pk))] + [(i, min(20, len(pk) - i)) for i in range(0, len(pk), 20)]
    ref = ref_decode.decode_chains(pk, chains, ix["channels"])
    got = host_decode(hc, pk, chains, ix["channels"])
    for i in range(len(chains)):
        pcm, ns, rg, stop, _ = got[i]
        assert stop == int(ref["status"][i]), i
        assert np.array_equal(ns, ref["nsamp"][i]) and np.array_equal(rg, ref["rng"][i]), i
        assert np.array_equal(pcm, ref["pcm"][i]), i


@pytest.mark.parametrize("seed,channels", [(42, 2), (44, 2), (45, 1), (48, 1), (49, 1)])
def test_host_decoder_inband_fec_matches_libopus(hc, seed, channels):
    """Streams encoded with in-band FEC (LBRR) and DTX, packets lost at random:
    with FEC on, a lost packet is rebuilt from the next packet's LBRR frames
    (opus_decode(next, 5760, decode_fec = 1)); every sample, count and final
    range matches libopus, and FEC changes the output of some lost packets."""
    try:
        corpus.ref_lib()
    except OSError as e:
        pytest.skip(str(e))
    d = corpus.make_stream(dict(kind="mixed", seed=seed, seconds=5.0, channels=channels, inband_fec=1,
                                loss_perc=25, dtx=1))
    ix = ogg_port.demux(d)
    pk = _lossy(ix["packets"], seed, 0.15, 0.0)
    chains = [(0, len(pk))] + [(i, min(25, len(pk) - i)) for i in range(0, len(pk), 25)]
    ref = ref_decode.decode_chains(pk, chains, ix["channels"], fec=1)
    ref0 = ref_decode.decode_chains(pk, chains[:1], ix["channels"], fec=0)
    assert not np.array_equal(ref["pcm"][0], ref0["pcm"][0]), "no packet used its FEC data"
    got = host_decode(hc, pk, chains, ix["channels"], fec=1)
    for i in range(len(chains)):
        pcm, ns, rg, stop, _ = got[i]
        assert stop == int(ref["status"][i]), i
        assert np.array_equal(ns, ref["nsamp"][i]) and np.array_equal(rg, ref["rng"][i]), i
        assert np.array_equal(pcm, ref["pcm"][i]), i


def test_parallel_demux_reports_like_the_sequential_one(cn, monkeypatch):
    """CUOPUS_DEMUX_THREADS: the file entry points demux on several host
    threads and still report the lowest-numbered bad file, with the same code
    and message as on the calling thread alone (no GPU needed: the demux comes
    first)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the pre-GPU part of the call on a machine without a GPU")
    lib = cn.lib()
    good = [_stream(n) for n in ("mixed_stereo_a", "mixed_mono_b", "plain_b", "long_hybrid")]
    bad = b"OggS" + b"\x07" * 200
    files = [good[0], good[1], bad, good[2], bad, good[3]]
    n = len(files)
    ba = (ctypes.c_char_p * n)(*files)
    la = (ctypes.c_size_t * n)(*[len(f) for f in files])
    outs = (ctypes.c_void_p * n)()
    caps = (ctypes.c_size_t * n)()
    lens = (ctypes.c_int64 * n)()
    chans = (ctypes.c_int32 * n)()
    seen = set()
    for threads in ("1", "4", "16"):
        monkeypatch.setenv("CUOPUS_DEMUX_THREADS", threads)
        err = ctypes.create_string_buffer(512)
        rc = lib.cuopus_decode_i16_multi(ba, la, n, outs, caps, lens, chans, None, err, 512)
        assert rc == 1
        seen.add(err.value)
    assert len(seen) == 1 and next(iter(seen)).startswith(b"file 2:")


def _pvq_v(n, k):
    """Number of integer vectors of length n with magnitudes summing to k."""
    from math import comb
    return sum((1 << j) * comb(n, j) * comb(k - 1, j - 1) for j in range(1, min(n, k) + 1))


def test_pvq_codewords_match_libopus(hc):
    """CELT PVQ codewords (celt/cwrs.c): random pulse vectors, encoded by
    libopus's encode_pulses, decode to the same vector through libopus's
    decode_pulses and through the decoder's cwrsi (host build), over band
    sizes 2-176 and pulse counts up to 30 within the codeword tables."""
    lib = corpus.ref_lib()
    lib.oref_pvq_roundtrip.restype = ctypes.c_int
    rng = np.random.default_rng(17)
    # (n, k) pairs whose codebook size fits 32 bits and lies inside the U table
    # rows the decoder indexes (min(n, k + 1) <= 5 with n <= 160, or small n and k)
    pairs = []
    for n in list(range(2, 33)) + [40, 48, 64, 72, 88, 96, 128, 144, 160, 176]:
        for k in range(1, 31):
            if _pvq_v(n, k) >= 1 << 32:
                continue
            r = min(n, k + 1)
            if (r <= 5 and max(n, k + 1) < 170) or (r <= 10 and max(n, k + 1) <= 20):
                pairs.append((n, k))
    checked = 0
    buf = (ctypes.c_ubyte * 64)()
    for n, k in pairs:
        for _ in range(3):
            y = np.zeros(n, np.int32)
            for _ in range(k):
                y[int(rng.integers(0, n))] += 1
            y *= np.where(rng.random(n) < 0.5, -1, 1).astype(np.int32)
            yin = np.ascontiguousarray(y, np.int32)
            yref = np.zeros(n, np.int32)
            assert lib.oref_pvq_roundtrip(n, k, yin.ctypes.data_as(ctypes.c_void_p), buf, 64,
                                          yref.ctypes.data_as(ctypes.c_void_p)) == 0
            assert np.array_equal(yref, yin), (n, k)
            got = np.zeros(n, np.int32)
            hc.hc_pvq_decode(buf, 64, n, k, got.ctypes.data_as(ctypes.c_void_p))
            assert np.array_equal(got, yin), (n, k, yin, got)
            checked += 1
    assert checked > 600


def test_imdct_matches_libopus(hc):
    """The decoder's inverse MDCT against libopus's clt_mdct_backward_c of the
    48 kHz mode: every block size (shift 0-3) and the short-block strides,
    random coefficients, random overlap history; every output word equal."""
    lib = corpus.ref_lib()
    lib.oref_imdct.restype = ctypes.c_int
    rng = np.random.default_rng(23)
    n_mdct, overlap = 1920, 120
    checked = 0
    # the decoder's calls: long blocks of every size (shift 3 - LM, stride 1)
    # and the short blocks of transient frames (shift 3, stride 1 << LM)
    for shift, stride in [(0, 1), (1, 1), (2, 1), (3, 1), (3, 2), (3, 4), (3, 8)]:
        for trial in range(12):
            scale = 1 << int(rng.integers(8, 22))
            x = rng.integers(-scale, scale, n_mdct, dtype=np.int64).astype(np.int32)
            hist = rng.integers(-scale, scale, overlap, dtype=np.int64).astype(np.int32)
            want = np.zeros(n_mdct + overlap, np.int32)
            want[:overlap] = hist
            got = want.copy()
            assert lib.oref_imdct(x.ctypes.data_as(ctypes.c_void_p), want.ctypes.data_as(ctypes.c_void_p),
                                  shift, stride) == 0
            hc.hc_imdct(x.ctypes.data_as(ctypes.c_void_p), got.ctypes.data_as(ctypes.c_void_p), shift, stride)
            assert np.array_equal(got, want), (shift, stride, trial)
            checked += 1
    assert checked == 7 * 12


def test_nlsf2a_matches_libopus(hc):
    """SILK NLSF to LPC (silk/NLSF2A.c, with its bandwidth-expansion loop for
    unstable filters) on random increasing NLSF vectors of order 10 and 16."""
    lib = corpus.ref_lib()
    rng = np.random.default_rng(29)
    for trial in range(400):
        d = 16 if trial % 2 else 10
        gap = int(rng.integers(1, 400))
        v = np.sort(rng.integers(1, 32767 - gap * d, d)) + gap * np.arange(1, d + 1)
        nlsf = np.ascontiguousarray(np.clip(v, 1, 32766).astype(np.int16))
        want = np.zeros(d, np.int16)
        got = np.zeros(d, np.int16)
        lib.oref_nlsf2a(want.ctypes.data_as(ctypes.c_void_p), nlsf.ctypes.data_as(ctypes.c_void_p), d)
        hc.hc_nlsf2a(got.ctypes.data_as(ctypes.c_void_p), nlsf.ctypes.data_as(ctypes.c_void_p), d)
        assert np.array_equal(got, want), (trial, nlsf)


@pytest.mark.parametrize("fs_in", [8000, 12000, 16000])
def test_silk_resampler_matches_libopus(hc, fs_in):
    """The SILK decoder's resampler to 48 kHz (silk/resampler.c, IIR_FIR: up2
    all-pass + fractional FIR) over a stream fed frame by frame: 10 and 20 ms
    frames of noise, tones and full-scale steps, every output sample equal."""
    lib = corpus.ref_lib()
    rng = np.random.default_rng(fs_in)
    n = fs_in * 2
    t = np.arange(n)
    x = (8000 * np.sin(2 * np.pi * 440 * t / fs_in) + rng.normal(0, 3000, n)).astype(np.int64)
    x[n // 3:n // 3 + 50] = 32767
    x[n // 2:n // 2 + 50] = -32768
    x = np.ascontiguousarray(np.clip(x, -32768, 32767).astype(np.int16))
    for ms in (10, 20):
        frame = fs_in * ms // 1000
        want = np.zeros(n * (48000 // fs_in), np.int16)
        got = np.zeros_like(want)
        a = lib.oref_silk_resample(fs_in, x.ctypes.data_as(ctypes.c_void_p), n, frame,
                                   want.ctypes.data_as(ctypes.c_void_p))
        b = hc.hc_silk_resample(fs_in, x.ctypes.data_as(ctypes.c_void_p), n, frame,
                                got.ctypes.data_as(ctypes.c_void_p))
        assert a == b > 0
        assert np.array_equal(got, want), (fs_in, ms)


@pytest.mark.parametrize("lanes", [0, 1])
def test_comb_filter_matches_libopus(hc, lanes):
    """The CELT comb (post-)filter (celt/celt.c comb_filter, in place, the
    decoder's use) in the serial form and in the block-parallel form: random
    pitch periods 15-1022 across the cross-fade, gains and tapsets, 2.5-20 ms."""
    lib = corpus.ref_lib()
    rng = np.random.default_rng(31 + lanes)
    off = 1100
    for trial in range(300):
        N = int(rng.choice([120, 240, 480, 960]))
        T0, T1 = (int(v) for v in rng.integers(15, 1023, 2))
        g0, g1 = (int(3072 * v) for v in rng.integers(0, 9, 2))
        t0, t1 = (int(v) for v in rng.integers(0, 3, 2))
        buf = rng.integers(-1 << 22, 1 << 22, off + N, dtype=np.int64).astype(np.int32)
        want = np.ascontiguousarray(buf.copy())
        got = np.ascontiguousarray(buf.copy())
        assert lib.oref_comb_filter(want.ctypes.data_as(ctypes.c_void_p), off, T0, T1, N, g0, g1, t0, t1) == 0
        hc.hc_comb_filter(got.ctypes.data_as(ctypes.c_void_p), off, T0, T1, N, g0, g1, t0, t1, lanes)
        assert np.array_equal(got, want), (trial, N, T0, T1, g0, g1, t0, t1)


def test_celt_allocation_matches_libopus(hc):
    """CELT bit allocation (celt/rate.c clt_compute_allocation in decode mode,
    caps from init_caps): random budgets, trims, dynalloc boosts, band ranges
    (CELT and hybrid), mono and stereo, every frame size; the decisions it
    reads from the range decoder come from random bytes.  Coded bands,
    intensity, dual stereo, balance, pulses, fine bits and priorities, and the
    range decoder's state after it all equal."""
    lib = corpus.ref_lib()
    rng = np.random.default_rng(37)
    out_w = np.zeros(4 + 63 + 2, np.int32)
    out_g = np.zeros_like(out_w)
    for trial in range(1500):
        start = 17 if trial % 4 == 0 else 0
        end = int(rng.choice([13, 17, 19, 21])) if start == 0 else int(rng.choice([19, 21]))
        C, LM = 1 + int(rng.integers(0, 2)), int(rng.integers(0, 4))
        trim = int(rng.integers(0, 11))
        total = int(rng.integers(0, 8 * 8 * 300))
        offsets = np.zeros(21, np.int32)
        for i in rng.integers(start, end, int(rng.integers(0, 4))):
            offsets[i] = int(rng.integers(1, 4)) * 8 * C
        buf = (ctypes.c_ubyte * 160)(*rng.integers(0, 256, 160).tolist())
        args = (buf, 160, start, end, offsets.ctypes.data_as(ctypes.c_void_p), trim, total, C, LM)
        assert lib.oref_alloc(*args, out_w.ctypes.data_as(ctypes.c_void_p)) == 0
        hc.hc_alloc(*args, out_g.ctypes.data_as(ctypes.c_void_p))
        assert np.array_equal(out_g, out_w), (trial, start, end, C, LM, trim, total)


def test_celt_band_decoding_matches_libopus(hc):
    """CELT band shapes (celt/bands.c quant_all_bands, decode mode, after the
    allocation, on one range decoder over random bytes): PVQ codewords, theta
    splits, folding and noise fill, stereo (intensity, dual, mid/side merge,
    phase inversion on or off), transient short blocks with time-frequency
    changes, every spread.  Every coefficient, collapse mask, the folding seed
    and the range decoder's state equal."""
    lib = corpus.ref_lib()
    rng = np.random.default_rng(41)
    for trial in range(1200):
        start = 17 if trial % 5 == 0 else 0
        end = int(rng.choice([13, 17, 19, 21])) if start == 0 else int(rng.choice([19, 21]))
        C, LM = 1 + int(rng.integers(0, 2)), int(rng.integers(0, 4))
        transient = LM > 0 and rng.random() < 0.3
        shortBlocks = (1 << LM) if transient else 0
        tf = np.zeros(21, np.int32)
        if LM > 0 and rng.random() < 0.5:
            tf[:] = rng.choice([0, 1] if transient else [0, -1], 21)
        offsets = np.zeros(21, np.int32)
        for i in rng.integers(start, end, int(rng.integers(0, 4))):
            offsets[i] = int(rng.integers(1, 4)) * 8 * C
        nbytes = int(rng.integers(8, 200))
        buf = (ctypes.c_ubyte * nbytes)(*rng.integers(0, 256, nbytes).tolist())
        spread, trim, inv = int(rng.integers(0, 4)), int(rng.integers(0, 11)), int(rng.integers(0, 2))
        seed = int(rng.integers(0, 1 << 32))
        outs = []
        for f in (lib.oref_bands, hc.hc_bands):
            X = np.zeros(2 * 960, np.int16)
            cm = np.zeros(42, np.uint8)
            tail = np.zeros(3, np.uint32)
            f(buf, nbytes, start, end, offsets.ctypes.data_as(ctypes.c_void_p), trim, C, LM, shortBlocks, spread,
              tf.ctypes.data_as(ctypes.c_void_p), inv, ctypes.c_uint32(seed), X.ctypes.data_as(ctypes.c_void_p),
              cm.ctypes.data_as(ctypes.c_void_p), tail.ctypes.data_as(ctypes.c_void_p))
            outs.append((X, cm, tail))
        (Xw, cw, tw), (Xg, cg, tg) = outs
        assert np.array_equal(Xg, Xw) and np.array_equal(cg, cw) and np.array_equal(tg, tw), \
            (trial, start, end, C, LM, shortBlocks, spread, trim, inv)


def test_celt_energy_decoding_matches_libopus(hc):
    """CELT band energies (celt/quant_bands.c): coarse energy (Laplace-coded,
    intra and inter prediction, every frame size), the allocation, fine energy
    and the final bits, on random bytes from random previous energies, mono and
    stereo; the energies and the range decoder's state equal."""
    lib = corpus.ref_lib()
    rng = np.random.default_rng(43)
    for trial in range(1500):
        start = 17 if trial % 5 == 0 else 0
        end = int(rng.choice([13, 17, 19, 21])) if start == 0 else int(rng.choice([19, 21]))
        C, LM, intra = 1 + int(rng.integers(0, 2)), int(rng.integers(0, 4)), int(rng.integers(0, 2))
        offsets = np.zeros(21, np.int32)
        for i in rng.integers(start, end, int(rng.integers(0, 4))):
            offsets[i] = int(rng.integers(1, 4)) * 8 * C
        nbytes = int(rng.integers(4, 200))
        buf = (ctypes.c_ubyte * nbytes)(*rng.integers(0, 256, nbytes).tolist())
        old = rng.integers(-28 << 8, 20 << 8, 42).astype(np.int16)
        trim = int(rng.integers(0, 11))
        res = []
        for f in (lib.oref_energy, hc.hc_energy):
            e = np.ascontiguousarray(old.copy())
            tail = np.zeros(2, np.uint32)
            f(buf, nbytes, start, end, intra, offsets.ctypes.data_as(ctypes.c_void_p), trim, C, LM,
              e.ctypes.data_as(ctypes.c_void_p), tail.ctypes.data_as(ctypes.c_void_p))
            res.append((e, tail))
        assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1]), \
            (trial, start, end, C, LM, intra)


def test_silk_entropy_decoding_matches_libopus(hc):
    """SILK side information and excitation pulses (silk/decode_indices.c,
    decode_pulses.c with the shell coder and signs): every internal rate,
    10 and 20 ms frames, up to three frames per packet, voiced / unvoiced VAD
    flags, independent and conditional coding of the first frame, on random
    bytes.  Every index, every pulse and the range decoder's state equal."""
    lib = corpus.ref_lib()
    rng = np.random.default_rng(47)
    for trial in range(1500):
        fs = int(rng.choice([8, 12, 16]))
        nb_subfr = int(rng.choice([2, 4]))
        frames = 1 if nb_subfr == 2 else int(rng.integers(1, 4))
        vad = np.ascontiguousarray(rng.integers(0, 2, 3).astype(np.int32))
        cond = int(rng.integers(0, 2))
        nbytes = int(rng.integers(10, 250))
        buf = (ctypes.c_ubyte * nbytes)(*rng.integers(0, 256, nbytes).tolist())
        res = []
        for f in (lib.oref_silk_entropy, hc.hc_silk_entropy):
            out = np.zeros(3 * (33 + 320), np.int32)
            tail = np.zeros(2, np.uint32)
            n = f(buf, nbytes, fs, nb_subfr, frames, vad.ctypes.data_as(ctypes.c_void_p), cond,
                  out.ctypes.data_as(ctypes.c_void_p), tail.ctypes.data_as(ctypes.c_void_p))
            res.append((n, out, tail))
        assert res[0][0] == res[1][0] > 0
        assert np.array_equal(res[0][1], res[1][1]) and np.array_equal(res[0][2], res[1][2]), \
            (trial, fs, nb_subfr, frames, cond)


def test_silk_frames_match_libopus(hc):
    """Whole SILK frames at the internal rate (silk/decode_frame.c: indices,
    pulses, NLSF / LPC / pitch / LTP parameters, excitation, LTP and LPC
    synthesis, concealment of lost frames, comfort noise), state carried over
    eight frames decoded from random bytes, every rate and frame length.
    Every sample and the range decoder's state equal."""
    lib = corpus.ref_lib()
    rng = np.random.default_rng(53)
    for trial in range(400):
        fs = int(rng.choice([8, 12, 16]))
        nb_subfr = int(rng.choice([2, 4]))
        frames = 8
        vad = np.ascontiguousarray(rng.integers(0, 2, frames).astype(np.int32))
        lost = np.ascontiguousarray((rng.random(frames) < 0.15).astype(np.int32))
        lost[0] = 0
        nbytes = int(rng.integers(40, 600))
        buf = (ctypes.c_ubyte * nbytes)(*rng.integers(0, 256, nbytes).tolist())
        res = []
        for f in (lib.oref_silk_frames, hc.hc_silk_frames):
            out = np.zeros(frames * 320, np.int16)
            tail = np.zeros(2, np.uint32)
            n = f(buf, nbytes, fs, nb_subfr, frames, vad.ctypes.data_as(ctypes.c_void_p),
                  lost.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p),
                  tail.ctypes.data_as(ctypes.c_void_p))
            res.append((n, out, tail))
        assert res[0][0] == res[1][0] == frames * nb_subfr * 5 * fs
        assert np.array_equal(res[0][1], res[1][1]) and np.array_equal(res[0][2], res[1][2]), \
            (trial, fs, nb_subfr, vad, lost)


def test_celt_frames_match_libopus(hc):
    """Whole CELT frames (celt/celt_decoder.c celt_decode_with_ec from a fresh
    decoder: energies, allocation, band shapes, anti-collapse, IMDCT, post
    filter, deemphasis, and the concealment of lost frames), ten frames of
    random bytes per stream with the state carried over, every frame size,
    mono and stereo, every end band.  Every sample and final range equal."""
    lib = corpus.ref_lib()
    rng = np.random.default_rng(59)
    for trial in range(300):
        C, LM = 1 + int(rng.integers(0, 2)), int(rng.integers(0, 4))
        end = int(rng.choice([13, 17, 19, 21]))
        frames = 10
        lens = rng.integers(2, 160, frames).astype(np.uint32)
        lens[rng.random(frames) < 0.12] = 0
        lens[0] = max(int(lens[0]), 2)
        data = rng.integers(0, 256, int(lens.sum()) + 1).astype(np.uint8)
        res = []
        for f in (lib.oref_celt_frames, hc.hc_celt_frames):
            out = np.zeros(frames * (120 << LM) * C, np.int16)
            fr = np.zeros(frames, np.uint32)
            f(data.ctypes.data_as(ctypes.c_void_p), lens.ctypes.data_as(ctypes.c_void_p), frames, C, LM, end,
              out.ctypes.data_as(ctypes.c_void_p), fr.ctypes.data_as(ctypes.c_void_p))
            res.append((out, fr))
        assert np.array_equal(res[0][1], res[1][1]), (trial, C, LM, end, lens)
        assert np.array_equal(res[0][0], res[1][0]), (trial, C, LM, end, lens)


def _mathops_cases(rng):
    """(op, a, b, q) arrays over each helper's input domain: exhaustive where it
    is 16-bit or a short range, random draws plus the ends elsewhere."""
    i32 = lambda x: np.asarray(x, np.int64).astype(np.int32)
    rnd = lambda lo, hi, n: rng.integers(lo, hi, n, dtype=np.int64)
    pos = np.concatenate([np.arange(1, 1 << 17), rnd(1, 1 << 31, 1 << 17), [2**31 - 1]])
    cases = []
    cases.append((0, i32(np.concatenate([np.arange(1, 1 << 17), rnd(1, 1 << 32, 1 << 17), [2**32 - 1]]))))
    cases.append((1, i32(pos)))
    b = rnd(1, 1 << 31, 1 << 17)
    a = (rng.random(len(b)) * 2 - 1) * b
    cases.append((2, i32(a), i32(b)))
    cases.append((3, i32(np.arange(16384, 65536))))
    cases.append((4, i32(np.concatenate([[0], pos]))))
    cases.append((5, i32(np.arange(-(1 << 18), (1 << 18) + 1))))
    cases.append((6, i32(np.arange(-32768, 32768))))
    cases.append((7, i32(np.arange(-32768, 32768))))
    cases.append((8,))              # bitexact_log2tan: built from bitexact_cos in the test
    sgn = np.concatenate([pos, -pos[::7], [0]])
    cases.append((9, i32(sgn)))
    a = rnd(-(2**31 - 1), 2**31, 1 << 17)
    b = rnd(1, 2**31, 1 << 17) * rng.choice([-1, 1], 1 << 17)
    cases.append((10, i32(a), i32(b), i32(rnd(0, 31, 1 << 17))))
    cases.append((11, i32(b), None, i32(rnd(1, 62, 1 << 17))))
    cases.append((12, i32(np.arange(-256, 4300))))
    cases.append((13, i32(np.concatenate([np.arange(0, 1 << 17), rnd(1, 2**31, 1 << 17)]))))
    return cases, np.arange(0, 16385)


def test_fixed_point_helpers_match_libopus(hc):
    """The decoder's fixed-point helpers against libopus's own, elementwise over
    their input domains (celt/mathops.c isqrt32, celt_rcp, frac_div32,
    celt_rsqrt_norm, celt_sqrt, celt_cos_norm; celt/mathops.h celt_exp2;
    celt/bands.c:68-90 bitexact_cos, bitexact_log2tan; silk/Inlines.h:71-166
    silk_SQRT_APPROX, silk_DIV32_varQ, silk_INVERSE32_varQ; silk/log2lin.c,
    silk/lin2log.c).  Every output word equal."""
    lib = corpus.ref_lib()
    rng = np.random.default_rng(61)
    cases, theta = _mathops_cases(rng)

    def run(f, op, a, b=None, q=None):
        n = len(a)
        b = np.zeros(n, np.int32) if b is None else b
        q = np.zeros(n, np.int32) if q is None else q
        out = np.zeros(n, np.int32)
        vp = lambda x: x.ctypes.data_as(ctypes.c_void_p)
        assert f(op, vp(a), vp(b), vp(q), n, vp(out)) == 0
        return out

    for case in cases:
        op = case[0]
        if op == 8:
            # the decoder's own domain: the sine / cosine of every split angle
            c = run(lib.oref_mathops, 7, theta.astype(np.int32))
            s = run(lib.oref_mathops, 7, (16384 - theta).astype(np.int32))
            r1 = rng.integers(1, 32768, 1 << 16).astype(np.int32)
            r2 = rng.integers(1, 32768, 1 << 16).astype(np.int32)
            a, b, q = np.concatenate([s, r1]), np.concatenate([c, r2]), None
        else:
            a = case[1]
            b = case[2] if len(case) > 2 else None
            q = case[3] if len(case) > 3 else None
        want = run(lib.oref_mathops, op, a, b, q)
        got = run(hc.hc_mathops, op, a, b, q)
        bad = np.flatnonzero(want != got)
        assert bad.size == 0, (op, int(a[bad[0]]), None if b is None else int(b[bad[0]]), int(want[bad[0]]),
                               int(got[bad[0]]))
