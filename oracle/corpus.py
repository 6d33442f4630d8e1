"""Seeded synthetic OGG-Opus corpora for the parity tests and the benchmark.

TEST INFRASTRUCTURE.  Opus packets can only come from an Opus encoder, and the
only one here is the reference's vendored libopus 1.5.2 encoder built under
oracle/_ref (oracle/Makefile).  This module drives it through oref_encode
(oracle/ref_driver.c) and wraps the packets in Ogg pages with a muxer written
here (RFC 3533 pages, RFC 7845 OpusHead/OpusTags, pre-skip and end trim).  It
runs before any timing and never on the decode path.

Signals (all numpy, seeded):
  speech  glottal pulse train, pitch 80-250 Hz with vibrato, through 3-4
          formant resonators, syllable envelope, plus pink noise at -30 dB
  sweep   log sine sweep 50 Hz - 20 kHz
  noise   white or pink noise
  chord   3-5 harmonic notes

Workloads (the reference's corpora are private; these stand in for them with
the shapes, sizes and mode mixes they were described with):
  plain64     64 mono streams of 1 s, SILK wideband 20 ms 24 kbps VBR, complexity 10
  mixed       N streams (default 4096), log-uniform 1-30 s, per-segment
              (0.5-3 s) forced SILK / hybrid / CELT, frame 2.5-60 ms,
              6-128 kbps log-uniform, mono or stereo
  long        one mono stream (default 7200 s), hybrid / SILK alternating,
              32 kbps, 20 ms frames
  pareto      N streams with Pareto(1.5, 0.25 s) lengths capped at 120 s, mixed modes
"""
from __future__ import annotations

import ctypes
import hashlib
import math
import os
import struct
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libopus_ref.so")

MODE_SILK, MODE_HYBRID, MODE_CELT = 1000, 1001, 1002
OPUS_AUTO = -1000
BW_NB, BW_MB, BW_WB, BW_SWB, BW_FB = 1101, 1102, 1103, 1104, 1105
APP_VOIP, APP_AUDIO = 2048, 2049
SR = 48000


class OrefSeg(ctypes.Structure):
    _fields_ = [("start", ctypes.c_int64), ("mode", ctypes.c_int32),
                ("bandwidth", ctypes.c_int32), ("frame_size", ctypes.c_int32),
                ("bitrate", ctypes.c_int32), ("force_channels", ctypes.c_int32)]


_lib = None


def ref_lib():
    """Load oracle/_ref/libopus_ref.so (built by oracle/Makefile)."""
    global _lib
    if _lib is None:
        if not os.path.exists(REF_LIB):
            raise OSError("oracle/_ref/libopus_ref.so is missing: run make -C oracle REF=<reference tree>")
        lib = ctypes.CDLL(REF_LIB)
        lib.oref_encode.restype = ctypes.c_int
        lib.oref_encode.argtypes = [
            ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(OrefSeg),
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int,
            ctypes.POINTER(ctypes.c_int)]
        lib.oref_encode_opts.restype = ctypes.c_int
        lib.oref_encode_opts.argtypes = lib.oref_encode.argtypes + [ctypes.c_int] * 3
        lib.oref_decode_chains.restype = ctypes.c_int
        lib.oref_decode_chains.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_int, ctypes.c_int] + \
            [ctypes.c_void_p] * 7 + [ctypes.c_int]
        lib.oref_decode_chains_fec.restype = ctypes.c_int
        lib.oref_decode_chains_fec.argtypes = lib.oref_decode_chains.argtypes + [ctypes.c_int]
        lib.oref_version.restype = ctypes.c_char_p
        _lib = lib
    return _lib


# ---------------------------------------------------------------- signals

def _pink(rng, n):
    """Pink noise by 1/f spectral shaping of white noise (unit RMS)."""
    w = rng.standard_normal(n)
    spec = np.fft.rfft(w)
    f = np.arange(spec.size, dtype=np.float64)
    f[0] = 1.0
    spec /= np.sqrt(f)
    x = np.fft.irfft(spec, n)
    return x / (np.sqrt(np.mean(x * x)) + 1e-12)


def _resonator(x, f0, bw):
    """Two-pole resonator (formant) at f0 Hz with bandwidth bw Hz."""
    from scipy.signal import lfilter
    r = math.exp(-math.pi * bw / SR)
    a1 = -2 * r * math.cos(2 * math.pi * f0 / SR)
    a2 = r * r
    g = (1 - r) * math.sqrt(1 - 2 * r * math.cos(4 * math.pi * f0 / SR) + r * r)
    return lfilter([g], [1.0, a1, a2], x)


def synth(kind, n, rng):
    """One channel of n float samples in [-1, 1] of the given kind."""
    t = np.arange(n) / SR
    if kind == "speech":
        f0 = rng.uniform(80, 250)
        vib = 1 + 0.03 * np.sin(2 * np.pi * rng.uniform(3, 7) * t)
        phase = np.cumsum(f0 * vib / SR)
        pulses = np.zeros(n)
        idx = np.nonzero(np.diff(np.floor(phase)) > 0)[0]
        pulses[idx] = 1.0
        # glottal shaping: short decaying pulse
        k = np.exp(-np.arange(64) / 8.0)
        src = np.convolve(pulses, k)[:n]
        y = np.zeros(n)
        for f, bw in zip(sorted(rng.uniform([300, 900, 2000, 3000], [900, 2000, 3000, 4500])),
                         rng.uniform(60, 200, 4)):
            y += _resonator(src, f, bw)
        # syllables: 3-6 Hz envelope with pauses
        env = 0.5 * (1 + np.sin(2 * np.pi * rng.uniform(3, 6) * t + rng.uniform(0, 6.28)))
        env = np.clip(env * 1.4 - 0.2, 0, 1)
        y = y * env
        y /= np.max(np.abs(y)) + 1e-9
        y = 0.6 * y + 10 ** (-30 / 20) * 0.3 * _pink(rng, n)
    elif kind == "sweep":
        f1, f2 = 50.0, 20000.0
        dur = max(n / SR, 1e-3)
        k = math.log(f2 / f1)
        y = 0.5 * np.sin(2 * np.pi * f1 * dur / k * (np.exp(t / dur * k) - 1))
    elif kind == "white":
        y = 0.3 * rng.standard_normal(n)
    elif kind == "pink":
        y = 0.25 * _pink(rng, n)
    elif kind == "chord":
        y = np.zeros(n)
        nn = int(rng.integers(3, 6))
        base = rng.uniform(110, 440)
        for j in range(nn):
            f = base * 2 ** (rng.integers(0, 24) / 12)
            for h in range(1, 5):
                if f * h < 20000:
                    y += np.sin(2 * np.pi * f * h * t + rng.uniform(0, 6.28)) / (h * nn)
        y *= 0.5
    else:
        raise ValueError(kind)
    return np.clip(y, -1, 1)


def to_i16(x):
    return np.clip(np.round(x * 32767), -32768, 32767).astype(np.int16)


# ---------------------------------------------------------------- encode

@dataclass
class Seg:
    start: int          # first input sample of the segment
    mode: int
    bandwidth: int
    frame_size: int     # at 48 kHz
    bitrate: int
    force_channels: int = OPUS_AUTO


def encode(pcm_i16, channels, segs, application=APP_AUDIO, complexity=10, vbr=1, inband_fec=0, loss_perc=0,
           dtx=0):
    """Encode interleaved int16 pcm (n*channels) -> (list of packets, preskip).
    inband_fec / loss_perc / dtx: OPUS_SET_INBAND_FEC, OPUS_SET_PACKET_LOSS_PERC
    and OPUS_SET_DTX (all 0 for the corpora)."""
    lib = ref_lib()
    pcm = np.ascontiguousarray(pcm_i16, dtype=np.int16)
    n = pcm.size // channels
    arr = (OrefSeg * len(segs))(*[OrefSeg(s.start, s.mode, s.bandwidth, s.frame_size,
                                          s.bitrate, s.force_channels) for s in segs])
    max_pkts = n // 120 + 64
    cap = max_pkts * 1500 + 4096
    out = np.zeros(cap, dtype=np.uint8)
    lens = np.zeros(max_pkts, dtype=np.uint32)
    pre = ctypes.c_int(0)
    np_ = lib.oref_encode_opts(pcm.ctypes.data, n, channels, arr, len(segs), application,
                               complexity, vbr, out.ctypes.data, cap, lens.ctypes.data,
                               max_pkts, ctypes.byref(pre), inband_fec, loss_perc, dtx)
    if np_ < 0:
        raise RuntimeError("oref_encode failed: %d" % np_)
    pkts, w = [], 0
    for i in range(np_):
        L = int(lens[i])
        pkts.append(bytes(out[w:w + L]))
        w += L
    return pkts, pre.value


# ---------------------------------------------------------------- ogg mux

_CRC = []
for _i in range(256):
    _r = _i << 24
    for _ in range(8):
        _r = ((_r << 1) ^ 0x04C11DB7) & 0xFFFFFFFF if _r & 0x80000000 else (_r << 1) & 0xFFFFFFFF
    _CRC.append(_r)
_CRC = np.array(_CRC, dtype=np.uint32)


def ogg_crc(buf):
    r = 0
    for b in buf:
        r = ((r << 8) & 0xFFFFFFFF) ^ int(_CRC[((r >> 24) & 0xFF) ^ b])
    return r


def toc_samples48(pkt):
    """Samples at 48 kHz of one packet from its TOC byte (RFC 6716 sec. 3.1)."""
    if not pkt:
        return 0
    cfg, code = pkt[0] >> 3, pkt[0] & 3
    if cfg < 12:
        q = (10, 20, 40, 60)[cfg & 3] * 4
    elif cfg < 16:
        q = (10, 20)[cfg & 1] * 4
    else:
        q = (10, 20, 40, 80)[cfg & 3]
    nf = 1 if code == 0 else 2 if code < 3 else (pkt[1] & 0x3F if len(pkt) > 1 else 0)
    return q * 12 * nf


def _page(serial, seq, granule, flags, segs_payload):
    lacing, body = [], bytearray()
    for payload, complete in segs_payload:
        L = len(payload)
        lacing += [255] * (L // 255)
        if complete:
            lacing.append(L % 255)
        body += payload
    hdr = bytearray(b"OggS" + struct.pack("<BBqIIIB", 0, flags, granule, serial, seq, 0,
                                          len(lacing)) + bytes(lacing))
    page = hdr + body
    struct.pack_into("<I", page, 22, ogg_crc(page))
    return bytes(page)


def mux_ogg(packets, preskip, channels, n_play, serial=0x43550001, max_page_bytes=4000,
            max_page_packets=50):
    """Ogg Opus byte stream.  Granules are cumulative TOC sample counts; the last
    page carries preskip + n_play (end trim, RFC 7845 sec. 4.4)."""
    head = b"OpusHead" + struct.pack("<BBHIhB", 1, channels, preskip, 48000, 0, 0)
    tags = b"OpusTags" + struct.pack("<I", 10) + b"cuopus-syn" + struct.pack("<I", 0)
    out = [_page(serial, 0, 0, 0x02, [(head, True)]), _page(serial, 1, 0, 0, [(tags, True)])]
    seq, cum, i = 2, 0, 0
    end_gran = preskip + n_play
    while i < len(packets):
        group, size = [], 0
        while i < len(packets) and len(group) < max_page_packets and \
                (not group or size + len(packets[i]) <= max_page_bytes) and \
                sum((len(p) // 255 + 1) for p in group) + len(packets[i]) // 255 + 1 <= 255:
            group.append(packets[i])
            size += len(packets[i])
            cum += toc_samples48(packets[i])
            i += 1
        last = i >= len(packets)
        gran = min(cum, end_gran) if last else cum
        out.append(_page(serial, seq, gran, 0x04 if last else 0, [(p, True) for p in group]))
        seq += 1
    return b"".join(out)


# ---------------------------------------------------------------- workloads

_FS = {2.5: 120, 5: 240, 10: 480, 20: 960, 40: 1920, 60: 2880}


def _mixed_segments(rng, n, channels):
    """Per-segment forced mode / bandwidth / frame size / bitrate over n samples."""
    segs, pos = [], 0
    while pos < n:
        mode = int(rng.choice([MODE_SILK, MODE_HYBRID, MODE_CELT]))
        if mode == MODE_SILK:
            bw = int(rng.choice([BW_NB, BW_MB, BW_WB]))
            fms = float(rng.choice([10, 20, 40, 60]))
        elif mode == MODE_HYBRID:
            bw = int(rng.choice([BW_SWB, BW_FB]))
            fms = float(rng.choice([10, 20]))
        else:
            bw = int(rng.choice([BW_NB, BW_WB, BW_SWB, BW_FB]))
            fms = float(rng.choice([2.5, 5, 10, 20, 40, 60]))
        br = int(round(math.exp(rng.uniform(math.log(6000), math.log(128000)))))
        segs.append(Seg(pos, mode, bw, _FS[fms], br))
        pos += int(rng.uniform(0.5, 3.0) * SR)
    return segs


def _signal(rng, n, channels):
    kinds = ["speech", "sweep", "white", "pink", "chord"]
    kind = kinds[int(rng.integers(0, len(kinds)))]
    x = synth(kind, n, rng)
    if channels == 2:
        kind2 = kinds[int(rng.integers(0, len(kinds)))]
        x2 = 0.6 * x + 0.4 * synth(kind2, n, rng)
        return to_i16(np.stack([x, x2], axis=1).reshape(-1)), kind
    return to_i16(x), kind


def make_stream(spec):
    """Build one stream from a spec dict -> Ogg bytes.  Deterministic in spec."""
    rng = np.random.default_rng(spec["seed"])
    n = int(spec["seconds"] * SR)
    ch = spec["channels"]
    kind = spec["kind"]
    if kind == "plain":
        x = to_i16(synth("speech", n, rng))
        segs = [Seg(0, MODE_SILK, BW_WB, 960, 24000)]
        pkts, pre = encode(x, 1, segs, APP_VOIP, complexity=10, vbr=1)
    elif kind == "mixed":
        x, _ = _signal(rng, n, ch)
        segs = _mixed_segments(rng, n, ch)
        pkts, pre = encode(x, ch, segs, APP_AUDIO, complexity=spec.get("complexity", 5),
                           inband_fec=spec.get("inband_fec", 0), loss_perc=spec.get("loss_perc", 0),
                           dtx=spec.get("dtx", 0))
    elif kind == "long":
        x = to_i16(synth("speech", n, rng))
        segs, pos, j = [], 0, 0
        while pos < n:
            if j % 2 == 0:
                segs.append(Seg(pos, MODE_HYBRID, BW_SWB, 960, 32000))
            else:
                segs.append(Seg(pos, MODE_SILK, BW_WB, 960, 32000))
            pos += int(rng.uniform(2.0, 20.0) * SR)
            j += 1
        pkts, pre = encode(x, 1, segs, APP_AUDIO, complexity=spec.get("complexity", 5))
    else:
        raise ValueError(kind)
    return mux_ogg(pkts, pre, ch, n)


def workload_specs(name, seed=1234, count=None, seconds=None):
    """Stream specs (seeded) for a named workload."""
    rng = np.random.default_rng(seed)
    specs = []
    if name == "plain64":
        for i in range(count or 64):
            specs.append(dict(kind="plain", seed=seed * 1000003 + i, seconds=seconds or 1.0,
                              channels=1))
    elif name == "mixed":
        for i in range(count or 4096):
            L = float(math.exp(rng.uniform(math.log(1.0), math.log(seconds or 30.0))))
            specs.append(dict(kind="mixed", seed=seed * 1000003 + i, seconds=round(L, 3),
                              channels=int(rng.choice([1, 2]))))
    elif name == "long":
        specs.append(dict(kind="long", seed=seed, seconds=seconds or 7200.0, channels=1))
    elif name == "pareto":
        for i in range(count or 16384):
            L = 0.25 / (1.0 - rng.uniform(0, 1)) ** (1 / 1.5)
            L = min(L, seconds or 120.0)
            specs.append(dict(kind="mixed", seed=seed * 1000003 + i, seconds=round(L, 3),
                              channels=int(rng.choice([1, 2]))))
    elif name == "lognormal":
        # serving requests: log-normal lengths, median 30 s, sigma 1, clipped
        # to [5 s, seconds] (2 h for the serving workload; a draw that long is
        # rare, and encoding it takes minutes)
        for i in range(count or 256):
            L = float(np.clip(30.0 * math.exp(rng.normal(0.0, 1.0)), 5.0, seconds or 600.0))
            specs.append(dict(kind="mixed", seed=seed * 1000003 + i, seconds=round(L, 3),
                              channels=int(rng.choice([1, 2]))))
    else:
        raise ValueError(name)
    return specs


def _build_one(args):
    spec, path = args
    if not os.path.exists(path):
        data = make_stream(spec)
        tmp = path + ".tmp%d" % os.getpid()
        with open(tmp, "wb") as f:
            f.write(data)
        os.replace(tmp, path)
    return path


def build_corpus(name, root, seed=1234, count=None, seconds=None, workers=None):
    """Generate (or reuse) a cached corpus directory; returns the file paths."""
    specs = workload_specs(name, seed, count, seconds)
    key = hashlib.sha1(repr((name, specs)).encode()).hexdigest()[:12]
    d = os.path.join(root, "%s-%s" % (name, key))
    os.makedirs(d, exist_ok=True)
    jobs = [(s, os.path.join(d, "%05d.opus" % i)) for i, s in enumerate(specs)]
    todo = [j for j in jobs if not os.path.exists(j[1])]
    if todo:
        workers = workers or os.cpu_count() or 1
        if workers > 1 and len(todo) > 1:
            import multiprocessing as mp
            with mp.get_context("spawn").Pool(min(workers, len(todo))) as pool:
                for _ in pool.imap_unordered(_build_one, todo, chunksize=4):
                    pass
        else:
            for j in todo:
                _build_one(j)
    return [p for _, p in jobs]
