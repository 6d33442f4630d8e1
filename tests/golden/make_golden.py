"""Generate the golden fixtures of the CPU tests (run once, in a checkout that
has the reference tree; the fixtures are committed and nothing reads the
reference at test time).

    python tests/golden/make_golden.py <reference source tree>

What it writes (all small):
  streams/*.opus    seeded synthetic Ogg Opus streams from the vendored libopus
                    encoder (oracle/corpus.py): SILK wideband speech, mixed
                    SILK / hybrid / CELT mono and stereo, hybrid/SILK long-form,
                    and edge cases (shorter than the preroll, one packet,
                    120 ms code-3 packets)
  index.json        the reference's own Python indexer (ogg_index.py:
                    build_index, build_chains2) on every stream: channels,
                    preskip, playable samples, packet lengths, per-packet
                    48 kHz offsets and the chain tables at 1 s / 250 ms and
                    0.5 s / 80 ms
  decode.json       libopus 1.5.2 fixed point (oracle/_ref, compiled from the
                    reference's vendored sources) on every 1 s / 250 ms chain:
                    per-packet sample counts and final ranges, the stop status
                    and a SHA-256 of the chain's int16 PCM
  resample.npz      the reference's torch resampler (gpu_resample.py:
                    resample_48k_to_16k) on seeded int16 vectors and on the
                    decoded PCM of one stream (first second): inputs and float32
                    outputs
  rangedec.json     the reference's range-decoder gate schedule
                    (schedule.inc:18-36) and a wider schedule, run through
                    libopus celt/entdec.c on seeded byte buffers
"""
from __future__ import annotations

import ctypes
import hashlib
import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import corpus, ref_decode  # noqa: E402

STREAMS = [
    # name, spec
    ("plain_a", dict(kind="plain", seed=101, seconds=2.0, channels=1)),
    ("plain_b", dict(kind="plain", seed=102, seconds=3.3, channels=1)),
    ("mixed_mono_a", dict(kind="mixed", seed=201, seconds=4.0, channels=1)),
    ("mixed_mono_b", dict(kind="mixed", seed=202, seconds=5.5, channels=1)),
    ("mixed_stereo_a", dict(kind="mixed", seed=301, seconds=4.0, channels=2)),
    ("mixed_stereo_b", dict(kind="mixed", seed=302, seconds=6.2, channels=2)),
    ("long_hybrid", dict(kind="long", seed=401, seconds=7.0, channels=1)),
    ("short_100ms", dict(kind="mixed", seed=501, seconds=0.1, channels=1)),
    ("short_stereo_300ms", dict(kind="mixed", seed=502, seconds=0.3, channels=2)),
]


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def one_packet_stream():
    """A stream of a single 20 ms CELT packet (the smallest legal stream)."""
    x = corpus.to_i16(corpus.synth("chord", 960, np.random.default_rng(7)))
    pk, pre = corpus.encode(x, 1, [corpus.Seg(0, corpus.MODE_CELT, corpus.BW_FB, 960, 64000)])
    n = max(1, 960 - pre)
    while len(pk) > 1:       # keep the first packet; trim the stream to what it covers
        pk.pop()
    return corpus.mux_ogg(pk, pre, 1, n)


def code3_stream():
    """SILK 60 ms frames packed two per packet (code-3, 120 ms packets)."""
    rng = np.random.default_rng(8)
    n = 48000 * 2
    x = corpus.to_i16(corpus.synth("speech", n, rng))
    pk, pre = corpus.encode(x, 1, [corpus.Seg(0, corpus.MODE_SILK, corpus.BW_WB, 2880, 20000)],
                            corpus.APP_VOIP)
    merged = []
    for i in range(0, len(pk) - 1, 2):
        a, b = pk[i], pk[i + 1]
        if (a[0] >> 2) != (b[0] >> 2):
            merged += [a, b]
            continue
        # code 3, CBR off: frame count 2, VBR flag set, first frame length coded
        toc = (a[0] & 0xFC) | 3
        la = len(a) - 1
        lenb = bytes([la]) if la < 252 else bytes([252 + (la - 252) % 4, (la - 252 - (la - 252) % 4) // 4])
        merged.append(bytes([toc, 0x80 | 2]) + lenb + a[1:] + b[1:])
    if len(pk) % 2:
        merged.append(pk[-1])
    total = sum(corpus.toc_samples48(p) for p in merged)
    return corpus.mux_ogg(merged, pre, 1, min(n, total - pre))


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference source tree>")
    ref_root = sys.argv[1]
    ogg_index = _load("ref_ogg_index", os.path.join(ref_root, "ogg_index.py"))
    gpu_resample = _load("ref_gpu_resample", os.path.join(ref_root, "gpu_resample.py"))
    import torch

    sdir = os.path.join(HERE, "streams")
    os.makedirs(sdir, exist_ok=True)
    streams = [(n, corpus.make_stream(s)) for n, s in STREAMS]
    streams.append(("one_packet", one_packet_stream()))
    streams.append(("code3_120ms", code3_stream()))
    index, decode = {}, {}
    for name, data in streams:
        path = os.path.join(sdir, name + ".opus")
        with open(path, "wb") as f:
            f.write(data)
        ix = ogg_index.build_index(path, check_crc=True)
        ent = dict(channels=ix["channels"], preskip=ix["preskip"], pcm_samples_48k=ix["pcm_samples_48k"],
                   n_packets=len(ix["audio_packets"]), packet_len=[len(p) for p in ix["audio_packets"]],
                   sample_off=ix["sample_off"], toc_total=ix["toc_total_samples"],
                   granule_checked=ix["granule_checked"], granule_match=ix["granule_match"],
                   crc_bad=ix["crc_bad"],
                   packets_sha256=hashlib.sha256(b"".join(ix["audio_packets"])).hexdigest())
        for seg, pre in ((1.0, 250), (0.5, 80)):
            try:
                ent["chains_%g_%d" % (seg, pre)] = [list(c) for c in ogg_index.build_chains2(ix, seg, pre)]
            except (ValueError, AssertionError) as e:
                ent["chains_%g_%d" % (seg, pre)] = "error: %s" % e
        index[name] = ent
        chains = ent["chains_1_250"]
        if isinstance(chains, list):
            r = ref_decode.decode_chains(ix["audio_packets"], chains, ix["channels"])
            decode[name] = [dict(status=int(r["status"][i]), samples=int(r["samples"][i]),
                                 nsamp=[int(v) for v in r["nsamp"][i]], rng=[int(v) for v in r["rng"][i]],
                                 pcm_sha256=hashlib.sha256(r["pcm"][i].astype("<i2").tobytes()).hexdigest())
                            for i in range(len(chains))]
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=0, sort_keys=True)
    with open(os.path.join(HERE, "decode.json"), "w") as f:
        json.dump(decode, f, indent=0, sort_keys=True)

    # resampler vectors: seeded noise, a full-scale square wave, silence with
    # clicks, and the decoded playable PCM of one stream
    rng = np.random.default_rng(99)
    vecs = {
        "noise": (rng.standard_normal(9001) * 6000).clip(-32768, 32767).astype(np.int16),
        "square": np.where((np.arange(6000) // 37) % 2 == 0, 32767, -32768).astype(np.int16),
        "clicks": np.zeros(3000, np.int16),
        "tiny": np.array([5, -7, 32767], np.int16),
    }
    vecs["clicks"][::501] = 30000
    from oracle import pipeline
    pcm, ch, _ = pipeline.i16(dict(streams)["plain_b"])
    vecs["decoded_plain_b"] = pcm[:48000]
    out = {}
    for k, v in vecs.items():
        out["in_" + k] = v
        out["out_" + k] = gpu_resample.resample_48k_to_16k(torch.from_numpy(v.copy())).numpy()
    np.savez_compressed(os.path.join(HERE, "resample.npz"), **out)

    # range decoder schedules
    lib = corpus.ref_lib()
    rng = np.random.default_rng(4242)
    cases = []
    bufs = [bytes(rng.integers(0, 256, int(n)).astype(np.uint8)) for n in rng.integers(1, 160, 40)]
    bufs += [b"", b"\x00" * 8, b"\xff" * 8, b"\x80"]
    bufs += [p for p in ogg_index.build_index(os.path.join(sdir, "mixed_stereo_a.opus"))["audio_packets"][:8]]
    for b in bufs:
        arr = np.frombuffer(b + b"\0", np.uint8)
        o1 = np.zeros(147, np.uint32)
        o2 = np.zeros(163, np.uint32)
        lib.oref_ec_schedule(ctypes.c_void_p(arr.ctypes.data), len(b), ctypes.c_void_p(o1.ctypes.data))
        lib.oref_ec_schedule2(ctypes.c_void_p(arr.ctypes.data), len(b), ctypes.c_void_p(o2.ctypes.data))
        cases.append(dict(buf=b.hex(), gate=[int(x) for x in o1], wide=[int(x) for x in o2]))
    with open(os.path.join(HERE, "rangedec.json"), "w") as f:
        json.dump(cases, f)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
