"""Pins of the oracle against the reference's own outputs (CPU only).

The golden fixtures under tests/golden were produced by
tests/golden/make_golden.py from the reference itself: its Python indexer
(ogg_index.py build_index / build_chains2), its torch resampler
(gpu_resample.py resample_48k_to_16k), its range-decoder gate schedule
(schedule.inc:18-36) through libopus celt/entdec.c, and libopus 1.5.2 fixed
point compiled from its vendored sources (oracle/_ref).  These tests check
that the oracle's CPU restatements reproduce them exactly, so that the GPU
parity tests, which compare against the oracle, compare against the
reference.
"""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import ogg_port, pipeline

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _json(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def _stream(name):
    with open(os.path.join(GOLD, "streams", name + ".opus"), "rb") as f:
        return f.read()


INDEX = _json("index.json")


@pytest.mark.parametrize("name", sorted(INDEX))
def test_demux_port_matches_reference_indexer(name):
    g = INDEX[name]
    ix = ogg_port.demux(_stream(name))
    assert ix["channels"] == g["channels"]
    assert ix["preskip"] == g["preskip"]
    assert ix["play48"] == g["pcm_samples_48k"]
    assert [len(p) for p in ix["packets"]] == g["packet_len"]
    assert hashlib.sha256(b"".join(ix["packets"])).hexdigest() == g["packets_sha256"]
    assert [ogg_port.toc_samples48(p) for p in ix["packets"]] == \
        list(np.diff(g["sample_off"] + [g["toc_total"]]))
    for seg, pre, key in ((1.0, 250.0, "chains_1_250"), (0.5, 80.0, "chains_0.5_80")):
        want = g[key]
        if isinstance(want, str):
            with pytest.raises(ogg_port.DemuxError):
                ogg_port.build_chains(ix, seg, pre)
        else:
            got = [list(c) for c in ogg_port.build_chains(ix, seg, pre)]
            assert got == want
            assert sum(c[3] for c in got) == g["pcm_samples_48k"]


def test_resample_port_matches_reference_torch():
    """The C restatement of the reference's fp32 resampler against the
    reference's torch twin (conv1d, stride 3, padding 24), run on the CPU.

    The reference kernel accumulates the 49 products in tap order with fused
    multiply-adds (cuopus_kernels.cuh:102-110); the port does the same.  Torch's
    CPU convolution keeps that order for some input lengths and not for others,
    so the twin agrees bit for bit on the decoded-speech vector and within a few
    fp32 ulps of full scale (2.5e-7) elsewhere.  Bit-exactness of the device
    kernel is checked on the GPU against the port."""
    z = np.load(os.path.join(GOLD, "resample.npz"))
    names = sorted(k[3:] for k in z.files if k.startswith("in_"))
    assert names
    for k in names:
        x, want = z["in_" + k], z["out_" + k]
        got = pipeline.resample(x, x.size // 3)
        assert got.dtype == np.float32 and got.shape == want.shape, k
        assert np.max(np.abs(got - want), initial=0.0) <= 2.5e-7, k
    for k in ("decoded_plain_b", "clicks", "tiny"):
        x, want = z["in_" + k], z["out_" + k]
        assert np.array_equal(pipeline.resample(x, x.size // 3), want), k


def test_resample_error_against_fp64_oracle():
    """Error of the fp32 resampler (float taps, fp32 accumulation) against the
    double-precision taps applied in double: |err| <= 4e-7 of full scale, under
    four fp32 ulps at 1.0 (measured: 1.3e-7 on noise and speech, 2.8e-7 on a
    full-scale square wave)."""
    z = np.load(os.path.join(GOLD, "resample.npz"))
    for k in ("noise", "square", "decoded_plain_b"):
        x = z["in_" + k]
        y32 = pipeline.resample(x, x.size // 3).astype(np.float64)
        y64 = pipeline.resample_f64(x, x.size // 3)
        assert np.max(np.abs(y32 - y64)) <= 4e-7, k


def test_resample_taps_are_the_reference_taps():
    """Kaiser beta 8.6, 49 taps, cutoff 1/3, unity DC gain, symmetric."""
    t = pipeline.taps()
    assert t.shape == (49,)
    assert abs(float(t.astype(np.float64).sum()) - 1.0) < 1e-6
    assert np.array_equal(t, t[::-1])
    assert int(np.argmax(t)) == 24


def _ref():
    from oracle.corpus import ref_lib
    try:
        return ref_lib()
    except OSError as e:
        pytest.skip(str(e))


def test_libopus_oracle_reproduces_golden_decode():
    """oracle/_ref (libopus 1.5.2 fixed point) decodes every golden chain to
    the recorded per-packet sample counts, final ranges and PCM."""
    _ref()
    from oracle import ref_decode
    gold = _json("decode.json")
    for name, chains_gold in sorted(gold.items()):
        ix = ogg_port.demux(_stream(name))
        chains = [tuple(c) for c in INDEX[name]["chains_1_250"]]
        r = ref_decode.decode_chains(ix["packets"], chains, ix["channels"])
        for i, cg in enumerate(chains_gold):
            assert int(r["status"][i]) == cg["status"]
            assert [int(v) for v in r["nsamp"][i]] == cg["nsamp"], (name, i)
            assert [int(v) for v in r["rng"][i]] == cg["rng"], (name, i)
            assert hashlib.sha256(r["pcm"][i].astype("<i2").tobytes()).hexdigest() == cg["pcm_sha256"]


def test_libopus_range_decoder_gate():
    lib = _ref()
    for case in _json("rangedec.json"):
        b = bytes.fromhex(case["buf"])
        arr = np.frombuffer(b + b"\0", np.uint8)
        o1 = np.zeros(147, np.uint32)
        o2 = np.zeros(163, np.uint32)
        lib.oref_ec_schedule(ctypes.c_void_p(arr.ctypes.data), len(b), ctypes.c_void_p(o1.ctypes.data))
        lib.oref_ec_schedule2(ctypes.c_void_p(arr.ctypes.data), len(b), ctypes.c_void_p(o2.ctypes.data))
        assert [int(x) for x in o1] == case["gate"]
        assert [int(x) for x in o2] == case["wide"]


def test_full_size_check_finds_planted_differences():
    """oref_check_chains, the full-size parity check the benchmark runs after
    its timed region: on a batch laid out as the decoder's chain table it must
    report nothing for libopus's own output, and exactly the differences
    planted into a copy of it (one sample, one final range, one sample count,
    one stop status)."""
    from oracle import ref_decode
    names = ["mixed_stereo_a", "mixed_mono_b", "long_hybrid", "code3_120ms"]
    data, off, lens, first, npk, chans, trim, keep, res, pcm, got_off = [], [], [], [], [], [], [], [], [], [], []
    base_p = base_b = base_o = 0
    for nm in names:
        ix = ogg_port.demux(_stream(nm))
        pk, ch = ix["packets"], ix["channels"]
        chains = ogg_port.build_chains(ix, 0.5, 250.0)
        ref = ref_decode.decode_chains(pk, chains, ch)
        for p in pk:
            off.append(base_b)
            lens.append(len(p))
            base_b += len(p)
        data.append(b"".join(pk))
        for i, (f, n, t, k) in enumerate(chains):
            first.append(f + base_p)
            npk.append(n)
            chans.append(ch)
            trim.append(t)
            keep.append(k)
            res.append([0, int(ref["samples"][i]), int(ref["rng"][i][-1]), 1])
            pcm.append(ref["pcm"][i][t * ch:(t + k) * ch])
            got_off.append(base_o)
            base_o += k * ch
        base_p += len(pk)
    blob = np.frombuffer(b"".join(data) + b"\0" * 16, np.uint8)
    got = np.concatenate(pcm)
    res = np.array(res, np.uint32)
    args = (blob, off, lens, first, npk, chans, trim, keep)
    r = ref_decode.check_batch(*args, got, got_off, res)
    assert len(first) > 20 and not r["bad"].any() and not r["flags"].any()
    got2, res2 = got.copy(), res.copy()
    got2[got_off[5] + 3] ^= 1
    res2[7, 2] ^= 0x100
    res2[9, 1] += 1
    res2[11, 0] = np.uint32(0xFFFFFFFC)   # -4, OPUS_INVALID_PACKET
    r = ref_decode.check_batch(*args, got2, got_off, res2)
    assert np.flatnonzero(r["bad"]).tolist() == [5] and int(r["bad"][5]) == 1
    assert {int(i): int(r["flags"][i]) for i in np.flatnonzero(r["flags"])} == {7: 4, 9: 2, 11: 1}
