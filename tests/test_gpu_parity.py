"""GPU parity: libcuopus against libopus 1.5.2 fixed point (the oracle).

Every chain is checked for per-packet sample counts, the final range after
every packet and every int16 sample (bit-exact), on seeded synthetic streams
made by the vendored encoder: SILK-only wideband speech, and mixed streams
with forced SILK / hybrid / CELT segments, 2.5-60 ms frames, 6-128 kbps,
mono and stereo.  The f16k path must match the CPU pipeline (libopus decode +
the resampler restatement) with max abs diff 0.
"""
import numpy as np
import pytest

from oracle import corpus, ogg_port, pipeline, ref_decode

pytestmark = pytest.mark.gpu


def _streams(kind, n, seconds, seed0):
    out = []
    for s in range(n):
        ch = 1 if kind == "plain" else 1 + (s % 2)
        out.append(corpus.make_stream(dict(kind=kind, seed=seed0 + s, seconds=seconds, channels=ch)))
    return out


def _check(gpu_chains, packets, chains, ch, whole):
    ref = ref_decode.decode_chains(packets, chains, ch)
    for i, g in enumerate(gpu_chains):
        assert g["stop"] == ref["status"][i] == 0
        assert np.array_equal(g["nsamp"], ref["nsamp"][i]), "chain %d nsamp" % i
        assert np.array_equal(g["rng"], ref["rng"][i]), "chain %d final range" % i
        trim, keep = chains[i][2], chains[i][3]
        want = ref["pcm"][i] if whole else ref["pcm"][i][trim * ch:(trim + keep) * ch]
        assert g["pcm"].shape == want.shape, "chain %d length" % i
        bad = np.nonzero(g["pcm"] != want)[0]
        assert bad.size == 0, "chain %d: %d samples differ, first at %d" % (i, bad.size, bad[0])


def test_plain_silk_whole_chains(cuda):
    from gpu_util import run_batch
    streams = _streams("plain", 8, 1.0, 5000)
    idx = [ogg_port.demux(d) for d in streams]
    pk = [ix["packets"] for ix in idx]
    ch = [(0, len(p), 0, 1 << 40) for p in pk]
    res, _ = run_batch(pk, [[c] for c in ch], [1] * len(pk), width=32)
    for s in range(len(pk)):
        _check([res[s]], pk[s], [(0, len(pk[s]), 0, res[s]["keep"])], 1, True)


@pytest.mark.parametrize("width,schedule", [(32, 0), (32, 1), (16, 1), (8, 0), (4, 1), (1, 0)])
def test_mixed_segmented_chains(cuda, width, schedule):
    from gpu_util import run_batch
    streams = _streams("mixed", 4, 4.0, 6000 + width)
    idx = [ogg_port.demux(d) for d in streams]
    pk = [ix["packets"] for ix in idx]
    chs = [ogg_port.build_chains(ix, 1.0, 250.0) for ix in idx]
    nch = [ix["channels"] for ix in idx]
    order = None
    total = sum(len(c) for c in chs)
    if schedule == 1:
        order = list(range(total))[::-1]
    res, _ = run_batch(pk, chs, nch, width=width, schedule=schedule, order=order)
    k = 0
    for s in range(len(pk)):
        _check(res[k:k + len(chs[s])], pk[s], chs[s], nch[s], False)
        k += len(chs[s])


def test_mixed_whole_streams_many(cuda):
    """Whole-stream chains (the uneven-batch workload shape), both schedules."""
    from gpu_util import run_batch
    rng = np.random.default_rng(77)
    streams = []
    for s in range(24):
        ch = int(rng.integers(1, 3))
        streams.append(corpus.make_stream(dict(kind="mixed", seed=7000 + s, seconds=float(rng.uniform(0.5, 6)),
                                               channels=ch)))
    idx = [ogg_port.demux(d) for d in streams]
    pk = [ix["packets"] for ix in idx]
    nch = [ix["channels"] for ix in idx]
    for schedule in (0, 1):
        res, _ = run_batch(pk, [[(0, len(p), 0, 1 << 40)] for p in pk], nch, width=32, schedule=schedule,
                           order=list(range(len(pk))) if schedule else None)
        for s in range(len(pk)):
            _check([res[s]], pk[s], [(0, len(pk[s]), 0, res[s]["keep"])], nch[s], True)


@pytest.mark.parametrize("channels,width", [(1, 32), (2, 32), (2, 4), (1, 1)])
def test_spliced_mode_changes(cuda, channels, width):
    """Mode changes without redundancy (CELT -> SILK / hybrid, SILK / hybrid ->
    CELT, hybrid -> SILK with the CELT layer's silence frame): the 5 ms
    concealment crossfades and silence frames of opus_decode_frame, bit-exact
    (tests/branches.py builds the chains; test_branches.py shows they reach
    those branches)."""
    from branches import spliced_chains
    from gpu_util import run_batch
    packets, chains = spliced_chains(channels)
    res, _ = run_batch([packets], [[(f, n, 0, 1 << 40) for f, n in chains]], [channels], width=width)
    for i, (f, n) in enumerate(chains):
        _check([res[i]], packets, [(f, n, 0, res[i]["keep"])], channels, True)


def test_f16k_matches_cpu_pipeline(cuda):
    import torch
    from cuopus_b200 import cuopus_native as cn
    for d in _streams("plain", 3, 2.5, 8000) + [corpus.make_stream(dict(kind="long", seed=8100, seconds=6.0,
                                                                          channels=1))]:
        want = pipeline.f16k(d)
        got = cn.decode_ogg_to_cuda_tensor(d)
        torch.cuda.synchronize()
        g = got.cpu().numpy()
        assert g.shape == want.shape
        assert np.max(np.abs(g - want)) == 0.0
        assert cn.probe(d) == want.size


def test_f16k_multi_equals_single(cuda):
    import torch
    from cuopus_b200 import cuopus_native as cn
    streams = _streams("plain", 5, 1.7, 8200)
    single = [cn.decode_ogg_to_cuda_tensor(d).cpu().numpy() for d in streams]
    multi = [t.cpu().numpy() for t in cn.decode_ogg_multi(streams)]
    for a, b in zip(single, multi):
        assert a.shape == b.shape and np.array_equal(a, b)


def test_f16k_channels_stereo_and_mono(cuda):
    """Stereo f16k: each channel resampled by the same filter, interleaved;
    max abs diff 0 against the resampler restatement per channel."""
    from cuopus_b200 import cuopus_native as cn
    streams = _streams("mixed", 4, 2.5, 8400)
    outs = cn.decode_ogg_to_f16k_channels(streams)
    for d, (t, ch) in zip(streams, outs):
        pcm, wch, _ = pipeline.i16(d)
        assert ch == wch
        play = pcm.size // ch
        n16 = max(0, (play - 48) // 3)
        want = np.stack([pipeline.resample(np.ascontiguousarray(pcm[c::ch]), n16) for c in range(ch)], 1).reshape(-1)
        got = t.cpu().numpy()
        assert got.shape == want.shape
        assert np.max(np.abs(got - want), initial=0.0) == 0.0
        if ch == 1:
            assert np.array_equal(got, cn.decode_ogg_to_cuda_tensor(d).cpu().numpy())


def test_i16_stereo_and_mono(cuda):
    """int16 48 kHz output, mono and stereo, against the CPU pipeline; the
    outputs back to back in one buffer (decoded in place) and the same outputs
    in buffers with gaps between them (decoded into the workspace, then
    copied) hold the same samples."""
    import ctypes
    import torch
    from cuopus_b200 import cuopus_native as cn
    streams = _streams("mixed", 4, 3.0, 8300)
    outs = cn.decode_ogg_to_int16(streams)
    for d, (t, ch) in zip(streams, outs):
        want, wch, _ = pipeline.i16(d)
        assert ch == wch
        assert np.array_equal(t.cpu().numpy(), want)
    caps = [t.numel() for t, _ in outs]
    gap = 4097
    big = torch.full((sum(caps) + gap * len(caps),), 7, dtype=torch.int16, device="cuda")
    starts = [sum(caps[:i]) + gap * (i + 1) for i in range(len(caps))]
    n = len(streams)
    lib = cn.lib()
    err = ctypes.create_string_buffer(512)
    ol, oc = (ctypes.c_int64 * n)(), (ctypes.c_int32 * n)()
    rc = lib.cuopus_decode_i16_multi((ctypes.c_char_p * n)(*streams), (ctypes.c_size_t * n)(*map(len, streams)), n,
                                     (ctypes.c_void_p * n)(*[big.data_ptr() + 2 * s for s in starts]),
                                     (ctypes.c_size_t * n)(*caps), ol, oc,
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), err, 512)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    h = big.cpu().numpy()
    for i, (t, _) in enumerate(outs):
        assert np.array_equal(h[starts[i]:starts[i] + caps[i]], t.cpu().numpy())
        assert np.all(h[starts[i] - gap:starts[i]] == 7)   # the gaps are untouched


def _lossy(packets, seed, p_lost, p_dtx):
    """Some packets empty (lost: concealment), some cut to the TOC byte (DTX)."""
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


@pytest.mark.parametrize("width", [32, 8])
def test_concealment_matches_libopus(cuda, width):
    """Lost and DTX packets in SILK / hybrid / CELT streams, mono and stereo:
    SILK PLC and CNG, CELT PLC and the transitions around them, bit-exact."""
    from gpu_util import run_batch
    pk, chs, nch = [], [], []
    for s in range(4):
        d = corpus.make_stream(dict(kind="mixed", seed=21 + s, seconds=4.0, channels=1 + s % 2))
        ix = ogg_port.demux(d)
        p = _lossy(ix["packets"], 21 + s, 0.12, 0.08)
        pk.append(p)
        chs.append([(0, len(p), 0, 1 << 40)] + [(i, min(20, len(p) - i), 0, 1 << 40) for i in range(0, len(p), 20)])
        nch.append(ix["channels"])
    res, _ = run_batch(pk, chs, nch, width=width, schedule=1, order=None)
    k = 0
    for s in range(len(pk)):
        _check(res[k:k + len(chs[s])], pk[s], [(c[0], c[1], 0, r["keep"]) for c, r in
                                               zip(chs[s], res[k:k + len(chs[s])])], nch[s], True)
        k += len(chs[s])


def test_damaged_packets_stop_like_libopus(cuda):
    """Truncated and bit-flipped packets: same stop status, per-packet counts,
    final ranges and samples as libopus up to the first error."""
    from gpu_util import run_batch
    rng = np.random.default_rng(5)
    pk, nch = [], []
    for s in range(6):
        ix = ogg_port.demux(corpus.make_stream(dict(kind="mixed", seed=31 + s, seconds=3.0, channels=1 + s % 2)))
        p = list(ix["packets"])
        for i in range(s % 5, len(p), 5 + s):
            b = bytearray(p[i])
            if i % 3 == 0 and len(b) > 3:
                b = b[: len(b) // 2]
            elif len(b) > 2:
                b[int(rng.integers(1, len(b)))] ^= 1 << int(rng.integers(0, 8))
            p[i] = bytes(b)
        pk.append(p)
        nch.append(ix["channels"])
    res, _ = run_batch(pk, [[(0, len(p), 0, 1 << 40)] for p in pk], nch, width=32, schedule=1)
    for s in range(len(pk)):
        ref = ref_decode.decode_chains(pk[s], [(0, len(pk[s]))], nch[s])
        g = res[s]
        assert g["stop"] == int(ref["status"][0])
        assert np.array_equal(g["nsamp"], ref["nsamp"][0]) and np.array_equal(g["rng"], ref["rng"][0])
        n = int(ref["samples"][0]) * nch[s]
        assert g["samples"] == int(ref["samples"][0])
        assert np.array_equal(g["pcm"][:n], ref["pcm"][0])


@pytest.mark.parametrize("fec", [1, 0])
def test_inband_fec_matches_libopus(cuda, fec):
    """Streams with in-band FEC (LBRR) and DTX, 15 % of packets lost: with
    cuopus_batch.fec = 1 a lost packet is rebuilt from the next packet's LBRR
    frames exactly as libopus's decode_fec = 1 does; with fec = 0 the same
    streams conceal like the reference's protocol."""
    from gpu_util import run_batch
    pk, chs, nch = [], [], []
    for seed, ch in [(42, 2), (44, 2), (45, 1), (48, 1), (49, 1)]:
        d = corpus.make_stream(dict(kind="mixed", seed=seed, seconds=5.0, channels=ch, inband_fec=1, loss_perc=25,
                                    dtx=1))
        ix = ogg_port.demux(d)
        p = _lossy(ix["packets"], seed, 0.15, 0.0)
        pk.append(p)
        chs.append([(0, len(p), 0, 1 << 40)] + [(i, min(25, len(p) - i), 0, 1 << 40) for i in range(0, len(p), 25)])
        nch.append(ix["channels"])
    res, _ = run_batch(pk, chs, nch, width=32, schedule=1, fec=fec)
    k = 0
    for s in range(len(pk)):
        ref = ref_decode.decode_chains(pk[s], [c[:2] for c in chs[s]], nch[s], fec=fec)
        for i, g in enumerate(res[k:k + len(chs[s])]):
            assert g["stop"] == int(ref["status"][i]) == 0
            assert np.array_equal(g["nsamp"], ref["nsamp"][i]) and np.array_equal(g["rng"], ref["rng"][i])
            assert np.array_equal(g["pcm"], ref["pcm"][i]), "stream %d chain %d" % (s, i)
        k += len(chs[s])


def test_autotuners_pick_a_launch_and_keep_the_bits(cuda):
    """cuopus_autotune (width x block) and cuopus_autotune_occupancy (decoder
    warps per SM) time real candidates, and the launch they pick decodes the
    same samples as libopus."""
    import torch
    from cuopus_b200 import cuopus_native as cn
    from gpu_util import device_batch, run_device_batch
    rng = np.random.default_rng(91)
    streams = [corpus.make_stream(dict(kind="mixed", seed=9100 + s, seconds=float(rng.uniform(0.5, 4)),
                                       channels=1 + s % 2)) for s in range(40)]
    idx = [ogg_port.demux(d) for d in streams]
    pk = [ix["packets"] for ix in idx]
    nch = [ix["channels"] for ix in idx]
    b, T, meta = device_batch(pk, [[(0, len(p))] for p in pk], nch)
    b.schedule, b.graph = 1, 1
    order = np.arange(meta["n"], dtype=np.uint32)[::-1].copy()
    b.order = order.ctypes.data
    st = torch.cuda.current_stream().cuda_stream
    w, blk, table = cn.autotune(b, widths=(8, 32), blocks=(64, 128), reps=1, stream=st)
    assert (w, blk) in table and table[(w, blk)] == min(v for v in table.values() if v is not None)
    b.width, b.block = w, blk
    mg, occ = cn.autotune_occupancy(b, warps_per_sm=(0, 6, 4), reps=1, stream=st)
    assert set(occ) == {0, 6, 4} and all(v is not None and v > 0 for v in occ.values())
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert mg in (0, 6 * sms * (32 // w), 4 * sms * (32 // w))
    b.max_groups = mg
    res = run_device_batch(b, meta, width=w, schedule=1, order=order, block=blk, graph=1)
    out = T["out"].cpu().numpy()
    for s in range(len(pk)):
        ref = ref_decode.decode_chains(pk[s], [(0, len(pk[s]))], nch[s])
        assert int(res[s, 0]) == 0 and int(res[s, 1]) == int(ref["samples"][0])
        o = int(meta["out_off"][s])
        assert np.array_equal(out[o:o + int(meta["keep"][s]) * nch[s]], ref["pcm"][0])


def test_tail_scheduling_keeps_the_bits(cuda):
    """Tail scheduling (cuopus_batch.light_sms): the longest chains run alone on
    their own SMs, the rest share the others; every chain still decodes to
    libopus's samples, whichever warp takes it."""
    import torch
    from gpu_util import device_batch, run_device_batch
    rng = np.random.default_rng(93)
    lens = [12.0, 9.0] + [float(rng.uniform(0.3, 3.0)) for _ in range(30)]
    streams = [corpus.make_stream(dict(kind="mixed", seed=9300 + s, seconds=L, channels=1 + s % 2))
               for s, L in enumerate(lens)]
    idx = [ogg_port.demux(d) for d in streams]
    pk = [ix["packets"] for ix in idx]
    nch = [ix["channels"] for ix in idx]
    b, T, meta = device_batch(pk, [[(0, len(p))] for p in pk], nch)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    order = np.argsort(-np.array([len(p) * c for p, c in zip(pk, nch)]), kind="stable").astype(np.uint32)
    for light, mg in ((4, 5 * sms), (2, 0)):
        b.light_sms, b.long_chains, b.max_groups = light, light, mg
        res = run_device_batch(b, meta, width=32, schedule=1, order=order, block=64, graph=1)
        out = T["out"].cpu().numpy()
        for s in range(len(pk)):
            ref = ref_decode.decode_chains(pk[s], [(0, len(pk[s]))], nch[s])
            assert int(res[s, 0]) == 0 and int(res[s, 1]) == int(ref["samples"][0])
            o = int(meta["out_off"][s])
            assert np.array_equal(out[o:o + int(meta["keep"][s]) * nch[s]], ref["pcm"][0]), (light, s)


@pytest.mark.gpu
def test_visiting_order_keeps_the_bits(cuda, monkeypatch):
    """The file entry points' chain order (fitted additive cost, or decoded
    samples with CUOPUS_ORDER=samples) changes no sample: int16 at 32 lanes
    per chain (whole streams) and f16k at 8 (1 s chains of a long stream)."""
    from cuopus_b200 import cuopus_native as cn
    streams = _streams("mixed", 6, 4.0, 8600)
    long_one = corpus.make_stream(dict(kind="mixed", seed=8700, seconds=20.0, channels=1))
    got = {}
    for order in (None, "samples"):
        if order:
            monkeypatch.setenv("CUOPUS_ORDER", order)
        else:
            monkeypatch.delenv("CUOPUS_ORDER", raising=False)
        monkeypatch.setenv("CUOPUS_SEG_S", "1e9")
        monkeypatch.delenv("CUOPUS_STRIDE", raising=False)
        i16 = [t.cpu().numpy() for t, _ in cn.decode_ogg_to_int16(streams)]
        monkeypatch.setenv("CUOPUS_SEG_S", "1.0")
        monkeypatch.setenv("CUOPUS_STRIDE", "8")
        f16 = cn.decode_ogg_to_cuda_tensor(long_one).cpu().numpy()
        got[order] = (i16, f16, cn.last_stats()["width"])
    a, b = got[None], got["samples"]
    assert all(np.array_equal(x, y) for x, y in zip(a[0], b[0]))
    assert np.array_equal(a[1], b[1])
    assert a[2] == b[2] == 8


@pytest.mark.gpu
def test_packet_staging_off_keeps_the_bits(cuda, monkeypatch):
    """CUOPUS_STAGE=0 (packets read in place instead of staged in shared
    memory) decodes the same samples, at 32 lanes per chain (whole streams,
    the full-register kernel instance) and at 8 (1 s chains, the 12-warp
    instance), packets larger than a staging buffer included."""
    from cuopus_b200 import cuopus_native as cn
    streams = _streams("mixed", 6, 4.0, 8800)
    big = corpus.make_stream(dict(kind="mixed", seed=8900, seconds=6.0, channels=2))
    # some packets exceed a staging buffer (480 bytes) and are read in place either way
    assert any(len(p) > 480 for f in streams + [big] for p in ogg_port.demux(f)["packets"])
    got = {}
    for stage in (None, "0"):
        if stage:
            monkeypatch.setenv("CUOPUS_STAGE", stage)
        else:
            monkeypatch.delenv("CUOPUS_STAGE", raising=False)
        out = []
        for seg, stride in (("1e9", "32"), ("1.0", "8")):
            monkeypatch.setenv("CUOPUS_SEG_S", seg)
            monkeypatch.setenv("CUOPUS_STRIDE", stride)
            out.append([t.cpu().numpy() for t, _ in cn.decode_ogg_to_int16(streams + [big])])
        got[stage] = out
    for a, b in zip(got[None], got["0"]):
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
