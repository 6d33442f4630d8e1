"""The continuous-batching server: every result equals the one-shot decode of
the same file (alone and in the mix), admission respects the device-memory
budget, and failures are reported per request."""
import os
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "streams")


def _read(name):
    return open(os.path.join(GOLD, name + ".opus"), "rb").read()


def _mix():
    from oracle import corpus
    files = [_read(n) for n in ("mixed_stereo_a", "mixed_mono_b", "long_hybrid", "mixed_stereo_b", "plain_b",
                                "code3_120ms", "short_100ms")]
    for s in range(6):
        files.append(corpus.make_stream(dict(kind="mixed", seed=41000 + s, seconds=2.0 + 1.5 * s,
                                             channels=1 + s % 2)))
    return files


def test_int16_results_alone_equal_results_in_the_mix(cuda):
    from cuopus_b200 import cuopus_native as cn
    from cuopus_b200.serving import Server
    files = _mix()
    alone = []
    for f in files:
        (t, ch), = cn.decode_ogg_to_int16([f])
        alone.append(t.cpu().numpy())
    # small waves so that chains of different requests share waves and
    # requests span several waves on both streams
    with Server(budget_bytes=1 << 30, wave_chains=7, max_inflight=2) as srv:
        ids = []
        for i, f in enumerate(files):            # staggered arrivals
            ids.append(srv.submit(f))
            if i % 3 == 2:
                time.sleep(0.01)
        # the server's own size of each request: samples per channel and channels as the probe gives
        import ctypes
        from cuopus_b200.serving import _lib
        for f, rid in zip(files, ids):
            n, ch, nb = ctypes.c_int64(0), ctypes.c_int32(0), ctypes.c_size_t(0)
            assert _lib().cuopus_server_request_size(srv._h, rid, ctypes.byref(n), ctypes.byref(ch),
                                                     ctypes.byref(nb)) == 0
            assert (n.value, ch.value) == cn.probe_pcm(f) and nb.value == 2 * n.value * ch.value
        assert _lib().cuopus_server_request_size(srv._h, 10 ** 9, None, None, None) == 3
        for i, rid in enumerate(ids):
            out, ch, lat = srv.wait(rid)
            assert lat > 0
            assert np.array_equal(out, alone[i]), "request %d differs from its one-shot decode" % i
        st = srv.stats()
        assert st["completed"] == len(files) and st["failed"] == 0
        assert st["waves"] >= 4 and st["p99_ms"] >= st["p50_ms"] > 0
    # the same file alone in a server
    with Server(budget_bytes=1 << 28) as srv:
        out, _, _ = srv.wait(srv.submit(files[2]))
        assert np.array_equal(out, alone[2])


def test_f16k_results_equal_the_library_call(cuda):
    from cuopus_b200 import cuopus_native as cn
    from cuopus_b200.serving import Server
    from oracle import corpus
    files = [_read("plain_b"), _read("long_hybrid")] + \
        [corpus.make_stream(dict(kind="long", seed=42000 + s, seconds=3.0 + s, channels=1)) for s in range(3)]
    want = [cn.decode_ogg_to_cuda_tensor(f).cpu().numpy() for f in files]
    with Server(budget_bytes=1 << 28, f16k=True, wave_chains=5) as srv:
        ids = [srv.submit(f) for f in files]
        for rid, w in zip(ids, want):
            out, ch, _ = srv.wait(rid)
            assert ch == 1 and out.shape == w.shape
            assert np.max(np.abs(out - w), initial=0.0) == 0.0


def test_admission_budget_and_concurrent_clients(cuda):
    from cuopus_b200 import cuopus_native as cn
    from cuopus_b200.serving import Server
    files = _mix()
    want = []
    for f in files:
        (t, ch), = cn.decode_ogg_to_int16([f])
        want.append(t.cpu().numpy())
    # room for roughly two of the larger requests at a time
    budget = 3 << 20
    peak = [0]
    with Server(budget_bytes=budget, wave_chains=16) as srv:
        results = {}

        def client(k):
            for i in range(k, len(files), 3):
                rid = srv.submit(files[i])
                results[i] = srv.wait(rid)[0]

        ths = [threading.Thread(target=client, args=(k,)) for k in range(3)]
        for t in ths:
            t.start()
        while any(t.is_alive() for t in ths):
            peak[0] = max(peak[0], srv.stats()["arena_used"])
            time.sleep(0.002)
        for t in ths:
            t.join()
        assert peak[0] <= budget
        for i in range(len(files)):
            assert np.array_equal(results[i], want[i]), i


def test_failures_are_per_request(cuda):
    from cuopus_b200 import cuopus_native as cn
    from cuopus_b200.serving import Server
    with Server(budget_bytes=1 << 16) as srv:
        with pytest.raises(cn.CuopusError) as e:
            srv.submit(b"not an ogg stream at all")
        assert e.value.rc == 1
        big = srv.submit(_read("mixed_stereo_b"))       # needs more than 64 KiB
        small = srv.submit(_read("short_100ms"))
        with pytest.raises(cn.CuopusError) as e:
            srv.wait(big)
        assert "budget" in str(e.value)
        out, ch, _ = srv.wait(small)
        (t, _), = cn.decode_ogg_to_int16([_read("short_100ms")])
        assert np.array_equal(out, t.cpu().numpy())
