"""cuopus_decode_batch_noalloc: the decode entry point for callers that
cannot allocate device memory (their device memory belongs to another
framework's pool, or they run on a latency-critical path where cudaMalloc /
cudaFree, which can synchronise the whole device, are not allowed).  It
decodes with decoder slots from a static device array instead of a library
workspace.

Called through the C ABI and checked against cuopus_decode_batch on the same
device tables: every chain's status, sample count, final range and every
int16 sample must be identical, on calls in a row (different batches, so
each call runs on slots the previous one left behind).  Later cases make one
lane group decode several chains in one call (max_groups = 3, and 141 chains
on the 63 groups of 96-thread blocks), so a slot is also reused within a
call, and one case leaves the block size to the entry point at one lane per
chain.  This file is collected last on purpose."""
import ctypes
import os

import numpy as np
import pytest

from oracle import ogg_port

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "streams")


def _tables(names, seg):
    pk, chs, nch = [], [], []
    for n in names:
        ix = ogg_port.demux(open(os.path.join(GOLD, n + ".opus"), "rb").read())
        pk.append(ix["packets"])
        chs.append(ogg_port.build_chains(ix, seg, 250.0))
        nch.append(ix["channels"])
    return pk, chs, nch


def _noalloc(lib, b):
    import torch
    err = ctypes.create_string_buffer(256)
    rc = lib.cuopus_decode_batch_noalloc(ctypes.byref(b), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                         err, 256)
    return rc, err.value.decode()


def test_noalloc_matches_decode_batch_twice(cuda):
    import torch
    from cuopus_b200 import cuopus_native as cn
    from gpu_util import device_batch, run_device_batch
    lib = cn.lib()
    lib.cuopus_decode_batch_noalloc.restype = ctypes.c_int
    lib.cuopus_decode_batch_noalloc.argtypes = [ctypes.POINTER(cn.Batch), ctypes.c_void_p, ctypes.c_char_p,
                                                ctypes.c_size_t]
    every = ["code3_120ms", "long_hybrid", "mixed_mono_a", "mixed_mono_b", "mixed_stereo_a", "mixed_stereo_b",
             "one_packet", "plain_a", "plain_b", "short_100ms", "short_stereo_300ms"]
    # (streams, seconds per chain, lanes per chain, block, max_groups)
    cases = [(["mixed_stereo_a", "mixed_mono_b", "long_hybrid"], 1.0, 32, 0, 0),
             (["mixed_stereo_b", "plain_b", "code3_120ms", "short_stereo_300ms"], 0.5, 16, 0, 0),
             (every, 0.25, 32, 96, 0),
             (["mixed_stereo_a", "mixed_mono_b", "long_hybrid"], 0.5, 8, 0, 3),
             (["plain_b", "code3_120ms", "short_stereo_300ms"], 0.5, 1, 0, 0)]
    for names, seg, width, block, max_groups in cases:
        pk, chs, nch = _tables(names, seg)
        b, keep_alive, meta = device_batch(pk, chs, nch)
        want = run_device_batch(b, meta, width=width, schedule=0)
        want_pcm = meta["T"]["out"].cpu().numpy().copy()
        assert np.all(want[:, 0] == 0)
        meta["T"]["out"].fill_(0x5A5A)
        meta["T"]["res"].fill_(-1)
        if names is every:
            assert meta["n"] > 64   # more chains than static slots: groups decode several each
        b.width, b.block, b.schedule, b.max_groups = width, block, 0, max_groups
        rc, msg = _noalloc(lib, b)
        assert rc == 0, msg
        torch.cuda.synchronize()
        got = meta["T"]["res"].cpu().numpy().view(np.uint32).reshape(-1, 4)[:meta["n"]]
        assert np.array_equal(got[:, :3], want[:, :3])
        assert np.array_equal(meta["T"]["out"].cpu().numpy(), want_pcm)


def test_noalloc_rejects_more_groups_than_slots(cuda):
    from cuopus_b200 import cuopus_native as cn
    from gpu_util import device_batch
    lib = cn.lib()
    lib.cuopus_decode_batch_noalloc.restype = ctypes.c_int
    lib.cuopus_decode_batch_noalloc.argtypes = [ctypes.POINTER(cn.Batch), ctypes.c_void_p, ctypes.c_char_p,
                                                ctypes.c_size_t]
    pk, chs, nch = _tables(["plain_a"], 1.0)
    b, keep_alive, meta = device_batch(pk, chs, nch)
    b.width, b.max_groups = 32, 65
    rc, msg = _noalloc(lib, b)
    assert rc == 3 and "static decoder slots" in msg
