"""Drop-in: this library behind the reference's own Python binding.

tests/golden/ref_binding.json is the binding table of the reference's
python/cuopus_native.py (every function it binds, with its ctypes argument
and return types), recorded from that module by make_ref_binding.py.  The
tests bind libcuopus.so exactly that way and make the calls the reference
module makes:

* CPU: every bound function resolves, the host-only probe gives the golden
  (play48 - 48) / 3 length, and the decode calls fail with RC 2 (no device)
  instead of decoding on the CPU;
* GPU: decode_ogg_to_cuda_tensor's and decode_ogg_multi's call sequences,
  through the same binding, on this library and on the reference's own
  libcuopus built unchanged for sm_100a (oracle/Makefile ref_gpu), give
  identical float32 16 kHz outputs (max abs diff 0: the decoder and the
  resampler against the reference's kernels, cuopus_kernels.cuh:41-149);
* GPU: every decode entry point refuses a stream that is capturing a CUDA
  graph with RC 3 (libcuopus.cu:259-267).
"""
import ctypes
import json
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
OURS = os.path.join(ROOT, "cuopus_b200", "lib", "libcuopus.so")
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libcuopus_refgpu.so")
with open(os.path.join(GOLD, "ref_binding.json")) as _f:
    BINDING = json.load(_f)
with open(os.path.join(GOLD, "index.json")) as _f:
    INDEX = json.load(_f)


def _ctype(name):
    if name is None:
        return None
    if name.startswith("POINTER("):
        return ctypes.POINTER(_ctype(name[8:-1]))
    return getattr(ctypes, name)


def bind(path):
    """Load a libcuopus and bind it as the reference's Python module does."""
    lib = ctypes.CDLL(path)
    for fn, sig in BINDING.items():
        f = getattr(lib, fn)
        f.argtypes = [_ctype(t) for t in sig["argtypes"]]
        f.restype = _ctype(sig["restype"])
    return lib


def _stream(name):
    with open(os.path.join(GOLD, "streams", name + ".opus"), "rb") as f:
        return f.read()


def ref_probe(lib, data):
    n16 = ctypes.c_int64(0)
    err = ctypes.create_string_buffer(512)
    rc = lib.cuopus_probe(data, len(data), ctypes.byref(n16), err, 512)
    return rc, n16.value, err.value.decode(errors="replace")


def ref_decode_f16k(lib, data):
    """decode_ogg_to_cuda_tensor of the reference module, on `lib`."""
    import torch
    rc, n16, msg = ref_probe(lib, data)
    assert rc == 0, msg
    out = torch.empty(n16, dtype=torch.float32, device="cuda")
    out_len = ctypes.c_int64(0)
    err = ctypes.create_string_buffer(512)
    rc = lib.cuopus_decode_f16k_on(data, len(data), ctypes.c_void_p(out.data_ptr()), n16, ctypes.byref(out_len),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), err, 512)
    assert rc == 0, err.value
    assert out_len.value == n16
    return out


def ref_decode_multi(lib, blobs):
    """decode_ogg_multi of the reference module, on `lib`."""
    import torch
    n = len(blobs)
    n16 = [ref_probe(lib, b)[1] for b in blobs]
    outs = [torch.empty(k, dtype=torch.float32, device="cuda") for k in n16]
    ba = (ctypes.c_char_p * n)(*blobs)
    la = (ctypes.c_size_t * n)(*[len(b) for b in blobs])
    oa = (ctypes.c_void_p * n)(*[o.data_ptr() for o in outs])
    ca = (ctypes.c_size_t * n)(*n16)
    ol = (ctypes.c_int64 * n)()
    err = ctypes.create_string_buffer(512)
    rc = lib.cuopus_decode_f16k_multi(ba, la, n, oa, ca, ol, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                      err, 512)
    assert rc == 0, err.value
    assert list(ol) == n16
    return outs


def test_reference_binding_on_this_library():
    """CPU: the reference module's binding resolves on libcuopus.so, probe is
    host-only and exact, and decoding without a device is not a CPU fallback."""
    assert set(BINDING) >= {"cuopus_probe", "cuopus_decode_f16k_on", "cuopus_decode_f16k_multi", "cuopus_warmup",
                            "cuopus_last_arena_overflow", "cuopus_workspace_bytes", "cuopus_release_workspaces"}
    lib = bind(OURS)
    for name in ("plain_a", "long_hybrid", "mixed_mono_a", "short_100ms"):
        rc, n16, msg = ref_probe(lib, _stream(name))
        assert rc == 0, msg
        assert n16 == max(0, (INDEX[name]["pcm_samples_48k"] - 48) // 3)
    rc, _, msg = ref_probe(lib, _stream("mixed_stereo_a"))
    assert rc == 1 and msg   # the reference's f16k path is mono only
    assert lib.cuopus_last_arena_overflow() == 0
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except ImportError:
        have_gpu = False
    if not have_gpu:
        d = _stream("plain_a")
        out_len = ctypes.c_int64(0)
        err = ctypes.create_string_buffer(512)
        rc = lib.cuopus_decode_f16k_on(d, len(d), ctypes.c_void_p(0x1000), 10, ctypes.byref(out_len), None, err, 512)
        assert rc in (2, 3), (rc, err.value)


@pytest.mark.gpu
def test_same_output_as_the_reference_library(cuda):
    """Through the reference module's calls, this library and the reference's
    own (built for sm_100a) give the same float32 16 kHz samples."""
    from oracle import corpus
    assert os.path.exists(REF_GPU), "oracle/_ref/libcuopus_refgpu.so must be built (make -C oracle ref_gpu)"
    ours, ref = bind(OURS), bind(REF_GPU)
    streams = [_stream(n) for n in ("plain_a", "plain_b", "long_hybrid", "mixed_mono_a", "mixed_mono_b",
                                    "code3_120ms", "short_100ms")]
    streams += [corpus.make_stream(dict(kind="mixed", seed=9300 + s, seconds=3.0, channels=1)) for s in range(4)]
    for d in streams:
        a = ref_decode_f16k(ours, d).cpu().numpy()
        b = ref_decode_f16k(ref, d).cpu().numpy()
        assert a.shape == b.shape and np.max(np.abs(a - b), initial=0.0) == 0.0
    ma = [t.cpu().numpy() for t in ref_decode_multi(ours, streams)]
    mb = [t.cpu().numpy() for t in ref_decode_multi(ref, streams)]
    for a, b in zip(ma, mb):
        assert a.shape == b.shape and np.max(np.abs(a - b), initial=0.0) == 0.0


@pytest.mark.gpu
def test_decode_refused_during_stream_capture(cuda):
    """A stream that is capturing a CUDA graph: every decode entry point
    returns RC 3 and enqueues nothing (the capture ends with an empty graph)."""
    import torch
    from cuopus_b200 import cuopus_native as cn
    mono, stereo = _stream("plain_a"), _stream("mixed_stereo_a")
    n16 = cn.probe(mono)
    out = torch.empty(n16, dtype=torch.float32, device="cuda")
    out16 = torch.empty(2 * INDEX["mixed_stereo_a"]["pcm_samples_48k"], dtype=torch.int16, device="cuda")
    lib = bind(OURS)
    ilib = cn.lib()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    rcs = {}
    with torch.cuda.graph(g, stream=s):
        st = ctypes.c_void_p(s.cuda_stream)
        err = ctypes.create_string_buffer(512)
        ol = ctypes.c_int64(0)
        rcs["f16k_on"] = lib.cuopus_decode_f16k_on(mono, len(mono), ctypes.c_void_p(out.data_ptr()), n16,
                                                   ctypes.byref(ol), st, err, 512)
        ba = (ctypes.c_char_p * 1)(mono)
        la = (ctypes.c_size_t * 1)(len(mono))
        oa = (ctypes.c_void_p * 1)(out.data_ptr())
        ca = (ctypes.c_size_t * 1)(n16)
        ola = (ctypes.c_int64 * 1)()
        rcs["f16k_multi"] = lib.cuopus_decode_f16k_multi(ba, la, 1, oa, ca, ola, st, err, 512)
        ba2 = (ctypes.c_char_p * 1)(stereo)
        la2 = (ctypes.c_size_t * 1)(len(stereo))
        oa2 = (ctypes.c_void_p * 1)(out16.data_ptr())
        ca2 = (ctypes.c_size_t * 1)(out16.numel())
        oc2 = (ctypes.c_int32 * 1)()
        rcs["i16_multi"] = ilib.cuopus_decode_i16_multi(ba2, la2, 1, oa2, ca2, ola, oc2, st, err, 512)
        rcs["message"] = err.value.decode()
    assert rcs["f16k_on"] == 3 and rcs["f16k_multi"] == 3 and rcs["i16_multi"] == 3, rcs
    assert "capture" in rcs["message"]
    # after the capture the same calls decode normally
    torch.cuda.synchronize()
    got = cn.decode_ogg_to_cuda_tensor(mono)
    assert got.numel() == n16
