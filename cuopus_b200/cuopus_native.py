"""cuopus_native: ctypes wrapper of libcuopus.so (batched Opus decode on B200).

Same surface as the reference's python/cuopus_native.py:30-180:
probe, decode_ogg_to_cuda_tensor, decode_ogg_multi, warmup, workspace_bytes,
last_arena_overflow, release_workspaces and CuopusError, with the same argument
meaning, the same (play48 - 48) // 3 output length contract and the same
errors (CuopusError carries the library's return code: 1 soft, 2 CUDA,
3 caller).  Work runs on torch's current CUDA device and stream; the library
creates no context, thread or stream and synchronises the stream before it
returns.  torch is used only to allocate the output tensors and to name the
stream.

Extensions: decode_ogg_to_int16 (48 kHz interleaved int16, mono or stereo) and
decode_batch (the device-resident engine, used by the benchmark and tests).

There is no CPU fallback: when libcuopus.so is missing or no GPU is present the
calls raise.
"""
from __future__ import annotations

import ctypes
import os

_ERRCAP = 512
_RC_NAMES = {1: "soft", 2: "cuda", 3: "caller"}
_HERE = os.path.dirname(os.path.abspath(__file__))


class CuopusError(RuntimeError):
    def __init__(self, rc, msg):
        super().__init__("cuopus[%s]: %s" % (_RC_NAMES.get(rc, rc), msg))
        self.rc = rc


def _find_lib():
    env = os.environ.get("CUOPUS_LIB")
    if env:
        return env
    cand = os.path.join(_HERE, "lib", "libcuopus.so")
    if os.path.exists(cand):
        return cand
    raise OSError("libcuopus.so not found (run `python -m cuopus_b200.build` or set CUOPUS_LIB)")


class Batch(ctypes.Structure):
    """cuopus_batch of include/cuopus.h."""
    _fields_ = [("data", ctypes.c_void_p), ("off", ctypes.c_void_p), ("len", ctypes.c_void_p),
                ("first", ctypes.c_void_p), ("npkts", ctypes.c_void_p), ("channels", ctypes.c_void_p),
                ("trim", ctypes.c_void_p), ("keep", ctypes.c_void_p), ("out_off", ctypes.c_void_p),
                ("out", ctypes.c_void_p), ("rec_off", ctypes.c_void_p), ("pkt_nsamp", ctypes.c_void_p),
                ("pkt_rng", ctypes.c_void_p), ("res", ctypes.c_void_p), ("nchains", ctypes.c_int32),
                ("width", ctypes.c_int32), ("schedule", ctypes.c_int32), ("max_groups", ctypes.c_int32),
                ("order", ctypes.c_void_p), ("block", ctypes.c_int32), ("graph", ctypes.c_int32),
                ("scalar", ctypes.c_int32), ("fec", ctypes.c_int32), ("light_sms", ctypes.c_int32),
                ("long_chains", ctypes.c_int32)]


_lib = None


def _load():
    global _lib
    if _lib is not None:
        return _lib
    lib = ctypes.CDLL(_find_lib())
    c_p = ctypes.c_void_p
    lib.cuopus_probe.restype = ctypes.c_int
    lib.cuopus_probe.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64),
                                 ctypes.c_char_p, ctypes.c_size_t]
    lib.cuopus_decode_f16k.restype = ctypes.c_int
    lib.cuopus_decode_f16k.argtypes = [ctypes.c_char_p, ctypes.c_size_t, c_p, ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_int64), ctypes.c_char_p, ctypes.c_size_t]
    lib.cuopus_decode_f16k_on.restype = ctypes.c_int
    lib.cuopus_decode_f16k_on.argtypes = [ctypes.c_char_p, ctypes.c_size_t, c_p, ctypes.c_size_t,
                                          ctypes.POINTER(ctypes.c_int64), c_p, ctypes.c_char_p, ctypes.c_size_t]
    lib.cuopus_decode_f16k_multi.restype = ctypes.c_int
    lib.cuopus_decode_f16k_multi.argtypes = [
        ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t), ctypes.c_int,
        ctypes.POINTER(c_p), ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int64), c_p,
        ctypes.c_char_p, ctypes.c_size_t]
    lib.cuopus_decode_i16_multi.restype = ctypes.c_int
    lib.cuopus_decode_i16_multi.argtypes = [
        ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t), ctypes.c_int,
        ctypes.POINTER(c_p), ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int64),
        ctypes.POINTER(ctypes.c_int32), c_p, ctypes.c_char_p, ctypes.c_size_t]
    lib.cuopus_decode_batch.restype = ctypes.c_int
    lib.cuopus_decode_batch.argtypes = [ctypes.POINTER(Batch), c_p, ctypes.POINTER(ctypes.c_float),
                                        ctypes.c_char_p, ctypes.c_size_t]
    lib.cuopus_autotune.restype = ctypes.c_int
    lib.cuopus_autotune.argtypes = [ctypes.POINTER(Batch), c_p, ctypes.c_int, c_p, ctypes.c_int, ctypes.c_int, c_p,
                                    ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32), c_p,
                                    ctypes.c_char_p, ctypes.c_size_t]
    lib.cuopus_autotune_occupancy.restype = ctypes.c_int
    lib.cuopus_autotune_occupancy.argtypes = [ctypes.POINTER(Batch), c_p, ctypes.c_int, ctypes.c_int, c_p,
                                              ctypes.POINTER(ctypes.c_int32), c_p, ctypes.c_char_p,
                                              ctypes.c_size_t]
    lib.cuopus_last_stats.restype = ctypes.c_int
    lib.cuopus_last_stats.argtypes = [c_p]
    lib.cuopus_resample48to16.restype = ctypes.c_int
    lib.cuopus_resample48to16.argtypes = [c_p, ctypes.c_int64, ctypes.c_int64, c_p, c_p, ctypes.c_char_p,
                                          ctypes.c_size_t]
    lib.cuopus_warmup.restype = ctypes.c_int
    lib.cuopus_warmup.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.cuopus_last_arena_overflow.restype = ctypes.c_int
    lib.cuopus_last_arena_overflow.argtypes = []
    lib.cuopus_workspace_bytes.restype = ctypes.c_longlong
    lib.cuopus_workspace_bytes.argtypes = []
    lib.cuopus_release_workspaces.restype = None
    lib.cuopus_release_workspaces.argtypes = []
    lib.cuopus_probe_pcm.restype = ctypes.c_int
    lib.cuopus_probe_pcm.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64),
                                     ctypes.POINTER(ctypes.c_int32), ctypes.c_char_p, ctypes.c_size_t]
    lib.cuopus_index.restype = ctypes.c_int
    lib.cuopus_index.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_double, ctypes.c_int] + \
        [ctypes.POINTER(ctypes.c_int64)] * 3 + [ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64)] + \
        [c_p] * 7 + [ctypes.c_char_p, ctypes.c_size_t]
    lib.cuopus_slot_bytes.restype = ctypes.c_longlong
    lib.cuopus_slot_bytes.argtypes = []
    lib.cuopus_default_width.restype = ctypes.c_int
    lib.cuopus_default_width.argtypes = []
    _lib = lib
    return lib


def lib():
    """The loaded libcuopus (ctypes.CDLL)."""
    return _load()


def _as_bytes(path_or_bytes):
    if isinstance(path_or_bytes, (bytes, bytearray, memoryview)):
        return bytes(path_or_bytes)
    with open(path_or_bytes, "rb") as f:
        return f.read()


def _check(rc, err):
    if rc:
        raise CuopusError(rc, err.value.decode(errors="replace"))


def probe(path_or_bytes) -> int:
    """Exact output length in float32 @16 kHz samples (host-only, no GPU)."""
    lib = _load()
    data = _as_bytes(path_or_bytes)
    n16 = ctypes.c_int64(0)
    err = ctypes.create_string_buffer(_ERRCAP)
    _check(lib.cuopus_probe(data, len(data), ctypes.byref(n16), err, _ERRCAP), err)
    return n16.value


def probe_pcm(path_or_bytes):
    """Extension: (playable samples per channel at 48 kHz, channels); host only."""
    lib = _load()
    data = _as_bytes(path_or_bytes)
    play = ctypes.c_int64(0)
    ch = ctypes.c_int32(0)
    err = ctypes.create_string_buffer(_ERRCAP)
    _check(lib.cuopus_probe_pcm(data, len(data), ctypes.byref(play), ctypes.byref(ch), err, _ERRCAP), err)
    return play.value, ch.value


class Index:
    """Host demux + chain table of one stream (cuopus_index)."""

    def __init__(self, blob, pkt_off, pkt_len, first, npkts, trim, keep, channels, play48):
        self.blob, self.pkt_off, self.pkt_len = blob, pkt_off, pkt_len
        self.first, self.npkts, self.trim, self.keep = first, npkts, trim, keep
        self.channels, self.play48 = channels, play48


def index(path_or_bytes, seg_s=1.0, preroll_ms=250.0, require_mono=False):
    """Extension: demux + chain table through the library's C++ demuxer."""
    import numpy as np
    lib = _load()
    data = _as_bytes(path_or_bytes)
    npk, nch, nb, play = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
    ch = ctypes.c_int32(0)
    err = ctypes.create_string_buffer(_ERRCAP)
    args = (data, len(data), float(seg_s), float(preroll_ms), int(require_mono), ctypes.byref(npk),
            ctypes.byref(nch), ctypes.byref(nb), ctypes.byref(ch), ctypes.byref(play))
    _check(lib.cuopus_index(*args, None, None, None, None, None, None, None, err, _ERRCAP), err)
    blob = np.zeros(max(nb.value, 1), np.uint8)
    off = np.zeros(max(npk.value, 1), np.uint64)
    ln = np.zeros(max(npk.value, 1), np.uint32)
    tabs = [np.zeros(max(nch.value, 1), np.uint32) for _ in range(4)]
    _check(lib.cuopus_index(*args, blob.ctypes.data, off.ctypes.data, ln.ctypes.data,
                            *[t.ctypes.data for t in tabs], err, _ERRCAP), err)
    k, c = npk.value, nch.value
    return Index(blob[:nb.value], off[:k], ln[:k], tabs[0][:c], tabs[1][:c], tabs[2][:c], tabs[3][:c],
                 ch.value, play.value)


def decode_ogg_to_cuda_tensor(path_or_bytes):
    """Decode an Ogg Opus file/bytes into a fresh torch CUDA float32 tensor at
    16 kHz on the current device/stream.  Raises CuopusError on failure."""
    import torch
    lib = _load()
    data = _as_bytes(path_or_bytes)
    n16 = probe(data)
    out = torch.empty(n16, dtype=torch.float32, device="cuda")
    if n16 == 0:
        return out
    stream = torch.cuda.current_stream().cuda_stream
    out_len = ctypes.c_int64(0)
    err = ctypes.create_string_buffer(_ERRCAP)
    _check(lib.cuopus_decode_f16k_on(data, len(data), ctypes.c_void_p(out.data_ptr()), n16,
                                     ctypes.byref(out_len), ctypes.c_void_p(stream), err, _ERRCAP), err)
    if out_len.value != n16:
        raise CuopusError(1, "decode wrote %d samples, probe said %d" % (out_len.value, n16))
    return out


def decode_ogg_multi(items):
    """Decode N Ogg Opus files/byte strings in one decode launch; returns a list
    of 1-D CUDA float32 tensors at 16 kHz, each identical to
    decode_ogg_to_cuda_tensor of that file.  rc 3 with a "max_batch" message
    means the merged chain count exceeds CUOPUS_MAX_BATCH."""
    import torch
    lib = _load()
    blobs = [_as_bytes(x) for x in items]
    n = len(blobs)
    if n == 0:
        return []
    n16 = [probe(b) for b in blobs]
    outs = [torch.empty(k, dtype=torch.float32, device="cuda") for k in n16]
    stream = torch.cuda.current_stream().cuda_stream
    ba = (ctypes.c_char_p * n)(*blobs)
    la = (ctypes.c_size_t * n)(*[len(b) for b in blobs])
    oa = (ctypes.c_void_p * n)(*[o.data_ptr() for o in outs])
    ca = (ctypes.c_size_t * n)(*n16)
    ol = (ctypes.c_int64 * n)()
    err = ctypes.create_string_buffer(_ERRCAP)
    _check(lib.cuopus_decode_f16k_multi(ba, la, n, oa, ca, ol, ctypes.c_void_p(stream), err, _ERRCAP), err)
    for i in range(n):
        if ol[i] != n16[i]:
            raise CuopusError(1, "file %d: decode wrote %d samples, probe said %d" % (i, ol[i], n16[i]))
    return outs


def decode_ogg_to_f16k_channels(items):
    """Extension: float32 16 kHz output for mono and stereo files (stereo
    channels resampled separately, interleaved).  Returns a list of
    (tensor[float32, samples*channels], channels)."""
    import torch
    lib = _load()
    if not getattr(lib, "_f16kc_bound", False):
        lib.cuopus_decode_f16k_channels.restype = ctypes.c_int
        lib.cuopus_decode_f16k_channels.argtypes = [
            ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t), ctypes.c_int,
            ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int64),
            ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
        lib._f16kc_bound = True
    blobs = [_as_bytes(x) for x in items]
    n = len(blobs)
    if n == 0:
        return []
    caps = []
    for b in blobs:
        play, ch = probe_pcm(b)
        caps.append(max(0, (play - 48) // 3) * ch)
    outs = [torch.empty(max(c, 1), dtype=torch.float32, device="cuda") for c in caps]
    stream = torch.cuda.current_stream().cuda_stream
    ba = (ctypes.c_char_p * n)(*blobs)
    la = (ctypes.c_size_t * n)(*[len(b) for b in blobs])
    oa = (ctypes.c_void_p * n)(*[o.data_ptr() for o in outs])
    ca = (ctypes.c_size_t * n)(*caps)
    ol = (ctypes.c_int64 * n)()
    oc = (ctypes.c_int32 * n)()
    err = ctypes.create_string_buffer(_ERRCAP)
    _check(lib.cuopus_decode_f16k_channels(ba, la, n, oa, ca, ol, oc, ctypes.c_void_p(stream), err, _ERRCAP), err)
    return [(outs[i][:ol[i] * oc[i]], oc[i]) for i in range(n)]


def decode_ogg_to_int16(items, capacities=None):
    """Extension: decode files to 48 kHz interleaved int16 playable PCM (mono or
    stereo).  Returns a list of (tensor[int16, samples*channels], channels):
    views of one device buffer holding the files back to back."""
    import numpy as np
    import torch
    lib = _load()
    blobs = [_as_bytes(x) for x in items]
    n = len(blobs)
    if n == 0:
        return []
    if capacities is None:
        capacities = []
        for b in blobs:
            play, ch = probe_pcm(b)
            capacities.append(play * ch)
    # one buffer, the files back to back: the library decodes straight into it
    bounds = np.concatenate([[0], np.cumsum([int(c) for c in capacities])]).astype(np.int64)
    whole = torch.empty(max(int(bounds[-1]), 1), dtype=torch.int16, device="cuda")
    outs = [whole[int(bounds[i]):int(bounds[i + 1])] for i in range(n)]
    stream = torch.cuda.current_stream().cuda_stream
    ba = (ctypes.c_char_p * n)(*blobs)
    la = (ctypes.c_size_t * n)(*[len(b) for b in blobs])
    oa = (ctypes.c_void_p * n)(*[o.data_ptr() for o in outs])
    ca = (ctypes.c_size_t * n)(*[int(c) for c in capacities])
    ol = (ctypes.c_int64 * n)()
    oc = (ctypes.c_int32 * n)()
    err = ctypes.create_string_buffer(_ERRCAP)
    _check(lib.cuopus_decode_i16_multi(ba, la, n, oa, ca, ol, oc, ctypes.c_void_p(stream), err, _ERRCAP), err)
    return [(outs[i][:ol[i] * oc[i]], oc[i]) for i in range(n)]


def decode_batch(batch: Batch, stream=None):
    """Extension: run the device-resident engine; returns the decode kernel ms."""
    lib = _load()
    ms = ctypes.c_float(0)
    err = ctypes.create_string_buffer(_ERRCAP)
    _check(lib.cuopus_decode_batch(ctypes.byref(batch), ctypes.c_void_p(stream or 0), ctypes.byref(ms), err,
                                   _ERRCAP), err)
    return ms.value


def autotune(batch: Batch, widths=(4, 8, 16, 32), blocks=(32, 64, 128), reps=1, stream=None):
    """Extension: time the batch at every (width, block) pair; returns
    (best_width, best_block, {(width, block): median ms or None})."""
    import numpy as np
    lib = _load()
    w = np.ascontiguousarray(np.array(widths, np.int32))
    b = np.ascontiguousarray(np.array(blocks, np.int32))
    t = np.zeros(len(w) * len(b), np.float32)
    bw, bb = ctypes.c_int32(0), ctypes.c_int32(0)
    err = ctypes.create_string_buffer(_ERRCAP)
    _check(lib.cuopus_autotune(ctypes.byref(batch), w.ctypes.data, len(w), b.ctypes.data, len(b), int(reps),
                               ctypes.c_void_p(stream or 0), ctypes.byref(bw), ctypes.byref(bb), t.ctypes.data,
                               err, _ERRCAP), err)
    table = {(int(w[i]), int(b[j])): (float(t[i * len(b) + j]) if t[i * len(b) + j] >= 0 else None)
             for i in range(len(w)) for j in range(len(b))}
    return bw.value, bb.value, table


def autotune_occupancy(batch: Batch, warps_per_sm=(0, 7, 6, 5, 4), reps=1, stream=None):
    """Extension: time the batch (its width and block kept) at every count of
    decoder warps per SM (0 = all resident groups); returns
    (best max_groups for cuopus_batch, {warps_per_sm: median ms or None})."""
    import numpy as np
    lib = _load()
    g = np.ascontiguousarray(np.array(warps_per_sm, np.int32))
    t = np.zeros(len(g), np.float32)
    best = ctypes.c_int32(0)
    err = ctypes.create_string_buffer(_ERRCAP)
    _check(lib.cuopus_autotune_occupancy(ctypes.byref(batch), g.ctypes.data, len(g), int(reps),
                                         ctypes.c_void_p(stream or 0), ctypes.byref(best), t.ctypes.data, err,
                                         _ERRCAP), err)
    return best.value, {int(g[i]): (float(t[i]) if t[i] >= 0 else None) for i in range(len(g))}


def autotune_tail(batch: Batch, light=(0, 8, 16, 32), reps=2, stream=None):
    """Extension: time the batch (queue schedule, its order longest first) with
    tail scheduling at every count of light SMs (the longest chains, one per
    light SM, each alone on its SM; 0 = off); sets batch.light_sms /
    long_chains to the fastest and returns (best count, {count: median ms})."""
    import statistics
    table = {}
    for k in light:
        batch.light_sms = batch.long_chains = int(k)
        table[int(k)] = statistics.median(decode_batch(batch, stream) for _ in range(max(1, reps)))
    best = min(table, key=table.get)
    batch.light_sms = batch.long_chains = best
    return best, table


class Stats(ctypes.Structure):
    """cuopus_stats of include/cuopus.h."""
    _fields_ = [("demux_ms", ctypes.c_double), ("h2d_ms", ctypes.c_float), ("kernel_ms", ctypes.c_float),
                ("resample_ms", ctypes.c_float), ("chains", ctypes.c_int64), ("packets", ctypes.c_int64),
                ("play48", ctypes.c_int64), ("width", ctypes.c_int32)]


def last_stats():
    """Extension: timings of the last successful decode call (dict)."""
    s = Stats()
    _load().cuopus_last_stats(ctypes.byref(s))
    return {k: getattr(s, k) for k, _ in Stats._fields_}


def warmup():
    """Pre-size the decoder slots and upload the resampler taps."""
    lib = _load()
    err = ctypes.create_string_buffer(_ERRCAP)
    _check(lib.cuopus_warmup(err, _ERRCAP), err)


def workspace_bytes() -> int:
    return int(_load().cuopus_workspace_bytes())


def last_arena_overflow() -> bool:
    return bool(_load().cuopus_last_arena_overflow())


def release_workspaces():
    _load().cuopus_release_workspaces()


# Decoder stages timed by the diagnostic build (libcuopus_phases.so), in the
# order of the device counters.  "packet" spans the whole of one packet's
# decode and contains the others; "keep_copy" (the PCM write) runs inside it.
PHASE_NAMES = ("packet", "silk_indices", "silk_pulses", "silk_params", "silk_core", "silk_plc", "silk_cng",
               "silk_stereo", "silk_resample", "celt_coarse", "celt_alloc", "celt_shift", "celt_bands",
               "celt_synth", "celt_comb", "celt_deemph", "keep_copy",
               # parts of the stages above
               "pvq_cwrsi", "pvq_rotation", "pvq_renormalise", "pvq_theta", "pvq_tf_haar_hadamard", "silk_lpc",
               "silk_ltp", "silk_shell")


def phases_lib_path():
    """Path of the diagnostic build with the decoder's stage timers."""
    return os.path.join(_HERE, "lib", "libcuopus_phases.so")


def phase_reset():
    """Zero the stage counters (diagnostic build only)."""
    lib = _load()
    if not hasattr(lib, "cuopus_phase_reset"):
        raise CuopusError(3, "the loaded library has no stage timers (load %s via CUOPUS_LIB)" % phases_lib_path())
    if lib.cuopus_phase_reset():
        raise CuopusError(2, "cuopus_phase_reset failed")


def phase_cycles():
    """Device clock cycles per decoder stage since phase_reset(), summed over
    the first lane of every chain (dict name -> cycles)."""
    lib = _load()
    if not hasattr(lib, "cuopus_phase_read"):
        raise CuopusError(3, "the loaded library has no stage timers (load %s via CUOPUS_LIB)" % phases_lib_path())
    n = int(lib.cuopus_phase_count())
    if n != len(PHASE_NAMES):
        raise CuopusError(3, "library has %d stage counters, this module knows %d" % (n, len(PHASE_NAMES)))
    buf = (ctypes.c_uint64 * n)()
    if lib.cuopus_phase_read(buf):
        raise CuopusError(2, "cuopus_phase_read failed")
    return dict(zip(PHASE_NAMES, (int(v) for v in buf)))
