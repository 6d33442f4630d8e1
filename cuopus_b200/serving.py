"""Continuous-batching decode server: Python front end of the library's
cuopus_server_* entry points (native C++ in csrc/server.cu).

    srv = Server(budget_bytes=40 << 30, f16k=True)
    rid = srv.submit(open("a.opus", "rb").read())     # returns at once
    pcm, channels, latency_ms = srv.wait(rid)          # numpy array
    srv.stats()                                        # p50 / p99 latency, throughput
    srv.close()

Requests are demuxed on the submitting thread, admitted by device-memory
budget, and their 1 s chains are decoded in waves together with whatever else
is in flight; each result equals the one-shot decode of the same file.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import cuopus_native as cn


class ServerConfig(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_int64), ("width", ctypes.c_int32), ("block", ctypes.c_int32),
                ("max_inflight", ctypes.c_int32), ("wave_chains", ctypes.c_int32), ("seg_s", ctypes.c_double),
                ("preroll_ms", ctypes.c_double), ("f16k", ctypes.c_int32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int64), ("failed", ctypes.c_int64), ("waves", ctypes.c_int64),
                ("chains", ctypes.c_int64), ("pending", ctypes.c_int64), ("active", ctypes.c_int64),
                ("arena_used", ctypes.c_int64), ("arena_bytes", ctypes.c_int64), ("wave_chains", ctypes.c_int64),
                ("audio_s", ctypes.c_double), ("wall_ms", ctypes.c_double), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double)]


def _lib():
    lib = cn.lib()
    if not getattr(lib, "_srv_bound", False):
        c_p = ctypes.c_void_p
        tail = [ctypes.c_char_p, ctypes.c_size_t]
        lib.cuopus_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(c_p)] + tail
        lib.cuopus_server_submit.argtypes = [c_p, ctypes.c_char_p, ctypes.c_size_t,
                                             ctypes.POINTER(ctypes.c_uint64)] + tail
        lib.cuopus_server_wait.argtypes = [c_p, ctypes.c_uint64, ctypes.c_int64, c_p, ctypes.c_size_t,
                                           ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_double)] + tail
        lib.cuopus_server_get_stats.argtypes = [c_p, ctypes.POINTER(ServerStats)]
        lib.cuopus_server_request_size.argtypes = [c_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int64),
                                                   ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_size_t)]
        lib.cuopus_server_destroy.argtypes = [c_p]
        lib.cuopus_server_destroy.restype = None
        for f in ("cuopus_server_create", "cuopus_server_submit", "cuopus_server_wait", "cuopus_server_get_stats",
                  "cuopus_server_request_size"):
            getattr(lib, f).restype = ctypes.c_int
        lib._srv_bound = True
    return lib


class Server:
    def __init__(self, budget_bytes=40 << 30, width=0, block=0, max_inflight=0, wave_chains=0, seg_s=1.0,
                 preroll_ms=250.0, f16k=False):
        self.f16k = bool(f16k)
        cfg = ServerConfig(int(budget_bytes), int(width), int(block), int(max_inflight), int(wave_chains),
                           float(seg_s), float(preroll_ms), int(self.f16k))
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = _lib().cuopus_server_create(ctypes.byref(cfg), ctypes.byref(self._h), err, 512)
        if rc:
            raise cn.CuopusError(rc, err.value.decode(errors="replace"))
        self._sizes = {}

    def submit(self, ogg):
        """Queue one Ogg Opus stream (bytes or path); returns its request id."""
        data = cn._as_bytes(ogg)
        rid = ctypes.c_uint64(0)
        err = ctypes.create_string_buffer(512)
        rc = _lib().cuopus_server_submit(self._h, data, len(data), ctypes.byref(rid), err, 512)
        if rc:
            raise cn.CuopusError(rc, err.value.decode(errors="replace"))
        # the output size, from the server's own demux of the request
        nbytes = ctypes.c_size_t(0)
        rc = _lib().cuopus_server_request_size(self._h, rid.value, None, None, ctypes.byref(nbytes))
        if rc:
            raise cn.CuopusError(rc, "request %d: no size" % rid.value)
        self._sizes[rid.value] = max(int(nbytes.value), 4)
        return rid.value

    def wait(self, rid, timeout_ms=-1):
        """(numpy output, channels, latency ms) of a request; releases it."""
        cap = self._sizes.pop(rid, 0)
        buf = np.empty(max(cap, 4), np.uint8)
        n = ctypes.c_int64(0)
        ch = ctypes.c_int32(0)
        lat = ctypes.c_double(0)
        err = ctypes.create_string_buffer(512)
        rc = _lib().cuopus_server_wait(self._h, int(rid), int(timeout_ms), buf.ctypes.data, buf.size,
                                       ctypes.byref(n), ctypes.byref(ch), ctypes.byref(lat), err, 512)
        if rc:
            raise cn.CuopusError(rc, err.value.decode(errors="replace"))
        # the buffer was sized from the server's demux, so the view is the whole output
        if self.f16k:
            out = buf[:4 * n.value].view(np.float32)
        else:
            out = buf[:2 * n.value * ch.value].view(np.int16)
        return out, ch.value, lat.value

    def stats(self):
        st = ServerStats()
        _lib().cuopus_server_get_stats(self._h, ctypes.byref(st))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self):
        if self._h:
            _lib().cuopus_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
