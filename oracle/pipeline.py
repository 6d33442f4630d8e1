"""CPU restatement of the reference's decode pipelines, for the parity tests.

TEST INFRASTRUCTURE (oracle).
  f16k(ogg)   = cuopus_decode_f16k_on (reference libcuopus.cu:238-460):
                demux + chains (1 s, 250 ms preroll; cuopus_demux.h:293-378),
                libopus decode of every chain with a fresh decoder, keep
                windows concatenated (cuopus_kernels.cuh:75-88), then the
                49-tap resampler (oracle/resample_port.c) to
                max(0, (playable - 48) // 3) samples.
  i16(ogg)    = the same decode, returning interleaved int16 48 kHz PCM.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import ogg_port, ref_decode

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "liboracle_port.so")
_port = None


def port_lib():
    global _port
    if _port is None:
        if not os.path.exists(PORT_LIB):
            raise OSError("oracle/_build/liboracle_port.so missing: run make -C oracle port")
        lib = ctypes.CDLL(PORT_LIB)
        lib.orp_resample.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p]
        lib.orp_resample_f64.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p]
        lib.orp_make_taps.argtypes = [ctypes.c_void_p]
        _port = lib
    return _port


def taps():
    t = np.zeros(49, np.float32)
    port_lib().orp_make_taps(t.ctypes.data)
    return t


def resample(pcm16, n_out=None):
    x = np.ascontiguousarray(pcm16, dtype=np.int16)
    if n_out is None:
        n_out = max(0, (x.size - 48) // 3)
    y = np.zeros(max(n_out, 1), np.float32)
    if n_out > 0:
        port_lib().orp_resample(x.ctypes.data, x.size, n_out, y.ctypes.data)
    return y[:n_out]


def resample_f64(pcm16, n_out=None):
    x = np.ascontiguousarray(pcm16, dtype=np.int16)
    if n_out is None:
        n_out = max(0, (x.size - 48) // 3)
    y = np.zeros(max(n_out, 1), np.float64)
    if n_out > 0:
        port_lib().orp_resample_f64(x.ctypes.data, x.size, n_out, y.ctypes.data)
    return y[:n_out]


def i16(ogg, seconds=1.0, preroll_ms=250.0, nthreads=None):
    """(interleaved int16 playable PCM, channels, per-chain results)."""
    ix = ogg_port.demux(ogg)
    chains = ogg_port.build_chains(ix, seconds, preroll_ms)
    ch = ix["channels"]
    r = ref_decode.decode_chains(ix["packets"], chains, ch, nthreads=nthreads)
    parts = []
    for i, (first, npk, trim, keep) in enumerate(chains):
        if r["status"][i] != 0:
            raise RuntimeError("libopus failed on chain %d: %d" % (i, r["status"][i]))
        parts.append(r["pcm"][i][trim * ch:(trim + keep) * ch])
    pcm = np.concatenate(parts) if parts else np.zeros(0, np.int16)
    return pcm, ch, r


def f16k(ogg, nthreads=None):
    pcm, ch, _ = i16(ogg, 1.0, 250.0, nthreads)
    if ch != 1:
        raise ValueError("only mono supported (channels=%d)" % ch)
    return resample(pcm)
