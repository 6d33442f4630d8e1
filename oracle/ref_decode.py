"""ctypes front end of the libopus chain-decode oracle (oracle/ref_driver.c).

TEST INFRASTRUCTURE.  decode_chains() runs the reference's vendored libopus
1.5.2 FIXED_POINT decoder with a fresh decoder per chain and returns, per chain,
the int16 PCM, per-packet sample counts and final ranges, and the stop status.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .corpus import ref_lib


def flatten(packets):
    """bytes blob + uint64 offsets + uint32 lengths of a packet list."""
    lens = np.array([len(p) for p in packets], dtype=np.uint32)
    off = np.zeros(len(packets), dtype=np.uint64)
    if len(packets) > 1:
        off[1:] = np.cumsum(lens[:-1], dtype=np.uint64)
    blob = np.frombuffer(b"".join(packets) or b"\0", dtype=np.uint8).copy()
    return blob, off, lens


def decode_chains(packets, chains, channels, nthreads=None, want_pcm=True, fec=0):
    """chains: sequence of (first, npkts[, trim, keep]) over `packets`.
    fec=1: in-band FEC for a lost (empty) packet followed by a non-empty one.

    Returns dict(pcm=list of int16 arrays (interleaved), nsamp=list of uint32
    arrays, rng=list of uint32 arrays, status=int32 array, samples=uint64 array)."""
    lib = ref_lib()
    blob, off, lens = flatten(packets)
    first = np.array([c[0] for c in chains], dtype=np.uint32)
    npk = np.array([c[1] for c in chains], dtype=np.uint32)
    nch = len(chains)
    rec_off = np.zeros(nch, dtype=np.uint64)
    if nch > 1:
        rec_off[1:] = np.cumsum(npk[:-1], dtype=np.uint64)
    cap = np.array([sum(_toc(packets[int(first[i]) + k]) for k in range(int(npk[i])))
                    for i in range(nch)], dtype=np.uint64)
    pcm_off = np.zeros(nch, dtype=np.uint64)
    if nch > 1:
        pcm_off[1:] = np.cumsum(cap[:-1] * channels, dtype=np.uint64)
    total = int(cap.sum()) * channels
    pcm = np.zeros(max(total, 1), dtype=np.int16) if want_pcm else None
    nrec = int(npk.sum())
    nsamp = np.zeros(max(nrec, 1), dtype=np.uint32)
    rng = np.zeros(max(nrec, 1), dtype=np.uint32)
    status = np.zeros(max(nch, 1), dtype=np.int32)
    samples = np.zeros(max(nch, 1), dtype=np.uint64)
    rc = lib.oref_decode_chains_fec(
        blob.ctypes.data, off.ctypes.data, lens.ctypes.data, first.ctypes.data,
        npk.ctypes.data, nch, channels,
        pcm.ctypes.data if want_pcm else None, pcm_off.ctypes.data, rec_off.ctypes.data,
        nsamp.ctypes.data, rng.ctypes.data, status.ctypes.data, samples.ctypes.data,
        nthreads or (os.cpu_count() or 1), fec)
    if rc != 0:
        raise RuntimeError("oref_decode_chains failed to start threads")
    out = dict(status=status[:nch], samples=samples[:nch], pcm=[], nsamp=[], rng=[])
    for i in range(nch):
        r0, r1 = int(rec_off[i]), int(rec_off[i]) + int(npk[i])
        out["nsamp"].append(nsamp[r0:r1])
        out["rng"].append(rng[r0:r1])
        if want_pcm:
            p0 = int(pcm_off[i])
            out["pcm"].append(pcm[p0:p0 + int(samples[i]) * channels])
    return out


def _toc(p):
    from .ogg_port import decode_capacity48
    return decode_capacity48(p)


def check_batch(data, off, lens, first, npkts, chans, trim, keep, got_pcm, got_off, got_res, nthreads=None):
    """Full-size parity of a decoded batch against libopus (oref_check_chains):
    every chain decoded afresh and compared in place with the batch under test
    (int16 PCM of its keep window at got_off, and the {stop, samples,
    final_range} of its result record got_res [n, 4] uint32).  All arrays are
    host numpy arrays laid out as the decoder's chain table.  Returns dict
    with per-chain differing sample counts (bad) and flags (bit 0 stop, bit 1
    samples, bit 2 final range)."""
    lib = ref_lib()
    fn = lib.oref_check_chains
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int] + [ctypes.c_void_p] * 7 + [ctypes.c_int]
    c = lambda a, dt: np.ascontiguousarray(a, dtype=dt)
    data, off, lens = c(data, np.uint8), c(off, np.uint64), c(lens, np.uint32)
    first, npkts, chans = c(first, np.uint32), c(npkts, np.uint32), c(chans, np.uint8)
    trim, keep, got_off = c(trim, np.uint64), c(keep, np.uint64), c(got_off, np.uint64)
    got_pcm, got_res = c(got_pcm, np.int16), c(got_res, np.uint32)
    n = len(first)
    assert got_res.size >= 4 * n
    need = int((keep * chans.astype(np.uint64) + got_off).max()) if n else 0
    assert got_pcm.size >= need, "PCM buffer shorter than the chain table's windows"
    bad = np.zeros(max(n, 1), np.uint64)
    flags = np.zeros(max(n, 1), np.uint32)
    rc = fn(data.ctypes.data, off.ctypes.data, lens.ctypes.data, first.ctypes.data, npkts.ctypes.data,
            chans.ctypes.data, n, trim.ctypes.data, keep.ctypes.data, got_pcm.ctypes.data, got_off.ctypes.data,
            got_res.ctypes.data, bad.ctypes.data, flags.ctypes.data, nthreads or (os.cpu_count() or 1))
    if rc != 0:
        raise RuntimeError("oref_check_chains failed to start threads")
    return dict(bad=bad[:n], flags=flags[:n])
