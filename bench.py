#!/usr/bin/env python
"""Benchmark of the batched Opus decoder: audio-seconds decoded per second.

Default workload (mixed4096): the mixed-mode uneven batch - 4096 seeded
synthetic Ogg Opus streams with log-uniform lengths 1-30 s, forced SILK /
hybrid / CELT segments of 0.5-3 s, frames 2.5-60 ms, 6-128 kbps, mono or
stereo; one chain per stream, decoded bit-exactly to int16 48 kHz PCM.  The
reference's corpora are private; the streams come from the vendored libopus
encoder (oracle/corpus.py), generated before anything is timed.

A step is one decode of the whole batch.
  value      scheduled form: persistent grid pulling chains from a device work
             queue, longest first by the learned cost model, replayed as a CUDA
             graph, width x block and decoder warps per SM picked by the
             autotuner; packets and chain
             tables already in HBM; CUDA-event time on the launching stream
  plain      the plain one-launch form on the same batch: one warp per chain,
             one launch, chains in index order (the reference kernel's layout)
  e2e        through the public C ABI (cuopus_decode_i16_multi) from host Ogg
             bytes: demux, host->device copy, decode, and a device->host read of
             all decoded PCM into pinned memory, every step
  cpu_baseline  libopus 1.5.2 fixed point (the reference's own decoder,
             compiled from its vendored sources) on all host cores, bounded
             sample of the same workload
Other workloads: pareto16384 (learned scheduling), long7200 (2 h mono file
cut in 1 s chains, f16k), plain64, serve (Poisson arrivals through the
continuous-batching server against one launch per request).
--impl reference runs only the CPU decoder (the reference arm).

Under torchrun every rank decodes its own batch of the same shape (weak
scaling, no data exchange); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (corpus kind, count, max seconds, chain segment seconds)
    "mixed4096": ("mixed", 4096, 30.0, 1e9),
    # the cost model's training set for mixed4096: the same generator, other seeds
    "mixed1024train": ("mixed", 1024, 30.0, 1e9),
    "pareto16384": ("pareto", 16384, 120.0, 1e9),
    "plain64": ("plain64", 64, 1.0, 1.0),
    "long7200": ("long", 1, 7200.0, 1.0),
    "serve": ("lognormal", 384, 7200.0, 1.0),
}
METRIC = "audio-sec decoded/sec on 1 B200 (bit-exact)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------ inputs

# the cost model trains on another corpus than the one it orders
TRAIN_ON = {"mixed4096": "mixed1024train", "pareto16384": "mixed4096"}
# client threads of the serving measurement
SERVE_CLIENTS = 8


def load_inputs(workload, count=None):
    """Input preparation (never timed): generate or reuse the cached corpus."""
    from oracle.corpus import build_corpus
    kind, n, secs, seg = WORKLOADS[workload]
    t = time.time()
    paths = build_corpus(kind, os.path.join(ROOT, "corpus"), seed=4321 if workload.endswith("train") else 1234,
                         count=count or n, seconds=secs if kind != "plain64" else None)
    files = [open(p, "rb").read() for p in paths]
    log("corpus %s: %d files, %.1f MB, %.1fs" % (workload, len(files), sum(map(len, files)) / 1e6,
                                                 time.time() - t))
    return files, seg


class DeviceBatch:
    """Packets + chain table of all files, resident on the device."""

    def __init__(self, files, seg, device):
        import torch
        from cuopus_b200 import cuopus_native as cn
        blobs, offs, lens, first, npk, chans, trim, keep = [], [], [], [], [], [], [], []
        base_b = 0
        base_p = 0
        self.audio_s = 0.0
        self.file_play = []
        self.pkt_bytes = 0
        self.pcm_bytes = 0
        for f in files:
            ix = cn.index(f, seg_s=seg, preroll_ms=250.0)
            blobs.append(ix.blob)
            offs.append(ix.pkt_off + base_b)
            lens.append(ix.pkt_len)
            first.append(ix.first + base_p)
            npk.append(ix.npkts)
            chans.append(np.full(len(ix.first), ix.channels, np.uint8))
            trim.append(ix.trim.astype(np.uint64))
            keep.append(ix.keep.astype(np.uint64))
            base_b += len(ix.blob)
            base_p += len(ix.pkt_len)
            self.audio_s += ix.play48 / 48000.0
            self.file_play.append(int(ix.play48) * ix.channels)
            self.pcm_bytes += int(ix.play48) * ix.channels * 2
            for c in range(len(ix.first)):   # packet bytes decoded, preroll packets included
                a, b = int(ix.first[c]), int(ix.first[c]) + int(ix.npkts[c])
                self.pkt_bytes += int(ix.pkt_len[a:b].sum())
        cat = lambda xs: np.ascontiguousarray(np.concatenate(xs))
        first, npk, chans = cat(first), cat(npk), cat(chans)
        trim, keep = cat(trim), cat(keep)
        out_off = np.zeros(len(first), np.uint64)
        out_off[1:] = np.cumsum(keep[:-1] * chans[:-1].astype(np.uint64))
        self.n = len(first)
        self.cap_pkts = npk
        self.chans = chans
        self.keep = keep
        tot = int((keep * chans.astype(np.uint64)).sum())
        # host copies of the chain table: the full-size parity check after the
        # timed region decodes every chain on the CPU from these
        self.host = dict(blob=np.concatenate(blobs + [np.zeros(16, np.uint8)]), off=cat(offs), len=cat(lens),
                         first=first, npkts=npk, chans=chans, trim=trim, keep=keep, out_off=out_off)
        dev = torch.device(device)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.t = dict(blob=T(np.concatenate(blobs + [np.zeros(16, np.uint8)])), off=T(cat(offs)),
                      len=T(cat(lens)), first=T(first), npkts=T(npk), chans=T(chans), trim=T(trim),
                      keep=T(keep), out_off=T(out_off))
        self.out = torch.empty(max(tot, 1), dtype=torch.int16, device=dev)
        self.res = torch.zeros(4 * self.n, dtype=torch.int32, device=dev)

    def batch(self, width, schedule, order=None, block=0, graph=0, scalar=0):
        from cuopus_b200 import cuopus_native as cn
        b = cn.Batch()
        b.scalar = scalar
        t = self.t
        b.data, b.off, b.len = t["blob"].data_ptr(), t["off"].data_ptr(), t["len"].data_ptr()
        b.first, b.npkts, b.channels = t["first"].data_ptr(), t["npkts"].data_ptr(), t["chans"].data_ptr()
        b.trim, b.keep, b.out_off = t["trim"].data_ptr(), t["keep"].data_ptr(), t["out_off"].data_ptr()
        b.out, b.res = self.out.data_ptr(), self.res.data_ptr()
        b.nchains, b.width, b.schedule, b.max_groups = self.n, width, schedule, 0
        b.block, b.graph = block, graph
        self._order = None
        if order is not None:
            self._order = np.ascontiguousarray(np.asarray(order, np.uint32))
            b.order = self._order.ctypes.data
        return b

    def results(self):
        return self.res.view(-1, 4).cpu().numpy().view(np.uint32)


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return None
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ------------------------------------------------------------------ CPU (oracle) decode

def cpu_decode(files, seg, budget_s, threads):
    """libopus on host threads over a prefix of the workload; returns
    (audio-s/s, audio seconds decoded, seconds, files used)."""
    from oracle import ogg_port, ref_decode
    audio = 0.0
    used = 0
    elapsed = 0.0
    group = max(threads * 4, 16)      # decode in groups so the sample stays bounded
    while used < len(files) and elapsed < budget_s:
        chunk = files[used:used + group]
        pk_all, ch_all, chains_all = [], [], []
        for f in chunk:
            ix = ogg_port.demux(f)
            pk_all.append(ix["packets"])
            ch_all.append(ix["channels"])
            chains_all.append(ogg_port.build_chains(ix, seg, 250.0))
            audio += ix["play48"] / 48000.0
        t0 = time.time()
        for want_ch in (1, 2):          # one oracle call per channel count
            pk, chains = [], []
            base = 0
            for p, ch, cs in zip(pk_all, ch_all, chains_all):
                if ch != want_ch:
                    continue
                pk += p
                chains += [(c[0] + base, c[1], c[2], c[3]) for c in cs]
                base += len(p)
            if chains:
                ref_decode.decode_chains(pk, chains, want_ch, nthreads=threads)
        elapsed += time.time() - t0
        used += len(chunk)
    return audio / elapsed if elapsed > 0 else 0.0, audio, elapsed, used


# ------------------------------------------------------------------ full-size parity

def full_parity(db, threads, e2e_host):
    """Untimed check of the timed batch's output after the timed region:
    every chain decoded by libopus 1.5.2 fixed point on the host threads and
    compared in place (every int16 sample of its keep window, its stop status,
    sample count and final range: oref_check_chains).  The e2e output of the
    last e2e step must equal the batch's PCM (int16), or the resampler oracle
    over it with max abs diff 0 (f16k)."""
    from oracle import ref_decode
    t0 = time.time()
    got = db.out.cpu().numpy()
    res = db.results()
    h = db.host
    r = ref_decode.check_batch(h["blob"], h["off"], h["len"], h["first"], h["npkts"], h["chans"], h["trim"],
                               h["keep"], got, h["out_off"], res, nthreads=threads)
    fl = r["flags"]
    out = {"oracle": "libopus 1.5.2 fixed point (oracle/_ref), fresh decoder per chain",
           "chains_checked": int(db.n), "chains_total": int(db.n),
           "pcm_mismatches": int(r["bad"].sum()), "chains_with_pcm_mismatch": int((r["bad"] > 0).sum()),
           "range_mismatches": int(((fl & 4) != 0).sum()), "sample_count_mismatches": int(((fl & 2) != 0).sum()),
           "stop_mismatches": int(((fl & 1) != 0).sum()), "samples_compared": int(got.size)}
    if e2e_host is not None:
        kind, buf, sizes = e2e_host
        if kind == "i16":
            hb = buf.numpy()[:got.size]
            out["e2e_equals_batch"] = bool(hb.size == got.size and np.array_equal(hb, got))
        else:
            from oracle import pipeline
            hb = buf.numpy()
            o16 = o48 = 0
            worst = 0.0
            for f_i, n16 in enumerate(sizes):     # one file per f16k workload stream
                n48 = int(db.file_play[f_i])
                want = pipeline.resample(got[o48:o48 + n48], n16)
                worst = max(worst, float(np.abs(hb[o16:o16 + n16] - want).max()) if n16 else 0.0)
                o16 += n16
                o48 += n48
            out["e2e_f16k_max_abs_diff"] = worst
    out["seconds"] = round(time.time() - t0, 1)
    log("parity: %s" % json.dumps(out))
    return out


# ------------------------------------------------------------------ the reference's GPU library

def reference_gpu_bench(args, files, seg):
    """--impl reference-gpu: the reference's own libcuopus (built unchanged for
    sm_100a by oracle/Makefile ref_gpu) against this library on the same GPU,
    through the identical f16k call (cuopus_decode_f16k_multi, bound as the
    reference's Python module binds it), on the workload's mono files (the
    reference's GPU path is mono only), in groups of at most 2,048 chains of
    1 s (the reference's one-launch limit).  Host Ogg bytes in, float32 16 kHz
    in device memory out, stream synchronised: end-to-end time, K steps after
    W warm-up steps, both libraries alternating step by step.  Outputs must
    be identical."""
    import ctypes
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_dropin import bind
    from cuopus_b200 import cuopus_native as cn
    ref_path = os.path.join(ROOT, "oracle", "_ref", "libcuopus_refgpu.so")
    if not os.path.exists(ref_path):
        return {"unavailable": "oracle/_ref/libcuopus_refgpu.so is not built (make -C oracle ref_gpu)"}
    torch.cuda.set_device(0)
    mono = [f for f in files if cn.probe_pcm(f)[1] == 1]
    chains = [len(cn.index(f, seg_s=1.0).first) for f in mono]
    groups, cur, cnt = [], [], 0
    for f, c in zip(mono, chains):
        if cur and cnt + c > 2048:
            groups.append(cur)
            cur, cnt = [], 0
        cur.append(f)
        cnt += c
    if cur:
        groups.append(cur)
    audio = sum(cn.probe_pcm(f)[0] for f in mono) / 48000.0
    stream = torch.cuda.current_stream()
    libs = {"reference": bind(ref_path), "ours": bind(os.path.join(ROOT, "cuopus_b200", "lib", "libcuopus.so"))}
    os.environ.setdefault("CUOPUS_SEG_S", "1")
    n16s = [[cn.probe(f) for f in g] for g in groups]
    outs = [[torch.empty(max(k, 1), dtype=torch.float32, device="cuda") for k in n] for n in n16s]
    err = ctypes.create_string_buffer(512)

    def step(lib):
        for g, n16, o in zip(groups, n16s, outs):
            n = len(g)
            ba = (ctypes.c_char_p * n)(*g)
            la = (ctypes.c_size_t * n)(*[len(f) for f in g])
            oa = (ctypes.c_void_p * n)(*[t.data_ptr() for t in o])
            ca = (ctypes.c_size_t * n)(*n16)
            ol = (ctypes.c_int64 * n)()
            rc = lib.cuopus_decode_f16k_multi(ba, la, n, oa, ca, ol, ctypes.c_void_p(stream.cuda_stream), err, 512)
            if rc:
                raise RuntimeError(err.value.decode())
        torch.cuda.synchronize()

    times = {k: [] for k in libs}
    for i in range(args.warmup + args.steps):
        for name, lib in libs.items():
            t0 = time.perf_counter()
            step(lib)
            if i >= args.warmup:
                times[name].append(time.perf_counter() - t0)
    # the last step of each library: identical samples
    same = True
    keep = [[t.cpu().numpy() for t in o] for o in outs]
    step(libs["reference"])
    for o, k in zip(outs, keep):
        for t, a in zip(o, k):
            same = same and np.array_equal(t.cpu().numpy(), a)
    med = {k: statistics.median(v) for k, v in times.items()}
    return {"files": len(mono), "groups": len(groups), "chains": int(sum(chains)), "audio_s": round(audio, 1),
            "reference": {"value": audio / med["reference"], "ms_per_step": med["reference"] * 1e3},
            "ours": {"value": audio / med["ours"], "ms_per_step": med["ours"] * 1e3},
            "speedup": med["reference"] / med["ours"], "identical_output": bool(same),
            "call": "cuopus_decode_f16k_multi (reference binding), 1 s chains, 250 ms preroll"}


# ------------------------------------------------------------------ helpers

def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def profile_traffic():
    """DRAM bytes per algorithmic byte of the decode kernel, from the committed
    ncu summary (profiles/k_decode_chains_traffic.json), or None."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "k_decode_chains_traffic.json")))
        return float(d["dram_bytes"]) / float(d["algorithmic_bytes"])
    except (OSError, ValueError, KeyError, ZeroDivisionError):
        return None


def timed_steps(cn, b, stream, steps):
    """K engine calls between two events on the stream; per-call kernel ms."""
    import torch
    kern = []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        kern.append(cn.decode_batch(b, stream.cuda_stream))
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, kern


def train_cost_model(args, stream):
    """The cost model of the scheduled form, trained (untimed) on another
    corpus than the timed batch (TRAIN_ON): that corpus is decoded once with
    the queue schedule in packet-count order, the decoder's per-chain decode
    times are the targets, and the MLP is trained on the GPU."""
    import torch
    from cuopus_b200 import costmodel
    from cuopus_b200 import cuopus_native as cn
    name = TRAIN_ON.get(args.workload, "mixed1024train")
    files, seg = load_inputs(name)
    tb = DeviceBatch(files, seg, stream.device)
    b = tb.batch(32, 1, costmodel.packet_order(tb.cap_pkts, tb.chans), 128, 0)
    cn.decode_batch(b, stream.cuda_stream)
    torch.cuda.synchronize()
    times = np.maximum(tb.results()[:, 3].astype(np.float64), 1.0)
    feats = costmodel.chain_features(b)
    model = costmodel.CostModel(seed=1)
    t0 = time.time()
    losses = model.fit(feats, times, steps=1500, lr=3e-3)
    train_s = time.time() - t0
    y, yh = np.log(times), np.log(model.predict(feats))
    r2 = 1.0 - np.sum((y - yh) ** 2) / np.sum((y - y.mean()) ** 2)
    del tb, b, feats
    torch.cuda.empty_cache()
    return model, {"train_corpus": name, "train_chains": int(len(times)), "train_s": round(train_s, 2),
                   "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
                   "r2_log_time_train": round(float(r2), 4)}


def compare_orders(cn, db, stream, b, info, reps=2):
    """Untimed comparison of visiting orders on the timed batch with the
    tuned launch: queue-schedule kernel time in learned and in packet-count
    order, and each order's makespan as the scheduler predicts it (list
    scheduling of the predicted, resp. packet-count-fitted, chain costs on the
    launch's decoder groups) against the measured kernel time."""
    import torch
    from cuopus_b200 import costmodel
    pred = info.pop("_pred", None)
    out = {}
    orders = {"packets": costmodel.packet_order(db.cap_pkts, db.chans)}
    if pred is not None:
        orders["learned"] = np.argsort(-pred, kind="stable")
    keep = b.order
    times = None
    for name, order in orders.items():
        arr = np.ascontiguousarray(order.astype(np.uint32))
        b.order = arr.ctypes.data
        ms = [cn.decode_batch(b, stream.cuda_stream) for _ in range(reps)]
        torch.cuda.synchronize()
        t = db.results()[:, 3].astype(np.float64)
        times = t if times is None else times
        out[name] = {"kernel_ms": float(min(ms))}
    b.order = keep
    groups = b.max_groups if b.max_groups > 0 else None
    if groups is None:
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        groups = sms * 8 * (32 // b.width)
    # per-chain costs in the unit of the measured chain times (us); the
    # packet-count fallback predicts cost proportional to packets x channels,
    # scaled to the measured total
    w = db.cap_pkts.astype(np.float64) * db.chans.astype(np.float64)
    pk_cost = w * (times.sum() / w.sum())
    out["packets"]["predicted_ms"] = costmodel.makespan(pk_cost, orders["packets"], groups) / 1e3
    if pred is not None:
        lt = np.log(np.maximum(times, 1.0))
        r2 = 1.0 - np.sum((lt - np.log(pred)) ** 2) / np.sum((lt - lt.mean()) ** 2)
        out["learned"]["predicted_ms"] = costmodel.makespan(pred, orders["learned"], groups) / 1e3
        out["r2_log_time_on_this_batch"] = round(float(r2), 4)
        out["learned_over_packets"] = out["packets"]["kernel_ms"] / out["learned"]["kernel_ms"]
    out["decoder_groups"] = int(groups)
    out["longest_chain_ms"] = float(times.max() / 1e3)
    return out


def schedule_batch(cn, db, stream, args):
    """Warm-up work of the scheduled form (untimed): plain form timing, cycle
    recording, cost model training, autotuning.  Returns (batch, info)."""
    import torch
    from cuopus_b200 import costmodel
    info = {}
    # plain one-launch forms, one warp per chain, index order: the reference
    # kernel's layout (one lane of the warp decodes) and with the lanes
    # splitting the independent loops
    reps = max(1, min(args.steps, 2))
    plain_ref = db.batch(32, 2, None, 128, 0, scalar=1)
    cn.decode_batch(plain_ref, stream.cuda_stream)
    torch.cuda.synchronize()
    ref_ms, _ = timed_steps(cn, plain_ref, stream, reps)
    plain_b = db.batch(32, 2, None, 128, 0)
    cn.decode_batch(plain_b, stream.cuda_stream)
    torch.cuda.synchronize()
    plain_ms, _ = timed_steps(cn, plain_b, stream, reps)
    info["plain"] = {"ms_per_step": ref_ms, "value": db.audio_s / (ref_ms / 1e3), "width": 32, "block": 128,
                     "schedule": "plain one-launch, one warp per chain, one lane decoding, index order",
                     "lane_split": {"ms_per_step": plain_ms, "value": db.audio_s / (plain_ms / 1e3),
                                    "schedule": "plain one-launch, one warp per chain, 32 lanes, index order"}}
    # learned order (the packet-count order is the fallback)
    order = costmodel.packet_order(db.cap_pkts, db.chans)
    info["order"] = "packets x channels"
    if args.order == "mlp":
        model, info["cost_model"] = train_cost_model(args, stream)
        feats = costmodel.chain_features(plain_b)
        pred = model.predict(feats)
        order = np.argsort(-pred, kind="stable")
        info["order"] = "learned (MLP 16-64-64-1, trained on %s)" % info["cost_model"]["train_corpus"]
        info["_pred"] = pred
    # autotune width x block on the scheduled form, then the decoder warps per SM
    width, block = args.width, args.block
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    max_groups = args.warps_per_sm * sms * (32 // width) if args.warps_per_sm > 0 else 0
    sched = {"queue": 1, "static": 0, "plain": 2}[args.schedule]
    if not args.no_tune:
        b = db.batch(32, 1, order, 128, 1)
        width, block, table = cn.autotune(b, widths=(8, 16, 32), blocks=(64, 128), reps=1,
                                          stream=stream.cuda_stream)
        info["autotune"] = {"%dx%d" % k: (round(v, 1) if v else None) for k, v in table.items()}
        if sched != 2:
            b = db.batch(width, sched, order if sched == 1 else None, block, 1)
            max_groups, occ = cn.autotune_occupancy(b, warps_per_sm=(0, 7, 6, 5, 4), reps=2,
                                                    stream=stream.cuda_stream)
            info["autotune_warps_per_sm"] = {str(k): (round(v, 1) if v else None) for k, v in occ.items()}
    b = db.batch(width, sched, order if sched == 1 else None, block, 1 if sched != 2 else 0)
    b.max_groups = max_groups
    if not args.no_tune and sched == 1 and width == 32:
        # tail scheduling: the longest chains alone on SMs of their own
        light, tails = cn.autotune_tail(b, light=(0, 8, 16, 32), reps=2, stream=stream.cuda_stream)
        info["autotune_light_sms"] = {str(k): round(v, 1) for k, v in tails.items()}
    info.update(width=width, block=block, max_groups=max_groups, light_sms=b.light_sms)
    if sched == 1:
        info["orders"] = compare_orders(cn, db, stream, b, info)
    info.pop("_pred", None)
    return b, info


# ------------------------------------------------------------------ serving workload

def serve_bench(args, files, dev):
    """Poisson arrivals through the continuous-batching server at each rate of
    --rates, against the plain form that decodes one request per launch in
    arrival order (the reference daemon's loop), both on the same arrival
    schedule and files.  Per rate: sustained audio-s/s (all requests' audio /
    first arrival to last completion) and p50 / p99 latency (arrival to
    result in host memory)."""
    import ctypes
    import torch
    from cuopus_b200 import cuopus_native as cn
    from cuopus_b200.serving import Server
    n = len(files)
    play = [cn.probe_pcm(f) for f in files]
    audio = [p / 48000.0 for p, _ in play]
    total_audio = float(sum(audio))
    rates = [float(r) for r in args.rates.split(",")]
    out = {"requests": n, "audio_s": total_audio, "longest_request_s": max(audio), "rates": {}}
    stream = torch.cuda.current_stream()
    caps = [p * c for p, c in play]
    buf = torch.empty(max(caps), dtype=torch.int16, device=dev)
    host = torch.empty(max(caps), dtype=torch.int16, pin_memory=True)
    lib = cn.lib()
    err = ctypes.create_string_buffer(512)
    with Server(budget_bytes=args.budget_gb << 30, width=args.serve_width, block=64,
                max_inflight=args.serve_inflight) as srv:
        srv.wait(srv.submit(files[0]))                      # warm-up (context, slots)
        for ri, rate in enumerate(rates):
            rng = np.random.default_rng(7 + ri)
            arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
            # continuous batching
            ids = [None] * n
            done_at = [0.0] * n
            t0 = time.perf_counter()

            # clients: each of SERVE_CLIENTS threads waits for every
            # SERVE_CLIENTS-th request in arrival order, so that one long
            # request does not hold back the results of the ones behind it
            def waiter(k):
                for i in range(k, n, SERVE_CLIENTS):
                    while ids[i] is None:
                        time.sleep(0.0002)
                    srv.wait(ids[i])
                    done_at[i] = time.perf_counter() - t0

            ths = [threading.Thread(target=waiter, args=(k,)) for k in range(SERVE_CLIENTS)]
            for th in ths:
                th.start()
            for i in range(n):
                d = arrivals[i] - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
                ids[i] = srv.submit(files[i])
            for th in ths:
                th.join()
            lat = (np.array(done_at) - arrivals) * 1e3
            wall = max(done_at)
            served = {"value": total_audio / wall, "p50_ms": float(np.percentile(lat, 50)),
                      "p99_ms": float(np.percentile(lat, 99)), "wall_s": wall}
            if args.serve_no_plain:
                out["rates"][str(int(rate))] = {"offered_audio_s_per_s": total_audio / float(arrivals[-1]),
                                                "served": served}
                log("serve %g/s: served %.0f audio-s/s p50 %.0f p99 %.0f ms" % (rate, served["value"],
                                                                             served["p50_ms"], served["p99_ms"]))
                continue
            # one launch per request, arrival order, one at a time
            lat2 = []
            t0 = time.perf_counter()
            for i, f in enumerate(files):
                d = arrivals[i] - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
                ba = (ctypes.c_char_p * 1)(f)
                la = (ctypes.c_size_t * 1)(len(f))
                oa = (ctypes.c_void_p * 1)(buf.data_ptr())
                ca = (ctypes.c_size_t * 1)(caps[i])
                ol = (ctypes.c_int64 * 1)()
                oc = (ctypes.c_int32 * 1)()
                rc = lib.cuopus_decode_i16_multi(ba, la, 1, oa, ca, ol, oc, ctypes.c_void_p(stream.cuda_stream),
                                                 err, 512)
                if rc:
                    raise RuntimeError(err.value.decode())
                host[:caps[i]].copy_(buf[:caps[i]], non_blocking=True)
                torch.cuda.synchronize()
                lat2.append((time.perf_counter() - t0 - arrivals[i]) * 1e3)
            wall2 = time.perf_counter() - t0
            lat2 = np.array(lat2)
            plain = {"value": total_audio / wall2, "p50_ms": float(np.percentile(lat2, 50)),
                     "p99_ms": float(np.percentile(lat2, 99)), "wall_s": wall2}
            out["rates"][str(int(rate))] = {"offered_audio_s_per_s": total_audio / float(arrivals[-1]),
                                            "served": served, "one_launch_per_request": plain,
                                            "throughput_ratio": served["value"] / plain["value"]}
            log("serve %g/s: served %.0f audio-s/s p50 %.0f p99 %.0f ms | one launch per request %.0f audio-s/s "
                "p50 %.0f p99 %.0f ms" % (rate, served["value"], served["p50_ms"], served["p99_ms"], plain["value"],
                                          plain["p50_ms"], plain["p99_ms"]))
        st = srv.stats()
        out["server"] = {"waves": st["waves"], "wave_chains": st["wave_chains"], "width": args.serve_width,
                         "max_inflight": args.serve_inflight, "budget_gb": args.budget_gb}
    return out


def fit_order(args):
    """Weights of the file entry points' visiting order (csrc/ordercost.cpp):
    the training corpus (never a timed workload) is cut in 1 s chains with
    250 ms preroll, as the file entry points cut, and decoded three times at 8
    and at 32 lanes per chain with the library's launch (64-thread blocks,
    queue schedule; every decoder group at 8 lanes, 5 warps per SM at 32); the
    median of each chain's recorded device time is the target of a
    non-negative least-squares fit on the chain's features.  Writes the
    weights to args.fit_order and prints one JSON line of fit statistics."""
    import torch
    from cuopus_b200 import cuopus_native as cn
    from cuopus_b200 import ordercost
    torch.cuda.set_device(0)
    cn.warmup()
    name = "mixed1024train"
    files, _ = load_inputs(name)
    db = DeviceBatch(files, 1.0, "cuda:0")
    stream = torch.cuda.current_stream()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    feats = ordercost.features(db.host)
    samples = db.keep.astype(np.float64) * db.chans
    order = np.argsort(-samples, kind="stable")
    out = {"train_corpus": name, "chains": int(db.n), "audio_s": round(db.audio_s, 1)}
    w = {}
    for width in (8, 32):
        b = db.batch(width, 1, order, 64, 0)
        b.max_groups = 5 * sms if width == 32 else 0
        runs = []
        for _ in range(3):
            cn.decode_batch(b, stream.cuda_stream)
            torch.cuda.synchronize()
            runs.append(db.results()[:, 3].astype(np.float64))
        t = np.median(np.stack(runs), axis=0)
        w[width], st = ordercost.fit(feats, t)
        st["mean_chain_us"] = round(float(t.mean()), 1)
        out["w%d" % width] = st
    ordercost.write_coefficients(args.fit_order, w[8], w[32], out)
    out["weights_us"] = {"w%d" % k: dict(zip(ordercost.FEATURE_NAMES, [round(float(x), 3) for x in v]))
                         for k, v in w.items()}
    print(json.dumps(out), flush=True)
    return 0


# ------------------------------------------------------------------ main

def phases_report(args):
    """Split of the decoder's time between its stages, from the stage timers of
    the diagnostic build: one decode of the workload in the lane-split form
    (the --width / --block given, packet-count order, queue schedule), one in
    the one-lane layout with the same order and schedule, and one in the
    one-lane reference layout (plain one-launch form, index order).  Prints one JSON line (not a bench line:
    the timers cost time of their own)."""
    import torch
    from cuopus_b200 import cuopus_native as cn
    # before the library is first loaded; a CUOPUS_LIB already set must name a
    # stage-timer build
    os.environ.setdefault("CUOPUS_LIB", cn.phases_lib_path())
    from cuopus_b200 import costmodel
    torch.cuda.set_device(0)
    files, seg = load_inputs(args.workload, args.count)
    cn.warmup()
    db = DeviceBatch(files, seg, "cuda:0")
    stream = torch.cuda.current_stream()
    order = costmodel.packet_order(db.cap_pkts, db.chans)
    # DeviceBatch.batch() keeps the order array of the latest batch alive only,
    # so each batch is made right before its use
    forms = {"lane_split": lambda: db.batch(args.width, 1, order, args.block, 0),
             "one_lane_queue": lambda: db.batch(32, 1, order, 128, 0, scalar=1),
             "one_lane": lambda: db.batch(32, 2, None, 128, 0, scalar=1)}
    out = {"report": "decoder stage cycles", "workload": args.workload, "chains": db.n,
           "audio_s": round(db.audio_s, 1), "width": args.width, "block": args.block}
    for name, make in forms.items():
        b = make()
        cn.decode_batch(b, stream.cuda_stream)     # warm
        torch.cuda.synchronize()
        cn.phase_reset()
        ms = cn.decode_batch(b, stream.cuda_stream)
        torch.cuda.synchronize()
        ph = cn.phase_cycles()
        chain_us = float(db.results()[:, 3].astype(np.float64).sum())
        tot = float(ph["packet"]) or 1.0
        out[name] = {"kernel_ms_with_timers": round(ms, 2), "chain_seconds": round(chain_us / 1e6, 2),
                     "cycles_per_audio_s": {k: round(v / db.audio_s) for k, v in ph.items()},
                     "share_of_packet": {k: round(v / tot, 4) for k, v in ph.items() if k != "packet"}}
        log(name, json.dumps(out[name]["share_of_packet"]))
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"],
                    help="reference: libopus on the host cores (the reference arm); reference-gpu: the "
                         "reference's own CUDA library against this one on the same GPU (mono files, f16k)")
    ap.add_argument("--workload", default="mixed4096", choices=sorted(WORKLOADS))
    ap.add_argument("--count", type=int, default=None, help="override the stream count (development)")
    ap.add_argument("--seg", type=float, default=None,
                    help="override the chain length in seconds (1e9: whole streams); small profiling cases")
    ap.add_argument("--width", type=int, default=32, help="lanes per chain when not autotuned")
    ap.add_argument("--block", type=int, default=128, help="threads per block when not autotuned")
    ap.add_argument("--warps-per-sm", type=int, default=0, help="decoder warps per SM when not autotuned (0 = all)")
    ap.add_argument("--schedule", default="queue", choices=["queue", "static", "plain"])
    ap.add_argument("--order", default="mlp", choices=["mlp", "packets"])
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the full-size parity check (development)")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--rates", default="50,100,250,500", help="serve: Poisson arrival rates per second")
    ap.add_argument("--serve-width", type=int, default=8, help="serve: lanes per chain of the server")
    ap.add_argument("--serve-inflight", type=int, default=8, help="serve: decode waves in flight")
    ap.add_argument("--budget-gb", type=int, default=40, help="serve: admission budget")
    ap.add_argument("--serve-no-plain", action="store_true",
                    help="serve: skip the one-launch-per-request comparison (development sweeps)")
    ap.add_argument("--phases", action="store_true",
                    help="diagnostics, not a bench line: per-stage decoder cycles from libcuopus_phases.so")
    ap.add_argument("--fit-order", metavar="INC", default=None,
                    help="not a bench line: fit the file entry points' visiting-order weights on the training "
                         "corpus and write them to INC (cuopus_b200/csrc/ordercost_coef.inc)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            return 0
        files, seg = load_inputs(args.workload, args.count)
        rates, els = [], []
        for i in range(args.warmup + args.steps):
            r, audio, el, used = cpu_decode(files, seg, args.cpu_budget / 2, threads)
            if i >= args.warmup:
                rates.append(r)
                els.append(el)
        v = statistics.median(rates)
        line = {"metric": METRIC, "value": v, "unit": "audio-s/s", "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.median(els) * 1e3,
                "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int16",
                "data": "synthetic (seeded, vendored libopus encoder)",
                "config": {"workload": args.workload, "sample_files": used},
                "cpu_baseline": {"value": v, "unit": "audio-s/s", "cores": threads, "kind": "reference",
                                 "sample": "libopus 1.5.2 fixed point, %d host threads, first %d streams "
                                           "(%.0f audio-s) per step" % (threads, used, audio)},
                "e2e": {"value": v, "unit": "audio-s/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    if args.phases:
        return phases_report(args)
    if args.fit_order:
        return fit_order(args)

    if args.impl == "reference-gpu":
        if rank != 0:
            return 0
        files, seg = load_inputs(args.workload, args.count)
        with ClockSampler(local) as clk:
            r = reference_gpu_bench(args, files, seg)
        line = {"metric": METRIC, "impl": "reference-gpu", "unit": "audio-s/s", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "dtype": "int16 decode, float32 16 kHz output",
                "data": "synthetic (seeded, vendored libopus encoder)",
                "config": {"workload": args.workload, "files": "mono files of the workload"},
                "value": r.get("reference", {}).get("value"), "compare": r, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = "cuda:%d" % local
    from cuopus_b200 import cuopus_native as cn

    files, seg = load_inputs(args.workload, args.count)
    if args.seg:
        seg = args.seg
    cn.warmup()

    if args.workload == "serve":
        with ClockSampler(local) as clk:
            r = serve_bench(args, files, dev)
        if rank == 0:
            top = r["rates"][max(r["rates"], key=float)]
            s = top["served"]
            line = {"metric": METRIC, "value": s["value"], "unit": "audio-s/s", "n_gpus": world, "steps": 1,
                    "warmup": 1, "ms_per_step": s["wall_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "int16", "data": "synthetic (seeded, vendored libopus encoder)",
                    "config": {"workload": "serve", "requests": r["requests"], "arrivals_per_s": args.rates,
                               "lengths": "log-normal median 30 s, sigma 1, clipped to [5 s, 2 h]; longest %.0f s"
                                          % r["longest_request_s"],
                               "budget_gb": args.budget_gb},
                    "latency_ms": {"p50": s["p50_ms"], "p99": s["p99_ms"]}, "serve": r, "clocks": clk.summary()}
            print(json.dumps(line), flush=True)
        return 0

    db = DeviceBatch(files, seg, dev)
    stream = torch.cuda.current_stream()
    b, info = schedule_batch(cn, db, stream, args)
    for _ in range(args.warmup):
        cn.decode_batch(b, stream.cuda_stream)
    res = db.results()
    bad = int((res[:, 0] != 0).sum())
    if bad:
        log("WARNING: %d chains stopped with a decode error" % bad)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        step_ms, kern = timed_steps(cn, b, stream, args.steps)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([step_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms = float(t.item())
    barrier()
    value = world * db.audio_s / (step_ms / 1e3)
    kern_ms = statistics.mean(kern)
    # the makespan floor: the most expensive single chain, from the decode time
    # the decoder records per chain
    us = db.results()[:, 3].astype(np.float64)
    tail = {"longest_chain_ms": float(us.max() / 1e3), "chain_seconds_total": float(us.sum() / 1e6),
            "kernel_ms": kern_ms}
    alg_bytes = db.pkt_bytes + db.pcm_bytes
    pk = peaks()
    peak = pk.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9
    ratio = profile_traffic()

    # e2e through the C ABI from host bytes, PCM read back to pinned host memory
    e2e = None
    e2e_host = None
    if not args.no_e2e:
        import ctypes
        play = [cn.probe_pcm(f) for f in files]
        caps = [p * c for p, c in play]
        # the files' outputs back to back in one device buffer, read back with one copy
        out_all = torch.empty(max(sum(caps), 1), dtype=torch.int16, device=dev)
        bounds = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
        outs = [out_all[int(bounds[i]):int(bounds[i + 1])] for i in range(len(caps))]
        host = torch.empty(max(sum(caps), 1), dtype=torch.int16, pin_memory=True)
        lib = cn.lib()
        n = len(files)
        ba = (ctypes.c_char_p * n)(*files)
        la = (ctypes.c_size_t * n)(*[len(f) for f in files])
        oa = (ctypes.c_void_p * n)(*[o.data_ptr() for o in outs])
        ca = (ctypes.c_size_t * n)(*caps)
        ol = (ctypes.c_int64 * n)()
        oc = (ctypes.c_int32 * n)()
        err = ctypes.create_string_buffer(512)
        os.environ["CUOPUS_SEG_S"] = str(seg)
        os.environ["CUOPUS_MAX_BATCH"] = str(10 ** 8)
        os.environ["CUOPUS_DEMUX_THREADS"] = str(threads)     # demux the files on every host core

        f16k = args.workload == "long7200"
        if f16k:     # the drop-in f16k path: float32 16 kHz output, read back
            n16 = [cn.probe(f) for f in files]
            outs16 = [torch.empty(max(c, 1), dtype=torch.float32, device=dev) for c in n16]
            host16 = torch.empty(max(sum(n16), 1), dtype=torch.float32, pin_memory=True)
            oa16 = (ctypes.c_void_p * n)(*[o.data_ptr() for o in outs16])
            ca16 = (ctypes.c_size_t * n)(*n16)

        def e2e_step():
            if f16k:
                rc = lib.cuopus_decode_f16k_multi(ba, la, n, oa16, ca16, ol, ctypes.c_void_p(stream.cuda_stream),
                                                  err, 512)
                if rc:
                    raise RuntimeError(err.value.decode())
                o = 0
                for t_, c in zip(outs16, n16):
                    host16[o:o + c].copy_(t_[:c], non_blocking=True)
                    o += c
                torch.cuda.synchronize()
                return
            rc = lib.cuopus_decode_i16_multi(ba, la, n, oa, ca, ol, oc, ctypes.c_void_p(stream.cuda_stream),
                                             err, 512)
            if rc:
                raise RuntimeError(err.value.decode())
            host.copy_(out_all, non_blocking=True)
            torch.cuda.synchronize()

        for _ in range(2):
            e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        e2e_s = (time.perf_counter() - t0) / args.steps
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([e2e_s], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        last = {k: (round(v, 2) if isinstance(v, float) else v) for k, v in cn.last_stats().items()}
        # the library's visiting order against the order by decoded samples
        # (one untimed call each way, same inputs)
        from cuopus_b200 import ordercost
        orders = {"model": "fitted additive cost" if ordercost.fitted() else "unfitted default (samples)"}
        for name, env in (("cost", None), ("samples", "samples")):
            if env:
                os.environ["CUOPUS_ORDER"] = env
            e2e_step()
            os.environ.pop("CUOPUS_ORDER", None)
            orders[name + "_kernel_ms"] = round(cn.last_stats()["kernel_ms"], 2)
        e2e_host = ("f16k", host16, n16) if f16k else ("i16", host, caps)
        e2e = {"value": world * db.audio_s / e2e_s, "unit": "audio-s/s",
               "h2d_bytes_per_step": int(sum(map(len, files))),
               "d2h_bytes_per_step": int(4 * sum(n16)) if f16k else int(2 * sum(caps)),
               "ms_per_step": e2e_s * 1e3, "api": "cuopus_decode_f16k_multi (float32 16 kHz)" if f16k else
               "cuopus_decode_i16_multi (int16 48 kHz)", "demux_threads": threads,
               "last_call": last, "library_order": orders}

    # full-size parity (after every timed region, untimed): every chain of the
    # timed batch against libopus, and the e2e output against the batch
    parity = None
    if rank == 0 and not args.no_parity:
        parity = full_parity(db, threads, e2e_host)

    cpu = None
    if rank == 0 and world == 1 and args.cpu_budget > 0:
        r, audio, el, used = cpu_decode(files, seg, args.cpu_budget, threads)
        cpu = {"value": r, "unit": "audio-s/s", "cores": threads, "kind": "reference",
               "sample": "libopus 1.5.2 fixed point on %d host threads: first %d of %d streams (%.0f audio-s, %.1fs)"
                         % (threads, used, len(files), audio, el)}

    if rank == 0:
        plain = info.pop("plain")
        line = {"metric": METRIC, "value": value, "unit": "audio-s/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int16", "data": "synthetic (seeded, vendored libopus encoder)",
                "config": {"workload": args.workload, "streams": len(files), "chains": db.n,
                           "audio_s_per_gpu": round(db.audio_s, 1), "schedule": args.schedule, **info,
                           "l2": "inputs and outputs exceed L2 (no flush needed)"},
                "plain": {**plain, "value": world * plain["value"], "speedup_of_scheduled": value /
                          (world * plain["value"]),
                          "speedup_of_scheduled_over_lane_split": value / (world * plain["lane_split"]["value"])},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_source": peak_src,
                             "traffic": alg_bytes * ratio if ratio else None,
                             "alg_bytes_per_launch": alg_bytes, "kernel_ms": kern_ms,
                             "kernel": "k_decode_chains"},
                "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(), "gpu_launches": args.steps,
                "decode_errors": bad, "tail": tail, "parity": parity}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
