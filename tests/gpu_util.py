"""Helpers for the GPU tests: move a chain table to the device and run the
engine (cuopus_decode_batch) through the C ABI."""
import numpy as np


def device_batch(packets_list, chains_list, channels_list):
    """Device-resident tables of several streams' chains (no per-packet
    records).  Returns (Batch, tensors to keep alive, meta dict)."""
    import torch
    from cuopus_b200 import cuopus_native as cn
    from oracle.ogg_port import decode_capacity48 as toc_samples48
    blob, off, lens, first, npk, chans, trim, keep, cap = [], [], [], [], [], [], [], [], []
    base_pkt = base_byte = 0
    for pk, chs, ch in zip(packets_list, chains_list, channels_list):
        for p in pk:
            off.append(base_byte)
            lens.append(len(p))
            blob.append(p)
            base_byte += len(p)
        for c in chs:
            first.append(c[0] + base_pkt)
            npk.append(c[1])
            chans.append(ch)
            cp = sum(toc_samples48(pk[c[0] + k]) for k in range(c[1]))
            t = c[2] if len(c) > 2 else 0
            trim.append(t)
            keep.append(min(c[3] if len(c) > 3 else cp, max(cp - t, 0)))
            cap.append(cp)
        base_pkt += len(pk)
    n = len(first)
    out_off = np.zeros(n, np.uint64)
    if n > 1:
        out_off[1:] = np.cumsum(np.array(keep[:-1], np.uint64) * np.array(chans[:-1], np.uint64))
    total = int(sum(k * c for k, c in zip(keep, chans)))
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(np.array(a, dtype=dt))).cuda()
    T = dict(blob=t(np.frombuffer(b"".join(blob) + b"\0" * 16, np.uint8), np.uint8), off=t(off, np.uint64),
             len=t(lens, np.uint32), first=t(first, np.uint32), npk=t(npk, np.uint32), ch=t(chans, np.uint8),
             trim=t(trim, np.uint64), keep=t(keep, np.uint64), ooff=t(out_off, np.uint64),
             out=torch.zeros(max(total, 1), dtype=torch.int16, device="cuda"),
             res=torch.zeros(4 * max(n, 1), dtype=torch.int32, device="cuda"))
    b = cn.Batch()
    b.data, b.off, b.len = T["blob"].data_ptr(), T["off"].data_ptr(), T["len"].data_ptr()
    b.first, b.npkts, b.channels = T["first"].data_ptr(), T["npk"].data_ptr(), T["ch"].data_ptr()
    b.trim, b.keep, b.out_off = T["trim"].data_ptr(), T["keep"].data_ptr(), T["ooff"].data_ptr()
    b.out, b.res = T["out"].data_ptr(), T["res"].data_ptr()
    b.nchains = n
    meta = dict(n=n, out_off=out_off, keep=np.array(keep), chans=np.array(chans), cap=np.array(cap),
                npkts=np.array(npk), T=T)
    return b, T, meta


def run_device_batch(b, meta, width=32, schedule=1, order=None, block=0, graph=0):
    """Run the engine on a device batch; returns res as uint32 [n, 4]."""
    import torch
    from cuopus_b200 import cuopus_native as cn
    b.width, b.schedule, b.block, b.graph = width, schedule, block, graph
    keep = None
    if order is not None:
        keep = np.ascontiguousarray(np.asarray(order, np.uint32))
        b.order = keep.ctypes.data
    else:
        b.order = None
    meta["T"]["res"].zero_()
    cn.decode_batch(b, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return meta["T"]["res"].cpu().numpy().view(np.uint32).reshape(-1, 4)[:meta["n"]]


def run_batch(packets_list, chains_list, channels_list, width=32, schedule=0, order=None, max_groups=0,
              records=True, fec=0):
    """Decode chains of several streams in one launch.

    packets_list[s]: list of packets of stream s; chains_list[s]: (first, npkts, trim, keep) over it;
    channels_list[s]: channels.  Returns per chain dicts with pcm (kept samples), nsamp, rng, res."""
    import torch
    from cuopus_b200 import cuopus_native as cn
    blob, off, lens = [], [], []
    first, npk, chans, trim, keep = [], [], [], [], []
    base_pkt = 0
    base_byte = 0
    for pk, chs, ch in zip(packets_list, chains_list, channels_list):
        for p in pk:
            off.append(base_byte)
            lens.append(len(p))
            blob.append(p)
            base_byte += len(p)
        for c in chs:
            first.append(c[0] + base_pkt)
            npk.append(c[1])
            chans.append(ch)
            trim.append(c[2] if len(c) > 2 else 0)
            keep.append(c[3] if len(c) > 3 else (1 << 40))
        base_pkt += len(pk)
    n = len(first)
    cap = []
    from oracle.ogg_port import decode_capacity48 as toc_samples48
    allp = [p for pk in packets_list for p in pk]
    for i in range(n):
        cap.append(sum(toc_samples48(allp[first[i] + k]) for k in range(npk[i])))
    keep = [min(keep[i], max(cap[i] - trim[i], 0)) for i in range(n)]
    out_off = np.zeros(n, np.uint64)
    if n > 1:
        out_off[1:] = np.cumsum(np.array(keep[:-1], np.uint64) * np.array(chans[:-1], np.uint64))
    total = int(sum(k * c for k, c in zip(keep, chans)))
    rec_off = np.zeros(n, np.uint64)
    if n > 1:
        rec_off[1:] = np.cumsum(np.array(npk[:-1], np.uint64))
    nrec = int(sum(npk))
    dev = "cuda"
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(np.array(a, dtype=dt))).to(dev)
    d_blob = t(np.frombuffer(b"".join(blob) + b"\0" * 16, np.uint8), np.uint8)
    d_off = t(off, np.uint64)
    d_len = t(lens, np.uint32)
    d_first = t(first, np.uint32)
    d_npk = t(npk, np.uint32)
    d_ch = t(chans, np.uint8)
    d_trim = t(trim, np.uint64)
    d_keep = t(keep, np.uint64)
    d_ooff = t(out_off, np.uint64)
    d_out = torch.zeros(max(total, 1), dtype=torch.int16, device=dev)
    d_roff = t(rec_off, np.uint64)
    d_ns = torch.zeros(max(nrec, 1), dtype=torch.int32, device=dev)
    d_rg = torch.zeros(max(nrec, 1), dtype=torch.int32, device=dev)
    d_res = torch.zeros(4 * max(n, 1), dtype=torch.int32, device=dev)
    b = cn.Batch()
    b.data, b.off, b.len = d_blob.data_ptr(), d_off.data_ptr(), d_len.data_ptr()
    b.first, b.npkts, b.channels = d_first.data_ptr(), d_npk.data_ptr(), d_ch.data_ptr()
    b.trim, b.keep, b.out_off, b.out = d_trim.data_ptr(), d_keep.data_ptr(), d_ooff.data_ptr(), d_out.data_ptr()
    if records:
        b.rec_off, b.pkt_nsamp, b.pkt_rng = d_roff.data_ptr(), d_ns.data_ptr(), d_rg.data_ptr()
    b.res = d_res.data_ptr()
    b.nchains, b.width, b.schedule, b.max_groups = n, width, schedule, max_groups
    b.fec = fec
    order_arr = None
    if order is not None:
        order_arr = np.ascontiguousarray(np.array(order, np.uint32))
        b.order = order_arr.ctypes.data
    ms = cn.decode_batch(b, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy()
    ns = d_ns.cpu().numpy().view(np.uint32)
    rg = d_rg.cpu().numpy().view(np.uint32)
    res = d_res.cpu().numpy().reshape(-1, 4)
    chains = []
    for i in range(n):
        o = int(out_off[i])
        r0 = int(rec_off[i])
        chains.append(dict(pcm=out[o:o + keep[i] * chans[i]], nsamp=ns[r0:r0 + npk[i]], rng=rg[r0:r0 + npk[i]],
                           stop=int(res[i, 0]), samples=int(res[i, 1].view(np.uint32) if hasattr(res[i, 1], 'view') else res[i, 1]),
                           final_range=int(np.uint32(res[i, 2])), time_us=int(np.uint32(res[i, 3])),
                           trim=trim[i], keep=keep[i], cap=cap[i]))
    return chains, ms
