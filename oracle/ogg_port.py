"""CPU restatement of the reference's Ogg-Opus indexer and chain builder.

TEST INFRASTRUCTURE (oracle).  Restates, in plain Python:
  * page parse + packet reassembly   ogg_index.py:75-170   (cuopus_demux.h:79-214)
  * TOC durations                    ogg_index.py:52-68    (cuopus_demux.h:46-60)
  * granule cross-check with the RFC 7845 end trim on the final data page
                                     ogg_index.py:172-190  (cuopus_demux.h:216-262)
  * playable-space chain table (first, npkts, trim, keep)
                                     ogg_index.py:319-367  (cuopus_demux.h:293-378)
Page CRCs are not checked (the reference's GPU path runs with check_crc=False).
The product's host demuxer (cuopus_b200/csrc/ogg_demux.cpp) is compared with
this module and with golden tables made by the reference's own ogg_index.py.
"""
from __future__ import annotations

import bisect
import struct

# quarter-milliseconds per frame for each TOC configuration (RFC 6716 sec. 3.1)
QMS = [40, 80, 160, 240] * 3 + [40, 80] * 2 + [10, 20, 40, 80] * 4


def toc_samples48(pkt: bytes) -> int:
    if not pkt:
        return 0
    code = pkt[0] & 3
    if code == 0:
        nf = 1
    elif code < 3:
        nf = 2
    else:
        if len(pkt) < 2:
            return 0
        nf = pkt[1] & 0x3F
    return QMS[pkt[0] >> 3] * 12 * nf


def decode_capacity48(pkt: bytes) -> int:
    """Samples per channel opus_decode(..., frame_size=5760, 0) can return for
    this packet: the TOC's count, or 5760 for an empty packet (a lost packet:
    opus_decode_native conceals until frame_size is filled,
    src/opus_decoder.c:715-729 of the vendored libopus)."""
    return 5760 if len(pkt) == 0 else toc_samples48(pkt)


class DemuxError(ValueError):
    pass


def demux(data: bytes) -> dict:
    """Parse an in-memory Ogg Opus stream."""
    n = len(data)
    pos = 0
    page_gran, spans = [], []          # spans: (start, end, complete, page)
    while pos < n:
        idx = data.find(b"OggS", pos)
        if idx < 0 or idx + 27 > n:
            break
        granule = struct.unpack_from("<q", data, idx + 6)[0]
        nseg = data[idx + 26]
        table = data[idx + 27: idx + 27 + nseg]
        body = idx + 27 + nseg
        blen = sum(table)
        if body + blen > n:
            break
        pg = len(page_gran)
        page_gran.append(granule)
        run_start, run_len, last = body, 0, 0
        for lac in table:
            run_len += lac
            last = lac
            if lac < 255:
                spans.append((run_start, run_start + run_len, True, pg))
                run_start += run_len
                run_len = 0
        if run_len > 0 or (nseg > 0 and last == 255):
            spans.append((run_start, run_start + run_len, False, pg))
        pos = body + blen
    if not page_gran:
        raise DemuxError("no OGG pages found")
    packets, pages, first_span = [], [], []
    part, start = b"", None
    for s, e, done, pg in spans:
        if start is None:
            start = e - s
        part += data[s:e]
        if done:
            packets.append(part)
            pages.append(pg)
            first_span.append(start)
            part, start = b"", None
    if len(packets) < 2:
        raise DemuxError("not an OGG Opus stream (fewer than 2 packets)")
    head = packets[0]
    # the header fields are read from the packet's first span (a page-split
    # OpusHead whose first piece is shorter than 12 bytes is refused)
    if len(head) < 19 or first_span[0] < 12 or not head.startswith(b"OpusHead"):
        raise DemuxError("not an OGG Opus stream (no OpusHead)")
    channels = head[9]
    preskip = head[10] | (head[11] << 8)
    audio = packets[2:]
    apages = pages[2:]
    sample_off, cum = [], 0
    for p in audio:
        sample_off.append(cum)
        cum += toc_samples48(p)
    pkt_end = {}
    for k, pg in enumerate(apages):
        pkt_end[pg] = sample_off[k] + toc_samples48(audio[k])
    final_page = max(pkt_end) if pkt_end else -1
    last_dur = toc_samples48(audio[-1]) if audio else 0
    checked = match = 0
    last_granule = 0
    for pg, g in enumerate(page_gran):
        if g != -1 and g > last_granule:
            last_granule = g
        if g == -1 or pg not in pkt_end:
            continue
        checked += 1
        if g == pkt_end[pg]:
            match += 1
        elif pg == final_page and 0 <= pkt_end[pg] - g < last_dur:
            match += 1
    return dict(packets=audio, sample_off=sample_off, channels=channels, preskip=preskip,
                toc_total=cum, last_granule=last_granule, play48=last_granule - preskip,
                end_trim=cum - last_granule, granule_checked=checked,
                granule_match=match, n_pages=len(page_gran))


def build_chains(ix: dict, seconds: float, preroll_ms: float):
    """(first, npkts, trim, keep) per chain over the playable samples."""
    step = int(seconds * 48000)
    preroll = int(preroll_ms * 48)
    pre = ix["preskip"]
    total = ix["play48"]
    so = ix["sample_off"]
    pk = ix["packets"]
    if total <= 0:
        raise DemuxError("no playable samples")
    if step <= 0:
        raise DemuxError("bad segment length")
    if not pk:
        # header pages may carry a granule with no audio packet after them
        # (cuopus_demux.h:293-378 reads past its prefix sums here)
        raise DemuxError("no audio packets")
    cum = [0]
    for p in pk:
        cum.append(cum[-1] + toc_samples48(p))
    out = []
    k = 0
    while k * step < total:
        ps, pe = k * step, min((k + 1) * step, total)
        ts, te = ps + pre, pe + pre
        target = max(0, ts - preroll)
        first = max(bisect.bisect_right(so, target) - 1, 0)
        if cum[first + 1] <= target:
            first += 1
        last = max(bisect.bisect_left(so, te) - 1, first)
        if first >= len(pk):
            raise DemuxError("chain %d: packet range beyond the stream" % k)
        trim, keep = ts - so[first], pe - ps
        if trim < 0:
            raise DemuxError("chain %d: negative trim %d" % (k, trim))
        if cum[last + 1] - cum[first] < trim + keep:
            raise DemuxError("chain %d: capacity %d < trim %d + keep %d"
                             % (k, cum[last + 1] - cum[first], trim, keep))
        out.append((first, last - first + 1, trim, keep))
        k += 1
    assert sum(c[3] for c in out) == total
    return out
