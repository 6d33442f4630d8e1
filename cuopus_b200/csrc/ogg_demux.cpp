// Host-side Ogg-Opus demuxer and chain builder (see ogg_demux.h).
#include "ogg_demux.h"

#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cstdio>

namespace cuo_host {

int toc_samples48(const uint8_t *p, uint32_t len)
{
    // frame duration in quarter milliseconds per TOC configuration
    static const int qms[32] = {40, 80, 160, 240, 40, 80, 160, 240, 40, 80, 160, 240, 40, 80, 40, 80,
                                10, 20, 40, 80, 10, 20, 40, 80, 10, 20, 40, 80, 10, 20, 40, 80};
    if (!len) return 0;
    int code = p[0] & 3, nf;
    if (code == 0) nf = 1;
    else if (code < 3) nf = 2;
    else {
        if (len < 2) return 0;
        nf = p[1] & 0x3F;
    }
    return qms[p[0] >> 3] * 12 * nf;
}

namespace {

int64_t rd_i64le(const uint8_t *p)
{
    uint64_t v = 0;
    for (int i = 7; i >= 0; i--) v = (v << 8) | p[i];
    return (int64_t)v;
}

std::string fmt(const char *f, long long a = 0, long long b = 0, long long c = 0, long long d = 0)
{
    char buf[256];
    snprintf(buf, sizeof buf, f, a, b, c, d);
    return buf;
}

// Ogg page CRC (RFC 3533): CRC-32, polynomial 0x04C11DB7, initial value 0,
// no reflection, over the whole page with its checksum field taken as zero.
uint32_t ogg_page_crc(const uint8_t *page, size_t len)
{
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; i++) {
            uint32_t r = i << 24;
            for (int k = 0; k < 8; k++) r = (r & 0x80000000u) ? (r << 1) ^ 0x04C11DB7u : r << 1;
            table[i] = r;
        }
        init = true;
    }
    uint32_t crc = 0;
    for (size_t i = 0; i < len; i++) {
        uint8_t b = (i >= 22 && i < 26) ? 0 : page[i];
        crc = (crc << 8) ^ table[((crc >> 24) ^ b) & 0xFF];
    }
    return crc;
}

} // namespace

Options options_from_env()
{
    Options o;
    const char *c = getenv("CUOPUS_OGG_CRC");
    o.check_crc = c && atoi(c) > 0;
    const char *g = getenv("CUOPUS_GRANULE");
    o.granule_warn = g && strcmp(g, "warn") == 0;
    return o;
}

bool demux(const uint8_t *data, size_t n, Demux &d, std::string &err)
{
    return demux(data, n, options_from_env(), d, err);
}

bool demux(const uint8_t *data, size_t n, const Options &opt, Demux &d, std::string &err)
{
    d = Demux();
    if (!data || n == 0) { err = "empty stream"; return false; }
    // One pass over the pages.  The body bytes of the audio packets (packet 2
    // on) are appended to the blob a page at a time, then the lacing table
    // cuts them into packets, each measured once from its TOC.
    std::vector<int64_t> page_granule;
    std::vector<int64_t> page_end;   // end sample of the last audio packet completed on the page, or -1
    page_granule.reserve(n / 2048 + 8);
    page_end.reserve(n / 2048 + 8);
    d.blob.reserve(n);
    d.off.reserve(n / 32 + 8);
    d.len.reserve(n / 32 + 8);
    d.sample_off.reserve(n / 32 + 8);
    uint64_t npk = 0;                          // completed packets, headers included
    uint64_t acc = 0;                          // bytes of the packet in progress
    uint64_t head_len = 0;                     // length of packet 0
    uint64_t head_start = 0, head_span = 0;    // first lacing run of packet 0
    bool head_seen = false, too_large = false;
    uint64_t w = 0;                            // blob offset of the audio packet in progress
    int64_t cum = 0, final_page = -1;
    int last_dur = 0;
    size_t pos = 0;
    static const uint8_t magic[4] = {'O', 'g', 'g', 'S'};
    while (pos < n) {
        const uint8_t *hit = std::search(data + pos, data + n, magic, magic + 4);
        if (hit == data + n) break;
        size_t idx = (size_t)(hit - data);
        if (idx + 27 > n) break;
        int64_t granule = rd_i64le(data + idx + 6);
        uint32_t nseg = data[idx + 26];
        const uint8_t *table = data + idx + 27;
        uint64_t body = idx + 27 + nseg;
        if (body > n) break;
        uint64_t blen = 0;
        for (uint32_t i = 0; i < nseg; i++) blen += table[i];
        if (body + blen > n) break;
        if (opt.check_crc) {
            uint32_t stored = (uint32_t)data[idx + 22] | (uint32_t)data[idx + 23] << 8 |
                              (uint32_t)data[idx + 24] << 16 | (uint32_t)data[idx + 25] << 24;
            if (ogg_page_crc(data + idx, (size_t)(body + blen - idx)) != stored) {
                err = fmt("page %lld: CRC mismatch", (long long)page_granule.size());
                return false;
            }
        }
        uint32_t pg = (uint32_t)page_granule.size();
        page_granule.push_back(granule);
        page_end.push_back(-1);
        // where this page's audio bytes begin (packets 0 and 1 are headers)
        uint64_t audio_from = UINT64_MAX;
        if (npk >= 2) {
            audio_from = body;
        } else {
            uint64_t k = npk, q = body, r = 0;
            for (uint32_t i = 0; i < nseg; i++) {
                r += table[i];
                if (table[i] < 255) {
                    q += r;
                    r = 0;
                    if (++k == 2) { audio_from = q; break; }
                }
            }
        }
        if (audio_from < body + blen) d.blob.insert(d.blob.end(), data + audio_from, data + body + blen);
        // lacing runs < 255 end a packet; a trailing run continues on the next page
        uint64_t run_start = body, run = 0;
        for (uint32_t i = 0; i < nseg; i++) {
            run += table[i];
            if (table[i] == 255) continue;
            if (!head_seen) { head_seen = true; head_start = run_start; head_span = run; }
            acc += run;
            if (acc > 0xFFFFFFFFull) too_large = true;
            if (npk >= 2 && !too_large) {
                uint32_t L = (uint32_t)acc;
                int ns = toc_samples48(d.blob.data() + w, L);
                d.off.push_back(w);
                d.len.push_back(L);
                d.sample_off.push_back(cum);
                cum += ns;
                last_dur = ns;
                page_end[pg] = cum;
                final_page = pg;
                w += L;
            } else if (npk == 0) {
                head_len = acc;
            }
            npk++;
            acc = 0;
            run_start += run;
            run = 0;
        }
        if (run > 0) {
            if (!head_seen) { head_seen = true; head_start = run_start; head_span = run; }
            acc += run;
            if (acc > 0xFFFFFFFFull) too_large = true;
        }
        pos = body + blen;
    }
    if (page_granule.empty()) { err = "no OGG pages found"; return false; }
    d.n_pages = (uint32_t)page_granule.size();
    if (too_large) { err = "packet too large"; return false; }
    if (npk < 2) { err = "not an OGG Opus stream (fewer than 2 packets)"; return false; }
    // OpusHead fields are read from packet 0's first lacing run, as the reference does
    if (head_len < 19 || head_span < 12 || memcmp(data + head_start, "OpusHead", 8) != 0) {
        err = "not an OGG Opus stream (no OpusHead)";
        return false;
    }
    d.channels = data[head_start + 9];
    d.preskip = data[head_start + 10] | (data[head_start + 11] << 8);
    if (w > 0xFFFFFFFFull) { err = "stream too large"; return false; }
    d.blob.resize(w);   // drops a partial packet at the end of the stream
    d.toc_total = cum;

    // granule cross-check
    int64_t last_granule = 0;
    for (size_t pg = 0; pg < page_granule.size(); pg++) {
        int64_t g = page_granule[pg];
        if (g != -1 && g > last_granule) last_granule = g;
        if (g == -1 || page_end[pg] < 0) continue;
        d.granule_checked++;
        if (g == page_end[pg]) d.granule_match++;
        else if ((int64_t)pg == final_page && page_end[pg] - g >= 0 && page_end[pg] - g < last_dur)
            d.granule_match++;
    }
    d.last_granule = last_granule;
    d.end_trim = d.toc_total - last_granule;
    d.play48 = last_granule - d.preskip;
    if (opt.granule_warn && d.granule_match != d.granule_checked) {
        // resync on the packets: their TOC durations are the timeline; the
        // final granule still trims the end when it is a legal end trim
        // (short of the TOC total by less than the last packet)
        d.granule_mismatch = d.granule_checked - d.granule_match;
        int64_t trim = d.toc_total - last_granule;
        if (!(trim >= 0 && trim < last_dur)) trim = 0;
        d.end_trim = trim;
        d.last_granule = d.toc_total - trim;
        d.play48 = d.last_granule - d.preskip;
        d.granule_match = d.granule_checked;
    }
    return true;
}

bool build_chains(const Demux &d, double seconds, double preroll_ms, Chains &c, std::string &err)
{
    c = Chains();
    int64_t step = (int64_t)(seconds * 48000);
    int64_t preroll = (int64_t)(preroll_ms * 48);
    int64_t total = d.play48;
    uint32_t npk = d.n_packets();
    if (total <= 0) { err = "no playable samples"; return false; }
    if (step <= 0) { err = "bad segment length"; return false; }
    // Header pages can carry a granule (hence playable samples) with no audio
    // packet after them; the reference's cu_build_chains2 then reads past its
    // prefix-sum array.
    if (npk == 0) { err = "no audio packets"; return false; }
    const std::vector<int64_t> &so = d.sample_off;
    // TOC samples before packet k (the demuxer's prefix sums)
    auto cum = [&](int64_t k) -> int64_t { return k < (int64_t)npk ? so[(size_t)k] : d.toc_total; };
    // a hint only: a damaged granule can claim far more chains than the packets
    // hold, and such a stream fails below
    const size_t nchains = std::min<size_t>((size_t)((total + step - 1) / step), (size_t)npk + 16);
    c.first.reserve(nchains);
    c.npkts.reserve(nchains);
    c.trim.reserve(nchains);
    c.keep.reserve(nchains);
    c.cap.reserve(nchains);
    int64_t kept = 0;
    for (int64_t k = 0; k * step < total; k++) {
        int64_t ps = k * step, pe = std::min((k + 1) * step, total);
        int64_t ts = ps + d.preskip, te = pe + d.preskip;
        int64_t target = std::max<int64_t>(0, ts - preroll);
        int64_t first = (int64_t)(std::upper_bound(so.begin(), so.end(), target) - so.begin()) - 1;
        if (first < 0) first = 0;
        if (cum(first + 1) <= target) first++;
        int64_t last = (int64_t)(std::lower_bound(so.begin(), so.end(), te) - so.begin()) - 1;
        if (last < first) last = first;
        if (first >= (int64_t)npk || last >= (int64_t)npk) {
            err = fmt("chain %lld: packet range beyond the stream", k);
            return false;
        }
        int64_t trim = ts - so[first], keep = pe - ps;
        if (trim < 0) { err = fmt("chain %lld: negative trim %lld", k, trim); return false; }
        int64_t capn = cum(last + 1) - cum(first);
        if (capn < trim + keep) {
            err = fmt("chain %lld: capacity %lld < trim %lld + keep %lld", k, capn, trim, keep);
            return false;
        }
        c.first.push_back((uint32_t)first);
        c.npkts.push_back((uint32_t)(last - first + 1));
        c.trim.push_back((uint32_t)trim);
        c.keep.push_back((uint32_t)keep);
        c.cap.push_back((uint64_t)capn);
        kept += keep;
    }
    if (kept != total) { err = fmt("internal: sum(keep) %lld != playable %lld", kept, total); return false; }
    return true;
}

bool demux_and_chain(const uint8_t *data, size_t n, double seconds, double preroll_ms, bool require_mono,
                     Demux &d, Chains *c, std::string &err)
{
    if (!demux(data, n, d, err)) return false;
    if (require_mono && d.channels != 1) {
        err = fmt("only mono supported (channels=%lld)", d.channels);
        return false;
    }
    if (d.channels != 1 && d.channels != 2) {
        err = fmt("unsupported channel count %lld", d.channels);
        return false;
    }
    if (d.granule_match != d.granule_checked) {
        err = fmt("granule cross-check failed (%lld/%lld)", d.granule_match, d.granule_checked);
        return false;
    }
    if (c && !build_chains(d, seconds, preroll_ms, *c, err)) return false;
    return true;
}

} // namespace cuo_host
