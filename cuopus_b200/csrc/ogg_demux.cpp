// Host-side Ogg-Opus demuxer and chain builder (see ogg_demux.h).
#include "ogg_demux.h"

#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cstdio>
#include <thread>

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

// What the serial walk knows of one page when it reaches it.
struct PageWalk {
    int64_t granule;
    uint64_t body, blen, table;   // body and lacing table offsets in the stream, body length
    uint64_t npk;                 // packets completed before the page, headers included
    uint64_t acc;                 // bytes of the packet in progress at the page start
    uint64_t audio_from;          // stream offset of the page's first audio byte (UINT64_MAX: none)
    uint64_t blob;                // blob offset of that byte (audio bytes before the page)
    uint64_t audio, done;         // audio packets completed before / on the page
    uint32_t nseg;
};

// Page ranges of about equal body bytes, at most `threads` of them and none
// below `range_bytes` (small streams stay on the calling thread).
std::vector<size_t> page_ranges(const std::vector<PageWalk> &pages, int threads, size_t range_bytes)
{
    uint64_t total = 0;
    for (const PageWalk &P : pages) total += P.blen;
    size_t t = (size_t)std::max(1, threads);
    t = std::min<size_t>(t, (size_t)(total / std::max<size_t>(range_bytes, 1)) + 1);
    std::vector<size_t> cut{0};
    uint64_t acc = 0;
    for (size_t pg = 0; pg < pages.size(); pg++) {
        acc += pages[pg].blen;
        if (cut.size() < t && acc * t >= total * cut.size() && pg + 1 < pages.size()) cut.push_back(pg + 1);
    }
    cut.push_back(pages.size());
    return cut;
}

// fn(begin, end) for every range of `cut`, the first on the calling thread.
template <class F> void run_ranges(const std::vector<size_t> &cut, F &&fn)
{
    std::vector<std::thread> pool;
    for (size_t r = 1; r + 1 < cut.size(); r++) {
        try {
            pool.emplace_back([&fn, &cut, r] { fn(cut[r], cut[r + 1]); });
        } catch (...) {
            fn(cut[r], cut[r + 1]);   // no thread: run it here
        }
    }
    fn(cut[0], cut[1]);
    for (auto &th : pool) th.join();
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
    // 1. A serial walk over the page headers and lacing tables decides
    //    everything structural: where each page's audio bytes go in the blob,
    //    which packets complete on it, the header checks and every error.
    // 2. Page ranges, in parallel: copy the audio bytes into the blob.
    // 3. Page ranges, in parallel: cut packets, read each TOC once.
    // 4. Prefix sums of the TOC durations and the granule cross-check.
    std::vector<PageWalk> pages;
    pages.reserve(n / 2048 + 8);
    uint64_t npk = 0;                          // completed packets, headers included
    uint64_t acc = 0;                          // bytes of the packet in progress
    uint64_t head_len = 0;                     // length of packet 0
    uint64_t head_start = 0, head_span = 0;    // first lacing run of packet 0
    bool head_seen = false, too_large = false;
    uint64_t appended = 0;                     // audio body bytes before the page
    uint64_t n_audio = 0, w = 0;               // completed audio packets and their bytes
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
                err = fmt("page %lld: CRC mismatch", (long long)pages.size());
                return false;
            }
        }
        PageWalk P;
        P.granule = granule;
        P.body = body;
        P.blen = blen;
        P.table = idx + 27;
        P.nseg = nseg;
        P.npk = npk;
        P.acc = acc;
        P.blob = appended;
        P.audio = n_audio;
        // where this page's audio bytes begin (packets 0 and 1 are headers)
        P.audio_from = UINT64_MAX;
        if (npk >= 2) {
            P.audio_from = body;
        } else {
            uint64_t k = npk, q = body, r = 0;
            for (uint32_t i = 0; i < nseg; i++) {
                r += table[i];
                if (table[i] < 255) {
                    q += r;
                    r = 0;
                    if (++k == 2) { P.audio_from = q; break; }
                }
            }
        }
        if (P.audio_from < body + blen) appended += body + blen - P.audio_from;
        // lacing runs < 255 end a packet; a trailing run continues on the next page
        uint64_t run_start = body, run = 0;
        for (uint32_t i = 0; i < nseg; i++) {
            run += table[i];
            if (table[i] == 255) continue;
            if (!head_seen) { head_seen = true; head_start = run_start; head_span = run; }
            acc += run;
            if (acc > 0xFFFFFFFFull) too_large = true;
            if (npk >= 2) {
                n_audio++;
                w += acc;
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
        P.done = n_audio - P.audio;
        pages.push_back(P);
        pos = body + blen;
    }
    if (pages.empty()) { err = "no OGG pages found"; return false; }
    d.n_pages = (uint32_t)pages.size();
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

    // the page ranges: audio bytes first (a packet's TOC can sit on an earlier
    // range's page), then packets; sample_off holds each packet's duration
    // until the prefix sums below
    d.blob.resize(appended);
    d.off.resize(n_audio);
    d.len.resize(n_audio);
    d.sample_off.resize(n_audio);
    const std::vector<size_t> cut = page_ranges(pages, opt.threads, opt.range_bytes);
    run_ranges(cut, [&](size_t a, size_t b) {
        for (size_t pg = a; pg < b; pg++) {
            const PageWalk &P = pages[pg];
            if (P.audio_from < P.body + P.blen)
                memcpy(d.blob.data() + P.blob, data + P.audio_from, P.body + P.blen - P.audio_from);
        }
    });
    run_ranges(cut, [&](size_t a, size_t b) {
        for (size_t pg = a; pg < b; pg++) {
            const PageWalk &P = pages[pg];
            const uint8_t *table = data + P.table;
            uint64_t k = P.audio, pk = P.npk, acc = P.acc, run_start = P.body, run = 0;
            for (uint32_t i = 0; i < P.nseg; i++) {
                run += table[i];
                if (table[i] == 255) continue;
                acc += run;
                if (pk >= 2) {
                    // blob offset of the packet's end, less its length
                    uint64_t off = P.blob + (run_start + run - P.audio_from) - acc;
                    d.off[k] = off;
                    d.len[k] = (uint32_t)acc;
                    d.sample_off[k] = toc_samples48(d.blob.data() + off, (uint32_t)acc);
                    k++;
                }
                pk++;
                acc = 0;
                run_start += run;
                run = 0;
            }
        }
    });
    d.blob.resize(w);   // drops a partial packet at the end of the stream
    int64_t cum = 0;
    int last_dur = 0;
    for (uint64_t k = 0; k < n_audio; k++) {
        int64_t ns = d.sample_off[k];
        d.sample_off[k] = cum;
        cum += ns;
        last_dur = (int)ns;
    }
    d.toc_total = cum;

    // granule cross-check: a page's end is that of the last audio packet completed on it
    int64_t final_page = -1;
    for (size_t pg = 0; pg < pages.size(); pg++)
        if (pages[pg].done) final_page = (int64_t)pg;
    int64_t last_granule = 0;
    for (size_t pg = 0; pg < pages.size(); pg++) {
        const PageWalk &P = pages[pg];
        int64_t g = P.granule;
        if (g != -1 && g > last_granule) last_granule = g;
        if (g == -1 || !P.done) continue;
        uint64_t k_end = P.audio + P.done;
        int64_t page_end = k_end < n_audio ? d.sample_off[k_end] : d.toc_total;
        d.granule_checked++;
        if (g == page_end) d.granule_match++;
        else if ((int64_t)pg == final_page && page_end - g >= 0 && page_end - g < last_dur)
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
    const Table<int64_t> &so = d.sample_off;
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
                     Demux &d, Chains *c, std::string &err, int threads)
{
    Options opt = options_from_env();
    opt.threads = threads;
    if (!demux(data, n, opt, d, err)) return false;
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
