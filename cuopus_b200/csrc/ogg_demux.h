// Host-side Ogg-Opus demuxer and chain builder.
//
// Behaviour of the reference's cu_demux_mem / cu_build_chains2
// (cuopus_demux.h:79-269, :293-378; Python twin ogg_index.py:75-209, :319-367):
//   * every "OggS" page is parsed (CRC not checked); lacing runs < 255 end a
//     packet, a trailing run continues on the next page; a partial packet at
//     end of file is dropped;
//   * packet 0 must be OpusHead (>= 19 bytes): channels = byte 9, pre-skip =
//     bytes 10-11; packets 0 and 1 (OpusTags) are headers;
//   * each audio packet's 48 kHz duration comes from its TOC (RFC 6716 3.1);
//   * every page with a granule and a completed packet is cross-checked
//     against the cumulative TOC sum; the final data page may be short by less
//     than the last packet's duration (RFC 7845 end trim);
//   * playable samples = last granule - pre-skip;
//   * chains: the playable range is cut every `seconds`; each chain starts
//     `preroll_ms` early (clamped at 0), `trim` drops preroll + pre-skip and
//     `keep` is exact, so sum(keep) == playable.
// The implementation is std::vector based and allocation-checked; errors are
// returned as a message, never by exiting.
#pragma once
#include <stdint.h>

#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace cuo_host {

int toc_samples48(const uint8_t *p, uint32_t len);

// std::allocator that leaves new elements uninitialised: tables that are
// written in full right after they are sized skip the zero fill.
template <class T> struct NoInit : std::allocator<T> {
    template <class U> struct rebind { using other = NoInit<U>; };
    NoInit() = default;
    template <class U> NoInit(const NoInit<U> &) {}
    template <class U> void construct(U *p) noexcept { ::new ((void *)p) U; }
    template <class U, class... A> void construct(U *p, A &&...a) { ::new ((void *)p) U(std::forward<A>(a)...); }
};
template <class T> using Table = std::vector<T, NoInit<T>>;

struct Demux {
    Table<uint8_t> blob;              // audio packets back to back
    Table<uint64_t> off;              // per packet offset into blob
    Table<uint32_t> len;              // per packet length
    Table<int64_t> sample_off;        // per packet cumulative 48 kHz offset
    int channels = 0;
    int preskip = 0;
    int64_t toc_total = 0;
    int64_t last_granule = 0;
    int64_t play48 = 0;               // last_granule - preskip
    int64_t end_trim = 0;
    uint32_t n_pages = 0;
    uint32_t granule_checked = 0, granule_match = 0;
    uint32_t granule_mismatch = 0;    // pages resynchronised under the "warn" granule policy
    uint32_t n_packets() const { return (uint32_t)len.size(); }
};

// Demux options (extensions; the defaults are the reference's behaviour):
//   check_crc     verify every page's CRC-32 (RFC 3533); a bad page fails the
//                 stream (the reference's GPU path does not check, ogg_index.py
//                 can: :103-111)
//   granule_warn  a page granule that disagrees with the TOC durations does not
//                 fail the stream: the packets' TOC durations are the timeline
//                 and the final granule trims the end only when it is a legal
//                 end trim (the reference fails such streams,
//                 cuopus_demux.h:240-258)
// options_from_env() reads them per call from CUOPUS_OGG_CRC=1 and
// CUOPUS_GRANULE=warn.
//   threads       host threads that copy the packets and read their TOCs,
//                 each over a range of pages of about equal bytes (the
//                 structural walk and every error stay on the calling thread;
//                 the result does not depend on the count)
//   range_bytes   the least page bytes per range (small streams: one range)
struct Options {
    bool check_crc = false;
    bool granule_warn = false;
    int threads = 1;
    size_t range_bytes = 256 << 10;
};
Options options_from_env();

struct Chains {
    std::vector<uint32_t> first, npkts, trim, keep;
    std::vector<uint64_t> cap;   // 48 kHz samples per channel the chain's packets decode to
    uint32_t size() const { return (uint32_t)first.size(); }
};

// Returns true on success; on failure `err` holds the reason.  The first form
// takes its options from the environment.
bool demux(const uint8_t *data, size_t n, Demux &d, std::string &err);
bool demux(const uint8_t *data, size_t n, const Options &opt, Demux &d, std::string &err);
bool build_chains(const Demux &d, double seconds, double preroll_ms, Chains &c, std::string &err);

// Demux (options from the environment, `threads` demux threads) + the
// reference's acceptance checks (granule cross-check; mono only when
// require_mono) + chain table.
bool demux_and_chain(const uint8_t *data, size_t n, double seconds, double preroll_ms, bool require_mono,
                     Demux &d, Chains *c, std::string &err, int threads = 1);

} // namespace cuo_host
