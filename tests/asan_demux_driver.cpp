// Test driver: the host demuxer and chain builder over a file of damaged Ogg
// streams, built with AddressSanitizer and UndefinedBehaviorSanitizer by
// tests/test_sanitizers.py.  Input records are [u32 length][bytes]; each
// stream is copied into a heap buffer of exactly its length (so a read past
// its end is reported) and parsed with the default options, the page-CRC
// check and the granule warn-and-resync policy.  One line per record and
// policy: "ok <play48> <channels> <packets> <chains> <sum keep>" or "refused".
// Each is also demuxed with its pages split over three threads (ranges of any
// size); a result that differs in any field is reported on stderr and the
// driver exits 3.
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "ogg_demux.h"

int main(int argc, char **argv)
{
    if (argc != 2) {
        fprintf(stderr, "usage: %s <records>\n", argv[0]);
        return 2;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 2;
    std::vector<uint8_t> all;
    uint8_t buf[65536];
    size_t r;
    while ((r = fread(buf, 1, sizeof buf, f)) > 0) all.insert(all.end(), buf, buf + r);
    fclose(f);
    size_t o = 0;
    int rec = 0, split_mismatch = 0;
    while (o + 4 <= all.size()) {
        uint32_t n;
        memcpy(&n, all.data() + o, 4);
        o += 4;
        if (o + n > all.size()) return 2;
        for (int policy = 0; policy < 3; policy++) {
            uint8_t *data = new uint8_t[n ? n : 1];
            memcpy(data, all.data() + o, n);
            cuo_host::Options opt;
            opt.check_crc = policy == 1;
            opt.granule_warn = policy == 2;
            cuo_host::Demux d;
            cuo_host::Chains c;
            std::string err;
            double seg = rec % 2 ? 1.0 : 0.5, pre = rec % 2 ? 250.0 : 80.0;
            bool dm = cuo_host::demux(n ? data : nullptr, n, opt, d, err);
            cuo_host::Options opt3 = opt;
            opt3.threads = 3;
            opt3.range_bytes = 1;
            cuo_host::Demux d3;
            std::string err3;
            bool dm3 = cuo_host::demux(n ? data : nullptr, n, opt3, d3, err3);
            if (dm != dm3 || err != err3 || d.blob != d3.blob || d.off != d3.off || d.len != d3.len ||
                d.sample_off != d3.sample_off || d.channels != d3.channels || d.preskip != d3.preskip ||
                d.toc_total != d3.toc_total || d.last_granule != d3.last_granule || d.play48 != d3.play48 ||
                d.end_trim != d3.end_trim || d.n_pages != d3.n_pages || d.granule_checked != d3.granule_checked ||
                d.granule_match != d3.granule_match || d.granule_mismatch != d3.granule_mismatch) {
                fprintf(stderr, "record %d policy %d: the split demux differs\n", rec, policy);
                split_mismatch++;
            }
            bool ok = dm && (d.channels == 1 || d.channels == 2) && d.granule_match == d.granule_checked &&
                      cuo_host::build_chains(d, seg, pre, c, err);
            if (ok) {
                long long keep = 0;
                for (uint32_t k : c.keep) keep += k;
                printf("ok %lld %lld %u %zu %lld\n", (long long)d.play48, (long long)d.channels, d.n_packets(),
                       c.keep.size(), keep);
            } else {
                printf("refused\n");
            }
            delete[] data;
        }
        o += n;
        rec++;
    }
    return split_mismatch ? 3 : 0;
}
