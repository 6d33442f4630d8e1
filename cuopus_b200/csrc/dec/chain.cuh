// One chain = a fresh 48 kHz Opus decoder run over a contiguous packet range,
// the protocol of the reference decode kernel (cuopus_kernels.cuh:41-69: a
// fresh cu_opus_decoder_init per chain, then one cu_opus_decode per packet,
// stopping at the first negative return).  Decoded samples whose chain-local
// index falls in [trim, trim + keep) are written, interleaved, to `out`; the
// other samples (preroll, pre-skip) are decoded and dropped, which fuses the
// reference's separate compaction kernel (cuopus_kernels.cuh:75-88) into the
// decode.
#pragma once
#include "opusdec.cuh"

namespace cuo {

struct ChainResult {
    int32_t stop;          // 0, or the first negative opus_decode return
    uint32_t samples;      // samples per channel decoded
    uint32_t final_range;  // OPUS_GET_FINAL_RANGE after the last packet
    uint32_t cycles;       // device clock cycles spent on the chain (0 on the host)
};

struct ChainSlot {         // per resident decoder group, in global memory
    OpusDec dec;
    OpusScratch scratch;
    int16_t frame_buf[2880 * 2];
};

struct KeepWindow {
    const Lanes *L;
    int16_t *out;
    int channels;
    uint64_t pos, trim, keep;
    MFN void operator()(const int16_t *frame, int n)
    {
        uint64_t lo = pos > trim ? pos : trim;
        uint64_t hi = pos + (uint64_t)n < trim + keep ? pos + (uint64_t)n : trim + keep;
        if (hi > lo) {
            int cnt = (int)(hi - lo) * channels;
            const int16_t *src = frame + (lo - pos) * channels;
            int16_t *dst = out + (lo - trim) * channels;
            LFOR((*L), i, 0, cnt) dst[i] = src[i];
        }
        lsync(*L);
        pos += (uint64_t)n;
    }
};

// Decode one chain.  pkt_nsamp / pkt_rng (optional) receive per-packet sample
// counts and final ranges; `out` may be null (decode only).
DNI void decode_chain(Lanes L, ChainSlot *slot, const uint8_t *data, const uint64_t *off,
                      const uint32_t *len, uint32_t first, uint32_t npkts, int channels, int16_t *out,
                      uint64_t trim, uint64_t keep, uint32_t *pkt_nsamp, uint32_t *pkt_rng, ChainResult *res)
{
    OpusDec *st = &slot->dec;
    opus_init(st, channels);
    lsync(L);
    KeepWindow win;
    win.L = &L;
    win.out = out;
    win.channels = channels;
    win.pos = 0;
    win.trim = out ? trim : 0;
    win.keep = out ? keep : 0;
    int32_t stop = 0;
    for (uint32_t k = 0; k < npkts; k++) {
        uint64_t p = (uint64_t)first + k;
        int ret = opus_decode_packet(L, st, data + off[p], (int32_t)len[p], slot->frame_buf, &slot->scratch, win);
        if (ret < 0) {
            stop = ret;
            if (L.id == 0) {
                if (pkt_nsamp) pkt_nsamp[k] = 0;
                if (pkt_rng) pkt_rng[k] = 0;
            }
            break;
        }
        if (L.id == 0) {
            if (pkt_nsamp) pkt_nsamp[k] = (uint32_t)ret;
            if (pkt_rng) pkt_rng[k] = st->rangeFinal;
        }
    }
    if (L.id == 0) {
        res->stop = stop;
        res->samples = (uint32_t)win.pos;
        res->final_range = st->rangeFinal;
    }
    lsync(L);
}

} // namespace cuo
