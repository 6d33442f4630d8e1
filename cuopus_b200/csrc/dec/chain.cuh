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

// ------------------------------------------------------------------ packet staging
//
// On the device each lane group stages its packets in shared memory with TMA
// bulk copies (cp.async.bulk global -> shared, completion on an mbarrier),
// double-buffered: packet k+1 is in flight while packet k is decoded, so the
// range decoder reads its bytes from shared memory.  Only bytes inside the
// packet are read from global memory: the 16-byte-aligned interior goes by
// TMA, the unaligned head and tail (< 16 bytes each) by plain lane loads, and
// byte a of the packet lands at buf + (a mod 16) so both sides of the copy
// stay 16-byte aligned.  Packets longer than a buffer are read in place.
// Every wait is bounded: if a copy does not complete in time the group stops
// staging (decoding continues from global memory, with the same result) and
// waits, again bounded, for its copies in flight before the chain returns.
// The buffers hold packets of up to 480 bytes (a 20 ms frame up to 192 kbps),
// larger ones are rare and read in place: staging takes its shared memory from
// the SM's L1, which the launches of narrow groups (48 chains per SM) need for
// the chains' state; with 1.5 KB buffers the 2 h file in 1 s chains decoded
// 3.5 % slower (178-179 ms against 172-173, same box, alternating).
enum { STAGE_BUF = 512, STAGE_BYTES = 2 * STAGE_BUF + 32 };   // per group: 2 buffers + 2 mbarriers

struct PacketStage {
    uint8_t *buf;        // 2 x STAGE_BUF bytes of shared memory, or null (host build / disabled)
    uint64_t *bar;       // 2 mbarriers
    unsigned parity;     // bit b: phase parity the next wait on buffer b expects
    unsigned pending;    // bit b: a TMA copy into buffer b was issued and not yet waited for
    int ok;              // staging usable (0 after a timed-out wait)
};

#ifdef __CUDACC__
DFN uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

DFN void stage_init(const Lanes &L, PacketStage &S, uint8_t *region)
{
    S.buf = region;
    S.bar = (uint64_t *)(region + 2 * STAGE_BUF);
    S.parity = 0;
    S.pending = 0;
    S.ok = 1;
    if (L.id == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    lsync(L);
}

DFN unsigned long long stage_clock_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the completion of buffer b's copy; false on timeout.  The
// limit is `polls` mbarrier.try_wait rounds and, when limit_ns > 0, also
// limit_ns of the device's global timer (whichever ends first is not a
// timeout: both must run out).
DFN bool stage_wait(PacketStage &S, int b, int polls = 1 << 20, unsigned long long limit_ns = 0)
{
    uint32_t addr = smem_u32(&S.bar[b]), par = (S.parity >> b) & 1u;
    const unsigned long long t0 = limit_ns ? stage_clock_ns() : 0;
    for (int it = 0;; it++) {
        uint32_t done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done)
                     : "r"(addr), "r"(par)
                     : "memory");
        if (done) {
            S.parity ^= 1u << b;
            S.pending &= ~(1u << b);
            return true;
        }
        if (it >= polls && (!limit_ns || stage_clock_ns() - t0 > limit_ns)) return false;
    }
}

// Start staging packet (src, n) into buffer b.  Returns false when the packet
// is read in place instead (too long, staging off).
DNI bool stage_issue(const Lanes &L, PacketStage &S, int b, const uint8_t *src, int n)
{
    if (!S.ok || n <= 0 || n > STAGE_BUF - 32) return false;
    uintptr_t a = (uintptr_t)src;
    uintptr_t lo = (a + 15) & ~(uintptr_t)15;         // first aligned byte inside the packet
    uintptr_t hi = (a + (uintptr_t)n) & ~(uintptr_t)15;   // end of the aligned interior
    uint8_t *dst = S.buf + b * STAGE_BUF + (a & 15);     // packet byte a at buf + (a mod 16)
    if (hi > lo) {
        if (L.id == 0) {
            uint32_t bytes = (uint32_t)(hi - lo);
            uint32_t bar = smem_u32(&S.bar[b]);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             smem_u32(dst + (lo - a))),
                         "l"((const void *)lo), "r"(bytes), "r"(bar)
                         : "memory");
        }
        S.pending |= 1u << b;
    } else {
        lo = hi = a + (uintptr_t)n;                  // no aligned interior: all bytes by lanes
    }
    int head = (int)(lo - a), tail0 = (int)(hi - a);
    LFOR(L, i, 0, head) dst[i] = src[i];
    LFOR(L, i, tail0, n) dst[i] = src[i];
    return true;
}

// Wait for buffer b (issued by stage_issue); false when staging gave up.  The
// lanes agree on the outcome, so a timeout switches the whole group to
// in-place reads.
DFN bool stage_ready(const Lanes &L, PacketStage &S, int b)
{
    bool ok = true;
    if (S.pending & (1u << b)) ok = stage_wait(S, b);
    ok = __all_sync(L.mask, ok);
    if (!ok) S.ok = 0;
    return ok;
}

// Before the group's region is reused or the kernel returns: let every copy in
// flight land.  A copy is at most STAGE_BUF bytes from global memory and
// lands within microseconds; the decode loop gives up on one after 2^20
// polls and reads the packet in place, but here the group must not leave its
// shared memory while the copy can still write it (a later block on the SM
// could own those bytes), so the wait runs for at least one second of the
// global timer as well.  A copy that has not landed by then means the memory
// system has failed; the group returns regardless (its chains' results are
// already written) rather than spin without end.
DFN void stage_drain(const Lanes &L, PacketStage &S)
{
    bool ok = true;
    for (int b = 0; b < 2; b++)
        if (S.pending & (1u << b)) ok = stage_wait(S, b, 1 << 20, 1000000000ull) && ok;
    if (!__all_sync(L.mask, ok)) S.ok = 0;
}
#endif

struct ChainResult {
    int32_t stop;          // 0, or the first negative opus_decode return
    uint32_t samples;      // samples per channel decoded
    uint32_t final_range;  // OPUS_GET_FINAL_RANGE after the last packet
    uint32_t time_us;      // microseconds the chain took on the device (0 on the host)
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
    // a call, not inlined: frames are emitted from several places
    MNI void operator()(const int16_t *frame, int n)
    {
        uint64_t lo = pos > trim ? pos : trim;
        uint64_t hi = pos + (uint64_t)n < trim + keep ? pos + (uint64_t)n : trim + keep;
        if (hi > lo) {
            int cnt = (int)(hi - lo) * channels;
            const int16_t *src = frame + (lo - pos) * channels;
            int16_t *dst = out + (lo - trim) * channels;
            PHASE_BEGIN(t_kc);
            LFOR((*L), i, 0, cnt) dst[i] = src[i];
            PHASE_END(PH_KEEP_COPY, t_kc, L->id);
        }
        lsync(*L);
        pos += (uint64_t)n;
    }
};

// Decode one chain.  pkt_nsamp / pkt_rng (optional) receive per-packet sample
// counts and final ranges; `out` may be null (decode only).
// `stage` (device only, may be null) stages the packets in shared memory.
// fec = 1 turns on in-band FEC: a lost (empty) packet followed by a non-empty
// one is decoded as opus_decode(next packet, 5760, decode_fec = 1), which
// conceals the same 5760 samples a lost packet always yields but takes the
// last frame's worth from the next packet's FEC (LBRR) data; the next packet
// is then decoded normally.
DNI void decode_chain(Lanes L, ChainSlot *slot, const uint8_t *data, const uint64_t *off,
                      const uint32_t *len, uint32_t first, uint32_t npkts, int channels, int16_t *out,
                      uint64_t trim, uint64_t keep, uint32_t *pkt_nsamp, uint32_t *pkt_rng, ChainResult *res,
                      PacketStage *stage, int fec)
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
#ifdef __CUDA_ARCH__
    bool next_staged = false;
    if (stage && npkts > 0) next_staged = stage_issue(L, *stage, 0, data + off[first], (int)len[first]);
#else
    (void)stage;
#endif
    for (uint32_t k = 0; k < npkts; k++) {
        uint64_t p = (uint64_t)first + k;
        const uint8_t *pk = data + off[p];
        int32_t n = (int32_t)len[p];
        int use_fec = fec && n == 0 && k + 1 < npkts && len[p + 1] > 0;
#ifdef __CUDA_ARCH__
        if (stage) {
            int b = (int)(k & 1u);
            bool cur = next_staged;
            next_staged = k + 1 < npkts && stage_issue(L, *stage, b ^ 1, data + off[p + 1], (int)len[p + 1]);
            if (cur && stage_ready(L, *stage, b)) pk = stage->buf + b * STAGE_BUF + ((uintptr_t)pk & 15);
        }
#endif
        PHASE_BEGIN(t_pk);
        if (use_fec) {   // the next packet, read in place (its staged copy is still in flight)
            pk = data + off[p + 1];
            n = (int32_t)len[p + 1];
        }
        int ret = opus_decode_packet(L, st, pk, n, slot->frame_buf, &slot->scratch, win, use_fec);
        PHASE_END(PH_PACKET, t_pk, L.id);
        lsync(L);   // every lane is done with this packet's buffer before it is refilled
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
#ifdef __CUDA_ARCH__
    if (stage) stage_drain(L, *stage);
#endif
    if (L.id == 0) {
        res->stop = stop;
        res->samples = (uint32_t)win.pos;
        res->final_range = st->rangeFinal;
    }
    lsync(L);
}

} // namespace cuo
