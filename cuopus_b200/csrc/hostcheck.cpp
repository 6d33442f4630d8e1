// Host build of the chain decoder (the same sources as the CUDA kernel,
// compiled by g++ with one lane per chain).  It is the host same-source
// check: the CPU parity tests run it against libopus to separate "the
// restatement is right" from "the CUDA execution is right".  Test-only; the
// product library never loads it and never falls back to it.
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CUO_FRAME_EVENTS 1
#include "dec/chain.cuh"

// Frame events of the host build (CUO_FRAME_EVENTS): counters the tests read
// with hc_frame_events to show which branches of the frame decode their
// streams exercise.  Index: 0 frames, 1 redundancy with celt_to_silk = 1,
// 2 redundancy with celt_to_silk = 0, 3 transitions with the 5 ms crossfade,
// 4 hybrid -> SILK silence frames, 5 concealment frames (depth 1),
// 6 SILK -> CELT transitions, 7 CELT -> SILK/hybrid transitions.
static unsigned long long g_events[8];
static pthread_mutex_t g_events_mu = PTHREAD_MUTEX_INITIALIZER;

void cuo::cuo_frame_event(int depth, int mode, int prev_mode, int redundancy, int celt_to_silk, int transition,
                          int silence_frame)
{
    pthread_mutex_lock(&g_events_mu);
    g_events[0]++;
    if (redundancy && celt_to_silk) g_events[1]++;
    if (redundancy && !celt_to_silk) g_events[2]++;
    if (transition) {
        g_events[3]++;
        if (mode == 1002) g_events[6]++;
        else g_events[7]++;
    }
    if (silence_frame) g_events[4]++;
    if (depth > 0) g_events[5]++;
    (void)prev_mode;
    pthread_mutex_unlock(&g_events_mu);
}

extern "C" {

struct hc_job {
    const uint8_t *data;
    const uint64_t *off;
    const uint32_t *len;
    const uint32_t *first, *npkts;
    const int32_t *channels;
    int16_t *pcm;
    const uint64_t *pcm_off;
    const uint64_t *trim, *keep;
    const uint64_t *rec_off;
    uint32_t *pkt_nsamp, *pkt_rng;
    cuo::ChainResult *res;
    int nchains;
    int fec;
    int next;
    pthread_mutex_t mu;
};

static void *hc_worker(void *arg)
{
    hc_job *j = (hc_job *)arg;
    cuo::ChainSlot *slot = (cuo::ChainSlot *)malloc(sizeof(cuo::ChainSlot));
    if (!slot) return nullptr;
    // poison the slot like fresh device memory: the decoder must not read
    // anything it has not initialised
    memset(slot, 0xA5, sizeof(cuo::ChainSlot));
    cuo::Lanes L{0, 1, 1u};
    for (;;) {
        pthread_mutex_lock(&j->mu);
        int c = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (c >= j->nchains) break;
        uint64_t r = j->rec_off ? j->rec_off[c] : 0;
        cuo::decode_chain(L, slot, j->data, j->off, j->len, j->first[c], j->npkts[c], j->channels[c],
                          j->pcm ? j->pcm + j->pcm_off[c] : nullptr, j->trim ? j->trim[c] : 0,
                          j->keep ? j->keep[c] : (uint64_t)-1 / 4, j->pkt_nsamp ? j->pkt_nsamp + r : nullptr,
                          j->pkt_rng ? j->pkt_rng + r : nullptr, &j->res[c], nullptr, j->fec);
    }
    free(slot);
    return nullptr;
}

// Same layout as the oracle's oref_decode_chains, plus per-chain channels and
// keep windows (trim/keep may be null: keep everything).  res: 4 words per chain.
int hc_decode_chains_fec(const uint8_t *data, const uint64_t *off, const uint32_t *len, const uint32_t *first,
                         const uint32_t *npkts, const int32_t *channels, int nchains, int16_t *pcm,
                         const uint64_t *pcm_off, const uint64_t *trim, const uint64_t *keep, const uint64_t *rec_off,
                         uint32_t *pkt_nsamp, uint32_t *pkt_rng, void *res, int nthreads, int fec)
{
    hc_job j;
    j.fec = fec;
    j.data = data; j.off = off; j.len = len; j.first = first; j.npkts = npkts; j.channels = channels;
    j.pcm = pcm; j.pcm_off = pcm_off; j.trim = trim; j.keep = keep; j.rec_off = rec_off;
    j.pkt_nsamp = pkt_nsamp; j.pkt_rng = pkt_rng; j.res = (cuo::ChainResult *)res;
    j.nchains = nchains; j.next = 0;
    pthread_mutex_init(&j.mu, nullptr);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    int started = 0;
    for (int t = 0; t < nthreads; t++) {
        if (pthread_create(&th[t], nullptr, hc_worker, &j) != 0) break;
        started++;
    }
    if (!started) hc_worker(&j);
    for (int t = 0; t < started; t++) pthread_join(th[t], nullptr);
    pthread_mutex_destroy(&j.mu);
    return 0;
}

int hc_decode_chains(const uint8_t *data, const uint64_t *off, const uint32_t *len, const uint32_t *first,
                     const uint32_t *npkts, const int32_t *channels, int nchains, int16_t *pcm,
                     const uint64_t *pcm_off, const uint64_t *trim, const uint64_t *keep, const uint64_t *rec_off,
                     uint32_t *pkt_nsamp, uint32_t *pkt_rng, void *res, int nthreads)
{
    return hc_decode_chains_fec(data, off, len, first, npkts, channels, nchains, pcm, pcm_off, trim, keep, rec_off,
                                pkt_nsamp, pkt_rng, res, nthreads, 0);
}

unsigned long hc_slot_bytes(void) { return sizeof(cuo::ChainSlot); }

// Copy the frame event counters (8 words, see cuo_frame_event) and reset them.
void hc_frame_events(unsigned long long *out)
{
    pthread_mutex_lock(&g_events_mu);
    for (int i = 0; i < 8; i++) {
        out[i] = g_events[i];
        g_events[i] = 0;
    }
    pthread_mutex_unlock(&g_events_mu);
}

}

// The range-decoder gate schedules (147 and 163 words) run through the
// decoder's own range decoder (dec/rangedec.cuh); the oracle runs the same
// schedules through libopus (oref_ec_schedule, oref_ec_schedule2).
extern "C" {

// The decoder's PVQ codeword decode (rd_uint of V(n, k), then cwrsi) on a
// buffer written by libopus's encode_pulses; y receives n pulses.
void hc_pvq_decode(const uint8_t *buf, uint32_t len, int n, int k, int32_t *y)
{
    cuo::RangeDec d;
    cuo::rd_init(&d, buf, len);
    cuo::cwrsi(n, k, cuo::rd_uint(&d, cuo::pvq_v(n, k)), y);
}

// The decoder's inverse MDCT (pre-rotation, FFT, post-rotation, TDAC
// mirror) for one block: the contract of clt_mdct_backward_c.
void hc_imdct(const int32_t *in, int32_t *out, int shift, int stride)
{
    cuo::Lanes L{0, 1, 1u};
    cuo::mdct_backward(L, in, out, shift, stride);
}

// SILK NLSF to LPC conversion of the decoder.
void hc_nlsf2a(int16_t *a_Q12, const int16_t *nlsf, int d)
{
    cuo::SilkWork sw;
    cuo::silk_nlsf2a(a_Q12, nlsf, d, &sw);
}

// The decoder's SILK resampler to 48 kHz (all-pass up2 + FIR interpolation),
// `frame` input samples per call; returns the output samples written.
int hc_silk_resample(int fs_in, const int16_t *in, int n_in, int frame, int16_t *out)
{
    cuo::Lanes L{0, 1, 1u};
    cuo::SilkResampler S;
    int16_t buf[2 * 160 + 8];
    cuo::silk_resampler_init48(&S, fs_in);
    int o = 0;
    for (int i = 0; i + frame <= n_in; i += frame) {
        cuo::silk_resample(L, &S, out + o, in + i, frame, buf);
        o += frame * (48000 / fs_in);
    }
    return o;
}

// The decoder's comb (post-)filter in place on buf + off: the serial form
// (lanes = 0) or the block-parallel form the decoder runs (lanes = 1, here
// with a single lane walking the same blocks).
void hc_comb_filter(int32_t *buf, int off, int T0, int T1, int N, int g0, int g1, int tapset0, int tapset1,
                    int lanes)
{
    if (lanes) {
        cuo::Lanes L{0, 1, 1u};
        cuo::comb_filter_lanes(L, buf + off, buf + off, T0, T1, N, (int16_t)g0, (int16_t)g1, tapset0, tapset1,
                               cuo::T_celt_window, cuo::CELT_OVERLAP);
    } else {
        cuo::comb_filter(buf + off, buf + off, T0, T1, N, (int16_t)g0, (int16_t)g1, tapset0, tapset1,
                         cuo::T_celt_window, cuo::CELT_OVERLAP);
    }
}

// The decoder's CELT bit allocation (clt_compute_allocation, decode mode)
// with its caps, same output layout as the oracle's oref_alloc.
int hc_alloc(const uint8_t *buf, uint32_t len, int start, int end, const int32_t *offsets, int alloc_trim,
             int32_t total, int C, int LM, int32_t *out)
{
    static thread_local cuo::CeltScratch w;
    int32_t cap[21], pulses[21] = {}, ebits[21] = {}, fine_priority[21] = {}, balance = 0;
    int intensity = 0, dual_stereo = 0;
    cuo::RangeDec d;
    cuo::init_caps(cap, LM, C);
    cuo::rd_init(&d, buf, len);
    int coded = cuo::clt_compute_allocation(start, end, offsets, cap, alloc_trim, &intensity, &dual_stereo, total,
                                            &balance, pulses, ebits, fine_priority, C, LM, &d, &w);
    int k = 0;
    out[k++] = coded;
    out[k++] = intensity;
    out[k++] = dual_stereo;
    out[k++] = balance;
    for (int i = 0; i < 21; i++) out[k++] = pulses[i];
    for (int i = 0; i < 21; i++) out[k++] = ebits[i];
    for (int i = 0; i < 21; i++) out[k++] = fine_priority[i];
    out[k++] = (int32_t)cuo::rd_tell_frac(&d);
    out[k++] = (int32_t)d.rng;
    return 0;
}

// Allocation then the decoder's band decoding (quant_all_bands_dec), the
// oracle's oref_bands layout.
int hc_bands(const uint8_t *buf, uint32_t len, int start, int end, const int32_t *offsets, int alloc_trim, int C,
             int LM, int shortBlocks, int spread, const int32_t *tf_res, int disable_inv, uint32_t seed,
             int16_t *X_out, uint8_t *cm_out, uint32_t *tail)
{
    static thread_local cuo::CeltScratch w;
    cuo::Lanes L{0, 1, 1u};
    int32_t cap[21], pulses[21] = {}, ebits[21] = {}, fine_priority[21] = {}, balance = 0;
    int intensity = 0, dual_stereo = 0;
    int N = 120 << LM;
    memset(w.X, 0, sizeof w.X);
    memset(w.collapse_masks, 0, sizeof w.collapse_masks);
    cuo::RangeDec d;
    cuo::init_caps(cap, LM, C);
    cuo::rd_init(&d, buf, len);
    int32_t bits = (int32_t)(len * 8 << 3) - (int32_t)cuo::rd_tell_frac(&d) - 1;
    int coded = cuo::clt_compute_allocation(start, end, offsets, cap, alloc_trim, &intensity, &dual_stereo, bits,
                                            &balance, pulses, ebits, fine_priority, C, LM, &d, &w);
    uint32_t s = seed;
    cuo::quant_all_bands_dec(L, start, end, w.X, C == 2 ? w.X + N : nullptr, w.collapse_masks, pulses, shortBlocks,
                             spread, dual_stereo, intensity, tf_res, (int32_t)(len * (8 << 3)), balance, &d, LM,
                             coded, &s, disable_inv, &w);
    memcpy(X_out, w.X, sizeof(int16_t) * C * N);
    memcpy(cm_out, w.collapse_masks, (size_t)C * 21);
    tail[0] = s;
    tail[1] = cuo::rd_tell_frac(&d);
    tail[2] = d.rng;
    return 0;
}

// The decoder's band-energy decoding around the allocation, the oracle's
// oref_energy layout.
int hc_energy(const uint8_t *buf, uint32_t len, int start, int end, int intra, const int32_t *offsets,
              int alloc_trim, int C, int LM, int16_t *oldE, uint32_t *tail)
{
    static thread_local cuo::CeltScratch w;
    int32_t cap[21], pulses[21] = {}, ebits[21] = {}, fine_priority[21] = {}, balance = 0;
    int intensity = 0, dual_stereo = 0;
    cuo::RangeDec d;
    cuo::rd_init(&d, buf, len);
    cuo::unquant_coarse_energy(start, end, oldE, intra, &d, C, LM);
    cuo::init_caps(cap, LM, C);
    int32_t bits = (int32_t)(len * 8 << 3) - (int32_t)cuo::rd_tell_frac(&d) - 1;
    cuo::clt_compute_allocation(start, end, offsets, cap, alloc_trim, &intensity, &dual_stereo, bits, &balance,
                                pulses, ebits, fine_priority, C, LM, &d, &w);
    cuo::unquant_fine_energy(start, end, oldE, ebits, &d, C);
    cuo::unquant_energy_finalise(start, end, oldE, ebits, fine_priority, (int)len * 8 - cuo::rd_tell(&d), &d, C);
    tail[0] = cuo::rd_tell_frac(&d);
    tail[1] = d.rng;
    return 0;
}

// The decoder's SILK entropy decoding (indices and pulses), the oracle's
// oref_silk_entropy layout.
int hc_silk_entropy(const uint8_t *buf, uint32_t len, int fs_kHz, int nb_subfr, int frames, const int32_t *vad,
                    int cond_first, int32_t *out, uint32_t *tail)
{
    static thread_local cuo::SilkChan c;
    static thread_local cuo::SilkScratch w;
    cuo::silk_reset_chan(&c);
    c.nb_subfr = nb_subfr;
    cuo::silk_decoder_set_fs(&c, fs_kHz, 48000);
    cuo::RangeDec d;
    cuo::rd_init(&d, buf, len);
    int k = 0;
    for (int f = 0; f < frames; f++) {
        c.VAD_flags[f] = vad[f];
        int cond = f == 0 ? (cond_first ? cuo::CODE_COND : cuo::CODE_INDEP) : cuo::CODE_COND;
        cuo::silk_decode_indices(&c, &d, f, 0, cond, &w.sw);
        cuo::silk_decode_pulses(&d, w.pulses, c.indices.signalType, c.indices.quantOffsetType, c.frame_length,
                                &w.sw);
        const cuo::SilkIndices *ix = &c.indices;
        out[k++] = ix->signalType;
        out[k++] = ix->quantOffsetType;
        for (int i = 0; i < 4; i++) out[k++] = ix->GainsIndices[i];
        for (int i = 0; i < 4; i++) out[k++] = ix->LTPIndex[i];
        for (int i = 0; i < 17; i++) out[k++] = ix->NLSFIndices[i];
        out[k++] = ix->lagIndex;
        out[k++] = ix->contourIndex;
        out[k++] = ix->NLSFInterpCoef_Q2;
        out[k++] = ix->PERIndex;
        out[k++] = ix->LTP_scaleIndex;
        out[k++] = ix->Seed;
        for (int i = 0; i < c.frame_length; i++) out[k++] = w.pulses[i];
    }
    tail[0] = (uint32_t)cuo::rd_tell(&d);
    tail[1] = d.rng;
    return k;
}

// The decoder's SILK frames at the internal rate, the oracle's
// oref_silk_frames layout.
int hc_silk_frames(const uint8_t *buf, uint32_t len, int fs_kHz, int nb_subfr, int frames, const int32_t *vad,
                   const int32_t *lost, int16_t *out, uint32_t *tail)
{
    static thread_local cuo::SilkChan c;
    static thread_local cuo::SilkScratch w;
    cuo::Lanes L{0, 1, 1u};
    cuo::silk_reset_chan(&c);
    c.nb_subfr = nb_subfr;
    c.nFramesPerPacket = 1;
    cuo::silk_decoder_set_fs(&c, fs_kHz, 48000);
    cuo::RangeDec d;
    cuo::rd_init(&d, buf, len);
    int o = 0;
    for (int f = 0; f < frames; f++) {
        int n = 0;
        c.nFramesDecoded = 0;
        c.VAD_flags[0] = vad[f];
        cuo::silk_decode_frame(L, &c, &d, out + o, &n, lost[f], f == 0 ? cuo::CODE_INDEP : cuo::CODE_COND, &w);
        o += n;
    }
    tail[0] = (uint32_t)cuo::rd_tell(&d);
    tail[1] = d.rng;
    return o;
}

// The decoder's CELT frames of one stream, the oracle's oref_celt_frames
// layout (its final range is the state's rng after each frame).
int hc_celt_frames(const uint8_t *data, const uint32_t *lens, int frames, int C, int LM, int end, int16_t *out,
                   uint32_t *rng)
{
    static thread_local cuo::CeltDec st;
    static thread_local cuo::CeltScratch w;
    cuo::Lanes L{0, 1, 1u};
    cuo::celt_init(&st, C);
    st.end = end;
    int N = 120 << LM;
    size_t off = 0;
    for (int f = 0; f < frames; f++) {
        int ret = cuo::celt_decode(L, &st, lens[f] ? data + off : nullptr, (int)lens[f], out + (size_t)f * N * C, N,
                                   nullptr, 0, &w);
        rng[f] = ret < 0 ? (uint32_t)ret : st.rng;
        off += lens[f];
    }
    return 0;
}

// The decoder's fixed-point helpers elementwise, numbered as the oracle's
// oref_mathops.
int hc_mathops(int op, const int32_t *a, const int32_t *b, const int32_t *q, int n, int32_t *out)
{
    for (int i = 0; i < n; i++) {
        int32_t r;
        switch (op) {
        case 0: r = (int32_t)cuo::c_isqrt32((uint32_t)a[i]); break;
        case 1: r = cuo::c_rcp(a[i]); break;
        case 2: r = cuo::c_frac_div32(a[i], b[i]); break;
        case 3: r = cuo::c_rsqrt_norm(a[i]); break;
        case 4: r = cuo::c_sqrt(a[i]); break;
        case 5: r = cuo::c_cos_norm(a[i]); break;
        case 6: r = cuo::c_exp2((int16_t)a[i]); break;
        case 7: r = cuo::bitexact_cos((int16_t)a[i]); break;
        case 8: r = cuo::bitexact_log2tan(a[i], b[i]); break;
        case 9: r = cuo::s_sqrt_approx(a[i]); break;
        case 10: r = cuo::s_div32_varq(a[i], b[i], q[i]); break;
        case 11: r = cuo::s_inverse32_varq(a[i], q[i]); break;
        case 12: r = cuo::s_log2lin(a[i]); break;
        case 13: r = cuo::s_lin2log(a[i]); break;
        default: return -1;
        }
        out[i] = r;
    }
    return 0;
}

void hc_ec_schedule(const uint8_t *buf, uint32_t len, uint32_t *out)
{
    static const uint8_t icdf_tab[8] = {120, 112, 96, 64, 32, 16, 8, 0};
    cuo::RangeDec d;
    int k = 0;
    cuo::rd_init(&d, buf, len);
    for (int i = 0; i < 64; i++) out[k++] = (uint32_t)cuo::rd_bit_logp(&d, 1);
    for (int i = 0; i < 32; i++) out[k++] = (uint32_t)cuo::rd_icdf(&d, icdf_tab, 7);
    for (int i = 0; i < 32; i++) out[k++] = cuo::rd_uint(&d, 2000);
    for (int i = 0; i < 16; i++) out[k++] = cuo::rd_bits(&d, 11);
    out[k++] = (uint32_t)cuo::rd_tell(&d);
    out[k++] = d.rng;
    out[k++] = (uint32_t)d.error;
}

void hc_ec_schedule2(const uint8_t *buf, uint32_t len, uint32_t *out)
{
    static const uint8_t icdf_tab[8] = {200, 150, 100, 60, 30, 12, 4, 0};
    cuo::RangeDec d;
    int k = 0;
    cuo::rd_init(&d, buf, len);
    for (int i = 0; i < 16; i++) {
        unsigned fs = 2000 + 1500 * (unsigned)(i & 7);
        int decay = 6000 + 1000 * (i & 7);
        out[k++] = (uint32_t)cuo::rd_laplace(&d, fs, decay);
        unsigned s = cuo::rd_decode_bin(&d, 9);
        cuo::rd_update(&d, s, s + 1, 512);
        out[k++] = s;
        out[k++] = (uint32_t)cuo::rd_bit_logp(&d, 1 + (i & 3));
        out[k++] = (uint32_t)cuo::rd_icdf(&d, icdf_tab, 8);
        out[k++] = cuo::rd_uint(&d, 3 + (unsigned)i);
        out[k++] = cuo::rd_uint(&d, 70000u + 977u * (unsigned)i);
        out[k++] = cuo::rd_bits(&d, 1 + (unsigned)(i % 16));
        out[k++] = cuo::rd_tell_frac(&d);
        out[k++] = (uint32_t)cuo::rd_tell(&d);
        out[k++] = d.rng;
    }
    out[k++] = cuo::rd_tell_frac(&d);
    out[k++] = d.rng;
    out[k++] = (uint32_t)d.error;
}

}
