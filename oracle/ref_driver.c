/* Oracle driver over the reference's vendored libopus 1.5.2 (FIXED_POINT).
 *
 * TEST INFRASTRUCTURE ONLY.  Linked into oracle/_ref/libopus_ref.so together
 * with the vendored libopus objects.  The product never loads this library.
 *
 * 1. oref_decode_chains: the bit-exactness oracle.  Every chain gets a FRESH
 *    OpusDecoder(48000, channels) and decodes its packet range in order with
 *    opus_decode(..., frame_size=5760, decode_fec=0) -- the chain protocol of the
 *    reference's decode kernel (cuopus_kernels.cuh:41-69, a fresh
 *    cu_opus_decoder_init per chain, then cu_opus_decode per packet) checked
 *    against libopus in harness2.cu:200-253.  Per packet it records the sample
 *    count and OPUS_GET_FINAL_RANGE; per chain the stop status and sample total.
 *    Chains run on a pthread pool (dynamic assignment) so the same entry point
 *    is the timed CPU baseline.  oref_decode_chains_fec adds in-band FEC: a
 *    lost (empty) packet followed by a non-empty one is decoded as
 *    opus_decode(next packet, 5760, decode_fec=1), the next packet then
 *    normally (the use of decode_fec in src/opus_demo.c, with the chain
 *    protocol's frame size).
 *
 * 2. oref_encode / oref_encode_opts: the corpus encoder.  Drives the vendored encoder frame by
 *    frame at 48 kHz with per-segment forced mode / bandwidth / frame size /
 *    bitrate (OPUS_SET_FORCE_MODE is the private request 11002 of
 *    src/opus_private.h:141; per-frame switching follows the idea of
 *    src/opus_demo.c:820-872).  It keeps encoding zero-padded frames until the
 *    packets cover pre-skip + input length, so an Ogg muxer can express the
 *    exact end trim (RFC 7845 sec. 4.4).
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "opus.h"

#define OREF_FORCE_MODE_REQUEST 11002   /* src/opus_private.h:141 */
#define OREF_MAX_PKT_SAMPLES 5760       /* 120 ms at 48 kHz */

/* ------------------------------------------------------------------ decode */

typedef struct {
    const uint8_t *data;
    const uint64_t *off;
    const uint32_t *len;
    const uint32_t *first;
    const uint32_t *npkts;
    const uint64_t *rec_off;    /* per chain: index of its first per-packet record */
    const uint64_t *pcm_off;    /* per chain: int16 element offset into pcm */
    int nchains, channels;
    int16_t *pcm;               /* may be NULL: decode into scratch only */
    uint32_t *pkt_nsamp;        /* per record (may be NULL) */
    uint32_t *pkt_rng;          /* per record (may be NULL) */
    int32_t *chain_status;      /* per chain: 0 or first negative opus_decode return */
    uint64_t *chain_samples;    /* per chain: samples per channel decoded */
    int fec;                    /* in-band FEC for lost packets */
    volatile int next;
    pthread_mutex_t mu;
} oref_job;

static void *oref_worker(void *arg)
{
    oref_job *j = (oref_job *)arg;
    int err = 0;
    OpusDecoder *dec = (OpusDecoder *)malloc((size_t)opus_decoder_get_size(j->channels));
    int16_t *scratch = (int16_t *)malloc(sizeof(int16_t) * OREF_MAX_PKT_SAMPLES * j->channels);
    if (!dec || !scratch) { free(dec); free(scratch); return NULL; }
    for (;;) {
        pthread_mutex_lock(&j->mu);
        int c = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (c >= j->nchains) break;
        err = opus_decoder_init(dec, 48000, j->channels);
        int32_t status = err;
        uint64_t total = 0;
        if (!err) {
            for (uint32_t k = 0; k < j->npkts[c]; k++) {
                uint64_t p = (uint64_t)j->first[c] + k;
                int16_t *out = j->pcm ? j->pcm + j->pcm_off[c] + total * (uint64_t)j->channels
                                      : scratch;
                int use_fec = j->fec && j->len[p] == 0 && k + 1 < j->npkts[c] && j->len[p + 1] > 0;
                uint64_t q = use_fec ? p + 1 : p;
                int ret = opus_decode(dec, j->data + j->off[q], (opus_int32)j->len[q], out,
                                      OREF_MAX_PKT_SAMPLES, use_fec);
                uint64_t r = j->rec_off ? j->rec_off[c] + k : 0;
                if (ret < 0) {
                    status = ret;
                    if (j->pkt_nsamp) j->pkt_nsamp[r] = 0;
                    if (j->pkt_rng) j->pkt_rng[r] = 0;
                    break;
                }
                opus_uint32 rng = 0;
                opus_decoder_ctl(dec, OPUS_GET_FINAL_RANGE(&rng));
                if (j->pkt_nsamp) j->pkt_nsamp[r] = (uint32_t)ret;
                if (j->pkt_rng) j->pkt_rng[r] = (uint32_t)rng;
                total += (uint64_t)ret;
            }
        }
        if (j->chain_status) j->chain_status[c] = status;
        if (j->chain_samples) j->chain_samples[c] = total;
    }
    free(dec);
    free(scratch);
    return NULL;
}

int oref_decode_chains_fec(const uint8_t *data, const uint64_t *off, const uint32_t *len,
                           const uint32_t *first, const uint32_t *npkts, int nchains,
                           int channels, int16_t *pcm, const uint64_t *pcm_off,
                           const uint64_t *rec_off, uint32_t *pkt_nsamp, uint32_t *pkt_rng,
                           int32_t *chain_status, uint64_t *chain_samples, int nthreads, int fec);

/* Decode nchains chains; returns 0, or -1 when a thread could not start. */
int oref_decode_chains(const uint8_t *data, const uint64_t *off, const uint32_t *len,
                       const uint32_t *first, const uint32_t *npkts, int nchains,
                       int channels, int16_t *pcm, const uint64_t *pcm_off,
                       const uint64_t *rec_off, uint32_t *pkt_nsamp, uint32_t *pkt_rng,
                       int32_t *chain_status, uint64_t *chain_samples, int nthreads)
{
    return oref_decode_chains_fec(data, off, len, first, npkts, nchains, channels, pcm, pcm_off, rec_off,
                                  pkt_nsamp, pkt_rng, chain_status, chain_samples, nthreads, 0);
}

int oref_decode_chains_fec(const uint8_t *data, const uint64_t *off, const uint32_t *len,
                           const uint32_t *first, const uint32_t *npkts, int nchains,
                           int channels, int16_t *pcm, const uint64_t *pcm_off,
                           const uint64_t *rec_off, uint32_t *pkt_nsamp, uint32_t *pkt_rng,
                           int32_t *chain_status, uint64_t *chain_samples, int nthreads, int fec)
{
    oref_job j;
    memset(&j, 0, sizeof(j));
    j.fec = fec;
    j.data = data; j.off = off; j.len = len; j.first = first; j.npkts = npkts;
    j.rec_off = rec_off; j.pcm_off = pcm_off; j.nchains = nchains; j.channels = channels;
    j.pcm = pcm; j.pkt_nsamp = pkt_nsamp; j.pkt_rng = pkt_rng;
    j.chain_status = chain_status; j.chain_samples = chain_samples;
    j.next = 0;
    pthread_mutex_init(&j.mu, NULL);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 1024) nthreads = 1024;
    pthread_t th[1024];
    int started = 0, rc = 0;
    for (int t = 0; t < nthreads; t++) {
        if (pthread_create(&th[t], NULL, oref_worker, &j) != 0) { rc = -1; break; }
        started++;
    }
    if (started == 0) oref_worker(&j);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&j.mu);
    return rc;
}

/* ------------------------------------------------------------------ full-size check
 *
 * oref_check_chains: the parity check of a whole decoded batch, for batches
 * whose PCM is too large to hold twice.  Every chain is decoded with a fresh
 * OpusDecoder(48000, chans[c]) under the chain protocol above (decode_fec = 0)
 * and compared, packet by packet, against the batch under test: the samples
 * of its keep window [trim, trim + keep) against got_pcm + got_off[c]
 * (interleaved int16), and at the end the stop status, the samples decoded
 * and the final range against got_res[4c + 0..2] ({stop, samples,
 * final_range, time}, the decoder's per-chain result record).  bad[c]
 * receives the number of differing int16 values of chain c; flags[c] bit 0 a
 * different stop status, bit 1 a different sample count, bit 2 a different
 * final range.  Chains run on a pthread pool.  Returns 0, or -1 when no thread
 * could start. */
typedef struct {
    const uint8_t *data;
    const uint64_t *off;
    const uint32_t *len;
    const uint32_t *first, *npkts;
    const uint8_t *chans;
    const uint64_t *trim, *keep, *got_off;
    const int16_t *got_pcm;
    const uint32_t *got_res;
    uint64_t *bad;
    uint32_t *flags;
    int nchains;
    volatile int next;
    pthread_mutex_t mu;
} oref_check_job;

static void *oref_check_worker(void *arg)
{
    oref_check_job *j = (oref_check_job *)arg;
    OpusDecoder *dec = (OpusDecoder *)malloc((size_t)opus_decoder_get_size(2));
    int16_t *buf = (int16_t *)malloc(sizeof(int16_t) * OREF_MAX_PKT_SAMPLES * 2);
    if (!dec || !buf) { free(dec); free(buf); return NULL; }
    for (;;) {
        pthread_mutex_lock(&j->mu);
        int c = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (c >= j->nchains) break;
        int ch = j->chans[c];
        int32_t status = opus_decoder_init(dec, 48000, ch);
        uint64_t pos = 0, bad = 0;
        opus_uint32 rng = 0;
        const uint64_t lo = j->trim[c], hi = j->trim[c] + j->keep[c];
        const int16_t *got = j->got_pcm + j->got_off[c];
        if (status == 0) {
            for (uint32_t k = 0; k < j->npkts[c]; k++) {
                uint64_t p = (uint64_t)j->first[c] + k;
                int ret = opus_decode(dec, j->data + j->off[p], (opus_int32)j->len[p], buf, OREF_MAX_PKT_SAMPLES, 0);
                if (ret < 0) { status = ret; break; }
                opus_decoder_ctl(dec, OPUS_GET_FINAL_RANGE(&rng));
                uint64_t a = pos > lo ? pos : lo, b = pos + (uint64_t)ret < hi ? pos + (uint64_t)ret : hi;
                for (uint64_t t = a; t < b; t++)
                    for (int q = 0; q < ch; q++)
                        bad += buf[(t - pos) * (uint64_t)ch + (uint64_t)q] != got[(t - lo) * (uint64_t)ch + (uint64_t)q];
                pos += (uint64_t)ret;
            }
        }
        if (pos < hi) bad += (hi - (pos > lo ? pos : lo)) * (uint64_t)ch;   /* window not covered */
        const uint32_t *r = j->got_res + 4 * (uint64_t)c;
        uint32_t f = 0;
        if ((int32_t)r[0] != status) f |= 1u;
        if ((uint64_t)r[1] != pos) f |= 2u;
        if (r[2] != (uint32_t)rng) f |= 4u;
        j->bad[c] = bad;
        j->flags[c] = f;
    }
    free(dec);
    free(buf);
    return NULL;
}

int oref_check_chains(const uint8_t *data, const uint64_t *off, const uint32_t *len, const uint32_t *first,
                      const uint32_t *npkts, const uint8_t *chans, int nchains, const uint64_t *trim,
                      const uint64_t *keep, const int16_t *got_pcm, const uint64_t *got_off,
                      const uint32_t *got_res, uint64_t *bad, uint32_t *flags, int nthreads)
{
    oref_check_job j;
    memset(&j, 0, sizeof(j));
    j.data = data; j.off = off; j.len = len; j.first = first; j.npkts = npkts; j.chans = chans;
    j.trim = trim; j.keep = keep; j.got_off = got_off; j.got_pcm = got_pcm; j.got_res = got_res;
    j.bad = bad; j.flags = flags; j.nchains = nchains; j.next = 0;
    pthread_mutex_init(&j.mu, NULL);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 1024) nthreads = 1024;
    pthread_t th[1024];
    int started = 0, rc = 0;
    for (int t = 0; t < nthreads; t++) {
        if (pthread_create(&th[t], NULL, oref_check_worker, &j) != 0) { rc = -1; break; }
        started++;
    }
    if (started == 0) oref_check_worker(&j);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&j.mu);
    return started == 0 && nchains > 0 && rc ? -1 : 0;
}

/* ------------------------------------------------------------------ encode */

typedef struct {
    int64_t start;      /* first input sample (per channel) of the segment */
    int32_t mode;       /* 1000 SILK, 1001 hybrid, 1002 CELT, -1000 = auto */
    int32_t bandwidth;  /* OPUS_BANDWIDTH_* or -1000 = auto */
    int32_t frame_size; /* samples at 48 kHz: 120 240 480 960 1920 2880 */
    int32_t bitrate;    /* bits per second */
    int32_t force_channels; /* -1000 auto, 1 or 2 */
} oref_seg;

/* Encode n samples per channel of interleaved pcm.  Writes packets back to back
 * into out (capacity out_cap bytes) and their lengths into pkt_len (capacity
 * max_pkts).  Returns the packet count, or a negative value on error.
 * *preskip receives OPUS_GET_LOOKAHEAD. */
int oref_encode_opts(const int16_t *pcm, int64_t n, int channels, const oref_seg *segs,
                     int nsegs, int application, int complexity, int vbr,
                     uint8_t *out, uint64_t out_cap, uint32_t *pkt_len, int max_pkts,
                     int *preskip, int inband_fec, int loss_perc, int dtx);

int oref_encode(const int16_t *pcm, int64_t n, int channels, const oref_seg *segs,
                int nsegs, int application, int complexity, int vbr,
                uint8_t *out, uint64_t out_cap, uint32_t *pkt_len, int max_pkts,
                int *preskip)
{
    return oref_encode_opts(pcm, n, channels, segs, nsegs, application, complexity, vbr, out, out_cap, pkt_len,
                            max_pkts, preskip, 0, 0, 0);
}

/* oref_encode with in-band FEC (LBRR frames, sized for loss_perc % loss) and
 * DTX switched on or off. */
int oref_encode_opts(const int16_t *pcm, int64_t n, int channels, const oref_seg *segs,
                     int nsegs, int application, int complexity, int vbr,
                     uint8_t *out, uint64_t out_cap, uint32_t *pkt_len, int max_pkts,
                     int *preskip, int inband_fec, int loss_perc, int dtx)
{
    int err = 0;
    OpusEncoder *enc = opus_encoder_create(48000, channels, application, &err);
    if (!enc || err) return -1000 + err;
    opus_encoder_ctl(enc, OPUS_SET_COMPLEXITY(complexity));
    opus_encoder_ctl(enc, OPUS_SET_VBR(vbr));
    opus_encoder_ctl(enc, OPUS_SET_INBAND_FEC(inband_fec));
    opus_encoder_ctl(enc, OPUS_SET_DTX(dtx));
    opus_encoder_ctl(enc, OPUS_SET_PACKET_LOSS_PERC(loss_perc));
    int la = 0;
    opus_encoder_ctl(enc, OPUS_GET_LOOKAHEAD(&la));
    if (preskip) *preskip = la;

    int16_t frame[2880 * 2];
    int64_t pos = 0, covered = 0;
    uint64_t w = 0;
    int np = 0, si = -1;
    while (covered < (int64_t)la + n) {
        /* segment in force at the current input position */
        int s = 0;
        while (s + 1 < nsegs && segs[s + 1].start <= pos) s++;
        if (s != si) {
            si = s;
            opus_encoder_ctl(enc, OREF_FORCE_MODE_REQUEST, (opus_int32)segs[s].mode);
            opus_encoder_ctl(enc, OPUS_SET_BANDWIDTH(segs[s].bandwidth));
            opus_encoder_ctl(enc, OPUS_SET_BITRATE(segs[s].bitrate));
            opus_encoder_ctl(enc, OPUS_SET_FORCE_CHANNELS(segs[s].force_channels));
        }
        int fs = segs[s].frame_size;
        for (int i = 0; i < fs; i++)
            for (int ch = 0; ch < channels; ch++) {
                int64_t at = pos + i;
                frame[i * channels + ch] = at < n ? pcm[at * channels + ch] : 0;
            }
        if (np >= max_pkts) { opus_encoder_destroy(enc); return -2000; }
        uint64_t room = out_cap - w;
        if (room > 1500) room = 1500;
        int nb = opus_encode(enc, frame, fs, out + w, (opus_int32)room);
        if (nb < 0) { opus_encoder_destroy(enc); return -3000 + nb; }
        pkt_len[np++] = (uint32_t)nb;
        w += (uint64_t)nb;
        pos += fs;
        covered += fs;
        if (out_cap - w < 1500) { opus_encoder_destroy(enc); return -4000; }
    }
    opus_encoder_destroy(enc);
    return np;
}

/* libopus version string of the oracle build, for logs. */
const char *oref_version(void) { return opus_get_version_string(); }

/* ------------------------------------------------------------------ range decoder schedules */

#include "entdec.h"
#include "laplace.h"

/* The reference's phase-1 range-decoder gate (schedule.inc:18-36) run through
 * libopus celt/entdec.c: on one buffer, 64 ec_dec_bit_logp(1), 32
 * ec_dec_icdf({120,112,96,64,32,16,8,0}, 7), 32 ec_dec_uint(2000), 16
 * ec_dec_bits(11), then ec_tell, rng and error: 147 words. */
void oref_ec_schedule(const uint8_t *buf, uint32_t len, uint32_t *out)
{
    static const unsigned char icdf_tab[8] = {120, 112, 96, 64, 32, 16, 8, 0};
    ec_dec dec;
    int i, k = 0;
    ec_dec_init(&dec, (unsigned char *)buf, len);
    for (i = 0; i < 64; i++) out[k++] = (uint32_t)ec_dec_bit_logp(&dec, 1);
    for (i = 0; i < 32; i++) out[k++] = (uint32_t)ec_dec_icdf(&dec, icdf_tab, 7);
    for (i = 0; i < 32; i++) out[k++] = (uint32_t)ec_dec_uint(&dec, 2000);
    for (i = 0; i < 16; i++) out[k++] = (uint32_t)ec_dec_bits(&dec, 11);
    out[k++] = (uint32_t)ec_tell(&dec);
    out[k++] = dec.rng;
    out[k++] = (uint32_t)dec.error;
}

/* A wider schedule over the same entry points plus those the gate leaves out
 * (ec_decode_bin + ec_dec_update, ec_laplace_decode, ec_tell_frac, small and
 * large ec_dec_uint): 16 rounds of 10 words, then tell_frac, rng, error. */
void oref_ec_schedule2(const uint8_t *buf, uint32_t len, uint32_t *out)
{
    static const unsigned char icdf_tab[8] = {200, 150, 100, 60, 30, 12, 4, 0};
    ec_dec dec;
    int i, k = 0;
    ec_dec_init(&dec, (unsigned char *)buf, len);
    for (i = 0; i < 16; i++) {
        unsigned fs = 2000 + 1500 * (unsigned)(i & 7);
        int decay = 6000 + 1000 * (i & 7);
        out[k++] = (uint32_t)ec_laplace_decode(&dec, fs, decay);
        unsigned s = ec_decode_bin(&dec, 9);
        ec_dec_update(&dec, s, s + 1, 512);
        out[k++] = s;
        out[k++] = (uint32_t)ec_dec_bit_logp(&dec, 1 + (i & 3));
        out[k++] = (uint32_t)ec_dec_icdf(&dec, icdf_tab, 8);
        out[k++] = ec_dec_uint(&dec, 3 + (unsigned)i);
        out[k++] = ec_dec_uint(&dec, 70000u + 977u * (unsigned)i);
        out[k++] = ec_dec_bits(&dec, 1 + (unsigned)(i % 16));
        out[k++] = ec_tell_frac(&dec);
        out[k++] = (uint32_t)ec_tell(&dec);
        out[k++] = dec.rng;
    }
    out[k++] = ec_tell_frac(&dec);
    out[k++] = dec.rng;
    out[k++] = (uint32_t)dec.error;
}

/* ------------------------------------------------------------------ PVQ codewords */

#include "entenc.h"
#include "cwrs.h"

/* celt/cwrs.c round trip: encode the pulse vector y (n entries, sum of
 * magnitudes k) with encode_pulses into buf (cap bytes, the range coder's
 * front and raw-bit tail both inside it), then decode it back with
 * decode_pulses into y_out.  Returns 0, or the encoder's error flag. */
int oref_pvq_roundtrip(int n, int k, const int *y, unsigned char *buf, uint32_t cap, int *y_out)
{
    ec_enc enc;
    ec_dec dec;
    memset(buf, 0, cap);
    ec_enc_init(&enc, buf, cap);
    encode_pulses(y, n, k, &enc);
    ec_enc_done(&enc);
    if (enc.error) return enc.error;
    ec_dec_init(&dec, buf, cap);
    decode_pulses(y_out, n, k, &dec);
    return dec.error;
}

/* ------------------------------------------------------------------ inverse MDCT */

#include "modes.h"
#include "mdct.h"

/* celt/mdct.c clt_mdct_backward_c of the 48 kHz / 960-sample mode (the one
 * the decoder uses) on in[] with the given shift (0 = 20 ms ... 3 = 2.5 ms)
 * and stride (short blocks); out[] holds the overlap history on entry, as in
 * celt_synthesis.  Returns 0, or -1 when the mode is unavailable. */
int oref_imdct(const int32_t *in, int32_t *out, int shift, int stride)
{
    int err = 0;
    const CELTMode *m = opus_custom_mode_create(48000, 960, &err);
    if (!m || err) return -1;
    clt_mdct_backward_c(&m->mdct, (kiss_fft_scalar *)in, out, m->window, m->overlap, shift, stride, 0);
    return 0;
}

/* ------------------------------------------------------------------ SILK / CELT components */

#include "SigProc_FIX.h"
#include "celt.h"

/* silk/NLSF2A.c: NLSF (Q15, d of them) to LPC coefficients (Q12). */
void oref_nlsf2a(int16_t *a_Q12, const int16_t *nlsf, int d)
{
    silk_NLSF2A(a_Q12, nlsf, d, 0);
}

/* silk/resampler.c from fs_in to 48 kHz, the decoder's set-up, fed `frame`
 * input samples per call for n_in samples: out receives n_in * 48000 / fs_in. */
int oref_silk_resample(int fs_in, const int16_t *in, int n_in, int frame, int16_t *out)
{
    silk_resampler_state_struct S;
    if (silk_resampler_init(&S, fs_in, 48000, 0)) return -1;
    int o = 0;
    for (int i = 0; i + frame <= n_in; i += frame) {
        if (silk_resampler(&S, out + o, in + i, frame)) return -2;
        o += frame * (48000 / fs_in);
    }
    return o;
}

/* celt/celt.c comb_filter in place on buf + off (the history before it is
 * read), with the 48 kHz mode's window and overlap. */
int oref_comb_filter(int32_t *buf, int off, int T0, int T1, int N, int g0, int g1, int tapset0, int tapset1)
{
    int err = 0;
    const CELTMode *m = opus_custom_mode_create(48000, 960, &err);
    if (!m || err) return -1;
    comb_filter(buf + off, buf + off, T0, T1, N, (opus_val16)g0, (opus_val16)g1, tapset0, tapset1, m->window,
                m->overlap, 0);
    return 0;
}

#include "rate.h"

/* celt/rate.c clt_compute_allocation in decode mode (bits read from a range
 * decoder over buf) for the 48 kHz mode, caps from celt/celt.c init_caps.
 * out: codedBands, intensity, dual_stereo, balance, then pulses[21],
 * ebits[21], fine_priority[21], then the decoder's tell_frac and rng. */
int oref_alloc(const uint8_t *buf, uint32_t len, int start, int end, const int *offsets, int alloc_trim,
               int32_t total, int C, int LM, int32_t *out)
{
    int err = 0, cap[21], pulses[21] = {0}, ebits[21] = {0}, fine_priority[21] = {0}, intensity = 0, dual_stereo = 0;
    opus_int32 balance = 0;
    ec_dec dec;
    const CELTMode *m = opus_custom_mode_create(48000, 960, &err);
    if (!m || err) return -1;
    init_caps(m, cap, LM, C);
    ec_dec_init(&dec, (unsigned char *)buf, len);
    int coded = clt_compute_allocation(m, start, end, offsets, cap, alloc_trim, &intensity, &dual_stereo, total,
                                       &balance, pulses, ebits, fine_priority, C, LM, &dec, 0, 0, 0);
    int k = 0;
    out[k++] = coded;
    out[k++] = intensity;
    out[k++] = dual_stereo;
    out[k++] = balance;
    for (int i = 0; i < 21; i++) out[k++] = pulses[i];
    for (int i = 0; i < 21; i++) out[k++] = ebits[i];
    for (int i = 0; i < 21; i++) out[k++] = fine_priority[i];
    out[k++] = (int32_t)ec_tell_frac(&dec);
    out[k++] = (int32_t)dec.rng;
    return 0;
}

#include "bands.h"

/* Allocation then celt/bands.c quant_all_bands in decode mode, on one range
 * decoder over buf (len bytes, the whole packet budget), as celt_decode_with_ec
 * runs them: X_out receives the C * (120 << LM) normalised coefficients,
 * cm_out the C * 21 collapse masks, tail the seed, tell_frac and rng. */
int oref_bands(const uint8_t *buf, uint32_t len, int start, int end, const int *offsets, int alloc_trim, int C,
               int LM, int shortBlocks, int spread, const int *tf_res, int disable_inv, uint32_t seed,
               int16_t *X_out, uint8_t *cm_out, uint32_t *tail)
{
    int err = 0, cap[21], pulses[21] = {0}, ebits[21] = {0}, fine_priority[21] = {0}, intensity = 0,
        dual_stereo = 0;
    opus_int32 balance = 0;
    celt_norm X[2 * 960];
    unsigned char masks[2 * 21];
    ec_dec dec;
    const CELTMode *m = opus_custom_mode_create(48000, 960, &err);
    if (!m || err) return -1;
    int N = 120 << LM;
    memset(X, 0, sizeof X);
    memset(masks, 0, sizeof masks);
    init_caps(m, cap, LM, C);
    ec_dec_init(&dec, (unsigned char *)buf, len);
    opus_int32 bits = (opus_int32)(len * 8 << 3) - (opus_int32)ec_tell_frac(&dec) - 1;
    int coded = clt_compute_allocation(m, start, end, offsets, cap, alloc_trim, &intensity, &dual_stereo, bits,
                                       &balance, pulses, ebits, fine_priority, C, LM, &dec, 0, 0, 0);
    opus_uint32 s = seed;
    quant_all_bands(0, m, start, end, X, C == 2 ? X + N : NULL, masks, NULL, pulses, shortBlocks, spread,
                    dual_stereo, intensity, (int *)tf_res, (opus_int32)(len * (8 << 3)), balance, &dec, LM, coded,
                    &s, 0, 0, disable_inv);
    memcpy(X_out, X, sizeof(int16_t) * C * N);
    memcpy(cm_out, masks, (size_t)C * 21);
    tail[0] = s;
    tail[1] = ec_tell_frac(&dec);
    tail[2] = dec.rng;
    return 0;
}

#include "quant_bands.h"

/* The band energies of one frame as celt_decode_with_ec decodes them around
 * the allocation: celt/quant_bands.c unquant_coarse_energy, then
 * clt_compute_allocation, unquant_fine_energy and unquant_energy_finalise with
 * the bits left.  oldE (2 x 21, Q8 log energies) is updated in place; tail
 * receives tell_frac and rng. */
int oref_energy(const uint8_t *buf, uint32_t len, int start, int end, int intra, const int *offsets,
                int alloc_trim, int C, int LM, int16_t *oldE, uint32_t *tail)
{
    int err = 0, cap[21], pulses[21] = {0}, ebits[21] = {0}, fine_priority[21] = {0}, intensity = 0,
        dual_stereo = 0;
    opus_int32 balance = 0;
    ec_dec dec;
    const CELTMode *m = opus_custom_mode_create(48000, 960, &err);
    if (!m || err) return -1;
    ec_dec_init(&dec, (unsigned char *)buf, len);
    unquant_coarse_energy(m, start, end, oldE, intra, &dec, C, LM);
    init_caps(m, cap, LM, C);
    opus_int32 bits = (opus_int32)(len * 8 << 3) - (opus_int32)ec_tell_frac(&dec) - 1;
    clt_compute_allocation(m, start, end, offsets, cap, alloc_trim, &intensity, &dual_stereo, bits, &balance,
                           pulses, ebits, fine_priority, C, LM, &dec, 0, 0, 0);
    unquant_fine_energy(m, start, end, oldE, ebits, &dec, C);
    unquant_energy_finalise(m, start, end, oldE, ebits, fine_priority, (int)len * 8 - ec_tell(&dec), &dec, C);
    tail[0] = ec_tell_frac(&dec);
    tail[1] = dec.rng;
    return 0;
}

#include "main.h"

/* SILK entropy decoding of `frames` frames of one channel (silk/decode_indices.c,
 * decode_pulses.c) at fs_kHz with nb_subfr subframes, from a fresh decoder
 * state: vad[f] is each frame's VAD flag, the first frame coded independently
 * (cond_first = 0) or not.  Per frame out receives 33 index words (signalType,
 * quantOffsetType, GainsIndices[4], LTPIndex[4], NLSFIndices[17], lagIndex,
 * contourIndex, NLSFInterpCoef_Q2, PERIndex, LTP_scaleIndex, Seed) and then
 * frame_length pulses; tail receives tell and rng.  Returns words written. */
int oref_silk_entropy(const uint8_t *buf, uint32_t len, int fs_kHz, int nb_subfr, int frames, const int *vad,
                      int cond_first, int32_t *out, uint32_t *tail)
{
    silk_decoder_state S;
    ec_dec dec;
    opus_int16 pulses[MAX_FRAME_LENGTH + SHELL_CODEC_FRAME_LENGTH];
    silk_init_decoder(&S);
    S.nb_subfr = nb_subfr;
    silk_decoder_set_fs(&S, fs_kHz, 48000);
    ec_dec_init(&dec, (unsigned char *)buf, len);
    int k = 0;
    for (int f = 0; f < frames; f++) {
        S.VAD_flags[f] = vad[f];
        silk_decode_indices(&S, &dec, f, 0, f == 0 ? (cond_first ? CODE_CONDITIONALLY : CODE_INDEPENDENTLY)
                                                    : CODE_CONDITIONALLY);
        silk_decode_pulses(&dec, pulses, S.indices.signalType, S.indices.quantOffsetType, S.frame_length);
        const SideInfoIndices *ix = &S.indices;
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
        for (int i = 0; i < S.frame_length; i++) out[k++] = pulses[i];
    }
    tail[0] = (uint32_t)ec_tell(&dec);
    tail[1] = dec.rng;
    return k;
}

/* SILK frames at the internal rate (silk/decode_frame.c: indices, pulses,
 * parameters, excitation, LTP / LPC synthesis, PLC and CNG) of one channel,
 * one frame per packet, the decoder state carried from frame to frame, all
 * bits from one range decoder: lost[f] conceals frame f, vad[f] is its VAD
 * flag.  out receives the frames back to back; tail tell and rng.  Returns
 * samples written. */
int oref_silk_frames(const uint8_t *buf, uint32_t len, int fs_kHz, int nb_subfr, int frames, const int *vad,
                     const int *lost, int16_t *out, uint32_t *tail)
{
    silk_decoder_state S;
    ec_dec dec;
    silk_init_decoder(&S);
    S.nb_subfr = nb_subfr;
    S.nFramesPerPacket = 1;
    silk_decoder_set_fs(&S, fs_kHz, 48000);
    ec_dec_init(&dec, (unsigned char *)buf, len);
    int o = 0;
    for (int f = 0; f < frames; f++) {
        opus_int32 n = 0;
        S.nFramesDecoded = 0;
        S.VAD_flags[0] = vad[f];
        silk_decode_frame(&S, &dec, out + o, &n, lost[f], f == 0 ? CODE_INDEPENDENTLY : CODE_CONDITIONALLY, 0);
        o += n;
    }
    tail[0] = (uint32_t)ec_tell(&dec);
    tail[1] = dec.rng;
    return o;
}

/* CELT frames (celt/celt_decoder.c celt_decode_with_ec: energies, allocation,
 * band shapes, anti-collapse, synthesis, post-filter, deemphasis, and the
 * concealment for lost frames) of one stream from a fresh 48 kHz decoder with
 * signalling off and end band `end`: frame f is lens[f] bytes of data (0 =
 * lost), 120 << LM samples per channel into out; rng[f] receives the final
 * range, or the error code when the decode fails.  Returns 0. */
int oref_celt_frames(const uint8_t *data, const uint32_t *lens, int frames, int C, int LM, int end, int16_t *out,
                     uint32_t *rng)
{
    CELTDecoder *st = (CELTDecoder *)malloc((size_t)celt_decoder_get_size(C));
    if (!st) return -1;
    celt_decoder_init(st, 48000, C);
    opus_custom_decoder_ctl(st, CELT_SET_SIGNALLING(0));
    opus_custom_decoder_ctl(st, CELT_SET_END_BAND(end));
    int N = 120 << LM;
    size_t off = 0;
    for (int f = 0; f < frames; f++) {
        int ret = celt_decode_with_ec(st, lens[f] ? data + off : NULL, (int)lens[f], out + (size_t)f * N * C, N,
                                      NULL, 0);
        opus_uint32 r = 0;
        opus_custom_decoder_ctl(st, OPUS_GET_FINAL_RANGE(&r));
        rng[f] = ret < 0 ? (uint32_t)ret : r;
        off += lens[f];
    }
    free(st);
    return 0;
}

/* Fixed-point helpers evaluated elementwise over arrays, for the decoder's
 * restatements of them: op 0 isqrt32, 1 celt_rcp, 2 frac_div32(a, b),
 * 3 celt_rsqrt_norm, 4 celt_sqrt, 5 celt_cos_norm, 6 celt_exp2 (celt/mathops.c,
 * celt/mathops.h), 7 bitexact_cos, 8 bitexact_log2tan(a, b) (celt/bands.c:68-90),
 * 9 silk_SQRT_APPROX, 10 silk_DIV32_varQ(a, b, q), 11 silk_INVERSE32_varQ(a, q)
 * (silk/Inlines.h:71-166), 12 silk_log2lin (silk/log2lin.c), 13 silk_lin2log
 * (silk/lin2log.c).  Returns -1 for an unknown op. */
#include "mathops.h"
int oref_mathops(int op, const int32_t *a, const int32_t *b, const int32_t *q, int n, int32_t *out)
{
    for (int i = 0; i < n; i++) {
        int32_t r;
        switch (op) {
        case 0: r = (int32_t)isqrt32((opus_uint32)a[i]); break;
        case 1: r = celt_rcp(a[i]); break;
        case 2: r = frac_div32(a[i], b[i]); break;
        case 3: r = celt_rsqrt_norm(a[i]); break;
        case 4: r = celt_sqrt(a[i]); break;
        case 5: r = celt_cos_norm(a[i]); break;
        case 6: r = celt_exp2((opus_val16)a[i]); break;
        case 7: r = bitexact_cos((opus_int16)a[i]); break;
        case 8: r = bitexact_log2tan(a[i], b[i]); break;
        case 9: r = silk_SQRT_APPROX(a[i]); break;
        case 10: r = silk_DIV32_varQ(a[i], b[i], q[i]); break;
        case 11: r = silk_INVERSE32_varQ(a[i], q[i]); break;
        case 12: r = silk_log2lin(a[i]); break;
        case 13: r = silk_lin2log(a[i]); break;
        default: return -1;
        }
        out[i] = r;
    }
    return 0;
}
