// CELT decoder (RFC 6716 section 4.3), fixed point, static 48 kHz / 960 mode.
//
// Restates libopus 1.5.2:
//   celt/celt_decoder.c   celt_decode_with_ec_dred, celt_decode_lost,
//                         prefilter_and_fold, celt_plc_pitch_search,
//                         tf_decode, celt_synthesis, deemphasis, reset
//   celt/quant_bands.c    unquant_coarse/fine_energy, unquant_energy_finalise
//   celt/rate.c           clt_compute_allocation, interp_bits2pulses
//   celt/rate.h           get_pulses, bits2pulses, pulses2bits
//   celt/bands.c          quant_all_bands (decode), quant_band(_stereo),
//                         quant_partition, compute_theta, anti_collapse,
//                         denormalise_bands, haar1, (de)interleave_hadamard,
//                         stereo_merge, special_hybrid_folding
//   celt/vq.c             alg_unquant, exp_rotation, renormalise_vector
//   celt/cwrs.c           cwrsi / decode_pulses (non-SMALL_FOOTPRINT)
//   celt/celt.c           comb_filter, init_caps
//   celt/mdct.c           clt_mdct_backward_c
//   celt/kiss_fft.c       opus_fft_impl, kf_bfly2/3/4/5
//   celt/pitch.c          pitch_downsample, pitch_search
//   celt/celt_lpc.c       _celt_lpc, celt_fir, celt_iir, _celt_autocorr
// The recursive band split (quant_partition) is unrolled at compile time by
// template depth (LM + 1 <= 4), so no device stack recursion is needed.
// Independent loops (IMDCT twiddles, FFT butterflies of one stage, band
// denormalisation, windowing, copies) are split over the chain's lanes.
#pragma once
#include "rangedec.cuh"

namespace cuo {

enum { CELT_NB = 21, CELT_OVERLAP = 120, CELT_DEC_BUF = 2048, CELT_LPC_ORDER = 24, CELT_MAX_PERIOD = 1024 };
enum { SPREAD_NONE = 0, SPREAD_LIGHT = 1, SPREAD_NORMAL = 2, SPREAD_AGGRESSIVE = 3 };
static const int CELT_SIG_SAT = 300000000;

struct CeltDec {
    int32_t channels, stream_channels, start, end, disable_inv;
    // reset region (DECODER_RESET_START = rng)
    uint32_t rng;
    int32_t error, last_pitch_index, loss_duration, skip_plc;
    int32_t postfilter_period, postfilter_period_old;
    int32_t postfilter_gain, postfilter_gain_old;
    int32_t postfilter_tapset, postfilter_tapset_old;
    int32_t prefilter_and_fold;
    int32_t preemph_memD[2];
    int32_t decode_mem[2][CELT_DEC_BUF + CELT_OVERLAP];
    int16_t lpc[2][CELT_LPC_ORDER];
    int16_t oldBandE[2 * CELT_NB], oldLogE[2 * CELT_NB], oldLogE2[2 * CELT_NB], backgroundLogE[2 * CELT_NB];
};

// One frame of quant_partition's explicit stack (the state of one split level).
struct QPFrame {
    int16_t *X, *Y, *lowband, *next_lowband2;
    int N, b, B, B0, LM, fill, mbits, sbits, itheta, stage;
    int32_t rebalance;
    int16_t gain, mid, side;
    unsigned cm;
};

// Per lane group, in the decoder slot.  Besides the frame buffers it holds
// what would otherwise be function-local arrays of the serial stages: every
// lane of a group computes the same values, so one copy per group serves all
// of them (a per-lane stack copy would multiply the memory these stages touch
// by the group width).
struct CeltScratch {
    QPFrame qp[5];                    // quant_partition's split stack
    int32_t bits1[CELT_NB], bits2[CELT_NB], thresh[CELT_NB], trim_offset[CELT_NB];   // allocation
    int16_t X[2 * 960];
    int32_t freq[960];
    int16_t norm[2 * 8 * 78];
    int16_t tmp[176];                 // (de)interleave staging
    int32_t iy[176];                  // PVQ pulses of one partition
    int32_t tf_res[CELT_NB], cap[CELT_NB], offsets[CELT_NB], fine_quant[CELT_NB], pulses[CELT_NB],
        fine_priority[CELT_NB];
    uint8_t collapse_masks[2 * CELT_NB];
    // PLC
    int16_t lp_pitch_buf[CELT_DEC_BUF >> 1];
    int16_t exc[CELT_MAX_PERIOD + CELT_LPC_ORDER];
    int16_t fir_tmp[CELT_MAX_PERIOD];
    int16_t x_lp4[(CELT_DEC_BUF - 720) >> 2];          // len >> 2, len = DEC_BUF - PLC_PITCH_LAG_MAX
    int16_t y_lp4[(CELT_DEC_BUF - 720 + 620) >> 2];    // (len + max_pitch) >> 2
    int32_t xcorr[CELT_MAX_PERIOD >> 1];
    int16_t ac_xx[CELT_MAX_PERIOD];
    int16_t iir_y[CELT_MAX_PERIOD + CELT_OVERLAP + CELT_LPC_ORDER];
    int32_t etmp[CELT_OVERLAP];
};

// ------------------------------------------------------------------ init / reset

DNI void celt_reset(CeltDec *st)
{
    st->rng = 0;
    st->error = 0;
    st->last_pitch_index = 0;
    st->loss_duration = 0;
    st->skip_plc = 0;
    st->postfilter_period = st->postfilter_period_old = 0;
    st->postfilter_gain = st->postfilter_gain_old = 0;
    st->postfilter_tapset = st->postfilter_tapset_old = 0;
    st->prefilter_and_fold = 0;
    st->preemph_memD[0] = st->preemph_memD[1] = 0;
    memset(st->decode_mem, 0, sizeof(st->decode_mem));
    memset(st->lpc, 0, sizeof(st->lpc));
    memset(st->oldBandE, 0, sizeof(st->oldBandE));
    memset(st->backgroundLogE, 0, sizeof(st->backgroundLogE));
    for (int i = 0; i < 2 * CELT_NB; i++) st->oldLogE[i] = st->oldLogE2[i] = -28672;   // -QCONST16(28.f, DB_SHIFT)
    st->skip_plc = 1;
}

// celt_decoder_init + CELT_SET_SIGNALLING(0) as done by opus_decoder_init
DFN void celt_init(CeltDec *st, int channels)
{
    st->channels = st->stream_channels = channels;
    st->start = 0;
    st->end = T_CELT_EFFEBANDS;
    st->disable_inv = channels == 1;
    celt_reset(st);
}

// ------------------------------------------------------------------ FFT / IMDCT

struct Cpx { int32_t r, i; };

DFN Cpx cmul(Cpx a, int16_t br, int16_t bi)
{
    Cpx m;
    m.r = wsub(c_mul16_32_q15(br, a.r), c_mul16_32_q15(bi, a.i));
    m.i = wadd(c_mul16_32_q15(bi, a.r), c_mul16_32_q15(br, a.i));
    return m;
}

// One radix-p stage of opus_fft_impl: N groups of m butterflies, group stride mm.
// Every butterfly touches its own p outputs, so the N*m of them are spread over lanes.
DNI void fft_stage(Lanes L, Cpx *F, int p, int fstride, int m, int N, int mm)
{
    const int16_t *tw = T_fft_twiddles;
    if (p == 2) {
        // kf_bfly2 (m == 4 in the static mode)
        const int16_t k = 23170;   // QCONST16(0.7071067812, 15)
        LFOR(L, i, 0, N) {
            Cpx *Fo = F + 8 * i, *F2 = Fo + 4, t;
            t = F2[0];
            F2[0].r = wsub(Fo[0].r, t.r); F2[0].i = wsub(Fo[0].i, t.i);
            Fo[0].r = wadd(Fo[0].r, t.r); Fo[0].i = wadd(Fo[0].i, t.i);
            t.r = c_mul16_32_q15(k, wadd(F2[1].r, F2[1].i));
            t.i = c_mul16_32_q15(k, wsub(F2[1].i, F2[1].r));
            F2[1].r = wsub(Fo[1].r, t.r); F2[1].i = wsub(Fo[1].i, t.i);
            Fo[1].r = wadd(Fo[1].r, t.r); Fo[1].i = wadd(Fo[1].i, t.i);
            t.r = F2[2].i; t.i = -F2[2].r;
            F2[2].r = wsub(Fo[2].r, t.r); F2[2].i = wsub(Fo[2].i, t.i);
            Fo[2].r = wadd(Fo[2].r, t.r); Fo[2].i = wadd(Fo[2].i, t.i);
            t.r = c_mul16_32_q15(k, wsub(F2[3].i, F2[3].r));
            t.i = c_mul16_32_q15(k, (int32_t)(0u - (uint32_t)wadd(F2[3].i, F2[3].r)));
            F2[3].r = wsub(Fo[3].r, t.r); F2[3].i = wsub(Fo[3].i, t.i);
            Fo[3].r = wadd(Fo[3].r, t.r); Fo[3].i = wadd(Fo[3].i, t.i);
        }
    } else if (p == 4) {
        if (m == 1) {
            LFOR(L, i, 0, N) {
                Cpx *Fo = F + 4 * i, s0, s1;
                s0.r = wsub(Fo[0].r, Fo[2].r); s0.i = wsub(Fo[0].i, Fo[2].i);
                Fo[0].r = wadd(Fo[0].r, Fo[2].r); Fo[0].i = wadd(Fo[0].i, Fo[2].i);
                s1.r = wadd(Fo[1].r, Fo[3].r); s1.i = wadd(Fo[1].i, Fo[3].i);
                Fo[2].r = wsub(Fo[0].r, s1.r); Fo[2].i = wsub(Fo[0].i, s1.i);
                Fo[0].r = wadd(Fo[0].r, s1.r); Fo[0].i = wadd(Fo[0].i, s1.i);
                s1.r = wsub(Fo[1].r, Fo[3].r); s1.i = wsub(Fo[1].i, Fo[3].i);
                Fo[1].r = wadd(s0.r, s1.i); Fo[1].i = wsub(s0.i, s1.r);
                Fo[3].r = wsub(s0.r, s1.i); Fo[3].i = wadd(s0.i, s1.r);
            }
        } else {
            LFOR(L, q, 0, N * m) {
                int i = q / m, j = q - i * m;
                Cpx *Fo = F + i * mm + j, s[6];
                s[0] = cmul(Fo[m], tw[2 * (j * fstride)], tw[2 * (j * fstride) + 1]);
                s[1] = cmul(Fo[2 * m], tw[2 * (2 * j * fstride)], tw[2 * (2 * j * fstride) + 1]);
                s[2] = cmul(Fo[3 * m], tw[2 * (3 * j * fstride)], tw[2 * (3 * j * fstride) + 1]);
                s[5].r = wsub(Fo[0].r, s[1].r); s[5].i = wsub(Fo[0].i, s[1].i);
                Fo[0].r = wadd(Fo[0].r, s[1].r); Fo[0].i = wadd(Fo[0].i, s[1].i);
                s[3].r = wadd(s[0].r, s[2].r); s[3].i = wadd(s[0].i, s[2].i);
                s[4].r = wsub(s[0].r, s[2].r); s[4].i = wsub(s[0].i, s[2].i);
                Fo[2 * m].r = wsub(Fo[0].r, s[3].r); Fo[2 * m].i = wsub(Fo[0].i, s[3].i);
                Fo[0].r = wadd(Fo[0].r, s[3].r); Fo[0].i = wadd(Fo[0].i, s[3].i);
                Fo[m].r = wadd(s[5].r, s[4].i); Fo[m].i = wsub(s[5].i, s[4].r);
                Fo[3 * m].r = wsub(s[5].r, s[4].i); Fo[3 * m].i = wadd(s[5].i, s[4].r);
            }
        }
    } else if (p == 3) {
        const int16_t epi3i = -28378;
        LFOR(L, q, 0, N * m) {
            int i = q / m, j = q - i * m;
            Cpx *Fo = F + i * mm + j, s[4];
            s[1] = cmul(Fo[m], tw[2 * (j * fstride)], tw[2 * (j * fstride) + 1]);
            s[2] = cmul(Fo[2 * m], tw[2 * (2 * j * fstride)], tw[2 * (2 * j * fstride) + 1]);
            s[3].r = wadd(s[1].r, s[2].r); s[3].i = wadd(s[1].i, s[2].i);
            s[0].r = wsub(s[1].r, s[2].r); s[0].i = wsub(s[1].i, s[2].i);
            Fo[m].r = wsub(Fo[0].r, s[3].r >> 1);
            Fo[m].i = wsub(Fo[0].i, s[3].i >> 1);
            s[0].r = c_mul16_32_q15(epi3i, s[0].r);
            s[0].i = c_mul16_32_q15(epi3i, s[0].i);
            Fo[0].r = wadd(Fo[0].r, s[3].r); Fo[0].i = wadd(Fo[0].i, s[3].i);
            Fo[2 * m].r = wadd(Fo[m].r, s[0].i);
            Fo[2 * m].i = wsub(Fo[m].i, s[0].r);
            Fo[m].r = wsub(Fo[m].r, s[0].i);
            Fo[m].i = wadd(Fo[m].i, s[0].r);
        }
    } else {
        // kf_bfly5
        const int16_t yar = 10126, yai = -31164, ybr = -26510, ybi = -19261;
        LFOR(L, q, 0, N * m) {
            int i = q / m, u = q - i * m;
            Cpx *F0 = F + i * mm + u, *F1 = F0 + m, *F2 = F0 + 2 * m, *F3 = F0 + 3 * m, *F4 = F0 + 4 * m;
            Cpx s[13];
            s[0] = *F0;
            s[1] = cmul(*F1, tw[2 * (u * fstride)], tw[2 * (u * fstride) + 1]);
            s[2] = cmul(*F2, tw[2 * (2 * u * fstride)], tw[2 * (2 * u * fstride) + 1]);
            s[3] = cmul(*F3, tw[2 * (3 * u * fstride)], tw[2 * (3 * u * fstride) + 1]);
            s[4] = cmul(*F4, tw[2 * (4 * u * fstride)], tw[2 * (4 * u * fstride) + 1]);
            s[7].r = wadd(s[1].r, s[4].r); s[7].i = wadd(s[1].i, s[4].i);
            s[10].r = wsub(s[1].r, s[4].r); s[10].i = wsub(s[1].i, s[4].i);
            s[8].r = wadd(s[2].r, s[3].r); s[8].i = wadd(s[2].i, s[3].i);
            s[9].r = wsub(s[2].r, s[3].r); s[9].i = wsub(s[2].i, s[3].i);
            F0->r = wadd(F0->r, wadd(s[7].r, s[8].r));
            F0->i = wadd(F0->i, wadd(s[7].i, s[8].i));
            s[5].r = wadd(s[0].r, wadd(c_mul16_32_q15(yar, s[7].r), c_mul16_32_q15(ybr, s[8].r)));
            s[5].i = wadd(s[0].i, wadd(c_mul16_32_q15(yar, s[7].i), c_mul16_32_q15(ybr, s[8].i)));
            s[6].r = wadd(c_mul16_32_q15(yai, s[10].i), c_mul16_32_q15(ybi, s[9].i));
            s[6].i = (int32_t)(0u - (uint32_t)wadd(c_mul16_32_q15(yai, s[10].r), c_mul16_32_q15(ybi, s[9].r)));
            F1->r = wsub(s[5].r, s[6].r); F1->i = wsub(s[5].i, s[6].i);
            F4->r = wadd(s[5].r, s[6].r); F4->i = wadd(s[5].i, s[6].i);
            s[11].r = wadd(s[0].r, wadd(c_mul16_32_q15(ybr, s[7].r), c_mul16_32_q15(yar, s[8].r)));
            s[11].i = wadd(s[0].i, wadd(c_mul16_32_q15(ybr, s[7].i), c_mul16_32_q15(yar, s[8].i)));
            s[12].r = wsub(c_mul16_32_q15(yai, s[9].i), c_mul16_32_q15(ybi, s[10].i));
            s[12].i = wsub(c_mul16_32_q15(ybi, s[10].r), c_mul16_32_q15(yai, s[9].r));
            F2->r = wadd(s[11].r, s[12].r); F2->i = wadd(s[11].i, s[12].i);
            F3->r = wsub(s[11].r, s[12].r); F3->i = wsub(s[11].i, s[12].i);
        }
    }
    lsync(L);
}

DNI void celt_fft(Lanes L, int shift_idx, Cpx *fout)
{
    const int16_t *factors;
    int sh;
    switch (shift_idx) {
    case 0: factors = T_fft0_factors; sh = T_FFT0_SHIFT; break;
    case 1: factors = T_fft1_factors; sh = T_FFT1_SHIFT; break;
    case 2: factors = T_fft2_factors; sh = T_FFT2_SHIFT; break;
    default: factors = T_fft3_factors; sh = T_FFT3_SHIFT; break;
    }
    int shift = sh > 0 ? sh : 0;
    int fstride[8];
    fstride[0] = 1;
    int Lf = 0, p, m;
    do {
        p = factors[2 * Lf];
        m = factors[2 * Lf + 1];
        fstride[Lf + 1] = fstride[Lf] * p;
        Lf++;
    } while (m != 1);
    m = factors[2 * Lf - 1];
    for (int i = Lf - 1; i >= 0; i--) {
        int m2 = i != 0 ? factors[2 * i - 1] : 1;
        fft_stage(L, fout, factors[2 * i], fstride[i] << shift, m, fstride[i], m2);
        m = m2;
    }
}

DFN const int16_t *fft_bitrev(int shift)
{
    return shift == 0 ? T_fft0_bitrev : shift == 1 ? T_fft1_bitrev : shift == 2 ? T_fft2_bitrev : T_fft3_bitrev;
}

// celt/mdct.c clt_mdct_backward_c
DNI void mdct_backward(Lanes L, const int32_t *in, int32_t *out, int shift, int stride)
{
    int N = T_CELT_MDCT_N;
    const int16_t *trig = T_celt_mdct_trig;
    for (int i = 0; i < shift; i++) { N >>= 1; trig += N; }
    int N2 = N >> 1, N4 = N >> 2;
    const int16_t *bitrev = fft_bitrev(shift);
    int32_t *yp = out + (CELT_OVERLAP >> 1);
    LFOR(L, i, 0, N4) {
        int rev = bitrev[i];
        int32_t x1 = in[2 * i * stride], x2 = in[stride * (N2 - 1) - 2 * i * stride];
        int32_t yr = wadd(c_mul16_32_q15(trig[i], x2), c_mul16_32_q15(trig[N4 + i], x1));
        int32_t yi = wsub(c_mul16_32_q15(trig[i], x1), c_mul16_32_q15(trig[N4 + i], x2));
        yp[2 * rev + 1] = yr;
        yp[2 * rev] = yi;
    }
    lsync(L);
    celt_fft(L, shift, (Cpx *)yp);
    LFOR(L, i, 0, (N4 + 1) >> 1) {
        int32_t *yp0 = yp + 2 * i, *yp1 = yp + N2 - 2 - 2 * i;
        int32_t re = yp0[1], im = yp0[0];
        int16_t t0 = trig[i], t1 = trig[N4 + i];
        int32_t yr = wadd(c_mul16_32_q15(t0, re), c_mul16_32_q15(t1, im));
        int32_t yi = wsub(c_mul16_32_q15(t1, re), c_mul16_32_q15(t0, im));
        re = yp1[1];
        im = yp1[0];
        yp0[0] = yr;
        yp1[1] = yi;
        t0 = trig[N4 - i - 1];
        t1 = trig[N2 - i - 1];
        yr = wadd(c_mul16_32_q15(t0, re), c_mul16_32_q15(t1, im));
        yi = wsub(c_mul16_32_q15(t1, re), c_mul16_32_q15(t0, im));
        yp1[0] = yr;
        yp0[1] = yi;
    }
    lsync(L);
    const int16_t *w = T_celt_window;
    LFOR(L, i, 0, CELT_OVERLAP / 2) {
        int32_t *xp1 = out + CELT_OVERLAP - 1 - i, *yp1 = out + i;
        int32_t x1 = *xp1, x2 = *yp1;
        int16_t w1 = w[i], w2 = w[CELT_OVERLAP - 1 - i];
        *yp1 = wsub(c_mul16_32_q15(w2, x2), c_mul16_32_q15(w1, x1));
        *xp1 = wadd(c_mul16_32_q15(w1, x2), c_mul16_32_q15(w2, x1));
    }
    lsync(L);
}

// ------------------------------------------------------------------ synthesis helpers

// celt/bands.c denormalise_bands (downsample 1)
DNI void denormalise_bands(Lanes L, const int16_t *X, int32_t *freq, const int16_t *bandLogE, int start,
                           int end, int M, int silence)
{
    const int16_t *eB = T_celt_eBands;
    int N = M * T_CELT_SHORTMDCT;
    int bound = M * eB[end];
    if (silence) { bound = 0; start = end = 0; }
    LFOR(L, i, 0, M * eB[start]) freq[i] = 0;
    for (int b = start; b < end; b++) {
        int j0 = M * eB[b], j1 = M * eB[b + 1];
        int16_t lg = c_sat16(wadd(bandLogE[b], shl32((int32_t)T_celt_eMeans[b], 6)));
        int shift = 16 - (lg >> 10);
        int16_t g;
        if (shift > 31) { shift = 0; g = 0; }
        else g = (int16_t)c_exp2_frac((int16_t)(lg & 1023));
        if (shift < 0) {
            if (shift <= -2) { g = 16384; shift = -2; }
            LFOR(L, j, j0, j1) freq[j] = shl32(c_mul16(X[j], g), -shift);
        } else {
            LFOR(L, j, j0, j1) freq[j] = c_mul16(X[j], g) >> shift;
        }
    }
    LFOR(L, i, bound, N) freq[i] = 0;
    lsync(L);
}

// celt/celt.c comb_filter (in place when y == x): the IIR recursion over lag T
// is kept serial.
// gains[3][3] of celt/celt.c (comb filter taps per tapset)
TABC(int16_t, T_comb_gains[3][3]) = {{10048, 7112, 4248}, {15200, 8784, 0}, {26208, 3280, 0}};

DNI void comb_filter(int32_t *y, int32_t *x, int T0, int T1, int N, int16_t g0, int16_t g1, int tapset0,
                     int tapset1, const int16_t *window, int overlap)
{
    const int16_t (*gains)[3] = T_comb_gains;
    if (g0 == 0 && g1 == 0) {
        if (x != y) for (int i = 0; i < N; i++) y[i] = x[i];
        return;
    }
    T0 = imax(T0, 15);
    T1 = imax(T1, 15);
    int16_t g00 = (int16_t)c_mul16_p15(g0, gains[tapset0][0]);
    int16_t g01 = (int16_t)c_mul16_p15(g0, gains[tapset0][1]);
    int16_t g02 = (int16_t)c_mul16_p15(g0, gains[tapset0][2]);
    int16_t g10 = (int16_t)c_mul16_p15(g1, gains[tapset1][0]);
    int16_t g11 = (int16_t)c_mul16_p15(g1, gains[tapset1][1]);
    int16_t g12 = (int16_t)c_mul16_p15(g1, gains[tapset1][2]);
    int32_t x0, x1 = x[-T1 + 1], x2 = x[-T1], x3 = x[-T1 - 1], x4 = x[-T1 - 2];
    if (g0 == g1 && T0 == T1 && tapset0 == tapset1) overlap = 0;
    int i;
    for (i = 0; i < overlap; i++) {
        x0 = x[i - T1 + 2];
        int16_t f = (int16_t)c_mul16_q15(window[i], window[i]);
        int32_t v = x[i];
        v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(32767 - f, g00), x[i - T0]));
        v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(32767 - f, g01), wadd(x[i - T0 + 1], x[i - T0 - 1])));
        v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(32767 - f, g02), wadd(x[i - T0 + 2], x[i - T0 - 2])));
        v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(f, g10), x2));
        v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(f, g11), wadd(x1, x3)));
        v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(f, g12), wadd(x0, x4)));
        y[i] = c_sat(v, CELT_SIG_SAT);
        x4 = x3; x3 = x2; x2 = x1; x1 = x0;
    }
    if (g1 == 0) {
        if (x != y) for (int k = overlap; k < N; k++) y[k] = x[k];
        return;
    }
    // comb_filter_const_c
    int32_t *yy = y + i, *xx = x + i;
    int Nc = N - i;
    x4 = xx[-T1 - 2]; x3 = xx[-T1 - 1]; x2 = xx[-T1]; x1 = xx[-T1 + 1];
    for (int k = 0; k < Nc; k++) {
        x0 = xx[k - T1 + 2];
        int32_t v = wadd(wadd(wadd(xx[k], c_mul16_32_q15(g10, x2)), c_mul16_32_q15(g11, wadd(x1, x3))),
                         c_mul16_32_q15(g12, wadd(x0, x4)));
        yy[k] = c_sat(v, CELT_SIG_SAT);
        x4 = x3; x3 = x2; x2 = x1; x1 = x0;
    }
}

// comb_filter split across the lanes.  In place (y == x) output i reads the
// input at i and outputs at i - T - 2 .. i - T + 2 (T >= 15), so a block of
// min(T0, T1) - 2 consecutive outputs depends only on earlier blocks: the
// blocks run in order with a barrier between them and the outputs of a block
// in parallel, each with the serial code's exact arithmetic.  Out of place
// every output depends on the input only and one block covers the frame.
DNI void comb_filter_lanes(Lanes L, int32_t *y, int32_t *x, int T0, int T1, int N, int16_t g0, int16_t g1,
                           int tapset0, int tapset1, const int16_t *window, int overlap)
{
    const int16_t (*gains)[3] = T_comb_gains;
    lsync(L);
    if (g0 == 0 && g1 == 0) {
        if (x != y) {
            LFOR(L, i, 0, N) y[i] = x[i];
            lsync(L);
        }
        return;
    }
    T0 = imax(T0, 15);
    T1 = imax(T1, 15);
    int16_t g00 = (int16_t)c_mul16_p15(g0, gains[tapset0][0]);
    int16_t g01 = (int16_t)c_mul16_p15(g0, gains[tapset0][1]);
    int16_t g02 = (int16_t)c_mul16_p15(g0, gains[tapset0][2]);
    int16_t g10 = (int16_t)c_mul16_p15(g1, gains[tapset1][0]);
    int16_t g11 = (int16_t)c_mul16_p15(g1, gains[tapset1][1]);
    int16_t g12 = (int16_t)c_mul16_p15(g1, gains[tapset1][2]);
    if (g0 == g1 && T0 == T1 && tapset0 == tapset1) overlap = 0;
    const int B = x == y ? imin(T0, T1) - 2 : imax(N, 1);
    for (int s = 0; s < overlap; s += B) {
        int e = imin(s + B, overlap);
        LFOR(L, i, s, e) {
            int16_t f = (int16_t)c_mul16_q15(window[i], window[i]);
            int32_t v = x[i];
            v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(32767 - f, g00), x[i - T0]));
            v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(32767 - f, g01), wadd(x[i - T0 + 1], x[i - T0 - 1])));
            v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(32767 - f, g02), wadd(x[i - T0 + 2], x[i - T0 - 2])));
            v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(f, g10), x[i - T1]));
            v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(f, g11), wadd(x[i - T1 + 1], x[i - T1 - 1])));
            v = wadd(v, c_mul16_32_q15((int16_t)c_mul16_q15(f, g12), wadd(x[i - T1 + 2], x[i - T1 - 2])));
            y[i] = c_sat(v, CELT_SIG_SAT);
        }
        lsync(L);
    }
    if (g1 == 0) {
        if (x != y) {
            LFOR(L, k, overlap, N) y[k] = x[k];
            lsync(L);
        }
        return;
    }
    for (int s = overlap; s < N; s += B) {
        int e = imin(s + B, N);
        LFOR(L, k, s, e) {
            int32_t v = wadd(wadd(wadd(x[k], c_mul16_32_q15(g10, x[k - T1])),
                                  c_mul16_32_q15(g11, wadd(x[k - T1 + 1], x[k - T1 - 1]))),
                             c_mul16_32_q15(g12, wadd(x[k - T1 + 2], x[k - T1 - 2])));
            y[k] = c_sat(v, CELT_SIG_SAT);
        }
        lsync(L);
    }
}

// celt/celt_decoder.c deemphasis (downsample 1): one-pole recursion, serial
DNI void deemphasis(Lanes L, int32_t *in0, int32_t *in1, int16_t *pcm, int N, int C, int32_t *mem,
                    int accum)
{
    const int16_t coef0 = T_CELT_PREEMPH0;
    // The channels are independent recursions: with two or more lanes, lane c
    // runs channel c, so a stereo frame's two recursions execute side by side
    // in the same instructions; a single lane runs them one after the other.
    lsync(L);
    int c0 = 0, c1 = C;
    if (L.n > 1) {
        c0 = L.id;
        c1 = L.id < C ? L.id + 1 : L.id;
    }
    for (int c = c0; c < c1; c++) {
        const int32_t *x = c == 0 ? in0 : in1;
        int16_t *y = pcm + c;
        int32_t m = mem[c];
        if (accum) {
            for (int j = 0; j < N; j++) {
                int32_t tmp = wadd(x[j], m);
                m = c_mul16_32_q15(coef0, tmp);
                y[j * C] = c_sat16((int32_t)y[j * C] + c_sig2word16(tmp));
            }
        } else {
            for (int j = 0; j < N; j++) {
                int32_t tmp = wadd(x[j], m);
                m = c_mul16_32_q15(coef0, tmp);
                y[j * C] = c_sig2word16(tmp);
            }
        }
        mem[c] = m;
    }
    lsync(L);
}

// celt/celt_decoder.c celt_synthesis (downsample 1)
DNI void celt_synthesis(Lanes L, CeltScratch *w, const int16_t *X, int32_t **out_syn,
                        const int16_t *oldBandE, int start, int effEnd, int C, int CC, int isTransient, int LM,
                        int silence)
{
    int M = 1 << LM;
    int N = T_CELT_SHORTMDCT << LM;
    int B, NB, shift;
    if (isTransient) { B = M; NB = T_CELT_SHORTMDCT; shift = T_CELT_MAXLM; }
    else { B = 1; NB = T_CELT_SHORTMDCT << LM; shift = T_CELT_MAXLM - LM; }
    int32_t *freq = w->freq;
    if (CC == 2 && C == 1) {
        denormalise_bands(L, X, freq, oldBandE, start, effEnd, M, silence);
        int32_t *freq2 = out_syn[1] + CELT_OVERLAP / 2;
        LFOR(L, i, 0, N) freq2[i] = freq[i];
        lsync(L);
        for (int b = 0; b < B; b++) mdct_backward(L, &freq2[b], out_syn[0] + NB * b, shift, B);
        for (int b = 0; b < B; b++) mdct_backward(L, &freq[b], out_syn[1] + NB * b, shift, B);
    } else if (CC == 1 && C == 2) {
        int32_t *freq2 = out_syn[0] + CELT_OVERLAP / 2;
        denormalise_bands(L, X, freq, oldBandE, start, effEnd, M, silence);
        denormalise_bands(L, X + N, freq2, oldBandE + CELT_NB, start, effEnd, M, silence);
        LFOR(L, i, 0, N) freq[i] = wadd(freq[i] >> 1, freq2[i] >> 1);
        lsync(L);
        for (int b = 0; b < B; b++) mdct_backward(L, &freq[b], out_syn[0] + NB * b, shift, B);
    } else {
        for (int c = 0; c < CC; c++) {
            denormalise_bands(L, X + c * N, freq, oldBandE + c * CELT_NB, start, effEnd, M, silence);
            for (int b = 0; b < B; b++) mdct_backward(L, &freq[b], out_syn[c] + NB * b, shift, B);
        }
    }
    for (int c = 0; c < CC; c++) {
        int32_t *o = out_syn[c];
        LFOR(L, i, 0, N) o[i] = c_sat(o[i], CELT_SIG_SAT);
    }
    lsync(L);
}

// ------------------------------------------------------------------ energy

DNI void unquant_coarse_energy(int start, int end, int16_t *oldEBands, int intra, RangeDec *dec, int C, int LM)
{
    const uint8_t *prob = &T_celt_e_prob_model[(LM * 2 + intra) * 42];
    int32_t prev[2] = {0, 0};
    int16_t coef, beta;
    if (intra) { coef = 0; beta = T_CELT_BETA_INTRA; }
    else { beta = T_celt_beta_coef[LM]; coef = T_celt_pred_coef[LM]; }
    int32_t budget = dec->storage * 8;
    for (int i = start; i < end; i++) {
        for (int c = 0; c < C; c++) {
            int qi;
            int32_t tell = rd_tell(dec);
            if (budget - tell >= 15) {
                int pi = 2 * imin(i, 20);
                qi = rd_laplace(dec, prob[pi] << 7, prob[pi + 1] << 6);
            } else if (budget - tell >= 2) {
                qi = rd_icdf(dec, T_celt_small_energy_icdf, 2);
                qi = (qi >> 1) ^ -(qi & 1);
            } else if (budget - tell >= 1) {
                qi = -rd_bit_logp(dec, 1);
            } else {
                qi = -1;
            }
            int32_t q = shl32(qi, 10);
            int16_t *e = &oldEBands[i + c * CELT_NB];
            *e = (int16_t)max32(-9216, *e);   // -QCONST16(9, DB_SHIFT)
            int32_t tmp = wadd(wadd(c_pshr(c_mul16(coef, *e), 8), prev[c]), shl32(q, 7));
            tmp = max32(-3670016, tmp);       // -QCONST32(28, DB_SHIFT + 7)
            *e = (int16_t)c_pshr(tmp, 7);
            prev[c] = wsub(wadd(prev[c], shl32(q, 7)), c_mul16(beta, c_pshr(q, 8)));
        }
    }
}

DNI void unquant_fine_energy(int start, int end, int16_t *oldEBands, const int32_t *fine_quant, RangeDec *dec,
                             int C)
{
    for (int i = start; i < end; i++) {
        if (fine_quant[i] <= 0) continue;
        for (int c = 0; c < C; c++) {
            int q2 = (int)rd_bits(dec, fine_quant[i]);
            int16_t offset = (int16_t)(((shl32(q2, 10) + 512) >> fine_quant[i]) - 512);
            oldEBands[i + c * CELT_NB] = (int16_t)(oldEBands[i + c * CELT_NB] + offset);
        }
    }
}

DNI void unquant_energy_finalise(int start, int end, int16_t *oldEBands, const int32_t *fine_quant,
                                 const int32_t *fine_priority, int bits_left, RangeDec *dec, int C)
{
    for (int prio = 0; prio < 2; prio++) {
        for (int i = start; i < end && bits_left >= C; i++) {
            if (fine_quant[i] >= 8 || fine_priority[i] != prio) continue;
            for (int c = 0; c < C; c++) {
                int q2 = (int)rd_bits(dec, 1);
                int16_t offset = (int16_t)((int16_t)((uint16_t)q2 << 10) - 512) >> (fine_quant[i] + 1);
                oldEBands[i + c * CELT_NB] = (int16_t)(oldEBands[i + c * CELT_NB] + offset);
                bits_left--;
            }
        }
    }
}

// ------------------------------------------------------------------ allocation

DFN int get_pulses(int i) { return i < 8 ? i : (8 + (i & 7)) << ((i >> 3) - 1); }

DFN const uint8_t *pulse_cache(int band, int LM)
{
    return T_celt_cache_bits + T_celt_cache_index[(LM + 1) * CELT_NB + band];
}

DFN int bits2pulses(int band, int LM, int bits)
{
    const uint8_t *cache = pulse_cache(band, LM);
    int lo = 0, hi = cache[0];
    bits--;
    for (int i = 0; i < 6; i++) {
        int mid = (lo + hi + 1) >> 1;
        if ((int)cache[mid] >= bits) hi = mid;
        else lo = mid;
    }
    if (bits - (lo == 0 ? -1 : (int)cache[lo]) <= (int)cache[hi] - bits) return lo;
    return hi;
}

DFN int pulses2bits(int band, int LM, int pulses)
{
    const uint8_t *cache = pulse_cache(band, LM);
    return pulses == 0 ? 0 : cache[pulses] + 1;
}

DFN void init_caps(int32_t *cap, int LM, int C)
{
    for (int i = 0; i < CELT_NB; i++) {
        int N = (T_celt_eBands[i + 1] - T_celt_eBands[i]) << LM;
        cap[i] = (T_celt_cache_caps[CELT_NB * (2 * LM + C - 1) + i] + 64) * C * N >> 2;
    }
}

DNI int interp_bits2pulses(int start, int end, int skip_start, const int32_t *bits1, const int32_t *bits2,
                           const int32_t *thresh, const int32_t *cap, int32_t total, int32_t *_balance,
                           int skip_rsv, int *intensity, int intensity_rsv, int *dual_stereo,
                           int dual_stereo_rsv, int32_t *bits, int32_t *ebits, int32_t *fine_priority, int C,
                           int LM, RangeDec *ec)
{
    const int16_t *eB = T_celt_eBands;
    int alloc_floor = C << 3;
    int stereo = C > 1;
    int logM = LM << 3;
    int lo = 0, hi = 1 << 6;
    int32_t psum;
    int done;
    for (int i = 0; i < 6; i++) {
        int mid = (lo + hi) >> 1;
        psum = 0;
        done = 0;
        for (int j = end; j-- > start;) {
            int tmp = bits1[j] + (mid * (int32_t)bits2[j] >> 6);
            if (tmp >= thresh[j] || done) {
                done = 1;
                psum += imin(tmp, cap[j]);
            } else if (tmp >= alloc_floor) {
                psum += alloc_floor;
            }
        }
        if (psum > total) hi = mid;
        else lo = mid;
    }
    psum = 0;
    done = 0;
    for (int j = end; j-- > start;) {
        int tmp = bits1[j] + ((int32_t)lo * bits2[j] >> 6);
        if (tmp < thresh[j] && !done) {
            if (tmp >= alloc_floor) tmp = alloc_floor;
            else tmp = 0;
        } else {
            done = 1;
        }
        tmp = imin(tmp, cap[j]);
        bits[j] = tmp;
        psum += tmp;
    }
    int codedBands;
    for (codedBands = end;; codedBands--) {
        int j = codedBands - 1;
        if (j <= skip_start) {
            total += skip_rsv;
            break;
        }
        int32_t left = total - psum;
        int32_t percoeff = (int32_t)((uint32_t)left / (uint32_t)(eB[codedBands] - eB[start]));
        left -= (eB[codedBands] - eB[start]) * percoeff;
        int rem = imax(left - (eB[j] - eB[start]), 0);
        int band_width = eB[codedBands] - eB[j];
        int band_bits = (int)(bits[j] + percoeff * band_width + rem);
        if (band_bits >= imax(thresh[j], alloc_floor + (1 << 3))) {
            if (rd_bit_logp(ec, 1)) break;
            psum += 1 << 3;
            band_bits -= 1 << 3;
        }
        psum -= bits[j] + intensity_rsv;
        if (intensity_rsv > 0) intensity_rsv = T_celt_log2_frac_table[j - start];
        psum += intensity_rsv;
        if (band_bits >= alloc_floor) {
            psum += alloc_floor;
            bits[j] = alloc_floor;
        } else {
            bits[j] = 0;
        }
    }
    if (intensity_rsv > 0) *intensity = start + (int)rd_uint(ec, codedBands + 1 - start);
    else *intensity = 0;
    if (*intensity <= start) {
        total += dual_stereo_rsv;
        dual_stereo_rsv = 0;
    }
    if (dual_stereo_rsv > 0) *dual_stereo = rd_bit_logp(ec, 1);
    else *dual_stereo = 0;
    int32_t left = total - psum;
    int32_t percoeff = (int32_t)((uint32_t)left / (uint32_t)(eB[codedBands] - eB[start]));
    left -= (eB[codedBands] - eB[start]) * percoeff;
    for (int j = start; j < codedBands; j++) bits[j] += (int)percoeff * (eB[j + 1] - eB[j]);
    for (int j = start; j < codedBands; j++) {
        int tmp = (int)imin(left, eB[j + 1] - eB[j]);
        bits[j] += tmp;
        left -= tmp;
    }
    int32_t balance = 0;
    int j;
    for (j = start; j < codedBands; j++) {
        int N0 = eB[j + 1] - eB[j];
        int N = N0 << LM;
        int32_t bit = (int32_t)bits[j] + balance;
        int32_t excess;
        if (N > 1) {
            excess = max32(bit - cap[j], 0);
            bits[j] = bit - excess;
            int den = C * N + ((C == 2 && N > 2 && !*dual_stereo && j < *intensity) ? 1 : 0);
            int NClogN = den * (T_celt_logN[j] + logM);
            int offset = (NClogN >> 1) - den * 21;   // FINE_OFFSET
            if (N == 2) offset += den << 3 >> 2;
            if (bits[j] + offset < den * 2 << 3) offset += NClogN >> 2;
            else if (bits[j] + offset < den * 3 << 3) offset += NClogN >> 3;
            ebits[j] = imax(0, bits[j] + offset + (den << 2));
            ebits[j] = (int32_t)((uint32_t)ebits[j] / (uint32_t)den) >> 3;
            if (C * ebits[j] > (bits[j] >> 3)) ebits[j] = bits[j] >> stereo >> 3;
            ebits[j] = imin(ebits[j], 8);
            fine_priority[j] = ebits[j] * (den << 3) >= bits[j] + offset;
            bits[j] -= C * ebits[j] << 3;
        } else {
            excess = max32(0, bit - (C << 3));
            bits[j] = bit - excess;
            ebits[j] = 0;
            fine_priority[j] = 1;
        }
        if (excess > 0) {
            int extra_fine = imin(excess >> (stereo + 3), 8 - ebits[j]);
            ebits[j] += extra_fine;
            int extra_bits = extra_fine * C << 3;
            fine_priority[j] = extra_bits >= excess - balance;
            excess -= extra_bits;
        }
        balance = excess;
    }
    *_balance = balance;
    for (; j < end; j++) {
        ebits[j] = bits[j] >> stereo >> 3;
        bits[j] = 0;
        fine_priority[j] = ebits[j] < 1;
    }
    return codedBands;
}

DNI int clt_compute_allocation(int start, int end, const int32_t *offsets, const int32_t *cap, int alloc_trim,
                               int *intensity, int *dual_stereo, int32_t total, int32_t *balance, int32_t *pulses,
                               int32_t *ebits, int32_t *fine_priority, int C, int LM, RangeDec *ec, CeltScratch *w)
{
    const int16_t *eB = T_celt_eBands;
    int32_t *bits1 = w->bits1, *bits2 = w->bits2, *thresh = w->thresh, *trim_offset = w->trim_offset;
    total = max32(total, 0);
    int skip_start = start;
    int skip_rsv = total >= 1 << 3 ? 1 << 3 : 0;
    total -= skip_rsv;
    int intensity_rsv = 0, dual_stereo_rsv = 0;
    if (C == 2) {
        intensity_rsv = T_celt_log2_frac_table[end - start];
        if (intensity_rsv > total) {
            intensity_rsv = 0;
        } else {
            total -= intensity_rsv;
            dual_stereo_rsv = total >= 1 << 3 ? 1 << 3 : 0;
            total -= dual_stereo_rsv;
        }
    }
    for (int j = start; j < end; j++) {
        thresh[j] = imax(C << 3, (3 * (eB[j + 1] - eB[j]) << LM << 3) >> 4);
        trim_offset[j] = C * (eB[j + 1] - eB[j]) * (alloc_trim - 5 - LM) * (end - j - 1) * (1 << (LM + 3)) >> 6;
        if ((eB[j + 1] - eB[j]) << LM == 1) trim_offset[j] -= C << 3;
    }
    int lo = 1, hi = T_CELT_NBALLOCV - 1;
    do {
        int done = 0, psum = 0;
        int mid = (lo + hi) >> 1;
        for (int j = end; j-- > start;) {
            int N = eB[j + 1] - eB[j];
            int bitsj = C * N * T_celt_allocVectors[mid * CELT_NB + j] << LM >> 2;
            if (bitsj > 0) bitsj = imax(0, bitsj + trim_offset[j]);
            bitsj += offsets[j];
            if (bitsj >= thresh[j] || done) {
                done = 1;
                psum += imin(bitsj, cap[j]);
            } else if (bitsj >= C << 3) {
                psum += C << 3;
            }
        }
        if (psum > total) hi = mid - 1;
        else lo = mid + 1;
    } while (lo <= hi);
    hi = lo--;
    for (int j = start; j < end; j++) {
        int N = eB[j + 1] - eB[j];
        int bits1j = C * N * T_celt_allocVectors[lo * CELT_NB + j] << LM >> 2;
        int bits2j = hi >= T_CELT_NBALLOCV ? cap[j] : C * N * T_celt_allocVectors[hi * CELT_NB + j] << LM >> 2;
        if (bits1j > 0) bits1j = imax(0, bits1j + trim_offset[j]);
        if (bits2j > 0) bits2j = imax(0, bits2j + trim_offset[j]);
        if (lo > 0) bits1j += offsets[j];
        bits2j += offsets[j];
        if (offsets[j] > 0) skip_start = j;
        bits2j = imax(0, bits2j - bits1j);
        bits1[j] = bits1j;
        bits2[j] = bits2j;
    }
    return interp_bits2pulses(start, end, skip_start, bits1, bits2, thresh, cap, total, balance, skip_rsv,
                              intensity, intensity_rsv, dual_stereo, dual_stereo_rsv, pulses, ebits,
                              fine_priority, C, LM, ec);
}

// ------------------------------------------------------------------ PVQ

DFN uint32_t pvq_u(int n, int k)
{
    int a = imin(n, k), b = imax(n, k);
    return T_celt_pvq_u_data[T_celt_pvq_u_row[a] + b];
}
DFN uint32_t pvq_v(int n, int k) { return pvq_u(n, k) + pvq_u(n, k + 1); }
DFN uint32_t pvq_row(int r, int c) { return T_celt_pvq_u_data[T_celt_pvq_u_row[r] + c]; }

// celt/cwrs.c cwrsi: combinatorial index -> pulse vector; returns sum of squares
DNI int32_t cwrsi(int n, int k, uint32_t idx, int32_t *y)
{
    uint32_t p;
    int s, k0;
    int16_t val;
    int32_t yy = 0;
    while (n > 2) {
        uint32_t q;
        if (k >= n) {
            p = pvq_row(n, k + 1);
            s = -(idx >= p);
            idx -= p & s;
            k0 = k;
            q = pvq_row(n, n);
            if (q > idx) {
                k = n;
                do p = pvq_row(--k, n);
                while (p > idx);
            } else {
                for (p = pvq_row(n, k); p > idx; p = pvq_row(n, k)) k--;
            }
            idx -= p;
            val = (int16_t)((k0 - k + s) ^ s);
            *y++ = val;
            yy = c_mac16(yy, val, val);
        } else {
            p = pvq_row(k, n);
            q = pvq_row(k + 1, n);
            if (p <= idx && idx < q) {
                idx -= p;
                *y++ = 0;
            } else {
                s = -(idx >= q);
                idx -= q & s;
                k0 = k;
                do p = pvq_row(--k, n);
                while (p > idx);
                idx -= p;
                val = (int16_t)((k0 - k + s) ^ s);
                *y++ = val;
                yy = c_mac16(yy, val, val);
            }
        }
        n--;
    }
    p = 2 * k + 1;
    s = -(idx >= p);
    idx -= p & s;
    k0 = k;
    k = (idx + 1) >> 1;
    if (k) idx -= 2 * k - 1;
    val = (int16_t)((k0 - k + s) ^ s);
    *y++ = val;
    yy = c_mac16(yy, val, val);
    s = -(int)idx;
    val = (int16_t)((k + s) ^ s);
    *y = val;
    yy = c_mac16(yy, val, val);
    return yy;
}

// celt/vq.c exp_rotation1.  Each pass rotates the pairs (X[i], X[i + stride])
// in order, and pair i + stride reads the element pair i has just written:
// the pass is `stride` independent recurrences, one per residue class of i
// mod stride.  Here each class runs on its own with the element it carries
// into the next pair kept in a register rather than stored and loaded back
// (a store-then-load round trip per step); every element gets the same
// arithmetic as in the serial pass.
DNI void exp_rotation1(int16_t *X, int len, int stride, int16_t c, int16_t s)
{
    const int16_t ms = (int16_t)-s;
    // forward: i = 0 .. len - stride - 1
    for (int j = 0; j < stride && j < len - stride; j++) {
        int16_t x1 = X[j];
        int i = j;
        for (; i < len - stride; i += stride) {
            int16_t x2 = X[i + stride];
            X[i] = (int16_t)c_pshr(c_mac16(c_mul16(c, x1), ms, x2), 15);
            x1 = (int16_t)c_pshr(c_mac16(c_mul16(c, x2), s, x1), 15);   // the new X[i + stride]
        }
        X[i] = x1;
    }
    // backward: i = len - 2 stride - 1 .. 0; pair i - stride reads the X[i]
    // pair i has written
    const int top = len - 2 * stride - 1;
    for (int j = 0; j < stride && top - j >= 0; j++) {
        int i = top - j;
        int16_t x2 = X[i + stride];
        for (; i >= 0; i -= stride) {
            int16_t x1 = X[i];
            X[i + stride] = (int16_t)c_pshr(c_mac16(c_mul16(c, x2), s, x1), 15);
            x2 = (int16_t)c_pshr(c_mac16(c_mul16(c, x1), ms, x2), 15);   // the new X[i]
        }
        X[i + stride] = x2;
    }
}

// celt/vq.c exp_rotation, dir = -1 (decoder)
DNI void exp_rotation_dec(int16_t *X, int len, int stride, int K, int spread)
{
    if (2 * K >= len || spread == SPREAD_NONE) return;
    int factor = spread == 1 ? 15 : spread == 2 ? 10 : 5;   // SPREAD_FACTOR[spread - 1] = {15, 10, 5}
    int16_t gain = (int16_t)c_mul32_q31(c_mul16(32767, len), c_rcp(len + factor * K));
    int16_t theta = (int16_t)(c_mul16_q15(gain, gain) >> 1);
    int16_t c = c_cos_norm(theta);
    int16_t s = c_cos_norm((int16_t)(32767 - theta));
    int stride2 = 0;
    if (len >= 8 * stride) {
        stride2 = 1;
        while ((stride2 * stride2 + stride2) * stride + (stride >> 2) < len) stride2++;
    }
    len = (int)((unsigned)len / (unsigned)stride);
    for (int i = 0; i < stride; i++) {
        if (stride2) exp_rotation1(X + i * len, len, stride2, s, c);
        exp_rotation1(X + i * len, len, 1, c, s);
    }
}

// celt/vq.c renormalise_vector
// (the energy is a wrap-around sum, so the lanes' partial sums give the serial
// value; every element is scaled on its own)
DNI void renormalise_vector(Lanes L, int16_t *X, int N, int16_t gain)
{
    PHASE_BEGIN(t_rn);
    int32_t E = 0;
    LFOR(L, i, 0, N) E = c_mac16(E, X[i], X[i]);
    E = wadd(lsum(L, E), 1);
    int k = c_ilog2(E) >> 1;
    int32_t t = c_vshr(E, 2 * (k - 7));
    int16_t g = (int16_t)c_mul16_p15(c_rsqrt_norm(t), gain);
    LFOR(L, i, 0, N) X[i] = (int16_t)c_pshr(c_mul16(g, X[i]), k + 1);
    lsync(L);
    PHASE_END(PH_PVQ_RENORM, t_rn, L.id);
}

// celt/vq.c alg_unquant
DNI unsigned alg_unquant(Lanes L, int16_t *X, int N, int K, int spread, int B, RangeDec *dec, int16_t gain,
                         int32_t *iy)
{
    PHASE_BEGIN(t_cw);
    int32_t Ryy = cwrsi(N, K, rd_uint(dec, pvq_v(N, K)), iy);
    PHASE_END(PH_PVQ_CWRSI, t_cw, L.id);
    // normalise_residual (every element on its own)
    int k = c_ilog2(Ryy) >> 1;
    int32_t t = c_vshr(Ryy, 2 * (k - 7));
    int16_t g = (int16_t)c_mul16_p15(c_rsqrt_norm(t), gain);
    LFOR(L, i, 0, N) X[i] = (int16_t)c_pshr(c_mul16(g, iy[i]), k + 1);
    lsync(L);
    PHASE_BEGIN(t_rt);
    exp_rotation_dec(X, N, B, K, spread);
    PHASE_END(PH_PVQ_ROT, t_rt, L.id);
    // extract_collapse_mask
    if (B <= 1) return 1;
    int N0 = (int)((unsigned)N / (unsigned)B);
    unsigned mask = 0;
    for (int i = 0; i < B; i++) {
        unsigned tmp = 0;
        for (int j = 0; j < N0; j++) tmp |= iy[i * N0 + j];
        mask |= (tmp != 0) << i;
    }
    return mask;
}

// ------------------------------------------------------------------ bands

DFN int16_t bitexact_cos(int16_t x)
{
    int32_t tmp = (4096 + (int32_t)x * x) >> 13;
    int16_t x2 = (int16_t)tmp;
    x2 = (int16_t)((32767 - x2) + c_frac_mul16(x2, (-7651 + c_frac_mul16(x2, (8277 + c_frac_mul16(-626, x2))))));
    return (int16_t)(1 + x2);
}

DFN int bitexact_log2tan(int isin, int icos)
{
    int lc = ilog((uint32_t)icos), ls = ilog((uint32_t)isin);
    icos <<= 15 - lc;
    isin <<= 15 - ls;
    return (ls - lc) * (1 << 11) + c_frac_mul16(isin, c_frac_mul16(isin, -2597) + 7932) -
           c_frac_mul16(icos, c_frac_mul16(icos, -2597) + 7932);
}

DNI void haar1(int16_t *X, int N0, int stride)
{
    N0 >>= 1;
    for (int i = 0; i < stride; i++)
        for (int j = 0; j < N0; j++) {
            int32_t t1 = c_mul16(23170, X[stride * 2 * j + i]);
            int32_t t2 = c_mul16(23170, X[stride * (2 * j + 1) + i]);
            X[stride * 2 * j + i] = (int16_t)c_pshr(wadd(t1, t2), 15);
            X[stride * (2 * j + 1) + i] = (int16_t)c_pshr(wsub(t1, t2), 15);
        }
}

DNI void deinterleave_hadamard(int16_t *X, int N0, int stride, int hadamard, int16_t *tmp)
{
    int N = N0 * stride;
    if (hadamard) {
        const int32_t *ordery = T_celt_ordery_table + stride - 2;
        for (int i = 0; i < stride; i++)
            for (int j = 0; j < N0; j++) tmp[ordery[i] * N0 + j] = X[j * stride + i];
    } else {
        for (int i = 0; i < stride; i++)
            for (int j = 0; j < N0; j++) tmp[i * N0 + j] = X[j * stride + i];
    }
    for (int i = 0; i < N; i++) X[i] = tmp[i];
}

DNI void interleave_hadamard(int16_t *X, int N0, int stride, int hadamard, int16_t *tmp)
{
    int N = N0 * stride;
    if (hadamard) {
        const int32_t *ordery = T_celt_ordery_table + stride - 2;
        for (int i = 0; i < stride; i++)
            for (int j = 0; j < N0; j++) tmp[j * stride + i] = X[ordery[i] * N0 + j];
    } else {
        for (int i = 0; i < stride; i++)
            for (int j = 0; j < N0; j++) tmp[j * stride + i] = X[i * N0 + j];
    }
    for (int i = 0; i < N; i++) X[i] = tmp[i];
}

struct BandCtx {
    Lanes L;
    int i;
    int intensity;
    int spread;
    int tf_change;
    RangeDec *ec;
    int32_t remaining_bits;
    uint32_t seed;
    int disable_inv;
    int avoid_split_noise;
    CeltScratch *w;
};

struct SplitCtx {
    int inv, imid, iside, delta, itheta, qalloc;
};

// exp2_table8 of celt/bands.c compute_qn
TABC(int16_t, T_exp2_table8[8]) = {16384, 17866, 19483, 21247, 23170, 25267, 27554, 30048};

DFN int compute_qn(int N, int b, int offset, int pulse_cap, int stereo)
{
    const int16_t *exp2_table8 = T_exp2_table8;
    int N2 = 2 * N - 1;
    if (stereo && N == 2) N2--;
    int qb = (b + N2 * offset) / N2;
    qb = imin(b - pulse_cap - (4 << 3), qb);
    qb = imin(8 << 3, qb);
    int qn;
    if (qb < (1 << 3 >> 1)) {
        qn = 1;
    } else {
        qn = exp2_table8[qb & 0x7] >> (14 - (qb >> 3));
        qn = (qn + 1) >> 1 << 1;
    }
    return qn;
}

// celt/bands.c compute_theta (decoder side)
DNI void compute_theta(BandCtx *ctx, SplitCtx *sctx, int N, int *b, int B, int B0, int LM, int stereo, int *fill)
{
    int itheta = 0, delta, imid, iside, inv = 0;
    RangeDec *ec = ctx->ec;
    int i = ctx->i;
    int pulse_cap = T_celt_logN[i] + LM * (1 << 3);
    int offset = (pulse_cap >> 1) - (stereo && N == 2 ? 16 : 4);
    int qn = compute_qn(N, *b, offset, pulse_cap, stereo);
    if (stereo && i >= ctx->intensity) qn = 1;
    int32_t tell = (int32_t)rd_tell_frac(ec);
    if (qn != 1) {
        if (stereo && N > 2) {
            int p0 = 3, x0 = qn / 2, ft = p0 * (x0 + 1) + x0, x;
            int fs = (int)rd_decode(ec, ft);
            if (fs < (x0 + 1) * p0) x = fs / p0;
            else x = x0 + 1 + (fs - (x0 + 1) * p0);
            rd_update(ec, x <= x0 ? p0 * x : (x - 1 - x0) + (x0 + 1) * p0,
                      x <= x0 ? p0 * (x + 1) : (x - x0) + (x0 + 1) * p0, ft);
            itheta = x;
        } else if (B0 > 1 || stereo) {
            itheta = (int)rd_uint(ec, qn + 1);
        } else {
            int fs = 1, fl = 0, ft = ((qn >> 1) + 1) * ((qn >> 1) + 1);
            int fm = (int)rd_decode(ec, ft);
            if (fm < ((qn >> 1) * ((qn >> 1) + 1) >> 1)) {
                itheta = (int)(c_isqrt32(8 * (uint32_t)fm + 1) - 1) >> 1;
                fs = itheta + 1;
                fl = itheta * (itheta + 1) >> 1;
            } else {
                itheta = (2 * (qn + 1) - (int)c_isqrt32(8 * (uint32_t)(ft - fm - 1) + 1)) >> 1;
                fs = qn + 1 - itheta;
                fl = ft - ((qn + 1 - itheta) * (qn + 2 - itheta) >> 1);
            }
            rd_update(ec, fl, fl + fs, ft);
        }
        itheta = (int)((uint32_t)((int32_t)itheta * 16384) / (uint32_t)qn);
    } else if (stereo) {
        if (*b > 2 << 3 && ctx->remaining_bits > 2 << 3) inv = rd_bit_logp(ec, 2);
        else inv = 0;
        if (ctx->disable_inv) inv = 0;
        itheta = 0;
    }
    int qalloc = (int)rd_tell_frac(ec) - tell;
    *b -= qalloc;
    if (itheta == 0) {
        imid = 32767; iside = 0;
        *fill &= (1 << B) - 1;
        delta = -16384;
    } else if (itheta == 16384) {
        imid = 0; iside = 32767;
        *fill &= ((1 << B) - 1) << B;
        delta = 16384;
    } else {
        imid = bitexact_cos((int16_t)itheta);
        iside = bitexact_cos((int16_t)(16384 - itheta));
        delta = c_frac_mul16((N - 1) << 7, bitexact_log2tan(iside, imid));
    }
    sctx->inv = inv; sctx->imid = imid; sctx->iside = iside;
    sctx->delta = delta; sctx->itheta = itheta; sctx->qalloc = qalloc;
}

DNI unsigned quant_band_n1(BandCtx *ctx, int16_t *X, int16_t *Y, int16_t *lowband_out)
{
    int16_t *x = X;
    int stereo = Y != 0;
    for (int c = 0; c < 1 + stereo; c++) {
        int sign = 0;
        if (ctx->remaining_bits >= 1 << 3) {
            sign = (int)rd_bits(ctx->ec, 1);
            ctx->remaining_bits -= 1 << 3;
        }
        x[0] = sign ? -16384 : 16384;
        x = Y;
    }
    if (lowband_out) lowband_out[0] = (int16_t)(X[0] >> 4);
    return 1;
}

// celt/bands.c quant_partition, leaf: pulses for the band piece (PVQ) or,
// with none, folding / noise fill.
DNI unsigned quant_partition_leaf(BandCtx *ctx, int16_t *X, int N, int b, int B, int16_t *lowband, int LM,
                                  int16_t gain, int fill)
{
    const int i = ctx->i;
    unsigned cm = 0;
    int q = bits2pulses(i, LM, b);
    int curr_bits = pulses2bits(i, LM, q);
    ctx->remaining_bits -= curr_bits;
    while (ctx->remaining_bits < 0 && q > 0) {
        ctx->remaining_bits += curr_bits;
        q--;
        curr_bits = pulses2bits(i, LM, q);
        ctx->remaining_bits -= curr_bits;
    }
    if (q != 0) {
        int K = get_pulses(q);
        cm = alg_unquant(ctx->L, X, N, K, ctx->spread, B, ctx->ec, gain, ctx->w->iy);
    } else {
        unsigned cm_mask = (unsigned)(1UL << B) - 1;
        fill &= cm_mask;
        if (!fill) {
            for (int j = 0; j < N; j++) X[j] = 0;
        } else {
            if (lowband == 0) {
                for (int j = 0; j < N; j++) {
                    ctx->seed = c_lcg_rand(ctx->seed);
                    X[j] = (int16_t)((int32_t)ctx->seed >> 20);
                }
                cm = cm_mask;
            } else {
                for (int j = 0; j < N; j++) {
                    ctx->seed = c_lcg_rand(ctx->seed);
                    int16_t tmp = (ctx->seed & 0x8000) ? 4 : -4;   // QCONST16(1.0f/256, 10)
                    X[j] = (int16_t)(lowband[j] + tmp);
                }
                cm = fill;
            }
            renormalise_vector(ctx->L, X, N, gain);
        }
    }
    return cm;
}

// celt/bands.c quant_partition.  libopus recurses into the two halves of a
// split band; here one loop walks an explicit stack of frames instead, so a
// single copy of the code serves every depth (the split depth is bounded by
// LM + 1 <= 4, five frames).  A frame resumes after each half: stage 1 / 2
// when the mid half went first, 3 / 4 when the side half did; the bit
// rebalancing between the halves and the collapse-mask combination happen at
// those points, in libopus's order.
DNI unsigned quant_partition(BandCtx *ctx, int16_t *X, int N, int b, int B, int16_t *lowband, int LM,
                             int16_t gain, int fill)
{
    QPFrame *st = ctx->w->qp;
    int sp = 0;
    st[0].X = X;
    st[0].N = N;
    st[0].b = b;
    st[0].B = B;
    st[0].lowband = lowband;
    st[0].LM = LM;
    st[0].gain = gain;
    st[0].fill = fill;
    st[0].stage = 0;
    unsigned ret = 0;
    const int i = ctx->i;
    while (sp >= 0) {
        QPFrame *f = &st[sp];
        QPFrame *c = &st[sp + 1 < 5 ? sp + 1 : 4];
        if (f->stage == 0) {
            const uint8_t *cache = T_celt_cache_bits + T_celt_cache_index[(f->LM + 1) * CELT_NB + i];
            if (f->LM != -1 && f->b > cache[cache[0]] + 12 && f->N > 2 && sp < 4) {
                SplitCtx sctx;
                int B0 = f->B;
                int N2 = f->N >> 1;
                int fill2 = f->fill;
                if (f->B == 1) fill2 = (fill2 & 1) | (fill2 << 1);
                int B2 = (f->B + 1) >> 1;
                int LM2 = f->LM - 1;
                int b2 = f->b;
                PHASE_BEGIN(t_th);
                compute_theta(ctx, &sctx, N2, &b2, B2, B0, LM2, 0, &fill2);
                PHASE_END(PH_PVQ_THETA, t_th, ctx->L.id);
                int delta = sctx.delta, itheta = sctx.itheta;
                if (B0 > 1 && (itheta & 0x3fff)) {
                    if (itheta > 8192) delta -= delta >> (4 - LM2);
                    else delta = imin(0, delta + (N2 << 3 >> (5 - LM2)));
                }
                int mbits = imax(0, imin(b2, (b2 - delta) / 2));
                int sbits = b2 - mbits;
                ctx->remaining_bits -= sctx.qalloc;
                f->Y = f->X + N2;
                f->N = N2;
                f->B = B2;
                f->B0 = B0;
                f->LM = LM2;
                f->fill = fill2;
                f->mid = (int16_t)sctx.imid;
                f->side = (int16_t)sctx.iside;
                f->itheta = itheta;
                f->mbits = mbits;
                f->sbits = sbits;
                f->next_lowband2 = f->lowband ? f->lowband + N2 : 0;
                f->rebalance = ctx->remaining_bits;
                c->stage = 0;
                c->N = N2;
                c->B = B2;
                c->LM = LM2;
                if (mbits >= sbits) {
                    f->stage = 1;
                    c->X = f->X;
                    c->b = mbits;
                    c->lowband = f->lowband;
                    c->gain = (int16_t)c_mul16_p15(f->gain, f->mid);
                    c->fill = fill2;
                } else {
                    f->stage = 3;
                    c->X = f->Y;
                    c->b = sbits;
                    c->lowband = f->next_lowband2;
                    c->gain = (int16_t)c_mul16_p15(f->gain, f->side);
                    c->fill = fill2 >> B2;
                }
                sp++;
                continue;
            }
            ret = quant_partition_leaf(ctx, f->X, f->N, f->b, f->B, f->lowband, f->LM, f->gain, f->fill);
            sp--;
            continue;
        }
        if (f->stage == 1 || f->stage == 3) {
            c->stage = 0;
            c->N = f->N;
            c->B = f->B;
            c->LM = f->LM;
            if (f->stage == 1) {            // mid half done: rebalance, then the side half
                f->cm = ret;
                int32_t rebalance = f->mbits - (f->rebalance - ctx->remaining_bits);
                if (rebalance > 3 << 3 && f->itheta != 0) f->sbits += rebalance - (3 << 3);
                c->X = f->Y;
                c->b = f->sbits;
                c->lowband = f->next_lowband2;
                c->gain = (int16_t)c_mul16_p15(f->gain, f->side);
                c->fill = f->fill >> f->B;
                f->stage = 2;
            } else {                        // side half done: rebalance, then the mid half
                f->cm = ret << (f->B0 >> 1);
                int32_t rebalance = f->sbits - (f->rebalance - ctx->remaining_bits);
                if (rebalance > 3 << 3 && f->itheta != 16384) f->mbits += rebalance - (3 << 3);
                c->X = f->X;
                c->b = f->mbits;
                c->lowband = f->lowband;
                c->gain = (int16_t)c_mul16_p15(f->gain, f->mid);
                c->fill = f->fill;
                f->stage = 4;
            }
            sp++;
            continue;
        }
        ret = f->stage == 2 ? f->cm | (ret << (f->B0 >> 1)) : f->cm | ret;
        sp--;
    }
    return ret;
}

// bit_interleave_table / bit_deinterleave_table of celt/bands.c quant_band
TABC(uint8_t, T_bit_interleave[16]) = {0, 1, 1, 1, 2, 3, 3, 3, 2, 3, 3, 3, 2, 3, 3, 3};
TABC(uint8_t, T_bit_deinterleave[16]) = {0x00, 0x03, 0x0C, 0x0F, 0x30, 0x33, 0x3C, 0x3F,
                                         0xC0, 0xC3, 0xCC, 0xCF, 0xF0, 0xF3, 0xFC, 0xFF};

// celt/bands.c quant_band (decoder, resynth always on)
DNI unsigned quant_band(BandCtx *ctx, int16_t *X, int N, int b, int B, int16_t *lowband, int LM,
                        int16_t *lowband_out, int16_t gain, int16_t *lowband_scratch, int fill)
{
    const uint8_t *bit_interleave_table = T_bit_interleave;
    const uint8_t *bit_deinterleave_table = T_bit_deinterleave;
    int N0 = N, N_B = N, N_B0, B0 = B, time_divide = 0, recombine = 0;
    int longBlocks = B0 == 1;
    unsigned cm = 0;
    int tf_change = ctx->tf_change;
    N_B = (int)((unsigned)N_B / (unsigned)B);
    if (N == 1) return quant_band_n1(ctx, X, 0, lowband_out);
    if (tf_change > 0) recombine = tf_change;
    PHASE_BEGIN(t_tf);
    if (lowband_scratch && lowband && (recombine || ((N_B & 1) == 0 && tf_change < 0) || B0 > 1)) {
        for (int j = 0; j < N; j++) lowband_scratch[j] = lowband[j];
        lowband = lowband_scratch;
    }
    for (int k = 0; k < recombine; k++) {
        if (lowband) haar1(lowband, N >> k, 1 << k);
        fill = bit_interleave_table[fill & 0xF] | bit_interleave_table[fill >> 4] << 2;
    }
    B >>= recombine;
    N_B <<= recombine;
    while ((N_B & 1) == 0 && tf_change < 0) {
        if (lowband) haar1(lowband, N_B, B);
        fill |= fill << B;
        B <<= 1;
        N_B >>= 1;
        time_divide++;
        tf_change++;
    }
    B0 = B;
    N_B0 = N_B;
    if (B0 > 1 && lowband)
        deinterleave_hadamard(lowband, N_B >> recombine, B0 << recombine, longBlocks, ctx->w->tmp);
    PHASE_END(PH_PVQ_TF, t_tf, ctx->L.id);
    cm = quant_partition(ctx, X, N, b, B, lowband, LM, gain, fill);
    PHASE_BEGIN(t_tf2);
    if (B0 > 1) interleave_hadamard(X, N_B >> recombine, B0 << recombine, longBlocks, ctx->w->tmp);
    N_B = N_B0;
    B = B0;
    for (int k = 0; k < time_divide; k++) {
        B >>= 1;
        N_B <<= 1;
        cm |= cm >> B;
        haar1(X, N_B, B);
    }
    for (int k = 0; k < recombine; k++) {
        cm = bit_deinterleave_table[cm];
        haar1(X, N0 >> k, 1 << k);
    }
    PHASE_END(PH_PVQ_TF, t_tf2, ctx->L.id);
    B <<= recombine;
    if (lowband_out) {
        int16_t n = (int16_t)c_sqrt(shl32(N0, 22));
        for (int j = 0; j < N0; j++) lowband_out[j] = (int16_t)c_mul16_q15(n, X[j]);
    }
    cm &= (1 << B) - 1;
    return cm;
}

// (the two dot products are wrap-around sums, so the lanes' partial sums give
// the serial values; every element is mixed on its own)
DNI void stereo_merge(Lanes L, int16_t *X, int16_t *Y, int16_t mid, int N)
{
    int32_t xp = 0, side = 0;
    LFOR(L, j, 0, N) {
        xp = c_mac16(xp, Y[j], X[j]);
        side = c_mac16(side, Y[j], Y[j]);
    }
    xp = lsum(L, xp);
    side = lsum(L, side);
    xp = c_mul16_32_q15(mid, xp);
    int16_t mid2 = (int16_t)(mid >> 1);
    int32_t El = wsub(wadd(c_mul16(mid2, mid2), side), 2 * xp);
    int32_t Er = wadd(wadd(c_mul16(mid2, mid2), side), 2 * xp);
    if (Er < 161061 || El < 161061) {   // QCONST32(6e-4f, 28)
        LFOR(L, j, 0, N) Y[j] = X[j];
        lsync(L);
        return;
    }
    int kl = c_ilog2(El) >> 1, kr = c_ilog2(Er) >> 1;
    int32_t t = c_vshr(El, (kl - 7) << 1);
    int16_t lgain = c_rsqrt_norm(t);
    t = c_vshr(Er, (kr - 7) << 1);
    int16_t rgain = c_rsqrt_norm(t);
    if (kl < 7) kl = 7;
    if (kr < 7) kr = 7;
    LFOR(L, j, 0, N) {
        int16_t l = (int16_t)c_mul16_p15(mid, X[j]);
        int16_t r = Y[j];
        X[j] = (int16_t)c_pshr(c_mul16(lgain, (int16_t)(l - r)), kl + 1);
        Y[j] = (int16_t)c_pshr(c_mul16(rgain, (int16_t)(l + r)), kr + 1);
    }
    lsync(L);
}

DNI unsigned quant_band_stereo(BandCtx *ctx, int16_t *X, int16_t *Y, int N, int b, int B, int16_t *lowband,
                               int LM, int16_t *lowband_out, int16_t *lowband_scratch, int fill)
{
    unsigned cm = 0;
    SplitCtx sctx;
    if (N == 1) return quant_band_n1(ctx, X, Y, lowband_out);
    int orig_fill = fill;
    PHASE_BEGIN(t_th);
    compute_theta(ctx, &sctx, N, &b, B, B, LM, 1, &fill);
    PHASE_END(PH_PVQ_THETA, t_th, ctx->L.id);
    int inv = sctx.inv, delta = sctx.delta, itheta = sctx.itheta, qalloc = sctx.qalloc;
    int16_t mid = (int16_t)sctx.imid, side = (int16_t)sctx.iside;
    int mbits, sbits;
    if (N == 2) {
        int sign = 0;
        mbits = b;
        sbits = 0;
        if (itheta != 0 && itheta != 16384) sbits = 1 << 3;
        mbits -= sbits;
        int c = itheta > 8192;
        ctx->remaining_bits -= qalloc + sbits;
        int16_t *x2 = c ? Y : X, *y2 = c ? X : Y;
        if (sbits) sign = (int)rd_bits(ctx->ec, 1);
        sign = 1 - 2 * sign;
        cm = quant_band(ctx, x2, N, mbits, B, lowband, LM, lowband_out, 32767, lowband_scratch, orig_fill);
        y2[0] = (int16_t)(-sign * x2[1]);
        y2[1] = (int16_t)(sign * x2[0]);
        X[0] = (int16_t)c_mul16_q15(mid, X[0]);
        X[1] = (int16_t)c_mul16_q15(mid, X[1]);
        Y[0] = (int16_t)c_mul16_q15(side, Y[0]);
        Y[1] = (int16_t)c_mul16_q15(side, Y[1]);
        int16_t tmp = X[0];
        X[0] = (int16_t)(tmp - Y[0]);
        Y[0] = (int16_t)(tmp + Y[0]);
        tmp = X[1];
        X[1] = (int16_t)(tmp - Y[1]);
        Y[1] = (int16_t)(tmp + Y[1]);
    } else {
        mbits = imax(0, imin(b, (b - delta) / 2));
        sbits = b - mbits;
        ctx->remaining_bits -= qalloc;
        int32_t rebalance = ctx->remaining_bits;
        if (mbits >= sbits) {
            cm = quant_band(ctx, X, N, mbits, B, lowband, LM, lowband_out, 32767, lowband_scratch, fill);
            rebalance = mbits - (rebalance - ctx->remaining_bits);
            if (rebalance > 3 << 3 && itheta != 0) sbits += rebalance - (3 << 3);
            cm |= quant_band(ctx, Y, N, sbits, B, 0, LM, 0, side, 0, fill >> B);
        } else {
            cm = quant_band(ctx, Y, N, sbits, B, 0, LM, 0, side, 0, fill >> B);
            rebalance = sbits - (rebalance - ctx->remaining_bits);
            if (rebalance > 3 << 3 && itheta != 16384) mbits += rebalance - (3 << 3);
            cm |= quant_band(ctx, X, N, mbits, B, lowband, LM, lowband_out, 32767, lowband_scratch, fill);
        }
    }
    if (N != 2) stereo_merge(ctx->L, X, Y, mid, N);
    if (inv)
        for (int j = 0; j < N; j++) Y[j] = (int16_t)-Y[j];
    return cm;
}

// celt/bands.c quant_all_bands, decoder path (encode = 0, resynth = 1, no theta RDO)
DNI void quant_all_bands_dec(Lanes L, int start, int end, int16_t *X_, int16_t *Y_, uint8_t *collapse_masks,
                             const int32_t *pulses, int shortBlocks, int spread, int dual_stereo, int intensity,
                             const int32_t *tf_res, int32_t total_bits, int32_t balance, RangeDec *ec, int LM,
                             int codedBands, uint32_t *seed, int disable_inv, CeltScratch *w)
{
    const int16_t *eB = T_celt_eBands;
    int M = 1 << LM;
    int B = shortBlocks ? M : 1;
    int norm_offset = M * eB[start];
    int C = Y_ != 0 ? 2 : 1;
    int16_t *norm = w->norm;
    int16_t *norm2 = norm + M * eB[CELT_NB - 1] - norm_offset;
    int16_t *lowband_scratch = X_ + M * eB[T_CELT_EFFEBANDS - 1];
    int lowband_offset = 0, update_lowband = 1;
    BandCtx ctx;
    ctx.ec = ec;
    ctx.intensity = intensity;
    ctx.seed = *seed;
    ctx.spread = spread;
    ctx.disable_inv = disable_inv;
    ctx.avoid_split_noise = B > 1;
    ctx.w = w;
    ctx.L = L;
    for (int i = start; i < end; i++) {
        int effective_lowband = -1;
        unsigned x_cm, y_cm;
        ctx.i = i;
        int last = i == end - 1;
        int16_t *X = X_ + M * eB[i];
        int16_t *Y = Y_ != 0 ? Y_ + M * eB[i] : 0;
        int N = M * eB[i + 1] - M * eB[i];
        int32_t tell = (int32_t)rd_tell_frac(ec);
        if (i != start) balance -= tell;
        int32_t remaining_bits = total_bits - tell - 1;
        ctx.remaining_bits = remaining_bits;
        int b;
        if (i <= codedBands - 1) {
            int32_t curr_balance = balance / imin(3, codedBands - i);
            b = imax(0, imin(16383, imin(remaining_bits + 1, pulses[i] + curr_balance)));
        } else {
            b = 0;
        }
        if ((M * eB[i] - N >= M * eB[start] || i == start + 1) && (update_lowband || lowband_offset == 0))
            lowband_offset = i;
        if (i == start + 1) {
            // special_hybrid_folding
            int n1 = M * (eB[start + 1] - eB[start]);
            int n2 = M * (eB[start + 2] - eB[start + 1]);
            for (int j = 0; j < n2 - n1; j++) norm[n1 + j] = norm[2 * n1 - n2 + j];
            if (dual_stereo)
                for (int j = 0; j < n2 - n1; j++) norm2[n1 + j] = norm2[2 * n1 - n2 + j];
        }
        int tf_change = tf_res[i];
        ctx.tf_change = tf_change;
        if (i >= T_CELT_EFFEBANDS) {
            X = norm;
            if (Y_ != 0) Y = norm;
            lowband_scratch = 0;
        }
        if (last) lowband_scratch = 0;
        if (lowband_offset != 0 && (spread != SPREAD_AGGRESSIVE || B > 1 || tf_change < 0)) {
            effective_lowband = imax(0, M * eB[lowband_offset] - norm_offset - N);
            int fold_start = lowband_offset;
            while (M * eB[--fold_start] > effective_lowband + norm_offset) {}
            int fold_end = lowband_offset - 1;
            while (++fold_end < i && M * eB[fold_end] < effective_lowband + norm_offset + N) {}
            x_cm = y_cm = 0;
            int fold_i = fold_start;
            do {
                x_cm |= collapse_masks[fold_i * C + 0];
                y_cm |= collapse_masks[fold_i * C + C - 1];
            } while (++fold_i < fold_end);
        } else {
            x_cm = y_cm = (1 << B) - 1;
        }
        if (dual_stereo && i == intensity) {
            dual_stereo = 0;
            for (int j = 0; j < M * eB[i] - norm_offset; j++) norm[j] = (int16_t)((norm[j] + norm2[j]) >> 1);
        }
        if (dual_stereo) {
            x_cm = quant_band(&ctx, X, N, b / 2, B, effective_lowband != -1 ? norm + effective_lowband : 0, LM,
                              last ? 0 : norm + M * eB[i] - norm_offset, 32767, lowband_scratch, (int)x_cm);
            y_cm = quant_band(&ctx, Y, N, b / 2, B, effective_lowband != -1 ? norm2 + effective_lowband : 0, LM,
                              last ? 0 : norm2 + M * eB[i] - norm_offset, 32767, lowband_scratch, (int)y_cm);
        } else {
            if (Y != 0) {
                x_cm = quant_band_stereo(&ctx, X, Y, N, b, B,
                                         effective_lowband != -1 ? norm + effective_lowband : 0, LM,
                                         last ? 0 : norm + M * eB[i] - norm_offset, lowband_scratch,
                                         (int)(x_cm | y_cm));
            } else {
                x_cm = quant_band(&ctx, X, N, b, B, effective_lowband != -1 ? norm + effective_lowband : 0, LM,
                                  last ? 0 : norm + M * eB[i] - norm_offset, 32767, lowband_scratch,
                                  (int)(x_cm | y_cm));
            }
            y_cm = x_cm;
        }
        collapse_masks[i * C + 0] = (uint8_t)x_cm;
        collapse_masks[i * C + C - 1] = (uint8_t)y_cm;
        balance += pulses[i] + tell;
        update_lowband = b > (N << 3);
        ctx.avoid_split_noise = 0;
    }
    *seed = ctx.seed;
    lsync(L);
}

// celt/bands.c anti_collapse
DNI void anti_collapse(Lanes L, int16_t *X_, const uint8_t *collapse_masks, int LM, int C, int size, int start,
                       int end,
                       const int16_t *logE, const int16_t *prev1logE, const int16_t *prev2logE,
                       const int32_t *pulses, uint32_t seed)
{
    const int16_t *eB = T_celt_eBands;
    for (int i = start; i < end; i++) {
        int N0 = eB[i + 1] - eB[i];
        int depth = (int)((uint32_t)(1 + pulses[i]) / (uint32_t)N0) >> LM;
        int32_t thresh32 = c_exp2((int16_t)-(int16_t)((uint16_t)depth << 7)) >> 1;
        int16_t thresh = (int16_t)c_mul16_32_q15(16384, min32(32767, thresh32));
        int32_t t = N0 << LM;
        int shift = c_ilog2(t) >> 1;
        t = shl32(t, (7 - shift) << 1);
        int16_t sqrt_1 = c_rsqrt_norm(t);
        for (int c = 0; c < C; c++) {
            int renormalize = 0;
            int16_t prev1 = prev1logE[c * CELT_NB + i], prev2 = prev2logE[c * CELT_NB + i];
            if (C == 1) {
                prev1 = prev1 > prev1logE[CELT_NB + i] ? prev1 : prev1logE[CELT_NB + i];
                prev2 = prev2 > prev2logE[CELT_NB + i] ? prev2 : prev2logE[CELT_NB + i];
            }
            int32_t Ediff = (int32_t)logE[c * CELT_NB + i] - (int32_t)(prev1 < prev2 ? prev1 : prev2);
            Ediff = max32(0, Ediff);
            int16_t r;
            if (Ediff < 16384) {
                int32_t r32 = c_exp2((int16_t)-(int16_t)Ediff) >> 1;
                r = (int16_t)(2 * (r32 < 16383 ? r32 : 16383));
            } else {
                r = 0;
            }
            if (LM == 3) r = (int16_t)c_mul16_q14(23170, min32(23169, r));
            r = (int16_t)((thresh < r ? thresh : r) >> 1);
            r = (int16_t)(c_mul16_q15(sqrt_1, r) >> shift);
            int16_t *X = X_ + c * size + (eB[i] << LM);
            for (int k = 0; k < 1 << LM; k++) {
                if (!(collapse_masks[i * C + c] & 1 << k)) {
                    for (int j = 0; j < N0; j++) {
                        seed = c_lcg_rand(seed);
                        X[(j << LM) + k] = (seed & 0x8000) ? r : (int16_t)-r;
                    }
                    renormalize = 1;
                }
            }
            if (renormalize) renormalise_vector(L, X, N0 << LM, 32767);
        }
    }
}

DNI void tf_decode(int start, int end, int isTransient, int32_t *tf_res, int LM, RangeDec *dec)
{
    uint32_t budget = dec->storage * 8;
    uint32_t tell = (uint32_t)rd_tell(dec);
    int logp = isTransient ? 2 : 4;
    int tf_select_rsv = LM > 0 && tell + logp + 1 <= budget;
    budget -= tf_select_rsv;
    int tf_changed = 0, curr = 0;
    for (int i = start; i < end; i++) {
        if (tell + logp <= budget) {
            curr ^= rd_bit_logp(dec, logp);
            tell = (uint32_t)rd_tell(dec);
            tf_changed |= curr;
        }
        tf_res[i] = curr;
        logp = isTransient ? 4 : 5;
    }
    int tf_select = 0;
    const int8_t *tt = &T_celt_tf_select_table[LM * 8];
    if (tf_select_rsv && tt[4 * isTransient + 0 + tf_changed] != tt[4 * isTransient + 2 + tf_changed])
        tf_select = rd_bit_logp(dec, 1);
    for (int i = start; i < end; i++) tf_res[i] = tt[4 * isTransient + 2 * tf_select + tf_res[i]];
}

// ------------------------------------------------------------------ PLC (pitch / LPC)

DNI int32_t celt_autocorr(const int16_t *x, int32_t *ac, const int16_t *window, int overlap, int lag, int n,
                          int16_t *xx)
{
    int fastN = n - lag, shift;
    const int16_t *xptr;
    if (overlap == 0) {
        xptr = x;
    } else {
        for (int i = 0; i < n; i++) xx[i] = x[i];
        for (int i = 0; i < overlap; i++) {
            xx[i] = (int16_t)c_mul16_q15(x[i], window[i]);
            xx[n - i - 1] = (int16_t)c_mul16_q15(x[n - i - 1], window[i]);
        }
        xptr = xx;
    }
    {
        int32_t ac0 = 1 + (n << 7);
        if (n & 1) ac0 = wadd(ac0, c_mul16(xptr[0], xptr[0]) >> 9);
        for (int i = (n & 1); i < n; i += 2) {
            ac0 = wadd(ac0, c_mul16(xptr[i], xptr[i]) >> 9);
            ac0 = wadd(ac0, c_mul16(xptr[i + 1], xptr[i + 1]) >> 9);
        }
        shift = c_ilog2(ac0) - 30 + 10;
        shift = shift / 2;
        if (shift > 0) {
            for (int i = 0; i < n; i++) xx[i] = (int16_t)c_pshr(xptr[i], shift);
            xptr = xx;
        } else {
            shift = 0;
        }
    }
    for (int k = 0; k <= lag; k++) {
        int32_t s = 0;
        for (int j = 0; j < fastN; j++) s = c_mac16(s, xptr[j], xptr[j + k]);
        ac[k] = s;
    }
    for (int k = 0; k <= lag; k++) {
        int32_t d = 0;
        for (int i = k + fastN; i < n; i++) d = c_mac16(d, xptr[i], xptr[i - k]);
        ac[k] = wadd(ac[k], d);
    }
    shift = 2 * shift;
    if (shift <= 0) ac[0] = wadd(ac[0], shl32(1, -shift));
    if (ac[0] < 268435456) {
        int shift2 = 29 - ilog((uint32_t)ac[0]);
        for (int i = 0; i <= lag; i++) ac[i] = shl32(ac[i], shift2);
        shift -= shift2;
    } else if (ac[0] >= 536870912) {
        int shift2 = 1;
        if (ac[0] >= 1073741824) shift2++;
        for (int i = 0; i <= lag; i++) ac[i] = ac[i] >> shift2;
        shift += shift2;
    }
    return shift;
}

DNI void celt_lpc(int16_t *_lpc, const int32_t *ac, int p)
{
    int32_t error = ac[0];
    int32_t lpc[CELT_LPC_ORDER];
    for (int i = 0; i < p; i++) lpc[i] = 0;
    if (ac[0] != 0) {
        for (int i = 0; i < p; i++) {
            int32_t rr = 0;
            for (int j = 0; j < i; j++) rr = wadd(rr, c_mul32_q31(lpc[j], ac[i - j]));
            rr = wadd(rr, ac[i + 1] >> 6);
            int32_t r = -c_frac_div32(shl32(rr, 6), error);
            lpc[i] = r >> 6;
            for (int j = 0; j < (i + 1) >> 1; j++) {
                int32_t t1 = lpc[j], t2 = lpc[i - 1 - j];
                lpc[j] = wadd(t1, c_mul32_q31(r, t2));
                lpc[i - 1 - j] = wadd(t2, c_mul32_q31(r, t1));
            }
            error = wsub(error, c_mul32_q31(c_mul32_q31(r, r), error));
            if (error <= (ac[0] >> 10)) break;
        }
    }
    int iter, idx = 0;
    for (iter = 0; iter < 10; iter++) {
        int32_t maxabs = 0;
        for (int i = 0; i < p; i++) {
            int32_t a = lpc[i] < 0 ? -lpc[i] : lpc[i];
            if (a > maxabs) { maxabs = a; idx = i; }
        }
        maxabs = c_pshr(maxabs, 13);
        if (maxabs > 32767) {
            maxabs = min32(maxabs, 163838);
            int32_t chirp_Q16 = 65470 - shl32(maxabs - 32767, 14) / (wmul(maxabs, idx + 1) >> 2);
            int32_t cm1 = chirp_Q16 - 65536;
            for (int i = 0; i < p - 1; i++) {
                lpc[i] = c_mul32_q16(chirp_Q16, lpc[i]);
                chirp_Q16 += c_pshr(wmul(chirp_Q16, cm1), 16);
            }
            lpc[p - 1] = c_mul32_q16(chirp_Q16, lpc[p - 1]);
        } else {
            break;
        }
    }
    if (iter == 10) {
        _lpc[0] = 4096;   // the remaining outputs keep their previous values, as in libopus
    } else {
        for (int i = 0; i < p; i++) _lpc[i] = (int16_t)c_pshr(lpc[i], 13);
    }
}

DNI void celt_fir(const int16_t *x, const int16_t *num, int16_t *y, int N, int ord)
{
    for (int i = 0; i < N; i++) {
        int32_t sum = shl32((int32_t)x[i], 12);
        for (int j = 0; j < ord; j++) sum = c_mac16(sum, num[ord - j - 1], x[i + j - ord]);
        y[i] = c_sround16(sum, 12);
    }
}

// celt/celt_lpc.c celt_iir (the 4-way unrolled form computes the same values)
DNI void celt_iir(const int32_t *_x, const int16_t *den, int32_t *_y, int N, int ord, int16_t *mem, int16_t *y)
{
    for (int i = 0; i < ord; i++) y[i] = (int16_t)-mem[ord - i - 1];
    for (int i = ord; i < N + ord; i++) y[i] = 0;
    for (int i = 0; i < N; i++) {
        int32_t sum = _x[i];
        for (int j = 0; j < ord; j++) sum = c_mac16(sum, den[ord - j - 1], y[i + j]);
        y[i + ord] = (int16_t)-c_sround16(sum, 12);
        _y[i] = sum;
    }
    for (int i = 0; i < ord; i++) mem[i] = (int16_t)_y[N - i - 1];
}

DNI void find_best_pitch(const int32_t *xcorr, const int16_t *y, int len, int max_pitch, int *best_pitch,
                         int yshift, int32_t maxcorr)
{
    int32_t Syy = 1;
    int16_t best_num[2] = {-1, -1};
    int32_t best_den[2] = {0, 0};
    int xshift = c_ilog2(maxcorr) - 14;
    best_pitch[0] = 0;
    best_pitch[1] = 1;
    for (int j = 0; j < len; j++) Syy = wadd(Syy, c_mul16(y[j], y[j]) >> yshift);
    for (int i = 0; i < max_pitch; i++) {
        if (xcorr[i] > 0) {
            int16_t xcorr16 = (int16_t)c_vshr(xcorr[i], xshift);
            int16_t num = (int16_t)c_mul16_q15(xcorr16, xcorr16);
            if (c_mul16_32_q15(num, best_den[1]) > c_mul16_32_q15(best_num[1], Syy)) {
                if (c_mul16_32_q15(num, best_den[0]) > c_mul16_32_q15(best_num[0], Syy)) {
                    best_num[1] = best_num[0];
                    best_den[1] = best_den[0];
                    best_pitch[1] = best_pitch[0];
                    best_num[0] = num;
                    best_den[0] = Syy;
                    best_pitch[0] = i;
                } else {
                    best_num[1] = num;
                    best_den[1] = Syy;
                    best_pitch[1] = i;
                }
            }
        }
        Syy = wadd(Syy, wsub(c_mul16(y[i + len], y[i + len]) >> yshift, c_mul16(y[i], y[i]) >> yshift));
        Syy = max32(1, Syy);
    }
}

DNI void pitch_downsample(int32_t *x0, int32_t *x1, int16_t *x_lp, int len, int C, int16_t *xx)
{
    int32_t ac[5];
    int16_t tmp = 32767, lpc[4], lpc2[5];
    const int16_t c1 = 26214;   // QCONST16(.8f, 15)
    int32_t maxabs = c_maxabs32(x0, len);
    if (C == 2) maxabs = max32(maxabs, c_maxabs32(x1, len));
    if (maxabs < 1) maxabs = 1;
    int shift = c_ilog2(maxabs) - 10;
    if (shift < 0) shift = 0;
    if (C == 2) shift++;
    for (int i = 1; i < len >> 1; i++)
        x_lp[i] = (int16_t)((x0[2 * i - 1] >> (shift + 2)) + (x0[2 * i + 1] >> (shift + 2)) + (x0[2 * i] >> (shift + 1)));
    x_lp[0] = (int16_t)((x0[1] >> (shift + 2)) + (x0[0] >> (shift + 1)));
    if (C == 2) {
        for (int i = 1; i < len >> 1; i++)
            x_lp[i] = (int16_t)(x_lp[i] + (x1[2 * i - 1] >> (shift + 2)) + (x1[2 * i + 1] >> (shift + 2)) +
                                (x1[2 * i] >> (shift + 1)));
        x_lp[0] = (int16_t)(x_lp[0] + (x1[1] >> (shift + 2)) + (x1[0] >> (shift + 1)));
    }
    celt_autocorr(x_lp, ac, 0, 0, 4, len >> 1, xx);
    ac[0] = wadd(ac[0], ac[0] >> 13);
    for (int i = 1; i <= 4; i++) ac[i] = wsub(ac[i], c_mul16_32_q15(2 * i * i, ac[i]));
    celt_lpc(lpc, ac, 4);
    for (int i = 0; i < 4; i++) {
        tmp = (int16_t)c_mul16_q15(29491, tmp);   // QCONST16(.9f, 15)
        lpc[i] = (int16_t)c_mul16_q15(lpc[i], tmp);
    }
    lpc2[0] = (int16_t)(lpc[0] + 3277);   // QCONST16(.8f, SIG_SHIFT)
    lpc2[1] = (int16_t)(lpc[1] + c_mul16_q15(c1, lpc[0]));
    lpc2[2] = (int16_t)(lpc[2] + c_mul16_q15(c1, lpc[1]));
    lpc2[3] = (int16_t)(lpc[3] + c_mul16_q15(c1, lpc[2]));
    lpc2[4] = (int16_t)c_mul16_q15(c1, lpc[3]);
    // celt_fir5 in place
    int32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0, m4 = 0;
    for (int i = 0; i < len >> 1; i++) {
        int32_t sum = shl32((int32_t)x_lp[i], 12);
        sum = c_mac16(sum, lpc2[0], m0);
        sum = c_mac16(sum, lpc2[1], m1);
        sum = c_mac16(sum, lpc2[2], m2);
        sum = c_mac16(sum, lpc2[3], m3);
        sum = c_mac16(sum, lpc2[4], m4);
        m4 = m3; m3 = m2; m2 = m1; m1 = m0;
        m0 = x_lp[i];
        x_lp[i] = (int16_t)c_pshr(sum, 12);
    }
}

DNI void pitch_search(Lanes L, const int16_t *x_lp, int16_t *y, int len, int max_pitch, int *pitch,
                      CeltScratch *w)
{
    int lag = len + max_pitch;
    int best_pitch[2] = {0, 0};
    int16_t *x_lp4 = w->x_lp4, *y_lp4 = w->y_lp4;
    int32_t *xcorr = w->xcorr;
    for (int j = 0; j < len >> 2; j++) x_lp4[j] = x_lp[2 * j];
    for (int j = 0; j < lag >> 2; j++) y_lp4[j] = y[2 * j];
    int32_t xmax = c_maxabs16(x_lp4, len >> 2), ymax = c_maxabs16(y_lp4, lag >> 2);
    int shift = c_ilog2(max32(1, max32(xmax, ymax))) - 11;
    if (shift > 0) {
        for (int j = 0; j < len >> 2; j++) x_lp4[j] = (int16_t)(x_lp4[j] >> shift);
        for (int j = 0; j < lag >> 2; j++) y_lp4[j] = (int16_t)(y_lp4[j] >> shift);
        shift *= 2;
    } else {
        shift = 0;
    }
    lsync(L);
    // celt_pitch_xcorr: every lag is an independent dot product
    LFOR(L, i, 0, max_pitch >> 2) {
        int32_t s = 0;
        for (int j = 0; j < len >> 2; j++) s = c_mac16(s, x_lp4[j], y_lp4[i + j]);
        xcorr[i] = s;
    }
    lsync(L);
    int32_t maxcorr = 1;
    for (int i = 0; i < max_pitch >> 2; i++) maxcorr = max32(maxcorr, xcorr[i]);
    find_best_pitch(xcorr, y_lp4, len >> 2, max_pitch >> 2, best_pitch, 0, maxcorr);
    lsync(L);
    LFOR(L, i, 0, max_pitch >> 1) {
        xcorr[i] = 0;
        int d0 = i - 2 * best_pitch[0], d1 = i - 2 * best_pitch[1];
        if (!((d0 < 0 ? -d0 : d0) > 2 && (d1 < 0 ? -d1 : d1) > 2)) {
            int32_t s = 0;
            for (int j = 0; j < len >> 1; j++) s = wadd(s, c_mul16(x_lp[j], y[i + j]) >> shift);
            xcorr[i] = max32(-1, s);
        }
    }
    lsync(L);
    // libopus tracks max(1, raw sums); the -1 floor and the zeroed lags cannot exceed 1
    maxcorr = 1;
    for (int i = 0; i < max_pitch >> 1; i++) maxcorr = max32(maxcorr, xcorr[i]);
    find_best_pitch(xcorr, y, len >> 1, max_pitch >> 1, best_pitch, shift + 1, maxcorr);
    int offset;
    if (best_pitch[0] > 0 && best_pitch[0] < (max_pitch >> 1) - 1) {
        int32_t a = xcorr[best_pitch[0] - 1], b = xcorr[best_pitch[0]], c = xcorr[best_pitch[0] + 1];
        if ((c - a) > c_mul16_32_q15(22938, b - a)) offset = 1;          // QCONST16(.7f, 15)
        else if ((a - c) > c_mul16_32_q15(22938, b - c)) offset = -1;
        else offset = 0;
    } else {
        offset = 0;
    }
    *pitch = 2 * best_pitch[0] - offset;
}

DNI void prefilter_and_fold(CeltDec *st, int N, CeltScratch *w)
{
    for (int c = 0; c < st->channels; c++) {
        int32_t *dm = st->decode_mem[c];
        comb_filter(w->etmp, dm + CELT_DEC_BUF - N, st->postfilter_period_old, st->postfilter_period, CELT_OVERLAP,
                    (int16_t)-st->postfilter_gain_old, (int16_t)-st->postfilter_gain, st->postfilter_tapset_old,
                    st->postfilter_tapset, 0, 0);
        for (int i = 0; i < CELT_OVERLAP / 2; i++)
            dm[CELT_DEC_BUF - N + i] = wadd(c_mul16_32_q15(T_celt_window[i], w->etmp[CELT_OVERLAP - 1 - i]),
                                            c_mul16_32_q15(T_celt_window[CELT_OVERLAP - i - 1], w->etmp[i]));
    }
}

// celt/celt_decoder.c celt_decode_lost (no deep PLC)
DNI void celt_decode_lost(Lanes L, CeltDec *st, int N, int LM, CeltScratch *w)
{
    const int C = st->channels;
    const int16_t *eB = T_celt_eBands;
    int32_t *out_syn[2];
    for (int c = 0; c < C; c++) out_syn[c] = st->decode_mem[c] + CELT_DEC_BUF - N;
    int loss_duration = st->loss_duration;
    int start = st->start;
    int noise_based = loss_duration >= 40 || start != 0 || st->skip_plc;
    if (noise_based) {
        int end = st->end;
        int effEnd = imax(start, imin(end, T_CELT_EFFEBANDS));
        int16_t *X = w->X;
        for (int c = 0; c < C; c++) lshift_copy(L, st->decode_mem[c], CELT_DEC_BUF - N + CELT_OVERLAP, N);
        if (st->prefilter_and_fold) prefilter_and_fold(st, N, w);
        int16_t decay = loss_duration == 0 ? 1536 : 512;   // QCONST16(1.5f / .5f, DB_SHIFT)
        for (int c = 0; c < C; c++)
            for (int i = start; i < end; i++) {
                int32_t a = st->backgroundLogE[c * CELT_NB + i];
                int32_t b = st->oldBandE[c * CELT_NB + i] - decay;
                st->oldBandE[c * CELT_NB + i] = (int16_t)(a > b ? a : b);
            }
        uint32_t seed = st->rng;
        for (int c = 0; c < C; c++) {
            for (int i = start; i < effEnd; i++) {
                int boffs = N * c + (eB[i] << LM);
                int blen = (eB[i + 1] - eB[i]) << LM;
                for (int j = 0; j < blen; j++) {
                    seed = c_lcg_rand(seed);
                    X[boffs + j] = (int16_t)((int32_t)seed >> 20);
                }
                renormalise_vector(L, X + boffs, blen, 32767);
            }
        }
        st->rng = seed;
        lsync(L);
        celt_synthesis(L, w, X, out_syn, st->oldBandE, start, effEnd, C, C, 0, LM, 0);
        st->prefilter_and_fold = 0;
        st->skip_plc = 1;
    } else {
        int16_t fade = 32767;
        int pitch_index;
        if (loss_duration == 0) {
            pitch_downsample(st->decode_mem[0], st->decode_mem[1], w->lp_pitch_buf, CELT_DEC_BUF, C, w->ac_xx);
            lsync(L);
            pitch_search(L, w->lp_pitch_buf + (720 >> 1), w->lp_pitch_buf, CELT_DEC_BUF - 720, 720 - 100,
                         &pitch_index, w);
            pitch_index = 720 - pitch_index;
            st->last_pitch_index = pitch_index;
        } else {
            pitch_index = st->last_pitch_index;
            fade = 26214;   // QCONST16(.8f, 15)
        }
        int exc_length = imin(2 * pitch_index, CELT_MAX_PERIOD);
        int16_t *exc = w->exc + CELT_LPC_ORDER;
        const int16_t *window = T_celt_window;
        for (int c = 0; c < C; c++) {
            int32_t *buf = st->decode_mem[c];
            int16_t *lpc = st->lpc[c];
            int32_t S1 = 0;
            for (int i = 0; i < CELT_MAX_PERIOD + CELT_LPC_ORDER; i++)
                exc[i - CELT_LPC_ORDER] = c_sround16(buf[CELT_DEC_BUF - CELT_MAX_PERIOD - CELT_LPC_ORDER + i], 12);
            if (loss_duration == 0) {
                int32_t ac[CELT_LPC_ORDER + 1];
                celt_autocorr(exc, ac, window, CELT_OVERLAP, CELT_LPC_ORDER, CELT_MAX_PERIOD, w->ac_xx);
                ac[0] = wadd(ac[0], ac[0] >> 13);
                for (int i = 1; i <= CELT_LPC_ORDER; i++) ac[i] = wsub(ac[i], c_mul16_32_q15(2 * i * i, ac[i]));
                celt_lpc(lpc, ac, CELT_LPC_ORDER);
                while (1) {
                    int16_t tmp = 32767;
                    int32_t sum = 4096;   // QCONST16(1., SIG_SHIFT)
                    for (int i = 0; i < CELT_LPC_ORDER; i++) sum += lpc[i] < 0 ? -lpc[i] : lpc[i];
                    if (sum < 65535) break;
                    for (int i = 0; i < CELT_LPC_ORDER; i++) {
                        tmp = (int16_t)c_mul16_q15(32440, tmp);   // QCONST16(.99f, 15)
                        lpc[i] = (int16_t)c_mul16_q15(lpc[i], tmp);
                    }
                }
            }
            celt_fir(exc + CELT_MAX_PERIOD - exc_length, lpc, w->fir_tmp, exc_length, CELT_LPC_ORDER);
            for (int i = 0; i < exc_length; i++) exc[CELT_MAX_PERIOD - exc_length + i] = w->fir_tmp[i];
            int16_t decay;
            {
                int32_t E1 = 1, E2 = 1;
                int shift = imax(0, 2 * c_zlog2(c_maxabs16(&exc[CELT_MAX_PERIOD - exc_length], exc_length)) - 20);
                int decay_length = exc_length >> 1;
                for (int i = 0; i < decay_length; i++) {
                    int16_t e = exc[CELT_MAX_PERIOD - decay_length + i];
                    E1 = wadd(E1, c_mul16(e, e) >> shift);
                    e = exc[CELT_MAX_PERIOD - 2 * decay_length + i];
                    E2 = wadd(E2, c_mul16(e, e) >> shift);
                }
                E1 = min32(E1, E2);
                decay = (int16_t)c_sqrt(c_frac_div32(E1 >> 1, E2));
            }
            for (int i = 0; i < CELT_DEC_BUF - N; i++) buf[i] = buf[i + N];
            int extrapolation_offset = CELT_MAX_PERIOD - pitch_index;
            int extrapolation_len = N + CELT_OVERLAP;
            int16_t attenuation = (int16_t)c_mul16_q15(fade, decay);
            for (int i = 0, j = 0; i < extrapolation_len; i++, j++) {
                if (j >= pitch_index) {
                    j -= pitch_index;
                    attenuation = (int16_t)c_mul16_q15(attenuation, decay);
                }
                buf[CELT_DEC_BUF - N + i] = shl32((int32_t)(int16_t)c_mul16_q15(attenuation,
                                                  exc[extrapolation_offset + j]), 12);
                int16_t tmp = c_sround16(buf[CELT_DEC_BUF - CELT_MAX_PERIOD - N + extrapolation_offset + j], 12);
                S1 = wadd(S1, c_mul16(tmp, tmp) >> 10);
            }
            {
                int16_t lpc_mem[CELT_LPC_ORDER];
                for (int i = 0; i < CELT_LPC_ORDER; i++) lpc_mem[i] = c_sround16(buf[CELT_DEC_BUF - N - 1 - i], 12);
                celt_iir(buf + CELT_DEC_BUF - N, lpc, buf + CELT_DEC_BUF - N, extrapolation_len, CELT_LPC_ORDER,
                         lpc_mem, w->iir_y);
                for (int i = 0; i < extrapolation_len; i++)
                    buf[CELT_DEC_BUF - N + i] = c_sat(buf[CELT_DEC_BUF - N + i], CELT_SIG_SAT);
            }
            {
                int32_t S2 = 0;
                for (int i = 0; i < extrapolation_len; i++) {
                    int16_t tmp = c_sround16(buf[CELT_DEC_BUF - N + i], 12);
                    S2 = wadd(S2, c_mul16(tmp, tmp) >> 10);
                }
                if (!(S1 > (S2 >> 2))) {
                    for (int i = 0; i < extrapolation_len; i++) buf[CELT_DEC_BUF - N + i] = 0;
                } else if (S1 < S2) {
                    int16_t ratio = (int16_t)c_sqrt(c_frac_div32((S1 >> 1) + 1, S2 + 1));
                    for (int i = 0; i < CELT_OVERLAP; i++) {
                        int16_t tmp_g = (int16_t)(32767 - c_mul16_q15(window[i], (int16_t)(32767 - ratio)));
                        buf[CELT_DEC_BUF - N + i] = c_mul16_32_q15(tmp_g, buf[CELT_DEC_BUF - N + i]);
                    }
                    for (int i = CELT_OVERLAP; i < extrapolation_len; i++)
                        buf[CELT_DEC_BUF - N + i] = c_mul16_32_q15(ratio, buf[CELT_DEC_BUF - N + i]);
                }
            }
        }
        st->prefilter_and_fold = 1;
    }
    st->loss_duration = imin(10000, loss_duration + (1 << LM));
    lsync(L);
}

// ------------------------------------------------------------------ frame decode

// The band energies of the first frame after a loss that is not intra coded
// (celt/celt_decoder.c, in celt_decode_with_ec_dred before unquant_coarse_energy):
// each energy may rise at most as the previous two frames did, less a safety
// margin.  Its own function, so the code of the lossless path stays small.
DNI void energy_after_loss(CeltDec *st, int start, int end, int LM)
{
    int16_t *oldBandE = st->oldBandE, *oldLogE = st->oldLogE, *oldLogE2 = st->oldLogE2;
    for (int c = 0; c < 2; c++) {
        int16_t safety = 0;
        int missing = imin(10, st->loss_duration >> LM);
        if (LM == 0) safety = 1536;
        else if (LM == 1) safety = 512;
        for (int i = start; i < end; i++) {
            int16_t *e0 = &oldBandE[c * CELT_NB + i];
            int16_t e1 = oldLogE[c * CELT_NB + i], e2 = oldLogE2[c * CELT_NB + i];
            if (*e0 < (e1 > e2 ? e1 : e2)) {
                int32_t E0 = *e0, E1 = e1, E2 = e2;
                int32_t slope = max32(E1 - E0, (E2 - E0) >> 1);
                E0 -= max32(0, (1 + missing) * slope);
                *e0 = (int16_t)max32(-20480, E0);   // -QCONST16(20.f, DB_SHIFT)
            } else {
                int16_t m = *e0 < e1 ? *e0 : e1;
                *e0 = m < e2 ? m : e2;
            }
            *e0 = (int16_t)(*e0 - safety);
        }
    }
}

// celt/celt_decoder.c celt_decode_with_ec_dred (downsample 1, no deep PLC).
// data == 0 or len <= 1 runs the concealment.  Returns samples or < 0.
DNI int celt_decode(Lanes L, CeltDec *st, const uint8_t *data, int len, int16_t *pcm, int frame_size,
                    RangeDec *dec, int accum, CeltScratch *w)
{
    const int16_t *eB = T_celt_eBands;
    const int CC = st->channels;
    int C = st->stream_channels;
    int start = st->start, end = st->end;
    int LM;
    for (LM = 0; LM <= T_CELT_MAXLM; LM++)
        if (T_CELT_SHORTMDCT << LM == frame_size) break;
    if (LM > T_CELT_MAXLM) return -1;   // OPUS_BAD_ARG
    int M = 1 << LM;
    if (len < 0 || len > 1275 || pcm == 0) return -1;
    int N = M * T_CELT_SHORTMDCT;
    int32_t *out_syn[2];
    for (int c = 0; c < CC; c++) out_syn[c] = st->decode_mem[c] + CELT_DEC_BUF - N;
    if (CC == 1) out_syn[1] = out_syn[0];
    int effEnd = end;
    if (effEnd > T_CELT_EFFEBANDS) effEnd = T_CELT_EFFEBANDS;
    if (data == 0 || len <= 1) {
        // concealment (mode transitions, lost packets): serial extrapolation
        // and state updates in place, on the first lane as a group of one
        lead(L, [&]() CUO_INLINE { celt_decode_lost(lone(L), st, N, LM, w); });
        deemphasis(L, out_syn[0], out_syn[1], pcm, N, CC, st->preemph_memD, accum);
        return frame_size;
    }
    RangeDec _dec;
    if (dec == 0) {
        rd_init(&_dec, data, len);
        dec = &_dec;
    }
    int16_t *oldBandE = st->oldBandE, *oldLogE = st->oldLogE, *oldLogE2 = st->oldLogE2,
            *backgroundLogE = st->backgroundLogE;
    if (C == 1) {
        LFOR(L, i, 0, CELT_NB) oldBandE[i] = oldBandE[i] > oldBandE[CELT_NB + i] ? oldBandE[i] : oldBandE[CELT_NB + i];
    }
    int32_t *tf_res = w->tf_res;
    int32_t *pulses = w->pulses, *fine_quant = w->fine_quant, *fine_priority = w->fine_priority;
    // The frame header, the energies and the bit allocation: entropy decoding
    // and state updates in place, on the first lane; every lane gets the
    // outcome (the per-band tables stay in the scratch).
    enum { H_SILENCE, H_PF_GAIN, H_PF_PITCH, H_PF_TAPSET, H_TRANSIENT, H_SPREAD, H_AC_RSV, H_INTENSITY, H_DUAL,
           H_BALANCE, H_CODED, H_N };
    int32_t hv[H_N] = {0};
    lead_rd(L, dec, [&]() CUO_INLINE {
        if (st->loss_duration == 0) st->skip_plc = 0;
        int32_t total_bits = len * 8;
        int32_t tell = rd_tell(dec);
        int silence;
        if (tell >= total_bits) silence = 1;
        else if (tell == 1) silence = rd_bit_logp(dec, 15);
        else silence = 0;
        if (silence) {
            tell = len * 8;
            dec->nbits_total += tell - rd_tell(dec);
        }
        int16_t postfilter_gain = 0;
        int postfilter_pitch = 0, postfilter_tapset = 0;
        if (start == 0 && tell + 16 <= total_bits) {
            if (rd_bit_logp(dec, 1)) {
                int octave = (int)rd_uint(dec, 6);
                postfilter_pitch = (16 << octave) + (int)rd_bits(dec, 4 + octave) - 1;
                int qg = (int)rd_bits(dec, 3);
                if (rd_tell(dec) + 2 <= total_bits) postfilter_tapset = rd_icdf(dec, T_celt_tapset_icdf, 2);
                postfilter_gain = (int16_t)(3072 * (qg + 1));   // QCONST16(.09375f, 15)
            }
            tell = rd_tell(dec);
        }
        int isTransient;
        if (LM > 0 && tell + 3 <= total_bits) {
            isTransient = rd_bit_logp(dec, 3);
            tell = rd_tell(dec);
        } else {
            isTransient = 0;
        }
        int intra_ener = tell + 3 <= total_bits ? rd_bit_logp(dec, 3) : 0;
        if (!intra_ener && st->loss_duration != 0) energy_after_loss(st, start, end, LM);
        PHASE_BEGIN(t_ce);
        unquant_coarse_energy(start, end, oldBandE, intra_ener, dec, C, LM);
        PHASE_END(PH_CELT_COARSE, t_ce, L.id);
        tf_decode(start, end, isTransient, tf_res, LM, dec);
        tell = rd_tell(dec);
        int spread_decision = SPREAD_NORMAL;
        if (tell + 4 <= total_bits) spread_decision = rd_icdf(dec, T_celt_spread_icdf, 5);
        int32_t *cap = w->cap, *offsets = w->offsets;
        init_caps(cap, LM, C);
        int dynalloc_logp = 6;
        total_bits <<= 3;
        tell = (int32_t)rd_tell_frac(dec);
        for (int i = start; i < end; i++) {
            int width = C * (eB[i + 1] - eB[i]) << LM;
            int quanta = imin(width << 3, imax(6 << 3, width));
            int dll = dynalloc_logp, boost = 0;
            while (tell + (dll << 3) < total_bits && boost < cap[i]) {
                int flag = rd_bit_logp(dec, dll);
                tell = (int32_t)rd_tell_frac(dec);
                if (!flag) break;
                boost += quanta;
                total_bits -= quanta;
                dll = 1;
            }
            offsets[i] = boost;
            if (boost > 0) dynalloc_logp = imax(2, dynalloc_logp - 1);
        }
        int alloc_trim = tell + (6 << 3) <= total_bits ? rd_icdf(dec, T_celt_trim_icdf, 7) : 5;
        int32_t bits = (((int32_t)len * 8) << 3) - (int32_t)rd_tell_frac(dec) - 1;
        int anti_collapse_rsv = isTransient && LM >= 2 && bits >= ((LM + 2) << 3) ? (1 << 3) : 0;
        bits -= anti_collapse_rsv;
        int intensity = 0, dual_stereo = 0;
        int32_t balance;
        PHASE_BEGIN(t_al);
        int codedBands = clt_compute_allocation(start, end, offsets, cap, alloc_trim, &intensity, &dual_stereo,
                                                bits, &balance, pulses, fine_quant, fine_priority, C, LM, dec, w);
        PHASE_END(PH_CELT_ALLOC, t_al, L.id);
        unquant_fine_energy(start, end, oldBandE, fine_quant, dec, C);
        hv[H_SILENCE] = silence;
        hv[H_PF_GAIN] = postfilter_gain;
        hv[H_PF_PITCH] = postfilter_pitch;
        hv[H_PF_TAPSET] = postfilter_tapset;
        hv[H_TRANSIENT] = isTransient;
        hv[H_SPREAD] = spread_decision;
        hv[H_AC_RSV] = anti_collapse_rsv;
        hv[H_INTENSITY] = intensity;
        hv[H_DUAL] = dual_stereo;
        hv[H_BALANCE] = balance;
        hv[H_CODED] = codedBands;
    });
    for (int k = 0; k < H_N; k++) hv[k] = lbcast(L, hv[k]);
    const int silence = hv[H_SILENCE];
    const int16_t postfilter_gain = (int16_t)hv[H_PF_GAIN];
    const int postfilter_pitch = hv[H_PF_PITCH], postfilter_tapset = hv[H_PF_TAPSET];
    const int isTransient = hv[H_TRANSIENT], shortBlocks = isTransient ? M : 0;
    const int spread_decision = hv[H_SPREAD], anti_collapse_rsv = hv[H_AC_RSV];
    const int intensity = hv[H_INTENSITY], dual_stereo = hv[H_DUAL];
    const int32_t balance = hv[H_BALANCE];
    const int codedBands = hv[H_CODED];
    PHASE_BEGIN(t_sh);
    for (int c = 0; c < CC; c++) lshift_copy(L, st->decode_mem[c], CELT_DEC_BUF - N + CELT_OVERLAP, N);
    PHASE_END(PH_CELT_SHIFT, t_sh, L.id);
    int16_t *X = w->X;
    // The band shapes: the PVQ split recursion updates its stack, the band
    // vectors and the folding buffer in place from entropy-decoded values,
    // so it runs on the first lane as a group of one.
    PHASE_BEGIN(t_qb);
    lead_rd(L, dec, [&]() CUO_INLINE {
        quant_all_bands_dec(lone(L), start, end, X, C == 2 ? X + N : 0, w->collapse_masks, pulses, shortBlocks,
                            spread_decision, dual_stereo, intensity, tf_res, len * (8 << 3) - anti_collapse_rsv,
                            balance, dec, LM, codedBands, &st->rng, st->disable_inv, w);
    });
    PHASE_END(PH_CELT_BANDS, t_qb, L.id);
    int anti_collapse_on = 0;
    lead_rd(L, dec, [&]() CUO_INLINE {
        if (anti_collapse_rsv > 0) anti_collapse_on = (int)rd_bits(dec, 1);
        unquant_energy_finalise(start, end, oldBandE, fine_quant, fine_priority, len * 8 - rd_tell(dec), dec, C);
    });
    anti_collapse_on = lbcast(L, anti_collapse_on);
    lead(L, [&]() CUO_INLINE {
        if (anti_collapse_on)
            anti_collapse(lone(L), X, w->collapse_masks, LM, C, N, start, end, oldBandE, oldLogE, oldLogE2, pulses,
                          st->rng);
        if (silence)
            for (int i = 0; i < C * CELT_NB; i++) oldBandE[i] = -28672;   // -QCONST16(28.f, DB_SHIFT)
        if (st->prefilter_and_fold) prefilter_and_fold(st, N, w);
    });
    PHASE_BEGIN(t_sy);
    celt_synthesis(L, w, X, out_syn, oldBandE, start, effEnd, C, CC, isTransient, LM, silence);
    PHASE_END(PH_CELT_SYNTH, t_sy, L.id);
    PHASE_BEGIN(t_cb);
    // the post-filter state is read once into registers here and written back
    // on the first lane after the filter, both with the period floored at 15
    const int pf_period = imax(st->postfilter_period, 15), pf_period_old = imax(st->postfilter_period_old, 15);
    const int16_t pf_gain = (int16_t)st->postfilter_gain, pf_gain_old = (int16_t)st->postfilter_gain_old;
    const int pf_tapset = st->postfilter_tapset, pf_tapset_old = st->postfilter_tapset_old;
    for (int c = 0; c < CC; c++) {
        comb_filter_lanes(L, out_syn[c], out_syn[c], pf_period_old, pf_period, T_CELT_SHORTMDCT, pf_gain_old,
                          pf_gain, pf_tapset_old, pf_tapset, T_celt_window, CELT_OVERLAP);
        if (LM != 0)
            comb_filter_lanes(L, out_syn[c] + T_CELT_SHORTMDCT, out_syn[c] + T_CELT_SHORTMDCT, pf_period,
                              postfilter_pitch, N - T_CELT_SHORTMDCT, pf_gain, postfilter_gain, pf_tapset,
                              postfilter_tapset, T_celt_window, CELT_OVERLAP);
    }
    PHASE_END(PH_CELT_COMB, t_cb, L.id);
    lead(L, [&]() CUO_INLINE {
        st->postfilter_period_old = pf_period;
        st->postfilter_gain_old = pf_gain;
        st->postfilter_tapset_old = pf_tapset;
        st->postfilter_period = postfilter_pitch;
        st->postfilter_gain = postfilter_gain;
        st->postfilter_tapset = postfilter_tapset;
        if (LM != 0) {
            st->postfilter_period_old = st->postfilter_period;
            st->postfilter_gain_old = st->postfilter_gain;
            st->postfilter_tapset_old = st->postfilter_tapset;
        }
    });
    // energy history: every band of both channels on its own, so lanes split them
    if (C == 1) {
        LFOR(L, i, 0, CELT_NB) oldBandE[CELT_NB + i] = oldBandE[i];
        lsync(L);
    }
    int32_t mbi = imin(160, st->loss_duration + M) * 1;   // QCONST16(0.001f, DB_SHIFT) == 1
    LFOR(L, j, 0, 2 * CELT_NB) {
        int16_t e = oldBandE[j];
        if (!isTransient) {
            oldLogE2[j] = oldLogE[j];
            oldLogE[j] = e;
        } else {
            oldLogE[j] = oldLogE[j] < e ? oldLogE[j] : e;
        }
        int32_t v = backgroundLogE[j] + mbi;
        backgroundLogE[j] = (int16_t)(v < e ? v : e);
        int i = j < CELT_NB ? j : j - CELT_NB;
        if (i < start || i >= end) {
            oldBandE[j] = 0;
            oldLogE[j] = oldLogE2[j] = -28672;
        }
    }
    PHASE_BEGIN(t_de);
    deemphasis(L, out_syn[0], out_syn[1], pcm, N, CC, st->preemph_memD, accum);
    PHASE_END(PH_CELT_DEEMPH, t_de, L.id);
    lead(L, [&]() CUO_INLINE {
        st->rng = dec->rng;
        st->loss_duration = 0;
        st->prefilter_and_fold = 0;
        if (rd_tell(dec) <= 8 * len && dec->error) st->error = 1;
    });
    if (rd_tell(dec) > 8 * len) return -3;   // OPUS_INTERNAL_ERROR
    return frame_size;
}

} // namespace cuo
