// SILK decoder (RFC 6716 section 4.2), fixed point, API rate 48 kHz.
//
// Restates the libopus 1.5.2 decode path file by file:
//   silk/dec_API.c            silk_Decode, silk_InitDecoder, silk_ResetDecoder
//   silk/init_decoder.c       silk_init_decoder / silk_reset_decoder
//   silk/decoder_set_fs.c     silk_decoder_set_fs
//   silk/decode_frame.c       silk_decode_frame
//   silk/decode_indices.c     silk_decode_indices
//   silk/decode_pulses.c, shell_coder.c, code_signs.c
//   silk/decode_parameters.c, gain_quant.c (silk_gains_dequant), NLSF_decode.c,
//   NLSF_unpack.c, NLSF_stabilize.c, NLSF2A.c, LPC_fit.c, LPC_inv_pred_gain.c,
//   bwexpander.c, bwexpander_32.c, decode_pitch.c, sort.c
//   silk/decode_core.c, LPC_analysis_filter.c
//   silk/PLC.c, CNG.c, sum_sqr_shift.c
//   silk/stereo_decode_pred.c, stereo_MS_to_LR.c
//   silk/resampler.c, resampler_private_IIR_FIR.c, resampler_private_up2_HQ.c
// The decoder always runs at an API rate of 48 kHz, so the resampler is the
// IIR_FIR (2x all-pass + 12-phase FIR) path of silk_resampler_init for 8, 12
// and 16 kHz input.  Deep PLC / OSCE are compiled out, as in the fixed-point
// build the reference decodes with.
#pragma once
#include "rangedec.cuh"

namespace cuo {

enum { SILK_MAX_FRAME = 320, SILK_MAX_SUBFR_LEN = 80, SILK_MAX_ORDER = 16, SILK_LTP_ORDER = 5 };
enum { SIG_NO_VOICE = 0, SIG_UNVOICED = 1, SIG_VOICED = 2 };
enum { CODE_INDEP = 0, CODE_INDEP_NO_LTP_SCALING = 1, CODE_COND = 2 };
enum { LOSS_NONE = 0, LOSS_LOST = 1, LOSS_LBRR = 2 };

struct SilkResampler {
    int32_t sIIR[6];
    int16_t sFIR[8];
    int16_t delayBuf[48];
    int32_t invRatio_Q16;
    int16_t batchSize, Fs_in_kHz, Fs_out_kHz, inputDelay;
};

struct SilkIndices {
    int8_t GainsIndices[4];
    int8_t LTPIndex[4];
    int8_t NLSFIndices[17];
    int16_t lagIndex;
    int8_t contourIndex, signalType, quantOffsetType, NLSFInterpCoef_Q2, PERIndex, LTP_scaleIndex,
        Seed;
};

struct SilkPLC {
    int32_t pitchL_Q8;
    int16_t LTPCoef_Q14[5];
    int16_t prevLPC_Q12[16];
    int32_t last_frame_lost;
    int32_t rand_seed;
    int16_t randScale_Q14;
    int32_t conc_energy;
    int32_t conc_energy_shift;
    int16_t prevLTP_scale_Q14;
    int32_t prevGain_Q16[2];
    int32_t fs_kHz, nb_subfr, subfr_length;
};

struct SilkCNG {
    int32_t CNG_exc_buf_Q14[SILK_MAX_FRAME];
    int16_t CNG_smth_NLSF_Q15[16];
    int32_t CNG_synth_state[16];
    int32_t CNG_smth_Gain_Q16;
    int32_t rand_seed;
    int32_t fs_kHz;
};

// silk_decoder_state (silk/structs.h); the reset region starts at prev_gain_Q16
struct SilkChan {
    int32_t prev_gain_Q16;
    int32_t exc_Q14[SILK_MAX_FRAME];
    int32_t sLPC_Q14_buf[16];
    int16_t outBuf[SILK_MAX_FRAME + 2 * SILK_MAX_SUBFR_LEN];
    int32_t lagPrev;
    int32_t LastGainIndex;
    int32_t fs_kHz;
    int32_t fs_API_hz;
    int32_t nb_subfr, frame_length, subfr_length, ltp_mem_length, LPC_order;
    int16_t prevNLSF_Q15[16];
    int32_t first_frame_after_reset;
    int32_t nFramesDecoded, nFramesPerPacket;
    int32_t ec_prevSignalType;
    int32_t ec_prevLagIndex;
    int32_t VAD_flags[3];
    int32_t LBRR_flag;
    int32_t LBRR_flags[3];
    SilkResampler resampler_state;
    SilkIndices indices;
    SilkCNG sCNG;
    int32_t lossCnt;
    int32_t prevSignalType;
    SilkPLC sPLC;
};

struct SilkStereo {
    int16_t pred_prev_Q13[2];
    int16_t sMid[2];
    int16_t sSide[2];
};

// silk_decoder super struct (silk/dec_API.c)
struct SilkDec {
    SilkChan ch[2];
    SilkStereo sStereo;
    int32_t nChannelsAPI, nChannelsInternal, prev_decode_only_middle;
};

struct SilkCtrl {     // silk_decoder_control
    int32_t pitchL[4];
    int32_t Gains_Q16[4];
    int16_t PredCoef_Q12[2][16];
    int16_t LTPCoef_Q14[5 * 4];
    int32_t LTP_scale_Q14;
};

struct SilkDecControl {   // silk_DecControlStruct (decoder fields)
    int32_t nChannelsAPI, nChannelsInternal, API_sampleRate, internalSampleRate, payloadSize_ms;
};

// Per-slot scratch of the SILK decoder (replaces the stack arrays of libopus).
// Arrays of the serial SILK stages (NLSF decoding and NLSF2A, inverse
// prediction gain, pulse counts and the shell split tree).  Every lane of a
// group computes the same values, so they live once per group in the decoder
// slot rather than once per lane on the stack.
struct SilkWork {
    int32_t A[16];                                        // silk_lpc_inv_pred_gain
    int32_t cos_LSF_QA[16], P[9], Q[9], a32_QA1[16];      // silk_nlsf2a
    int16_t ec_ix[16], res_Q10[16];                       // NLSF unpack / residuals
    uint8_t pred_Q8[16];
    int16_t pNLSF_Q15[16], pNLSF0_Q15[16];                // silk_decode_parameters
    int32_t sum_pulses[20], nLshifts[20];                 // silk_decode_pulses
    int16_t shell[14];                                    // shell split tree walk: stack
    uint8_t sign_icdf[2];
};

struct SilkScratch {
    SilkWork sw;
    int16_t pulses[SILK_MAX_FRAME + 16];
    int16_t lbrr_pulses[SILK_MAX_FRAME + 16];
    int16_t sLTP[SILK_MAX_FRAME];
    int32_t sLTP_Q15[2 * SILK_MAX_FRAME];
    int32_t res_Q14[SILK_MAX_SUBFR_LEN];
    int32_t sLPC_Q14[SILK_MAX_SUBFR_LEN + 16];
    int16_t tmp[2][SILK_MAX_FRAME + 2];        // samplesOut1_tmp of silk_Decode
    int16_t rs_out[960];                      // samplesOut2_tmp (stereo interleave staging)
    int16_t rs_buf[2 * 160 + 8];              // IIR_FIR work buffer
    int32_t CNG_sig_Q14[SILK_MAX_FRAME + 16];
    int16_t plc_exc[2 * SILK_MAX_SUBFR_LEN];
    SilkCtrl ctrl;
};

// ------------------------------------------------------------------ tables by context

DFN const uint8_t *silk_pitch_contour_tab(int fs_kHz, int nb_subfr)
{
    if (fs_kHz == 8) return nb_subfr == 4 ? T_silk_pitch_contour_NB_iCDF : T_silk_pitch_contour_10_ms_NB_iCDF;
    return nb_subfr == 4 ? T_silk_pitch_contour_iCDF : T_silk_pitch_contour_10_ms_iCDF;
}
DFN const uint8_t *silk_pitch_lowbits_tab(int fs_kHz)
{
    return fs_kHz == 16 ? T_silk_uniform8_iCDF : (fs_kHz == 12 ? T_silk_uniform6_iCDF : T_silk_uniform4_iCDF);
}

struct NlsfCB {
    int nVectors, order, quantStepSize_Q16;
    const uint8_t *CB1_NLSF_Q8;
    const int16_t *CB1_Wght_Q9;
    const uint8_t *CB1_iCDF, *pred_Q8, *ec_sel, *ec_iCDF;
    const int16_t *deltaMin_Q15;
};
DFN NlsfCB silk_nlsf_cb(int order)
{
    NlsfCB c;
    if (order == 16) {
        c.nVectors = T_NLSF_WB_NVECTORS; c.order = 16; c.quantStepSize_Q16 = T_NLSF_WB_QSTEP_Q16;
        c.CB1_NLSF_Q8 = T_NLSF_WB_CB1_Q8; c.CB1_Wght_Q9 = T_NLSF_WB_CB1_Wght_Q9;
        c.CB1_iCDF = T_NLSF_WB_CB1_iCDF; c.pred_Q8 = T_NLSF_WB_pred_Q8; c.ec_sel = T_NLSF_WB_ec_sel;
        c.ec_iCDF = T_NLSF_WB_ec_iCDF; c.deltaMin_Q15 = T_NLSF_WB_deltaMin_Q15;
    } else {
        c.nVectors = T_NLSF_NB_MB_NVECTORS; c.order = 10; c.quantStepSize_Q16 = T_NLSF_NB_MB_QSTEP_Q16;
        c.CB1_NLSF_Q8 = T_NLSF_NB_MB_CB1_Q8; c.CB1_Wght_Q9 = T_NLSF_NB_MB_CB1_Wght_Q9;
        c.CB1_iCDF = T_NLSF_NB_MB_CB1_iCDF; c.pred_Q8 = T_NLSF_NB_MB_pred_Q8;
        c.ec_sel = T_NLSF_NB_MB_ec_sel; c.ec_iCDF = T_NLSF_NB_MB_ec_iCDF;
        c.deltaMin_Q15 = T_NLSF_NB_MB_deltaMin_Q15;
    }
    return c;
}

// ------------------------------------------------------------------ resampler

// silk_resampler_init(S, Fs_in, 48000, forEnc=0) for Fs_in in {8000,12000,16000}
DNI void silk_resampler_init48(SilkResampler *S, int32_t Fs_Hz_in)
{
    memset(S, 0, sizeof(*S));
    // delay_matrix_dec row for the input rate, column for 48 kHz
    S->inputDelay = (int16_t)(Fs_Hz_in == 8000 ? 0 : (Fs_Hz_in == 12000 ? 4 : 7));
    S->Fs_in_kHz = (int16_t)(Fs_Hz_in / 1000);
    S->Fs_out_kHz = 48;
    S->batchSize = (int16_t)(S->Fs_in_kHz * 10);
    // IIR_FIR with 2x up-sampling: invRatio = ((Fs_in << 15) / Fs_out) << 2, rounded up
    int32_t inv = shl32((int32_t)(((int64_t)Fs_Hz_in << 15) / 48000), 2);
    while (s_smulww(inv, 48000) < shl32(Fs_Hz_in, 1)) inv++;
    S->invRatio_Q16 = inv;
}

// silk/resampler_private_up2_HQ.c: 2x up-sampling by two 3-stage all-pass chains
// The even and the odd outputs come from two all-pass cascades that share
// only the input (states S[0..2] and S[3..5]), so two lanes run one cascade
// each; a group of one lane runs them one after the other.
DNI void silk_up2_hq(Lanes L, int32_t *S, int16_t *out, const int16_t *in, int32_t len)
{
    const int step = L.n > 1 ? 2 : 1;
    for (int ph = L.n > 1 ? L.id : 0; ph < 2; ph += step) {
        const int16_t *a = ph ? T_silk_resampler_up2_hq_1 : T_silk_resampler_up2_hq_0;
        int32_t s0 = S[3 * ph], s1 = S[3 * ph + 1], s2 = S[3 * ph + 2];
        for (int32_t k = 0; k < len; k++) {
            int32_t in32 = shl32((int32_t)in[k], 10), Y, X, o1, o2;
            Y = wsub(in32, s0); X = s_smulwb(Y, a[0]); o1 = wadd(s0, X); s0 = wadd(in32, X);
            Y = wsub(o1, s1); X = s_smulwb(Y, a[1]); o2 = wadd(s1, X); s1 = wadd(o1, X);
            Y = wsub(o2, s2); X = s_smlawb(Y, Y, a[2]); o1 = wadd(s2, X); s2 = wadd(o2, X);
            out[2 * k + ph] = (int16_t)s_sat16(s_rshift_round(o1, 10));
        }
        S[3 * ph] = s0; S[3 * ph + 1] = s1; S[3 * ph + 2] = s2;
    }
    lsync(L);
}

// silk/resampler_private_IIR_FIR.c; the FIR interpolation is split over lanes
DNI int16_t *silk_iir_fir(Lanes L, SilkResampler *S, int16_t *out, const int16_t *in,
                          int32_t inLen, int16_t *buf)
{
    LFOR(L, i, 0, 8) buf[i] = S->sFIR[i];
    lsync(L);
    const int32_t inc = S->invRatio_Q16;
    int32_t nIn = 0;
    while (1) {
        nIn = inLen < S->batchSize ? inLen : S->batchSize;
        silk_up2_hq(L, S->sIIR, &buf[8], in, nIn);
        lsync(L);
        int32_t max_index_Q16 = shl32(nIn, 17);
        int32_t nOut = (max_index_Q16 + inc - 1) / inc;
        LFOR(L, o, 0, nOut) {
            int32_t index_Q16 = o * inc;
            int32_t ti = s_smulwb(index_Q16 & 0xFFFF, 12);
            const int16_t *bp = &buf[index_Q16 >> 16];
            const int16_t *fa = &T_silk_resampler_frac_FIR_12[ti * 4];
            const int16_t *fb = &T_silk_resampler_frac_FIR_12[(11 - ti) * 4];
            int32_t r = s_smulbb(bp[0], fa[0]);
            r = s_smlabb(r, bp[1], fa[1]);
            r = s_smlabb(r, bp[2], fa[2]);
            r = s_smlabb(r, bp[3], fa[3]);
            r = s_smlabb(r, bp[4], fb[3]);
            r = s_smlabb(r, bp[5], fb[2]);
            r = s_smlabb(r, bp[6], fb[1]);
            r = s_smlabb(r, bp[7], fb[0]);
            out[o] = (int16_t)s_sat16(s_rshift_round(r, 15));
        }
        out += nOut;
        lsync(L);
        in += nIn;
        inLen -= nIn;
        if (inLen > 0) {
            int16_t keep[8];
            for (int i = 0; i < 8; i++) keep[i] = buf[(nIn << 1) + i];
            lsync(L);
            LFOR(L, i, 0, 8) buf[i] = keep[i];
            lsync(L);
        } else {
            break;
        }
    }
    for (int i = 0; i < 8; i++) S->sFIR[i] = buf[(nIn << 1) + i];
    lsync(L);
    return out;
}

// silk/resampler.c silk_resampler (IIR_FIR case)
DNI void silk_resample(Lanes L, SilkResampler *S, int16_t *out, const int16_t *in,
                       int32_t inLen, int16_t *buf)
{
    int nSamples = S->Fs_in_kHz - S->inputDelay;
    LFOR(L, i, 0, nSamples) S->delayBuf[S->inputDelay + i] = in[i];
    lsync(L);
    silk_iir_fir(L, S, out, S->delayBuf, S->Fs_in_kHz, buf);
    silk_iir_fir(L, S, &out[S->Fs_out_kHz], &in[nSamples], inLen - S->Fs_in_kHz, buf);
    LFOR(L, i, 0, S->inputDelay) S->delayBuf[i] = in[inLen - S->inputDelay + i];
    lsync(L);
}

// ------------------------------------------------------------------ LPC helpers

DFN void silk_bwexpander(int16_t *ar, int d, int32_t chirp_Q16)
{
    int32_t cm1 = chirp_Q16 - 65536;
    for (int i = 0; i < d - 1; i++) {
        ar[i] = (int16_t)s_rshift_round(wmul(chirp_Q16, ar[i]), 16);
        chirp_Q16 += s_rshift_round(wmul(chirp_Q16, cm1), 16);
    }
    ar[d - 1] = (int16_t)s_rshift_round(wmul(chirp_Q16, ar[d - 1]), 16);
}

DFN void silk_bwexpander_32(int32_t *ar, int d, int32_t chirp_Q16)
{
    int32_t cm1 = chirp_Q16 - 65536;
    for (int i = 0; i < d - 1; i++) {
        ar[i] = s_smulww(chirp_Q16, ar[i]);
        chirp_Q16 += s_rshift_round(wmul(chirp_Q16, cm1), 16);
    }
    ar[d - 1] = s_smulww(chirp_Q16, ar[d - 1]);
}

// silk/LPC_inv_pred_gain.c (QA = 24); returns 0 when the filter is unstable
DNI int32_t silk_lpc_inv_pred_gain(const int16_t *A_Q12, int order, int32_t *A)
{
    const int32_t A_LIMIT = 16773022;   // SILK_FIX_CONST(0.99975, 24)
    const int32_t MIN_INVG = 107374;    // SILK_FIX_CONST(1 / MAX_PREDICTION_POWER_GAIN, 30)
    int32_t DC = 0;
    for (int k = 0; k < order; k++) {
        DC += A_Q12[k];
        A[k] = shl32((int32_t)A_Q12[k], 12);
    }
    if (DC >= 4096) return 0;
    int32_t invGain_Q30 = 1 << 30;
    int k;
    for (k = order - 1; k > 0; k--) {
        if (A[k] > A_LIMIT || A[k] < -A_LIMIT) return 0;
        int32_t rc_Q31 = -shl32(A[k], 7);
        int32_t rc_mult1_Q30 = (1 << 30) - s_smmul(rc_Q31, rc_Q31);
        invGain_Q30 = shl32(s_smmul(invGain_Q30, rc_mult1_Q30), 2);
        if (invGain_Q30 < MIN_INVG) return 0;
        int mult2Q = 32 - s_clz32(s_abs(rc_mult1_Q30));
        int32_t rc_mult2 = s_inverse32_varq(rc_mult1_Q30, mult2Q + 30);
        for (int n = 0; n < (k + 1) >> 1; n++) {
            int32_t t1 = A[n], t2 = A[k - n - 1];
            int64_t v = s_rshift_round64(s_smull(s_sub_sat32(t1,
                (int32_t)s_rshift_round64(s_smull(t2, rc_Q31), 31)), rc_mult2), mult2Q);
            if (v > 2147483647LL || v < -2147483648LL) return 0;
            A[n] = (int32_t)v;
            v = s_rshift_round64(s_smull(s_sub_sat32(t2,
                (int32_t)s_rshift_round64(s_smull(t1, rc_Q31), 31)), rc_mult2), mult2Q);
            if (v > 2147483647LL || v < -2147483648LL) return 0;
            A[k - n - 1] = (int32_t)v;
        }
    }
    if (A[k] > A_LIMIT || A[k] < -A_LIMIT) return 0;
    int32_t rc_Q31 = -shl32(A[0], 7);
    int32_t rc_mult1_Q30 = (1 << 30) - s_smmul(rc_Q31, rc_Q31);
    invGain_Q30 = shl32(s_smmul(invGain_Q30, rc_mult1_Q30), 2);
    if (invGain_Q30 < MIN_INVG) return 0;
    return invGain_Q30;
}

// silk/LPC_fit.c
DNI void silk_lpc_fit(int16_t *a_QOUT, int32_t *a_QIN, int QOUT, int QIN, int d)
{
    int i, k, idx = 0;
    for (i = 0; i < 10; i++) {
        int32_t maxabs = 0;
        for (k = 0; k < d; k++) {
            int32_t absval = s_abs(a_QIN[k]);
            if (absval > maxabs) { maxabs = absval; idx = k; }
        }
        maxabs = s_rshift_round(maxabs, QIN - QOUT);
        if (maxabs > 32767) {
            maxabs = maxabs < 163838 ? maxabs : 163838;
            int32_t chirp_Q16 = 65470 - shl32(maxabs - 32767, 14) / ((wmul(maxabs, idx + 1)) >> 2);
            silk_bwexpander_32(a_QIN, d, chirp_Q16);
        } else {
            break;
        }
    }
    if (i == 10) {
        for (k = 0; k < d; k++) {
            a_QOUT[k] = (int16_t)s_sat16(s_rshift_round(a_QIN[k], QIN - QOUT));
            a_QIN[k] = shl32((int32_t)a_QOUT[k], QIN - QOUT);
        }
    } else {
        for (k = 0; k < d; k++) a_QOUT[k] = (int16_t)s_rshift_round(a_QIN[k], QIN - QOUT);
    }
}

// silk/NLSF2A.c (QA = 16): NLSF -> LPC via the P/Q polynomial expansion
DFN void silk_nlsf2a_poly(int32_t *out, const int32_t *cLSF, int dd)
{
    out[0] = 1 << 16;
    out[1] = -cLSF[0];
    for (int k = 1; k < dd; k++) {
        int32_t ftmp = cLSF[2 * k];
        out[k + 1] = wsub(shl32(out[k - 1], 1), (int32_t)s_rshift_round64(s_smull(ftmp, out[k]), 16));
        for (int n = k; n > 1; n--)
            out[n] = wadd(out[n], wsub(out[n - 2], (int32_t)s_rshift_round64(s_smull(ftmp, out[n - 1]), 16)));
        out[1] = wsub(out[1], ftmp);
    }
}

// ordering16 / ordering10 of silk/NLSF2A.c
TABC(uint8_t, T_nlsf2a_ord16[16]) = {0, 15, 8, 7, 4, 11, 12, 3, 2, 13, 10, 5, 6, 9, 14, 1};
TABC(uint8_t, T_nlsf2a_ord10[10]) = {0, 9, 6, 3, 4, 5, 8, 1, 2, 7};

DNI void silk_nlsf2a(int16_t *a_Q12, const int16_t *NLSF, int d, SilkWork *sw)
{
    const uint8_t *ordering = d == 16 ? T_nlsf2a_ord16 : T_nlsf2a_ord10;
    int32_t *cos_LSF_QA = sw->cos_LSF_QA, *P = sw->P, *Q = sw->Q, *a32_QA1 = sw->a32_QA1;
    for (int k = 0; k < d; k++) {
        int32_t f_int = NLSF[k] >> 8;
        int32_t f_frac = NLSF[k] - shl32(f_int, 8);
        int32_t cos_val = T_silk_LSFCosTab_FIX_Q12[f_int];
        int32_t delta = T_silk_LSFCosTab_FIX_Q12[f_int + 1] - cos_val;
        cos_LSF_QA[ordering[k]] = s_rshift_round(wadd(shl32(cos_val, 8), wmul(delta, f_frac)), 4);
    }
    int dd = d >> 1;
    silk_nlsf2a_poly(P, &cos_LSF_QA[0], dd);
    silk_nlsf2a_poly(Q, &cos_LSF_QA[1], dd);
    for (int k = 0; k < dd; k++) {
        int32_t Ptmp = wadd(P[k + 1], P[k]);
        int32_t Qtmp = wsub(Q[k + 1], Q[k]);
        a32_QA1[k] = wsub(-Qtmp, Ptmp);
        a32_QA1[d - k - 1] = wsub(Qtmp, Ptmp);
    }
    silk_lpc_fit(a_Q12, a32_QA1, 12, 17, d);
    for (int i = 0; silk_lpc_inv_pred_gain(a_Q12, d, sw->A) == 0 && i < 16; i++) {
        silk_bwexpander_32(a32_QA1, d, 65536 - shl32(2, i));
        for (int k = 0; k < d; k++) a_Q12[k] = (int16_t)s_rshift_round(a32_QA1[k], 5);
    }
}

// silk/NLSF_stabilize.c (MAX_LOOPS 20) with the sort.c insertion sort fallback
DNI void silk_nlsf_stabilize(int16_t *NLSF_Q15, const int16_t *NDeltaMin_Q15, int L)
{
    int loops, I = 0;
    for (loops = 0; loops < 20; loops++) {
        int32_t min_diff = NLSF_Q15[0] - NDeltaMin_Q15[0];
        I = 0;
        for (int i = 1; i <= L - 1; i++) {
            int32_t diff = NLSF_Q15[i] - (NLSF_Q15[i - 1] + NDeltaMin_Q15[i]);
            if (diff < min_diff) { min_diff = diff; I = i; }
        }
        int32_t diff = (1 << 15) - (NLSF_Q15[L - 1] + NDeltaMin_Q15[L]);
        if (diff < min_diff) { min_diff = diff; I = L; }
        if (min_diff >= 0) return;
        if (I == 0) {
            NLSF_Q15[0] = NDeltaMin_Q15[0];
        } else if (I == L) {
            NLSF_Q15[L - 1] = (int16_t)((1 << 15) - NDeltaMin_Q15[L]);
        } else {
            int32_t min_center = 0;
            for (int k = 0; k < I; k++) min_center += NDeltaMin_Q15[k];
            min_center += NDeltaMin_Q15[I] >> 1;
            int32_t max_center = 1 << 15;
            for (int k = L; k > I; k--) max_center -= NDeltaMin_Q15[k];
            max_center -= NDeltaMin_Q15[I] >> 1;
            int16_t center = (int16_t)s_limit(s_rshift_round((int32_t)NLSF_Q15[I - 1] + (int32_t)NLSF_Q15[I], 1),
                                              min_center, max_center);
            NLSF_Q15[I - 1] = (int16_t)(center - (NDeltaMin_Q15[I] >> 1));
            NLSF_Q15[I] = (int16_t)(NLSF_Q15[I - 1] + NDeltaMin_Q15[I]);
        }
    }
    if (loops == 20) {
        for (int i = 1; i < L; i++) {
            int value = NLSF_Q15[i], j;
            for (j = i - 1; j >= 0 && value < NLSF_Q15[j]; j--) NLSF_Q15[j + 1] = NLSF_Q15[j];
            NLSF_Q15[j + 1] = (int16_t)value;
        }
        NLSF_Q15[0] = (int16_t)imax(NLSF_Q15[0], NDeltaMin_Q15[0]);
        for (int i = 1; i < L; i++)
            NLSF_Q15[i] = (int16_t)imax(NLSF_Q15[i], (int16_t)s_sat16(NLSF_Q15[i - 1] + NDeltaMin_Q15[i]));
        NLSF_Q15[L - 1] = (int16_t)imin(NLSF_Q15[L - 1], (1 << 15) - NDeltaMin_Q15[L]);
        for (int i = L - 2; i >= 0; i--)
            NLSF_Q15[i] = (int16_t)imin(NLSF_Q15[i], NLSF_Q15[i + 1] - NDeltaMin_Q15[i + 1]);
    }
}

DFN void silk_nlsf_unpack(int16_t *ec_ix, uint8_t *pred_Q8, const NlsfCB &cb, int CB1_index)
{
    const uint8_t *sel = &cb.ec_sel[CB1_index * cb.order / 2];
    for (int i = 0; i < cb.order; i += 2) {
        uint8_t entry = *sel++;
        ec_ix[i] = (int16_t)(((entry >> 1) & 7) * 9);
        pred_Q8[i] = cb.pred_Q8[i + (entry & 1) * (cb.order - 1)];
        ec_ix[i + 1] = (int16_t)(((entry >> 5) & 7) * 9);
        pred_Q8[i + 1] = cb.pred_Q8[i + ((entry >> 4) & 1) * (cb.order - 1) + 1];
    }
}

// silk/NLSF_decode.c
DNI void silk_nlsf_decode(int16_t *pNLSF_Q15, const int8_t *NLSFIndices, const NlsfCB &cb, SilkWork *sw)
{
    uint8_t *pred_Q8 = sw->pred_Q8;
    int16_t *ec_ix = sw->ec_ix, *res_Q10 = sw->res_Q10;
    silk_nlsf_unpack(ec_ix, pred_Q8, cb, NLSFIndices[0]);
    int32_t out_Q10 = 0;
    for (int i = cb.order - 1; i >= 0; i--) {
        int32_t pred_Q10 = s_smulbb(out_Q10, (int16_t)pred_Q8[i]) >> 8;
        out_Q10 = shl32(NLSFIndices[i + 1], 10);
        if (out_Q10 > 0) out_Q10 -= 102;            // SILK_FIX_CONST(NLSF_QUANT_LEVEL_ADJ, 10)
        else if (out_Q10 < 0) out_Q10 += 102;
        out_Q10 = s_smlawb(pred_Q10, out_Q10, cb.quantStepSize_Q16);
        res_Q10[i] = (int16_t)out_Q10;
    }
    const uint8_t *el = &cb.CB1_NLSF_Q8[NLSFIndices[0] * cb.order];
    const int16_t *w = &cb.CB1_Wght_Q9[NLSFIndices[0] * cb.order];
    for (int i = 0; i < cb.order; i++) {
        int32_t t = wadd(shl32((int32_t)res_Q10[i], 14) / w[i], shl32((int16_t)el[i], 7));
        pNLSF_Q15[i] = (int16_t)s_limit(t, 0, 32767);
    }
    silk_nlsf_stabilize(pNLSF_Q15, cb.deltaMin_Q15, cb.order);
}

// silk/LPC_analysis_filter.c, split over lanes (each output is independent)
DNI void silk_lpc_analysis_filter(Lanes L, int16_t *out, const int16_t *in,
                                  const int16_t *B, int32_t len, int32_t d)
{
    LFOR(L, ix, d, len) {
        const int16_t *ip = &in[ix - 1];
        int32_t acc = s_smulbb(ip[0], B[0]);
        for (int j = 1; j < d; j++) acc = s_smlabb(acc, ip[-j], B[j]);
        acc = wsub(shl32((int32_t)ip[1], 12), acc);
        out[ix] = (int16_t)s_sat16(s_rshift_round(acc, 12));
    }
    LFOR(L, j, 0, d) out[j] = 0;
    lsync(L);
}

// silk/sum_sqr_shift.c
DNI void silk_sum_sqr_shift(int32_t *energy, int *shift, const int16_t *x, int len)
{
    int i, shft = 31 - s_clz32(len);
    int32_t nrg = len;
    for (i = 0; i < len - 1; i += 2) {
        uint32_t t = (uint32_t)s_smulbb(x[i], x[i]);
        t = (uint32_t)s_smlabb((int32_t)t, x[i + 1], x[i + 1]);
        nrg = (int32_t)((uint32_t)nrg + (t >> shft));
    }
    if (i < len) nrg = (int32_t)((uint32_t)nrg + ((uint32_t)s_smulbb(x[i], x[i]) >> shft));
    shft = imax(0, shft + 3 - s_clz32(nrg));
    nrg = 0;
    for (i = 0; i < len - 1; i += 2) {
        uint32_t t = (uint32_t)s_smulbb(x[i], x[i]);
        t = (uint32_t)s_smlabb((int32_t)t, x[i + 1], x[i + 1]);
        nrg = (int32_t)((uint32_t)nrg + (t >> shft));
    }
    if (i < len) nrg = (int32_t)((uint32_t)nrg + ((uint32_t)s_smulbb(x[i], x[i]) >> shft));
    *shift = shft;
    *energy = nrg;
}

// ------------------------------------------------------------------ state init

DFN void silk_cng_reset(SilkChan *c)
{
    int32_t step = 32767 / (c->LPC_order + 1), acc = 0;
    for (int i = 0; i < c->LPC_order; i++) {
        acc += step;
        c->sCNG.CNG_smth_NLSF_Q15[i] = (int16_t)acc;
    }
    c->sCNG.CNG_smth_Gain_Q16 = 0;
    c->sCNG.rand_seed = 3176576;
}

DFN void silk_plc_reset(SilkChan *c)
{
    c->sPLC.pitchL_Q8 = shl32(c->frame_length, 7);
    c->sPLC.prevGain_Q16[0] = 65536;
    c->sPLC.prevGain_Q16[1] = 65536;
    c->sPLC.subfr_length = 20;
    c->sPLC.nb_subfr = 2;
}

// silk_reset_decoder: clear from prev_gain_Q16 onwards
DNI void silk_reset_chan(SilkChan *c)
{
    memset(c, 0, sizeof(*c));
    c->first_frame_after_reset = 1;
    c->prev_gain_Q16 = 65536;
    silk_cng_reset(c);
    silk_plc_reset(c);
}

DFN void silk_init_dec(SilkDec *d)
{
    silk_reset_chan(&d->ch[0]);
    silk_reset_chan(&d->ch[1]);
    memset(&d->sStereo, 0, sizeof(d->sStereo));
    d->prev_decode_only_middle = 0;
    d->nChannelsAPI = 0;
    d->nChannelsInternal = 0;
}

// silk_ResetDecoder: like init, but silk_reset_decoder keeps nothing before
// prev_gain_Q16, which is the start of the state here as well
DFN void silk_reset_dec(SilkDec *d)
{
    silk_reset_chan(&d->ch[0]);
    silk_reset_chan(&d->ch[1]);
    memset(&d->sStereo, 0, sizeof(d->sStereo));
    d->prev_decode_only_middle = 0;
}

// silk/decoder_set_fs.c with API rate 48 kHz
DNI void silk_decoder_set_fs(SilkChan *c, int fs_kHz, int32_t fs_API_Hz)
{
    c->subfr_length = 5 * fs_kHz;
    int frame_length = c->nb_subfr * c->subfr_length;
    if (c->fs_kHz != fs_kHz || c->fs_API_hz != fs_API_Hz) {
        silk_resampler_init48(&c->resampler_state, fs_kHz * 1000);
        c->fs_API_hz = fs_API_Hz;
    }
    if (c->fs_kHz != fs_kHz || frame_length != c->frame_length) {
        if (c->fs_kHz != fs_kHz) {
            c->ltp_mem_length = 20 * fs_kHz;
            c->LPC_order = (fs_kHz == 8 || fs_kHz == 12) ? 10 : 16;
            c->first_frame_after_reset = 1;
            c->lagPrev = 100;
            c->LastGainIndex = 10;
            c->prevSignalType = SIG_NO_VOICE;
            memset(c->outBuf, 0, sizeof(c->outBuf));
            memset(c->sLPC_Q14_buf, 0, sizeof(c->sLPC_Q14_buf));
        }
        c->fs_kHz = fs_kHz;
        c->frame_length = frame_length;
    }
}

// ------------------------------------------------------------------ entropy decoding

DNI void silk_decode_indices(SilkChan *c, RangeDec *rd, int FrameIndex, int decode_LBRR, int condCoding,
                             SilkWork *sw)
{
    SilkIndices *ix = &c->indices;
    int Ix;
    if (decode_LBRR || c->VAD_flags[FrameIndex]) Ix = rd_icdf(rd, T_silk_type_offset_VAD_iCDF, 8) + 2;
    else Ix = rd_icdf(rd, T_silk_type_offset_no_VAD_iCDF, 8);
    ix->signalType = (int8_t)(Ix >> 1);
    ix->quantOffsetType = (int8_t)(Ix & 1);

    if (condCoding == CODE_COND) {
        ix->GainsIndices[0] = (int8_t)rd_icdf(rd, T_silk_delta_gain_iCDF, 8);
    } else {
        ix->GainsIndices[0] = (int8_t)shl32(rd_icdf(rd, &T_silk_gain_iCDF[ix->signalType * 8], 8), 3);
        ix->GainsIndices[0] = (int8_t)(ix->GainsIndices[0] + rd_icdf(rd, T_silk_uniform8_iCDF, 8));
    }
    for (int i = 1; i < c->nb_subfr; i++) ix->GainsIndices[i] = (int8_t)rd_icdf(rd, T_silk_delta_gain_iCDF, 8);

    NlsfCB cb = silk_nlsf_cb(c->LPC_order);
    ix->NLSFIndices[0] = (int8_t)rd_icdf(rd, &cb.CB1_iCDF[(ix->signalType >> 1) * cb.nVectors], 8);
    int16_t *ec_ix = sw->ec_ix;
    silk_nlsf_unpack(ec_ix, sw->pred_Q8, cb, ix->NLSFIndices[0]);
    for (int i = 0; i < cb.order; i++) {
        Ix = rd_icdf(rd, &cb.ec_iCDF[ec_ix[i]], 8);
        if (Ix == 0) Ix -= rd_icdf(rd, T_silk_NLSF_EXT_iCDF, 8);
        else if (Ix == 8) Ix += rd_icdf(rd, T_silk_NLSF_EXT_iCDF, 8);
        ix->NLSFIndices[i + 1] = (int8_t)(Ix - 4);
    }
    if (c->nb_subfr == 4) ix->NLSFInterpCoef_Q2 = (int8_t)rd_icdf(rd, T_silk_NLSF_interpolation_factor_iCDF, 8);
    else ix->NLSFInterpCoef_Q2 = 4;

    if (ix->signalType == SIG_VOICED) {
        int decode_abs = 1;
        if (condCoding == CODE_COND && c->ec_prevSignalType == SIG_VOICED) {
            int delta = (int16_t)rd_icdf(rd, T_silk_pitch_delta_iCDF, 8);
            if (delta > 0) {
                delta = delta - 9;
                ix->lagIndex = (int16_t)(c->ec_prevLagIndex + delta);
                decode_abs = 0;
            }
        }
        if (decode_abs) {
            ix->lagIndex = (int16_t)(rd_icdf(rd, T_silk_pitch_lag_iCDF, 8) * (c->fs_kHz >> 1));
            ix->lagIndex = (int16_t)(ix->lagIndex + rd_icdf(rd, silk_pitch_lowbits_tab(c->fs_kHz), 8));
        }
        c->ec_prevLagIndex = ix->lagIndex;
        ix->contourIndex = (int8_t)rd_icdf(rd, silk_pitch_contour_tab(c->fs_kHz, c->nb_subfr), 8);
        ix->PERIndex = (int8_t)rd_icdf(rd, T_silk_LTP_per_index_iCDF, 8);
        const uint8_t *gt = ix->PERIndex == 0 ? T_silk_LTP_gain_iCDF_0
                          : (ix->PERIndex == 1 ? T_silk_LTP_gain_iCDF_1 : T_silk_LTP_gain_iCDF_2);
        for (int k = 0; k < c->nb_subfr; k++) ix->LTPIndex[k] = (int8_t)rd_icdf(rd, gt, 8);
        if (condCoding == CODE_INDEP) ix->LTP_scaleIndex = (int8_t)rd_icdf(rd, T_silk_LTPscale_iCDF, 8);
        else ix->LTP_scaleIndex = 0;
    }
    c->ec_prevSignalType = ix->signalType;
    ix->Seed = (int8_t)rd_icdf(rd, T_silk_uniform4_iCDF, 8);
}

// silk/shell_coder.c silk_shell_decoder: a binary split tree over 16 pulses.
// libopus unrolls the tree; here one loop walks it depth first, left half
// before right half, which reads the splits in the same order.  A node at
// level L (3 = the root) holds the pulse count of 2^(L+1) positions; its split
// gives the left child's count from the level-L table, the right child gets
// the rest.  `tree` is scratch for the walk's stack (8 entries).
DNI void silk_shell_decoder(int16_t *p0, RangeDec *rd, int pulses4, int16_t *tree)
{
    int sp = 0;
    tree[sp++] = (int16_t)(pulses4 | 3 << 5);                 // count | level << 5 | first position << 8
    while (sp > 0) {
        int node = tree[--sp];
        int p = node & 31, lvl = (node >> 5) & 3, pos = node >> 8;
        int left = 0;
        if (p > 0) {
            const uint8_t *t = lvl == 3 ? T_silk_shell_code_table3
                             : lvl == 2 ? T_silk_shell_code_table2
                             : lvl == 1 ? T_silk_shell_code_table1 : T_silk_shell_code_table0;
            left = rd_icdf(rd, &t[T_silk_shell_code_table_offsets[p]], 8);
        }
        int right = p - left;
        if (lvl == 0) {
            p0[pos] = (int16_t)left;
            p0[pos + 1] = (int16_t)right;
        } else {
            int half = 1 << lvl;                                  // positions under each child
            tree[sp++] = (int16_t)(right | (lvl - 1) << 5 | (pos + half) << 8);
            tree[sp++] = (int16_t)(left | (lvl - 1) << 5 | pos << 8);
        }
    }
}

// silk/decode_pulses.c + code_signs.c silk_decode_signs
DNI void silk_decode_pulses(RangeDec *rd, int16_t *pulses, int signalType, int quantOffsetType,
                            int frame_length, SilkWork *sw)
{
    int32_t *sum_pulses = sw->sum_pulses, *nLshifts = sw->nLshifts;
    int RateLevelIndex = rd_icdf(rd, &T_silk_rate_levels_iCDF[(signalType >> 1) * 9], 8);
    int iter = frame_length >> 4;
    if (iter * 16 < frame_length) iter++;
    const uint8_t *cdf = &T_silk_pulses_per_block_iCDF[RateLevelIndex * 18];
    for (int i = 0; i < iter; i++) {
        nLshifts[i] = 0;
        sum_pulses[i] = rd_icdf(rd, cdf, 8);
        while (sum_pulses[i] == 17) {
            nLshifts[i]++;
            sum_pulses[i] = rd_icdf(rd, &T_silk_pulses_per_block_iCDF[9 * 18] + (nLshifts[i] == 10), 8);
        }
    }
    for (int i = 0; i < iter; i++) {
        if (sum_pulses[i] > 0) {
            PHASE_BEGIN(t_sh);
            silk_shell_decoder(&pulses[i * 16], rd, sum_pulses[i], sw->shell);
            PHASE_END(PH_SILK_SHELL, t_sh, 0);
        }
        else for (int k = 0; k < 16; k++) pulses[i * 16 + k] = 0;
    }
    for (int i = 0; i < iter; i++) {
        if (nLshifts[i] > 0) {
            int nLS = nLshifts[i];
            int16_t *pp = &pulses[i * 16];
            for (int k = 0; k < 16; k++) {
                int abs_q = pp[k];
                for (int j = 0; j < nLS; j++) {
                    abs_q = shl32(abs_q, 1);
                    abs_q += rd_icdf(rd, T_silk_lsb_iCDF, 8);
                }
                pp[k] = (int16_t)abs_q;
            }
            sum_pulses[i] |= nLS << 5;
        }
    }
    // signs
    uint8_t *icdf = sw->sign_icdf;
    icdf[1] = 0;
    const uint8_t *icdf_ptr = &T_silk_sign_iCDF[7 * (quantOffsetType + (signalType << 1))];
    int len = (frame_length + 8) >> 4;
    int16_t *q = pulses;
    for (int i = 0; i < len; i++) {
        int p = sum_pulses[i];
        if (p > 0) {
            icdf[0] = icdf_ptr[imin(p & 0x1F, 6)];
            for (int j = 0; j < 16; j++)
                if (q[j] > 0) q[j] = (int16_t)(q[j] * (shl32(rd_icdf(rd, icdf, 8), 1) - 1));
        }
        q += 16;
    }
}

// silk/stereo_decode_pred.c
DNI void silk_stereo_decode_pred(RangeDec *rd, int32_t *pred_Q13)
{
    int ix[2][3];
    int n = rd_icdf(rd, T_silk_stereo_pred_joint_iCDF, 8);
    ix[0][2] = n / 5;
    ix[1][2] = n - 5 * ix[0][2];
    for (n = 0; n < 2; n++) {
        ix[n][0] = rd_icdf(rd, T_silk_uniform3_iCDF, 8);
        ix[n][1] = rd_icdf(rd, T_silk_uniform5_iCDF, 8);
    }
    for (n = 0; n < 2; n++) {
        ix[n][0] += 3 * ix[n][2];
        int32_t low = T_silk_stereo_pred_quant_Q13[ix[n][0]];
        int32_t step = s_smulwb(T_silk_stereo_pred_quant_Q13[ix[n][0] + 1] - low, 6554);
        pred_Q13[n] = s_smlabb(low, step, 2 * ix[n][1] + 1);
    }
    pred_Q13[0] -= pred_Q13[1];
}

// ------------------------------------------------------------------ parameters

DNI void silk_decode_pitch(int lagIndex, int contourIndex, int32_t *pitch_lags, int Fs_kHz, int nb_subfr)
{
    const int8_t *cb;
    int cbk_size;
    if (Fs_kHz == 8) {
        if (nb_subfr == 4) { cb = T_silk_CB_lags_stage2; cbk_size = T_SILK_PE_NB_CBKS_STAGE2_EXT; }
        else { cb = T_silk_CB_lags_stage2_10_ms; cbk_size = T_SILK_PE_NB_CBKS_STAGE2_10MS; }
    } else {
        if (nb_subfr == 4) { cb = T_silk_CB_lags_stage3; cbk_size = T_SILK_PE_NB_CBKS_STAGE3_MAX; }
        else { cb = T_silk_CB_lags_stage3_10_ms; cbk_size = T_SILK_PE_NB_CBKS_STAGE3_10MS; }
    }
    int min_lag = 2 * Fs_kHz, max_lag = 18 * Fs_kHz;
    int lag = min_lag + lagIndex;
    for (int k = 0; k < nb_subfr; k++) {
        pitch_lags[k] = lag + cb[k * cbk_size + contourIndex];
        pitch_lags[k] = s_limit(pitch_lags[k], min_lag, max_lag);
    }
}

DNI void silk_gains_dequant(int32_t *gain_Q16, const int8_t *ind, int32_t *prev_ind, int conditional,
                            int nb_subfr)
{
    for (int k = 0; k < nb_subfr; k++) {
        if (k == 0 && conditional == 0) {
            *prev_ind = imax(ind[k], *prev_ind - 16);
        } else {
            int ind_tmp = ind[k] - 4;
            int thr = 2 * 36 - 64 + *prev_ind;
            if (ind_tmp > thr) *prev_ind += shl32(ind_tmp, 1) - thr;
            else *prev_ind += ind_tmp;
        }
        *prev_ind = s_limit(*prev_ind, 0, 63);
        // INV_SCALE_Q16 = 1907825, OFFSET = 2090
        gain_Q16[k] = s_log2lin(min32(s_smulwb(1907825, *prev_ind) + 2090, 3967));
    }
}

DNI void silk_decode_parameters(SilkChan *c, SilkCtrl *ctrl, int condCoding, SilkWork *sw)
{
    int16_t *pNLSF_Q15 = sw->pNLSF_Q15, *pNLSF0_Q15 = sw->pNLSF0_Q15;
    SilkIndices *ix = &c->indices;
    silk_gains_dequant(ctrl->Gains_Q16, ix->GainsIndices, &c->LastGainIndex, condCoding == CODE_COND,
                       c->nb_subfr);
    NlsfCB cb = silk_nlsf_cb(c->LPC_order);
    silk_nlsf_decode(pNLSF_Q15, ix->NLSFIndices, cb, sw);
    silk_nlsf2a(ctrl->PredCoef_Q12[1], pNLSF_Q15, c->LPC_order, sw);
    if (c->first_frame_after_reset == 1) ix->NLSFInterpCoef_Q2 = 4;
    if (ix->NLSFInterpCoef_Q2 < 4) {
        for (int i = 0; i < c->LPC_order; i++)
            pNLSF0_Q15[i] = (int16_t)(c->prevNLSF_Q15[i] +
                ((ix->NLSFInterpCoef_Q2 * (pNLSF_Q15[i] - c->prevNLSF_Q15[i])) >> 2));
        silk_nlsf2a(ctrl->PredCoef_Q12[0], pNLSF0_Q15, c->LPC_order, sw);
    } else {
        for (int i = 0; i < c->LPC_order; i++) ctrl->PredCoef_Q12[0][i] = ctrl->PredCoef_Q12[1][i];
    }
    for (int i = 0; i < c->LPC_order; i++) c->prevNLSF_Q15[i] = pNLSF_Q15[i];
    if (c->lossCnt) {
        silk_bwexpander(ctrl->PredCoef_Q12[0], c->LPC_order, 63570);
        silk_bwexpander(ctrl->PredCoef_Q12[1], c->LPC_order, 63570);
    }
    if (ix->signalType == SIG_VOICED) {
        silk_decode_pitch(ix->lagIndex, ix->contourIndex, ctrl->pitchL, c->fs_kHz, c->nb_subfr);
        const int8_t *cbk = ix->PERIndex == 0 ? T_silk_LTP_gain_vq_0
                          : (ix->PERIndex == 1 ? T_silk_LTP_gain_vq_1 : T_silk_LTP_gain_vq_2);
        for (int k = 0; k < c->nb_subfr; k++) {
            int I = ix->LTPIndex[k];
            for (int i = 0; i < 5; i++) ctrl->LTPCoef_Q14[k * 5 + i] = (int16_t)shl32(cbk[I * 5 + i], 7);
        }
        ctrl->LTP_scale_Q14 = T_silk_LTPScales_table_Q14[ix->LTP_scaleIndex];
    } else {
        for (int k = 0; k < c->nb_subfr; k++) ctrl->pitchL[k] = 0;
        for (int k = 0; k < 5 * c->nb_subfr; k++) ctrl->LTPCoef_Q14[k] = 0;
        ix->PERIndex = 0;
        ctrl->LTP_scale_Q14 = 0;
    }
}

// ------------------------------------------------------------------ synthesis

// silk/decode_core.c: excitation, LTP and LPC synthesis for one frame
DNI void silk_decode_core(Lanes L, SilkChan *c, SilkCtrl *ctrl, int16_t *xq, const int16_t *pulses,
                          SilkScratch *w)
{
    int16_t *sLTP = w->sLTP;
    int32_t *sLTP_Q15 = w->sLTP_Q15;
    const SilkIndices *ix = &c->indices;
    int32_t offset_Q10 = T_silk_Quantization_Offsets_Q10[(ix->signalType >> 1) * 2 + ix->quantOffsetType];
    int NLSF_interpolation_flag = ix->NLSFInterpCoef_Q2 < 4;

    // excitation.  Sample i's sign comes from an LCG seed that then advances
    // by the sample's pulse: t[i+1] = A (t[i] + p[i]) + B mod 2^32, an affine
    // recurrence.  Each lane takes a contiguous run of samples, composes its
    // run's maps, and a prefix composition over the lanes gives every run its
    // first seed -- the serial seeds exactly (modular arithmetic).
    {
        const uint32_t A = 196314165u, B = 907633515u;   // silk_RAND
        const int n = c->frame_length;
        const int run = (n + L.n - 1) / L.n;
        const int i0 = imin(n, L.id * run), i1 = imin(n, i0 + run);
        uint32_t ma = 1, mb = 0;
        for (int i = i0; i < i1; i++) {
            mb = A * (mb + (uint32_t)(int32_t)pulses[i]) + B;
            ma = A * ma;
        }
        lscan_affine(L, ma, mb);
        uint32_t t = ma * (uint32_t)s_rand(ix->Seed) + mb;
        for (int i = i0; i < i1; i++) {
            int32_t e = shl32((int32_t)pulses[i], 14);
            if (e > 0) e -= 80 << 4;
            else if (e < 0) e += 80 << 4;
            e += offset_Q10 << 4;
            if ((int32_t)t < 0) e = -e;
            c->exc_Q14[i] = e;
            t = A * (t + (uint32_t)(int32_t)pulses[i]) + B;
        }
        lsync(L);
    }
    // LPC synthesis history: the last 16 outputs, in registers (win[15] newest);
    // the previous subframe's gain, also in a register: both are written back
    // after the frame's last barrier
    int32_t prev_gain_Q16 = c->prev_gain_Q16;
    int32_t win[16];
#pragma unroll
    for (int t = 0; t < 16; t++) win[t] = c->sLPC_Q14_buf[t];
    const int32_t *pexc = c->exc_Q14;
    int16_t *pxq = xq;
    int sLTP_buf_idx = c->ltp_mem_length;
    int lag = 0;
    for (int k = 0; k < c->nb_subfr; k++) {
        const int32_t *pres;
        int16_t A_Q12[16];
        const int16_t *Acoef = ctrl->PredCoef_Q12[k >> 1];
        for (int i = 0; i < c->LPC_order; i++) A_Q12[i] = Acoef[i];
        int16_t *B_Q14 = &ctrl->LTPCoef_Q14[k * 5];
        int signalType = ix->signalType;
        int32_t Gain_Q10 = ctrl->Gains_Q16[k] >> 6;
        int32_t inv_gain_Q31 = s_inverse32_varq(ctrl->Gains_Q16[k], 47);
        int32_t gain_adj_Q16;
        if (ctrl->Gains_Q16[k] != prev_gain_Q16) {
            gain_adj_Q16 = s_div32_varq(prev_gain_Q16, ctrl->Gains_Q16[k], 16);
#pragma unroll
            for (int t = 0; t < 16; t++) win[t] = s_smulww(gain_adj_Q16, win[t]);
        } else {
            gain_adj_Q16 = 1 << 16;
        }
        prev_gain_Q16 = ctrl->Gains_Q16[k];
        if (c->lossCnt && c->prevSignalType == SIG_VOICED && ix->signalType != SIG_VOICED && k < 2) {
            for (int i = 0; i < 5; i++) B_Q14[i] = 0;
            B_Q14[2] = 4096;   // SILK_FIX_CONST(0.25, 14)
            signalType = SIG_VOICED;
            ctrl->pitchL[k] = c->lagPrev;
        }
        if (signalType == SIG_VOICED) {
            lag = ctrl->pitchL[k];
            if (k == 0 || (k == 2 && NLSF_interpolation_flag)) {
                int start_idx = c->ltp_mem_length - lag - c->LPC_order - 2;
                if (k == 2) {
                    LFOR(L, i, 0, 2 * c->subfr_length) c->outBuf[c->ltp_mem_length + i] = xq[i];
                    lsync(L);
                }
                silk_lpc_analysis_filter(L, &sLTP[start_idx], &c->outBuf[start_idx + k * c->subfr_length],
                                         A_Q12, c->ltp_mem_length - start_idx, c->LPC_order);
                if (k == 0) inv_gain_Q31 = shl32(s_smulwb(inv_gain_Q31, ctrl->LTP_scale_Q14), 2);
                LFOR(L, i, 0, lag + 2)
                    sLTP_Q15[sLTP_buf_idx - i - 1] = s_smulwb(inv_gain_Q31, sLTP[c->ltp_mem_length - i - 1]);
                lsync(L);
            } else if (gain_adj_Q16 != 1 << 16) {
                LFOR(L, i, 0, lag + 2)
                    sLTP_Q15[sLTP_buf_idx - i - 1] = s_smulww(gain_adj_Q16, sLTP_Q15[sLTP_buf_idx - i - 1]);
                lsync(L);
            }
        }
        int32_t *res = w->res_Q14;
        PHASE_BEGIN(t_ltp);
        if (signalType == SIG_VOICED) {
            // the 5-tap LTP reads samples at least lag - 2 back, so blocks of
            // lag - 2 outputs depend only on earlier blocks: lanes split a
            // block, blocks run in order
            const int32_t *pl = &sLTP_Q15[sLTP_buf_idx - lag + 2];
            const int blk = imax(lag - 2, 1);   // lag >= 16 in a valid stream
            for (int s0 = 0; s0 < c->subfr_length; s0 += blk) {
                int e0 = imin(s0 + blk, c->subfr_length);
                LFOR(L, i, s0, e0) {
                    int32_t p = 2;
                    p = s_smlawb(p, pl[i], B_Q14[0]);
                    p = s_smlawb(p, pl[i - 1], B_Q14[1]);
                    p = s_smlawb(p, pl[i - 2], B_Q14[2]);
                    p = s_smlawb(p, pl[i - 3], B_Q14[3]);
                    p = s_smlawb(p, pl[i - 4], B_Q14[4]);
                    int32_t r = wadd(pexc[i], shl32(p, 1));
                    res[i] = r;
                    sLTP_Q15[sLTP_buf_idx + i] = shl32(r, 1);
                }
                lsync(L);
            }
            sLTP_buf_idx += c->subfr_length;
            pres = res;
        } else {
            pres = pexc;
        }
        PHASE_END(PH_SILK_LTP, t_ltp, L.id);
        PHASE_BEGIN(t_lpc);
        // LPC synthesis: order-10/16 recursion per sample.  The prediction is
        // order/2 plus one truncated product per tap, summed with wrap-around
        // adds, so the sum may be taken in any order: the taps on samples
        // older than the newest one are summed while the newest sample is
        // still being computed, and only tap 0 stays on the recursion's path.
        const int order = c->LPC_order;
        int32_t pold = order >> 1;     // order/2 + taps 1.. on the current window
#pragma unroll
        for (int j = 1; j < 16; j++)
            if (j < order) pold = wadd(pold, s_smulwb(win[15 - j], A_Q12[j]));
        for (int i = 0; i < c->subfr_length; i++) {
            int32_t p = wadd(pold, s_smulwb(win[15], A_Q12[0]));
            // taps 1.. of the next sample read win[16 - j]: known already
            int32_t pa = order >> 1, pb = 0;
#pragma unroll
            for (int j = 1; j < 16; j += 2) {
                if (j < order) pa = wadd(pa, s_smulwb(win[16 - j], A_Q12[j]));
                if (j + 1 < order) pb = wadd(pb, s_smulwb(win[15 - j], A_Q12[j + 1]));
            }
            pold = wadd(pa, pb);
            int32_t v = s_add_sat32(pres[i], s_lshift_sat32(p, 4));
#pragma unroll
            for (int t = 0; t < 15; t++) win[t] = win[t + 1];
            win[15] = v;
            pxq[i] = (int16_t)s_sat16(s_rshift_round(s_smulww(v, Gain_Q10), 8));
        }
        pexc += c->subfr_length;
        pxq += c->subfr_length;
        PHASE_END(PH_SILK_LPC, t_lpc, L.id);
        lsync(L);   // the next subframe's LTP rewrites res_Q14, which this one's synthesis reads
    }
    lsync(L);
#pragma unroll
    for (int t = 0; t < 16; t++) c->sLPC_Q14_buf[t] = win[t];
    c->prev_gain_Q16 = prev_gain_Q16;
    lsync(L);
}

// ------------------------------------------------------------------ PLC

DNI void silk_plc_update(SilkChan *c, const SilkCtrl *ctrl)
{
    SilkPLC *p = &c->sPLC;
    c->prevSignalType = c->indices.signalType;
    int32_t LTP_Gain_Q14 = 0;
    if (c->indices.signalType == SIG_VOICED) {
        for (int j = 0; j * c->subfr_length < ctrl->pitchL[c->nb_subfr - 1]; j++) {
            if (j == c->nb_subfr) break;
            int32_t t = 0;
            for (int i = 0; i < 5; i++) t += ctrl->LTPCoef_Q14[(c->nb_subfr - 1 - j) * 5 + i];
            if (t > LTP_Gain_Q14) {
                LTP_Gain_Q14 = t;
                for (int i = 0; i < 5; i++) p->LTPCoef_Q14[i] = ctrl->LTPCoef_Q14[(c->nb_subfr - 1 - j) * 5 + i];
                p->pitchL_Q8 = shl32(ctrl->pitchL[c->nb_subfr - 1 - j], 8);
            }
        }
        for (int i = 0; i < 5; i++) p->LTPCoef_Q14[i] = 0;
        p->LTPCoef_Q14[2] = (int16_t)LTP_Gain_Q14;
        if (LTP_Gain_Q14 < 11469) {
            int32_t scale_Q10 = shl32(11469, 10) / imax(LTP_Gain_Q14, 1);
            for (int i = 0; i < 5; i++) p->LTPCoef_Q14[i] = (int16_t)(s_smulbb(p->LTPCoef_Q14[i], scale_Q10) >> 10);
        } else if (LTP_Gain_Q14 > 15565) {
            int32_t scale_Q14 = shl32(15565, 14) / imax(LTP_Gain_Q14, 1);
            for (int i = 0; i < 5; i++) p->LTPCoef_Q14[i] = (int16_t)(s_smulbb(p->LTPCoef_Q14[i], scale_Q14) >> 14);
        }
    } else {
        p->pitchL_Q8 = shl32(s_smulbb(c->fs_kHz, 18), 8);
        for (int i = 0; i < 5; i++) p->LTPCoef_Q14[i] = 0;
    }
    for (int i = 0; i < c->LPC_order; i++) p->prevLPC_Q12[i] = ctrl->PredCoef_Q12[1][i];
    p->prevLTP_scale_Q14 = (int16_t)ctrl->LTP_scale_Q14;
    p->prevGain_Q16[0] = ctrl->Gains_Q16[c->nb_subfr - 2];
    p->prevGain_Q16[1] = ctrl->Gains_Q16[c->nb_subfr - 1];
    p->subfr_length = c->subfr_length;
    p->nb_subfr = c->nb_subfr;
}

DNI void silk_plc_conceal(Lanes L, SilkChan *c, SilkCtrl *ctrl, int16_t *frame, SilkScratch *w)
{
    // HARM_ATT_Q15 {32440, 31130}, RAND_ATT_V_Q15 {31130, 26214}, RAND_ATT_UV_Q15
    // {32440, 29491} of silk/PLC.c, indexed by min(1, lossCnt)
    SilkPLC *p = &c->sPLC;
    int32_t *sLTP_Q14 = w->sLTP_Q15;
    int16_t *sLTP = w->sLTP;
    // The serial parts (energies, gains, the LPC chirp in place, the LTP
    // excitation and the LPC synthesis) run on the first lane; the lanes split
    // the LPC analysis filtering between them.  What the first lane computes
    // for the second serial part stays in its registers.
    int32_t prevGain_Q10[2] = {0, 0};
    const int32_t *rand_ptr = nullptr;
    int16_t *B_Q14 = p->LTPCoef_Q14;
    int16_t rand_scale_Q14 = 0;
    int32_t harm_Gain_Q15 = 0, rand_Gain_Q15 = 0;
    lead(L, [&]() CUO_INLINE {
        prevGain_Q10[0] = p->prevGain_Q16[0] >> 6;
        prevGain_Q10[1] = p->prevGain_Q16[1] >> 6;
        if (c->first_frame_after_reset) for (int i = 0; i < 16; i++) p->prevLPC_Q12[i] = 0;

        // silk_PLC_energy
        int32_t energy1, energy2;
        int shift1, shift2;
        {
            int16_t *eb = w->plc_exc;
            for (int k = 0; k < 2; k++)
                for (int i = 0; i < c->subfr_length; i++)
                    eb[k * c->subfr_length + i] = (int16_t)s_sat16(s_smulww(
                        c->exc_Q14[i + (k + c->nb_subfr - 2) * c->subfr_length], prevGain_Q10[k]) >> 8);
            silk_sum_sqr_shift(&energy1, &shift1, eb, c->subfr_length);
            silk_sum_sqr_shift(&energy2, &shift2, &eb[c->subfr_length], c->subfr_length);
        }
        if ((energy1 >> shift2) < (energy2 >> shift1))
            rand_ptr = &c->exc_Q14[imax(0, (p->nb_subfr - 1) * p->subfr_length - 128)];
        else
            rand_ptr = &c->exc_Q14[imax(0, p->nb_subfr * p->subfr_length - 128)];
        rand_scale_Q14 = p->randScale_Q14;
        const int first_loss = c->lossCnt == 0;
        harm_Gain_Q15 = first_loss ? 32440 : 31130;
        rand_Gain_Q15 = c->prevSignalType == SIG_VOICED ? (first_loss ? 31130 : 26214)
                                                        : (first_loss ? 32440 : 29491);
        silk_bwexpander(p->prevLPC_Q12, c->LPC_order, 64881);   // SILK_FIX_CONST(0.99, 16)
        if (c->lossCnt == 0) {
            rand_scale_Q14 = 1 << 14;
            if (c->prevSignalType == SIG_VOICED) {
                for (int i = 0; i < 5; i++) rand_scale_Q14 = (int16_t)(rand_scale_Q14 - B_Q14[i]);
                rand_scale_Q14 = rand_scale_Q14 > 3277 ? rand_scale_Q14 : 3277;
                rand_scale_Q14 = (int16_t)(s_smulbb(rand_scale_Q14, p->prevLTP_scale_Q14) >> 14);
            } else {
                int32_t invGain_Q30 = silk_lpc_inv_pred_gain(p->prevLPC_Q12, c->LPC_order, w->sw.A);
                int32_t down = min32((1 << 30) >> 3, invGain_Q30);
                down = max32((1 << 30) >> 8, down);
                down = shl32(down, 3);
                rand_Gain_Q15 = s_smulwb(down, rand_Gain_Q15) >> 14;
            }
        }
    });
    int16_t A_Q12[16];
    for (int i = 0; i < c->LPC_order; i++) A_Q12[i] = p->prevLPC_Q12[i];
    int lag = s_rshift_round(p->pitchL_Q8, 8);
    int idx = c->ltp_mem_length - lag - c->LPC_order - 2;
    silk_lpc_analysis_filter(L, &sLTP[idx], &c->outBuf[idx], A_Q12, c->ltp_mem_length - idx, c->LPC_order);
    int32_t inv_gain_Q30 = s_inverse32_varq(p->prevGain_Q16[1], 46);
    inv_gain_Q30 = min32(inv_gain_Q30, 0x7FFFFFFF >> 1);
    LFOR(L, i, idx + c->LPC_order, c->ltp_mem_length) sLTP_Q14[i] = s_smulwb(inv_gain_Q30, sLTP[i]);
    lead(L, [&]() CUO_INLINE {
        int32_t rand_seed = p->rand_seed;
        int sLTP_buf_idx = c->ltp_mem_length;
        for (int k = 0; k < c->nb_subfr; k++) {
            const int32_t *pl = &sLTP_Q14[sLTP_buf_idx - lag + 2];
            for (int i = 0; i < c->subfr_length; i++) {
                int32_t pr = 2;
                pr = s_smlawb(pr, pl[i], B_Q14[0]);
                pr = s_smlawb(pr, pl[i - 1], B_Q14[1]);
                pr = s_smlawb(pr, pl[i - 2], B_Q14[2]);
                pr = s_smlawb(pr, pl[i - 3], B_Q14[3]);
                pr = s_smlawb(pr, pl[i - 4], B_Q14[4]);
                rand_seed = s_rand(rand_seed);
                int ri = (rand_seed >> 25) & 127;
                sLTP_Q14[sLTP_buf_idx] = shl32(s_smlawb(pr, rand_ptr[ri], rand_scale_Q14), 2);
                sLTP_buf_idx++;
            }
            for (int j = 0; j < 5; j++) B_Q14[j] = (int16_t)(s_smulbb(harm_Gain_Q15, B_Q14[j]) >> 15);
            rand_scale_Q14 = (int16_t)(s_smulbb(rand_scale_Q14, rand_Gain_Q15) >> 15);
            p->pitchL_Q8 = s_smlawb(p->pitchL_Q8, p->pitchL_Q8, 655);
            p->pitchL_Q8 = min32(p->pitchL_Q8, shl32(s_smulbb(18, c->fs_kHz), 8));
            lag = s_rshift_round(p->pitchL_Q8, 8);
        }
        int32_t *sl = &sLTP_Q14[c->ltp_mem_length - 16];
        for (int i = 0; i < 16; i++) sl[i] = c->sLPC_Q14_buf[i];
        for (int i = 0; i < c->frame_length; i++) {
            int32_t pr = c->LPC_order >> 1;
            for (int j = 0; j < c->LPC_order; j++) pr = s_smlawb(pr, sl[16 + i - j - 1], A_Q12[j]);
            sl[16 + i] = s_add_sat32(sl[16 + i], s_lshift_sat32(pr, 4));
            frame[i] = (int16_t)s_sat16(s_sat16(s_rshift_round(s_smulww(sl[16 + i], prevGain_Q10[1]), 8)));
        }
        for (int i = 0; i < 16; i++) c->sLPC_Q14_buf[i] = sl[c->frame_length + i];
        p->rand_seed = rand_seed;
        p->randScale_Q14 = rand_scale_Q14;
        for (int i = 0; i < 4; i++) ctrl->pitchL[i] = lag;
    });
}

DNI void silk_plc(Lanes L, SilkChan *c, SilkCtrl *ctrl, int16_t *frame, int lost, SilkScratch *w)
{
    lead(L, [&]() CUO_INLINE {
        if (c->fs_kHz != c->sPLC.fs_kHz) {
            silk_plc_reset(c);
            c->sPLC.fs_kHz = c->fs_kHz;
        }
        if (!lost) silk_plc_update(c, ctrl);
    });
    if (lost) {
        silk_plc_conceal(L, c, ctrl, frame, w);
        lead(L, [&]() CUO_INLINE { c->lossCnt++; });
    }
}

DNI void silk_plc_glue_frames(SilkChan *c, int16_t *frame, int length)
{
    SilkPLC *p = &c->sPLC;
    if (c->lossCnt) {
        silk_sum_sqr_shift(&p->conc_energy, &p->conc_energy_shift, frame, length);
        p->last_frame_lost = 1;
    } else {
        if (p->last_frame_lost) {
            int32_t energy;
            int energy_shift;
            silk_sum_sqr_shift(&energy, &energy_shift, frame, length);
            if (energy_shift > p->conc_energy_shift)
                p->conc_energy = p->conc_energy >> (energy_shift - p->conc_energy_shift);
            else if (energy_shift < p->conc_energy_shift)
                energy = energy >> (p->conc_energy_shift - energy_shift);
            if (energy > p->conc_energy) {
                int32_t LZ = s_clz32(p->conc_energy) - 1;
                p->conc_energy = shl32(p->conc_energy, LZ);
                energy = energy >> imax(24 - LZ, 0);
                int32_t frac_Q24 = p->conc_energy / imax(energy, 1);
                int32_t gain_Q16 = shl32(s_sqrt_approx(frac_Q24), 4);
                int32_t slope_Q16 = ((1 << 16) - gain_Q16) / length;
                slope_Q16 = shl32(slope_Q16, 2);
                for (int i = 0; i < length; i++) {
                    frame[i] = (int16_t)s_smulwb(gain_Q16, frame[i]);
                    gain_Q16 += slope_Q16;
                    if (gain_Q16 > (1 << 16)) break;
                }
            }
        }
        p->last_frame_lost = 0;
    }
}

// silk/CNG.c
// The comfort-noise generation of silk_CNG (only after a lost frame): its own
// function, so the code of the per-frame update stays small.
DNI void silk_cng_generate(SilkChan *c, int16_t *frame, int length, SilkScratch *w)
{
    SilkCNG *g = &c->sCNG;
    int32_t *sig = w->CNG_sig_Q14;
    int32_t gain_Q16 = s_smulww(c->sPLC.randScale_Q14, c->sPLC.prevGain_Q16[1]);
    if (gain_Q16 >= (1 << 21) || g->CNG_smth_Gain_Q16 > (1 << 23)) {
        gain_Q16 = s_smultt(gain_Q16, gain_Q16);
        gain_Q16 = wsub(s_smultt(g->CNG_smth_Gain_Q16, g->CNG_smth_Gain_Q16), shl32(gain_Q16, 5));
        gain_Q16 = shl32(s_sqrt_approx(gain_Q16), 16);
    } else {
        gain_Q16 = s_smulww(gain_Q16, gain_Q16);
        gain_Q16 = wsub(s_smulww(g->CNG_smth_Gain_Q16, g->CNG_smth_Gain_Q16), shl32(gain_Q16, 5));
        gain_Q16 = shl32(s_sqrt_approx(gain_Q16), 8);
    }
    int32_t gain_Q10 = gain_Q16 >> 6;
    // silk_CNG_exc
    int exc_mask = 255;
    while (exc_mask > length) exc_mask >>= 1;
    int32_t seed = g->rand_seed;
    for (int i = 0; i < length; i++) {
        seed = s_rand(seed);
        sig[16 + i] = g->CNG_exc_buf_Q14[(seed >> 24) & exc_mask];
    }
    g->rand_seed = seed;
    int16_t A_Q12[16];
    silk_nlsf2a(A_Q12, g->CNG_smth_NLSF_Q15, c->LPC_order, &w->sw);
    for (int i = 0; i < 16; i++) sig[i] = g->CNG_synth_state[i];
    for (int i = 0; i < length; i++) {
        int32_t pr = c->LPC_order >> 1;
        for (int j = 0; j < c->LPC_order; j++) pr = s_smlawb(pr, sig[16 + i - j - 1], A_Q12[j]);
        sig[16 + i] = s_add_sat32(sig[16 + i], s_lshift_sat32(pr, 4));
        frame[i] = (int16_t)s_sat16((int32_t)frame[i] +
            s_sat16(s_rshift_round(s_smulww(sig[16 + i], gain_Q10), 8)));
    }
    for (int i = 0; i < 16; i++) g->CNG_synth_state[i] = sig[length + i];
}

DNI void silk_cng(Lanes L, SilkChan *c, const SilkCtrl *ctrl, int16_t *frame, int length, SilkScratch *w)
{
    SilkCNG *g = &c->sCNG;
    // state updates in place on the first lane; the lanes split the
    // excitation history move
    lead(L, [&]() CUO_INLINE {
        if (c->fs_kHz != g->fs_kHz) {
            silk_cng_reset(c);
            g->fs_kHz = c->fs_kHz;
        }
        if (c->lossCnt == 0 && c->prevSignalType == SIG_NO_VOICE)
            for (int i = 0; i < c->LPC_order; i++)
                g->CNG_smth_NLSF_Q15[i] = (int16_t)(g->CNG_smth_NLSF_Q15[i] +
                    s_smulwb((int32_t)c->prevNLSF_Q15[i] - (int32_t)g->CNG_smth_NLSF_Q15[i], 16348));
    });
    if (c->lossCnt == 0 && c->prevSignalType == SIG_NO_VOICE) {
        int32_t max_Gain_Q16 = 0;
        int subfr = 0;
        for (int i = 0; i < c->nb_subfr; i++)
            if (ctrl->Gains_Q16[i] > max_Gain_Q16) { max_Gain_Q16 = ctrl->Gains_Q16[i]; subfr = i; }
        // the excitation history moves up by one subframe: blocks of one
        // subframe from the top, each reading only what the block before it
        // has already moved; lanes split a block
        const int S = c->subfr_length;
        for (int hi = (c->nb_subfr - 1) * S; hi > 0; hi -= S) {
            LFOR(L, i, hi - S, hi) g->CNG_exc_buf_Q14[S + i] = g->CNG_exc_buf_Q14[i];
            lsync(L);
        }
        LFOR(L, i, 0, S) g->CNG_exc_buf_Q14[i] = c->exc_Q14[subfr * S + i];
        lead(L, [&]() CUO_INLINE {
            for (int i = 0; i < c->nb_subfr; i++) {
                g->CNG_smth_Gain_Q16 += s_smulwb(ctrl->Gains_Q16[i] - g->CNG_smth_Gain_Q16, 4634);
                if (s_smulww(g->CNG_smth_Gain_Q16, 46396) > ctrl->Gains_Q16[i])
                    g->CNG_smth_Gain_Q16 = ctrl->Gains_Q16[i];
            }
        });
    }
    lead(L, [&]() CUO_INLINE {
        if (c->lossCnt) silk_cng_generate(c, frame, length, w);
        else
            for (int i = 0; i < c->LPC_order; i++) g->CNG_synth_state[i] = 0;
    });
}

// ------------------------------------------------------------------ frame

// silk/decode_frame.c
DNI void silk_decode_frame(Lanes L, SilkChan *c, RangeDec *rd, int16_t *pOut, int *pN, int lostFlag,
                           int condCoding, SilkScratch *w)
{
    SilkCtrl *ctrl = &w->ctrl;
    int Lf = c->frame_length;
    if (lostFlag == LOSS_NONE || (lostFlag == LOSS_LBRR && c->LBRR_flags[c->nFramesDecoded] == 1)) {
        int16_t *pulses = w->pulses;
        // side information, pulses and parameters: entropy decoding and
        // state updates in place, on the first lane
        lead_rd(L, rd, [&]() CUO_INLINE {
            ctrl->LTP_scale_Q14 = 0;
            PHASE_BEGIN(t_ix);
            silk_decode_indices(c, rd, c->nFramesDecoded, lostFlag, condCoding, &w->sw);
            PHASE_END(PH_SILK_INDICES, t_ix, L.id);
            PHASE_BEGIN(t_pu);
            silk_decode_pulses(rd, pulses, c->indices.signalType, c->indices.quantOffsetType, c->frame_length,
                               &w->sw);
            PHASE_END(PH_SILK_PULSES, t_pu, L.id);
            PHASE_BEGIN(t_pa);
            silk_decode_parameters(c, ctrl, condCoding, &w->sw);
            PHASE_END(PH_SILK_PARAMS, t_pa, L.id);
        });
        PHASE_BEGIN(t_co);
        silk_decode_core(L, c, ctrl, pOut, pulses, w);
        PHASE_END(PH_SILK_CORE, t_co, L.id);
        int mv = c->ltp_mem_length - c->frame_length;
        lshift_copy(L, c->outBuf, mv, c->frame_length);
        LFOR(L, i, 0, c->frame_length) c->outBuf[mv + i] = pOut[i];
        lsync(L);
        PHASE_BEGIN(t_pl);
        silk_plc(L, c, ctrl, pOut, 0, w);
        PHASE_END(PH_SILK_PLC, t_pl, L.id);
        lead(L, [&]() CUO_INLINE {
            c->lossCnt = 0;
            c->prevSignalType = c->indices.signalType;
            c->first_frame_after_reset = 0;
        });
    } else {
        lead(L, [&]() CUO_INLINE { ctrl->LTP_scale_Q14 = 0; });
        silk_plc(L, c, ctrl, pOut, 1, w);
        int mv = c->ltp_mem_length - c->frame_length;
        lshift_copy(L, c->outBuf, mv, c->frame_length);
        LFOR(L, i, 0, c->frame_length) c->outBuf[mv + i] = pOut[i];
        lsync(L);
    }
    PHASE_BEGIN(t_cn);
    silk_cng(L, c, ctrl, pOut, Lf, w);
    PHASE_END(PH_SILK_CNG, t_cn, L.id);
    lead(L, [&]() CUO_INLINE {
        silk_plc_glue_frames(c, pOut, Lf);
        c->lagPrev = ctrl->pitchL[c->nb_subfr - 1];
    });
    *pN = Lf;
}

// silk/stereo_MS_to_LR.c; all samples depend only on inputs, so lanes split them
DNI void silk_stereo_ms_to_lr(Lanes L, SilkStereo *st, int16_t *x1, int16_t *x2, const int32_t *pred_Q13,
                              int fs_kHz, int frame_length)
{
    int16_t m0 = st->sMid[0], m1 = st->sMid[1], s0 = st->sSide[0], s1 = st->sSide[1];
    int16_t nm0 = x1[frame_length], nm1 = x1[frame_length + 1];
    int16_t ns0 = x2[frame_length], ns1 = x2[frame_length + 1];
    lsync(L);
    if (L.id == 0) { x1[0] = m0; x1[1] = m1; x2[0] = s0; x2[1] = s1; }
    st->sMid[0] = nm0; st->sMid[1] = nm1; st->sSide[0] = ns0; st->sSide[1] = ns1;
    lsync(L);
    int32_t pred0 = st->pred_prev_Q13[0], pred1 = st->pred_prev_Q13[1];
    int interp = 8 * fs_kHz;
    int32_t denom_Q16 = (1 << 16) / interp;
    int32_t d0 = s_rshift_round(s_smulbb(pred_Q13[0] - st->pred_prev_Q13[0], denom_Q16), 16);
    int32_t d1 = s_rshift_round(s_smulbb(pred_Q13[1] - st->pred_prev_Q13[1], denom_Q16), 16);
    // side channel rewrite: x2[n+1] from x1[n..n+2] and x2[n+1]
    LFOR(L, n, 0, frame_length) {
        int32_t p0 = n < interp ? pred0 + (n + 1) * d0 : pred_Q13[0];
        int32_t p1 = n < interp ? pred1 + (n + 1) * d1 : pred_Q13[1];
        int32_t sum = shl32(wadd((int32_t)x1[n] + (int32_t)x1[n + 2], shl32(x1[n + 1], 1)), 9);
        sum = s_smlawb(shl32((int32_t)x2[n + 1], 8), sum, p0);
        sum = s_smlawb(sum, shl32((int32_t)x1[n + 1], 11), p1);
        x2[n + 1] = (int16_t)s_sat16(s_rshift_round(sum, 8));
    }
    lsync(L);
    st->pred_prev_Q13[0] = (int16_t)pred_Q13[0];
    st->pred_prev_Q13[1] = (int16_t)pred_Q13[1];
    LFOR(L, n, 0, frame_length) {
        int32_t sum = x1[n + 1] + (int32_t)x2[n + 1];
        int32_t diff = x1[n + 1] - (int32_t)x2[n + 1];
        x1[n + 1] = (int16_t)s_sat16(sum);
        x2[n + 1] = (int16_t)s_sat16(diff);
    }
    lsync(L);
}

// silk/dec_API.c silk_Decode (API rate 48 kHz, no deep PLC).  Returns nonzero
// on an invalid configuration.
// Regular decoding reads past the packet's LBRR (in-band FEC) frames: their
// indices and pulses are decoded and dropped (silk/dec_API.c).  Returns the
// mid-only flag as the last LBRR frame left it.
DNI int silk_skip_lbrr(SilkChan *cs, int nChannelsInternal, RangeDec *rd, int32_t *MS_pred_Q13,
                       int decode_only_middle, SilkScratch *w)
{
    for (int i = 0; i < cs[0].nFramesPerPacket; i++) {
        for (int n = 0; n < nChannelsInternal; n++) {
            if (cs[n].LBRR_flags[i]) {
                if (nChannelsInternal == 2 && n == 0) {
                    silk_stereo_decode_pred(rd, MS_pred_Q13);
                    if (cs[1].LBRR_flags[i] == 0)
                        decode_only_middle = rd_icdf(rd, T_silk_stereo_only_code_mid_iCDF, 8);
                }
                int cond = (i > 0 && cs[n].LBRR_flags[i - 1]) ? CODE_COND : CODE_INDEP;
                silk_decode_indices(&cs[n], rd, i, 1, cond, &w->sw);
                silk_decode_pulses(rd, w->lbrr_pulses, cs[n].indices.signalType, cs[n].indices.quantOffsetType,
                                   cs[n].frame_length, &w->sw);
            }
        }
    }
    return decode_only_middle;
}

DNI int silk_decode(Lanes L, SilkDec *dec, SilkDecControl *ctl, int lostFlag, int newPacketFlag,
                    RangeDec *rd, int16_t *samplesOut, int32_t *nSamplesOut, SilkScratch *w)
{
    int ret = 0;
    int32_t nSamplesOutDec = 0;
    int32_t MS_pred_Q13[2] = {0, 0};
    SilkChan *cs = dec->ch;

    // The packet header: VAD and LBRR flags, skipped LBRR frames, stereo
    // prediction, channel (re)configuration -- entropy decoding and state
    // updates in place, on the first lane; every lane gets the outcome.
    int hdr[6] = {0, 0, 0, 0, 0, 0};   // status, mid only, stereo to mono, MS pred 0 / 1, has side
    lead_rd(L, rd, [&]() CUO_INLINE {
    int32_t ms_pred[2] = {0, 0};
        int decode_only_middle = 0;
        if (newPacketFlag)
            for (int n = 0; n < ctl->nChannelsInternal; n++) cs[n].nFramesDecoded = 0;
        if (ctl->nChannelsInternal > dec->nChannelsInternal) {
            silk_reset_chan(&cs[1]);   // silk_init_decoder
        }
        hdr[2] = ctl->nChannelsInternal == 1 && dec->nChannelsInternal == 2 &&
                             ctl->internalSampleRate == 1000 * cs[0].fs_kHz;
        if (cs[0].nFramesDecoded == 0) {
            for (int n = 0; n < ctl->nChannelsInternal; n++) {
                int ms = ctl->payloadSize_ms;
                if (ms == 0 || ms == 10) { cs[n].nFramesPerPacket = 1; cs[n].nb_subfr = 2; }
                else if (ms == 20) { cs[n].nFramesPerPacket = 1; cs[n].nb_subfr = 4; }
                else if (ms == 40) { cs[n].nFramesPerPacket = 2; cs[n].nb_subfr = 4; }
                else if (ms == 60) { cs[n].nFramesPerPacket = 3; cs[n].nb_subfr = 4; }
                else { hdr[0] = -203; return; }   // SILK_DEC_INVALID_FRAME_SIZE
                int fs_kHz_dec = (ctl->internalSampleRate >> 10) + 1;
                if (fs_kHz_dec != 8 && fs_kHz_dec != 12 && fs_kHz_dec != 16) { hdr[0] = -200; return; }
                silk_decoder_set_fs(&cs[n], fs_kHz_dec, ctl->API_sampleRate);
            }
        }
        if (ctl->nChannelsAPI == 2 && ctl->nChannelsInternal == 2 &&
            (dec->nChannelsAPI == 1 || dec->nChannelsInternal == 1)) {
            dec->sStereo.pred_prev_Q13[0] = dec->sStereo.pred_prev_Q13[1] = 0;
            dec->sStereo.sSide[0] = dec->sStereo.sSide[1] = 0;
            cs[1].resampler_state = cs[0].resampler_state;
        }
        dec->nChannelsAPI = ctl->nChannelsAPI;
        dec->nChannelsInternal = ctl->nChannelsInternal;

        if (lostFlag != LOSS_LOST && cs[0].nFramesDecoded == 0) {
            for (int n = 0; n < ctl->nChannelsInternal; n++) {
                for (int i = 0; i < cs[n].nFramesPerPacket; i++) cs[n].VAD_flags[i] = rd_bit_logp(rd, 1);
                cs[n].LBRR_flag = rd_bit_logp(rd, 1);
            }
            for (int n = 0; n < ctl->nChannelsInternal; n++) {
                cs[n].LBRR_flags[0] = cs[n].LBRR_flags[1] = cs[n].LBRR_flags[2] = 0;
                if (cs[n].LBRR_flag) {
                    if (cs[n].nFramesPerPacket == 1) {
                        cs[n].LBRR_flags[0] = 1;
                    } else {
                        const uint8_t *t = cs[n].nFramesPerPacket == 2 ? T_silk_LBRR_flags_2_iCDF
                                                                       : T_silk_LBRR_flags_3_iCDF;
                        int sym = rd_icdf(rd, t, 8) + 1;
                        for (int i = 0; i < cs[n].nFramesPerPacket; i++) cs[n].LBRR_flags[i] = (sym >> i) & 1;
                    }
                }
            }
            if (lostFlag == LOSS_NONE && (cs[0].LBRR_flag || (ctl->nChannelsInternal == 2 && cs[1].LBRR_flag)))
                decode_only_middle = silk_skip_lbrr(cs, ctl->nChannelsInternal, rd, ms_pred, decode_only_middle, w);
        }
        if (ctl->nChannelsInternal == 2) {
            if (lostFlag == LOSS_NONE ||
                (lostFlag == LOSS_LBRR && cs[0].LBRR_flags[cs[0].nFramesDecoded] == 1)) {
                silk_stereo_decode_pred(rd, ms_pred);
                if ((lostFlag == LOSS_NONE && cs[1].VAD_flags[cs[0].nFramesDecoded] == 0) ||
                    (lostFlag == LOSS_LBRR && cs[1].LBRR_flags[cs[0].nFramesDecoded] == 0))
                    decode_only_middle = rd_icdf(rd, T_silk_stereo_only_code_mid_iCDF, 8);
                else
                    decode_only_middle = 0;
            } else {
                ms_pred[0] = dec->sStereo.pred_prev_Q13[0];
                ms_pred[1] = dec->sStereo.pred_prev_Q13[1];
            }
        }
        if (ctl->nChannelsInternal == 2 && decode_only_middle == 0 && dec->prev_decode_only_middle == 1) {
            memset(cs[1].outBuf, 0, sizeof(cs[1].outBuf));
            memset(cs[1].sLPC_Q14_buf, 0, sizeof(cs[1].sLPC_Q14_buf));
            cs[1].lagPrev = 100;
            cs[1].LastGainIndex = 10;
            cs[1].prevSignalType = SIG_NO_VOICE;
            cs[1].first_frame_after_reset = 1;
        }
        if (lostFlag == LOSS_NONE) hdr[5] = !decode_only_middle;
        else hdr[5] = !dec->prev_decode_only_middle ||
                        (ctl->nChannelsInternal == 2 && lostFlag == LOSS_LBRR &&
                         cs[1].LBRR_flags[cs[1].nFramesDecoded] == 1);
        hdr[1] = decode_only_middle;
        hdr[3] = ms_pred[0];
        hdr[4] = ms_pred[1];
    });
    for (int k = 0; k < 6; k++) hdr[k] = lbcast(L, hdr[k]);
    if (hdr[0]) return hdr[0];
    const int decode_only_middle = hdr[1], stereo_to_mono = hdr[2], has_side = hdr[5];
    MS_pred_Q13[0] = hdr[3];
    MS_pred_Q13[1] = hdr[4];
    int16_t *tmp[2] = {w->tmp[0], w->tmp[1]};
    for (int n = 0; n < ctl->nChannelsInternal; n++) {
        if (n == 0 || has_side) {
            int FrameIndex = cs[0].nFramesDecoded - n;
            int cond;
            if (FrameIndex <= 0) cond = CODE_INDEP;
            else if (lostFlag == LOSS_LBRR) cond = cs[n].LBRR_flags[FrameIndex - 1] ? CODE_COND : CODE_INDEP;
            else if (n > 0 && dec->prev_decode_only_middle) cond = CODE_INDEP_NO_LTP_SCALING;
            else cond = CODE_COND;
            int nOut;
            silk_decode_frame(L, &cs[n], rd, &tmp[n][2], &nOut, lostFlag, cond, w);
            nSamplesOutDec = nOut;
        } else {
            LFOR(L, i, 0, nSamplesOutDec) tmp[n][2 + i] = 0;
        }
        lead(L, [&]() CUO_INLINE { cs[n].nFramesDecoded++; });
    }
    if (ctl->nChannelsAPI == 2 && ctl->nChannelsInternal == 2) {
        PHASE_BEGIN(t_st);
        silk_stereo_ms_to_lr(L, &dec->sStereo, tmp[0], tmp[1], MS_pred_Q13, cs[0].fs_kHz, nSamplesOutDec);
        PHASE_END(PH_SILK_STEREO, t_st, L.id);
    } else {
        int16_t m0 = dec->sStereo.sMid[0], m1 = dec->sStereo.sMid[1];
        int16_t n0 = tmp[0][nSamplesOutDec], n1 = tmp[0][nSamplesOutDec + 1];
        lsync(L);
        if (L.id == 0) { tmp[0][0] = m0; tmp[0][1] = m1; }
        dec->sStereo.sMid[0] = n0;
        dec->sStereo.sMid[1] = n1;
        lsync(L);
    }
    *nSamplesOut = nSamplesOutDec * ctl->API_sampleRate / s_smulbb(cs[0].fs_kHz, 1000);
    int16_t *rs_out = ctl->nChannelsAPI == 2 ? w->rs_out : samplesOut;
    int nres = imin(ctl->nChannelsAPI, ctl->nChannelsInternal);
    for (int n = 0; n < nres; n++) {
        PHASE_BEGIN(t_rs);
        silk_resample(L, &cs[n].resampler_state, rs_out, &tmp[n][1], nSamplesOutDec, w->rs_buf);
        PHASE_END(PH_SILK_RESAMPLE, t_rs, L.id);
        if (ctl->nChannelsAPI == 2) {
            LFOR(L, i, 0, *nSamplesOut) samplesOut[n + 2 * i] = rs_out[i];
            lsync(L);
        }
    }
    if (ctl->nChannelsAPI == 2 && ctl->nChannelsInternal == 1) {
        if (stereo_to_mono) {
            silk_resample(L, &cs[1].resampler_state, rs_out, &tmp[0][1], nSamplesOutDec, w->rs_buf);
            LFOR(L, i, 0, *nSamplesOut) samplesOut[1 + 2 * i] = rs_out[i];
        } else {
            LFOR(L, i, 0, *nSamplesOut) samplesOut[1 + 2 * i] = samplesOut[2 * i];
        }
        lsync(L);
    }
    lead(L, [&]() CUO_INLINE {
        if (lostFlag == LOSS_LOST) {
            for (int i = 0; i < dec->nChannelsInternal; i++) cs[i].LastGainIndex = 10;
        } else {
            dec->prev_decode_only_middle = decode_only_middle;
        }
    });
    return ret;
}

} // namespace cuo
