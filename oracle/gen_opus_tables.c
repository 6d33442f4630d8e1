/* Dumps the normative Opus decoder tables (RFC 6716 codebooks, iCDFs and the
 * static 48 kHz / 960-sample CELT mode) into opus_tables.inc.
 *
 * The tables are data the decoder must reproduce exactly, so they are not
 * retyped: this program is compiled against the vendored libopus 1.5.2
 * sources (FIXED_POINT) and prints every table from the compiled objects.
 * It is a one-off generator; its output, opus_tables.inc, is committed.
 *
 *   make -C oracle REF=<reference tree> tables
 *
 * builds it (oracle/_build/gen_opus_tables, linked with oracle/_ref's
 * libopus) and rewrites cuopus_b200/csrc/dec/opus_tables.inc.  It lives
 * beside the oracle because it compiles the reference's vendored sources; the
 * product only includes its output.
 *
 * File-static tables (coarse-energy model, PVQ counts, log2 fractions, band
 * ordering) are reached by including the vendor translation units that own
 * them; everything else goes through the exported symbols and the mode
 * returned by opus_custom_mode_create(48000, 960).
 */
#include <stdio.h>
#include <stdint.h>

#include "celt/quant_bands.c"
#include "celt/rate.c"
#include "celt/cwrs.c"
#include "celt/bands.c"
#include "celt/celt.h"
#include "celt/modes.h"
#include "silk/main.h"
#include "silk/resampler_rom.h"
#include "silk/pitch_est_defines.h"

static void emit_hdr(const char *cls, const char *type, const char *name, long n)
{
    printf("%s(%s, %s[%ld]) = {", cls, type, name, n);
}

#define EMITS(cls, type, name, src, n) do {                                 \
    long _n = (long)(n);                                                      \
    emit_hdr(cls, #type, name, _n);                                            \
    for (long _i = 0; _i < _n; _i++)                                          \
        printf("%s%s%ld", _i ? "," : "", (_i % 16) ? "" : "\n  ", (long)(src)[_i]); \
    printf("\n};\n");                                                         \
} while (0)

#define EMITU(cls, type, name, src, n) do {                                 \
    long _n = (long)(n);                                                      \
    emit_hdr(cls, #type, #name, _n);                                            \
    for (long _i = 0; _i < _n; _i++)                                          \
        printf("%s%s%luu", _i ? "," : "", (_i % 8) ? "" : "\n  ", (unsigned long)(src)[_i]); \
    printf("\n};\n");                                                         \
} while (0)

#define EMIT(cls, type, name, src, n) EMITS(cls, type, #name, src, n)

int main(void)
{
    int i;
    printf("/* GENERATED by gen_opus_tables.c from the vendored libopus 1.5.2\n"
           " * (FIXED_POINT). Normative RFC 6716 decoder tables; do not edit. */\n\n");

    /* ---------------- SILK ---------------- */
    EMIT("TABC", uint8_t, T_silk_gain_iCDF, &silk_gain_iCDF[0][0], 3 * 8);
    EMIT("TABC", uint8_t, T_silk_delta_gain_iCDF, silk_delta_gain_iCDF, 41);
    EMIT("TABC", uint8_t, T_silk_pitch_lag_iCDF, silk_pitch_lag_iCDF, 32);
    EMIT("TABC", uint8_t, T_silk_pitch_delta_iCDF, silk_pitch_delta_iCDF, 21);
    EMIT("TABC", uint8_t, T_silk_pitch_contour_iCDF, silk_pitch_contour_iCDF, 34);
    EMIT("TABC", uint8_t, T_silk_pitch_contour_NB_iCDF, silk_pitch_contour_NB_iCDF, 11);
    EMIT("TABC", uint8_t, T_silk_pitch_contour_10_ms_iCDF, silk_pitch_contour_10_ms_iCDF, 12);
    EMIT("TABC", uint8_t, T_silk_pitch_contour_10_ms_NB_iCDF, silk_pitch_contour_10_ms_NB_iCDF, 3);
    EMIT("TABC", uint8_t, T_silk_pulses_per_block_iCDF, &silk_pulses_per_block_iCDF[0][0], 10 * 18);
    EMIT("TABC", uint8_t, T_silk_rate_levels_iCDF, &silk_rate_levels_iCDF[0][0], 2 * 9);
    EMIT("TABC", uint8_t, T_silk_shell_code_table0, silk_shell_code_table0, 152);
    EMIT("TABC", uint8_t, T_silk_shell_code_table1, silk_shell_code_table1, 152);
    EMIT("TABC", uint8_t, T_silk_shell_code_table2, silk_shell_code_table2, 152);
    EMIT("TABC", uint8_t, T_silk_shell_code_table3, silk_shell_code_table3, 152);
    EMIT("TABC", uint8_t, T_silk_shell_code_table_offsets, silk_shell_code_table_offsets, 17);
    EMIT("TABC", uint8_t, T_silk_sign_iCDF, silk_sign_iCDF, 42);
    EMIT("TABC", uint8_t, T_silk_lsb_iCDF, silk_lsb_iCDF, 2);
    EMIT("TABC", uint8_t, T_silk_LTP_per_index_iCDF, silk_LTP_per_index_iCDF, 3);
    EMIT("TABC", uint8_t, T_silk_LTP_gain_iCDF_0, silk_LTP_gain_iCDF_ptrs[0], 8);
    EMIT("TABC", uint8_t, T_silk_LTP_gain_iCDF_1, silk_LTP_gain_iCDF_ptrs[1], 16);
    EMIT("TABC", uint8_t, T_silk_LTP_gain_iCDF_2, silk_LTP_gain_iCDF_ptrs[2], 32);
    EMIT("TABC", int8_t, T_silk_LTP_gain_vq_0, silk_LTP_vq_ptrs_Q7[0], 8 * 5);
    EMIT("TABC", int8_t, T_silk_LTP_gain_vq_1, silk_LTP_vq_ptrs_Q7[1], 16 * 5);
    EMIT("TABC", int8_t, T_silk_LTP_gain_vq_2, silk_LTP_vq_ptrs_Q7[2], 32 * 5);
    EMIT("TABC", int16_t, T_silk_LTPScales_table_Q14, silk_LTPScales_table_Q14, 3);
    EMIT("TABC", uint8_t, T_silk_LTPscale_iCDF, silk_LTPscale_iCDF, 3);
    EMIT("TABC", uint8_t, T_silk_type_offset_VAD_iCDF, silk_type_offset_VAD_iCDF, 4);
    EMIT("TABC", uint8_t, T_silk_type_offset_no_VAD_iCDF, silk_type_offset_no_VAD_iCDF, 2);
    EMIT("TABC", uint8_t, T_silk_NLSF_interpolation_factor_iCDF, silk_NLSF_interpolation_factor_iCDF, 5);
    EMIT("TABC", int16_t, T_silk_Quantization_Offsets_Q10, &silk_Quantization_Offsets_Q10[0][0], 4);
    EMIT("TABC", uint8_t, T_silk_uniform3_iCDF, silk_uniform3_iCDF, 3);
    EMIT("TABC", uint8_t, T_silk_uniform4_iCDF, silk_uniform4_iCDF, 4);
    EMIT("TABC", uint8_t, T_silk_uniform5_iCDF, silk_uniform5_iCDF, 5);
    EMIT("TABC", uint8_t, T_silk_uniform6_iCDF, silk_uniform6_iCDF, 6);
    EMIT("TABC", uint8_t, T_silk_uniform8_iCDF, silk_uniform8_iCDF, 8);
    EMIT("TABC", uint8_t, T_silk_NLSF_EXT_iCDF, silk_NLSF_EXT_iCDF, 7);
    EMIT("TABC", uint8_t, T_silk_LBRR_flags_2_iCDF, silk_LBRR_flags_iCDF_ptr[0], 3);
    EMIT("TABC", uint8_t, T_silk_LBRR_flags_3_iCDF, silk_LBRR_flags_iCDF_ptr[1], 7);
    EMIT("TABC", int16_t, T_silk_stereo_pred_quant_Q13, silk_stereo_pred_quant_Q13, 16);
    EMIT("TABC", uint8_t, T_silk_stereo_pred_joint_iCDF, silk_stereo_pred_joint_iCDF, 25);
    EMIT("TABC", uint8_t, T_silk_stereo_only_code_mid_iCDF, silk_stereo_only_code_mid_iCDF, 2);
    EMIT("TABG", int16_t, T_silk_LSFCosTab_FIX_Q12, silk_LSFCosTab_FIX_Q12, 129);
    EMIT("TABC", int8_t, T_silk_CB_lags_stage2, &silk_CB_lags_stage2[0][0], 4 * 11);
    EMIT("TABC", int8_t, T_silk_CB_lags_stage3, &silk_CB_lags_stage3[0][0], 4 * 34);
    EMIT("TABC", int8_t, T_silk_CB_lags_stage2_10_ms, &silk_CB_lags_stage2_10_ms[0][0], 2 * 3);
    EMIT("TABC", int8_t, T_silk_CB_lags_stage3_10_ms, &silk_CB_lags_stage3_10_ms[0][0], 2 * 12);
    EMIT("TABG", int16_t, T_silk_resampler_frac_FIR_12, &silk_resampler_frac_FIR_12[0][0], 12 * 4);
    EMIT("TABC", int16_t, T_silk_resampler_up2_hq_0, silk_resampler_up2_hq_0, 3);
    EMIT("TABC", int16_t, T_silk_resampler_up2_hq_1, silk_resampler_up2_hq_1, 3);
    printf("#define T_SILK_PE_NB_CBKS_STAGE2_EXT %d\n#define T_SILK_PE_NB_CBKS_STAGE3_MAX %d\n"
           "#define T_SILK_PE_NB_CBKS_STAGE2_10MS %d\n#define T_SILK_PE_NB_CBKS_STAGE3_10MS %d\n",
           PE_NB_CBKS_STAGE2_EXT, PE_NB_CBKS_STAGE3_MAX, PE_NB_CBKS_STAGE2_10MS,
           PE_NB_CBKS_STAGE3_10MS);

    {
        const silk_NLSF_CB_struct *cb[2] = { &silk_NLSF_CB_NB_MB, &silk_NLSF_CB_WB };
        const char *nm[2] = { "NB_MB", "WB" };
        for (int k = 0; k < 2; k++) {
            const silk_NLSF_CB_struct *c = cb[k];
            char buf[96];
            int nv = c->nVectors, o = c->order;
            printf("#define T_NLSF_%s_NVECTORS %d\n#define T_NLSF_%s_ORDER %d\n"
                   "#define T_NLSF_%s_QSTEP_Q16 %d\n", nm[k], nv, nm[k], o, nm[k],
                   c->quantStepSize_Q16);
            snprintf(buf, sizeof buf, "T_NLSF_%s_CB1_Q8", nm[k]);
            EMITS("TABC", uint8_t, buf, c->CB1_NLSF_Q8, nv * o);
            snprintf(buf, sizeof buf, "T_NLSF_%s_CB1_Wght_Q9", nm[k]);
            EMITS("TABC", int16_t, buf, c->CB1_Wght_Q9, nv * o);
            snprintf(buf, sizeof buf, "T_NLSF_%s_CB1_iCDF", nm[k]);
            EMITS("TABC", uint8_t, buf, c->CB1_iCDF, 2 * nv);
            snprintf(buf, sizeof buf, "T_NLSF_%s_pred_Q8", nm[k]);
            EMITS("TABC", uint8_t, buf, c->pred_Q8, 2 * (o - 1));
            snprintf(buf, sizeof buf, "T_NLSF_%s_ec_sel", nm[k]);
            EMITS("TABC", uint8_t, buf, c->ec_sel, nv * o / 2);
            snprintf(buf, sizeof buf, "T_NLSF_%s_ec_iCDF", nm[k]);
            EMITS("TABC", uint8_t, buf, c->ec_iCDF, 72);
            snprintf(buf, sizeof buf, "T_NLSF_%s_deltaMin_Q15", nm[k]);
            EMITS("TABC", int16_t, buf, c->deltaMin_Q15, o + 1);
        }
    }

    /* ---------------- CELT ---------------- */
    {
        const CELTMode *m = opus_custom_mode_create(48000, 960, NULL);
        printf("#define T_CELT_NBEBANDS %d\n#define T_CELT_EFFEBANDS %d\n#define T_CELT_OVERLAP %d\n"
               "#define T_CELT_MAXLM %d\n#define T_CELT_SHORTMDCT %d\n#define T_CELT_NBALLOCV %d\n"
               "#define T_CELT_PREEMPH0 %d\n#define T_CELT_MDCT_N %d\n#define T_CELT_CACHE_SIZE %d\n",
               m->nbEBands, m->effEBands, m->overlap, m->maxLM, m->shortMdctSize,
               m->nbAllocVectors, m->preemph[0], m->mdct.n, m->cache.size);
        EMIT("TABC", int16_t, T_celt_eBands, m->eBands, m->nbEBands + 1);
        EMIT("TABC", int16_t, T_celt_logN, m->logN, m->nbEBands);
        EMIT("TABC", uint8_t, T_celt_allocVectors, m->allocVectors, m->nbAllocVectors * m->nbEBands);
        EMIT("TABG", int16_t, T_celt_window, m->window, m->overlap);
        EMIT("TABC", int16_t, T_celt_cache_index, m->cache.index, m->nbEBands * (m->maxLM + 2));
        EMIT("TABC", uint8_t, T_celt_cache_bits, m->cache.bits, m->cache.size);
        EMIT("TABC", uint8_t, T_celt_cache_caps, m->cache.caps, (m->maxLM + 1) * 2 * m->nbEBands);
        {
            int n = m->mdct.n, tot = 0;
            for (i = 0; i <= m->mdct.maxshift; i++) { n >>= 1; tot += n; }
            EMIT("TABG", int16_t, T_celt_mdct_trig, m->mdct.trig, tot);
        }
        for (i = 0; i <= m->mdct.maxshift; i++) {
            const kiss_fft_state *s = m->mdct.kfft[i];
            char buf[64];
            int nf = 0;
            while (nf < MAXFACTORS && s->factors[2 * nf + 1] != 1) nf++;
            nf++;
            printf("#define T_FFT%d_NFFT %d\n#define T_FFT%d_SHIFT %d\n#define T_FFT%d_NFACT %d\n",
                   i, s->nfft, i, s->shift, i, nf);
            snprintf(buf, sizeof buf, "T_fft%d_factors", i);
            EMITS("TABC", int16_t, buf, s->factors, 2 * MAXFACTORS);
            snprintf(buf, sizeof buf, "T_fft%d_bitrev", i);
            EMITS("TABG", int16_t, buf, s->bitrev, s->nfft);
        }
        {
            const kiss_fft_state *s = m->mdct.kfft[0];
            static int16_t tw[2 * 480];
            for (i = 0; i < s->nfft; i++) { tw[2 * i] = s->twiddles[i].r; tw[2 * i + 1] = s->twiddles[i].i; }
            EMIT("TABG", int16_t, T_fft_twiddles, tw, 2 * s->nfft);
        }
    }
    EMIT("TABC", uint8_t, T_celt_e_prob_model, &e_prob_model[0][0][0], 4 * 2 * 42);
    EMIT("TABC", int16_t, T_celt_pred_coef, pred_coef, 4);
    EMIT("TABC", int16_t, T_celt_beta_coef, beta_coef, 4);
    printf("#define T_CELT_BETA_INTRA %d\n", beta_intra);
    EMIT("TABC", uint8_t, T_celt_small_energy_icdf, small_energy_icdf, 3);
    EMIT("TABC", int8_t, T_celt_eMeans, eMeans, 25);
    EMIT("TABC", int8_t, T_celt_tf_select_table, &tf_select_table[0][0], 32);
    EMIT("TABC", uint8_t, T_celt_trim_icdf, trim_icdf, 11);
    EMIT("TABC", uint8_t, T_celt_spread_icdf, spread_icdf, 4);
    EMIT("TABC", uint8_t, T_celt_tapset_icdf, tapset_icdf, 3);
    EMIT("TABC", uint8_t, T_celt_log2_frac_table, LOG2_FRAC_TABLE, 24);
    EMIT("TABC", int32_t, T_celt_ordery_table, ordery_table, 30);
    EMITU("TABC", uint32_t, T_celt_pvq_u_data, CELT_PVQ_U_DATA, sizeof(CELT_PVQ_U_DATA) / 4);
    {
        int rows[15];
        for (i = 0; i < 15; i++) rows[i] = (int)(CELT_PVQ_U_ROW[i] - CELT_PVQ_U_DATA);
        EMIT("TABC", int16_t, T_celt_pvq_u_row, rows, 15);
    }
    return 0;
}
