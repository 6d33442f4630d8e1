/* Stage timers of the diagnostic build, libcuopus_phases.so.
 *
 * libcuopus_phases.so is libcuopus.so (every entry point of cuopus.h) built
 * with the decoder's stage timers on: the first lane of each chain's lane
 * group reads the SM clock around each decoder stage and adds the cycles to a
 * device counter per stage.  The timers cost time of their own, so the
 * figures are for the split between stages, never for throughput; the
 * product library, libcuopus.so, has no timers and does not export these.
 *
 * No counterpart in the reference, which has no per-stage timing of its
 * decode kernel.
 *
 * Stage order (cuopus_phase_read's out[i]): packet (one whole opus_decode of
 * a packet; contains the others), silk_indices, silk_pulses, silk_params,
 * silk_core, silk_plc, silk_cng, silk_stereo, silk_resample, celt_coarse,
 * celt_alloc, celt_shift, celt_bands, celt_synth, celt_comb, celt_deemph,
 * keep_copy (the PCM write, inside "packet").
 */
#ifndef CUOPUS_PHASES_H
#define CUOPUS_PHASES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Number of stage counters (17).  Host only. */
int cuopus_phase_count(void);

/* Copy the counters of the current device (cycles summed since the last
 * cuopus_phase_reset) to out[0 .. cuopus_phase_count()).  0, or 2 on a CUDA
 * error.  Synchronous with respect to the device. */
int cuopus_phase_read(uint64_t *out);

/* Zero the counters of the current device.  0, or 2 on a CUDA error. */
int cuopus_phase_reset(void);

#ifdef __cplusplus
}
#endif

#endif
