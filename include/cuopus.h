/* libcuopus — batched Opus decode on NVIDIA Blackwell (sm_100a).
 *
 * C ABI of the drop-in library.  The first eight entry points have exactly the
 * signatures and semantics of the reference's libcuopus.cu (cited per entry);
 * the rest extend it and say so.
 *
 * Return codes (reference libcuopus.cu:48-51): 0 ok; 1 soft failure (bad
 * stream or decode validation; the CUDA context is healthy, the caller may
 * fall back to a CPU decoder); 2 CUDA error (context suspect); 3 caller error
 * (capacity, NULL pointer, stream capture in progress, too many merged
 * chains).  errbuf, when not NULL, always receives a NUL-terminated message.
 *
 * Threading: the library never creates a context, thread or stream; all work
 * is issued on the caller's stream (or stream 0) of the current device, and
 * every call synchronises that stream before it returns.  It refuses to run
 * while that stream is capturing a CUDA graph.  Workspaces are process-global
 * and grow-only; calls must not run concurrently from several host threads.
 */
#ifndef CUOPUS_H
#define CUOPUS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Demux + validate (mono, granule cross-check) and return the exact f16k
 * output length max(0, (playable48 - 48) / 3).  Host only.
 * Replaces reference libcuopus.cu:223-236 (cuopus_probe). */
int cuopus_probe(const uint8_t *ogg, size_t n, int64_t *samples16k, char *errbuf, size_t errcap);

/* cuopus_decode_f16k_on on stream 0.  Replaces libcuopus.cu:462-468. */
int cuopus_decode_f16k(const uint8_t *ogg, size_t n, float *out_dev, size_t out_cap, int64_t *out_len,
                       char *errbuf, size_t errcap);

/* Decode a mono Ogg Opus stream cut into CUOPUS_SEG_S chains (default 1 s)
 * with CUOPUS_PREROLL_MS preroll (default 250 ms) and resample 48->16 kHz into
 * out_dev (float32, out_cap samples) on cuda_stream.  Replaces
 * libcuopus.cu:238-460 (cuopus_decode_f16k_on). */
int cuopus_decode_f16k_on(const uint8_t *ogg, size_t n, float *out_dev, size_t out_cap, int64_t *out_len,
                          void *cuda_stream, char *errbuf, size_t errcap);

/* N files in one decode launch; per-file output identical to the single-file
 * call.  RC 3 when the merged chain count exceeds CUOPUS_MAX_BATCH.
 * Replaces libcuopus.cu:482-741 (cuopus_decode_f16k_multi). */
int cuopus_decode_f16k_multi(const uint8_t *const *oggs, const size_t *ns, int nfiles, float *const *out_devs,
                             const size_t *out_caps, int64_t *out_lens, void *cuda_stream, char *errbuf,
                             size_t errcap);

/* Pre-size the decoder slots and upload the resampler taps on the current
 * device so the first decode pays only for the decode.  Replaces
 * libcuopus.cu:746-776 (cuopus_warmup). */
int cuopus_warmup(char *errbuf, size_t errcap);

/* 1 if the last call failed on decoder scratch overflow.  This decoder sizes
 * all scratch statically per slot, so it always returns 0.  Replaces
 * libcuopus.cu:201. */
int cuopus_last_arena_overflow(void);

/* Bytes held in grow-only device workspaces.  Replaces libcuopus.cu:203. */
long long cuopus_workspace_bytes(void);

/* Free every workspace.  Replaces libcuopus.cu:205-221. */
void cuopus_release_workspaces(void);

/* ------------------------------------------------------------------ extensions */

/* Extension (no counterpart in the reference, whose f16k paths reject stereo):
 * cuopus_decode_f16k_multi for mono and stereo files.  Each channel of a
 * stereo file is resampled on its own with the same filter and the float32
 * 16 kHz output interleaves the channels; out_caps count floats over all
 * channels, out_lens receive samples per channel, out_channels (may be NULL)
 * the channel count.  Mono output equals cuopus_decode_f16k_multi's. */
int cuopus_decode_f16k_channels(const uint8_t *const *oggs, const size_t *ns, int nfiles, float *const *out_devs,
                                const size_t *out_caps, int64_t *out_lens, int32_t *out_channels, void *cuda_stream,
                                char *errbuf, size_t errcap);

/* Extension (the reference CLI's int16 "DECODE" output, for mono and stereo):
 * decode N files to 48 kHz interleaved int16 playable PCM.  out_caps are in
 * int16 elements; out_lens receive samples per channel; out_channels (may be
 * NULL) the channel count.  Chains as in cuopus_decode_f16k_on.  When the
 * outputs are one buffer with the files back to back in order (out_devs[f] =
 * out_devs[0] + the play samples x channels of the files before f), the
 * decoder writes into it directly, with no workspace and no copy. */
int cuopus_decode_i16_multi(const uint8_t *const *oggs, const size_t *ns, int nfiles, int16_t *const *out_devs,
                            const size_t *out_caps, int64_t *out_lens, int32_t *out_channels, void *cuda_stream,
                            char *errbuf, size_t errcap);

/* Extension: device-resident batch decode, the engine under every entry
 * above.  All pointers are device pointers unless noted.  Chains are decoded
 * by groups of `width` lanes (1..32, a power of two: the reference's
 * "stride"); blocks have `block` threads (32, 64, 96 or 128; 0 = 128).
 * `schedule` 0 = static persistent grid (chain c on group c mod groups),
 * 1 = persistent grid pulling from a device work queue in `order` (host
 * pointer or NULL = identity), 2 = plain one-launch form (one group per
 * chain, the reference kernel's layout).  `max_groups` bounds the groups
 * (0 = fill the GPU).  `graph` != 0 replays the launch (queue reset +
 * kernel) as a CUDA graph, captured on first use for these arguments.
 * pkt_nsamp / pkt_rng (device, may be NULL) receive per-packet sample counts
 * and final ranges at rec_off[c] + k.  res: 4 x uint32 per chain
 * {stop, samples, final_range, time_us}: time_us is the chain's decode time in
 * microseconds (device global timer, at least 1).  kernel_ms (host, may be NULL)
 * receives the decode kernel time measured with events on the stream. */
typedef struct cuopus_batch {
    const uint8_t *data;
    const uint64_t *off;
    const uint32_t *len;
    const uint32_t *first;
    const uint32_t *npkts;
    const uint8_t *channels;
    const uint64_t *trim;
    const uint64_t *keep;
    const uint64_t *out_off;
    int16_t *out;
    const uint64_t *rec_off;
    uint32_t *pkt_nsamp;
    uint32_t *pkt_rng;
    uint32_t *res;
    int32_t nchains;
    int32_t width;
    int32_t schedule;
    int32_t max_groups;
    const uint32_t *order;
    int32_t block;
    int32_t graph;
    int32_t scalar;      /* 1: only the first lane of each group decodes (lane-split loops run
                            serially): the reference kernel's slot layout, for comparison */
    int32_t fec;         /* 1: in-band FEC.  A lost (empty) packet followed by a non-empty one
                            is decoded as opus_decode(next, 5760, decode_fec = 1): the same
                            5760 concealed samples as without FEC, the last frame's worth
                            rebuilt from the next packet's LBRR data.  0: the reference's
                            protocol (decode_fec = 0 for every packet). */
    int32_t light_sms;   /* tail scheduling (queue schedule, not scalar; 0 = off): on the SMs
                            with id < light_sms one decoder warp runs alone and takes the first
                            long_chains positions of `order` first, so the longest chains of an
                            uneven batch decode at the speed of an unshared SM; every other SM
                            runs max_groups / SMs warps (all resident if max_groups is 0).  The
                            launch grid is then every resident group. */
    int32_t long_chains;
} cuopus_batch;

int cuopus_decode_batch(const cuopus_batch *b, void *cuda_stream, float *kernel_ms, char *errbuf, size_t errcap);

/* Extension with no counterpart in the reference: cuopus_decode_batch for
 * callers that cannot allocate device memory -- a process whose device memory
 * is all handed to another framework's pool, or a latency-critical thread that
 * must not call cudaMalloc / cudaFree (they can synchronise the whole device).
 * The caller passes every table and output buffer, as for cuopus_decode_batch;
 * the library allocates nothing: the decoder slots are a static device array
 * of CUOPUS_NOALLOC_MAX_SLOTS slots (about 4.9 MiB) that every GPU loading the
 * library holds until the process exits.  Chains are dealt round-robin to at
 * most that many lane groups; schedule, order, graph, light_sms and
 * long_chains of *b are ignored (there is no queue counter to allocate),
 * width, scalar and fec are honoured as in cuopus_decode_batch (width 0 =
 * cuopus_default_width()), and block 0 picks the largest block whose lane
 * groups fit in the slots (64 threads at width 1, 128 otherwise).
 * max_groups above CUOPUS_NOALLOC_MAX_SLOTS, or a block holding more lane
 * groups than that, is rejected with RC 3.  Packets are staged in shared
 * memory as in cuopus_decode_batch.  The first
 * call on each device looks up the array's device address (with that device
 * current), so make that first call before any stream capture; the call
 * itself refuses to run during capture.  All calls share the one array:
 * calls whose work overlaps on the GPU (other streams, other host threads)
 * race on it and must be serialised by the caller.  Synchronises the stream
 * before it returns. */
#define CUOPUS_NOALLOC_MAX_SLOTS 64
int cuopus_decode_batch_noalloc(const cuopus_batch *b, void *cuda_stream, char *errbuf, size_t errcap);

/* Extension: autotuner of the decode launch.  Decodes the batch `reps` times
 * for every width in widths[0..nwidths) and block size in blocks[0..nblocks)
 * (the schedule, order and graph flag of *b are kept) and returns the pair
 * with the lowest median kernel time.  times_ms (host, may be NULL) receives
 * nwidths x nblocks medians, -1 where the launch was rejected. */
int cuopus_autotune(const cuopus_batch *b, const int32_t *widths, int nwidths, const int32_t *blocks, int nblocks,
                    int reps, void *cuda_stream, int32_t *best_width, int32_t *best_block, float *times_ms,
                    char *errbuf, size_t errcap);

/* Extension: occupancy autotuner of the persistent launch.  Decodes the batch
 * (width, block, schedule, order and graph of *b kept) `reps` times for every
 * count of decoder warps per SM in warps_per_sm[0..n) (0 = every resident
 * group) and returns in *best_max_groups the cuopus_batch.max_groups value
 * (warps per SM x SMs x lane groups per warp, 0 for all) with the lowest
 * median kernel time.
 * Fewer resident warps than the GPU holds can decode faster: the decoder is
 * one large body of code, and with fewer warps per SM at different places in
 * it each warp waits less for instructions, so a chain decodes faster and the
 * longest chains finish sooner.  times_ms (may be NULL) receives n medians. */
int cuopus_autotune_occupancy(const cuopus_batch *b, const int32_t *warps_per_sm, int n, int reps,
                              void *cuda_stream, int32_t *best_max_groups, float *times_ms, char *errbuf,
                              size_t errcap);

/* ---- Extension: learned cost model of the queue schedule (no counterpart in
 * the reference).  An FP32 MLP 16 -> 64 -> 64 -> 1 (ReLU) predicts a chain's
 * log decode time from 16 features of its packets' TOC bytes; chains are
 * queued longest first by the prediction.  It orders work only: decoded
 * samples do not depend on it.  All buffers are device pointers. */
#define CUOPUS_MLP_FEATURES 16
#define CUOPUS_MLP_HIDDEN 64
#define CUOPUS_MLP_NPARAM (16 * 64 + 64 + 64 * 64 + 64 + 64 + 1)

/* feat_dev[c * 16 + k]: log1p packets, log1p bytes, log1p frames, log1p
 * seconds, channels - 1, SILK / hybrid / CELT frame fractions, 2.5 / 5 / 10 /
 * 20 / >= 40 ms frame fractions, mean bandwidth / 4, stereo-flag packet
 * fraction, log1p bytes per second; from the tables of *b. */
int cuopus_chain_features(const cuopus_batch *b, float *feat_dev, void *cuda_stream, char *errbuf, size_t errcap);
/* He-uniform weights from `seed`, zero biases. */
int cuopus_mlp_init(float *params_dev, uint64_t seed, void *cuda_stream, char *errbuf, size_t errcap);
/* y_dev[s] = network(x_dev[s * 16 ..]). */
int cuopus_mlp_predict(const float *params_dev, const float *x_dev, int n, float *y_dev, void *cuda_stream,
                       char *errbuf, size_t errcap);
/* Gradient of mean_s (y_s - t_s)^2 in the parameter layout, and the loss. */
int cuopus_mlp_grad(const float *params_dev, const float *x_dev, const float *t_dev, int n, float *grad_dev,
                    float *loss_dev, void *cuda_stream, char *errbuf, size_t errcap);
/* Full-batch Adam (steps rounded up to a multiple of 50, replayed as a CUDA
 * graph); losses (host, may be NULL) receives the loss before each step. */
int cuopus_mlp_train(float *params_dev, const float *x_dev, const float *t_dev, int n, int steps, float lr,
                     float *losses, void *cuda_stream, char *errbuf, size_t errcap);

/* ---- Extension: the visiting order of the file entry points (no counterpart
 * in the reference).  They queue chains longest first by an additive cost: the
 * sum over a chain's packets of non-negative weights times the packet's
 * features, plus a constant per chain.  The weights are fitted by
 * non-negative least squares to per-chain device times of a training corpus,
 * one set for 8 lanes per chain and one for 32.  Host pointers; the tables are
 * those of cuopus_batch.  feat receives nchains x CUOPUS_ORDER_FEATURES values:
 * 1 (chain constant), packets, bytes / 100, frames per (mode, duration) class
 * and TOC stereo bit (SILK 10/20/40/60 ms, hybrid 10/20, CELT 2.5/5/10/20;
 * mono then stereo for each), SILK ms x bandwidth (NB 0..WB 2), CELT ms x
 * bandwidth (NB 0..FB 3), ms decoded to a stereo output, empty packets.
 * cost[c] = weights(width) . feat[c].  cuopus_order_model_fitted() is 0 while
 * the weights are the unfitted default (decoded duration x channels). */
#define CUOPUS_ORDER_FEATURES 27
int cuopus_order_features(const uint8_t *blob, const uint64_t *off, const uint32_t *len, const uint32_t *first,
                          const uint32_t *npkts, const uint8_t *channels, int32_t nchains, double *feat);
int cuopus_order_costs(const uint8_t *blob, const uint64_t *off, const uint32_t *len, const uint32_t *first,
                       const uint32_t *npkts, const uint8_t *channels, int32_t nchains, int32_t width,
                       double *cost);
int cuopus_order_model_fitted(void);
/* w receives the CUOPUS_ORDER_FEATURES weights used for `width` lanes. */
int cuopus_order_weights(int32_t width, double *w);

/* ---- Extension: continuous-batching decode server (no counterpart in the
 * reference, whose daemon decodes one request at a time, decode_cli.cu:572-678).
 * Requests are demuxed on the submitting thread and admitted, oldest first,
 * when their packets, PCM and output fit in a device arena of budget_bytes
 * allocated once at creation; their chains are packed into decode waves of at
 * most wave_chains chains, up to max_inflight waves in flight on the server's
 * own streams, so requests that arrive while others decode join the next wave.
 * The server owns one host thread and max_inflight streams on the device that
 * is current at creation.  Results are identical to the one-shot entry points
 * (a fresh decoder per chain).  Return codes as above, plus 4 = timeout. */
typedef struct cuopus_server cuopus_server;
typedef struct cuopus_server_config {
    int64_t budget_bytes;   /* device arena for admitted requests (0 = 40 GiB) */
    int32_t width;          /* lanes per chain (0 = 8 for chains of up to 4 s, else 32) */
    int32_t block;          /* threads per block (0 = 64) */
    int32_t max_inflight;   /* decode waves in flight (0 = 8); with two or more in flight a
                               wave waits until it is half full or its oldest chain has
                               waited 5 ms */
    int32_t wave_chains;    /* chains per wave (0 = the resident lane groups of the GPU) */
    double seg_s;           /* chain length (0 = 1 s) */
    double preroll_ms;      /* chain preroll (0 = 250 ms) */
    int32_t f16k;           /* 1: float32 16 kHz output (mono only); 0: int16 48 kHz interleaved */
} cuopus_server_config;
typedef struct cuopus_server_stats {
    int64_t completed, failed, waves, chains, pending, active;
    int64_t arena_used, arena_bytes, wave_chains;
    double audio_s;         /* playable audio seconds of completed requests */
    double wall_ms;         /* first submit to last completion */
    double p50_ms, p99_ms, max_ms;   /* request latency, submit to completion */
} cuopus_server_stats;

int cuopus_server_create(const cuopus_server_config *cfg, cuopus_server **out, char *errbuf, size_t errcap);
/* Queue one Ogg Opus stream; *id identifies it.  RC 1 for a stream that does
 * not demux (nothing is queued). */
int cuopus_server_submit(cuopus_server *s, const uint8_t *ogg, size_t n, uint64_t *id, char *errbuf, size_t errcap);
/* Wait for a request (timeout_ms < 0: forever), copy its output to host_out
 * (may be NULL) and release it.  out_samples: samples per channel (int16) or
 * 16 kHz samples (f16k); latency_ms: submit to completion. */
int cuopus_server_wait(cuopus_server *s, uint64_t id, int64_t timeout_ms, void *host_out, size_t out_cap_bytes,
                       int64_t *out_samples, int32_t *channels, double *latency_ms, char *errbuf, size_t errcap);
int cuopus_server_get_stats(cuopus_server *s, cuopus_server_stats *st);
/* Output size of a submitted request, known from its demux at submit: samples
 * per channel (int16) or 16 kHz samples (f16k), the channel count, and the
 * bytes cuopus_server_wait writes.  RC 3 for an unknown id. */
int cuopus_server_request_size(cuopus_server *s, uint64_t id, int64_t *out_samples, int32_t *channels,
                               size_t *out_bytes);
/* Finish admitted work, drop queued requests, free everything. */
void cuopus_server_destroy(cuopus_server *s);

/* Extension: fp32 48->16 kHz resample of a device int16 mono stream (the
 * kernel behind the f16k entries): out[i], i < n_out, from in[0..avail). */
int cuopus_resample48to16(const int16_t *in_dev, int64_t avail, int64_t n_out, float *out_dev, void *cuda_stream,
                          char *errbuf, size_t errcap);

/* Extension (host only, mono or stereo): demux + validate; play48 receives
 * the playable samples per channel at 48 kHz and channels the channel count. */
int cuopus_probe_pcm(const uint8_t *ogg, size_t n, int64_t *play48, int32_t *channels, char *errbuf,
                     size_t errcap);

/* Extension: the host demuxer and chain builder (the reference CLI's
 * --dump-blob / --dump-chains data, cuopus_demux.h:79-378).  Two calls: with
 * blob == NULL only the counts are returned; then pass arrays of those sizes.
 * seg_s / preroll_ms choose the chains (1.0 / 250.0 in the entry points above);
 * require_mono applies the f16k entry points' mono check. */
int cuopus_index(const uint8_t *ogg, size_t n, double seg_s, double preroll_ms, int require_mono,
                 int64_t *n_packets, int64_t *n_chains, int64_t *blob_bytes, int32_t *channels, int64_t *play48,
                 uint8_t *blob, uint64_t *pkt_off, uint32_t *pkt_len, uint32_t *first, uint32_t *npkts,
                 uint32_t *trim, uint32_t *keep, char *errbuf, size_t errcap);

/* Extension: timings and sizes of the last successful decode call of the
 * entry points above (the reference CLI's per-request report,
 * decode_cli.cu:486-491, 656-664): host demux, upload, decode kernel and
 * resampler times, chains, packets and playable samples at 48 kHz. */
typedef struct cuopus_stats {
    double demux_ms;
    float h2d_ms;
    float kernel_ms;
    float resample_ms;
    int64_t chains;
    int64_t packets;
    int64_t play48;
    int32_t width;      /* lanes per chain the call decoded with */
} cuopus_stats;

int cuopus_last_stats(cuopus_stats *s);

/* Extension: bytes of device state per decoder slot, and the number of lanes
 * per chain cuopus_decode_batch uses when its width is 0 (CUOPUS_STRIDE,
 * default 32).  The file entry points choose 32 or 8 lanes per call from the
 * chains' lengths unless CUOPUS_STRIDE is set (cuopus_stats.width reports it). */
long long cuopus_slot_bytes(void);
int cuopus_default_width(void);

#ifdef __cplusplus
}
#endif

#endif /* CUOPUS_H */
