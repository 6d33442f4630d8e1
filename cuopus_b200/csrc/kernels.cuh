// Device kernels of libcuopus (sm_100a).
//
//   k_decode_chains   one decoder per group of `width` lanes; the groups of a
//                     launch are resident decoder slots.  Two schedules:
//                       plain      chain c goes to group c % ngroups (static)
//                       queue      groups pull chain indices from a device
//                                  counter in the order given by `order`
//                                  (longest first when the host sorts it);
//                                  the loop is bounded by the chain count
//   k_resample48to16  49-tap Kaiser-windowed sinc, 3:1 decimation of the
//                     compacted int16 48 kHz stream into fp32 16 kHz: input
//                     tiles staged in shared memory, each thread emits four
//                     consecutive outputs as one float4 store.
//
// Arithmetic of the resampler follows the reference kernel
// (cuopus_kernels.cuh:96-111): acc starts at 0 and adds taps[t] * x/32768
// for t = 0..48 in order with a fused multiply-add, samples outside the
// stream read as zero.
#pragma once
#include "dec/chain.cuh"

namespace cuo {

struct DecodeArgs {
    const uint8_t *data;        // packet bytes
    const uint64_t *off;        // per packet offset
    const uint32_t *len;        // per packet length
    const uint32_t *first;      // per chain first packet
    const uint32_t *npkts;      // per chain packet count
    const uint8_t *channels;    // per chain channel count (1 or 2)
    const uint64_t *trim;       // per chain samples to drop (per channel)
    const uint64_t *keep;       // per chain samples to keep (per channel)
    const uint64_t *out_off;    // per chain int16 element offset into out
    int16_t *out;               // kept PCM, interleaved
    const uint32_t *order;      // queue schedule: chain visiting order (may be null)
    const uint64_t *rec_off;    // per chain first per-packet record (may be null)
    uint32_t *pkt_nsamp;        // per-packet records (may be null)
    uint32_t *pkt_rng;
    ChainResult *res;           // per chain result
    ChainSlot *slots;           // one per group of the launch
    unsigned *queue_head;       // queue schedule: next position in `order`
    int nchains;
    int width;                  // lanes per chain: 1, 2, 4, 8, 16 or 32
    int use_queue;
    int stage;                  // packets staged in shared memory (STAGE_BYTES per group)
    int scalar;                 // one active lane per group (the reference kernel's slot layout)
    int fec;                    // in-band FEC for lost packets (decode_chain)
    // Tail scheduling (queue schedule, light_sms > 0): the warps of SMs whose id
    // is below light_sms keep only light_warps of themselves and take the
    // first long_chains positions of the order first; every other SM keeps
    // heavy_warps.  queue_head[0] counts the long positions, queue_head[1] the
    // rest; sm_rank[smid] counts the warps that arrived on each SM.
    unsigned *sm_rank;
    int light_sms, light_warps, heavy_warps, long_chains;
};

// Number of SM ids sm_rank covers (%smid is masked to it).
enum { SM_RANK_SLOTS = 256 };

// Shared memory a block of `block` threads at `width` lanes per chain uses for
// packet staging; 0 (no staging) when it would exceed 48 KB per block.
// Packet staging takes shared memory from the SM's unified L1 / shared
// storage; CUOPUS_STAGE=0 turns it off (all of that storage stays L1).
inline int stage_smem_bytes(int block, int width)
{
    const char *e = getenv("CUOPUS_STAGE");
    if (e && e[0] == '0' && e[1] == 0) return 0;
    int bytes = (block / width) * (int)STAGE_BYTES;
    return bytes <= 48 * 1024 ? bytes : 0;
}

// Decoder kernel: defined in decode_kernel.cu, which is compiled on its own
// (see the note there); the host side reaches it through these calls.  The
// launch decides packet staging from block and width (stage_smem_bytes).
cudaError_t decode_kernel_occupancy(int block, int width, int *blocks_per_sm);
cudaError_t decode_kernel_launch(const DecodeArgs &a, int blocks, int block, cudaStream_t st);

// The 48 -> 16 kHz resampler of libcuopus.cu for other host translation units:
// uploads the taps to the current device on first use, then launches on st.
cudaError_t resample_into(const int16_t *in, long long avail, long long n_out, float *out, cudaStream_t st);

#ifdef CUO_DECODE_KERNEL_TU
// The device's global nanosecond timer (PTX %globaltimer).
__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Next queue position under tail scheduling: light groups take the long
// positions [0, long_chains) first, the others the rest; each takes from the
// other part when its own is used up.  nchains when nothing is left.
__device__ __forceinline__ unsigned queue_next(const DecodeArgs &a, int light)
{
    const unsigned K = (unsigned)a.long_chains, n = (unsigned)a.nchains;
    if (light) {
        unsigned v = atomicAdd(&a.queue_head[0], 1u);
        if (v < K) return v;
        v = K + atomicAdd(&a.queue_head[1], 1u);
        return v < n ? v : n;
    }
    unsigned v = K + atomicAdd(&a.queue_head[1], 1u);
    if (v < n) return v;
    v = atomicAdd(&a.queue_head[0], 1u);
    return v < K ? v : n;
}

// MIN_BLOCKS: resident 128-thread blocks per SM the register allocation is
// sized for (decode_kernel.cu instantiates 1 and 3 and says which runs when).
template <int MIN_BLOCKS>
__global__ void __launch_bounds__(128, MIN_BLOCKS) k_decode_chains(DecodeArgs a)
{
    const int W = a.width;
    const int lane = threadIdx.x & 31;
    const int sub = lane / W;
    Lanes L;
    L.id = lane - sub * W;
    L.n = W;
    L.mask = W == 32 ? 0xffffffffu : (((1u << W) - 1u) << (sub * W));
    if (a.scalar) {            // the group's first lane decodes alone; the others idle
        if (L.id != 0) return;
        L.n = 1;
        L.mask = 1u << lane;
    }
    const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int group = (int)(gtid / W);
    const int ngroups = (int)((long long)gridDim.x * blockDim.x / W);
    ChainSlot *slot = a.slots + group;
    extern __shared__ __align__(16) uint8_t s_stage[];
    PacketStage S;
    PacketStage *stage = nullptr;
    if (a.stage) {
        stage_init(L, S, s_stage + (size_t)(threadIdx.x / W) * STAGE_BYTES);
        stage = &S;
    }
    int light = 0;
    if (a.light_sms > 0) {   // tail scheduling: keep this warp or leave (whole warps, before any decoding)
        unsigned smid, r = 0;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        if (lane == 0) r = atomicAdd(&a.sm_rank[smid % SM_RANK_SLOTS], 1u);
        r = __shfl_sync(0xffffffffu, r, 0);
        light = smid < (unsigned)a.light_sms;
        if ((int)r >= (light ? a.light_warps : a.heavy_warps)) {
            if (stage) stage_drain(L, *stage);
            return;
        }
    }
    for (int it = 0; it < a.nchains; it++) {
        int pos;
        if (a.use_queue) {
            unsigned v = 0;
            if (L.id == 0) v = a.long_chains > 0 ? queue_next(a, light) : atomicAdd(a.queue_head, 1u);
            v = __shfl_sync(L.mask, v, sub * W);
            pos = (int)v;
        } else {
            pos = group + it * ngroups;
        }
        if (pos >= a.nchains) break;
        int c = a.order ? (int)a.order[pos] : pos;
        unsigned long long t0 = globaltimer_ns();
        decode_chain(L, slot, a.data, a.off, a.len, a.first[c], a.npkts[c], a.channels[c],
                     a.out ? a.out + a.out_off[c] : nullptr, a.trim[c], a.keep[c],
                     a.pkt_nsamp ? a.pkt_nsamp + a.rec_off[c] : nullptr,
                     a.pkt_rng ? a.pkt_rng + a.rec_off[c] : nullptr, &a.res[c], stage, a.fec);
        unsigned long long us = (globaltimer_ns() - t0) / 1000ull;
        if (L.id == 0) a.res[c].time_us = (uint32_t)(us < 1 ? 1 : us > 0xffffffffull ? 0xffffffffull : us);
    }
}
#endif

// The resampler kernel and its taps belong to libcuopus.cu; other host
// translation units define CUO_NO_RESAMPLE_KERNEL and use resample_into.
#if !defined(CUO_DECODE_KERNEL_TU) && !defined(CUO_NO_RESAMPLE_KERNEL)
enum { RS_TAPS = 49, RS_PAD = 24, RS_OUT_PER_THREAD = 4, RS_THREADS = 256,
       RS_TILE_OUT = RS_THREADS * RS_OUT_PER_THREAD, RS_TILE_IN = 3 * RS_TILE_OUT + RS_TAPS - 1 };

__constant__ float c_rs_taps[RS_TAPS];

// out[i * chans] for i in [0, n_out): taps over in[(3 i - 24 + t) * chans], the
// input valid for sample indices [0, avail); chans > 1 resamples one channel of
// an interleaved stream into one channel of an interleaved output.
__global__ void __launch_bounds__(RS_THREADS) k_resample48to16(const int16_t *__restrict__ in, long long avail,
                                                               long long n_out, float *__restrict__ out, int chans)
{
    __shared__ float xs[RS_TILE_IN];
    const long long o0 = (long long)blockIdx.x * RS_TILE_OUT;
    const long long base = 3 * o0 - RS_PAD;
    for (int i = threadIdx.x; i < RS_TILE_IN; i += RS_THREADS) {
        long long g = base + i;
        xs[i] = (g >= 0 && g < avail) ? (float)in[g * chans] * (1.0f / 32768.0f) : 0.0f;
    }
    __syncthreads();
    const int j0 = threadIdx.x * RS_OUT_PER_THREAD;
    float acc[RS_OUT_PER_THREAD];
#pragma unroll
    for (int k = 0; k < RS_OUT_PER_THREAD; k++) {
        float a = 0.0f;
        const float *x = xs + 3 * (j0 + k);
#pragma unroll
        for (int t = 0; t < RS_TAPS; t++) a = __fmaf_rn(c_rs_taps[t], x[t], a);
        acc[k] = a;
    }
    long long i0 = o0 + j0;
    if (chans == 1 && i0 + RS_OUT_PER_THREAD <= n_out && ((((uintptr_t)(out + i0)) & 15) == 0)) {
        *reinterpret_cast<float4 *>(out + i0) = make_float4(acc[0], acc[1], acc[2], acc[3]);
    } else {
#pragma unroll
        for (int k = 0; k < RS_OUT_PER_THREAD; k++)
            if (i0 + k < n_out) out[(i0 + k) * chans] = acc[k];
    }
}
#endif

} // namespace cuo
