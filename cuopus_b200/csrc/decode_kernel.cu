// Translation unit of the chain decoder kernel (k_decode_chains).
//
// It is compiled apart from the rest of libcuopus, at NVVM -O1 and ptxas -O1:
//   * code size: the kernel is one large body of codec paths (SILK, CELT,
//     hybrid, PLC), and with every decoder slot busy its warps stall mostly on
//     instruction fetch (ncu: 6.1 cycles per issued instruction).  NVVM -O1
//     unrolls and duplicates less; the machine code shrinks from 1.17 MB to
//     0.79 MB and a loaded GPU decodes about 20 % more audio per second, with
//     identical output;
//   * with NVVM -O3, ptxas -O2 and -O3 decoded stereo SILK and hybrid frames
//     with wrong samples (the mid/side to left/right stage diverged from
//     libopus on the first stereo frame), while ptxas -O0 / -O1, nvcc -G and
//     the same sources built for the host with g++ (also under ASan / UBSan,
//     and with every local variable pattern-initialised) were bit-exact.
// The GPU parity tests hold the shipped build to libopus on stereo streams.
#define CUO_DECODE_KERNEL_TU 1
#include <cuda_runtime.h>
#include <stdio.h>

#include <atomic>
#include <string.h>

#include "../../include/cuopus.h"
#include "kernels.cuh"

namespace cuo {

// Two instances of the decoder kernel.  Groups of 8 lanes or fewer put 4 or
// more chains in each warp, and throughput is what such launches are for (1 s
// chains of long files, the server's waves): they run the instance compiled
// for 3 resident 128-thread blocks (at most 170 registers, so 12 warps per SM
// at 64-thread blocks instead of 8), whose chains each decode slower (spills)
// but more of them are in flight: the 2 h file in 1 s chains at 8 lanes,
// 179-180 ms against 188-189 (same box, alternating; sized for 4 blocks, 128
// registers, 239 ms: the spills outweigh the extra warps).  Wider groups decode the
// long chains that set an uneven batch's step, with few warps per SM: they
// run the instance with the full register budget (255), which decodes each
// chain faster (the mixed batch at 5 warps per SM: 2,401-2,496 ms against
// 2,798-2,803 with the register cap).
static bool dense_instance(int width) { return width <= 8; }

cudaError_t decode_kernel_occupancy(int block, int width, int *blocks_per_sm)
{
    size_t smem = (size_t)stage_smem_bytes(block, width);
    if (dense_instance(width))
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_decode_chains<3>, block, smem);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_decode_chains<1>, block, smem);
}

cudaError_t decode_kernel_launch(const DecodeArgs &a, int blocks, int block, cudaStream_t st)
{
    DecodeArgs b = a;
    int smem = stage_smem_bytes(block, a.width);
    b.stage = smem > 0;
    if (dense_instance(a.width)) k_decode_chains<3><<<blocks, block, (size_t)smem, st>>>(b);
    else k_decode_chains<1><<<blocks, block, (size_t)smem, st>>>(b);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ allocation-free decode

// Decoder slots of cuopus_decode_batch_noalloc: a fixed array in the
// library's device image instead of a cudaMalloc'd workspace.  Every GPU that
// loads the library holds it (CUOPUS_NOALLOC_MAX_SLOTS x sizeof(ChainSlot),
// about 4.9 MiB) until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_slots[CUOPUS_NOALLOC_MAX_SLOTS * sizeof(ChainSlot)];

// Device address of g_noalloc_slots per device, looked up once with that
// device current.  In host code the array's name is only a host-side stand-in
// for the symbol, never a device address, so the kernel gets this pointer.
// Atomic so that first calls from several host threads (on one device or on
// different ones) do not race on the lookup; a lookup done twice stores the
// same address.
static std::atomic<void *> g_noalloc_ptr[64];

} // namespace cuo

static int noalloc_err(char *errbuf, size_t errcap, int rc, const char *msg, cudaError_t e)
{
    if (errbuf && errcap) {
        if (e != cudaSuccess) snprintf(errbuf, errcap, "%s: %s", msg, cudaGetErrorString(e));
        else snprintf(errbuf, errcap, "%s", msg);
    }
    return rc;
}

extern "C" int cuopus_default_width(void);

// The caller owns every table and output buffer (as in cuopus_decode_batch);
// this entry point allocates nothing: decoder slots come from the static
// array above, chains are dealt round-robin to at most
// CUOPUS_NOALLOC_MAX_SLOTS resident groups, and no events, streams or graphs
// are created.  Packets are staged in the launch's dynamic shared memory, as
// in cuopus_decode_batch.  Nothing in the slots needs clearing: a group
// initialises its slot at the start of every chain and reads nothing it has
// not written.
extern "C" int cuopus_decode_batch_noalloc(const cuopus_batch *b, void *cuda_stream, char *errbuf, size_t errcap)
{
    using namespace cuo;
    if (errbuf && errcap) errbuf[0] = 0;
    if (!b) return noalloc_err(errbuf, errcap, 3, "batch is NULL", cudaSuccess);
    if (b->nchains <= 0) return 0;
    int width = b->width > 0 ? b->width : cuopus_default_width();
    if (width != 1 && width != 2 && width != 4 && width != 8 && width != 16 && width != 32)
        return noalloc_err(errbuf, errcap, 3, "width is not a power of two <= 32", cudaSuccess);
    int block = b->block;
    if (block <= 0) {   // the largest block whose lane groups fit in the static slots
        block = 0;
        for (int cand = 128; cand >= 32 && !block; cand -= 32)
            if (cand % width == 0 && cand / width <= CUOPUS_NOALLOC_MAX_SLOTS) block = cand;
    }
    if ((block != 32 && block != 64 && block != 96 && block != 128) || block % width)
        return noalloc_err(errbuf, errcap, 3, "block must be 32, 64, 96 or 128 threads and a multiple of width",
                           cudaSuccess);
    if (block / width > CUOPUS_NOALLOC_MAX_SLOTS)
        return noalloc_err(errbuf, errcap, 3, "block holds more lane groups than there are static decoder slots",
                           cudaSuccess);
    if (!b->data || !b->off || !b->len || !b->first || !b->npkts || !b->channels || !b->trim || !b->keep ||
        !b->res || (b->out && !b->out_off) || ((b->pkt_nsamp || b->pkt_rng) && !b->rec_off))
        return noalloc_err(errbuf, errcap, 3, "batch has a NULL table", cudaSuccess);
    if (b->max_groups > CUOPUS_NOALLOC_MAX_SLOTS) {
        char m[128];
        snprintf(m, sizeof m, "max_groups %d exceeds the %d static decoder slots", b->max_groups,
                 CUOPUS_NOALLOC_MAX_SLOTS);
        return noalloc_err(errbuf, errcap, 3, m, cudaSuccess);
    }
    cudaStream_t st = (cudaStream_t)cuda_stream;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
        return noalloc_err(errbuf, errcap, 3, "refusing to decode during CUDA stream capture", cudaSuccess);
    cudaGetLastError();
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_err(errbuf, errcap, 2, "cudaGetDevice", e);
    if (dev < 0 || dev >= 64) return noalloc_err(errbuf, errcap, 3, "device index out of range", cudaSuccess);
    void *slots = g_noalloc_ptr[dev].load(std::memory_order_acquire);
    if (!slots) {
        e = cudaGetSymbolAddress(&slots, g_noalloc_slots);
        if (e != cudaSuccess) return noalloc_err(errbuf, errcap, 2, "cudaGetSymbolAddress of the decoder slots", e);
        g_noalloc_ptr[dev].store(slots, std::memory_order_release);
    }
    long long groups = b->nchains;
    long long cap = b->max_groups > 0 ? b->max_groups : CUOPUS_NOALLOC_MAX_SLOTS;
    if (groups > cap) groups = cap;
    int gpb = block / width;
    int blocks = (int)((groups + gpb - 1) / gpb);
    if ((long long)blocks * gpb > CUOPUS_NOALLOC_MAX_SLOTS) blocks = CUOPUS_NOALLOC_MAX_SLOTS / gpb;
    DecodeArgs a;
    memset(&a, 0, sizeof a);
    a.data = b->data;
    a.off = b->off;
    a.len = b->len;
    a.first = b->first;
    a.npkts = b->npkts;
    a.channels = b->channels;
    a.trim = b->trim;
    a.keep = b->keep;
    a.out_off = b->out_off;
    a.out = b->out;
    a.order = nullptr;
    a.rec_off = b->rec_off;
    a.pkt_nsamp = b->pkt_nsamp;
    a.pkt_rng = b->pkt_rng;
    a.res = (ChainResult *)b->res;
    a.slots = (ChainSlot *)slots;
    a.queue_head = nullptr;
    a.nchains = b->nchains;
    a.width = width;
    a.use_queue = 0;
    a.scalar = b->scalar != 0;
    a.fec = b->fec != 0;
    e = decode_kernel_launch(a, blocks, block, st);
    if (e != cudaSuccess) return noalloc_err(errbuf, errcap, 2, "decode launch", e);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return noalloc_err(errbuf, errcap, 2, "decode", e);
    return 0;
}

#ifdef CUO_PHASE_TIMERS
#include "../../include/cuopus_phases.h"

// Stage timers of the diagnostic build (libcuopus_phases.so only): cycles per
// decoder stage summed over every chain of every launch since the last reset.
namespace cuo {
__device__ unsigned long long g_phase_cycles[PH_COUNT];
__device__ void cuo_phase_add(int stage, long long cycles)
{
    atomicAdd(&g_phase_cycles[stage], (unsigned long long)cycles);
}
} // namespace cuo

extern "C" int cuopus_phase_count(void) { return cuo::PH_COUNT; }

extern "C" int cuopus_phase_read(uint64_t *out)
{
    return cudaMemcpyFromSymbol(out, cuo::g_phase_cycles, sizeof(cuo::g_phase_cycles)) == cudaSuccess ? 0 : 2;
}

extern "C" int cuopus_phase_reset(void)
{
    static const unsigned long long zero[cuo::PH_COUNT] = {};
    return cudaMemcpyToSymbol(cuo::g_phase_cycles, zero, sizeof zero) == cudaSuccess ? 0 : 2;
}
#endif
