// libcuopus.so: C ABI of the batch decoder (declarations and the meaning of
// every entry point: include/cuopus.h).
//
// Host orchestration restated from the reference's libcuopus.cu: demux and
// chain tables on the host, validation of every chain against its TOC
// capacity before success is returned, RC / errbuf conventions, the refusal
// to run while the caller's stream captures, grow-only process-global
// workspaces.  The B200 design differs in how the work is laid out:
//   * all chains of a call go to one decode launch (no 2048-chain batching
//     with resampler carries); the launch is sized to the resident decoder
//     slots of the GPU and chains are assigned statically or pulled from a
//     device work queue;
//   * the decode kernel writes only the kept samples, straight into the
//     compacted stream (no separate compaction kernel, no preroll PCM buffer);
//   * decoder state and scratch live in per-slot global memory (no per-thread
//     bump arena), so arena overflow cannot happen.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <functional>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cuopus.h"
#include "kernels.cuh"
#include "ogg_demux.h"
#include "ordercost.h"

namespace {

enum { RC_OK = 0, RC_SOFT = 1, RC_CUDA = 2, RC_ARG = 3 };
const int BLOCK = 128;
// work queue: two position counters (tail scheduling uses both) and the
// per-SM warp counters of tail scheduling
const size_t QUEUE_BYTES = (2 + cuo::SM_RANK_SLOTS) * sizeof(unsigned);
const double SWR_TAIL_48K = 48;   // samples the CPU path never flushes (libcuopus.cu:195-199)

struct Err {
    char *buf;
    size_t cap;
    char scratch[8];
    Err(char *b, size_t c)
    {
        if (b && c) { buf = b; cap = c; }
        else { buf = scratch; cap = sizeof scratch; }
        buf[0] = 0;
    }
    int set(int rc, const char *fmt, ...)
    {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, cap, fmt, ap);
        va_end(ap);
        return rc;
    }
};

#define CK(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return err.set(RC_CUDA, "CUDA error %s at %s:%d: %s", #call, __FILE__, __LINE__,       \
                           cudaGetErrorString(e_));                                                 \
    } while (0)

struct Grow {
    void *p = nullptr;
    size_t cap = 0;
};

struct State {
    Grow data, off, len, first, npkts, chans, trim, keep, out_off, order, res, slots, queue, pcm;
    Grow hpin;
    long long dev_bytes = 0;
    int taps_dev = -1;
    int occ_dev = -1, occ_blocks = 0, sm_count = 0;
    int occ[5][6] = {};                          // resident blocks per SM by [warps per block][log2 width]
    // decode launch captured as a CUDA graph (queue reset + kernel) and its key
    cudaGraphExec_t gexec = nullptr;
    cudaStream_t cap_stream = nullptr;
    int cap_dev = -1, g_dev = -1, g_blocks = 0, g_block = 0;
    cuo::DecodeArgs g_args;
    float last_kernel_ms = 0.f;
    int last_ovf = 0;
    int last_width = 0;                          // lanes per chain of the last file-entry decode
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;     // decode kernel
    cudaEvent_t evh0 = nullptr, evh1 = nullptr;   // packet / table upload
    cudaEvent_t evr0 = nullptr, evr1 = nullptr;   // resampler
    int ev_dev = -1;
    cuopus_stats last{};
} G;

std::mutex g_mu;

int gpu_grow(Grow &g, size_t need, Err &err)
{
    if (need == 0) need = 1;
    if (need <= g.cap) return RC_OK;
    if (g.p) {
        cudaFree(g.p);
        G.dev_bytes -= (long long)g.cap;
        g.p = nullptr;
        g.cap = 0;
    }
    cudaError_t e = cudaMalloc(&g.p, need);
    if (e != cudaSuccess) return err.set(RC_CUDA, "cudaMalloc %zu bytes: %s", need, cudaGetErrorString(e));
    g.cap = need;
    G.dev_bytes += (long long)need;
    return RC_OK;
}

int pin_grow(Grow &g, size_t need, Err &err)
{
    if (need == 0) need = 1;
    if (need <= g.cap) return RC_OK;
    if (g.p) cudaFreeHost(g.p);
    g.p = nullptr;
    g.cap = 0;
    cudaError_t e = cudaMallocHost(&g.p, need);
    if (e != cudaSuccess) return err.set(RC_CUDA, "cudaMallocHost %zu bytes: %s", need, cudaGetErrorString(e));
    g.cap = need;
    return RC_OK;
}

double env_f(const char *name, double dflt)
{
    const char *e = getenv(name);
    return (e && *e) ? atof(e) : dflt;
}
int env_i(const char *name, int dflt)
{
    const char *e = getenv(name);
    return (e && atoi(e) > 0) ? atoi(e) : dflt;
}

int default_width()
{
    int w = env_i("CUOPUS_STRIDE", 32);
    int p = 1;
    while (p * 2 <= w && p < 32) p *= 2;
    return p;
}

// Decoder warps per SM of the library's own launches (CUOPUS_WARPS_PER_SM).
// At 32 lanes per chain the default is 5, fewer than the GPU holds (8 at
// 128-thread blocks): the decoder waits on instruction fetch when more of its
// warps share an SM, so each chain decodes faster and the longest chains
// finish sooner (the occupancy autotuner measured 5 per SM best on the mixed
// batch).  At narrower widths a warp decodes several chains and the default
// is every resident group (the 2 h file in 1 s chains at 8 lanes per chain
// decoded in 151 ms with every group, 232 ms at 5 warps per SM).  Returns the
// cuopus_batch.max_groups value for `width` lanes per chain (0 = all).
int default_max_groups(int width)
{
    int wps = env_i("CUOPUS_WARPS_PER_SM", width == 32 ? 5 : 0);
    if (G.sm_count <= 0 || wps <= 0) return 0;
    return wps * G.sm_count * (32 / width);
}

int refuse_capture(cudaStream_t st, Err &err)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cs);
    if (e == cudaSuccess && cs != cudaStreamCaptureStatusNone)
        return err.set(RC_ARG, "refusing to decode during CUDA stream capture");
    cudaGetLastError();
    return RC_OK;
}

// Kaiser-windowed sinc low-pass at 1/3 of the 48 kHz Nyquist rate, 49 taps,
// beta 8.6, normalised to unity DC gain; computed in double, rounded to float.
void make_taps(float *taps)
{
    const int n = cuo::RS_TAPS;
    const double beta = 8.6, cutoff = 1.0 / 3.0;
    auto i0 = [](double x) {   // modified Bessel function of order 0, power series
        double sum = 1.0, term = 1.0, q = x * x / 4.0;
        for (int k = 1; k < 64; k++) {
            term *= q / ((double)k * k);
            sum += term;
            if (term < 1e-18 * sum) break;
        }
        return sum;
    };
    double h[cuo::RS_TAPS], total = 0.0;
    for (int i = 0; i < n; i++) {
        double m = i - (n - 1) / 2.0;
        double sinc = (m == 0.0) ? cutoff : sin(M_PI * cutoff * m) / (M_PI * m);
        double r = 2.0 * i / (n - 1) - 1.0;
        double win = i0(beta * sqrt(1.0 - r * r)) / i0(beta);
        h[i] = sinc * win;
        total += h[i];
    }
    for (int i = 0; i < n; i++) taps[i] = (float)(h[i] / total);
}

std::mutex g_taps_mu;   // the taps upload is also reached from the server thread

int ensure_taps(cudaStream_t st, Err &err)
{
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_taps_mu);
    if (G.taps_dev == dev) return RC_OK;
    float taps[cuo::RS_TAPS];
    make_taps(taps);
    CK(cudaMemcpyToSymbolAsync(cuo::c_rs_taps, taps, sizeof taps, 0, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    G.taps_dev = dev;
    return RC_OK;
}

// Resident blocks per SM of the decode kernel at the block sizes the engine
// launches (32, 64, 96 or 128 threads), per device.
int ensure_occupancy(Err &err)
{
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (G.occ_dev == dev) return RC_OK;
    CK(cudaDeviceGetAttribute(&G.sm_count, cudaDevAttrMultiProcessorCount, dev));
    for (int w = 1; w <= 4; w++)
        for (int lw = 0; lw <= 5; lw++) {
            int nb = 0;
            CK(cuo::decode_kernel_occupancy(32 * w, 1 << lw, &nb));
            G.occ[w][lw] = nb < 1 ? 1 : nb;
        }
    G.occ_blocks = G.occ[BLOCK / 32][5];
    G.occ_dev = dev;
    return RC_OK;
}

int block_threads(const cuopus_batch *b)
{
    int t = b->block > 0 ? b->block : BLOCK;
    return t;
}

// Decoder groups resident on the whole GPU for a block size and width.
long long resident_groups(int block, int width)
{
    int lw = 0;
    while ((1 << lw) < width) lw++;
    return (long long)G.sm_count * G.occ[block / 32][lw] * (block / width);
}

int ensure_events(Err &err)
{
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (G.ev_dev == dev && G.ev0) return RC_OK;
    cudaEvent_t *evs[] = {&G.ev0, &G.ev1, &G.evh0, &G.evh1, &G.evr0, &G.evr1};
    for (cudaEvent_t *e : evs) CK(cudaEventCreate(e));
    G.ev_dev = dev;
    return RC_OK;
}

double now_ms()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

// ------------------------------------------------------------------ engine

void drop_graph()
{
    if (G.gexec) cudaGraphExecDestroy(G.gexec);
    G.gexec = nullptr;
    G.g_dev = -1;
}

// The decode launch as a CUDA graph: the work-queue reset and the kernel,
// captured once on a library-private stream and replayed on the caller's
// stream.  The key is the full argument block and grid, so a launch with
// other tables, sizes or workspaces captures again (the previous executable
// graph is released first).
int launch_graph(const cuo::DecodeArgs &a, int blocks, int block, cudaStream_t st, Err &err)
{
    int dev = 0;
    CK(cudaGetDevice(&dev));
    bool hit = G.gexec && G.g_dev == dev && G.g_blocks == blocks && G.g_block == block &&
               memcmp(&G.g_args, &a, sizeof a) == 0;
    if (!hit) {
        drop_graph();
        if (!G.cap_stream || G.cap_dev != dev) {
            CK(cudaStreamCreateWithFlags(&G.cap_stream, cudaStreamNonBlocking));
            G.cap_dev = dev;
        }
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(G.cap_stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e1 = a.use_queue ? cudaMemsetAsync(G.queue.p, 0, QUEUE_BYTES, G.cap_stream) : cudaSuccess;
        cudaError_t e2 = cuo::decode_kernel_launch(a, blocks, block, G.cap_stream);
        cudaError_t e3 = cudaStreamEndCapture(G.cap_stream, &g);
        if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaError_t e = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3);
            return err.set(RC_CUDA, "graph capture of the decode launch: %s", cudaGetErrorString(e));
        }
        cudaError_t e = cudaGraphInstantiate(&G.gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            G.gexec = nullptr;
            return err.set(RC_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        }
        G.g_dev = dev;
        G.g_blocks = blocks;
        G.g_block = block;
        G.g_args = a;
    }
    CK(cudaGraphLaunch(G.gexec, st));
    return RC_OK;
}

int decode_batch(const cuopus_batch *b, cudaStream_t st, float *kernel_ms, Err &err)
{
    if (!b) return err.set(RC_ARG, "batch is NULL");
    if (b->nchains <= 0) return RC_OK;
    int width = b->width > 0 ? b->width : default_width();
    if (width != 1 && width != 2 && width != 4 && width != 8 && width != 16 && width != 32)
        return err.set(RC_ARG, "width %d is not a power of two <= 32", width);
    if (!b->data || !b->off || !b->len || !b->first || !b->npkts || !b->channels || !b->trim || !b->keep ||
        !b->res)
        return err.set(RC_ARG, "batch has a NULL table");
    if (b->out && !b->out_off) return err.set(RC_ARG, "out without out_off");
    if ((b->pkt_nsamp || b->pkt_rng) && !b->rec_off) return err.set(RC_ARG, "per-packet records without rec_off");
    if (b->schedule < 0 || b->schedule > 2) return err.set(RC_ARG, "schedule %d is not 0, 1 or 2", b->schedule);
    int block = block_threads(b);
    if (block != 32 && block != 64 && block != 96 && block != 128)
        return err.set(RC_ARG, "block %d is not 32, 64, 96 or 128 threads", block);
    if (block % width) return err.set(RC_ARG, "width %d does not divide block %d", width, block);
    const bool tail = b->light_sms > 0;
    if (tail && (b->schedule != 1 || b->scalar))
        return err.set(RC_ARG, "tail scheduling (light_sms) needs the queue schedule and every lane");
    if (b->light_sms < 0 || b->long_chains < 0) return err.set(RC_ARG, "light_sms / long_chains < 0");
    int rc = ensure_occupancy(err);
    if (rc) return rc;
    if ((rc = ensure_events(err))) return rc;
    // plain: one group per chain, the hardware block scheduler assigns them;
    // static / queue: a persistent grid of the resident groups (under tail
    // scheduling all of them: the warps themselves decide which stay)
    long long groups = b->schedule == 2 ? (long long)b->nchains
                                        : std::min<long long>(b->nchains, resident_groups(block, width));
    if (tail) groups = resident_groups(block, width);
    else if (b->max_groups > 0) groups = std::min<long long>(groups, b->max_groups);
    int gpb = block / width;
    long long blocks_ll = (groups + gpb - 1) / gpb;
    if (blocks_ll > 0x7fffffffLL) return err.set(RC_ARG, "too many chains for one launch");
    int blocks = (int)blocks_ll;
    long long nslots = blocks_ll * gpb;
    if ((rc = gpu_grow(G.slots, (size_t)nslots * sizeof(cuo::ChainSlot), err))) return rc;
    if ((rc = gpu_grow(G.queue, QUEUE_BYTES, err))) return rc;
    const uint32_t *order_dev = nullptr;
    if (b->schedule == 1 && b->order) {
        if ((rc = gpu_grow(G.order, 4ull * b->nchains, err))) return rc;
        CK(cudaMemcpyAsync(G.order.p, b->order, 4ull * b->nchains, cudaMemcpyHostToDevice, st));
        order_dev = (const uint32_t *)G.order.p;
    }
    cuo::DecodeArgs a;
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
    a.order = order_dev;
    a.rec_off = b->rec_off;
    a.pkt_nsamp = b->pkt_nsamp;
    a.pkt_rng = b->pkt_rng;
    a.res = (cuo::ChainResult *)b->res;
    a.slots = (cuo::ChainSlot *)G.slots.p;
    a.queue_head = (unsigned *)G.queue.p;
    a.nchains = b->nchains;
    a.width = width;
    a.use_queue = b->schedule == 1;
    a.scalar = b->scalar != 0;
    a.fec = b->fec != 0;
    if (tail) {
        int gpw = 32 / width;
        a.sm_rank = (unsigned *)G.queue.p + 2;
        a.light_sms = b->light_sms;
        a.light_warps = 1;
        a.heavy_warps = b->max_groups > 0 ? std::max(1, (int)(b->max_groups / ((long long)G.sm_count * gpw))) : 64;
        a.long_chains = std::min(b->long_chains, b->nchains);
    }
    CK(cudaEventRecord(G.ev0, st));
    if (b->graph) {
        if ((rc = launch_graph(a, blocks, block, st, err))) return rc;
    } else {
        if (a.use_queue) CK(cudaMemsetAsync(G.queue.p, 0, QUEUE_BYTES, st));
        CK(cuo::decode_kernel_launch(a, blocks, block, st));
    }
    CK(cudaEventRecord(G.ev1, st));
    if (kernel_ms) {
        CK(cudaEventSynchronize(G.ev1));
        CK(cudaEventElapsedTime(kernel_ms, G.ev0, G.ev1));
        G.last_kernel_ms = *kernel_ms;
    }
    return RC_OK;
}

// One call's worth of files merged into a single chain table (the packet
// tables uninitialised when sized: they are written in full right after).
struct Plan {
    cuo_host::Table<uint8_t> blob;
    cuo_host::Table<uint64_t> off;
    cuo_host::Table<uint32_t> len;
    std::vector<uint32_t> first, npkts;
    std::vector<uint8_t> chans;
    std::vector<uint64_t> trim, keep, out_off, cap;
    std::vector<uint64_t> file_out0, file_keep;   // per file: element offset / kept samples per channel
    std::vector<int> file_chans;
    std::vector<int64_t> file_play48;
    uint64_t out_elems = 0;
};

// One file's demux and chain table (with each chain's decode capacity).
struct FilePlan {
    cuo_host::Demux d;
    cuo_host::Chains c;
    std::string e;
    bool ok = false;
};

void plan_one(const uint8_t *ogg, size_t n, double seg_s, double preroll_ms, bool require_mono, FilePlan &F,
              int threads)
{
    F.ok = cuo_host::demux_and_chain(ogg, n, seg_s, preroll_ms, require_mono, F.d, &F.c, F.e, threads);
}

// Demux every file and merge the tables.  The files are demuxed and merged on
// CUOPUS_DEMUX_THREADS host threads (default 1: the calling thread only, as
// the reference's library, which starts no threads); with fewer files than
// threads, each file's demux splits its pages over the threads left.  Errors
// are reported for the lowest-numbered failing file, whatever the thread count.
int plan_files(const uint8_t *const *oggs, const size_t *ns, int nfiles, bool require_mono, Plan &P, Err &err)
{
    double seg_s = env_f("CUOPUS_SEG_S", 1.0);
    double preroll_ms = env_f("CUOPUS_PREROLL_MS", 250.0);
    for (int f = 0; f < nfiles; f++)
        if (!oggs || !ns || !oggs[f] || !ns[f]) return err.set(RC_ARG, "file %d: empty input", f);
    std::vector<FilePlan> F((size_t)std::max(nfiles, 0));
    const int all_threads = std::min(env_i("CUOPUS_DEMUX_THREADS", 1), 64);
    int nthreads = std::min(all_threads, std::max(nfiles, 1));
    const int per_file = std::max(1, all_threads / std::max(nfiles, 1));
    std::atomic<int> next(0);
    auto work = [&]() {
        for (int f; (f = next.fetch_add(1)) < nfiles;)
            plan_one(oggs[f], ns[f], seg_s, preroll_ms, require_mono, F[f], per_file);
    };
    auto run = [&](const std::function<void()> &fn) {
        next = 0;
        std::vector<std::thread> pool;
        for (int t = 1; t < nthreads; t++) {
            try {
                pool.emplace_back(fn);
            } catch (...) {
                break;   // fewer threads; the calling thread does the rest
            }
        }
        fn();
        for (auto &t : pool) t.join();
    };
    run(work);
    // sizes and errors, file by file (the first failing file is reported)
    std::vector<uint64_t> pkt0(nfiles + 1, 0), byte0(nfiles + 1, 0), ch0(nfiles + 1, 0);
    P.file_out0.resize(nfiles);
    P.file_keep.resize(nfiles);
    P.file_chans.resize(nfiles);
    P.file_play48.resize(nfiles);
    for (int f = 0; f < nfiles; f++) {
        FilePlan &Fp = F[f];
        if (!Fp.ok) {
            if (nfiles > 1) return err.set(RC_SOFT, "file %d: %s", f, Fp.e.c_str());
            return err.set(RC_SOFT, "%s", Fp.e.c_str());
        }
        const cuo_host::Chains &c = Fp.c;
        uint64_t fkeep = 0;
        for (uint32_t i = 0; i < c.size(); i++) {
            if (c.cap[i] < (uint64_t)c.trim[i] + c.keep[i])
                return err.set(RC_SOFT, "chain %u capacity %llu < trim %u + keep %u", i,
                               (unsigned long long)c.cap[i], c.trim[i], c.keep[i]);
            fkeep += c.keep[i];
        }
        pkt0[f + 1] = pkt0[f] + Fp.d.n_packets();
        byte0[f + 1] = byte0[f] + Fp.d.blob.size();
        ch0[f + 1] = ch0[f] + c.size();
        P.file_out0[f] = P.out_elems;
        P.file_keep[f] = fkeep;
        P.file_chans[f] = Fp.d.channels;
        P.file_play48[f] = Fp.d.play48;
        P.out_elems += fkeep * (uint64_t)Fp.d.channels;
    }
    // merged tables: every file fills its own ranges (on the same threads); a
    // single file's packet tables are taken over as they are
    const bool take = nfiles == 1;
    if (take) {
        P.blob.swap(F[0].d.blob);
        P.off.swap(F[0].d.off);
        P.len.swap(F[0].d.len);
    } else {
        P.blob.resize(byte0[nfiles]);
        P.off.resize(pkt0[nfiles]);
        P.len.resize(pkt0[nfiles]);
    }
    size_t nch = ch0[nfiles];
    P.first.resize(nch);
    P.npkts.resize(nch);
    P.chans.resize(nch);
    P.trim.resize(nch);
    P.keep.resize(nch);
    P.out_off.resize(nch);
    P.cap.resize(nch);
    run([&]() {
        for (int f; (f = next.fetch_add(1)) < nfiles;) {
            FilePlan &Fp = F[f];
            const cuo_host::Demux &d = Fp.d;
            const cuo_host::Chains &c = Fp.c;
            if (!take) {
                if (!d.blob.empty()) memcpy(P.blob.data() + byte0[f], d.blob.data(), d.blob.size());
                for (uint32_t k = 0; k < d.n_packets(); k++) {
                    P.off[pkt0[f] + k] = d.off[k] + byte0[f];
                    P.len[pkt0[f] + k] = d.len[k];
                }
            }
            uint64_t fkeep = 0;
            for (uint32_t i = 0; i < c.size(); i++) {
                size_t j = ch0[f] + i;
                P.first[j] = c.first[i] + (uint32_t)pkt0[f];
                P.npkts[j] = c.npkts[i];
                P.chans[j] = (uint8_t)d.channels;
                P.trim[j] = c.trim[i];
                P.keep[j] = c.keep[i];
                P.out_off[j] = P.file_out0[f] + fkeep * d.channels;
                P.cap[j] = c.cap[i];
                fkeep += c.keep[i];
            }
            Fp = FilePlan();   // release this file's tables on this thread
        }
    });
    return RC_OK;
}

// Threads per block of the file entry points' launch: the autotuner's choice at
// both widths they use (the 2 h file in 1 s chains at 8 lanes: 164 ms at 64
// threads against 200 ms at 128; whole streams at 32 lanes: equal).
const int FILE_BLOCK = 64;

// Lanes per chain of a file batch (CUOPUS_STRIDE, when set, decides).  A
// batch's decode time is about max(longest chain, total work / decoder
// groups) / per-group speed.  At 32 lanes a group decodes about 3x faster
// than at 8 (lane-split loops), but 8 lanes give 6.4x the groups (every
// resident group at 8 against 5 warps per SM at 32): long or uneven chains
// (whole streams) decode faster at 32, many short chains (a long file cut in
// 1 s chains) at 8.  Chain cost: its TOC samples x channels.
int choose_width(const Plan &P)
{
    const char *e = getenv("CUOPUS_STRIDE");
    if (e && atoi(e) > 0) return default_width();
    double sum = 0.0, mx = 0.0;
    for (size_t c = 0; c < P.first.size(); c++) {
        double w = (double)P.cap[c] * (double)P.chans[c];
        sum += w;
        mx = std::max(mx, w);
    }
    long long g32 = default_max_groups(32);
    if (g32 <= 0) g32 = resident_groups(FILE_BLOCK, 32);
    long long g8 = resident_groups(FILE_BLOCK, 8);
    const double speed32 = 3.0;   // per-group speed at 32 lanes relative to 8
    double t32 = std::max(mx, sum / (double)std::max(g32, 1LL)) / speed32;
    double t8 = std::max(mx, sum / (double)std::max(g8, 1LL));
    return t8 < t32 ? 8 : 32;
}

// fn(begin, end) over [0, n) in up to `threads` contiguous ranges, the first
// on the calling thread.
template <class F> void run_chunks(int threads, size_t n, F &&fn)
{
    size_t t = (size_t)std::max(1, std::min(threads, 64));
    t = std::min(t, std::max<size_t>(1, n / 256));
    std::vector<std::thread> pool;
    for (size_t r = 1; r < t; r++) {
        size_t a = n * r / t, b = n * (r + 1) / t;
        try {
            pool.emplace_back([&fn, a, b] { fn(a, b); });
        } catch (...) {
            fn(a, b);   // no thread: run it here
        }
    }
    fn(0, n / t);
    for (auto &th : pool) th.join();
}

// H2D of a plan and one decode launch into G.pcm, or into `direct_out` when
// the caller's outputs are one buffer laid out as the plan's (the decoder
// writes exactly each chain's kept samples at its offset, nothing else).
int run_plan(const Plan &P, cudaStream_t st, Err &err, int16_t *direct_out = nullptr)
{
    int rc;
    uint32_t nch = (uint32_t)P.first.size();
    auto r16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    size_t tbl = r16(P.blob.size()) + r16(8ull * P.off.size()) + r16(4ull * P.len.size()) + 2 * r16(4ull * nch) +
                 r16(nch) + 3 * r16(8ull * nch);
    if ((rc = pin_grow(G.hpin, tbl, err))) return rc;
    if ((rc = gpu_grow(G.data, P.blob.size() + 16, err))) return rc;
    if ((rc = gpu_grow(G.off, 8ull * P.off.size(), err))) return rc;
    if ((rc = gpu_grow(G.len, 4ull * P.len.size(), err))) return rc;
    if ((rc = gpu_grow(G.first, 4ull * nch, err))) return rc;
    if ((rc = gpu_grow(G.npkts, 4ull * nch, err))) return rc;
    if ((rc = gpu_grow(G.chans, nch, err))) return rc;
    if ((rc = gpu_grow(G.trim, 8ull * nch, err))) return rc;
    if ((rc = gpu_grow(G.keep, 8ull * nch, err))) return rc;
    if ((rc = gpu_grow(G.out_off, 8ull * nch, err))) return rc;
    if ((rc = gpu_grow(G.res, 16ull * nch, err))) return rc;
    if (!direct_out && (rc = gpu_grow(G.pcm, 2ull * P.out_elems + 16, err))) return rc;
    // stage everything through one pinned buffer, then one async copy per table
    if ((rc = ensure_events(err))) return rc;
    CK(cudaEventRecord(G.evh0, st));
    uint8_t *h = (uint8_t *)G.hpin.p;
    size_t o = 0;
    auto stage = [&](Grow &dst, const void *src, size_t bytes) -> int {
        if (!bytes) return RC_OK;
        memcpy(h + o, src, bytes);
        cudaError_t e = cudaMemcpyAsync(dst.p, h + o, bytes, cudaMemcpyHostToDevice, st);
        o += (bytes + 15) & ~(size_t)15;
        if (e != cudaSuccess) return err.set(RC_CUDA, "cudaMemcpyAsync: %s", cudaGetErrorString(e));
        return RC_OK;
    };
    if ((rc = stage(G.data, P.blob.data(), P.blob.size()))) return rc;
    if ((rc = stage(G.off, P.off.data(), 8ull * P.off.size()))) return rc;
    if ((rc = stage(G.len, P.len.data(), 4ull * P.len.size()))) return rc;
    if ((rc = stage(G.first, P.first.data(), 4ull * nch))) return rc;
    if ((rc = stage(G.npkts, P.npkts.data(), 4ull * nch))) return rc;
    if ((rc = stage(G.chans, P.chans.data(), nch))) return rc;
    if ((rc = stage(G.trim, P.trim.data(), 8ull * nch))) return rc;
    if ((rc = stage(G.keep, P.keep.data(), 8ull * nch))) return rc;
    if ((rc = stage(G.out_off, P.out_off.data(), 8ull * nch))) return rc;
    CK(cudaEventRecord(G.evh1, st));
    cuopus_batch b;
    memset(&b, 0, sizeof b);
    b.data = (const uint8_t *)G.data.p;
    b.off = (const uint64_t *)G.off.p;
    b.len = (const uint32_t *)G.len.p;
    b.first = (const uint32_t *)G.first.p;
    b.npkts = (const uint32_t *)G.npkts.p;
    b.channels = (const uint8_t *)G.chans.p;
    b.trim = (const uint64_t *)G.trim.p;
    b.keep = (const uint64_t *)G.keep.p;
    b.out_off = (const uint64_t *)G.out_off.p;
    b.out = direct_out ? direct_out : (int16_t *)G.pcm.p;
    b.res = (uint32_t *)G.res.p;
    b.nchains = (int32_t)nch;
    if ((rc = ensure_occupancy(err))) return rc;
    b.width = choose_width(P);
    b.block = FILE_BLOCK;
    b.max_groups = default_max_groups(b.width);
    G.last_width = b.width;
    // longest chains first through the device queue, by the fitted additive
    // cost of their packets (CUOPUS_ORDER=samples: by decoded samples x channels)
    std::vector<uint32_t> order(nch);
    std::iota(order.begin(), order.end(), 0u);
    const char *oenv = getenv("CUOPUS_ORDER");
    if (oenv && strcmp(oenv, "samples") == 0) {
        std::stable_sort(order.begin(), order.end(),
                         [&](uint32_t x, uint32_t y) { return P.cap[x] * P.chans[x] > P.cap[y] * P.chans[y]; });
    } else {
        const cuo_host::OrderCost oc(cuo_host::order_coefficients(b.width));
        std::vector<double> cost(nch);
        run_chunks(env_i("CUOPUS_DEMUX_THREADS", 1), nch, [&](size_t c0, size_t c1) {
            for (size_t c = c0; c < c1; c++) {
                double s = oc.chain;
                for (uint32_t k = 0; k < P.npkts[c]; k++) {
                    uint64_t q = (uint64_t)P.first[c] + k;
                    s += oc.of(P.blob.data() + P.off[q], P.len[q], P.chans[c]);
                }
                cost[c] = s;
            }
        });
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return cost[x] > cost[y]; });
    }
    b.schedule = 1;
    b.order = order.data();
    float kms = 0.f;
    if ((rc = decode_batch(&b, st, &kms, err))) return rc;
    return RC_OK;
}

int validate(const Plan &P, cudaStream_t st, Err &err)
{
    uint32_t nch = (uint32_t)P.first.size();
    std::vector<uint32_t> res(4ull * nch);
    CK(cudaMemcpyAsync(res.data(), G.res.p, 16ull * nch, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (uint32_t c = 0; c < nch; c++) {
        int32_t stop = (int32_t)res[4 * c];
        uint32_t samples = res[4 * c + 1];
        if (stop != 0) return err.set(RC_SOFT, "chain %u: device decode error %d", c, stop);
        if (samples != P.cap[c])
            return err.set(RC_SOFT, "chain %u: decoded %u samples, expected %llu", c, samples,
                           (unsigned long long)P.cap[c]);
    }
    return RC_OK;
}

// Timings of the call that just completed (its stream is synchronised).
struct Plan;
void record_stats(const Plan &P, bool resampled);

int64_t out16_of(int64_t play48)
{
    int64_t v = (int64_t)((play48 - (int64_t)SWR_TAIL_48K) / 3);
    return v < 0 ? 0 : v;
}

int resample(const int16_t *in, int64_t avail, int64_t n_out, float *out, cudaStream_t st, Err &err, int chans = 1)
{
    if (n_out <= 0) return RC_OK;
    int rc = ensure_taps(st, err);
    if (rc) return rc;
    long long blocks = (n_out + cuo::RS_TILE_OUT - 1) / cuo::RS_TILE_OUT;
    if (blocks > 0x7fffffffLL) return err.set(RC_ARG, "resample length too large");
    cuo::k_resample48to16<<<(unsigned)blocks, cuo::RS_THREADS, 0, st>>>(in, avail, n_out, out, chans);
    CK(cudaGetLastError());
    return RC_OK;
}

// f16k decode of N files.  The reference entry points are mono only
// (allow_stereo false); with allow_stereo each channel of a stereo file is
// resampled on its own and the output interleaves them (out_caps then count
// floats over all channels).
int f16k_impl(const uint8_t *const *oggs, const size_t *ns, int nfiles, float *const *out_devs,
              const size_t *out_caps, int64_t *out_lens, cudaStream_t st, bool enforce_max_batch, Err &err,
              bool allow_stereo = false, int32_t *out_channels = nullptr)
{
    G.last_ovf = 0;
    if (out_lens) for (int f = 0; f < nfiles; f++) out_lens[f] = 0;
    if (nfiles <= 0) return RC_OK;
    int rc = refuse_capture(st, err);
    if (rc) return rc;
    Plan P;
    G.last = cuopus_stats{};
    double t0 = now_ms();
    if ((rc = plan_files(oggs, ns, nfiles, !allow_stereo, P, err))) return rc;
    G.last.demux_ms = now_ms() - t0;
    if (P.first.empty()) return err.set(RC_SOFT, "no chains");
    if (enforce_max_batch) {
        int max_batch = env_i("CUOPUS_MAX_BATCH", 2048);
        if ((int)P.first.size() > max_batch)
            return err.set(RC_ARG, "merged chains %zu > max_batch %d (decode files individually)", P.first.size(),
                           max_batch);
    }
    std::vector<int64_t> n16(nfiles);
    for (int f = 0; f < nfiles; f++) {
        n16[f] = out16_of((int64_t)P.file_keep[f]);   // sum(keep) == playable samples
        uint64_t need = (uint64_t)n16[f] * (uint64_t)P.file_chans[f];
        if (!out_caps || need > out_caps[f])
            return err.set(RC_ARG, "file %d: output capacity %zu < required %llu", f, out_caps ? out_caps[f] : 0,
                           (unsigned long long)need);
        if (n16[f] > 0 && (!out_devs || !out_devs[f])) return err.set(RC_ARG, "file %d: out_dev is NULL", f);
    }
    int64_t total16 = 0;
    for (int f = 0; f < nfiles; f++) total16 += n16[f];
    if (total16 == 0) return RC_OK;
    if ((rc = run_plan(P, st, err))) return rc;
    CK(cudaEventRecord(G.evr0, st));
    for (int f = 0; f < nfiles; f++) {
        int ch = P.file_chans[f];
        for (int c = 0; c < ch; c++) {
            const int16_t *in = (const int16_t *)G.pcm.p + P.file_out0[f] + c;
            if ((rc = resample(in, (int64_t)P.file_keep[f], n16[f], out_devs[f] + c, st, err, ch))) return rc;
        }
    }
    CK(cudaEventRecord(G.evr1, st));
    if ((rc = validate(P, st, err))) return rc;
    record_stats(P, true);
    if (out_lens) for (int f = 0; f < nfiles; f++) out_lens[f] = n16[f];
    if (out_channels) for (int f = 0; f < nfiles; f++) out_channels[f] = P.file_chans[f];
    return RC_OK;
}

void record_stats(const Plan &P, bool resampled)
{
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, G.evh0, G.evh1) == cudaSuccess) G.last.h2d_ms = ms;
    if (cudaEventElapsedTime(&ms, G.ev0, G.ev1) == cudaSuccess) G.last.kernel_ms = ms;
    if (resampled && cudaEventElapsedTime(&ms, G.evr0, G.evr1) == cudaSuccess) G.last.resample_ms = ms;
    G.last.chains = (int64_t)P.first.size();
    G.last.width = G.last_width;
    G.last.packets = (int64_t)P.len.size();
    int64_t play = 0;
    for (int64_t v : P.file_play48) play += v;
    G.last.play48 = play;
    cudaGetLastError();
}

} // namespace

cudaError_t cuo::resample_into(const int16_t *in, long long avail, long long n_out, float *out, cudaStream_t st)
{
    Err err(nullptr, 0);
    int rc = resample(in, avail, n_out, out, st, err);
    if (rc == RC_OK) return cudaSuccess;
    cudaError_t e = cudaGetLastError();
    return e != cudaSuccess ? e : cudaErrorInvalidValue;
}

// ====================================================================== C ABI

extern "C" int cuopus_last_stats(cuopus_stats *s)
{
    if (!s) return RC_ARG;
    *s = G.last;
    return RC_OK;
}

extern "C" int cuopus_last_arena_overflow(void) { return G.last_ovf; }

extern "C" long long cuopus_workspace_bytes(void) { return G.dev_bytes; }

extern "C" void cuopus_release_workspaces(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    drop_graph();
    Grow *all[] = {&G.data, &G.off, &G.len, &G.first, &G.npkts, &G.chans, &G.trim, &G.keep,
                   &G.out_off, &G.order, &G.res, &G.slots, &G.queue, &G.pcm};
    for (Grow *g : all) {
        if (g->p) cudaFree(g->p);
        g->p = nullptr;
        g->cap = 0;
    }
    if (G.hpin.p) cudaFreeHost(G.hpin.p);
    G.hpin.p = nullptr;
    G.hpin.cap = 0;
    G.dev_bytes = 0;
    G.taps_dev = -1;
}

extern "C" int cuopus_probe(const uint8_t *ogg, size_t n, int64_t *samples16k, char *errbuf, size_t errcap)
{
    Err err(errbuf, errcap);
    if (!samples16k) return err.set(RC_ARG, "samples16k is NULL");
    if (!ogg || !n) return err.set(RC_ARG, "empty input");
    cuo_host::Demux d;
    std::string e;
    if (!cuo_host::demux_and_chain(ogg, n, 1.0, 250.0, true, d, nullptr, e)) return err.set(RC_SOFT, "%s", e.c_str());
    *samples16k = out16_of(d.play48);
    return RC_OK;
}

extern "C" int cuopus_probe_pcm(const uint8_t *ogg, size_t n, int64_t *play48, int32_t *channels, char *errbuf,
                                size_t errcap)
{
    Err err(errbuf, errcap);
    if (!play48) return err.set(RC_ARG, "play48 is NULL");
    if (!ogg || !n) return err.set(RC_ARG, "empty input");
    cuo_host::Demux d;
    std::string e;
    if (!cuo_host::demux_and_chain(ogg, n, 1.0, 250.0, false, d, nullptr, e)) return err.set(RC_SOFT, "%s", e.c_str());
    *play48 = d.play48 > 0 ? d.play48 : 0;
    if (channels) *channels = d.channels;
    return RC_OK;
}

extern "C" int cuopus_index(const uint8_t *ogg, size_t n, double seg_s, double preroll_ms, int require_mono,
                            int64_t *n_packets, int64_t *n_chains, int64_t *blob_bytes, int32_t *channels,
                            int64_t *play48, uint8_t *blob, uint64_t *pkt_off, uint32_t *pkt_len, uint32_t *first,
                            uint32_t *npkts, uint32_t *trim, uint32_t *keep, char *errbuf, size_t errcap)
{
    Err err(errbuf, errcap);
    if (!ogg || !n) return err.set(RC_ARG, "empty input");
    cuo_host::Demux d;
    cuo_host::Chains c;
    std::string e;
    if (!cuo_host::demux_and_chain(ogg, n, seg_s, preroll_ms, require_mono != 0, d, &c, e))
        return err.set(RC_SOFT, "%s", e.c_str());
    if (n_packets) *n_packets = d.n_packets();
    if (n_chains) *n_chains = c.size();
    if (blob_bytes) *blob_bytes = (int64_t)d.blob.size();
    if (channels) *channels = d.channels;
    if (play48) *play48 = d.play48;
    if (!blob) return RC_OK;
    if (!pkt_off || !pkt_len || !first || !npkts || !trim || !keep) return err.set(RC_ARG, "NULL output array");
    memcpy(blob, d.blob.data(), d.blob.size());
    memcpy(pkt_off, d.off.data(), 8 * d.off.size());
    memcpy(pkt_len, d.len.data(), 4 * d.len.size());
    memcpy(first, c.first.data(), 4 * c.size());
    memcpy(npkts, c.npkts.data(), 4 * c.size());
    memcpy(trim, c.trim.data(), 4 * c.size());
    memcpy(keep, c.keep.data(), 4 * c.size());
    return RC_OK;
}

extern "C" int cuopus_decode_f16k_on(const uint8_t *ogg, size_t n, float *out_dev, size_t out_cap, int64_t *out_len,
                                     void *cuda_stream, char *errbuf, size_t errcap)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Err err(errbuf, errcap);
    const uint8_t *oggs[1] = {ogg};
    size_t ns[1] = {n};
    float *outs[1] = {out_dev};
    size_t caps[1] = {out_cap};
    if (!ogg || !n) return err.set(RC_ARG, "empty input");
    return f16k_impl(oggs, ns, 1, outs, caps, out_len, (cudaStream_t)cuda_stream, false, err);
}

extern "C" int cuopus_decode_f16k(const uint8_t *ogg, size_t n, float *out_dev, size_t out_cap, int64_t *out_len,
                                  char *errbuf, size_t errcap)
{
    return cuopus_decode_f16k_on(ogg, n, out_dev, out_cap, out_len, nullptr, errbuf, errcap);
}

extern "C" int cuopus_decode_f16k_multi(const uint8_t *const *oggs, const size_t *ns, int nfiles,
                                        float *const *out_devs, const size_t *out_caps, int64_t *out_lens,
                                        void *cuda_stream, char *errbuf, size_t errcap)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Err err(errbuf, errcap);
    return f16k_impl(oggs, ns, nfiles, out_devs, out_caps, out_lens, (cudaStream_t)cuda_stream, nfiles > 1, err);
}

extern "C" int cuopus_decode_f16k_channels(const uint8_t *const *oggs, const size_t *ns, int nfiles,
                                           float *const *out_devs, const size_t *out_caps, int64_t *out_lens,
                                           int32_t *out_channels, void *cuda_stream, char *errbuf, size_t errcap)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Err err(errbuf, errcap);
    return f16k_impl(oggs, ns, nfiles, out_devs, out_caps, out_lens, (cudaStream_t)cuda_stream, false, err, true,
                     out_channels);
}

extern "C" int cuopus_decode_i16_multi(const uint8_t *const *oggs, const size_t *ns, int nfiles,
                                       int16_t *const *out_devs, const size_t *out_caps, int64_t *out_lens,
                                       int32_t *out_channels, void *cuda_stream, char *errbuf, size_t errcap)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Err err(errbuf, errcap);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    if (out_lens) for (int f = 0; f < nfiles; f++) out_lens[f] = 0;
    if (nfiles <= 0) return RC_OK;
    int rc = refuse_capture(st, err);
    if (rc) return rc;
    Plan P;
    G.last = cuopus_stats{};
    double t0 = now_ms();
    if ((rc = plan_files(oggs, ns, nfiles, false, P, err))) return rc;
    G.last.demux_ms = now_ms() - t0;
    if (P.first.empty()) return err.set(RC_SOFT, "no chains");
    for (int f = 0; f < nfiles; f++) {
        uint64_t need = P.file_keep[f] * (uint64_t)P.file_chans[f];
        if (!out_caps || need > out_caps[f])
            return err.set(RC_ARG, "file %d: output capacity %zu < required %llu", f, out_caps ? out_caps[f] : 0,
                           (unsigned long long)need);
        if (need && (!out_devs || !out_devs[f])) return err.set(RC_ARG, "file %d: out_dev is NULL", f);
    }
    // outputs back to back in file order, as the plan lays them out: decode
    // straight into them; otherwise into the workspace, then one copy per file
    bool direct = out_devs && out_devs[0] != nullptr;
    for (int f = 0; f < nfiles && direct; f++) {
        uint64_t need = P.file_keep[f] * (uint64_t)P.file_chans[f];
        if (need && out_devs[f] != out_devs[0] + P.file_out0[f]) direct = false;
    }
    if ((rc = run_plan(P, st, err, direct ? out_devs[0] : nullptr))) return rc;
    for (int f = 0; f < nfiles && !direct; f++) {
        uint64_t need = P.file_keep[f] * (uint64_t)P.file_chans[f];
        if (need)
            CK(cudaMemcpyAsync(out_devs[f], (const int16_t *)G.pcm.p + P.file_out0[f], 2 * need,
                               cudaMemcpyDeviceToDevice, st));
    }
    if ((rc = validate(P, st, err))) return rc;
    record_stats(P, false);
    for (int f = 0; f < nfiles; f++) {
        if (out_lens) out_lens[f] = (int64_t)P.file_keep[f];
        if (out_channels) out_channels[f] = P.file_chans[f];
    }
    return RC_OK;
}

extern "C" int cuopus_decode_batch(const cuopus_batch *b, void *cuda_stream, float *kernel_ms, char *errbuf,
                                   size_t errcap)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Err err(errbuf, errcap);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    int rc = refuse_capture(st, err);
    if (rc) return rc;
    if ((rc = decode_batch(b, st, kernel_ms, err))) return rc;
    CK(cudaStreamSynchronize(st));
    return RC_OK;
}

// Autotuner: every (width, block) candidate decodes the batch as given
// (schedule, order, graph) `reps` times; the candidate with the lowest
// median kernel time wins.  Candidates whose launch is rejected are skipped.
extern "C" int cuopus_autotune(const cuopus_batch *b, const int32_t *widths, int nwidths, const int32_t *blocks,
                               int nblocks, int reps, void *cuda_stream, int32_t *best_width, int32_t *best_block,
                               float *times_ms, char *errbuf, size_t errcap)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Err err(errbuf, errcap);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    if (!b || !widths || !blocks || nwidths <= 0 || nblocks <= 0 || !best_width || !best_block)
        return err.set(RC_ARG, "autotune: bad arguments");
    int rc = refuse_capture(st, err);
    if (rc) return rc;
    if (reps < 1) reps = 1;
    float best = -1.f;
    for (int i = 0; i < nwidths; i++)
        for (int j = 0; j < nblocks; j++) {
            cuopus_batch c = *b;
            c.width = widths[i];
            c.block = blocks[j];
            std::vector<float> t;
            bool ok = true;
            for (int r = 0; r < reps && ok; r++) {
                float ms = 0.f;
                Err e2(nullptr, 0);
                int rc2 = decode_batch(&c, st, &ms, e2);
                if (rc2 == RC_CUDA) return err.set(rc2, "autotune: %s", e2.buf);
                ok = rc2 == RC_OK;
                t.push_back(ms);
            }
            float med = -1.f;
            if (ok) {
                std::sort(t.begin(), t.end());
                med = t[t.size() / 2];
                if (best < 0.f || med < best) {
                    best = med;
                    *best_width = c.width;
                    *best_block = c.block;
                }
            }
            if (times_ms) times_ms[i * nblocks + j] = med;
        }
    CK(cudaStreamSynchronize(st));
    if (best < 0.f) return err.set(RC_ARG, "autotune: no candidate could be launched");
    return RC_OK;
}

extern "C" int cuopus_autotune_occupancy(const cuopus_batch *b, const int32_t *warps_per_sm, int n, int reps,
                                         void *cuda_stream, int32_t *best_max_groups, float *times_ms,
                                         char *errbuf, size_t errcap)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Err err(errbuf, errcap);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    if (!b || !warps_per_sm || n <= 0 || !best_max_groups) return err.set(RC_ARG, "autotune: bad arguments");
    int rc = refuse_capture(st, err);
    if (rc) return rc;
    if ((rc = ensure_occupancy(err))) return rc;
    if (reps < 1) reps = 1;
    float best = -1.f;
    for (int i = 0; i < n; i++) {
        cuopus_batch c = *b;
        int width = c.width > 0 ? c.width : 32;
        c.max_groups = warps_per_sm[i] > 0 ? warps_per_sm[i] * G.sm_count * (32 / width) : 0;
        std::vector<float> t;
        bool ok = warps_per_sm[i] >= 0 && width >= 1 && width <= 32;
        for (int r = 0; r < reps && ok; r++) {
            float ms = 0.f;
            Err e2(nullptr, 0);
            int rc2 = decode_batch(&c, st, &ms, e2);
            if (rc2 == RC_CUDA) return err.set(rc2, "autotune: %s", e2.buf);
            ok = rc2 == RC_OK;
            t.push_back(ms);
        }
        float med = -1.f;
        if (ok) {
            std::sort(t.begin(), t.end());
            med = t[t.size() / 2];
            if (best < 0.f || med < best) {
                best = med;
                *best_max_groups = c.max_groups;
            }
        }
        if (times_ms) times_ms[i] = med;
    }
    CK(cudaStreamSynchronize(st));
    if (best < 0.f) return err.set(RC_ARG, "autotune: no candidate could be launched");
    return RC_OK;
}

extern "C" int cuopus_resample48to16(const int16_t *in_dev, int64_t avail, int64_t n_out, float *out_dev,
                                     void *cuda_stream, char *errbuf, size_t errcap)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Err err(errbuf, errcap);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    int rc = refuse_capture(st, err);
    if (rc) return rc;
    if (n_out > 0 && (!in_dev || !out_dev)) return err.set(RC_ARG, "NULL buffer");
    if ((rc = resample(in_dev, avail, n_out, out_dev, st, err))) return rc;
    CK(cudaStreamSynchronize(st));
    return RC_OK;
}

extern "C" int cuopus_warmup(char *errbuf, size_t errcap)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Err err(errbuf, errcap);
    int rc = ensure_occupancy(err);
    if (rc) return rc;
    if ((rc = ensure_events(err))) return rc;
    int width = default_width();
    long long nslots = resident_groups(BLOCK, width);
    if ((rc = gpu_grow(G.slots, (size_t)nslots * sizeof(cuo::ChainSlot), err))) return rc;
    if ((rc = ensure_taps(nullptr, err))) return rc;
    CK(cudaDeviceSynchronize());
    return RC_OK;
}

extern "C" long long cuopus_slot_bytes(void) { return (long long)sizeof(cuo::ChainSlot); }

extern "C" int cuopus_default_width(void) { return default_width(); }
