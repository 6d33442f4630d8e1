// Continuous-batching decode server (extension; the reference serves one
// request at a time from its daemon, decode_cli.cu:572-678).
//
// Requests (Ogg Opus files) are demuxed and cut into chains on the caller's
// thread at submit time and queued.  One server thread owns the GPU work:
//   * admission: a queued request is admitted when its packets, PCM and output
//     fit in the free space of one device arena of `budget_bytes`, allocated
//     once at start (first fit over 256-byte granules, host-side bookkeeping)
//     and kept resident with the decoder slots between requests;
//   * waves: chains of admitted requests, oldest request first, are packed into
//     decode waves of at most `wave_chains` chains; up to `max_inflight` waves
//     run at once, each on its own stream with its own decoder slots and
//     tables, so a request that arrives while others decode joins the next
//     wave and its work overlaps theirs on the device.  While two or more
//     waves are in flight a new wave is held back until it can take half of
//     `wave_chains` or its oldest chain has waited BATCH_WAIT_MS: launching
//     every trickle of arrivals as its own small wave would spend the in-flight
//     waves on a few chains each and leave most of the GPU idle;
//   * completion: after a wave the per-chain results are checked (status and
//     sample count against the TOC capacity, as in the one-shot entry points);
//     when every chain of a request is done its PCM is resampled (f16k) and
//     the request completes with its latency from submit.
// Each chain is decoded by a fresh decoder over its own packets into its own
// keep window, so a request's output does not depend on what it was batched
// with.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cuopus.h"
#define CUO_NO_RESAMPLE_KERNEL 1
#include "kernels.cuh"
#include "ogg_demux.h"

namespace {

double now_ms()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

int fail(char *errbuf, size_t errcap, int rc, const char *fmt, ...)
{
    if (errbuf && errcap) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(errbuf, errcap, fmt, ap);
        va_end(ap);
    }
    return rc;
}

const size_t GRAN = 256;
size_t rup(size_t x) { return (x + GRAN - 1) & ~(GRAN - 1); }

// First-fit allocator of byte ranges of the device arena (host bookkeeping).
struct RangeAlloc {
    std::map<size_t, size_t> free_;   // offset -> size
    size_t total = 0, used = 0;
    void init(size_t n)
    {
        free_.clear();
        free_[0] = n;
        total = n;
        used = 0;
    }
    bool alloc(size_t n, size_t *off)
    {
        n = rup(n ? n : 1);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                *off = it->first;
                size_t rest = it->second - n, o = it->first + n;
                free_.erase(it);
                if (rest) free_[o] = rest;
                used += n;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t n)
    {
        n = rup(n ? n : 1);
        used -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Request {
    uint64_t id = 0;
    double t_submit = 0, t_done = 0, t_admit = 0;
    cuo_host::Demux d;
    cuo_host::Chains c;
    std::vector<uint64_t> cap;             // per chain TOC capacity
    uint64_t keep_total = 0;               // kept samples per channel
    int64_t n16 = 0;                       // f16k output samples
    size_t arena_off = 0, arena_bytes = 0, blob_off = 0, pcm_off = 0, f32_off = 0;
    uint32_t next_chain = 0, chains_done = 0;
    bool admitted = false, done = false, failed = false;
    // packets are uploaded on the stream of the first wave that holds one of
    // the request's chains; waves on other streams wait for this event
    cudaStream_t up_st = nullptr;
    cudaEvent_t up_ev = nullptr;
    ~Request()
    {
        if (up_ev) cudaEventDestroy(up_ev);
    }
    std::string error;
    std::vector<uint64_t> chain_out;       // per chain int16 element offset in its PCM
};

struct Wave {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    bool busy = false;
    double t_launch = 0;
    // device tables (grow-only) and pinned staging
    void *d_tab = nullptr;
    size_t d_cap = 0;
    void *h_tab = nullptr;
    size_t h_cap = 0;
    void *slots = nullptr;
    // chain results land in the pinned table (a copy into pageable memory
    // would return only after the kernel, holding every other wave back)
    uint32_t *d_res = nullptr;
    const uint32_t *h_res = nullptr;
    std::vector<std::pair<Request *, uint32_t>> chains;   // (request, chain index)
    // resample jobs issued on this stream after the decode
    std::vector<Request *> finishing;
};

} // namespace

struct cuopus_server {
    cuopus_server_config cfg{};
    int dev = 0;
    int width = 32, block = 128, groups = 0;
    uint8_t *arena = nullptr;
    RangeAlloc ra;
    std::vector<Wave> waves;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> pending;                 // submitted, not admitted (FIFO)
    std::vector<Request *> active;                 // admitted, chains left to launch or finish
    std::map<uint64_t, std::unique_ptr<Request>> reqs;
    uint64_t next_id = 1;
    bool stop = false;
    std::string fatal;
    std::thread th;
    // statistics
    int64_t n_done = 0, n_failed = 0, n_waves = 0, n_chains = 0;
    double audio_s = 0, t_first_submit = -1, t_last_done = 0, busy_ms = 0;
    std::vector<double> lat;

    void run();
    bool admit_locked();
    bool worth_launching_locked();
    bool build_wave_locked(Wave &w);
    void finish_wave(Wave &w);
};

namespace {

struct Tab {   // per-wave table layout inside one device / pinned buffer
    size_t off, len, first, npkts, chans, trim, keep, out_off, res, blobs, total;
};

// `blob_bytes`: packets of the requests this wave uploads, staged in the
// pinned buffer only (the device table does not hold them)
Tab layout(size_t npk, size_t nch, size_t blob_bytes = 0)
{
    Tab t;
    size_t o = 0;
    auto put = [&](size_t bytes) { size_t r = o; o = rup(o + bytes); return r; };
    t.off = put(8 * npk);
    t.len = put(4 * npk);
    t.first = put(4 * nch);
    t.npkts = put(4 * nch);
    t.chans = put(nch);
    t.trim = put(8 * nch);
    t.keep = put(8 * nch);
    t.out_off = put(8 * nch);
    t.res = put(16 * nch);
    t.blobs = put(blob_bytes);
    t.total = o;
    return t;
}

} // namespace

// Admit queued requests, oldest first, while their bytes fit in the arena.
// Stops at the first request that does not fit so admission stays in order.
bool cuopus_server::admit_locked()
{
    bool any = false;
    while (!pending.empty()) {
        Request *r = pending.front();
        size_t blob = rup(r->d.blob.size() + 16);
        size_t pcm = rup(2 * (size_t)r->keep_total * (size_t)r->d.channels + 16);
        size_t f32 = cfg.f16k ? rup(4 * (size_t)std::max<int64_t>(r->n16, 1)) : 0;
        size_t need = blob + pcm + f32;
        size_t off = 0;
        if (!ra.alloc(need, &off)) {
            if (need > ra.total) {     // can never fit: fail it instead of blocking the queue
                pending.pop_front();
                r->failed = r->done = true;
                r->error = "request needs more device memory than the admission budget";
                n_failed++;
                cv_done.notify_all();
                continue;
            }
            break;
        }
        pending.pop_front();
        r->arena_off = off;
        r->arena_bytes = need;
        r->blob_off = off;
        r->pcm_off = off + blob;
        r->f32_off = off + blob + pcm;
        r->admitted = true;
        r->t_admit = now_ms();
        active.push_back(r);
        any = true;
    }
    return any;
}

const double BATCH_WAIT_MS = 5.0;

// Whether a wave should be launched now (see the header comment).
bool cuopus_server::worth_launching_locked()
{
    size_t avail = 0;
    double oldest = -1;
    for (Request *r : active) {
        size_t left = r->c.size() - r->next_chain;
        if (left && oldest < 0) oldest = r->t_admit;
        avail += left;
    }
    if (!avail) return false;
    int busy = 0;
    for (const Wave &w : waves) busy += w.busy;
    return busy < 2 || stop || avail >= (size_t)std::max(groups / 2, 1) || now_ms() - oldest >= BATCH_WAIT_MS;
}

// Pack up to wave_chains chains of admitted requests (oldest first) into w.
bool cuopus_server::build_wave_locked(Wave &w)
{
    w.chains.clear();
    size_t npk = 0;
    for (Request *r : active) {
        while (r->next_chain < r->c.size() && (int)w.chains.size() < groups) {
            uint32_t i = r->next_chain++;
            w.chains.push_back({r, i});
            npk += r->c.npkts[i];
        }
        if ((int)w.chains.size() >= groups) break;
    }
    return !w.chains.empty();
}

void cuopus_server::run()
{
    cudaSetDevice(dev);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        if (stop && pending.empty() && active.empty()) break;
        if (!fatal.empty()) break;
        admit_locked();
        // upload the packets of newly admitted requests happens at wave build
        // time (the blob copy is issued on the wave's stream before the kernel)
        bool launched = false;
        for (Wave &w : waves) {
            if (w.busy) continue;
            if (!worth_launching_locked() || !build_wave_locked(w)) break;
            // host tables for this wave
            size_t npk = 0, nch = w.chains.size(), blob_bytes = 0;
            for (size_t c = 0; c < nch; c++) {
                const Request *r = w.chains[c].first;
                npk += r->c.npkts[w.chains[c].second];
                if (!r->up_st && (c == 0 || w.chains[c - 1].first != r)) blob_bytes += rup(r->d.blob.size());
            }
            Tab t = layout(npk, nch, blob_bytes);
            lk.unlock();
            cudaError_t e = cudaSuccess;
            if (t.total > w.h_cap) {
                if (w.h_tab) cudaFreeHost(w.h_tab);
                w.h_tab = nullptr;
                e = cudaMallocHost(&w.h_tab, t.total * 2);
                w.h_cap = e == cudaSuccess ? t.total * 2 : 0;
            }
            if (e == cudaSuccess && t.blobs > w.d_cap) {
                if (w.d_tab) cudaFree(w.d_tab);
                w.d_tab = nullptr;
                e = cudaMalloc(&w.d_tab, t.blobs * 2);
                w.d_cap = e == cudaSuccess ? t.blobs * 2 : 0;
            }
            if (e == cudaSuccess) {
                uint8_t *h = (uint8_t *)w.h_tab;
                uint64_t *off = (uint64_t *)(h + t.off);
                uint32_t *len = (uint32_t *)(h + t.len);
                uint32_t *first = (uint32_t *)(h + t.first), *npkts = (uint32_t *)(h + t.npkts);
                uint8_t *chans = h + t.chans;
                uint64_t *trim = (uint64_t *)(h + t.trim), *keep = (uint64_t *)(h + t.keep);
                uint64_t *out_off = (uint64_t *)(h + t.out_off);
                size_t p = 0, staged = t.blobs;
                for (size_t c = 0; c < nch; c++) {
                    Request *r = w.chains[c].first;
                    uint32_t i = w.chains[c].second;
                    if (!r->up_st) {
                        // first wave to hold one of the request's chains: upload its
                        // packets through the pinned table, so that the copy returns
                        // at once instead of waiting for the stream's earlier work
                        memcpy(h + staged, r->d.blob.data(), r->d.blob.size());
                        e = cudaMemcpyAsync(arena + r->blob_off, h + staged, r->d.blob.size(),
                                            cudaMemcpyHostToDevice, w.st);
                        staged += rup(r->d.blob.size());
                        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->up_ev, cudaEventDisableTiming);
                        if (e == cudaSuccess) e = cudaEventRecord(r->up_ev, w.st);
                        r->up_st = w.st;
                    } else if (r->up_st != w.st && (c == 0 || w.chains[c - 1].first != r)) {
                        e = cudaStreamWaitEvent(w.st, r->up_ev, 0);
                    }
                    first[c] = (uint32_t)p;
                    npkts[c] = r->c.npkts[i];
                    for (uint32_t k = 0; k < r->c.npkts[i]; k++, p++) {
                        uint32_t q = r->c.first[i] + k;
                        off[p] = (uint64_t)r->blob_off + r->d.off[q];
                        len[p] = r->d.len[q];
                    }
                    chans[c] = (uint8_t)r->d.channels;
                    trim[c] = r->c.trim[i];
                    keep[c] = r->c.keep[i];
                    out_off[c] = r->pcm_off / 2 + r->chain_out[i];
                }
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(w.d_tab, w.h_tab, t.res, cudaMemcpyHostToDevice, w.st);
            }
            if (e == cudaSuccess) {
                uint8_t *d = (uint8_t *)w.d_tab;
                cuo::DecodeArgs a;
                memset(&a, 0, sizeof a);
                a.data = arena;
                a.off = (const uint64_t *)(d + t.off);
                a.len = (const uint32_t *)(d + t.len);
                a.first = (const uint32_t *)(d + t.first);
                a.npkts = (const uint32_t *)(d + t.npkts);
                a.channels = d + t.chans;
                a.trim = (const uint64_t *)(d + t.trim);
                a.keep = (const uint64_t *)(d + t.keep);
                a.out_off = (const uint64_t *)(d + t.out_off);
                a.out = (int16_t *)arena;
                a.res = (cuo::ChainResult *)(d + t.res);
                a.slots = (cuo::ChainSlot *)w.slots;
                a.nchains = (int)nch;
                a.width = width;
                int gpb = block / width;
                int blocks = (int)((nch + gpb - 1) / gpb);
                w.d_res = (uint32_t *)(d + t.res);
                w.t_launch = now_ms();
                e = cuo::decode_kernel_launch(a, blocks, block, w.st);
                if (e == cudaSuccess) {
                    w.h_res = (const uint32_t *)((uint8_t *)w.h_tab + t.res);
                    e = cudaMemcpyAsync((uint8_t *)w.h_tab + t.res, w.d_res, 16 * nch, cudaMemcpyDeviceToHost,
                                        w.st);
                }
                if (e == cudaSuccess) e = cudaEventRecord(w.ev, w.st);
            }
            lk.lock();
            if (e != cudaSuccess) {
                fatal = std::string("server decode launch: ") + cudaGetErrorString(e);
                break;
            }
            w.busy = true;
            n_waves++;
            n_chains += (int64_t)nch;
            launched = true;
        }
        if (!fatal.empty()) break;
        // completions
        bool completed = false;
        for (Wave &w : waves) {
            if (!w.busy) continue;
            if (cudaEventQuery(w.ev) == cudaErrorNotReady) continue;
            lk.unlock();
            finish_wave(w);
            lk.lock();
            w.busy = false;
            completed = true;
        }
        if (!fatal.empty()) break;
        if (!launched && !completed) {
            bool any_busy = false;
            for (Wave &w : waves) any_busy |= w.busy;
            if (any_busy) {
                lk.unlock();
                // a short sleep instead of a blocking sync keeps admission live
                struct timespec ts = {0, 200000};
                nanosleep(&ts, nullptr);
                lk.lock();
            } else {
                cv_work.wait_for(lk, std::chrono::milliseconds(50));
            }
        }
    }
    if (!fatal.empty()) {
        for (auto &kv : reqs)
            if (!kv.second->done) {
                kv.second->failed = kv.second->done = true;
                kv.second->error = fatal;
            }
        cv_done.notify_all();
    }
}

// Check a finished wave's chains; complete the requests whose chains are all
// done (resample first when the server produces f16k).
void cuopus_server::finish_wave(Wave &w)
{
    cudaError_t e = cudaEventSynchronize(w.ev);
    std::vector<Request *> finished;
    {
        std::lock_guard<std::mutex> g(mu);
        busy_ms += now_ms() - w.t_launch;
        for (size_t c = 0; c < w.chains.size(); c++) {
            Request *r = w.chains[c].first;
            uint32_t i = w.chains[c].second;
            int32_t stop_ = (int32_t)w.h_res[4 * c];
            uint32_t samples = w.h_res[4 * c + 1];
            if (e != cudaSuccess) {
                fatal = std::string("server decode: ") + cudaGetErrorString(e);
            } else if (!r->failed && (stop_ != 0 || samples != r->cap[i])) {
                r->failed = true;
                char m[160];
                snprintf(m, sizeof m, "chain %u: status %d, %u of %llu samples", i, stop_, samples,
                         (unsigned long long)r->cap[i]);
                r->error = m;
            }
            if (++r->chains_done == r->c.size()) finished.push_back(r);
        }
    }
    for (Request *r : finished) {
        if (!r->failed && cfg.f16k && r->n16 > 0) {
            cudaError_t e2 = cuo::resample_into((const int16_t *)(arena + r->pcm_off), (long long)r->keep_total,
                                                r->n16, (float *)(arena + r->f32_off), w.st);
            if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(w.st);
            if (e2 != cudaSuccess) {
                std::lock_guard<std::mutex> g(mu);
                fatal = std::string("server resample: ") + cudaGetErrorString(e2);
            }
        }
        std::lock_guard<std::mutex> g(mu);
        r->done = true;
        r->t_done = now_ms();
        active.erase(std::remove(active.begin(), active.end(), r), active.end());
        if (r->failed) {
            n_failed++;
        } else {
            n_done++;
            audio_s += (double)r->d.play48 / 48000.0;
            lat.push_back(r->t_done - r->t_submit);
            t_last_done = r->t_done;
        }
    }
    if (!finished.empty()) cv_done.notify_all();
}

// ====================================================================== C ABI

extern "C" int cuopus_server_create(const cuopus_server_config *cfg, cuopus_server **out, char *errbuf,
                                    size_t errcap)
{
    if (!out) return fail(errbuf, errcap, 3, "out is NULL");
    *out = nullptr;
    std::unique_ptr<cuopus_server> s(new cuopus_server());
    if (cfg) s->cfg = *cfg;
    if (s->cfg.budget_bytes <= 0) s->cfg.budget_bytes = 40ll << 30;
    if (s->cfg.max_inflight <= 0) s->cfg.max_inflight = 8;
    if (s->cfg.seg_s <= 0) s->cfg.seg_s = 1.0;
    if (s->cfg.preroll_ms < 0) s->cfg.preroll_ms = 250.0;
    if (s->cfg.preroll_ms == 0 && !(cfg && cfg->preroll_ms == 0)) s->cfg.preroll_ms = 250.0;
    // chains of a few seconds at most: many short chains decode faster at 8
    // lanes on every resident group than at 32 (the file entry points' rule)
    s->width = s->cfg.width > 0 ? s->cfg.width : (s->cfg.seg_s <= 4.0 ? 8 : 32);
    s->block = s->cfg.block > 0 ? s->cfg.block : 64;
    if ((s->width & (s->width - 1)) || s->width > 32 || s->block % s->width || s->block > 128 || s->block % 32)
        return fail(errbuf, errcap, 3, "bad width %d / block %d", s->width, s->block);
    cudaError_t e = cudaGetDevice(&s->dev);
    if (e != cudaSuccess) return fail(errbuf, errcap, 2, "cudaGetDevice: %s", cudaGetErrorString(e));
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->dev);
    e = cuo::decode_kernel_occupancy(s->block, s->width, &per_sm);
    if (e != cudaSuccess) return fail(errbuf, errcap, 2, "occupancy: %s", cudaGetErrorString(e));
    long long resident = (long long)sms * std::max(per_sm, 1) * (s->block / s->width);
    s->groups = (int)(s->cfg.wave_chains > 0 ? std::min<long long>(s->cfg.wave_chains, resident) : resident);
    s->cfg.wave_chains = s->groups;
    e = cudaMalloc((void **)&s->arena, (size_t)s->cfg.budget_bytes);
    if (e != cudaSuccess)
        return fail(errbuf, errcap, 2, "arena of %lld bytes: %s", (long long)s->cfg.budget_bytes,
                    cudaGetErrorString(e));
    s->ra.init((size_t)s->cfg.budget_bytes);
    s->waves.resize(s->cfg.max_inflight);
    int gpb = s->block / s->width;
    size_t nslots = (size_t)((s->groups + gpb - 1) / gpb) * gpb;
    for (Wave &w : s->waves) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&w.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w.ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&w.slots, nslots * sizeof(cuo::ChainSlot));
    }
    if (e != cudaSuccess) {
        cuopus_server_destroy(s.release());
        return fail(errbuf, errcap, 2, "server setup: %s", cudaGetErrorString(e));
    }
    cuopus_server *p = s.release();
    p->th = std::thread([p] { p->run(); });
    *out = p;
    return 0;
}

extern "C" int cuopus_server_submit(cuopus_server *s, const uint8_t *ogg, size_t n, uint64_t *id, char *errbuf,
                                    size_t errcap)
{
    if (!s || !ogg || !n || !id) return fail(errbuf, errcap, 3, "bad argument");
    std::unique_ptr<Request> r(new Request());
    r->t_submit = now_ms();
    std::string e;
    if (!cuo_host::demux_and_chain(ogg, n, s->cfg.seg_s, s->cfg.preroll_ms, s->cfg.f16k != 0, r->d, &r->c, e))
        return fail(errbuf, errcap, 1, "%s", e.c_str());
    if (r->c.size() == 0) return fail(errbuf, errcap, 1, "no chains");
    r->cap.resize(r->c.size());
    r->chain_out.resize(r->c.size());
    for (uint32_t i = 0; i < r->c.size(); i++) {
        uint64_t cap = r->c.cap[i];
        if (cap < (uint64_t)r->c.trim[i] + r->c.keep[i])
            return fail(errbuf, errcap, 1, "chain %u capacity %llu < trim + keep", i, (unsigned long long)cap);
        r->cap[i] = cap;
        r->chain_out[i] = r->keep_total * (uint64_t)r->d.channels;
        r->keep_total += r->c.keep[i];
    }
    int64_t v = ((int64_t)r->keep_total - 48) / 3;
    r->n16 = v < 0 ? 0 : v;
    std::lock_guard<std::mutex> g(s->mu);
    if (!s->fatal.empty()) return fail(errbuf, errcap, 2, "%s", s->fatal.c_str());
    if (s->stop) return fail(errbuf, errcap, 3, "server is stopping");
    r->id = s->next_id++;
    *id = r->id;
    if (s->t_first_submit < 0) s->t_first_submit = r->t_submit;
    s->pending.push_back(r.get());
    s->reqs[r->id] = std::move(r);
    s->cv_work.notify_all();
    return 0;
}

extern "C" int cuopus_server_wait(cuopus_server *s, uint64_t id, int64_t timeout_ms, void *host_out,
                                  size_t out_cap_bytes, int64_t *out_samples, int32_t *channels, double *latency_ms,
                                  char *errbuf, size_t errcap)
{
    if (!s) return fail(errbuf, errcap, 3, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(errbuf, errcap, 3, "unknown request %llu", (unsigned long long)id);
    Request *r = it->second.get();
    auto ready = [&] { return r->done; };
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
        return fail(errbuf, errcap, 4, "request %llu not done", (unsigned long long)id);
    std::unique_ptr<Request> own = std::move(it->second);
    s->reqs.erase(it);
    if (r->failed) {
        if (r->admitted) s->ra.release(r->arena_off, r->arena_bytes);
        s->cv_work.notify_all();
        return fail(errbuf, errcap, 1, "%s", r->error.c_str());
    }
    size_t bytes = s->cfg.f16k ? 4 * (size_t)r->n16 : 2 * (size_t)r->keep_total * (size_t)r->d.channels;
    if (out_samples) *out_samples = s->cfg.f16k ? r->n16 : (int64_t)r->keep_total;
    if (channels) *channels = r->d.channels;
    if (latency_ms) *latency_ms = r->t_done - r->t_submit;
    int rc = 0;
    if (host_out) {
        if (out_cap_bytes < bytes) {
            rc = fail(errbuf, errcap, 3, "output capacity %zu < %zu bytes", out_cap_bytes, bytes);
        } else if (bytes) {
            const uint8_t *src = s->arena + (s->cfg.f16k ? r->f32_off : r->pcm_off);
            lk.unlock();
            cudaError_t e = cudaMemcpy(host_out, src, bytes, cudaMemcpyDeviceToHost);
            lk.lock();
            if (e != cudaSuccess) rc = fail(errbuf, errcap, 2, "result copy: %s", cudaGetErrorString(e));
        }
    }
    s->ra.release(r->arena_off, r->arena_bytes);
    s->cv_work.notify_all();
    return rc;
}

extern "C" int cuopus_server_request_size(cuopus_server *s, uint64_t id, int64_t *out_samples,
                                          int32_t *channels, size_t *out_bytes)
{
    if (!s) return 3;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return 3;
    const Request *r = it->second.get();
    int64_t n = s->cfg.f16k ? r->n16 : (int64_t)r->keep_total;
    if (out_samples) *out_samples = n;
    if (channels) *channels = r->d.channels;
    if (out_bytes) *out_bytes = s->cfg.f16k ? 4 * (size_t)r->n16 : 2 * (size_t)r->keep_total * (size_t)r->d.channels;
    return 0;
}

extern "C" int cuopus_server_get_stats(cuopus_server *s, cuopus_server_stats *st)
{
    if (!s || !st) return 3;
    std::lock_guard<std::mutex> g(s->mu);
    memset(st, 0, sizeof *st);
    st->completed = s->n_done;
    st->failed = s->n_failed;
    st->waves = s->n_waves;
    st->chains = s->n_chains;
    st->pending = (int64_t)s->pending.size();
    st->active = (int64_t)s->active.size();
    st->audio_s = s->audio_s;
    st->wall_ms = s->t_first_submit >= 0 ? s->t_last_done - s->t_first_submit : 0;
    st->arena_used = (int64_t)s->ra.used;
    st->arena_bytes = (int64_t)s->ra.total;
    st->wave_chains = s->groups;
    std::vector<double> l = s->lat;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        st->p50_ms = l[(size_t)(0.50 * (l.size() - 1) + 0.5)];
        st->p99_ms = l[(size_t)(0.99 * (l.size() - 1) + 0.5)];
        st->max_ms = l.back();
    }
    return 0;
}

extern "C" void cuopus_server_destroy(cuopus_server *s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        s->pending.clear();
        s->cv_work.notify_all();
    }
    if (s->th.joinable()) s->th.join();
    for (Wave &w : s->waves) {
        if (w.st) cudaStreamSynchronize(w.st);
        if (w.ev) cudaEventDestroy(w.ev);
        if (w.st) cudaStreamDestroy(w.st);
        if (w.slots) cudaFree(w.slots);
        if (w.d_tab) cudaFree(w.d_tab);
        if (w.h_tab) cudaFreeHost(w.h_tab);
    }
    if (s->arena) cudaFree(s->arena);
    delete s;
}
