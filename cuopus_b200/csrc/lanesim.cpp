// Lane-interleaving host build of the chain decoder (test only).
//
// The CUDA kernel decodes one chain with a group of `width` lanes that run the
// decoder's scalar code redundantly on the same data and split independent
// loops between them (dec/common.cuh).  Nothing in the CUDA programming model
// keeps the lanes of a group in lockstep between two __syncwarp barriers, so
// the decoder is correct only if every stretch of code between two barriers
// gives the same result whatever the order in which the lanes' memory
// accesses interleave.  This build checks exactly that on the host:
//
//   * every lane of a group is a fiber (ucontext) with a stack of its own, all
//     fibers of a group on one OS thread, sharing one decoder slot as the
//     lanes of a group share theirs in device memory;
//   * the decoder sources are compiled with -finstrument-functions, so every
//     function entry (the fixed-point helpers included) is a point at which
//     the running fiber may be switched out; after a random run of `max_run`
//     entries at most, a random other runnable lane is switched in
//     (max_run = 0: lanes switch only at barriers, each one running a whole
//     stretch before the next starts);
//   * lsync is a barrier over the fibers, lsum and lscan_affine exchange their
//     values through the barrier, as the warp shuffles do on the device.
//
// A stretch whose result depends on the lanes staying in lockstep (a lane
// overwriting group memory that another lane has yet to read) then decodes
// wrong samples, and the CPU tests compare every sample with libopus.
// Test-only; the product library never loads it.
#include <dlfcn.h>
#include <execinfo.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <ucontext.h>

#include "dec/chain.cuh"

#define NOINSTR __attribute__((no_instrument_function))

namespace cuo {

enum { SIM_MAX_LANES = 32, SIM_STACK = 1 << 20 };
enum LaneState { RUNNABLE = 0, AT_BARRIER = 1, FINISHED = 2 };

struct LaneSim {
    int n;
    int cur;
    int arrived;
    uint64_t gen;
    uint64_t rng;
    int max_run;
    long budget;
    int busy;                      // inside the scheduler: no switching
    unsigned long long switches;
    ucontext_t main_ctx;
    ucontext_t ctx[SIM_MAX_LANES];
    char *stack[SIM_MAX_LANES];
    int state[SIM_MAX_LANES];
    int32_t xv[SIM_MAX_LANES];
    uint32_t xa[SIM_MAX_LANES], xb[SIM_MAX_LANES];
    unsigned char xbytes[256];
    // the chain every lane decodes
    ChainSlot *slot;
    const uint8_t *data;
    const uint64_t *off;
    const uint32_t *len;
    uint32_t first, npkts;
    int channels;
    int16_t *out;
    uint64_t trim, keep;
    uint32_t *pkt_nsamp, *pkt_rng;
    ChainResult *res;
    int fec;
    // hazard detector (barrier-only schedule): the slot as the barrier released
    // (s0) and as the previous lane arrived (sp)
    int detect;
    unsigned char *s0, *sp;
    unsigned long long hazards;
    char prev_at[SIM_MAX_LANES][160];   // where each lane's previous barrier was
};

static int g_detect_reports = 0;

static __thread LaneSim *t_sim;

NOINSTR static uint64_t sim_rand(LaneSim *s)
{
    uint64_t x = s->rng;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    s->rng = x;
    return x;
}

NOINSTR static long sim_run_length(LaneSim *s)
{
    return s->max_run > 0 ? 1 + (long)(sim_rand(s) % (uint64_t)s->max_run) : 0x7fffffffffffL;
}

// Switch to a random runnable lane other than the current one, if there is
// one; the current lane must itself be runnable then, or be waiting.
NOINSTR static void sim_switch(LaneSim *s)
{
    int cand[SIM_MAX_LANES], k = 0;
    for (int i = 0; i < s->n; i++)
        if (i != s->cur && s->state[i] == RUNNABLE) cand[k++] = i;
    if (k == 0) return;
    int from = s->cur, to = cand[sim_rand(s) % (uint64_t)k];
    s->cur = to;
    s->switches++;
    s->busy = 0;
    swapcontext(&s->ctx[from], &s->ctx[to]);
    s->busy = 1;
}

// Detector of the barrier-only schedule: lanes run their stretches one after
// another, so the bytes a lane changes are exactly its stretch's writes.  A
// byte that an earlier lane of the same stretch changed and this lane changes
// again (to another value) was computed from what the earlier lane had
// already overwritten: a hazard.
NOINSTR static void sim_where(char *at, size_t cap)
{
    void *fr[7];
    int nf = backtrace(fr, 7);
    int o = 0;
    at[0] = 0;
    for (int k = 2; k < nf && o < (int)cap - 20; k++) {
        Dl_info di;
        uintptr_t rel = (uintptr_t)fr[k];
        if (dladdr(fr[k], &di) && di.dli_fbase) rel -= (uintptr_t)di.dli_fbase;
        o += snprintf(at + o, cap - (size_t)o, " +0x%lx", (unsigned long)rel);
    }
}

NOINSTR static void sim_detect(LaneSim *s, int id, void *where)
{
    const unsigned char *cur = (const unsigned char *)s->slot;
    const size_t nb = sizeof(ChainSlot);
    long first = -1, count = 0;
    long runs[8];
    int nruns = 0;
    for (size_t i = 0; i < nb; i++)
        if (cur[i] != s->sp[i] && s->sp[i] != s->s0[i]) {
            if (first < 0) first = (long)i;
            if (nruns < 8 && (nruns == 0 || (long)i > runs[nruns - 1] + 8)) runs[nruns++] = (long)i;
            count++;
        }
    if (count) {
        s->hazards++;
        if (s->hazards == 1 && g_detect_reports < 400) {   // the first of a chain: later ones may follow from it
            g_detect_reports++;
            void *fr[6];
            int nf = backtrace(fr, 6);
            char at[160];
            int o = 0;
            for (int k = 1; k < nf && o < 140; k++) {
                Dl_info di;
                uintptr_t rel = (uintptr_t)fr[k];
                if (dladdr(fr[k], &di) && di.dli_fbase) rel -= (uintptr_t)di.dli_fbase;
                o += snprintf(at + o, sizeof at - (size_t)o, " +0x%lx", (unsigned long)rel);
            }
            (void)where;
            char rs[128];
            int ro = 0;
            for (int k = 0; k < nruns; k++) ro += snprintf(rs + ro, sizeof rs - (size_t)ro, " %ld", runs[k]);
            fprintf(stderr, "lanesim: hazard (barrier %llu, lane %d): %ld bytes at slot+%s, stack%s, from%s\n",
                    (unsigned long long)s->gen, id, count, rs, at, s->prev_at[id]);
        }
    }
    memcpy(s->sp, cur, nb);
    sim_where(s->prev_at[id], sizeof s->prev_at[id]);
}

void lanesim_sync(LaneSim *s, int id) NOINSTR;
void lanesim_sync(LaneSim *s, int id)
{
    s->busy = 1;
    uint64_t g = s->gen;
    if (s->detect) sim_detect(s, id, __builtin_return_address(0));
    if (++s->arrived == s->n) {   // the last lane in releases the others
        if (s->detect) memcpy(s->s0, s->slot, sizeof(ChainSlot));
        s->arrived = 0;
        s->gen++;
        for (int i = 0; i < s->n; i++)
            if (s->state[i] == AT_BARRIER) s->state[i] = RUNNABLE;
        s->budget = sim_run_length(s);
        sim_switch(s);            // let a random lane go first after the barrier
    } else {
        s->state[id] = AT_BARRIER;
        while (s->gen == g) {
            int runnable = 0;
            for (int i = 0; i < s->n; i++) runnable += s->state[i] == RUNNABLE;
            if (!runnable) {      // lanes disagree on the number of barriers
                fprintf(stderr, "lanesim: lane %d waits at a barrier no other lane will reach\n", id);
                abort();
            }
            sim_switch(s);
        }
    }
    s->busy = 0;
}

int32_t lanesim_sum(LaneSim *s, int id, int32_t v) NOINSTR;
int32_t lanesim_sum(LaneSim *s, int id, int32_t v)
{
    s->xv[id] = v;
    lanesim_sync(s, id);
    uint32_t t = 0;
    for (int i = 0; i < s->n; i++) t += (uint32_t)s->xv[i];
    lanesim_sync(s, id);          // nobody refills xv before every lane has read it
    return (int32_t)t;
}

void lanesim_scan_affine(LaneSim *s, int id, uint32_t *a, uint32_t *b) NOINSTR;
void lanesim_scan_affine(LaneSim *s, int id, uint32_t *a, uint32_t *b)
{
    s->xa[id] = *a;
    s->xb[id] = *b;
    lanesim_sync(s, id);
    uint32_t A = 1, B = 0;        // maps of lanes 0 .. id-1, lane 0's applied first
    for (int i = 0; i < id; i++) {
        B = s->xa[i] * B + s->xb[i];
        A = s->xa[i] * A;
    }
    lanesim_sync(s, id);
    *a = A;
    *b = B;
}

void lanesim_bcast(LaneSim *s, int id, void *p, int bytes) NOINSTR;
void lanesim_bcast(LaneSim *s, int id, void *p, int bytes)
{
    if (id == 0) memcpy(s->xbytes, p, (size_t)bytes);
    lanesim_sync(s, id);
    if (id != 0) memcpy(p, s->xbytes, (size_t)bytes);
    lanesim_sync(s, id);
}

NOINSTR static void sim_lane_main(unsigned lo, unsigned hi, int id)
{
    LaneSim *s = (LaneSim *)(((uintptr_t)hi << 32) | (uintptr_t)lo);
    Lanes L;
    L.id = id;
    L.n = s->n;
    L.mask = s->n == 32 ? 0xffffffffu : ((1u << s->n) - 1u);
    L.sim = s;
    s->busy = 0;
    decode_chain(L, s->slot, s->data, s->off, s->len, s->first, s->npkts, s->channels, s->out, s->trim, s->keep,
                 L.id == 0 ? s->pkt_nsamp : nullptr, L.id == 0 ? s->pkt_rng : nullptr, s->res, nullptr, s->fec);
    s->busy = 1;
    s->state[id] = FINISHED;
    int left = 0;
    for (int i = 0; i < s->n; i++) left += s->state[i] != FINISHED;
    if (left == 0) {
        setcontext(&s->main_ctx);
    }
    sim_switch(s);                // never returns: another lane finishes us off
    setcontext(&s->main_ctx);
}

// Decode one chain with n fiber lanes.
NOINSTR static void sim_decode(LaneSim *s)
{
    s->arrived = 0;
    s->gen = 0;
    s->busy = 1;
    for (int i = 0; i < s->n; i++) {
        s->state[i] = RUNNABLE;
        getcontext(&s->ctx[i]);
        s->ctx[i].uc_stack.ss_sp = s->stack[i];
        s->ctx[i].uc_stack.ss_size = SIM_STACK;
        s->ctx[i].uc_link = &s->main_ctx;
        uintptr_t p = (uintptr_t)s;
        makecontext(&s->ctx[i], (void (*)())sim_lane_main, 3, (unsigned)(p & 0xffffffffu), (unsigned)(p >> 32), i);
    }
    s->cur = (int)(sim_rand(s) % (uint64_t)s->n);
    s->budget = sim_run_length(s);
    if (s->detect) {
        memcpy(s->s0, s->slot, sizeof(ChainSlot));
        memcpy(s->sp, s->slot, sizeof(ChainSlot));
    }
    t_sim = s;
    swapcontext(&s->main_ctx, &s->ctx[s->cur]);
    t_sim = nullptr;
}

} // namespace cuo

extern "C" {

NOINSTR void __cyg_profile_func_enter(void *, void *)
{
    cuo::LaneSim *s = cuo::t_sim;
    if (!s || s->busy) return;
    if (--s->budget > 0) return;
    s->busy = 1;
    s->budget = cuo::sim_run_length(s);
    cuo::sim_switch(s);
    s->busy = 0;
}

NOINSTR void __cyg_profile_func_exit(void *, void *) {}

struct ls_job {
    const uint8_t *data;
    const uint64_t *off;
    const uint32_t *len;
    const uint32_t *first, *npkts;
    const int32_t *channels;
    int16_t *pcm;
    const uint64_t *pcm_off, *trim, *keep, *rec_off;
    uint32_t *pkt_nsamp, *pkt_rng;
    cuo::ChainResult *res;
    int nchains, width, max_run, fec, detect;
    uint64_t seed;
    unsigned long long switches, hazards;
    int next;
    pthread_mutex_t mu;
};

NOINSTR static void *ls_worker(void *arg)
{
    ls_job *j = (ls_job *)arg;
    cuo::LaneSim *s = (cuo::LaneSim *)calloc(1, sizeof(cuo::LaneSim));
    cuo::ChainSlot *slot = (cuo::ChainSlot *)malloc(sizeof(cuo::ChainSlot));
    bool ok = s && slot;
    for (int i = 0; ok && i < j->width; i++) ok = (s->stack[i] = (char *)malloc(cuo::SIM_STACK)) != nullptr;
    if (ok) {
        memset(slot, 0xA5, sizeof(cuo::ChainSlot));   // like fresh device memory
        s->n = j->width;
        s->max_run = j->max_run;
        s->slot = slot;
        s->data = j->data;
        s->off = j->off;
        s->len = j->len;
        s->fec = j->fec;
        s->detect = j->max_run == 0 && j->detect;
        if (s->detect) {
            s->s0 = (unsigned char *)malloc(sizeof(cuo::ChainSlot));
            s->sp = (unsigned char *)malloc(sizeof(cuo::ChainSlot));
            if (!s->s0 || !s->sp) s->detect = 0;
        }
        for (;;) {
            pthread_mutex_lock(&j->mu);
            int c = j->next++;
            pthread_mutex_unlock(&j->mu);
            if (c >= j->nchains) break;
            uint64_t r = j->rec_off ? j->rec_off[c] : 0;
            s->rng = (j->seed + 0x9E3779B97F4A7C15ull * (uint64_t)(c + 1)) | 1;
            s->first = j->first[c];
            s->npkts = j->npkts[c];
            s->channels = j->channels[c];
            s->out = j->pcm ? j->pcm + j->pcm_off[c] : nullptr;
            s->trim = j->trim ? j->trim[c] : 0;
            s->keep = j->keep ? j->keep[c] : (uint64_t)-1 / 4;
            s->pkt_nsamp = j->pkt_nsamp ? j->pkt_nsamp + r : nullptr;
            s->pkt_rng = j->pkt_rng ? j->pkt_rng + r : nullptr;
            s->res = &j->res[c];
            unsigned long long before = s->hazards;
            s->hazards = 0;
            cuo::sim_decode(s);
            s->hazards += before;
        }
        pthread_mutex_lock(&j->mu);
        j->switches += s->switches;
        j->hazards += s->hazards;
        pthread_mutex_unlock(&j->mu);
    }
    if (s) {
        free(s->s0);
        free(s->sp);
    }
    if (s)
        for (int i = 0; i < cuo::SIM_MAX_LANES; i++) free(s->stack[i]);
    free(s);
    free(slot);
    return nullptr;
}

// hc_decode_chains_fec of the one-lane host build, with `width` fiber lanes
// per chain, switching after at most `max_run` instrumented function entries
// (0: only at barriers), seeded by `seed`.  With max_run 0 and detect set,
// every stretch between barriers is also checked for bytes of the decoder
// slot that a later lane rewrote after an earlier lane had changed them; the
// count goes to *hazards (may be null) and the first hazard of each chain is
// reported on stderr with the code locations of the stretch's two barriers.
// Returns the number of lane switches made, or -1 on bad arguments.
NOINSTR long long ls_decode_chains(const uint8_t *data, const uint64_t *off, const uint32_t *len,
                                   const uint32_t *first, const uint32_t *npkts, const int32_t *channels,
                                   int nchains, int16_t *pcm, const uint64_t *pcm_off, const uint64_t *trim,
                                   const uint64_t *keep, const uint64_t *rec_off, uint32_t *pkt_nsamp,
                                   uint32_t *pkt_rng, void *res, int nthreads, int fec, int width, int max_run,
                                   uint64_t seed, int detect, unsigned long long *hazards)
{
    if (width < 1 || width > cuo::SIM_MAX_LANES || (width & (width - 1)) || max_run < 0) return -1;
    ls_job j;
    memset(&j, 0, sizeof j);
    j.data = data; j.off = off; j.len = len; j.first = first; j.npkts = npkts; j.channels = channels;
    j.pcm = pcm; j.pcm_off = pcm_off; j.trim = trim; j.keep = keep; j.rec_off = rec_off;
    j.pkt_nsamp = pkt_nsamp; j.pkt_rng = pkt_rng; j.res = (cuo::ChainResult *)res;
    j.nchains = nchains; j.width = width; j.max_run = max_run; j.fec = fec; j.seed = seed; j.detect = detect;
    pthread_mutex_init(&j.mu, nullptr);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 64) nthreads = 64;
    pthread_t th[64];
    int started = 0;
    for (int t = 0; t < nthreads; t++) {
        if (pthread_create(&th[t], nullptr, ls_worker, &j) != 0) break;
        started++;
    }
    if (!started) ls_worker(&j);
    for (int t = 0; t < started; t++) pthread_join(th[t], nullptr);
    pthread_mutex_destroy(&j.mu);
    if (hazards) *hazards = j.hazards;
    return (long long)j.switches;
}

}
