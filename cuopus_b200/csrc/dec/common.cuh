// Shared definitions of the chain decoder: compilation-target macros, the lane
// group abstraction, and the fixed-point arithmetic of the libopus 1.5.2
// FIXED_POINT decoder.
//
// Execution model.  One Opus chain is decoded by a group of `width` lanes of a
// warp (width 1..32).  All lanes of the group execute the scalar decoder code
// redundantly on identical data (they stay converged, and every store writes
// the same value), while loops whose iterations are independent are split
// across the lanes with LFOR and closed with lsync().  Big per-chain arrays
// live in a per-slot work area in global memory that every lane addresses
// identically; small temporaries stay in registers.  The same source compiles
// for the host with width 1 (g++), which the host-side parity tests use.
//
// Arithmetic.  The helpers below restate the operators of silk/macros.h,
// silk/SigProc_FIX.h, silk/Inlines.h (SILK) and celt/fixed_generic.h,
// celt/mathops.{h,c} (CELT).  Each is written from its definition as exact
// integer arithmetic: products are formed in 64 bits and shifted, 32-bit sums
// wrap, and saturation is explicit.  The 32-bit-only variants libopus selects
// when OPUS_FAST_INT64 is 0 compute the same values, so bit-exactness holds
// against either build.
#pragma once
#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define DFN static __device__ __forceinline__
#define MFN __device__ __forceinline__
#define DNI static __device__ __noinline__
#define MNI __device__ __noinline__
#define TABC(type, decl) static __constant__ type decl
#define TABG(type, decl) static __device__ const type decl
#else
#define DFN static inline
#define MFN inline
#define DNI static
#define MNI
#define TABC(type, decl) static const type decl
#define TABG(type, decl) static const type decl
#endif

namespace cuo {

#include "opus_tables.inc"

// ------------------------------------------------------------------ lanes

#if defined(CUO_LANE_SIM) && !defined(__CUDACC__)
// Lane-interleaving host build (test only, lanesim.cpp): every lane of a group
// is a fiber of its own and the fibers switch at random points of the decoder
// code, so an access to group memory that depends on the lanes running in
// lockstep shows up as a wrong sample.  The lane primitives below become
// barriers and exchanges between the fibers.
struct LaneSim;
void lanesim_sync(LaneSim *s, int id);
int32_t lanesim_sum(LaneSim *s, int id, int32_t v);
void lanesim_scan_affine(LaneSim *s, int id, uint32_t *a, uint32_t *b);
void lanesim_bcast(LaneSim *s, int id, void *p, int bytes);
#endif

struct Lanes {
    int id;          // lane index inside the chain's group
    int n;           // group width
    unsigned mask;   // warp mask of the group
#if defined(CUO_LANE_SIM) && !defined(__CUDACC__)
    LaneSim *sim;    // the group's fibers (null: one lane)
#endif
};

DFN void lsync(const Lanes &L)
{
#ifdef __CUDA_ARCH__
    __syncwarp(L.mask);
#elif defined(CUO_LANE_SIM)
    if (L.sim) lanesim_sync(L.sim, L.id);
#else
    (void)L;
#endif
}

// A serial stretch on the group's first lane alone; the other lanes wait at
// the barrier after it.  Code that updates group memory in place (reads a
// location, then writes it) is correct only if no lane writes a location that
// another lane has yet to read, and nothing keeps the lanes of a group in
// lockstep between barriers; with one lane doing all of the stretch's reads
// and writes, and barriers on both sides, that holds by construction.  Values
// the other lanes need afterwards go through group memory (or lbcast /
// rd_bcast).
// Lead bodies are written [&]() CUO_INLINE { ... }: inlined into the caller, so
// the variables they share with it stay in registers.
#define CUO_INLINE __attribute__((always_inline))
template <class F> DFN void lead(const Lanes &L, F &&body)
{
    lsync(L);
    if (L.id == 0) body();
    lsync(L);
}

// This lane as a group of its own, for a lead stretch that calls lane-split
// code: every LFOR iteration then runs on this lane and the barriers and
// lane sums reduce to nothing.
DFN Lanes lone(const Lanes &L)
{
    Lanes s = L;
    s.id = 0;
    s.n = 1;
#ifdef __CUDA_ARCH__
    s.mask = 1u << (threadIdx.x & 31);
#endif
#if defined(CUO_LANE_SIM) && !defined(__CUDACC__)
    s.sim = nullptr;
#endif
    return s;
}

// The first lane's value of v, on every lane of the group.
DFN int32_t lbcast(const Lanes &L, int32_t v)
{
#ifdef __CUDA_ARCH__
    if (L.n > 1) v = __shfl_sync(L.mask, v, (int)(threadIdx.x & 31) - L.id);
#elif defined(CUO_LANE_SIM)
    if (L.sim) lanesim_bcast(L.sim, L.id, &v, (int)sizeof v);
#else
    (void)L;
#endif
    return v;
}

// for (i = start; i < end; i++) split across the lanes of the group.  The
// iterations of an LFOR loop must not depend on each other; a host test build
// (CUO_LFOR_REVERSE) runs them in reverse order to check that they do not.
#ifdef CUO_LFOR_REVERSE
#define LFOR(L, i, start, end) for (int i = (end) - 1 - (L).id; i >= (start); i -= (L).n)
#else
#define LFOR(L, i, start, end) for (int i = (start) + (L).id; i < (end); i += (L).n)
#endif

// Stage timers of the diagnostic build (CUO_PHASE_TIMERS, libcuopus_phases.so):
// the first lane of each group adds the clock cycles a decoder stage took to
// that stage's device counter (cuopus_phase_read).  Other builds compile them
// to nothing.  Stage numbers: PH_* below.
enum {
    PH_PACKET = 0, PH_SILK_INDICES, PH_SILK_PULSES, PH_SILK_PARAMS, PH_SILK_CORE, PH_SILK_PLC, PH_SILK_CNG,
    PH_SILK_STEREO, PH_SILK_RESAMPLE, PH_CELT_COARSE, PH_CELT_ALLOC, PH_CELT_SHIFT, PH_CELT_BANDS,
    PH_CELT_SYNTH, PH_CELT_COMB, PH_CELT_DEEMPH, PH_KEEP_COPY,
    // parts of the stages above (nested in them)
    PH_PVQ_CWRSI, PH_PVQ_ROT, PH_PVQ_RENORM, PH_PVQ_THETA, PH_PVQ_TF, PH_SILK_LPC, PH_SILK_LTP, PH_SILK_SHELL,
    PH_COUNT
};
#if defined(CUO_PHASE_TIMERS) && defined(__CUDA_ARCH__)
__device__ void cuo_phase_add(int stage, long long cycles);
#define PHASE_BEGIN(v) long long v = clock64()
#define PHASE_END(k, v, lane)                                                                        \
    do {                                                                                             \
        if ((lane) == 0) cuo_phase_add((k), clock64() - (v));                                        \
    } while (0)
#else
#define PHASE_BEGIN(v) \
    do {               \
    } while (0)
#define PHASE_END(k, v, lane) \
    do {                      \
    } while (0)
#endif

// Sum of v over the lanes of the group with wrap-around 32-bit adds (so the
// order of the terms does not change the result); every lane gets the total.
DFN int32_t lsum(const Lanes &L, int32_t v)
{
#ifdef __CUDA_ARCH__
    for (int off = L.n >> 1; off > 0; off >>= 1) v = (int32_t)((uint32_t)v + (uint32_t)__shfl_xor_sync(L.mask, v, off));
#elif defined(CUO_LANE_SIM)
    if (L.sim) v = lanesim_sum(L.sim, L.id, v);
#else
    (void)L;
#endif
    return v;
}

// Exclusive prefix composition of affine maps x -> a*x + b (mod 2^32) over the
// lanes of the group, lane 0's map first: on return (a, b) is the composition
// of the maps of the lanes before this one, the identity on lane 0.  Modular
// arithmetic is exact, so any grouping of the compositions gives the serial
// result.
DFN void lscan_affine(const Lanes &L, uint32_t &a, uint32_t &b)
{
#ifdef __CUDA_ARCH__
    for (int off = 1; off < L.n; off <<= 1) {
        uint32_t pa = __shfl_up_sync(L.mask, a, off, L.n), pb = __shfl_up_sync(L.mask, b, off, L.n);
        if (L.id >= off) {   // this lane's span after the earlier one
            b = a * pb + b;
            a = a * pa;
        }
    }
    uint32_t pa = __shfl_up_sync(L.mask, a, 1, L.n), pb = __shfl_up_sync(L.mask, b, 1, L.n);
    if (L.id == 0) {
        a = 1;
        b = 0;
    } else {
        a = pa;
        b = pb;
    }
#elif defined(CUO_LANE_SIM)
    if (L.sim) {
        lanesim_scan_affine(L.sim, L.id, &a, &b);
    } else {
        a = 1;
        b = 0;
    }
#else
    (void)L;
    a = 1;
    b = 0;
#endif
}

// buf[i] = buf[i + shift] for i = 0 .. n-1 (the forward in-place copy that
// drops the oldest `shift` samples of a history buffer), split across the
// lanes.  Positions go in blocks of `shift`: block k reads only block k+1,
// which no lane writes before the barrier that ends block k, so the result is
// the serial copy's.
template <class T> DFN void lshift_copy(const Lanes &L, T *buf, int n, int shift)
{
    lsync(L);
    for (int b = 0; b < n; b += shift) {
        int e = b + shift < n ? b + shift : n;
        LFOR(L, i, b, e) buf[i] = buf[i + shift];
        lsync(L);
    }
}

// ------------------------------------------------------------------ basic ops

DFN int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
DFN int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
DFN int32_t wmul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }
DFN int32_t shl32(int32_t a, int s) { return (int32_t)((uint32_t)a << s); }
DFN int imin(int a, int b) { return a < b ? a : b; }
DFN int imax(int a, int b) { return a > b ? a : b; }
DFN int32_t min32(int32_t a, int32_t b) { return a < b ? a : b; }
DFN int32_t max32(int32_t a, int32_t b) { return a > b ? a : b; }

// number of significant bits; 0 for 0
DFN int ilog(uint32_t x)
{
#ifdef __CUDA_ARCH__
    return 32 - __clz((int)x);
#else
    return x ? 32 - __builtin_clz(x) : 0;
#endif
}

// ------------------------------------------------------------------ SILK ops

DFN int32_t s_smulwb(int32_t a, int32_t b) { return (int32_t)(((int64_t)a * (int16_t)b) >> 16); }
DFN int32_t s_smlawb(int32_t a, int32_t b, int32_t c) { return wadd(a, s_smulwb(b, c)); }
DFN int32_t s_smulwt(int32_t a, int32_t b) { return (int32_t)(((int64_t)a * (b >> 16)) >> 16); }
DFN int32_t s_smulbb(int32_t a, int32_t b) { return (int32_t)(int16_t)a * (int32_t)(int16_t)b; }
DFN int32_t s_smlabb(int32_t a, int32_t b, int32_t c) { return wadd(a, s_smulbb(b, c)); }
DFN int32_t s_smultt(int32_t a, int32_t b) { return (a >> 16) * (b >> 16); }
DFN int32_t s_smulww(int32_t a, int32_t b) { return (int32_t)(((int64_t)a * b) >> 16); }
DFN int32_t s_smlaww(int32_t a, int32_t b, int32_t c) { return wadd(a, s_smulww(b, c)); }
DFN int32_t s_smmul(int32_t a, int32_t b) { return (int32_t)(((int64_t)a * b) >> 32); }
DFN int64_t s_smull(int32_t a, int32_t b) { return (int64_t)a * b; }

DFN int32_t s_rshift_round(int32_t a, int s)
{
    return s == 1 ? (a >> 1) + (a & 1) : ((a >> (s - 1)) + 1) >> 1;
}
DFN int64_t s_rshift_round64(int64_t a, int s)
{
    return s == 1 ? (a >> 1) + (a & 1) : ((a >> (s - 1)) + 1) >> 1;
}
DFN int32_t s_sat16(int32_t a) { return a > 32767 ? 32767 : (a < -32768 ? -32768 : a); }
DFN int32_t s_limit(int32_t a, int32_t l1, int32_t l2)
{
    if (l1 > l2) return a > l1 ? l1 : (a < l2 ? l2 : a);
    return a > l2 ? l2 : (a < l1 ? l1 : a);
}
DFN int32_t s_add_sat32(int32_t a, int32_t b)
{
    int64_t s = (int64_t)a + b;
    return s > 2147483647LL ? 2147483647 : (s < -2147483648LL ? (int32_t)0x80000000 : (int32_t)s);
}
DFN int32_t s_sub_sat32(int32_t a, int32_t b)
{
    int64_t s = (int64_t)a - b;
    return s > 2147483647LL ? 2147483647 : (s < -2147483648LL ? (int32_t)0x80000000 : (int32_t)s);
}
DFN int32_t s_lshift_sat32(int32_t a, int s)
{
    return shl32(s_limit(a, (int32_t)0x80000000 >> s, 0x7FFFFFFF >> s), s);
}
DFN int32_t s_abs(int32_t a) { return a > 0 ? a : -a; }
DFN int32_t s_clz32(int32_t x) { return x ? 32 - ilog((uint32_t)x) : 32; }
DFN int32_t s_clz16(int16_t x) { return 32 - ilog(((uint32_t)(uint16_t)x << 16) | 0x8000u); }
DFN int32_t s_ror32(int32_t a, int rot)
{
    uint32_t x = (uint32_t)a, r = (uint32_t)rot, m = (uint32_t)-rot;
    if (rot == 0) return a;
    if (rot < 0) return (int32_t)((x << m) | (x >> (32 - m)));
    return (int32_t)((x << (32 - r)) | (x >> r));
}
DFN int32_t s_rand(int32_t seed) { return (int32_t)(907633515u + (uint32_t)seed * 196314165u); }

DFN void s_clz_frac(int32_t in, int32_t *lz, int32_t *frac_Q7)
{
    int32_t l = s_clz32(in);
    *lz = l;
    *frac_Q7 = s_ror32(in, 24 - l) & 0x7f;
}

// silk/Inlines.h silk_SQRT_APPROX
DFN int32_t s_sqrt_approx(int32_t x)
{
    int32_t y, lz, frac;
    if (x <= 0) return 0;
    s_clz_frac(x, &lz, &frac);
    y = (lz & 1) ? 32768 : 46214;
    y >>= (lz >> 1);
    return s_smlawb(y, y, s_smulbb(213, frac));
}

// silk/Inlines.h silk_DIV32_varQ
DFN int32_t s_div32_varq(int32_t a32, int32_t b32, int Qres)
{
    int a_h = s_clz32(s_abs(a32)) - 1;
    int32_t a_n = shl32(a32, a_h);
    int b_h = s_clz32(s_abs(b32)) - 1;
    int32_t b_n = shl32(b32, b_h);
    int32_t b_inv = (0x7FFFFFFF >> 2) / (b_n >> 16);
    int32_t result = s_smulwb(a_n, b_inv);
    a_n = wsub(a_n, shl32(s_smmul(b_n, result), 3));
    result = s_smlawb(result, a_n, b_inv);
    int ls = 29 + a_h - b_h - Qres;
    if (ls < 0) return s_lshift_sat32(result, -ls);
    return ls < 32 ? (result >> ls) : 0;
}

// silk/Inlines.h silk_INVERSE32_varQ
DFN int32_t s_inverse32_varq(int32_t b32, int Qres)
{
    int b_h = s_clz32(s_abs(b32)) - 1;
    int32_t b_n = shl32(b32, b_h);
    int32_t b_inv = (0x7FFFFFFF >> 2) / (b_n >> 16);
    int32_t result = shl32(b_inv, 16);
    int32_t err = shl32((1 << 29) - s_smulwb(b_n, b_inv), 3);
    result = s_smlaww(result, err, b_inv);
    int ls = 61 - b_h - Qres;
    if (ls <= 0) return s_lshift_sat32(result, -ls);
    return ls < 32 ? (result >> ls) : 0;
}

// silk/log2lin.c
DFN int32_t s_log2lin(int32_t inLog_Q7)
{
    if (inLog_Q7 < 0) return 0;
    if (inLog_Q7 >= 3967) return 0x7FFFFFFF;
    int32_t out = shl32(1, inLog_Q7 >> 7);
    int32_t frac = inLog_Q7 & 0x7F;
    int32_t poly = s_smlawb(frac, s_smulbb(frac, 128 - frac), -174);
    if (inLog_Q7 < 2048)
        return wadd(out, wmul(out, poly) >> 7);
    return wadd(out, wmul(out >> 7, poly));
}

// silk/lin2log.c
DFN int32_t s_lin2log(int32_t inLin)
{
    int32_t lz, frac;
    s_clz_frac(inLin, &lz, &frac);
    return wadd(s_smlawb(frac, wmul(frac, 128 - frac), 179), shl32(31 - lz, 7));
}

// ------------------------------------------------------------------ CELT ops

DFN int32_t c_mul16(int32_t a, int32_t b) { return (int32_t)(int16_t)a * (int32_t)(int16_t)b; }
DFN int32_t c_mac16(int32_t c, int32_t a, int32_t b) { return wadd(c, c_mul16(a, b)); }
DFN int32_t c_mul16_q15(int32_t a, int32_t b) { return c_mul16(a, b) >> 15; }
DFN int32_t c_mul16_q14(int32_t a, int32_t b) { return c_mul16(a, b) >> 14; }
DFN int32_t c_mul16_p15(int32_t a, int32_t b) { return (16384 + c_mul16(a, b)) >> 15; }
DFN int32_t c_mul16_32_q15(int32_t a, int32_t b) { return (int32_t)(((int64_t)(int16_t)a * b) >> 15); }
DFN int32_t c_mul16_32_q16(int32_t a, int32_t b) { return (int32_t)(((int64_t)(int16_t)a * b) >> 16); }
DFN int32_t c_mul16_32_p16(int32_t a, int32_t b)
{
    return (int32_t)(((int64_t)(int16_t)a * b + 32768) >> 16);
}
DFN int32_t c_mul32_q31(int32_t a, int32_t b) { return (int32_t)(((int64_t)a * b) >> 31); }
DFN int32_t c_mul32_q16(int32_t a, int32_t b) { return (int32_t)(((int64_t)a * b) >> 16); }
DFN int32_t c_pshr(int32_t a, int s) { return wadd(a, (1 << s) >> 1) >> s; }
DFN int32_t c_vshr(int32_t a, int s) { return s > 0 ? a >> s : shl32(a, -s); }
DFN int32_t c_sat(int32_t x, int32_t a) { return x > a ? a : (x < -a ? -a : x); }
DFN int16_t c_sat16(int32_t x) { return (int16_t)(x > 32767 ? 32767 : (x < -32768 ? -32768 : x)); }
DFN int16_t c_sround16(int32_t x, int a) { return (int16_t)c_sat(c_pshr(x, a), 32767); }
DFN int32_t c_frac_mul16(int32_t a, int32_t b) { return (16384 + (int32_t)(int16_t)a * (int16_t)b) >> 15; }
DFN int c_ilog2(int32_t x) { return ilog((uint32_t)x) - 1; }
DFN int c_zlog2(int32_t x) { return x <= 0 ? 0 : c_ilog2(x); }

// celt/fixed_generic.h SIG2WORD16 (SIG_SHIFT 12)
DFN int16_t c_sig2word16(int32_t x)
{
    x = c_pshr(x, 12);
    x = x < -32768 ? -32768 : x;
    x = x > 32767 ? 32767 : x;
    return (int16_t)x;
}

// celt/mathops.h celt_maxabs16 / celt_maxabs32 (scalar)
DFN int32_t c_maxabs16(const int16_t *x, int len)
{
    int16_t mx = 0, mn = 0;
    for (int i = 0; i < len; i++) { mx = x[i] > mx ? x[i] : mx; mn = x[i] < mn ? x[i] : mn; }
    return max32(mx, -(int32_t)mn);
}
DFN int32_t c_maxabs32(const int32_t *x, int len)
{
    int32_t mx = 0, mn = 0;
    for (int i = 0; i < len; i++) { mx = max32(mx, x[i]); mn = min32(mn, x[i]); }
    return max32(mx, -mn);
}

// celt/mathops.c isqrt32 (bit-by-bit integer square root)
DFN unsigned c_isqrt32(uint32_t val)
{
    unsigned g = 0;
    int bshift = (ilog(val) - 1) >> 1;
    unsigned b = 1u << bshift;
    do {
        uint32_t t = (((uint32_t)g << 1) + b) << bshift;
        if (t <= val) { g += b; val -= t; }
        b >>= 1;
        bshift--;
    } while (bshift >= 0);
    return g;
}

// celt/mathops.c celt_rcp: Q15 reciprocal with two Newton steps
DFN int32_t c_rcp(int32_t x)
{
    int i = c_ilog2(x);
    int16_t n = (int16_t)(c_vshr(x, i - 15) - 32768);
    int16_t r = (int16_t)(30840 + c_mul16_q15(-15420, n));
    r = (int16_t)(r - c_mul16_q15(r, (int16_t)(c_mul16_q15(r, n) + (int16_t)(r - 32768))));
    r = (int16_t)(r - (int16_t)(1 + c_mul16_q15(r, (int16_t)(c_mul16_q15(r, n) + (int16_t)(r - 32768)))));
    return c_vshr((int32_t)r, i - 16);
}

// celt/mathops.c frac_div32
DFN int32_t c_frac_div32(int32_t a, int32_t b)
{
    int shift = c_ilog2(b) - 29;
    a = c_vshr(a, shift);
    b = c_vshr(b, shift);
    int16_t rcp = (int16_t)c_pshr(c_rcp((int16_t)c_pshr(b, 16)), 3);
    int32_t result = c_mul16_32_q15(rcp, a);
    int32_t rem = wsub(c_pshr(a, 2), c_mul32_q31(result, b));
    result = wadd(result, shl32(c_mul16_32_q15(rcp, rem), 2));
    if (result >= 536870912) return 2147483647;
    if (result <= -536870912) return -2147483647;
    return shl32(result, 2);
}

// celt/mathops.c celt_rsqrt_norm
DFN int16_t c_rsqrt_norm(int32_t x)
{
    int16_t n = (int16_t)(x - 32768);
    int16_t r = (int16_t)(23557 + c_mul16_q15(n, (int16_t)(-13490 + c_mul16_q15(n, 6713))));
    int16_t r2 = (int16_t)c_mul16_q15(r, r);
    int16_t y = (int16_t)((uint16_t)(int16_t)((int16_t)(c_mul16_q15(r2, n) + r2) - 16384) << 1);
    return (int16_t)(r + c_mul16_q15(r, (int16_t)c_mul16_q15(y, (int16_t)(c_mul16_q15(y, 12288) - 16384))));
}

// celt/mathops.c celt_sqrt
DFN int32_t c_sqrt(int32_t x)
{
    if (x == 0) return 0;
    if (x >= 1073741824) return 32767;
    int k = (c_ilog2(x) >> 1) - 7;
    x = c_vshr(x, 2 * k);
    int16_t n = (int16_t)(x - 32768);
    int16_t rt = (int16_t)(23175 + c_mul16_q15(n, (int16_t)(11561 + c_mul16_q15(n,
        (int16_t)(-3011 + c_mul16_q15(n, (int16_t)(1699 + c_mul16_q15(n, -664))))))));
    return c_vshr((int32_t)rt, 7 - k);
}

// celt/mathops.c _celt_cos_pi_2 / celt_cos_norm
DFN int16_t c_cos_pi_2(int16_t x)
{
    int16_t x2 = (int16_t)c_mul16_p15(x, x);
    int32_t in = wadd((int16_t)(32767 - x2), c_mul16_p15(x2, wadd(-7651,
                   c_mul16_p15(x2, wadd(8277, c_mul16_p15(-626, x2))))));
    return (int16_t)(1 + (int16_t)(in < 32766 ? in : 32766));
}
DFN int16_t c_cos_norm(int32_t x)
{
    x = x & 0x0001ffff;
    if (x > (1 << 16)) x = (1 << 17) - x;
    if (x & 0x00007fff) {
        if (x < (1 << 15)) return c_cos_pi_2((int16_t)x);
        return (int16_t)-c_cos_pi_2((int16_t)(65536 - x));
    }
    if (x & 0x0000ffff) return 0;
    if (x & 0x0001ffff) return -32767;
    return 32767;
}

// celt/mathops.h celt_exp2_frac / celt_exp2 (DB_SHIFT 10)
DFN int32_t c_exp2_frac(int16_t x)
{
    int16_t frac = (int16_t)((uint16_t)x << 4);
    return (int16_t)(16383 + c_mul16_q15(frac, (int16_t)(22804 + c_mul16_q15(frac,
            (int16_t)(14819 + c_mul16_q15(10204, frac))))));
}
DFN int32_t c_exp2(int16_t x)
{
    int integer = x >> 10;
    if (integer > 14) return 0x7f000000;
    if (integer < -15) return 0;
    int16_t frac = (int16_t)c_exp2_frac((int16_t)(x - (int16_t)((uint16_t)integer << 10)));
    return c_vshr((int32_t)frac, -integer - 2);
}

// celt/bands.c celt_lcg_rand
DFN uint32_t c_lcg_rand(uint32_t seed) { return 1664525u * seed + 1013904223u; }

} // namespace cuo
