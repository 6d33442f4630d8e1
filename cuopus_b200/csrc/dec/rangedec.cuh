// Range decoder of RFC 6716 section 4.1: 32-bit range/value normalised byte by
// byte from the front of the frame, raw bits read from the back.  Restates
// celt/entdec.c (ec_dec_init, ec_decode, ec_decode_bin, ec_dec_update,
// ec_dec_bit_logp, ec_dec_icdf, ec_dec_icdf16, ec_dec_uint, ec_dec_bits),
// celt/entcode.c ec_tell_frac, celt/entcode.h ec_tell and celt/laplace.c
// ec_laplace_decode of libopus 1.5.2.
//
// The decoder state lives in registers of every lane of the chain's group
// (all lanes decode the same symbols).  `buf` points at the frame bytes; the
// chain kernel stages those into shared memory when it can.
//
// Symbol log (two-phase decoding).  What the range decoder hands the decoder
// -- every symbol, raw bit field, uniform integer, Laplace value, tell and
// final range -- depends on the packet's bytes and on decisions taken from
// earlier such values of the same packet, never on decoder state carried
// from earlier packets: SILK codes frames conditionally only inside a packet,
// CELT's energy prediction, folding and noise seed act on the reconstruction
// only, and the Opus layer's mode and bandwidth come from the TOC.  So a
// packet can be decoded once on its own from a fresh decoder, recording those
// values in order (SYM_RECORD), and decoded again inside its chain with the
// range decoder replaying them (SYM_REPLAY) instead of decoding: the same
// values in the same order, without the range coder's arithmetic on the
// chain's serial path.  The one range decode that depends on earlier packets
// -- the constant silence frame CELT decodes when hybrid switches to SILK --
// is not logged.  Every lane keeps its own cursor (rd_bcast carries the first
// lane's after a lead stretch), as it keeps its own decoder state.
#pragma once
#include "common.cuh"

namespace cuo {

enum { SYM_OFF = 0, SYM_RECORD = 1, SYM_REPLAY = 2 };

struct SymLog {
    uint32_t *base;   // this packet's entries
    uint32_t pos;     // next entry
    uint32_t cap;     // entries available; a record beyond it sets overflow
    int mode;
    int overflow;     // recording: an entry did not fit; replaying: out of step
};

// Symbol-log tables of a batch (null: decode normally): per packet p, entries
// base + off[p] .. base + off[p + 1]; len[p] = entries recorded, or
// SYM_BAD when the packet's record is unusable (overflow, decode error), in
// which case the chain decodes that packet normally.
struct SymArgs {
    uint32_t *base;
    const uint64_t *off;
    uint32_t *len;
    int mode;
};
constexpr uint32_t SYM_BAD = 0xFFFFFFFFu;

struct RangeDec {
    const uint8_t *buf;
    uint32_t storage;
    uint32_t end_offs;
    uint32_t end_window;
    int nend_bits;
    int nbits_total;
    uint32_t offs;
    uint32_t rng;
    uint32_t val;
    uint32_t ext;
    int rem;
    int error;
    SymLog *lg;   // this lane's symbol log of the packet, or null
};

DFN bool sym_replay(const RangeDec *d) { return d->lg && d->lg->mode == SYM_REPLAY; }
// The next replayed value, which must be below `limit` (0: any value).  A
// value out of range, or a log read past its end, means the replay is out of
// step with the decoder: the log is marked so and this and every later call
// return 0, a value every primitive can return -- the decode goes on over
// valid (wrong) values and never reads or writes out of bounds.
DFN uint32_t sym_pop(const RangeDec *d, uint32_t limit = 0)
{
    SymLog *g = d->lg;
    if (g->overflow) return 0u;
    uint32_t v = 0u;
    if (g->pos < g->cap) v = g->base[g->pos];
    else g->overflow = 1;
    g->pos++;
    if (limit && v >= limit) {
        g->overflow = 1;
        v = 0u;
    }
    return g->overflow ? 0u : v;
}
// v, recorded when the log records
DFN uint32_t sym_note(const RangeDec *d, uint32_t v)
{
    SymLog *g = d->lg;
    if (g && g->mode == SYM_RECORD) {
        if (g->pos < g->cap) g->base[g->pos] = v;
        else g->overflow = 1;
        g->pos++;
    }
    return v;
}

// The first lane's decoder state on every lane of the group, after a lead
// stretch (common.cuh) decoded symbols on the first lane only.  buf and
// storage are the same on every lane already.
DFN void rd_bcast(const Lanes &L, RangeDec *d)
{
#ifdef __CUDA_ARCH__
    if (L.n == 1) return;
    const int src = (int)(threadIdx.x & 31) - L.id;
    d->end_offs = __shfl_sync(L.mask, d->end_offs, src);
    d->end_window = __shfl_sync(L.mask, d->end_window, src);
    d->nend_bits = __shfl_sync(L.mask, d->nend_bits, src);
    d->nbits_total = __shfl_sync(L.mask, d->nbits_total, src);
    d->offs = __shfl_sync(L.mask, d->offs, src);
    d->rng = __shfl_sync(L.mask, d->rng, src);
    d->val = __shfl_sync(L.mask, d->val, src);
    d->ext = __shfl_sync(L.mask, d->ext, src);
    d->rem = __shfl_sync(L.mask, d->rem, src);
    d->error = __shfl_sync(L.mask, d->error, src);
    if (d->lg) {
        d->lg->pos = __shfl_sync(L.mask, d->lg->pos, src);
        d->lg->overflow = __shfl_sync(L.mask, d->lg->overflow, src);
    }
#elif defined(CUO_LANE_SIM)
    if (L.sim) {
        SymLog *own = d->lg;   // every lane keeps its own log cursor
        lanesim_bcast(L.sim, L.id, d, (int)sizeof *d);
        d->lg = own;
        if (own) lanesim_bcast(L.sim, L.id, own, (int)sizeof *own);
    }
#else
    (void)L;
    (void)d;
#endif
}

// A lead stretch that decodes symbols: the body runs on the first lane, then
// every lane continues from that lane's decoder state.
template <class F> DFN void lead_rd(const Lanes &L, RangeDec *rd, F &&body)
{
    lead(L, body);
    rd_bcast(L, rd);
}

DFN int rd_read_byte(RangeDec *d) { return d->offs < d->storage ? d->buf[d->offs++] : 0; }
DFN int rd_read_byte_end(RangeDec *d)
{
    return d->end_offs < d->storage ? d->buf[d->storage - ++(d->end_offs)] : 0;
}

DFN void rd_normalize(RangeDec *d)
{
    while (d->rng <= (1u << 23)) {
        d->nbits_total += 8;
        d->rng <<= 8;
        int sym = d->rem;
        d->rem = rd_read_byte(d);
        sym = (sym << 8 | d->rem) >> 1;
        d->val = ((d->val << 8) + (255u & ~(uint32_t)sym)) & 0x7FFFFFFFu;
    }
}

DNI void rd_init(RangeDec *d, const uint8_t *buf, uint32_t storage, SymLog *lg = nullptr)
{
    d->buf = buf;
    d->storage = storage;
    d->end_offs = 0;
    d->end_window = 0;
    d->nend_bits = 0;
    d->nbits_total = 33 - 24;   // EC_CODE_BITS+1 - ((EC_CODE_BITS-EC_CODE_EXTRA)/8)*8
    d->offs = 0;
    d->rng = 1u << 7;
    d->rem = rd_read_byte(d);
    d->val = d->rng - 1 - (d->rem >> 1);
    d->error = 0;
    d->lg = lg;
    rd_normalize(d);
}

// The range coder's arithmetic (rdr_*: never logged; the composite decodes
// below are built from these) ...
DFN unsigned rdr_decode(RangeDec *d, unsigned ft)
{
    d->ext = d->rng / ft;
    unsigned s = d->val / d->ext;
    return ft - (s + 1 < ft ? s + 1 : ft);
}

DFN unsigned rdr_decode_bin(RangeDec *d, unsigned bits)
{
    d->ext = d->rng >> bits;
    unsigned s = d->val / d->ext;
    unsigned t = 1u << bits;
    return t - (s + 1u < t ? s + 1u : t);
}

DFN void rdr_update(RangeDec *d, unsigned fl, unsigned fh, unsigned ft)
{
    uint32_t s = d->ext * (ft - fh);
    d->val -= s;
    d->rng = fl > 0 ? d->ext * (fh - fl) : d->rng - s;
    rd_normalize(d);
}

DFN uint32_t rdr_bits(RangeDec *d, unsigned bits)
{
    uint32_t window = d->end_window;
    int available = d->nend_bits;
    if ((unsigned)available < bits) {
        do {
            window |= (uint32_t)rd_read_byte_end(d) << available;
            available += 8;
        } while (available <= 32 - 8);
    }
    uint32_t ret = window & ((1u << bits) - 1u);
    window >>= bits;
    available -= bits;
    d->end_window = window;
    d->nend_bits = available;
    d->nbits_total += bits;
    return ret;
}

// ... and the calls the decoder makes (rd_*): each value the decoder receives
// is replayed from the packet's symbol log, or recorded into it, when the
// packet has one.
DNI unsigned rd_decode(RangeDec *d, unsigned ft)
{
    if (sym_replay(d)) return sym_pop(d, ft);
    return sym_note(d, rdr_decode(d, ft));
}

DNI unsigned rd_decode_bin(RangeDec *d, unsigned bits)
{
    if (sym_replay(d)) return sym_pop(d, 1u << bits);
    return sym_note(d, rdr_decode_bin(d, bits));
}

// follows rd_decode: nothing to do when that value was replayed
DNI void rd_update(RangeDec *d, unsigned fl, unsigned fh, unsigned ft)
{
    if (sym_replay(d)) return;
    rdr_update(d, fl, fh, ft);
}

DNI int rd_bit_logp(RangeDec *d, unsigned logp)
{
    if (sym_replay(d)) return (int)sym_pop(d, 2u);
    uint32_t r = d->rng, v = d->val;
    uint32_t s = r >> logp;
    int ret = v < s;
    if (!ret) d->val = v - s;
    d->rng = ret ? s : r - s;
    rd_normalize(d);
    return (int)sym_note(d, (uint32_t)ret);
}

DNI int rd_icdf(RangeDec *d, const uint8_t *icdf, unsigned ftb)
{
    if (sym_replay(d)) {
        // a symbol of this table: no terminating zero before it
        uint32_t v = sym_pop(d, 256u);
        for (uint32_t i = 0; i < v; i++)
            if (icdf[i] == 0) {
                d->lg->overflow = 1;
                return 0;
            }
        return (int)v;
    }
    uint32_t s = d->rng, v = d->val, r = s >> ftb, t;
    int ret = -1;
    do {
        t = s;
        s = r * icdf[++ret];
    } while (v < s);
    d->val = v - s;
    d->rng = t - s;
    rd_normalize(d);
    return (int)sym_note(d, (uint32_t)ret);
}

DNI uint32_t rd_bits(RangeDec *d, unsigned bits)
{
    if (sym_replay(d)) return bits >= 32 ? sym_pop(d) : sym_pop(d, 1u << bits);
    return sym_note(d, rdr_bits(d, bits));
}

DNI uint32_t rd_uint(RangeDec *d, uint32_t ft)
{
    if (sym_replay(d)) return sym_pop(d, ft);
    uint32_t v;
    ft--;
    int ftb = ilog(ft);
    if (ftb > 8) {
        ftb -= 8;
        unsigned f = (unsigned)(ft >> ftb) + 1;
        unsigned s = rdr_decode(d, f);
        rdr_update(d, s, s + 1, f);
        uint32_t t = (uint32_t)s << ftb | rdr_bits(d, ftb);
        if (t <= ft) {
            v = t;
        } else {
            d->error = 1;
            v = ft;
        }
    } else {
        ft++;
        unsigned s = rdr_decode(d, (unsigned)ft);
        rdr_update(d, s, s + 1, (unsigned)ft);
        v = s;
    }
    return sym_note(d, v);
}

// Replayed tells are bounded by the frame's bits plus 64 (callers size frames
// and budgets from them); a recorded tell beyond that marks the packet's log
// unusable, so the bound never changes a decode.
DFN uint32_t rd_tell_bound(const RangeDec *d) { return 8u * d->storage + 64u; }
DNI int rd_tell_logged(const RangeDec *d)
{
    if (sym_replay(d)) return (int)sym_pop(d, rd_tell_bound(d) + 1u);
    int t = d->nbits_total - ilog(d->rng);
    if (d->lg->mode == SYM_RECORD && (t < 0 || (uint32_t)t > rd_tell_bound(d))) d->lg->overflow = 1;
    return (int)sym_note(d, (uint32_t)t);
}
DFN int rd_tell(const RangeDec *d)
{
    if (d->lg) return rd_tell_logged(d);
    return d->nbits_total - ilog(d->rng);
}

// correction thresholds of celt/entcode.c ec_tell_frac
TABC(unsigned, T_tell_frac_corr[8]) = {35733, 38967, 42495, 46340, 50535, 55109, 60097, 65535};

DFN uint32_t rdr_tell_frac(const RangeDec *d)
{
    // 1/8-bit resolution: a linear estimate corrected against fixed thresholds
    const unsigned *corr = T_tell_frac_corr;
    uint32_t nbits = (uint32_t)d->nbits_total << 3;
    int l = ilog(d->rng);
    uint32_t r = d->rng >> (l - 16);
    unsigned b = (r >> 12) - 8;
    b += r > corr[b];
    l = (l << 3) + b;
    return nbits - l;
}
DNI uint32_t rd_tell_frac_logged(const RangeDec *d)
{
    if (sym_replay(d)) return sym_pop(d, 8u * rd_tell_bound(d) + 1u);
    uint32_t t = rdr_tell_frac(d);
    if (d->lg->mode == SYM_RECORD && t > 8u * rd_tell_bound(d)) d->lg->overflow = 1;
    return sym_note(d, t);
}
DFN uint32_t rd_tell_frac(const RangeDec *d)
{
    if (d->lg) return rd_tell_frac_logged(d);
    return rdr_tell_frac(d);
}

// The final range (OPUS_GET_FINAL_RANGE, the CELT noise seed) and the error
// flag, as the decoder reads them at the end of a frame.
DNI uint32_t rd_final_logged(const RangeDec *d)
{
    if (sym_replay(d)) return sym_pop(d);
    return sym_note(d, d->rng);
}
DFN uint32_t rd_final(const RangeDec *d)
{
    if (d->lg) return rd_final_logged(d);
    return d->rng;
}
DNI int rd_err_logged(const RangeDec *d)
{
    if (sym_replay(d)) return (int)sym_pop(d);
    return (int)sym_note(d, (uint32_t)d->error);
}
DFN int rd_err(const RangeDec *d)
{
    if (d->lg) return rd_err_logged(d);
    return d->error;
}

// celt/laplace.c ec_laplace_decode (LAPLACE_MINP 1, LAPLACE_NMIN 16)
DNI int rd_laplace(RangeDec *d, unsigned fs, int decay)
{
    if (sym_replay(d)) return (int)sym_pop(d);
    int val = 0;
    unsigned fl = 0;
    unsigned fm = rdr_decode_bin(d, 15);
    if (fm >= fs) {
        val++;
        fl = fs;
        fs = ((32768u - 32u - fs) * (int32_t)(16384 - decay) >> 15) + 1;
        while (fs > 1 && fm >= fl + 2 * fs) {
            fs *= 2;
            fl += fs;
            fs = ((fs - 2) * (int32_t)decay) >> 15;
            fs += 1;
            val++;
        }
        if (fs <= 1) {
            int di = (fm - fl) >> 1;
            val += di;
            fl += 2 * di;
        }
        if (fm < fl + fs) val = -val;
        else fl += fs;
    }
    rdr_update(d, fl, (fl + fs) < 32768u ? fl + fs : 32768u, 32768);
    return (int)sym_note(d, (uint32_t)val);
}

} // namespace cuo
