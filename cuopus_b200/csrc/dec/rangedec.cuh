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
#pragma once
#include "common.cuh"

namespace cuo {

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
};

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
#elif defined(CUO_LANE_SIM)
    if (L.sim) lanesim_bcast(L.sim, L.id, d, (int)sizeof *d);
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

DNI void rd_init(RangeDec *d, const uint8_t *buf, uint32_t storage)
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
    rd_normalize(d);
}

DNI unsigned rd_decode(RangeDec *d, unsigned ft)
{
    d->ext = d->rng / ft;
    unsigned s = d->val / d->ext;
    return ft - (s + 1 < ft ? s + 1 : ft);
}

DNI unsigned rd_decode_bin(RangeDec *d, unsigned bits)
{
    d->ext = d->rng >> bits;
    unsigned s = d->val / d->ext;
    unsigned t = 1u << bits;
    return t - (s + 1u < t ? s + 1u : t);
}

DNI void rd_update(RangeDec *d, unsigned fl, unsigned fh, unsigned ft)
{
    uint32_t s = d->ext * (ft - fh);
    d->val -= s;
    d->rng = fl > 0 ? d->ext * (fh - fl) : d->rng - s;
    rd_normalize(d);
}

DNI int rd_bit_logp(RangeDec *d, unsigned logp)
{
    uint32_t r = d->rng, v = d->val;
    uint32_t s = r >> logp;
    int ret = v < s;
    if (!ret) d->val = v - s;
    d->rng = ret ? s : r - s;
    rd_normalize(d);
    return ret;
}

DNI int rd_icdf(RangeDec *d, const uint8_t *icdf, unsigned ftb)
{
    uint32_t s = d->rng, v = d->val, r = s >> ftb, t;
    int ret = -1;
    do {
        t = s;
        s = r * icdf[++ret];
    } while (v < s);
    d->val = v - s;
    d->rng = t - s;
    rd_normalize(d);
    return ret;
}

DNI uint32_t rd_bits(RangeDec *d, unsigned bits)
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

DNI uint32_t rd_uint(RangeDec *d, uint32_t ft)
{
    ft--;
    int ftb = ilog(ft);
    if (ftb > 8) {
        ftb -= 8;
        unsigned f = (unsigned)(ft >> ftb) + 1;
        unsigned s = rd_decode(d, f);
        rd_update(d, s, s + 1, f);
        uint32_t t = (uint32_t)s << ftb | rd_bits(d, ftb);
        if (t <= ft) return t;
        d->error = 1;
        return ft;
    }
    ft++;
    unsigned s = rd_decode(d, (unsigned)ft);
    rd_update(d, s, s + 1, (unsigned)ft);
    return s;
}

DFN int rd_tell(const RangeDec *d) { return d->nbits_total - ilog(d->rng); }

// correction thresholds of celt/entcode.c ec_tell_frac
TABC(unsigned, T_tell_frac_corr[8]) = {35733, 38967, 42495, 46340, 50535, 55109, 60097, 65535};

DFN uint32_t rd_tell_frac(const RangeDec *d)
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

// celt/laplace.c ec_laplace_decode (LAPLACE_MINP 1, LAPLACE_NMIN 16)
DNI int rd_laplace(RangeDec *d, unsigned fs, int decay)
{
    int val = 0;
    unsigned fl = 0;
    unsigned fm = rd_decode_bin(d, 15);
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
    rd_update(d, fl, (fl + fs) < 32768u ? fl + fs : 32768u, 32768);
    return val;
}

} // namespace cuo
