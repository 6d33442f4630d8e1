// Visiting order of the file entry points: an additive cost per chain.
//
// The file entry points pull chains from a device queue in a host-given
// order, longest first (list scheduling).  When the chains of a call are few
// per decoder group (the 2 h file in 1 s chains: 7,200 chains on 4,736 groups
// of 8 lanes), the makespan depends on which chains go first, and a chain's
// sample count does not tell them apart: a second of hybrid costs more than a
// second of SILK.  The cost of a chain is modelled as the sum of its packets'
// costs (plus a constant), each packet a non-negative combination of the
// features below, so chain costs are prefix-sum differences.  The weights are
// fitted by non-negative least squares to per-chain device times measured on
// a training corpus (cuopus_b200/fit_order_cost.py writes ordercost_coef.inc);
// they change no decoded sample, only the order in which chains start.
//
// Features of one packet (TOC of RFC 6716 section 3.1):
//   0  chain constant (1 per chain, not per packet)
//   1  packets
//   2  packet bytes / 100
//   3 + 2 * class + s   frames of each (mode, frame duration) class, s = the
//                       TOC stereo bit; classes: SILK 10/20/40/60 ms (0-3),
//                       hybrid 10/20 ms (4-5), CELT 2.5/5/10/20 ms (6-9)
//   23 SILK milliseconds x bandwidth (NB 0, MB 1, WB 2)
//   24 CELT milliseconds x bandwidth (NB 0, WB 1, SWB 2, FB 3)
//   25 milliseconds decoded to a stereo output
//   26 empty packets (concealment)
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/cuopus.h"
#include "ordercost.h"

namespace cuo_host {
namespace {

#include "ordercost_coef.inc"

static_assert(sizeof(kOrderCoef8) / sizeof(double) == CUOPUS_ORDER_FEATURES, "coefficients");
static_assert(sizeof(kOrderCoef32) / sizeof(double) == CUOPUS_ORDER_FEATURES, "coefficients");

// frame duration in quarter milliseconds per TOC configuration
const int kQms[32] = {40, 80, 160, 240, 40, 80, 160, 240, 40, 80, 160, 240, 40, 80, 40, 80,
                      10, 20, 40, 80, 10, 20, 40, 80, 10, 20, 40, 80, 10, 20, 40, 80};

} // namespace

void packet_order_features(const uint8_t *p, uint32_t len, int out_channels, double *f)
{
    f[1] += 1.0;
    f[2] += len / 100.0;
    if (!len) {
        f[26] += 1.0;
        return;
    }
    int toc = p[0], cfg = toc >> 3, code = toc & 3;
    int nf = code == 0 ? 1 : code < 3 ? 2 : (len > 1 ? (p[1] & 63) : 0);
    int s = (toc >> 2) & 1;
    int cls;
    if (cfg < 12) cls = cfg & 3;
    else if (cfg < 16) cls = 4 + (cfg & 1);
    else cls = 6 + (cfg & 3);
    double ms = nf * kQms[cfg] / 4.0;
    f[3 + 2 * cls + s] += nf;
    if (cfg < 12) f[23] += ms * (cfg >> 2);
    else if (cfg >= 16) f[24] += ms * ((cfg - 16) >> 2);
    if (out_channels == 2) f[25] += ms;
}

const double *order_coefficients(int width)
{
    return width >= 32 ? kOrderCoef32 : kOrderCoef8;
}

bool order_model_fitted()
{
    return CUO_ORDER_FITTED != 0;
}

OrderCost::OrderCost(const double *w)
{
    chain = w[0];
    packet = w[1];
    per_byte = w[2] / 100.0;
    empty = w[26];
    for (int cfg = 0; cfg < 32; cfg++)
        for (int s = 0; s < 2; s++)
            for (int so = 0; so < 2; so++) {
                // one frame of this configuration: its features are linear in the frame count
                uint8_t toc[2] = {(uint8_t)(cfg << 3 | s << 2), 0};
                double f[CUOPUS_ORDER_FEATURES];
                memset(f, 0, sizeof f);
                packet_order_features(toc, 1, so ? 2 : 1, f);
                double c = 0.0;
                for (int k = 3; k < 26; k++) c += w[k] * f[k];
                frame[cfg][s][so] = c;
            }
}

} // namespace cuo_host

extern "C" int cuopus_order_features(const uint8_t *blob, const uint64_t *off, const uint32_t *len,
                                     const uint32_t *first, const uint32_t *npkts, const uint8_t *channels,
                                     int32_t nchains, double *feat)
{
    if (nchains < 0 || (nchains > 0 && (!blob || !off || !len || !first || !npkts || !channels || !feat)))
        return 3;
    for (int32_t c = 0; c < nchains; c++) {
        double *f = feat + (size_t)c * CUOPUS_ORDER_FEATURES;
        memset(f, 0, CUOPUS_ORDER_FEATURES * sizeof(double));
        f[0] = 1.0;
        for (uint32_t k = 0; k < npkts[c]; k++) {
            uint64_t q = (uint64_t)first[c] + k;
            cuo_host::packet_order_features(blob + off[q], len[q], channels[c], f);
        }
    }
    return 0;
}

extern "C" int cuopus_order_costs(const uint8_t *blob, const uint64_t *off, const uint32_t *len,
                                  const uint32_t *first, const uint32_t *npkts, const uint8_t *channels,
                                  int32_t nchains, int32_t width, double *cost)
{
    if (nchains < 0 || (nchains > 0 && (!blob || !off || !len || !first || !npkts || !channels || !cost)))
        return 3;
    const cuo_host::OrderCost oc(cuo_host::order_coefficients(width));
    for (int32_t c = 0; c < nchains; c++) {
        double s = oc.chain;
        for (uint32_t k = 0; k < npkts[c]; k++) {
            uint64_t q = (uint64_t)first[c] + k;
            s += oc.of(blob + off[q], len[q], channels[c]);
        }
        cost[c] = s;
    }
    return 0;
}

extern "C" int cuopus_order_model_fitted(void)
{
    return cuo_host::order_model_fitted() ? 1 : 0;
}

extern "C" int cuopus_order_weights(int32_t width, double *w)
{
    if (!w) return 3;
    memcpy(w, cuo_host::order_coefficients(width), CUOPUS_ORDER_FEATURES * sizeof(double));
    return 0;
}
