// Additive per-chain cost of the file entry points' visiting order
// (ordercost.cpp): features of a packet, the fitted weights per lane width.
#pragma once
#include <stdint.h>

namespace cuo_host {

// Adds one packet's features (all but the chain constant, index 0) to f.
void packet_order_features(const uint8_t *p, uint32_t len, int out_channels, double *f);

// The weights folded per packet: the frame features are linear in the frame
// count, so a packet costs packet + per_byte * len + frames * frame[cfg][s][stereo out].
struct OrderCost {
    double chain, packet, per_byte, empty;
    double frame[32][2][2];
    explicit OrderCost(const double *w);
    double of(const uint8_t *p, uint32_t len, int out_channels) const
    {
        if (!len) return packet + empty;
        int toc = p[0], code = toc & 3;
        int nf = code == 0 ? 1 : code < 3 ? 2 : (len > 1 ? (p[1] & 63) : 0);
        return packet + per_byte * len + nf * frame[toc >> 3][(toc >> 2) & 1][out_channels == 2];
    }
};
// Weights for chains decoded by groups of `width` lanes (8 and below, or 32).
const double *order_coefficients(int width);
// False while the weights are the unfitted default (cost = decoded duration).
bool order_model_fitted();

} // namespace cuo_host
