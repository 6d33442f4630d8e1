// Opus layer of the chain decoder: packet framing and the per-frame mode logic
// of RFC 6716 (SILK / hybrid / CELT, mode transitions with a 5 ms concealed
// cross-fade, embedded CELT redundancy, the hybrid->SILK silence frame).
//
// Restates libopus 1.5.2 src/opus_decoder.c (opus_decoder_init,
// opus_decode_frame, opus_decode_native with decode_fec = 0, smooth_fade) and
// src/opus.c (opus_packet_parse_impl, opus_packet_get_samples_per_frame), for
// a decoder created at 48 kHz with decode_gain 0 and the int16 output of the
// FIXED_POINT build.
//
// opus_decode_frame calls itself for concealment (mode transitions and
// len <= 1 frames); that recursion is at most two deep and is unrolled here
// with a depth template parameter, so the device code uses no call stack
// recursion.
#pragma once
#include "silk.cuh"
#include "celt.cuh"

namespace cuo {

enum { MODE_SILK_ONLY = 1000, MODE_HYBRID = 1001, MODE_CELT_ONLY = 1002 };
enum { BW_NB = 1101, BW_MB = 1102, BW_WB = 1103, BW_SWB = 1104, BW_FB = 1105 };
enum { OPUS_OK = 0, OPUS_BAD_ARG = -1, OPUS_BUFFER_TOO_SMALL = -2, OPUS_INTERNAL_ERROR = -3,
       OPUS_INVALID_PACKET = -4 };
enum { MAX_PACKET_SAMPLES = 5760 };

struct OpusDec {
    int32_t channels;
    int32_t stream_channels, bandwidth, mode, prev_mode, frame_size, prev_redundancy, last_packet_duration;
    uint32_t rangeFinal;
    SilkDecControl DecControl;
    SilkDec silk;
    CeltDec celt;
};

struct OpusScratch {
    SilkScratch silk;
    CeltScratch celt;
    int16_t pcm_silk[2][480 * 2];       // per recursion depth, IMAX(F10, frame_size) * channels
    int16_t pcm_transition[240 * 2];
    int16_t redundant_audio[240 * 2];
    int16_t sizes[48];                  // frame sizes of the packet being decoded
};

DNI void opus_init(OpusDec *st, int channels)
{
    st->channels = channels;
    st->stream_channels = channels;
    st->bandwidth = 0;
    st->mode = 0;
    st->prev_mode = 0;
    st->frame_size = 48000 / 400;
    st->prev_redundancy = 0;
    st->last_packet_duration = 0;
    st->rangeFinal = 0;
    st->DecControl.nChannelsAPI = channels;
    st->DecControl.nChannelsInternal = 0;
    st->DecControl.API_sampleRate = 48000;
    st->DecControl.internalSampleRate = 0;
    st->DecControl.payloadSize_ms = 0;
    silk_init_dec(&st->silk);
    celt_init(&st->celt, channels);
}

DFN int toc_mode(uint8_t toc)
{
    if (toc & 0x80) return MODE_CELT_ONLY;
    if ((toc & 0x60) == 0x60) return MODE_HYBRID;
    return MODE_SILK_ONLY;
}
DFN int toc_bandwidth(uint8_t toc)
{
    if (toc & 0x80) {
        int bw = BW_MB + ((toc >> 5) & 0x3);
        return bw == BW_MB ? BW_NB : bw;
    }
    if ((toc & 0x60) == 0x60) return (toc & 0x10) ? BW_FB : BW_SWB;
    return BW_NB + ((toc >> 5) & 0x3);
}
DFN int toc_samples_per_frame(uint8_t toc)
{
    const int Fs = 48000;
    if (toc & 0x80) return (Fs << ((toc >> 3) & 0x3)) / 400;
    if ((toc & 0x60) == 0x60) return (toc & 0x08) ? Fs / 50 : Fs / 100;
    int a = (toc >> 3) & 0x3;
    return a == 3 ? Fs * 60 / 1000 : (Fs << a) / 100;
}

DFN int parse_size(const uint8_t *data, int32_t len, int16_t *size)
{
    if (len < 1) { *size = -1; return -1; }
    if (data[0] < 252) { *size = data[0]; return 1; }
    if (len < 2) { *size = -1; return -1; }
    *size = (int16_t)(4 * data[1] + data[0]);
    return 2;
}

// src/opus.c opus_packet_parse_impl (self_delimited = 0)
DNI int packet_parse(const uint8_t *data, int32_t len, int16_t *size, int *payload_offset)
{
    if (len < 0) return OPUS_BAD_ARG;
    if (len == 0) return OPUS_INVALID_PACKET;
    const uint8_t *data0 = data;
    int framesize = toc_samples_per_frame(data[0]);
    uint8_t toc = *data++;
    len--;
    int32_t last_size = len;
    int count, bytes;
    switch (toc & 0x3) {
    case 0:
        count = 1;
        break;
    case 1:
        count = 2;
        if (len & 0x1) return OPUS_INVALID_PACKET;
        last_size = len / 2;
        size[0] = (int16_t)last_size;
        break;
    case 2:
        count = 2;
        bytes = parse_size(data, len, size);
        len -= bytes;
        if (size[0] < 0 || size[0] > len) return OPUS_INVALID_PACKET;
        data += bytes;
        last_size = len - size[0];
        break;
    default: {
        if (len < 1) return OPUS_INVALID_PACKET;
        uint8_t ch = *data++;
        count = ch & 0x3F;
        if (count <= 0 || framesize * (int32_t)count > 5760) return OPUS_INVALID_PACKET;
        len--;
        if (ch & 0x40) {
            int p;
            do {
                if (len <= 0) return OPUS_INVALID_PACKET;
                p = *data++;
                len--;
                int tmp = p == 255 ? 254 : p;
                len -= tmp;
            } while (p == 255);
        }
        if (len < 0) return OPUS_INVALID_PACKET;
        int cbr = !(ch & 0x80);
        if (!cbr) {
            last_size = len;
            for (int i = 0; i < count - 1; i++) {
                bytes = parse_size(data, len, size + i);
                len -= bytes;
                if (size[i] < 0 || size[i] > len) return OPUS_INVALID_PACKET;
                data += bytes;
                last_size -= bytes + size[i];
            }
            if (last_size < 0) return OPUS_INVALID_PACKET;
        } else {
            last_size = len / count;
            if (last_size * count != len) return OPUS_INVALID_PACKET;
            for (int i = 0; i < count - 1; i++) size[i] = (int16_t)last_size;
        }
        break;
    }
    }
    if (last_size > 1275) return OPUS_INVALID_PACKET;
    size[count - 1] = (int16_t)last_size;
    *payload_offset = (int)(data - data0);
    return count;
}

#ifdef CUO_FRAME_EVENTS
// Defined by a test build: called once per decoded frame with the recursion
// depth, the frame's mode, the previous mode, the redundancy flags, the
// transition flag (5 ms concealment crossfade) and the hybrid -> SILK silence
// frame flag.
void cuo_frame_event(int depth, int mode, int prev_mode, int redundancy, int celt_to_silk, int transition,
                     int silence_frame);
#endif

// src/opus_decoder.c smooth_fade (Fs 48 kHz: window increment 1)
DNI void smooth_fade(Lanes L, const int16_t *in1, const int16_t *in2, int16_t *out, int overlap, int channels)
{
    lsync(L);
    LFOR(L, q, 0, overlap * channels) {
        int i = q / channels, c = q - i * channels;
        int16_t wv = (int16_t)c_mul16_q15(T_celt_window[i], T_celt_window[i]);
        int16_t a = in1[i * channels + c], b = in2[i * channels + c];
        out[i * channels + c] = (int16_t)(c_mac16(c_mul16(wv, b), 32767 - wv, a) >> 15);
    }
    lsync(L);
}

// src/opus_decoder.c opus_decode_frame (:237-668).  D is the recursion depth;
// fec = 1 decodes the SILK layer's in-band FEC (LBRR) frames of `data` and
// conceals the CELT layer.
template <int D>
DNI int opus_frame(Lanes L, OpusDec *st, const uint8_t *data, int32_t len, int16_t *pcm, int frame_size,
                   OpusScratch *w, int fec)
{
    const int F20 = 960, F10 = 480, F5 = 240, F2_5 = 120;
    const int C = st->channels;
    RangeDec dec;
    int silk_ret = 0, celt_ret = 0;
    int audiosize, mode, bandwidth;
    int transition = 0, redundancy = 0, redundancy_bytes = 0, celt_to_silk = 0;
    uint32_t redundant_rng = 0;
    int16_t *pcm_transition = 0;
    if (frame_size < F2_5) return OPUS_BUFFER_TOO_SMALL;
    frame_size = imin(frame_size, 48000 / 25 * 3);
    if (len <= 1) {
        data = 0;
        frame_size = imin(frame_size, st->frame_size);
    }
    if (data != 0) {
        audiosize = st->frame_size;
        mode = st->mode;
        bandwidth = st->bandwidth;
        rd_init(&dec, data, (uint32_t)len);
    } else {
        audiosize = frame_size;
        mode = st->prev_redundancy ? MODE_CELT_ONLY : st->prev_mode;
        bandwidth = 0;
        if (mode == 0) {
            LFOR(L, i, 0, audiosize * C) pcm[i] = 0;
            lsync(L);
            return audiosize;
        }
        if (audiosize > F20) {
            if constexpr (D == 0) {
                do {
                    int ret = opus_frame<1>(L, st, 0, 0, pcm, imin(audiosize, F20), w, 0);
                    if (ret < 0) return ret;
                    pcm += ret * C;
                    audiosize -= ret;
                } while (audiosize > 0);
                return frame_size;
            } else {
                return OPUS_INTERNAL_ERROR;   // unreachable: nested concealment is at most 20 ms
            }
        } else if (audiosize < F20) {
            if (audiosize > F10) audiosize = F10;
            else if (mode != MODE_SILK_ONLY && audiosize > F5 && audiosize < F10) audiosize = F5;
        }
    }
    int celt_accum = (mode != MODE_CELT_ONLY) && (frame_size >= F10);
    if (data != 0 && st->prev_mode > 0 &&
        ((mode == MODE_CELT_ONLY && st->prev_mode != MODE_CELT_ONLY && !st->prev_redundancy) ||
         (mode != MODE_CELT_ONLY && st->prev_mode == MODE_CELT_ONLY)))
        transition = 1;
    if (transition && mode == MODE_CELT_ONLY) {
        if constexpr (D == 0) {
            pcm_transition = w->pcm_transition;
            opus_frame<1>(L, st, 0, 0, pcm_transition, imin(F5, audiosize), w, 0);
        }
    }
    if (audiosize > frame_size) return OPUS_BAD_ARG;
    frame_size = audiosize;
    int16_t *pcm_silk = w->pcm_silk[D];

    // Every write of decoder state below happens in a lead stretch (first
    // lane only, barriers on both sides), so that no lane changes a field
    // another lane may still be reading.
    if (mode != MODE_CELT_ONLY) {
        int16_t *pcm_ptr = celt_accum ? pcm : pcm_silk;
        lead(L, [&]() CUO_INLINE {
            if (st->prev_mode == MODE_CELT_ONLY) silk_reset_dec(&st->silk);
            st->DecControl.payloadSize_ms = imax(10, 1000 * audiosize / 48000);
            if (data != 0) {
                st->DecControl.nChannelsInternal = st->stream_channels;
                if (mode == MODE_SILK_ONLY) {
                    if (bandwidth == BW_NB) st->DecControl.internalSampleRate = 8000;
                    else if (bandwidth == BW_MB) st->DecControl.internalSampleRate = 12000;
                    else st->DecControl.internalSampleRate = 16000;
                } else {
                    st->DecControl.internalSampleRate = 16000;
                }
            }
        });
        int lost_flag = data == 0 ? 1 : (fec ? 2 : 0);
        int decoded_samples = 0;
        do {
            int first_frame = decoded_samples == 0;
            int32_t silk_frame_size = 0;
            silk_ret = silk_decode(L, &st->silk, &st->DecControl, lost_flag, first_frame, &dec, pcm_ptr,
                                   &silk_frame_size, &w->silk);
            if (silk_ret) {
                if (lost_flag) {
                    silk_frame_size = frame_size;
                    LFOR(L, i, 0, frame_size * C) pcm_ptr[i] = 0;
                    lsync(L);
                } else {
                    return OPUS_INTERNAL_ERROR;
                }
            }
            pcm_ptr += silk_frame_size * C;
            decoded_samples += silk_frame_size;
        } while (decoded_samples < frame_size);
    }

    int start_band = 0;
    if (!fec && mode != MODE_CELT_ONLY && data != 0 && rd_tell(&dec) + 17 + 20 * (mode == MODE_HYBRID) <= 8 * len) {
        if (mode == MODE_HYBRID) redundancy = rd_bit_logp(&dec, 12);
        else redundancy = 1;
        if (redundancy) {
            celt_to_silk = rd_bit_logp(&dec, 1);
            redundancy_bytes = mode == MODE_HYBRID ? (int32_t)rd_uint(&dec, 256) + 2
                                                   : len - ((rd_tell(&dec) + 7) >> 3);
            len -= redundancy_bytes;
            if (len * 8 < rd_tell(&dec)) {
                len = 0;
                redundancy_bytes = 0;
                redundancy = 0;
            }
            dec.storage -= redundancy_bytes;
        }
    }
    if (mode != MODE_CELT_ONLY) start_band = 17;
    if (redundancy) transition = 0;
    if (transition && mode != MODE_CELT_ONLY) {
        if constexpr (D == 0) {
            pcm_transition = w->pcm_transition;
            opus_frame<1>(L, st, 0, 0, pcm_transition, imin(F5, audiosize), w, 0);
        }
    }
    int16_t *redundant_audio = w->redundant_audio;
    lead(L, [&]() CUO_INLINE {
        if (bandwidth) {
            int endband = 21;
            switch (bandwidth) {
            case BW_NB: endband = 13; break;
            case BW_MB:
            case BW_WB: endband = 17; break;
            case BW_SWB: endband = 19; break;
            default: endband = 21; break;
            }
            st->celt.end = endband;
        }
        st->celt.stream_channels = st->stream_channels;
        if (redundancy && celt_to_silk) st->celt.start = 0;
    });
    if (redundancy && celt_to_silk) {
        celt_decode(L, &st->celt, data + len, redundancy_bytes, redundant_audio, F5, 0, 0, &w->celt);
        redundant_rng = st->celt.rng;
    }
    // the previous mode decides the CELT reset and the hybrid -> SILK silence
    // frame: read before the lead stretch that may change the CELT state
    const int prev_mode = st->prev_mode, prev_redundancy = st->prev_redundancy;
    const int silence_frame =
        mode == MODE_SILK_ONLY && prev_mode == MODE_HYBRID && !(redundancy && celt_to_silk && prev_redundancy);
    lead(L, [&]() CUO_INLINE {
        st->celt.start = start_band;
        if (mode != MODE_SILK_ONLY && mode != prev_mode && prev_mode > 0 && !prev_redundancy) celt_reset(&st->celt);
        if (silence_frame) st->celt.start = 0;
    });
    if (mode != MODE_SILK_ONLY) {
        int celt_frame_size = imin(F20, frame_size);
        celt_ret = celt_decode(L, &st->celt, fec ? 0 : data, len, pcm, celt_frame_size, (data && !fec) ? &dec : 0,
                               celt_accum,
                               &w->celt);
    } else {
        const uint8_t silence[2] = {0xFF, 0xFF};
        if (!celt_accum) {
            LFOR(L, i, 0, frame_size * C) pcm[i] = 0;
            lsync(L);
        }
        if (silence_frame) celt_decode(L, &st->celt, silence, 2, pcm, F2_5, 0, celt_accum, &w->celt);
    }
    if (mode != MODE_CELT_ONLY && !celt_accum) {
        LFOR(L, i, 0, frame_size * C) pcm[i] = c_sat16((int32_t)pcm[i] + pcm_silk[i]);
        lsync(L);
    }
    if (redundancy && !celt_to_silk) {
        lead(L, [&]() CUO_INLINE {
            celt_reset(&st->celt);
            st->celt.start = 0;
        });
        celt_decode(L, &st->celt, data + len, redundancy_bytes, redundant_audio, F5, 0, 0, &w->celt);
        redundant_rng = st->celt.rng;
        smooth_fade(L, pcm + C * (frame_size - F2_5), redundant_audio + C * F2_5, pcm + C * (frame_size - F2_5),
                    F2_5, C);
    }
    if (redundancy && celt_to_silk && (prev_mode != MODE_SILK_ONLY || prev_redundancy)) {
        LFOR(L, i, 0, F2_5 * C) pcm[i] = redundant_audio[i];
        smooth_fade(L, redundant_audio + C * F2_5, pcm + C * F2_5, pcm + C * F2_5, F2_5, C);
    }
    if (transition) {
        if (audiosize >= F5) {
            LFOR(L, i, 0, C * F2_5) pcm[i] = pcm_transition[i];
            smooth_fade(L, pcm_transition + C * F2_5, pcm + C * F2_5, pcm + C * F2_5, F2_5, C);
        } else {
            smooth_fade(L, pcm_transition, pcm, pcm, F2_5, C);
        }
    }
#ifdef CUO_FRAME_EVENTS
    // test builds only: which branches of the frame decode ran
    if (L.id == 0) cuo_frame_event(D, mode, prev_mode, redundancy, celt_to_silk, transition, silence_frame);
#endif
    lead(L, [&]() CUO_INLINE {
        if (len <= 1) st->rangeFinal = 0;
        else st->rangeFinal = dec.rng ^ redundant_rng;
        st->prev_mode = mode;
        st->prev_redundancy = redundancy && !celt_to_silk;
    });
    return celt_ret < 0 ? celt_ret : audiosize;
}

// Number of samples per channel a packet decodes to (opus_decode_native checks),
// or a negative Opus error code.
DFN int packet_nb_samples(const uint8_t *data, int32_t len)
{
    if (len < 1) return OPUS_BAD_ARG;
    int count, code = data[0] & 3;
    if (code == 0) count = 1;
    else if (code != 3) count = 2;
    else if (len < 2) return OPUS_INVALID_PACKET;
    else count = data[1] & 0x3F;
    int samples = count * toc_samples_per_frame(data[0]);
    if (samples * 25 > 48000 * 3) return OPUS_INVALID_PACKET;
    return samples;
}

// Concealment of n samples per channel (src/opus_decoder.c:715-729, the
// len == 0 branch of opus_decode_native), emitted frame by frame.
template <class Emit>
DNI int conceal_samples(Lanes L, OpusDec *st, int n, int16_t *frame_buf, OpusScratch *w, Emit &emit)
{
    int pcm_count = 0;
    do {
        int ret = opus_frame<0>(L, st, 0, 0, frame_buf, n - pcm_count, w, 0);
        if (ret < 0) return ret;
        emit(frame_buf, ret);
        pcm_count += ret;
    } while (pcm_count < n);
    return pcm_count;
}

// The decode_fec = 1 branch of opus_decode_native (src/opus_decoder.c:745-779)
// for a parsed packet whose first frame is data[0 .. size0): conceal up to the
// last frame, which comes from the packet's FEC data.  Its own function, so
// the code of the lossless path stays small.
template <class Emit>
DNI int decode_fec(Lanes L, OpusDec *st, const uint8_t *data, int size0, int packet_mode, int packet_bandwidth,
                   int packet_frame_size, int packet_stream_channels, int16_t *frame_buf, OpusScratch *w,
                   Emit &emit)
{
    const int frame_size = MAX_PACKET_SAMPLES;
    if (frame_size < packet_frame_size || packet_mode == MODE_CELT_ONLY || st->mode == MODE_CELT_ONLY) {
        int ret = conceal_samples(L, st, frame_size, frame_buf, w, emit);
        if (ret < 0) return ret;
        lead(L, [&]() CUO_INLINE { st->last_packet_duration = ret; });
        return ret;
    }
    int duration_copy = st->last_packet_duration;
    if (frame_size - packet_frame_size != 0) {
        int ret = conceal_samples(L, st, frame_size - packet_frame_size, frame_buf, w, emit);
        if (ret < 0) {
            lead(L, [&]() CUO_INLINE { st->last_packet_duration = duration_copy; });
            return ret;
        }
    }
    lead(L, [&]() CUO_INLINE {
        st->mode = packet_mode;
        st->bandwidth = packet_bandwidth;
        st->frame_size = packet_frame_size;
        st->stream_channels = packet_stream_channels;
    });
    int ret = opus_frame<0>(L, st, data, size0, frame_buf, packet_frame_size, w, 1);
    if (ret < 0) return ret;
    emit(frame_buf, ret);
    lead(L, [&]() CUO_INLINE { st->last_packet_duration = frame_size; });
    return frame_size;
}

// src/opus_decoder.c opus_decode_native (:670-811; not self-delimited,
// frame_size = MAX_PACKET_SAMPLES).  `emit(frame_pcm, n)` receives each decoded
// frame (n samples per channel, interleaved) so the caller can place it; the
// frame buffer is reused for the next frame.  fec = 1 is decode_fec = 1: the
// packet is the one after a lost packet, and the lost packet's audio is
// concealed up to the last frame, which comes from the packet's FEC data
// (:745-779).
template <class Emit>
DFN int opus_decode_packet(Lanes L, OpusDec *st, const uint8_t *data, int32_t len, int16_t *frame_buf,
                           OpusScratch *w, Emit &emit, int fec)
{
    const int frame_size = MAX_PACKET_SAMPLES;
    if (len == 0 || data == 0) {
        int ret = conceal_samples(L, st, frame_size, frame_buf, w, emit);
        if (ret < 0) return ret;
        lead(L, [&]() CUO_INLINE { st->last_packet_duration = ret; });
        return ret;
    }
    if (len < 0) return OPUS_BAD_ARG;
    int packet_mode = toc_mode(data[0]);
    int packet_bandwidth = toc_bandwidth(data[0]);
    int packet_frame_size = toc_samples_per_frame(data[0]);
    int packet_stream_channels = (data[0] & 0x4) ? 2 : 1;
    int16_t *size = w->sizes;
    int offset = 0;
    int count = packet_parse(data, len, size, &offset);
    if (count < 0) return count;
    data += offset;
    if (fec)
        return decode_fec(L, st, data, size[0], packet_mode, packet_bandwidth, packet_frame_size,
                          packet_stream_channels, frame_buf, w, emit);
    if (count * packet_frame_size > frame_size) return OPUS_BUFFER_TOO_SMALL;
    lead(L, [&]() CUO_INLINE {
        st->mode = packet_mode;
        st->bandwidth = packet_bandwidth;
        st->frame_size = packet_frame_size;
        st->stream_channels = packet_stream_channels;
    });
    int nb_samples = 0;
    for (int i = 0; i < count; i++) {
        int ret = opus_frame<0>(L, st, data, size[i], frame_buf, frame_size - nb_samples, w, 0);
        if (ret < 0) return ret;
        emit(frame_buf, ret);
        data += size[i];
        nb_samples += ret;
    }
    lead(L, [&]() CUO_INLINE { st->last_packet_duration = nb_samples; });
    return nb_samples;
}

} // namespace cuo
