/* CPU restatement of the reference's 48 -> 16 kHz resampler.
 *
 * TEST INFRASTRUCTURE (oracle).  Follows cuopus_kernels.cuh:96-149 of the
 * reference:
 *   taps  rs_make_taps (:136-149): 49-tap windowed sinc, cutoff 1/3 of the
 *         48 kHz Nyquist rate, Kaiser beta 8.6 (I0 by power series, :123-132),
 *         normalised to unity DC gain, computed in double and rounded to float
 *         (the same formula as gpu_resample.py:24-32);
 *   y[i]  cuopus_resample48to16 (:96-111): acc = 0; for t in 0..48 in order:
 *         acc = fma(taps[t], x, acc) with x = in[3i - 24 + t] / 32768 and
 *         samples outside [0, avail) read as 0 (nvcc contracts acc += a*b to an
 *         FMA; fmaf here is the same correctly rounded operation).
 * orp_resample_f64 applies the double-precision taps in double (the FP64 oracle
 * the fp32 error is reported against).
 */
#include <math.h>
#include <stdint.h>

#define ORP_TAPS 49
#define ORP_PAD 24

static double orp_i0(double x)
{
    double s = 1.0, t = 1.0, q = x * x / 4.0;
    for (int k = 1; k < 64; k++) {
        t *= q / ((double)k * k);
        s += t;
        if (t < 1e-18 * s) break;
    }
    return s;
}

void orp_make_taps_f64(double *h)
{
    double sum = 0.0;
    for (int i = 0; i < ORP_TAPS; i++) {
        double n = i - (ORP_TAPS - 1) / 2.0;
        double v = (n == 0.0) ? (1.0 / 3.0) : sin(M_PI * (1.0 / 3.0) * n) / (M_PI * n);
        double r = 2.0 * i / (ORP_TAPS - 1) - 1.0;
        double w = orp_i0(8.6 * sqrt(1.0 - r * r)) / orp_i0(8.6);
        h[i] = v * w;
        sum += h[i];
    }
    for (int i = 0; i < ORP_TAPS; i++) h[i] /= sum;
}

void orp_make_taps(float *taps)
{
    double h[ORP_TAPS];
    orp_make_taps_f64(h);
    for (int i = 0; i < ORP_TAPS; i++) taps[i] = (float)h[i];
}

void orp_resample(const int16_t *in, int64_t avail, int64_t n_out, float *out)
{
    float taps[ORP_TAPS];
    orp_make_taps(taps);
    for (int64_t i = 0; i < n_out; i++) {
        int64_t c = 3 * i;
        float acc = 0.0f;
        for (int t = 0; t < ORP_TAPS; t++) {
            int64_t li = c - ORP_PAD + t;
            float v = (li >= 0 && li < avail) ? (float)in[li] * (1.0f / 32768.0f) : 0.0f;
            acc = fmaf(taps[t], v, acc);
        }
        out[i] = acc;
    }
}

void orp_resample_f64(const int16_t *in, int64_t avail, int64_t n_out, double *out)
{
    double h[ORP_TAPS];
    orp_make_taps_f64(h);
    for (int64_t i = 0; i < n_out; i++) {
        double acc = 0.0;
        for (int t = 0; t < ORP_TAPS; t++) {
            int64_t li = 3 * i - ORP_PAD + t;
            if (li >= 0 && li < avail) acc += h[t] * (in[li] / 32768.0);
        }
        out[i] = acc;
    }
}
