// Learned cost model of the decode scheduler: per-chain features from the
// packets' TOC bytes, and an FP32 multilayer perceptron (16 -> 64 -> 64 -> 1,
// ReLU) that predicts the log decode time of a chain, trained and evaluated
// with the kernels below.  The queue schedule of the decoder visits chains in
// decreasing predicted cost (longest first); the packet-count order is the
// fallback.  None of this changes a decoded sample: it only orders the work.
//
// Parameter layout (floats, one contiguous device buffer of MLP_NPARAM):
//   W1[16][64] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3
// Training is full-batch Adam on the mean squared error.  Gradients are
// reduced deterministically: one kernel stores each sample's activations and
// back-propagated signals, a second sums them over samples in index order
// for every parameter (no atomics), so a training run is reproducible.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "../../include/cuopus.h"

namespace {

constexpr int F = CUOPUS_MLP_FEATURES;   // 16
constexpr int H = CUOPUS_MLP_HIDDEN;     // 64
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + F * H;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + H;
constexpr int NPARAM = OFF_B3 + 1;
static_assert(NPARAM == CUOPUS_MLP_NPARAM, "parameter layout");
// per-sample record of the training forward/backward pass
constexpr int R_X = 0, R_H1 = R_X + F, R_G1 = R_H1 + H, R_H2 = R_G1 + H, R_G2 = R_H2 + H, R_D = R_G2 + H;
constexpr int REC = R_D + 1;

// ------------------------------------------------------------------ features

// TOC of RFC 6716 section 3.1: config = toc >> 3.
__device__ __forceinline__ int toc_mode(int config) { return config < 12 ? 0 : (config < 16 ? 1 : 2); }
__device__ __forceinline__ int toc_qms(int config)   // frame duration in quarter milliseconds
{
    if (config < 12) return (config & 3) == 0 ? 40 : (config & 3) == 1 ? 80 : (config & 3) == 2 ? 160 : 240;
    if (config < 16) return (config & 1) ? 80 : 40;
    return 10 << (config & 3);
}
__device__ __forceinline__ int toc_bw(int config)   // 0 NB, 1 MB, 2 WB, 3 SWB, 4 FB
{
    if (config < 12) return config >> 2;
    if (config < 16) return config < 14 ? 3 : 4;
    int b = (config - 16) >> 2;          // NB, WB, SWB, FB
    return b == 0 ? 0 : b + 1;
}

// One thread per chain; feat[c * 16 + k].
__global__ void k_chain_features(const uint8_t *__restrict__ data, const uint64_t *__restrict__ off,
                                 const uint32_t *__restrict__ len, const uint32_t *__restrict__ first,
                                 const uint32_t *__restrict__ npkts, const uint8_t *__restrict__ channels,
                                 int nchains, float *__restrict__ feat)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchains) return;
    double bytes = 0, frames = 0, q = 0;
    double fm[3] = {0, 0, 0}, f25 = 0, f5 = 0, f10 = 0, f20 = 0, f40 = 0, bw = 0, stereo = 0;
    uint32_t n = npkts[c];
    for (uint32_t k = 0; k < n; k++) {
        uint64_t p = (uint64_t)first[c] + k;
        uint32_t L = len[p];
        bytes += L;
        if (!L) continue;
        const uint8_t *b = data + off[p];
        int toc = b[0], cfg = toc >> 3, code = toc & 3;
        int nf = code == 0 ? 1 : code < 3 ? 2 : (L > 1 ? (b[1] & 63) : 0);
        int qms = toc_qms(cfg);
        frames += nf;
        q += (double)nf * qms;
        fm[toc_mode(cfg)] += nf;
        if (qms == 10) f25 += nf;
        else if (qms == 20) f5 += nf;
        else if (qms == 40) f10 += nf;
        else if (qms == 80) f20 += nf;
        else f40 += nf;
        bw += (double)nf * toc_bw(cfg);
        stereo += (toc >> 2) & 1;
    }
    double secs = q / 4000.0;
    double fr = frames > 0 ? 1.0 / frames : 0.0;
    float *o = feat + (size_t)c * F;
    o[0] = (float)log1p((double)n);
    o[1] = (float)log1p(bytes);
    o[2] = (float)log1p(frames);
    o[3] = (float)log1p(secs);
    o[4] = (float)(channels[c] - 1);
    o[5] = (float)(fm[0] * fr);
    o[6] = (float)(fm[1] * fr);
    o[7] = (float)(fm[2] * fr);
    o[8] = (float)(f25 * fr);
    o[9] = (float)(f5 * fr);
    o[10] = (float)(f10 * fr);
    o[11] = (float)(f20 * fr);
    o[12] = (float)(f40 * fr);
    o[13] = (float)(bw * fr * 0.25);
    o[14] = (float)(n ? stereo / n : 0.0);
    o[15] = (float)log1p(secs > 0 ? bytes / secs : 0.0);
}

// ------------------------------------------------------------------ network

// Forward pass of one sample with the weights staged in shared memory.
// Returns the output; h1 / h2 receive the post-ReLU activations.
__device__ __forceinline__ float mlp_forward(const float *w, const float *x, float *h1, float *h2)
{
#pragma unroll 4
    for (int j = 0; j < H; j++) {
        float a = w[OFF_B1 + j];
#pragma unroll
        for (int i = 0; i < F; i++) a = fmaf(x[i], w[OFF_W1 + i * H + j], a);
        h1[j] = a > 0.f ? a : 0.f;
    }
    for (int j = 0; j < H; j++) {
        float a = w[OFF_B2 + j];
#pragma unroll 8
        for (int k = 0; k < H; k++) a = fmaf(h1[k], w[OFF_W2 + k * H + j], a);
        h2[j] = a > 0.f ? a : 0.f;
    }
    float y = w[OFF_B3];
#pragma unroll 8
    for (int j = 0; j < H; j++) y = fmaf(h2[j], w[OFF_W3 + j], y);
    return y;
}

__device__ void stage_weights(float *ws, const float *__restrict__ params)
{
    for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) ws[i] = params[i];
    __syncthreads();
}

__global__ void k_mlp_predict(const float *__restrict__ params, const float *__restrict__ X, int n,
                              float *__restrict__ y)
{
    extern __shared__ float ws[];
    stage_weights(ws, params);
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[F], h1[H], h2[H];
#pragma unroll
    for (int i = 0; i < F; i++) x[i] = X[(size_t)s * F + i];
    y[s] = mlp_forward(ws, x, h1, h2);
}

// Forward + back-propagated signals of one sample for the loss
// L = mean_s (y_s - t_s)^2: rec[s] = {x, h1, g1, h2, g2, dL/dy}, with
// g2 = dL/d(pre-activation 2) and g1 = dL/d(pre-activation 1).
__global__ void k_mlp_backprop(const float *__restrict__ params, const float *__restrict__ X,
                               const float *__restrict__ T, int n, float *__restrict__ rec, float *__restrict__ sqerr)
{
    extern __shared__ float ws[];
    stage_weights(ws, params);
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[F], h1[H], h2[H];
#pragma unroll
    for (int i = 0; i < F; i++) x[i] = X[(size_t)s * F + i];
    float y = mlp_forward(ws, x, h1, h2);
    float e = y - T[s];
    float d = 2.f * e / (float)n;
    float *r = rec + (size_t)s * REC;
#pragma unroll
    for (int i = 0; i < F; i++) r[R_X + i] = x[i];
    float g2[H];
    for (int j = 0; j < H; j++) {
        g2[j] = h2[j] > 0.f ? d * ws[OFF_W3 + j] : 0.f;
        r[R_H1 + j] = h1[j];
        r[R_H2 + j] = h2[j];
        r[R_G2 + j] = g2[j];
    }
    for (int k = 0; k < H; k++) {
        float a = 0.f;
        if (h1[k] > 0.f) {
#pragma unroll 8
            for (int j = 0; j < H; j++) a = fmaf(ws[OFF_W2 + k * H + j], g2[j], a);
        }
        r[R_G1 + k] = a;
    }
    r[R_D] = d;
    sqerr[s] = e * e;
}

// One thread per parameter: its gradient summed over samples in index order.
// Thread NPARAM also sums the squared errors into *loss.
__global__ void k_mlp_reduce(const float *__restrict__ rec, const float *__restrict__ sqerr, int n,
                             float *__restrict__ grad, float *__restrict__ loss)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > NPARAM) return;
    if (p == NPARAM) {
        float a = 0.f;
        for (int s = 0; s < n; s++) a += sqerr[s];
        *loss = a / (float)n;
        return;
    }
    int ca, cb;   // gradient = sum_s rec[s][ca] * rec[s][cb] (cb < 0: rec[s][ca] alone)
    if (p < OFF_B1) { ca = R_X + p / H; cb = R_G1 + p % H; }
    else if (p < OFF_W2) { ca = R_G1 + (p - OFF_B1); cb = -1; }
    else if (p < OFF_B2) { ca = R_H1 + (p - OFF_W2) / H; cb = R_G2 + (p - OFF_W2) % H; }
    else if (p < OFF_W3) { ca = R_G2 + (p - OFF_B2); cb = -1; }
    else if (p < OFF_B3) { ca = R_H2 + (p - OFF_W3); cb = R_D; }
    else { ca = R_D; cb = -1; }
    float a = 0.f;
    if (cb < 0)
        for (int s = 0; s < n; s++) a += rec[(size_t)s * REC + ca];
    else
        for (int s = 0; s < n; s++) a = fmaf(rec[(size_t)s * REC + ca], rec[(size_t)s * REC + cb], a);
    grad[p] = a;
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8).  `t` counts the steps taken on
// the device (k_tick advances it after each update), so a captured graph of
// several steps stays correct on replay.
__global__ void k_adam(float *__restrict__ params, const float *__restrict__ grad, float *__restrict__ m,
                       float *__restrict__ v, const int *__restrict__ t, float lr)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAM) return;
    float step = (float)(*t + 1);
    float g = grad[p];
    float mi = 0.9f * m[p] + 0.1f * g;
    float vi = 0.999f * v[p] + 0.001f * g * g;
    m[p] = mi;
    v[p] = vi;
    float mh = mi / (1.f - powf(0.9f, step));
    float vh = vi / (1.f - powf(0.999f, step));
    params[p] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

__global__ void k_tick(int *t) { *t += 1; }

const int THREADS = 128;
const size_t SMEM = NPARAM * sizeof(float);

int set_err(char *errbuf, size_t errcap, int rc, const char *msg, cudaError_t e)
{
    if (errbuf && errcap) {
        size_t n = strlen(msg);
        const char *es = cudaGetErrorString(e);
        size_t m = strlen(es);
        size_t k = 0;
        for (size_t i = 0; i < n && k + 1 < errcap; i++) errbuf[k++] = msg[i];
        if (k + 2 < errcap) { errbuf[k++] = ':'; errbuf[k++] = ' '; }
        for (size_t i = 0; i < m && k + 1 < errcap; i++) errbuf[k++] = es[i];
        errbuf[k] = 0;
    }
    return rc;
}

#define CKM(call, what)                                                                                \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return set_err(errbuf, errcap, 2, what, e_);                            \
    } while (0)

int grid_of(int n) { return (n + THREADS - 1) / THREADS; }

cudaError_t smem_attr()
{
    static bool done = false;
    if (done) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_mlp_predict, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_backprop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    done = e == cudaSuccess;
    return e;
}

cudaError_t grad_launches(const float *params, const float *X, const float *T, int n, float *rec, float *sqerr,
                          float *grad, float *loss, cudaStream_t st)
{
    k_mlp_backprop<<<grid_of(n), THREADS, SMEM, st>>>(params, X, T, n, rec, sqerr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_mlp_reduce<<<grid_of(NPARAM + 1), THREADS, 0, st>>>(rec, sqerr, n, grad, loss);
    return cudaGetLastError();
}

} // namespace

extern "C" int cuopus_chain_features(const cuopus_batch *b, float *feat_dev, void *cuda_stream, char *errbuf,
                                     size_t errcap)
{
    if (!b || !feat_dev || !b->data || !b->off || !b->len || !b->first || !b->npkts || !b->channels)
        return set_err(errbuf, errcap, 3, "chain_features: NULL argument", cudaSuccess);
    if (b->nchains <= 0) return 0;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    k_chain_features<<<grid_of(b->nchains), THREADS, 0, st>>>(b->data, b->off, b->len, b->first, b->npkts,
                                                              b->channels, b->nchains, feat_dev);
    CKM(cudaGetLastError(), "chain_features launch");
    CKM(cudaStreamSynchronize(st), "chain_features");
    return 0;
}

extern "C" int cuopus_mlp_init(float *params_dev, uint64_t seed, void *cuda_stream, char *errbuf, size_t errcap)
{
    if (!params_dev) return set_err(errbuf, errcap, 3, "mlp_init: NULL params", cudaSuccess);
    // He-uniform weights from a 64-bit LCG, zero biases
    std::vector<float> p(NPARAM, 0.f);
    uint64_t s = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto uni = [&]() {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        return (float)((double)(s >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
    };
    float a1 = sqrtf(6.f / F), a2 = sqrtf(6.f / H), a3 = sqrtf(3.f / H);
    for (int i = 0; i < F * H; i++) p[OFF_W1 + i] = a1 * uni();
    for (int i = 0; i < H * H; i++) p[OFF_W2 + i] = a2 * uni();
    for (int i = 0; i < H; i++) p[OFF_W3 + i] = a3 * uni();
    cudaStream_t st = (cudaStream_t)cuda_stream;
    CKM(cudaMemcpyAsync(params_dev, p.data(), NPARAM * sizeof(float), cudaMemcpyHostToDevice, st), "mlp_init copy");
    CKM(cudaStreamSynchronize(st), "mlp_init");
    return 0;
}

extern "C" int cuopus_mlp_predict(const float *params_dev, const float *x_dev, int n, float *y_dev,
                                  void *cuda_stream, char *errbuf, size_t errcap)
{
    if (!params_dev || (n > 0 && (!x_dev || !y_dev)))
        return set_err(errbuf, errcap, 3, "mlp_predict: NULL argument", cudaSuccess);
    if (n <= 0) return 0;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    CKM(smem_attr(), "mlp smem");
    k_mlp_predict<<<grid_of(n), THREADS, SMEM, st>>>(params_dev, x_dev, n, y_dev);
    CKM(cudaGetLastError(), "mlp_predict launch");
    CKM(cudaStreamSynchronize(st), "mlp_predict");
    return 0;
}

extern "C" int cuopus_mlp_grad(const float *params_dev, const float *x_dev, const float *t_dev, int n,
                               float *grad_dev, float *loss_dev, void *cuda_stream, char *errbuf, size_t errcap)
{
    if (!params_dev || !x_dev || !t_dev || !grad_dev || !loss_dev || n <= 0)
        return set_err(errbuf, errcap, 3, "mlp_grad: bad argument", cudaSuccess);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    CKM(smem_attr(), "mlp smem");
    float *rec = nullptr, *sq = nullptr;
    CKM(cudaMalloc(&rec, (size_t)n * REC * sizeof(float)), "mlp_grad alloc");
    cudaError_t e = cudaMalloc(&sq, (size_t)n * sizeof(float));
    if (e == cudaSuccess) e = grad_launches(params_dev, x_dev, t_dev, n, rec, sq, grad_dev, loss_dev, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(rec);
    cudaFree(sq);
    if (e != cudaSuccess) return set_err(errbuf, errcap, 2, "mlp_grad", e);
    return 0;
}

// Full-batch Adam at learning rate lr; the step (gradient kernels + update)
// is captured once as a CUDA graph of 50 steps and replayed, so the steps run
// are `steps` rounded up to a multiple of 50.  losses (host, may be NULL,
// `steps` entries) receives the loss before each step.
extern "C" int cuopus_mlp_train(float *params_dev, const float *x_dev, const float *t_dev, int n, int steps,
                                float lr, float *losses, void *cuda_stream, char *errbuf, size_t errcap)
{
    if (!params_dev || !x_dev || !t_dev || n <= 0 || steps < 0)
        return set_err(errbuf, errcap, 3, "mlp_train: bad argument", cudaSuccess);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    CKM(smem_attr(), "mlp smem");
    const int chunk = 50;
    float *rec = nullptr, *work = nullptr;
    int *tstep = nullptr;
    // work: sqerr[n] | grad | m | v | loss[chunk]
    size_t wn = (size_t)n + 3 * NPARAM + chunk;
    cudaError_t e = cudaMalloc(&rec, (size_t)n * REC * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&work, wn * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&tstep, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(work, 0, wn * sizeof(float), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(tstep, 0, sizeof(int), st);
    float *sq = work, *grad = sq + n, *m = grad + NPARAM, *v = m + NPARAM, *lossv = v + NPARAM;
    cudaStream_t cs = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t e1 = cudaSuccess;
            for (int k = 0; k < chunk && e1 == cudaSuccess; k++) {
                e1 = grad_launches(params_dev, x_dev, t_dev, n, rec, sq, grad, lossv + k, cs);
                if (e1 == cudaSuccess) {
                    k_adam<<<grid_of(NPARAM), THREADS, 0, cs>>>(params_dev, grad, m, v, tstep, lr);
                    k_tick<<<1, 1, 0, cs>>>(tstep);
                    e1 = cudaGetLastError();
                }
            }
            e = cudaStreamEndCapture(cs, &g);
            if (e == cudaSuccess) e = e1;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
        if (g) cudaGraphDestroy(g);
    }
    std::vector<float> lv(chunk);
    for (int done = 0; e == cudaSuccess && done < steps; done += chunk) {
        e = cudaGraphLaunch(exec, st);
        if (e == cudaSuccess && losses) {
            e = cudaMemcpyAsync(lv.data(), lossv, chunk * sizeof(float), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            for (int k = 0; k < chunk && done + k < steps; k++) losses[done + k] = lv[k];
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (exec) cudaGraphExecDestroy(exec);
    if (cs) cudaStreamDestroy(cs);
    cudaFree(rec);
    cudaFree(work);
    cudaFree(tstep);
    if (e != cudaSuccess) return set_err(errbuf, errcap, 2, "mlp_train", e);
    return 0;
}
