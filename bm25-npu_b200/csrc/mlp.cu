// Threshold MLP (32 -> 64 -> 64 -> 1, ReLU, FP32): forward, backward and Adam
// kernels, exported through the C ABI (include/bm25_b200.h).
//
// The network predicts, from per-query features, the log of the query's K-th
// best score; the pruned Search uses exp(prediction - margin) as its starting
// bound (a wrong guess costs a re-run on the plain path, never a wrong result).
// No counterpart in the reference: this is the learned part of the engine.
//
// Training is deterministic: each CTA of the backward kernel writes its partial
// gradient to its own slice of the scratch array and a second kernel sums the
// slices in a fixed order.
#include "bm25_b200.h"
#include "mlp.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>

namespace bm25mlp {

constexpr int kRows = 64;   // samples per forward CTA
constexpr int kBRows = 32;  // samples per backward CTA

__global__ void __launch_bounds__(kRows) ForwardKernel(const float *params, const float *x, long long batch, float *y)
{
    __shared__ float p[kParams];
    for (int i = threadIdx.x; i < kParams; i += kRows)
        p[i] = params[i];
    __syncthreads();
    const long long r = (long long)blockIdx.x * kRows + threadIdx.x;
    if (r >= batch)
        return;
    float xi[kIn], h1[kH], h2[kH];
    for (int j = 0; j < kIn; ++j)
        xi[j] = x[r * kIn + j];
    y[r] = Forward(p, xi, h1, h2);
}

// Loss per sample: w * (y - t)^2 with w = over_weight when y > t (an over-estimate
// of the K-th score sends the query to the plain path), else 1.  Mean over the batch.
// Each CTA writes its partial gradient (kParams floats) and its loss sum.
__global__ void __launch_bounds__(kBRows) BackwardKernel(const float *__restrict__ p, const float *x, const float *t,
                                                         long long batch, float over_weight, float *partial,
                                                         float *partial_loss)
{
    __shared__ float sx[kBRows][kIn + 1];
    __shared__ float sh1[kBRows][kH + 1], sd1[kBRows][kH + 1];
    __shared__ float sh2[kBRows][kH + 1], sd2[kBRows][kH + 1];
    __shared__ float sdy[kBRows], sloss[kBRows];
    const int tid = threadIdx.x;
    const long long r = (long long)blockIdx.x * kBRows + tid;
    const bool live = r < batch;
    float xi[kIn], h1[kH], h2[kH];
    for (int j = 0; j < kIn; ++j)
        xi[j] = live ? x[r * kIn + j] : 0.0f;
    float dy = 0.0f, loss = 0.0f;
    if (live) {
        const float y = Forward(p, xi, h1, h2);
        const float e = y - t[r];
        const float w = e > 0.0f ? over_weight : 1.0f;
        loss = w * e * e;
        dy = 2.0f * w * e / (float)batch;
    } else {
        for (int i = 0; i < kH; ++i)
            h1[i] = h2[i] = 0.0f;
    }
    // dh2 = dy * w3 (ReLU gate), dh1 = W2^T dh2 (ReLU gate)
    float d2[kH];
    for (int i = 0; i < kH; ++i)
        d2[i] = h2[i] > 0.0f ? dy * p[kOffW3 + i] : 0.0f;
    for (int j = 0; j < kH; ++j) {
        float acc = 0.0f;
        for (int i = 0; i < kH; ++i)
            acc = fmaf(p[kOffW2 + i * kH + j], d2[i], acc);
        sd1[tid][j] = h1[j] > 0.0f ? acc : 0.0f;
        sh1[tid][j] = h1[j];
        sh2[tid][j] = h2[j];
        sd2[tid][j] = d2[j];
    }
    for (int j = 0; j < kIn; ++j)
        sx[tid][j] = xi[j];
    sdy[tid] = dy;
    sloss[tid] = loss;
    __syncthreads();
    // this CTA's gradient, each parameter summed over the CTA's samples in row order
    float *out = partial + (long long)blockIdx.x * kParams;
    for (int q = tid; q < kParams; q += kBRows) {
        float g = 0.0f;
        if (q < kOffB1) {
            const int i = (q - kOffW1) / kIn, j = (q - kOffW1) % kIn;
            for (int s = 0; s < kBRows; ++s)
                g = fmaf(sd1[s][i], sx[s][j], g);
        } else if (q < kOffW2) {
            const int i = q - kOffB1;
            for (int s = 0; s < kBRows; ++s)
                g += sd1[s][i];
        } else if (q < kOffB2) {
            const int i = (q - kOffW2) / kH, j = (q - kOffW2) % kH;
            for (int s = 0; s < kBRows; ++s)
                g = fmaf(sd2[s][i], sh1[s][j], g);
        } else if (q < kOffW3) {
            const int i = q - kOffB2;
            for (int s = 0; s < kBRows; ++s)
                g += sd2[s][i];
        } else if (q < kOffB3) {
            const int j = q - kOffW3;
            for (int s = 0; s < kBRows; ++s)
                g = fmaf(sdy[s], sh2[s][j], g);
        } else {
            for (int s = 0; s < kBRows; ++s)
                g += sdy[s];
        }
        out[q] = g;
    }
    if (tid == 0) {
        float l = 0.0f;
        for (int s = 0; s < kBRows; ++s)
            l += sloss[s];
        partial_loss[blockIdx.x] = l;
    }
}

// grad[q] = sum over CTAs of partial[c][q] in CTA order; loss = sum of partial losses / batch.
__global__ void ReduceKernel(const float *partial, const float *partial_loss, int ctas, long long batch, float *grad,
                             float *loss)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < kParams) {
        float g = 0.0f;
        for (int c = 0; c < ctas; ++c)
            g += partial[(long long)c * kParams + q];
        grad[q] = g;
    }
    if (q == 0 && loss) {
        float l = 0.0f;
        for (int c = 0; c < ctas; ++c)
            l += partial_loss[c];
        *loss = l / (float)batch;
    }
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) with bias correction for step `step` (1-based).
__global__ void AdamKernel(float *params, float *m, float *v, const float *grad, float lr, int step)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kParams)
        return;
    const float g = grad[q];
    const float mq = 0.9f * m[q] + 0.1f * g, vq = 0.999f * v[q] + 0.001f * g * g;
    m[q] = mq;
    v[q] = vq;
    const float mh = mq / (1.0f - powf(0.9f, (float)step)), vh = vq / (1.0f - powf(0.999f, (float)step));
    params[q] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

} // namespace bm25mlp

namespace {
thread_local std::string g_mlp_error;
int Fail(int status, const std::string &m)
{
    g_mlp_error = m;
    return status;
}
int CudaStatus(cudaError_t e, const char *what)
{
    if (e == cudaSuccess)
        return BM25_OK;
    return Fail(BM25_ERR_INNER_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}
} // namespace

extern "C" int64_t bm25_mlp_param_count(void) { return bm25mlp::kParams; }

extern "C" int64_t bm25_mlp_scratch_floats(int64_t batch)
{
    const int64_t ctas = (batch + bm25mlp::kBRows - 1) / bm25mlp::kBRows;
    return ctas * (bm25mlp::kParams + 1);
}

extern "C" int bm25_mlp_forward(const float *params, const float *features, int64_t batch, float *out, void *stream)
{
    if (!params || !features || !out || batch < 1)
        return Fail(BM25_ERR_INVALID_PARAM, "Null buffer or empty batch");
    const int64_t ctas = (batch + bm25mlp::kRows - 1) / bm25mlp::kRows;
    bm25mlp::ForwardKernel<<<(unsigned)ctas, bm25mlp::kRows, 0, static_cast<cudaStream_t>(stream)>>>(
        params, features, batch, out);
    return CudaStatus(cudaGetLastError(), "MLP forward launch");
}

extern "C" int bm25_mlp_gradient(const float *params, const float *features, const float *targets, int64_t batch,
                                 float over_weight, float *scratch, float *grad, float *loss, void *stream)
{
    if (!params || !features || !targets || !scratch || !grad || batch < 1)
        return Fail(BM25_ERR_INVALID_PARAM, "Null buffer or empty batch");
    const int64_t ctas = (batch + bm25mlp::kBRows - 1) / bm25mlp::kBRows;
    if (ctas > (1 << 20))
        return Fail(BM25_ERR_INVALID_PARAM, "Batch too large");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float *partial = scratch, *partial_loss = scratch + ctas * bm25mlp::kParams;
    bm25mlp::BackwardKernel<<<(unsigned)ctas, bm25mlp::kBRows, 0, s>>>(params, features, targets, batch, over_weight,
                                                                      partial, partial_loss);
    int st = CudaStatus(cudaGetLastError(), "MLP backward launch");
    if (st != BM25_OK)
        return st;
    bm25mlp::ReduceKernel<<<(bm25mlp::kParams + 255) / 256, 256, 0, s>>>(partial, partial_loss, (int)ctas, batch,
                                                                          grad, loss);
    return CudaStatus(cudaGetLastError(), "MLP reduce launch");
}

extern "C" int bm25_mlp_adam(float *params, float *m, float *v, const float *grad, float lr, int32_t step,
                             void *stream)
{
    if (!params || !m || !v || !grad || step < 1)
        return Fail(BM25_ERR_INVALID_PARAM, "Null buffer or step < 1");
    bm25mlp::AdamKernel<<<(bm25mlp::kParams + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(params, m, v,
                                                                                                   grad, lr, step);
    return CudaStatus(cudaGetLastError(), "MLP Adam launch");
}

extern "C" int bm25_mlp_last_error(char *buffer, size_t length)
{
    if (buffer && length) {
        const size_t n = g_mlp_error.size() < length - 1 ? g_mlp_error.size() : length - 1;
        g_mlp_error.copy(buffer, n);
        buffer[n] = '\0';
    }
    return BM25_OK;
}
