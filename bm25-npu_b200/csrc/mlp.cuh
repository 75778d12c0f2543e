// Threshold MLP layout and per-sample forward pass, shared by the training
// kernels (mlp.cu) and the engine's learned-bound kernel.
//
// Parameters are one flat FP32 array (kParams floats):
//   W1 [64][32] | b1 [64] | W2 [64][64] | b2 [64] | w3 [64] | b3 [1]
// Layers: h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2), y = w3 . h2 + b3, each
// dot product a chain of fmaf in index order starting from the bias.
#pragma once

namespace bm25mlp {

constexpr int kIn = 32, kH = 64;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kIn, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH, kParams = kOffB3 + 1;

// Per-sample forward (parameters in shared or global memory); h1/h2 post-ReLU.
__device__ __forceinline__ float Forward(const float *p, const float *x, float *h1, float *h2)
{
    for (int i = 0; i < kH; ++i) {
        float acc = p[kOffB1 + i];
        for (int j = 0; j < kIn; ++j)
            acc = fmaf(p[kOffW1 + i * kIn + j], x[j], acc);
        h1[i] = fmaxf(acc, 0.0f);
    }
    for (int i = 0; i < kH; ++i) {
        float acc = p[kOffB2 + i];
        for (int j = 0; j < kH; ++j)
            acc = fmaf(p[kOffW2 + i * kH + j], h1[j], acc);
        h2[i] = fmaxf(acc, 0.0f);
    }
    float y = p[kOffB3];
    for (int j = 0; j < kH; ++j)
        y = fmaf(p[kOffW3 + j], h2[j], y);
    return y;
}

} // namespace bm25mlp
