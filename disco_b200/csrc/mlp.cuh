// Shape, parameter layout and activation of the learned far-image surrogate's
// network (14 -> 128 -> 128 -> 128 -> 3, SiLU), shared by its training kernels
// (mlp.cu) and its fused inference kernel (far.cu).
#pragma once

#include <cstdint>

#include <cuda_bf16.h>

namespace disco {
namespace mlp {

constexpr int kIn = 16, kHid = 128, kOut = 16;       // padded widths
constexpr int kInReal = 14, kOutReal = 3;
// parameter offsets (floats): W1 [128 x 16], b1, W2 [128 x 128], b2, W3, b3, W4 [16 x 128], b4
constexpr int oW1 = 0, ob1 = oW1 + kHid * kIn, oW2 = ob1 + kHid, ob2 = oW2 + kHid * kHid;
constexpr int oW3 = ob2 + kHid, ob3 = oW3 + kHid * kHid, oW4 = ob3 + kHid, ob4 = oW4 + kOut * kHid;
constexpr int kParams = ob4 + kOut;                  // 37 264

// SiLU(x) = x sigmoid(x) = u + u tanh(u) with u = x / 2, one MUFU tanh.
__device__ __forceinline__ float tanh_approx(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float silu_half(float u) { return fmaf(u, tanh_approx(u), u); }

// d SiLU / dx = s (1 + x (1 - s)), s = sigmoid(x) = (1 + tanh(x / 2)) / 2
__device__ __forceinline__ float dsilu(float x)
{
    const float s = fmaf(0.5f, tanh_approx(0.5f * x), 0.5f);
    return s * fmaf(x, 1.0f - s, 1.0f);
}

} // namespace mlp
} // namespace disco

struct disco_mlp {
    float* params = nullptr;   // FP32 master weights (device)
    float* grads = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    float* loss = nullptr;     // device scalar
    int64_t cap = 0;           // rows of the workspace below
    float *pre1 = nullptr, *pre2 = nullptr, *pre3 = nullptr, *y = nullptr, *dy = nullptr, *dpre = nullptr;
    __nv_bfloat16 *h1 = nullptr, *h2 = nullptr, *h3 = nullptr, *dpre_h = nullptr;
    int64_t step = 0;
    int* status = nullptr;
    unsigned char* packed = nullptr;   // inference image of the weights (far.cu)
};
