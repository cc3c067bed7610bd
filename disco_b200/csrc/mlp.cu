// The learned far-image surrogate's network: 14 -> 128 -> 128 -> 128 -> 3,
// SiLU, BF16 weights and activations on the tensor cores, FP32 accumulation,
// FP32 master weights and Adam.  Every matrix product, forward and backward,
// runs through one hand-written tcgen05 GEMM kernel:
//
//     C[M x N] = A[M x K] * B[N x K]^T        (BF16 x BF16 -> FP32 in TMEM)
//
// A and B are read from global memory (FP32 or BF16, stored as given or
// transposed) and written into shared memory in the no-swizzle K-major
// layout of tcgen05.cuh, converting to BF16 on the way; one elected thread
// issues the MMAs (K = 16 each) and commits them to an mbarrier; four warps
// read the accumulator back with tcgen05.ld (warp w owns rows 32w..32w+31)
// and apply a fused epilogue.  Transposed operands (dW = dpre^T h,
// dh = dpre W) are transposed by the loader, so every descriptor is K-major.
//
// Inputs are padded to 16 features and outputs to 16 (the MMA's N >= 16 for
// M = 128); the padding columns of W1 and rows of W4 are zero and stay zero
// (their gradients are masked).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "mlp.cuh"
#include "tcgen05.cuh"

namespace disco {
namespace mlp {

enum { kF32 = 0, kBF16 = 1 };
enum { EPI_STORE = 0, EPI_SILU = 1, EPI_DSILU = 2, EPI_ATOMIC = 3, EPI_ATOMIC_T = 4 };

struct Operand {
    const void* ptr;
    int32_t dtype;        // kF32 or kBF16
    int32_t transposed;   // 0: element (r, k) at r*ld + k; 1: at k*ld + r
    int64_t ld;
};

struct GemmArgs {
    Operand A, B;
    int32_t M, N, K;
    int32_t k_per_split;  // split-K: blockIdx.z takes K range [z*k_per_split, ...)
    int32_t epi;
    float* C;             // FP32 output (pre-activation, dpre, raw result or gradient)
    int64_t ldc;
    __nv_bfloat16* H;     // BF16 output (activation or dpre)
    int64_t ldh;
    const float* bias;    // per output column (EPI_STORE / EPI_SILU)
    const float* pre;     // EPI_DSILU: pre-activations
    int64_t ldp;
    int32_t n_valid;      // EPI_ATOMIC*: columns >= n_valid are not accumulated
    int32_t m_valid;      // EPI_ATOMIC*: rows >= m_valid are not accumulated
    int* status;
};

constexpr int kThreads = 128;
constexpr int kTileM = 128, kTileK = 128;

__device__ __forceinline__ float load_elem(const Operand& o, int64_t r, int64_t k)
{
    const int64_t idx = o.transposed ? k * o.ld + r : r * o.ld + k;
    return o.dtype == kF32 ? static_cast<const float*>(o.ptr)[idx]
                           : __bfloat162float(static_cast<const __nv_bfloat16*>(o.ptr)[idx]);
}

__device__ __forceinline__ uint32_t bf16x2(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// 8 consecutive elements (along the row in memory) at p as 8 floats
__device__ __forceinline__ void load8(const Operand& o, int64_t idx, float* v)
{
    if (o.dtype == kF32) {
        const float4* q = reinterpret_cast<const float4*>(static_cast<const float*>(o.ptr) + idx);
        const float4 a = q[0], b = q[1];
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    } else {
        const uint4 u = *reinterpret_cast<const uint4*>(static_cast<const __nv_bfloat16*>(o.ptr) + idx);
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 f = __bfloat1622float2(h[i]);
            v[2 * i] = f.x;
            v[2 * i + 1] = f.y;
        }
    }
}

// Whole tile in range and 16-byte aligned along memory rows: 8-element vector
// loads, and 16-byte shared stores of 8 K-consecutive values (transposed
// operands: 8 x 8 blocks transposed in registers).  Rows vary fastest across
// threads, so the stores of a warp fill whole 128-byte core matrices.
__device__ __forceinline__ bool tile_fast(const Operand& o, int rows, int64_t r0, int64_t rmax, int64_t k0, int kc,
                                          int64_t kmax)
{
    const int esz = o.dtype == kF32 ? 4 : 2;
    const bool in = r0 + rows <= rmax && k0 + kc <= kmax && (kc % 8) == 0;
    const bool al = ((reinterpret_cast<uintptr_t>(o.ptr) & 15) == 0) && ((o.ld * esz) % 16 == 0) &&
                    (((o.transposed ? r0 : k0) * esz) % 16 == 0);
    return in && al;
}

__device__ __forceinline__ void load_tile_fast(const Operand& o, unsigned char* base, int rows, int64_t r0,
                                               int64_t k0, int kc)
{
    if (!o.transposed) {
        const int total = rows * (kc / 8);
        for (int e = threadIdx.x; e < total; e += kThreads) {
            const int r = e % rows, k8 = (e / rows) * 8;
            float v[8];
            load8(o, (r0 + r) * o.ld + k0 + k8, v);
            *reinterpret_cast<uint4*>(base + tc::kmajor_offset(r, k8, rows)) =
                make_uint4(bf16x2(v[0], v[1]), bf16x2(v[2], v[3]), bf16x2(v[4], v[5]), bf16x2(v[6], v[7]));
        }
    } else {
        const int total = (rows / 8) * (kc / 8);
        for (int e = threadIdx.x; e < total; e += kThreads) {
            const int r8 = (e % (rows / 8)) * 8, k8 = (e / (rows / 8)) * 8;
            float v[8][8];                   // v[k][r]
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) load8(o, (k0 + k8 + kk) * o.ld + r0 + r8, v[kk]);
#pragma unroll
            for (int rr = 0; rr < 8; ++rr)
                *reinterpret_cast<uint4*>(base + tc::kmajor_offset(r8 + rr, k8, rows)) =
                    make_uint4(bf16x2(v[0][rr], v[1][rr]), bf16x2(v[2][rr], v[3][rr]), bf16x2(v[4][rr], v[5][rr]),
                               bf16x2(v[6][rr], v[7][rr]));
        }
    }
}

// rows x kc tile of an operand into shared memory (K-major, BF16), zero-padded
__device__ __forceinline__ void load_tile(const Operand& o, __nv_bfloat16* smem, int rows, int64_t r0, int64_t rmax,
                                          int64_t k0, int kc, int64_t kmax)
{
    unsigned char* base = reinterpret_cast<unsigned char*>(smem);
    if (tile_fast(o, rows, r0, rmax, k0, kc, kmax)) {
        load_tile_fast(o, base, rows, r0, k0, kc);
        return;
    }
    const int total = rows * kc;
    if (!o.transposed) {
        for (int e = threadIdx.x; e < total; e += kThreads) {
            const int r = e / kc, k = e % kc;
            const float v = (r0 + r < rmax && k0 + k < kmax) ? load_elem(o, r0 + r, k0 + k) : 0.0f;
            *reinterpret_cast<__nv_bfloat16*>(base + tc::kmajor_offset(r, k, rows)) = __float2bfloat16_rn(v);
        }
    } else {
        for (int e = threadIdx.x; e < total; e += kThreads) {
            const int k = e / rows, r = e % rows;
            const float v = (r0 + r < rmax && k0 + k < kmax) ? load_elem(o, r0 + r, k0 + k) : 0.0f;
            *reinterpret_cast<__nv_bfloat16*>(base + tc::kmajor_offset(r, k, rows)) = __float2bfloat16_rn(v);
        }
    }
}


template <int NT>
__global__ void __launch_bounds__(kThreads) gemm_kernel(const GemmArgs g)
{
    extern __shared__ __align__(128) unsigned char gemm_smem[];
    __nv_bfloat16* sA = reinterpret_cast<__nv_bfloat16*>(gemm_smem);
    __nv_bfloat16* sB = sA + kTileM * kTileK;
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    constexpr uint32_t kCols = NT < 32 ? 32 : NT;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t m0 = (int64_t)blockIdx.x * kTileM;
    const int64_t n0 = (int64_t)blockIdx.y * NT;
    const int64_t kbeg = (int64_t)blockIdx.z * g.k_per_split;
    const int64_t kend = ((int64_t)g.K < kbeg + g.k_per_split) ? (int64_t)g.K : kbeg + g.k_per_split;
    if (warp == 0) tc::alloc(&tmem_slot, kCols);
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = tc::idesc_bf16(kTileM, NT);
    const uint32_t lboA = (kTileM / 8) * 128, lboB = (NT / 8) * 128;
    uint32_t phase = 0;
    bool ok = true;
    for (int64_t kk = kbeg; kk < kend; kk += kTileK) {
        const int64_t rem = ((kend - kk + 15) / 16) * 16;
        const int kc = (int)(rem < kTileK ? rem : kTileK);
        load_tile(g.A, sA, kTileM, m0, g.M, kk, kc, kend);
        load_tile(g.B, sB, NT, n0, g.N, kk, kc, kend);
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc::fence_after_sync();
            const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sB);
            for (int j = 0; j < kc / 16; ++j) {
                const uint64_t ad = tc::smem_desc(a0 + j * 2 * lboA, lboA, 128);
                const uint64_t bd = tc::smem_desc(b0 + j * 2 * lboB, lboB, 128);
                tc::mma_bf16(tmem, ad, bd, idesc, kk > kbeg || j > 0);
            }
            tc::commit(&bar);
        }
        const bool mine = mbar_wait_bounded(&bar, phase);
        phase ^= 1;
        if (__syncthreads_or(!mine)) { ok = false; break; }     // every thread agrees
        tc::fence_after_sync();
    }
    if (ok) {
        const int64_t row = m0 + warp * 32 + lane;
        const bool rvalid = row < g.M && kend > kbeg;
        for (int c = 0; c < NT; c += 16) {
            float v[16];
            tc::ld16(tmem + ((uint32_t)(warp * 32) << 16) + c, v);
            if (!rvalid) continue;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int64_t col = n0 + c + i;
                if (col >= g.N) continue;
                float x = v[i];
                switch (g.epi) {
                case EPI_STORE:
                    if (g.bias) x += g.bias[col];
                    g.C[row * g.ldc + col] = x;
                    break;
                case EPI_SILU: {
                    if (g.bias) x += g.bias[col];
                    g.C[row * g.ldc + col] = x;
                    g.H[row * g.ldh + col] = __float2bfloat16_rn(silu_half(0.5f * x));
                    break;
                }
                case EPI_DSILU: {
                    const float p = g.pre[row * g.ldp + col];
                    const float d = x * dsilu(p);
                    g.C[row * g.ldc + col] = d;
                    g.H[row * g.ldh + col] = __float2bfloat16_rn(d);
                    break;
                }
                case EPI_ATOMIC:
                    if (row < g.m_valid && col < g.n_valid) atomicAdd(&g.C[row * g.ldc + col], x);
                    break;
                default:   // EPI_ATOMIC_T: C^T += D
                    if (row < g.m_valid && col < g.n_valid) atomicAdd(&g.C[col * g.ldc + row], x);
                    break;
                }
            }
        }
    } else if (threadIdx.x == 0) {
        report(g.status, DISCO_ETIMEOUT);
        mbar_wait_bounded(&bar, phase ^ 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::dealloc(tmem, kCols);
}

// dy = 2 (y - t) / n on the real outputs (0 on padding); loss += sum (y - t)^2 / n
__global__ void mse_grad_kernel(const float* y, const float* t, int64_t n, float* dy, float* loss)
{
    float acc = 0.0f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * kOut;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / kOut;
        const int c = (int)(i % kOut);
        float g = 0.0f;
        if (c < kOutReal) {
            const float d = y[i] - t[r * kOutReal + c];
            acc += d * d;
            g = 2.0f * d / (float)n;
        }
        dy[i] = g;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc / (float)n);
}

// grad[col] += sum over rows of x[row * ld + col] (cols < n_valid)
__global__ void colsum_kernel(const float* x, int64_t rows, int cols, int64_t ld, int n_valid, float* grad)
{
    const int col = blockIdx.x;
    float acc = 0.0f;
    for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) acc += x[r * ld + col];
    __shared__ float part[32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        float s = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0 && col < n_valid) grad[col] += s;
    }
    (void)cols;
}

__global__ void adam_kernel(float* p, float* g, float* m, float* v, int n, float lr, float b1, float b2,
                            float eps, float bc1, float bc2, float wd)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float upd = (mi / bc1) / (sqrtf(vi / bc2) + eps) + wd * p[i];
    p[i] -= lr * upd;
    g[i] = 0.0f;
}

} // namespace mlp
} // namespace disco

// ---- host ---------------------------------------------------------------------------------


namespace {

using namespace disco::mlp;

int mfail(int code, const std::string& msg)
{
    disco::set_last_error(msg);
    return code;
}

int mcuda(cudaError_t e, const char* what)
{
    disco::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? DISCO_ENOMEM : DISCO_ECUDA;
}

Operand op(const void* p, int dtype, int transposed, int64_t ld) { return Operand{ p, dtype, transposed, ld }; }

// One GEMM launch; split > 1 splits K over blockIdx.z (EPI_ATOMIC* only).
int gemm(const Operand& A, const Operand& B, int M, int N, int K, int epi, float* C, int64_t ldc,
         __nv_bfloat16* H, int64_t ldh, const float* bias, const float* pre, int64_t ldp, int split,
         int n_valid, int m_valid, int* status, cudaStream_t s)
{
    GemmArgs g;
    std::memset(&g, 0, sizeof(g));
    g.A = A; g.B = B; g.M = M; g.N = N; g.K = K;
    g.k_per_split = split > 1 ? (int)(((K + split - 1) / split + kTileK - 1) / kTileK * kTileK) : K;
    g.epi = epi; g.C = C; g.ldc = ldc; g.H = H; g.ldh = ldh; g.bias = bias; g.pre = pre; g.ldp = ldp;
    g.n_valid = n_valid; g.m_valid = m_valid; g.status = status;
    const int zs = (int)((K + g.k_per_split - 1) / g.k_per_split);
    if (N == 16) {
        const size_t smem = (size_t)(kTileM + 16) * kTileK * sizeof(__nv_bfloat16);
        cudaFuncSetAttribute(gemm_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        dim3 grid((M + kTileM - 1) / kTileM, 1, zs);
        gemm_kernel<16><<<grid, kThreads, smem, s>>>(g);
    } else if (N % 128 == 0) {
        const size_t smem = (size_t)(kTileM + 128) * kTileK * sizeof(__nv_bfloat16);
        cudaFuncSetAttribute(gemm_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        dim3 grid((M + kTileM - 1) / kTileM, N / 128, zs);
        gemm_kernel<128><<<grid, kThreads, smem, s>>>(g);
    } else {
        return mfail(DISCO_EINVAL, "GEMM N must be 16 or a multiple of 128");
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DISCO_OK : mcuda(e, "gemm launch");
}

void free_mlp(disco_mlp* p)
{
    if (!p) return;
    float* fs[] = { p->params, p->grads, p->m, p->v, p->loss, p->pre1, p->pre2, p->pre3, p->y, p->dy, p->dpre };
    for (float* f : fs) if (f) cudaFree(f);
    __nv_bfloat16* hs[] = { p->h1, p->h2, p->h3, p->dpre_h };
    for (auto* h : hs) if (h) cudaFree(h);
    if (p->status) cudaFree(p->status);
    if (p->packed) cudaFree(p->packed);
    delete p;
}

int ensure_workspace(disco_mlp* p, int64_t n)
{
    if (n <= p->cap) return DISCO_OK;
    float** fs[] = { &p->pre1, &p->pre2, &p->pre3, &p->dpre };
    for (float** f : fs) { if (*f) cudaFree(*f); *f = nullptr; }
    if (p->y) cudaFree(p->y);
    if (p->dy) cudaFree(p->dy);
    __nv_bfloat16** hs[] = { &p->h1, &p->h2, &p->h3, &p->dpre_h };
    for (auto** h : hs) { if (*h) cudaFree(*h); *h = nullptr; }
    p->y = p->dy = nullptr;
    cudaError_t e = cudaSuccess;
    for (float** f : fs) if (e == cudaSuccess) e = cudaMalloc(f, (size_t)n * kHid * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->y, (size_t)n * kOut * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->dy, (size_t)n * kOut * sizeof(float));
    for (auto** h : hs) if (e == cudaSuccess) e = cudaMalloc(h, (size_t)n * kHid * sizeof(__nv_bfloat16));
    if (e != cudaSuccess) { p->cap = 0; return mcuda(e, "MLP workspace"); }
    p->cap = n;
    return DISCO_OK;
}

// Forward over n rows of X [n x 16] (FP32): fills pre1..3, h1..3 and y [n x 16].
int forward(disco_mlp* p, const float* X, int64_t n, cudaStream_t s)
{
    const float* P = p->params;
    int st = gemm(op(X, kF32, 0, kIn), op(P + oW1, kF32, 0, kIn), (int)n, kHid, kIn, EPI_SILU,
                  p->pre1, kHid, p->h1, kHid, P + ob1, nullptr, 0, 1, 0, 0, p->status, s);
    if (!st) st = gemm(op(p->h1, kBF16, 0, kHid), op(P + oW2, kF32, 0, kHid), (int)n, kHid, kHid, EPI_SILU,
                       p->pre2, kHid, p->h2, kHid, P + ob2, nullptr, 0, 1, 0, 0, p->status, s);
    if (!st) st = gemm(op(p->h2, kBF16, 0, kHid), op(P + oW3, kF32, 0, kHid), (int)n, kHid, kHid, EPI_SILU,
                       p->pre3, kHid, p->h3, kHid, P + ob3, nullptr, 0, 1, 0, 0, p->status, s);
    if (!st) st = gemm(op(p->h3, kBF16, 0, kHid), op(P + oW4, kF32, 0, kHid), (int)n, kOut, kHid, EPI_STORE,
                       p->y, kOut, nullptr, 0, P + ob4, nullptr, 0, 1, 0, 0, p->status, s);
    return st;
}

// Backward of the MSE loss after forward(): accumulates into p->grads.
int backward(disco_mlp* p, const float* X, const float* T, int64_t n, cudaStream_t s)
{
    const float* P = p->params;
    float* G = p->grads;
    const int nb = (int)std::min<int64_t>(1024, (n * kOut + 255) / 256);
    mse_grad_kernel<<<nb, 256, 0, s>>>(p->y, T, n, p->dy, p->loss);
    const int split = (int)std::max<int64_t>(1, std::min<int64_t>(64, n / kTileK));
    const int N = (int)n;
    // layer 4: dW4^T = h3^T dy, db4, dh3 = dy W4 -> dpre3
    int st = gemm(op(p->h3, kBF16, 1, kHid), op(p->dy, kF32, 1, kOut), kHid, kOut, N, EPI_ATOMIC_T,
                  G + oW4, kHid, nullptr, 0, nullptr, nullptr, 0, split, kOutReal, kHid, p->status, s);
    if (!st) { colsum_kernel<<<kOut, 256, 0, s>>>(p->dy, n, kOut, kOut, kOutReal, G + ob4); }
    if (!st) st = gemm(op(p->dy, kF32, 0, kOut), op(P + oW4, kF32, 1, kHid), N, kHid, kOut, EPI_DSILU,
                       p->dpre, kHid, p->dpre_h, kHid, nullptr, p->pre3, kHid, 1, 0, 0, p->status, s);
    // layer 3
    if (!st) st = gemm(op(p->dpre_h, kBF16, 1, kHid), op(p->h2, kBF16, 1, kHid), kHid, kHid, N, EPI_ATOMIC,
                       G + oW3, kHid, nullptr, 0, nullptr, nullptr, 0, split, kHid, kHid, p->status, s);
    if (!st) { colsum_kernel<<<kHid, 256, 0, s>>>(p->dpre, n, kHid, kHid, kHid, G + ob3); }
    if (!st) st = gemm(op(p->dpre_h, kBF16, 0, kHid), op(P + oW3, kF32, 1, kHid), N, kHid, kHid, EPI_DSILU,
                       p->dpre, kHid, p->h3, kHid, nullptr, p->pre2, kHid, 1, 0, 0, p->status, s);
    // (h3 is free now and holds dpre2 in BF16)
    if (!st) st = gemm(op(p->h3, kBF16, 1, kHid), op(p->h1, kBF16, 1, kHid), kHid, kHid, N, EPI_ATOMIC,
                       G + oW2, kHid, nullptr, 0, nullptr, nullptr, 0, split, kHid, kHid, p->status, s);
    if (!st) { colsum_kernel<<<kHid, 256, 0, s>>>(p->dpre, n, kHid, kHid, kHid, G + ob2); }
    if (!st) st = gemm(op(p->h3, kBF16, 0, kHid), op(P + oW2, kF32, 1, kHid), N, kHid, kHid, EPI_DSILU,
                       p->dpre, kHid, p->dpre_h, kHid, nullptr, p->pre1, kHid, 1, 0, 0, p->status, s);
    // layer 1: dW1 = dpre1^T X (input padding columns masked), db1
    if (!st) st = gemm(op(p->dpre_h, kBF16, 1, kHid), op(X, kF32, 1, kIn), kHid, kIn, N, EPI_ATOMIC,
                       G + oW1, kIn, nullptr, 0, nullptr, nullptr, 0, split, kInReal, kHid, p->status, s);
    if (!st) { colsum_kernel<<<kHid, 256, 0, s>>>(p->dpre, n, kHid, kHid, kHid, G + ob1); }
    if (!st) {
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = mcuda(e, "MLP backward");
    }
    return st;
}

} // namespace

extern "C" {

int disco_b200_mlp_create(uint64_t seed, disco_mlp** out)
{
    if (!out) return mfail(DISCO_EINVAL, "null out");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return mfail(DISCO_ENODEV, "no CUDA device");
    disco_mlp* p = new disco_mlp();
    cudaError_t e = cudaSuccess;
    float** bufs[] = { &p->params, &p->grads, &p->m, &p->v };
    for (float** b : bufs) if (e == cudaSuccess) e = cudaMalloc(b, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->status, sizeof(int));
    if (e != cudaSuccess) { free_mlp(p); return mcuda(e, "MLP allocation"); }
    // Kaiming-uniform weights (a SplitMix64 stream), zero biases and padding
    std::vector<float> h(kParams, 0.0f);
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
    auto next = [&]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int rows, int cols, int rows_real, int cols_real) {
        const double bound = std::sqrt(6.0 / cols_real);
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c)
                h[off + r * cols + c] = (r < rows_real && c < cols_real) ? (float)((2.0 * next() - 1.0) * bound) : 0.0f;
    };
    fill(oW1, kHid, kIn, kHid, kInReal);
    fill(oW2, kHid, kHid, kHid, kHid);
    fill(oW3, kHid, kHid, kHid, kHid);
    fill(oW4, kOut, kHid, kOutReal, kHid);
    e = cudaMemcpy(p->params, h.data(), kParams * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(p->grads, 0, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(p->m, 0, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(p->v, 0, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(p->status, 0, sizeof(int));
    if (e != cudaSuccess) { free_mlp(p); return mcuda(e, "MLP init"); }
    *out = p;
    return DISCO_OK;
}

int disco_b200_mlp_destroy(disco_mlp* p)
{
    free_mlp(p);
    return DISCO_OK;
}

int disco_b200_mlp_param_count(void) { return kParams; }

int disco_b200_mlp_get_params(const disco_mlp* p, float* host)
{
    if (!p || !host) return mfail(DISCO_EINVAL, "null argument");
    const cudaError_t e = cudaMemcpy(host, p->params, kParams * sizeof(float), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? DISCO_OK : mcuda(e, "params download");
}

int disco_b200_mlp_set_params(disco_mlp* p, const float* host)
{
    if (!p || !host) return mfail(DISCO_EINVAL, "null argument");
    const cudaError_t e = cudaMemcpy(p->params, host, kParams * sizeof(float), cudaMemcpyHostToDevice);
    return e == cudaSuccess ? DISCO_OK : mcuda(e, "params upload");
}

int disco_b200_mlp_get_grads(const disco_mlp* p, float* host)
{
    if (!p || !host) return mfail(DISCO_EINVAL, "null argument");
    const cudaError_t e = cudaMemcpy(host, p->grads, kParams * sizeof(float), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? DISCO_OK : mcuda(e, "grads download");
}

int disco_b200_mlp_forward(disco_mlp* p, const float* X, int64_t n, float* Y, void* stream)
{
    if (!p || n < 0 || (n > 0 && (!X || !Y))) return mfail(DISCO_EINVAL, "bad argument");
    if (n == 0) return DISCO_OK;
    int st = ensure_workspace(p, n);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    st = forward(p, X, n, s);
    if (st) return st;
    const cudaError_t e = cudaMemcpyAsync(Y, p->y, (size_t)n * kOut * sizeof(float), cudaMemcpyDeviceToDevice, s);
    return e == cudaSuccess ? DISCO_OK : mcuda(e, "forward output");
}

// Forward + backward of the MSE loss over n rows; gradients accumulate in the
// model (zeroed by disco_b200_mlp_adam); *loss = mean squared error.
int disco_b200_mlp_grad(disco_mlp* p, const float* X, const float* T, int64_t n, float* loss, void* stream)
{
    if (!p || n <= 0 || !X || !T) return mfail(DISCO_EINVAL, "bad argument");
    int st = ensure_workspace(p, n);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(p->loss, 0, sizeof(float), s);
    if (e != cudaSuccess) return mcuda(e, "loss reset");
    st = forward(p, X, n, s);
    if (!st) st = backward(p, X, T, n, s);
    if (st) return st;
    if (loss) {
        e = cudaMemcpyAsync(loss, p->loss, sizeof(float), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return mcuda(e, "loss read");
    }
    return DISCO_OK;
}

int disco_b200_mlp_adam(disco_mlp* p, float lr, float beta1, float beta2, float eps, float weight_decay,
                        void* stream)
{
    if (!p) return mfail(DISCO_EINVAL, "null model");
    p->step++;
    const float bc1 = 1.0f - std::pow(beta1, (float)p->step), bc2 = 1.0f - std::pow(beta2, (float)p->step);
    adam_kernel<<<(kParams + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        p->params, p->grads, p->m, p->v, kParams, lr, beta1, beta2, eps, bc1, bc2, weight_decay);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DISCO_OK : mcuda(e, "adam");
}

int disco_b200_mlp_status(disco_mlp* p)
{
    if (!p) return mfail(DISCO_EINVAL, "null model");
    int st = 0;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&st, p->status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return mcuda(e, "status");
    if (st) { cudaMemset(p->status, 0, sizeof(int)); return mfail(st, "an MLP kernel's bounded wait gave up"); }
    return DISCO_OK;
}

} // extern "C"
