// Learned far-image surrogate: the network's features, its fused tcgen05
// inference kernel and the learned displacement (exact near images, network
// far shells, exact re-check on a random atom subsample with per-loop
// fallback).  The reference has no learned path; the exact sums it is checked
// against and falls back to are the plan and batch forms of this library.
//
// Fused inference (far_kernel): one CTA of 256 threads owns a tile of 128 atoms
// (row r = tensor-memory lane r; warps w and w + 4 read the same lanes and
// split the 128 columns of each epilogue) and walks the selected loops.  Per
// (tile, loop): the 16 features of each row go to shared memory as one BF16
// K-major A tile; layer 1 is one 128x128x16 MMA, layers 2 and 3 eight MMAs of
// K = 16 reading the previous activations from shared memory, layer 4 eight
// MMAs of N = 16.  Accumulators live in 128 tensor-memory columns; each
// epilogue (tcgen05.ld, bias, SiLU with one MUFU tanh, BF16 pack) writes the
// next A tile in place.  The weights (72 KB BF16, with layers 1-3 pre-halved so
// that the accumulator is u = x / 2 of SiLU(x) = u + u tanh(u)) are staged
// once per CTA by a bulk async copy.  About 110 KB of shared memory: two CTAs
// per SM, so one CTA's epilogue overlaps the other's MMAs.
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
namespace far {

using namespace disco::mlp;

struct FarLoop {
    double cx, cy, cz;   // loop centre (fan apex)
    float feat[11];      // features 3..13 (standardised)
    float gain;          // displacement (A) per unit network output
};

struct FeatNorm {
    double iLx, iLy, iLz;   // 1 / box lengths
    float mu[3], isd[3];    // standardisation of features 0..2
};

// byte offsets of the packed inference image
constexpr uint32_t kImgW1 = 0;                                  // [128 x 16]  K-major, halved
constexpr uint32_t kImgW2 = kImgW1 + kHid * kIn * 2;            // [128 x 128] K-major, halved
constexpr uint32_t kImgW3 = kImgW2 + kHid * kHid * 2;
constexpr uint32_t kImgW4 = kImgW3 + kHid * kHid * 2;           // [16 x 128]  K-major
constexpr uint32_t kImgBias = kImgW4 + kOut * kHid * 2;         // b1/2, b2/2, b3/2, b4 (FP32)
constexpr uint32_t kImgBytes = kImgBias + (3 * kHid + kOut) * 4;
static_assert(kImgBytes % 16 == 0, "bulk copies move multiples of 16 bytes");

constexpr int kFarThreads = 256;      // two threads per row: warps w and w + 4 split the columns
constexpr uint32_t kSmX = (kImgBytes + 127) / 128 * 128;       // features tile [128 x 16]
constexpr uint32_t kSmH = kSmX + 128 * kIn * 2;                 // activations [128 x 128]
constexpr uint32_t kSmBar = kSmH + 128 * kHid * 2;
constexpr uint32_t kSmTotal = kSmBar + 32;
constexpr uint32_t kTmemCols = 128;

struct FarArgs {
    const double *x, *y, *z;
    double *ux, *uy, *uz;
    int64_t n;
    const FarLoop* loops;
    const int32_t* sel;
    int32_t nsel, ntiles;
    float* per_loop;
    const unsigned char* image;
    FeatNorm fn;
    int* status;
};

__device__ __forceinline__ void features(double px, double py, double pz, const FarLoop& L, const FeatNorm& fn,
                                         float* f)
{
    f[0] = ((float)((px - L.cx) * fn.iLx) - fn.mu[0]) * fn.isd[0];
    f[1] = ((float)((py - L.cy) * fn.iLy) - fn.mu[1]) * fn.isd[1];
    f[2] = ((float)((pz - L.cz) * fn.iLz) - fn.mu[2]) * fn.isd[2];
#pragma unroll
    for (int k = 0; k < 11; ++k) f[3 + k] = L.feat[k];
    f[14] = 0.0f;
    f[15] = 0.0f;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// Raw or standardised features of every (selected loop, atom) pair, loop-major.
__global__ void features_kernel(const double* x, const double* y, const double* z, int64_t n,
                                const FarLoop* loops, int32_t nloops, FeatNorm fn, float* X)
{
    const int64_t total = n * nloops;
    for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < total;
         row += (int64_t)gridDim.x * blockDim.x) {
        const int64_t l = row / n, i = row % n;
        float f[16];
        features(x[i], y[i], z[i], loops[l], fn, f);
        float4* o = reinterpret_cast<float4*>(X + row * 16);
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] = make_float4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
    }
}

// FP32 master parameters -> the inference image (BF16 K-major weights, FP32 biases).
__global__ void pack_kernel(const float* P, unsigned char* img)
{
    float* bias = reinterpret_cast<float*>(img + kImgBias);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) {
        const float v = P[i];
        if (i < ob1) {
            const int r = (i - oW1) / kIn, k = (i - oW1) % kIn;
            *reinterpret_cast<__nv_bfloat16*>(img + kImgW1 + tc::kmajor_offset(r, k, kHid)) = __float2bfloat16_rn(0.5f * v);
        } else if (i < oW2) {
            bias[i - ob1] = 0.5f * v;
        } else if (i < ob2) {
            const int r = (i - oW2) / kHid, k = (i - oW2) % kHid;
            *reinterpret_cast<__nv_bfloat16*>(img + kImgW2 + tc::kmajor_offset(r, k, kHid)) = __float2bfloat16_rn(0.5f * v);
        } else if (i < oW3) {
            bias[kHid + i - ob2] = 0.5f * v;
        } else if (i < ob3) {
            const int r = (i - oW3) / kHid, k = (i - oW3) % kHid;
            *reinterpret_cast<__nv_bfloat16*>(img + kImgW3 + tc::kmajor_offset(r, k, kHid)) = __float2bfloat16_rn(0.5f * v);
        } else if (i < oW4) {
            bias[2 * kHid + i - ob3] = 0.5f * v;
        } else if (i < ob4) {
            const int r = (i - oW4) / kHid, k = (i - oW4) % kHid;
            *reinterpret_cast<__nv_bfloat16*>(img + kImgW4 + tc::kmajor_offset(r, k, kOut)) = __float2bfloat16_rn(v);
        } else {
            bias[3 * kHid + i - ob4] = v;
        }
    }
}

// Every thread: publish this thread's shared-memory tile writes and finished
// tensor-memory loads, then one thread issues nk MMAs of K = 16 and commits;
// all wait (bounded).  Returns false, agreed by the whole CTA, on a timeout.
__device__ __forceinline__ bool mma_step(uint32_t tmem, uint32_t a_addr, uint32_t a_lbo, uint32_t b_addr,
                                         uint32_t b_lbo, int nk, uint32_t idesc, uint64_t* bar, uint32_t& phase)
{
    fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc::fence_after_sync();
        for (int j = 0; j < nk; ++j)
            tc::mma_bf16(tmem, tc::smem_desc(a_addr + j * 2 * a_lbo, a_lbo, 128),
                         tc::smem_desc(b_addr + j * 2 * b_lbo, b_lbo, 128), idesc, j > 0);
        tc::commit(bar);
    }
    const bool mine = mbar_wait_bounded(bar, phase);
    phase ^= 1;
    const bool bad = __syncthreads_or(!mine);
    tc::fence_after_sync();
    return !bad;
}

// Hidden-layer epilogue of row `row`, columns [c0, c0 + 64): H[row, c] =
// SiLU(acc + b) in BF16 (acc and bh hold halves: h = u + u tanh(u)).
__device__ __forceinline__ void epilogue_hidden(uint32_t taddr, const float* bh, unsigned char* H, int row, int c0)
{
#pragma unroll 1
    for (int c = c0; c < c0 + kHid / 2; c += 32) {
        float v[32];
        tc::ld32(taddr + c, v);
        uint32_t w[16];
#pragma unroll
        for (int i = 0; i < 16; ++i)
            w[i] = pack_bf16(silu_half(v[2 * i] + bh[c + 2 * i]), silu_half(v[2 * i + 1] + bh[c + 2 * i + 1]));
#pragma unroll
        for (int q = 0; q < 4; ++q)
            *reinterpret_cast<uint4*>(H + tc::kmajor_offset(row, c + 8 * q, 128)) =
                make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
    }
}

__global__ void __launch_bounds__(kFarThreads, 2) far_kernel(const FarArgs a)
{
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kSmBar);    // [0] weights, [1] MMAs
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kSmBar + 16);
    const int t = threadIdx.x, warp = t >> 5;
    if (warp == 0) tc::alloc(tslot, kTmemCols);
    if (t == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    if (t == 0) stage_load(sm, a.image, kImgBytes, &bar[0]);
    bool ok = !__syncthreads_or(!mbar_wait_bounded(&bar[0], 0));
    if (!ok && t == 0) {
        report(a.status, DISCO_ETIMEOUT);
        mbar_wait_bounded(&bar[0], 0);
    }

    const float* bias = reinterpret_cast<const float*>(sm + kImgBias);
    unsigned char* X = sm + kSmX;
    unsigned char* H = sm + kSmH;
    const uint32_t aW1 = smem_addr(sm + kImgW1), aW2 = smem_addr(sm + kImgW2), aW3 = smem_addr(sm + kImgW3),
                   aW4 = smem_addr(sm + kImgW4), aX = smem_addr(X), aH = smem_addr(H);
    constexpr uint32_t lbo128 = (128 / 8) * 128, lbo16 = (16 / 8) * 128;
    const uint32_t id_hid = tc::idesc_bf16(128, kHid), id_out = tc::idesc_bf16(128, kOut);
    // warp w reads tensor-memory lanes 32 (w % 4) ...; warps 0-3 (half 0) own
    // the rows' features and outputs, both halves share the epilogues
    const int row = t & 127, half = t >> 7;
    const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    uint32_t phase = 0;

    for (int tile = blockIdx.x; ok && tile < a.ntiles; tile += gridDim.x) {
        const int64_t atom = (int64_t)tile * 128 + row;
        const bool valid = atom < a.n;
        double px = 0.0, py = 0.0, pz = 0.0;
        if (half == 0) {
            const int64_t ia = valid ? atom : a.n - 1;
            px = a.x[ia]; py = a.y[ia]; pz = a.z[ia];
        }
        float sx = 0.0f, sy = 0.0f, sz = 0.0f;
        FarLoop L;
        if (half == 0) L = a.loops[a.sel[0]];
        for (int s = 0; s < a.nsel; ++s) {
            FarLoop next;
            if (half == 0) {
                // the next loop's descriptor loads while this loop's layers run
                next = a.loops[a.sel[s + 1 < a.nsel ? s + 1 : s]];
                float f[16];
                features(px, py, pz, L, a.fn, f);
                uint32_t w[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) w[i] = pack_bf16(f[2 * i], f[2 * i + 1]);
                *reinterpret_cast<uint4*>(X + tc::kmajor_offset(row, 0, 128)) = make_uint4(w[0], w[1], w[2], w[3]);
                *reinterpret_cast<uint4*>(X + tc::kmajor_offset(row, 8, 128)) = make_uint4(w[4], w[5], w[6], w[7]);
            }
            ok = mma_step(tmem, aX, lbo128, aW1, lbo128, kIn / 16, id_hid, &bar[1], phase);
            if (!ok) break;
            epilogue_hidden(trow, bias, H, row, half * (kHid / 2));
            ok = mma_step(tmem, aH, lbo128, aW2, lbo128, kHid / 16, id_hid, &bar[1], phase);
            if (!ok) break;
            epilogue_hidden(trow, bias + kHid, H, row, half * (kHid / 2));
            ok = mma_step(tmem, aH, lbo128, aW3, lbo128, kHid / 16, id_hid, &bar[1], phase);
            if (!ok) break;
            epilogue_hidden(trow, bias + 2 * kHid, H, row, half * (kHid / 2));
            ok = mma_step(tmem, aH, lbo128, aW4, lbo16, kHid / 16, id_out, &bar[1], phase);
            if (!ok) break;
            if (half == 0) {
                float y[16];
                tc::ld16(trow, y);
                const float* b4 = bias + 3 * kHid;
                const float gx = (y[0] + b4[0]) * L.gain, gy = (y[1] + b4[1]) * L.gain,
                            gz = (y[2] + b4[2]) * L.gain;
                if (a.per_loop) {
                    if (valid) {
                        float* o = a.per_loop + (int64_t)s * 3 * a.n;
                        o[atom] = gx;
                        o[a.n + atom] = gy;
                        o[2 * a.n + atom] = gz;
                    }
                } else {
                    sx += gx;
                    sy += gy;
                    sz += gz;
                }
                L = next;
            }
        }
        if (ok && half == 0 && valid && !a.per_loop) {
            a.ux[atom] += sx;
            a.uy[atom] += sy;
            a.uz[atom] += sz;
        }
    }
    if (!ok && t == 0) {
        report(a.status, DISCO_ETIMEOUT);
        mbar_wait_bounded(&bar[1], phase ^ 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::dealloc(tmem, kTmemCols);
}

// ---- the subsample check --------------------------------------------------------

__global__ void gather_kernel(const double* x, const double* y, const double* z, const int64_t* idx, int64_t m,
                              double* gx, double* gy, double* gz)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = idx[j];
        gx[j] = x[i];
        gy[j] = y[i];
        gz[j] = z[i];
    }
}

// diff = network - exact per (loop, component, atom); loop_max[l] = max |diff|
__global__ void diff_kernel(const float* net, const double* exact, int64_t per_loop, float* diff, float* loop_max)
{
    const int l = blockIdx.y;
    float m = 0.0f;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < per_loop;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = (int64_t)l * per_loop + e;
        const float d = (float)((double)net[k] - exact[k]);
        diff[k] = d;
        m = fmaxf(m, d == d ? fabsf(d) : INFINITY);     // a NaN never passes
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int*>(loop_max + l), __float_as_int(m));
}

// total over the loops still on the network (keep[l] = 1) per (component, atom):
// out[0] = max |total| (as int bits), out_sq += total^2
__global__ void total_kernel(const float* diff, const int32_t* keep, int nloops, int64_t per_loop, float* out_max,
                             double* out_sq)
{
    float m = 0.0f;
    double sq = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < per_loop;
         e += (int64_t)gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int l = 0; l < nloops; ++l)
            if (keep[l]) s += diff[(int64_t)l * per_loop + e];
        m = fmaxf(m, s == s ? fabsf(s) : INFINITY);
        sq += (double)s * s;
    }
    for (int o = 16; o > 0; o >>= 1) {
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        sq += __shfl_xor_sync(0xffffffffu, sq, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(reinterpret_cast<int*>(out_max), __float_as_int(m));
        atomicAdd(out_sq, sq);
    }
}

} // namespace far
} // namespace disco

// ---- host ---------------------------------------------------------------------------------

namespace {

using namespace disco::far;

int ffail(int code, const std::string& msg)
{
    disco::set_last_error(msg);
    return code;
}

int fcuda(cudaError_t e, const char* what)
{
    disco::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? DISCO_ENOMEM : DISCO_ECUDA;
}

#define FAR_TRY(call, what)                                    \
    do {                                                       \
        const cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return fcuda(e_, what);         \
    } while (0)

// Host restatement of the loop-constant features (see disco_far_norm).
int build_far_loops(const disco_loop* loops, int32_t nloops, const double box[3], const disco_far_norm* norm,
                    std::vector<FarLoop>& out, std::vector<float>& gain)
{
    out.assign((size_t)nloops, FarLoop{});
    gain.assign((size_t)nloops, 0.0f);
    const double Lref = std::cbrt(box[0] * box[1] * box[2]);
    const double pi = 3.14159265358979323846;
    for (int l = 0; l < nloops; ++l) {
        const disco_loop& lp = loops[l];
        if (!lp.line || lp.n_vertices < 3 || !lp.vx || !lp.vy || !lp.vz)
            return ffail(DISCO_EINVAL, "learned far shells: loop " + std::to_string(l) + " is not a polyline");
        const double c[3] = { lp.cx, lp.cy, lp.cz };
        double av[3] = { 0, 0, 0 }, rmax = 0.0;
        for (int i = 0; i < lp.n_vertices; ++i) {
            const int j = (i + 1) % lp.n_vertices;
            const double p[3] = { lp.vx[i] - c[0], lp.vy[i] - c[1], lp.vz[i] - c[2] };
            const double q[3] = { lp.vx[j] - c[0], lp.vy[j] - c[1], lp.vz[j] - c[2] };
            av[0] += 0.5 * (p[1] * q[2] - p[2] * q[1]);
            av[1] += 0.5 * (p[2] * q[0] - p[0] * q[2]);
            av[2] += 0.5 * (p[0] * q[1] - p[1] * q[0]);
            rmax = std::max(rmax, std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]));
        }
        const double A = std::sqrt(av[0] * av[0] + av[1] * av[1] + av[2] * av[2]);
        double n[3] = { lp.phys.nx, lp.phys.ny, lp.phys.nz };
        const double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        const double b[3] = { lp.phys.bx * lp.phys.mx, lp.phys.by * lp.phys.my, lp.phys.bz * lp.phys.mz };
        const double bb = std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
        if (!(A > 0.0) || !(nn > 0.0) || !(bb > 0.0))
            return ffail(DISCO_EINVAL, "learned far shells: loop " + std::to_string(l) + " has no area, normal or b");
        for (double& v : n) v /= nn;
        const double bh[3] = { b[0] / bb, b[1] / bb, b[2] / bb };
        const double bn = bh[0] * n[0] + bh[1] * n[1] + bh[2] * n[2];
        const double req = std::sqrt(A / pi);
        const double raw[11] = { req / Lref, n[0], n[1], n[2], bh[0], bh[1], bh[2],
                                 box[1] / box[0] - 1.0, box[2] / box[0] - 1.0, rmax / req - 1.0, bn };
        FarLoop& F = out[l];
        F.cx = c[0]; F.cy = c[1]; F.cz = c[2];
        for (int k = 0; k < 11; ++k)
            F.feat[k] = norm ? (float)((raw[k] - norm->mu[3 + k]) * norm->inv_sd[3 + k]) : (float)raw[k];
        const double g = bb * A / (Lref * Lref);
        gain[l] = (float)g;
        F.gain = (float)(norm ? g * norm->out_scale : g);
    }
    return DISCO_OK;
}

FeatNorm feat_norm(const double box[3], const disco_far_norm* norm)
{
    FeatNorm fn;
    fn.iLx = 1.0 / box[0];
    fn.iLy = 1.0 / box[1];
    fn.iLz = 1.0 / box[2];
    for (int k = 0; k < 3; ++k) {
        fn.mu[k] = norm ? norm->mu[k] : 0.0f;
        fn.isd[k] = norm ? norm->inv_sd[k] : 1.0f;
    }
    return fn;
}

bool box_ok(const double* box) { return box && box[0] > 0.0 && box[1] > 0.0 && box[2] > 0.0; }

int apply_impl(disco_mlp* m, const disco_far_norm* norm, const disco_atoms* a, const disco_loop* loops,
               int32_t nloops, const double box[3], const int32_t* sel, int32_t nsel, float* per_loop,
               cudaStream_t s)
{
    if (!m || !norm || !a || nloops < 0 || (nloops > 0 && !loops) || !box_ok(box) || nsel < 0)
        return ffail(DISCO_EINVAL, "far_apply: bad argument");
    if (a->n < 0) return ffail(DISCO_EINVAL, "far_apply: negative atom count");
    std::vector<int32_t> idx;
    if (sel) {
        idx.assign(sel, sel + nsel);
        for (int32_t v : idx)
            if (v < 0 || v >= nloops) return ffail(DISCO_EINVAL, "far_apply: loop index out of range");
    } else {
        nsel = nloops;
        idx.resize((size_t)nloops);
        for (int l = 0; l < nloops; ++l) idx[l] = l;
    }
    if (a->n == 0 || nsel == 0) return DISCO_OK;
    if (!a->x || !a->y || !a->z || (!per_loop && (!a->ux || !a->uy || !a->uz)))
        return ffail(DISCO_EINVAL, "far_apply: null atom array");
    std::vector<FarLoop> fl;
    std::vector<float> gain;
    int st = build_far_loops(loops, nloops, box, norm, fl, gain);
    if (st) return st;
    if (!m->packed) FAR_TRY(cudaMalloc(&m->packed, kImgBytes), "far weights image");
    // per-call descriptor upload (a pageable copy returns once the source is consumed)
    const size_t bl = fl.size() * sizeof(FarLoop), bs = idx.size() * sizeof(int32_t);
    void* dbuf = nullptr;
    FAR_TRY(cudaMallocAsync(&dbuf, bl + bs, s), "far loop descriptors");
    cudaError_t e = cudaMemcpyAsync(dbuf, fl.data(), bl, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(static_cast<char*>(dbuf) + bl, idx.data(), bs, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { cudaFreeAsync(dbuf, s); return fcuda(e, "far descriptor upload"); }
    pack_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(m->params, m->packed);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    FarArgs fa;
    std::memset(&fa, 0, sizeof(fa));
    fa.x = a->x; fa.y = a->y; fa.z = a->z;
    fa.ux = a->ux; fa.uy = a->uy; fa.uz = a->uz;
    fa.n = a->n;
    fa.loops = static_cast<const FarLoop*>(dbuf);
    fa.sel = reinterpret_cast<const int32_t*>(static_cast<char*>(dbuf) + bl);
    fa.nsel = nsel;
    fa.ntiles = (int32_t)((a->n + 127) / 128);
    fa.per_loop = per_loop;
    fa.image = m->packed;
    fa.fn = feat_norm(box, norm);
    fa.status = m->status;
    e = cudaFuncSetAttribute(far_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmTotal);
    if (e == cudaSuccess) {
        const int grid = (int)std::min<int64_t>(fa.ntiles, 2 * (int64_t)std::max(sms, 1));
        far_kernel<<<grid, kFarThreads, kSmTotal, s>>>(fa);
        e = cudaGetLastError();
    }
    cudaFreeAsync(dbuf, s);
    return e == cudaSuccess ? DISCO_OK : fcuda(e, "far kernel launch");
}

struct Ev {
    cudaEvent_t a = nullptr, b = nullptr;
    Ev() { cudaEventCreate(&a); cudaEventCreate(&b); }
    ~Ev() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); }
    double seconds()
    {
        float ms = 0.0f;
        return cudaEventElapsedTime(&ms, a, b) == cudaSuccess ? ms * 1e-3 : 0.0;
    }
};

uint64_t splitmix(uint64_t& st)
{
    st += 0x9E3779B97F4A7C15ull;
    uint64_t z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Device buffers of one learned call, released on every exit path.
struct Bufs {
    std::vector<void*> ptrs;
    ~Bufs() { for (void* p : ptrs) cudaFree(p); }
    template <class T>
    cudaError_t get(T** out, size_t count)
    {
        void* p = nullptr;
        const cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(p);
        *out = static_cast<T*>(p);
        return e;
    }
};

} // namespace

extern "C" {

int disco_b200_far_features(const disco_atoms* a, const disco_loop* loops, int32_t nloops, const double box[3],
                            const disco_far_norm* norm, float* X, float* gain, void* stream)
{
    if (!a || nloops < 0 || (nloops > 0 && !loops) || !box_ok(box) || a->n < 0)
        return ffail(DISCO_EINVAL, "far_features: bad argument");
    std::vector<FarLoop> fl;
    std::vector<float> g;
    int st = build_far_loops(loops, nloops, box, norm, fl, g);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (gain && nloops > 0)
        FAR_TRY(cudaMemcpyAsync(gain, g.data(), g.size() * sizeof(float), cudaMemcpyHostToDevice, s), "gain");
    if (a->n == 0 || nloops == 0) return DISCO_OK;
    if (!a->x || !a->y || !a->z || !X) return ffail(DISCO_EINVAL, "far_features: null array");
    void* dl = nullptr;
    FAR_TRY(cudaMallocAsync(&dl, fl.size() * sizeof(FarLoop), s), "far loop descriptors");
    cudaError_t e = cudaMemcpyAsync(dl, fl.data(), fl.size() * sizeof(FarLoop), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        const int64_t rows = a->n * nloops;
        const int grid = (int)std::min<int64_t>((rows + 255) / 256, 148 * 16);
        features_kernel<<<grid, 256, 0, s>>>(a->x, a->y, a->z, a->n, static_cast<const FarLoop*>(dl), nloops,
                                             feat_norm(box, norm), X);
        e = cudaGetLastError();
    }
    cudaFreeAsync(dl, s);
    return e == cudaSuccess ? DISCO_OK : fcuda(e, "far features");
}

int disco_b200_far_apply(disco_mlp* m, const disco_far_norm* norm, const disco_atoms* a, const disco_loop* loops,
                         int32_t nloops, const double box[3], const int32_t* sel, int32_t nsel, float* per_loop,
                         void* stream)
{
    return apply_impl(m, norm, a, loops, nloops, box, sel, nsel, per_loop, static_cast<cudaStream_t>(stream));
}

int disco_b200_learned_displace(disco_mlp* m, const disco_far_norm* norm, const disco_atoms* a,
                                const disco_loop* loops, int32_t nloops, const double box[3],
                                const disco_learned_options* opt, disco_learned_report* rep, void* stream)
{
    if (!m || !norm || !a || !opt || nloops < 0 || (nloops > 0 && !loops) || !box_ok(box))
        return ffail(DISCO_EINVAL, "learned_displace: bad argument");
    if (norm->image_min < 1 || norm->images < norm->image_min || norm->images > 8)
        return ffail(DISCO_EINVAL, "learned_displace: the network's shells must satisfy 1 <= image_min <= images <= 8");
    if (!(opt->check_fraction >= 0.0 && opt->check_fraction <= 1.0) || !(opt->tol_loop >= 0.0) ||
        !(opt->tol_total >= 0.0))
        return ffail(DISCO_EINVAL, "learned_displace: bad check options");
    if (a->n < 0) return ffail(DISCO_EINVAL, "learned_displace: negative atom count");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    disco_learned_report R;
    std::memset(&R, 0, sizeof(R));
    if (rep) { R.loop_err = rep->loop_err; R.fallback = rep->fallback; }
    std::vector<int32_t> fb((size_t)nloops, 0);
    std::vector<float> lerr((size_t)nloops, 0.0f);
    const int64_t n = a->n;
    // kernels of one exact sum of line loops: FP32C adds the near-cut FP64 pass
    auto sum_launches = [](int precision) { return precision == DISCO_FP32C ? 2 : 1; };
    int launches = 0;
    Bufs B;
    Ev ec, en, ef, eb;

    // 1. exact far shells and the network, per loop, on the subsample
    int64_t nc = (n > 0 && nloops > 0 && opt->check_fraction > 0.0)
                     ? std::max<int64_t>(1, (int64_t)std::llround(opt->check_fraction * (double)n)) : 0;
    nc = std::min(nc, n);
    R.n_check = nc;
    cudaEventRecord(ec.a, s);
    if (nc > 0) {
        std::vector<int64_t> idx((size_t)nc);
        uint64_t st = opt->seed * 0x2545F4914F6CDD1Dull + 7;
        for (int64_t j = 0; j < nc; ++j) {
            const double u = (double)(splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
            const int64_t lo = j * n / nc, hi = (j + 1) * n / nc;
            idx[j] = std::min(hi - 1, lo + (int64_t)(u * (double)(hi - lo)));
        }
        int64_t* didx;
        double *gx, *gy, *gz, *exact, *dsq;
        float *net, *diff, *lmax, *tmax;
        int32_t* keep;
        const size_t per = 3 * (size_t)nc;
        FAR_TRY(B.get(&didx, nc), "check buffers");
        FAR_TRY(B.get(&gx, nc), "check buffers");
        FAR_TRY(B.get(&gy, nc), "check buffers");
        FAR_TRY(B.get(&gz, nc), "check buffers");
        FAR_TRY(B.get(&exact, per * nloops), "check buffers");
        FAR_TRY(B.get(&net, per * nloops), "check buffers");
        FAR_TRY(B.get(&diff, per * nloops), "check buffers");
        FAR_TRY(B.get(&lmax, nloops), "check buffers");
        FAR_TRY(B.get(&tmax, 1), "check buffers");
        FAR_TRY(B.get(&dsq, 1), "check buffers");
        FAR_TRY(B.get(&keep, nloops), "check buffers");
        FAR_TRY(cudaMemcpyAsync(didx, idx.data(), nc * sizeof(int64_t), cudaMemcpyHostToDevice, s), "subsample");
        gather_kernel<<<(int)std::min<int64_t>((nc + 255) / 256, 4096), 256, 0, s>>>(a->x, a->y, a->z, didx, nc,
                                                                                     gx, gy, gz);
        launches += 1;
        FAR_TRY(cudaMemsetAsync(exact, 0, per * nloops * sizeof(double), s), "check buffers");
        // exact: one batch sample per loop over the subsample's atoms
        std::vector<disco_sample> smp((size_t)nloops);
        for (int l = 0; l < nloops; ++l) {
            disco_sample& d = smp[l];
            std::memset(&d, 0, sizeof(d));
            d.atoms.x = gx; d.atoms.y = gy; d.atoms.z = gz;
            d.atoms.ux = exact + per * l;
            d.atoms.uy = exact + per * l + nc;
            d.atoms.uz = exact + per * l + 2 * nc;
            d.atoms.n = nc;
            d.loops = &loops[l];
            d.nloops = 1;
            d.images = norm->images;
            d.image_min = norm->image_min;
            for (int k = 0; k < 3; ++k) d.box[k] = box[k];
        }
        disco_options bo;
        disco_b200_options_default(&bo);
        bo.precision = opt->check_precision;
        bo.nu = opt->nu;
        disco_batch_plan* bp = nullptr;
        int st2 = disco_b200_batch_plan_create(smp.data(), nloops, &bo, &bp);
        if (st2) return st2;
        st2 = disco_b200_batch_plan_execute(bp, s);
        if (!st2) st2 = disco_b200_batch_plan_sync(bp, s);
        disco_b200_batch_plan_destroy(bp);
        if (st2) return st2;
        launches += sum_launches(opt->check_precision);
        disco_atoms ga = { gx, gy, gz, nullptr, nullptr, nullptr, nc };
        st2 = apply_impl(m, norm, &ga, loops, nloops, box, nullptr, nloops, net, s);
        if (st2) return st2;
        launches += 3;                     // weights image, far kernel, differences
        FAR_TRY(cudaMemsetAsync(lmax, 0, nloops * sizeof(float), s), "check buffers");
        diff_kernel<<<dim3((unsigned)std::min<int64_t>((per + 255) / 256, 256), nloops), 256, 0, s>>>(
            net, exact, (int64_t)per, diff, lmax);
        FAR_TRY(cudaMemcpyAsync(lerr.data(), lmax, nloops * sizeof(float), cudaMemcpyDeviceToHost, s), "check");
        FAR_TRY(cudaStreamSynchronize(s), "check");
        int dst = disco_b200_mlp_status(m);
        if (dst) return dst;
        for (int l = 0; l < nloops; ++l) {
            R.worst_loop = std::max(R.worst_loop, (double)lerr[l]);
            if (!(lerr[l] <= opt->tol_loop)) fb[l] = 1;
        }
        // further loops, largest error first, until the subsample total is within tol_total
        for (;;) {
            std::vector<int32_t> kp((size_t)nloops);
            for (int l = 0; l < nloops; ++l) kp[l] = fb[l] ? 0 : 1;
            FAR_TRY(cudaMemcpyAsync(keep, kp.data(), nloops * sizeof(int32_t), cudaMemcpyHostToDevice, s), "check");
            FAR_TRY(cudaMemsetAsync(tmax, 0, sizeof(float), s), "check");
            FAR_TRY(cudaMemsetAsync(dsq, 0, sizeof(double), s), "check");
            total_kernel<<<(unsigned)std::min<int64_t>((per + 255) / 256, 1024), 256, 0, s>>>(diff, keep, nloops,
                                                                                              (int64_t)per, tmax, dsq);
            launches += 1;
            float tm = 0.0f;
            double sq = 0.0;
            FAR_TRY(cudaMemcpyAsync(&tm, tmax, sizeof(float), cudaMemcpyDeviceToHost, s), "check");
            FAR_TRY(cudaMemcpyAsync(&sq, dsq, sizeof(double), cudaMemcpyDeviceToHost, s), "check");
            FAR_TRY(cudaStreamSynchronize(s), "check");
            R.check_max = tm;
            R.check_rms = std::sqrt(sq / (double)per);
            if (tm <= opt->tol_total) break;
            int worst = -1;
            for (int l = 0; l < nloops; ++l)
                if (!fb[l] && (worst < 0 || lerr[l] > lerr[worst])) worst = l;
            if (worst < 0) break;
            fb[worst] = 1;
        }
    }
    cudaEventRecord(ec.b, s);

    // 2. exact near images, every loop
    cudaEventRecord(en.a, s);
    if (n > 0 && nloops > 0) {
        disco_options no;
        disco_b200_options_default(&no);
        no.precision = opt->precision;
        no.nu = opt->nu;
        no.images = norm->image_min - 1;
        disco_plan* p = nullptr;
        int st2 = disco_b200_plan_create(loops, nloops, box, &no, n, &p);
        if (st2) return st2;
        st2 = disco_b200_plan_execute(p, a, s);
        if (!st2) st2 = disco_b200_plan_sync(p, s);
        disco_b200_plan_destroy(p);
        if (st2) return st2;
        launches += sum_launches(opt->precision);
    }
    cudaEventRecord(en.b, s);

    // 3. the network's far shells for the loops that passed
    std::vector<int32_t> on, off;
    for (int l = 0; l < nloops; ++l) (fb[l] ? off : on).push_back(l);
    cudaEventRecord(ef.a, s);
    if (n > 0 && !on.empty()) {
        int st2 = apply_impl(m, norm, a, loops, nloops, box, on.data(), (int32_t)on.size(), nullptr, s);
        if (st2) return st2;
        launches += 2;
    }
    cudaEventRecord(ef.b, s);

    // 4. exact far shells for the loops that fell back
    cudaEventRecord(eb.a, s);
    if (n > 0 && !off.empty()) {
        std::vector<disco_loop> sub;
        for (int l : off) sub.push_back(loops[l]);
        disco_options fo;
        disco_b200_options_default(&fo);
        fo.precision = opt->precision;
        fo.nu = opt->nu;
        fo.images = norm->images;
        fo.image_min = norm->image_min;
        disco_plan* p = nullptr;
        int st2 = disco_b200_plan_create(sub.data(), (int32_t)sub.size(), box, &fo, n, &p);
        if (st2) return st2;
        st2 = disco_b200_plan_execute(p, a, s);
        if (!st2) st2 = disco_b200_plan_sync(p, s);
        disco_b200_plan_destroy(p);
        if (st2) return st2;
        launches += sum_launches(opt->precision);
    }
    cudaEventRecord(eb.b, s);
    FAR_TRY(cudaStreamSynchronize(s), "learned displacement");
    const int dst = disco_b200_mlp_status(m);
    if (dst) return dst;
    R.t_check = ec.seconds();
    R.t_near = en.seconds();
    R.t_far = ef.seconds();
    R.t_fallback = eb.seconds();
    R.n_fallback = (int32_t)off.size();
    R.launches = launches;
    if (R.loop_err)
        for (int l = 0; l < nloops; ++l) R.loop_err[l] = lerr[l];
    if (R.fallback)
        for (int l = 0; l < nloops; ++l) R.fallback[l] = fb[l];
    if (rep) *rep = R;
    return DISCO_OK;
}

} // extern "C"
