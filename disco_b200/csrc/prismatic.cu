// Prismatic matter step on the GPU (Code/prismatic.cpp:36-74 driven as
// Code/main.cpp:586-687), and the fused output epilogue (Code/main.cpp:733-743,
// 797-818).
//
// Slab membership of an atom is the reference's FP64 predicate evaluated with
// explicit round-to-nearest intrinsics in the reference's operation order, so
// no FMA contraction can change it: the atom sets are bit-exact with the
// contract-off oracle, and the oracle's margin report shows that the
// reference's own contracted build selects the same sets.
//
// Stream compaction, order-preserving, in three passes over tiles of 2048
// atoms (8 rounds of 256):
//   count    per tile and category (survivors, and the slab of every loop),
//            warp ballots + shared-memory counters;
//   scan     one CTA: exclusive scan over tiles per category, per-loop bases;
//   scatter  the predicate again (cheaper than storing it), ranks from warp
//            ballots and a per-round scan over the 8 warps; survivors are
//            compacted (x, y, z and the new-index map) and slab entries
//            written at base + tile offset + rank, i.e. ascending atom order.
// A fourth single-CTA pass gathers the interstitial copies in loop order then
// slab order, drops those of removed atoms and renumbers their sources.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "common.cuh"

namespace disco {

constexpr int kSlabThreads = 256;
constexpr int kSlabRounds = 8;
constexpr int kSlabTile = kSlabThreads * kSlabRounds;   // atoms per tile
constexpr int kMaxSlabLoops = 64;                       // active slab loops per call
constexpr int kSlabWarps = kSlabThreads / 32;

struct SlabLoopDev {
    disco_slab_loop L;
    double tLo, tHi;       // slab bounds in units of d (Code/prismatic.cpp:58-59)
    double cuv, det;       // u.v and 1 - (u.v)^2 (Code/loop.cpp:327-328)
    float nf[3], cf[3];    // the pre-test only: n, c, 1 / spacing, its margin in planes
    float inv_df, margin;
    int32_t type;          // DISCO_MATTER_VACANCY or DISCO_MATTER_INTERSTITIAL
    int32_t pad;
};

// ---- the predicate, FP64 round-to-nearest, reference operation order -------------------

__device__ __forceinline__ double min_image(double r, double L)
{
    // r - L * floor(r / L + 0.5)   (Code/prismatic.cpp:31-34)
    return __dsub_rn(r, __dmul_rn(L, floor(__dadd_rn(__ddiv_rn(r, L), 0.5))));
}

__device__ __forceinline__ double dot3_rn(double a0, double a1, double a2, double b0, double b1, double b2)
{
    return __dadd_rn(__dadd_rn(__dmul_rn(a0, b0), __dmul_rn(a1, b1)), __dmul_rn(a2, b2));
}

// Code/loop.cpp:281-316
__device__ bool inside_uv_rn(const disco_slab_loop& g, double u, double v)
{
    const double eps = 1e-9;
    if (g.shape == DISCO_SHAPE_CIRCLE)
        return __dsqrt_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v))) < __dsub_rn(g.radius, eps);
    if (g.shape == DISCO_SHAPE_POLYGON) {
        const int N = g.n_poly;
        bool inner = true;
        for (int i = 0; i < N && inner; i++)
            if (__dadd_rn(__dmul_rn(g.nu[i], __dsub_rn(u, g.pu[i])), __dmul_rn(g.nv[i], __dsub_rn(v, g.pv[i])))
                < __dsub_rn(g.r_corner, eps))
                inner = false;
        if (inner) return true;
        if (g.r_corner <= 0.) return false;
        double d2 = 1e300;
        for (int i = 0; i < N; i++) {
            const int j = (i + 1) % N;
            const double eu = __dsub_rn(g.qu[j], g.qu[i]), ev = __dsub_rn(g.qv[j], g.qv[i]);
            const double l2 = __dadd_rn(__dmul_rn(eu, eu), __dmul_rn(ev, ev));
            double t = l2 > 0. ? __ddiv_rn(__dadd_rn(__dmul_rn(__dsub_rn(u, g.qu[i]), eu),
                                                     __dmul_rn(__dsub_rn(v, g.qv[i]), ev)), l2) : 0.;
            t = fmin(fmax(t, 0.), 1.);
            const double wu = __dsub_rn(__dsub_rn(u, g.qu[i]), __dmul_rn(t, eu));
            const double wv = __dsub_rn(__dsub_rn(v, g.qv[i]), __dmul_rn(t, ev));
            d2 = fmin(d2, __dadd_rn(__dmul_rn(wu, wu), __dmul_rn(wv, wv)));
        }
        return d2 <= __dadd_rn(__dmul_rn(g.r_corner, g.r_corner), eps);
    }
    const double du = fmax(__dsub_rn(fabs(u), fmax(__dsub_rn(g.half_m, g.r_corner), 0.0)), 0.0);
    const double dv = fmax(__dsub_rn(fabs(v), fmax(__dsub_rn(g.half_p, g.r_corner), 0.0)), 0.0);
    return __dadd_rn(__dmul_rn(du, du), __dmul_rn(dv, dv)) <= __dadd_rn(__dmul_rn(g.r_corner, g.r_corner), eps);
}

// Cheap pre-test in FP32: true only if the atom's t is outside [tLo, tHi) by
// more than `margin` planes.  With the atom and the centre rounded to FP32
// and the nearest image unambiguous (r/L + 1/2 at least 1e-5 from an integer
// and |r/L| < 2, else it returns false), the FP32 t differs from the exactly
// rounded t of slab_member by less than 1.5e-6 (Lx + Ly + Lz) / d + 1e-6
// planes; the margin is 1e-5 (Lx + Ly + Lz) / d + 1e-3.  So it never rejects
// a member: the exact test below decides every atom it passes, and atom sets
// stay bit-exact.
__device__ __forceinline__ bool clearly_outside(const SlabLoopDev& S, const float (&p)[3], const float (&L)[3],
                                                const float (&iL)[3])
{
    float s = 0.0f;
    bool sure = true;                     // branch-free, so that loops interleave
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float r = p[k] - S.cf[k];
        const float q = r * iL[k];
        const float h = q + 0.5f;
        const float f = floorf(h);
        const float fr = h - f;
        sure = sure && fabsf(q) < 2.0f && fr >= 1e-5f && fr <= 1.0f - 1e-5f;
        s = fmaf(S.nf[k], fmaf(-L[k], f, r), s);
    }
    const float t = s * S.inv_df;
    return sure && (t < (float)S.tLo - S.margin || t >= (float)S.tHi + S.margin);
}

// Slab membership of one atom (Code/prismatic.cpp:61-72); side = sign of s.
__device__ __forceinline__ bool slab_member(const SlabLoopDev& S, double x, double y, double z,
                                            double Lx, double Ly, double Lz, bool& pos_side)
{
    const disco_slab_loop& g = S.L;
    const double r0 = min_image(__dsub_rn(x, g.c[0]), Lx);
    const double r1 = min_image(__dsub_rn(y, g.c[1]), Ly);
    const double r2 = min_image(__dsub_rn(z, g.c[2]), Lz);
    const double s = dot3_rn(r0, r1, r2, g.n[0], g.n[1], g.n[2]);
    const double t = __ddiv_rn(s, g.spacing);
    if (t < S.tLo || t >= S.tHi) return false;
    const double ru = dot3_rn(r0, r1, r2, g.u[0], g.u[1], g.u[2]);
    const double rv = dot3_rn(r0, r1, r2, g.v[0], g.v[1], g.v[2]);
    const double uu = __ddiv_rn(__dsub_rn(ru, __dmul_rn(S.cuv, rv)), S.det);
    const double vv = __ddiv_rn(__dsub_rn(rv, __dmul_rn(S.cuv, ru)), S.det);
    if (!inside_uv_rn(g, uu, vv)) return false;
    pos_side = s > 0.;
    return true;
}

struct SlabArgs {
    const double *x, *y, *z;
    int64_t n;
    const SlabLoopDev* loops;
    int32_t nl;
    double Lx, Ly, Lz;
    float iLx, iLy, iLz;      // 1 / box lengths in FP32 (the pre-test only)
    int32_t* tile_counts;     // [ntiles][nl + 1]
    int32_t* tile_offsets;    // [ntiles][nl + 1]
    int64_t* totals;          // [nl + 1] totals, [nl] loop bases, [1] copies
    double *xo, *yo, *zo;
    int32_t* new_index;
    int32_t* slab_atoms;
    int8_t* slab_side;
};

// Every atom's membership mask over the active loops, sides and removal.
__device__ __forceinline__ void atom_masks(const SlabLoopDev* sl, int nl, double x, double y, double z,
                                           const SlabArgs& a, uint64_t& mask, uint64_t& sides, bool& removed)
{
    const double Lx = a.Lx, Ly = a.Ly, Lz = a.Lz;
    mask = 0; sides = 0; removed = false;
    const float L[3] = { (float)Lx, (float)Ly, (float)Lz };
    const float iL[3] = { a.iLx, a.iLy, a.iLz };
    const float p[3] = { (float)x, (float)y, (float)z };
    // the pre-test for every loop first (independent, interleaved), then the
    // exact test for the loops it could not exclude, in loop order
    uint64_t cand = 0;
#pragma unroll 4
    for (int l = 0; l < nl; ++l)
        if (!clearly_outside(sl[l], p, L, iL)) cand |= 1ull << l;
    while (cand) {
        const int l = __ffsll((long long)cand) - 1;
        cand &= cand - 1;
        bool ps = false;
        if (slab_member(sl[l], x, y, z, Lx, Ly, Lz, ps)) {
            mask |= 1ull << l;
            if (ps) sides |= 1ull << l;
            if (sl[l].type == DISCO_MATTER_VACANCY) removed = true;
        }
    }
}

__device__ __forceinline__ void load_loops(SlabLoopDev* dst, const SlabLoopDev* src, int nl)
{
    const int words = nl * (int)(sizeof(SlabLoopDev) / 8);
    const uint64_t* s = reinterpret_cast<const uint64_t*>(src);
    uint64_t* d = reinterpret_cast<uint64_t*>(dst);
    for (int i = threadIdx.x; i < words; i += blockDim.x) d[i] = s[i];
}

// CTA b takes tiles b, b + grid, ... (with the grid of slab_grid: tile b).
__global__ void __launch_bounds__(kSlabThreads) slab_count_kernel(const SlabArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SlabLoopDev* sl = reinterpret_cast<SlabLoopDev*>(smem_raw);
    __shared__ int cnt[kMaxSlabLoops + 1];
    const int C = a.nl + 1;
    load_loops(sl, a.loops, a.nl);
    const int lane = threadIdx.x & 31;
    const int64_t ntiles = (a.n + kSlabTile - 1) / kSlabTile;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        for (int i = threadIdx.x; i < C; i += blockDim.x) cnt[i] = 0;
        __syncthreads();
        const int64_t base = tile * kSlabTile;
        for (int r = 0; r < kSlabRounds; ++r) {
            const int64_t i = base + r * kSlabThreads + threadIdx.x;
            const bool valid = i < a.n;
            uint64_t mask = 0, sides = 0;
            bool removed = false;
            if (valid) atom_masks(sl, a.nl, a.x[i], a.y[i], a.z[i], a, mask, sides, removed);
            const unsigned b0 = __ballot_sync(0xffffffffu, valid && !removed);
            if (lane == 0 && b0) atomicAdd(&cnt[0], __popc(b0));
            for (int l = 0; l < a.nl; ++l) {
                const unsigned b = __ballot_sync(0xffffffffu, (mask >> l) & 1ull);
                if (lane == 0 && b) atomicAdd(&cnt[1 + l], __popc(b));
            }
        }
        __syncthreads();
        for (int c = threadIdx.x; c < C; c += blockDim.x)
            a.tile_counts[tile * C + c] = cnt[c];
        __syncthreads();
    }
}

// One CTA per category (survivors, then each loop): exclusive scan over the
// tiles, the category's total; the last CTA to finish (a counter in
// totals[2 C], zeroed with the totals) writes the loops' bases.
__global__ void __launch_bounds__(1024) slab_scan_kernel(const SlabArgs a, int64_t ntiles)
{
    __shared__ int64_t warp_sum[32];
    __shared__ int64_t carry;
    __shared__ bool last;
    const int C = a.nl + 1;
    const int c = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t t0 = 0; t0 < ntiles; t0 += blockDim.x) {
        const int64_t t = t0 + threadIdx.x;
        const int64_t v = t < ntiles ? a.tile_counts[t * C + c] : 0;
        int64_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int64_t s = lane < (int)(blockDim.x >> 5) ? warp_sum[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            warp_sum[lane] = s;           // inclusive over warps
        }
        __syncthreads();
        const int64_t excl = carry + (warp > 0 ? warp_sum[warp - 1] : 0) + x - v;
        if (t < ntiles) a.tile_offsets[t * C + c] = (int32_t)excl;
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_sum[(blockDim.x >> 5) - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        a.totals[c] = carry;
        __threadfence();
        const unsigned long long done =
            atomicAdd(reinterpret_cast<unsigned long long*>(&a.totals[2 * C]), 1ull);
        last = done == (unsigned long long)(C - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const volatile int64_t* tot = a.totals;
        int64_t acc = 0;
        for (int l = 0; l < a.nl; ++l) { a.totals[C + l] = acc; acc += tot[1 + l]; }
    }
}

__global__ void __launch_bounds__(kSlabThreads) slab_scatter_kernel(const SlabArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SlabLoopDev* sl = reinterpret_cast<SlabLoopDev*>(smem_raw);
    __shared__ int wcnt[kSlabWarps][kMaxSlabLoops + 1];    // per-warp counts, then prefixes
    __shared__ int run[kMaxSlabLoops + 1];                 // running count within the tile
    __shared__ int64_t base_off[kMaxSlabLoops + 1];        // global offset of this tile per category
    const int C = a.nl + 1;
    load_loops(sl, a.loops, a.nl);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t ntiles = (a.n + kSlabTile - 1) / kSlabTile;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        for (int c = threadIdx.x; c < C; c += blockDim.x) {
            run[c] = 0;
            const int64_t t = a.tile_offsets[tile * C + c];
            base_off[c] = c == 0 ? t : a.totals[C + (c - 1)] + t;
        }
        __syncthreads();
        const int64_t base = tile * kSlabTile;
        for (int r = 0; r < kSlabRounds; ++r) {
            const int64_t i = base + r * kSlabThreads + threadIdx.x;
            const bool valid = i < a.n;
            uint64_t mask = 0, sides = 0;
            bool removed = false;
            double x = 0., y = 0., z = 0.;
            if (valid) {
                x = a.x[i]; y = a.y[i]; z = a.z[i];
                atom_masks(sl, a.nl, x, y, z, a, mask, sides, removed);
            }
            const bool surv = valid && !removed;
            const unsigned b0 = __ballot_sync(0xffffffffu, surv);
            const int r0 = __popc(b0 & lt);
            if (lane == 0) wcnt[warp][0] = __popc(b0);
            for (int l = 0; l < a.nl; ++l) {
                const unsigned b = __ballot_sync(0xffffffffu, (mask >> l) & 1ull);
                if (lane == 0) wcnt[warp][1 + l] = __popc(b);
            }
            __syncthreads();
            // exclusive prefix over the warps of this round, per category
            for (int c = threadIdx.x; c < C; c += blockDim.x) {
                int acc = run[c];
                for (int w = 0; w < kSlabWarps; ++w) {
                    const int v = wcnt[w][c];
                    wcnt[w][c] = acc;
                    acc += v;
                }
                run[c] = acc;
            }
            __syncthreads();
            if (valid) {
                if (surv) {
                    const int64_t p = base_off[0] + wcnt[warp][0] + r0;
                    a.xo[p] = x; a.yo[p] = y; a.zo[p] = z;
                    a.new_index[i] = (int32_t)p;
                } else {
                    a.new_index[i] = -1;
                }
            }
            for (int l = 0; l < a.nl; ++l) {
                const bool m = (mask >> l) & 1ull;
                const unsigned b = __ballot_sync(0xffffffffu, m);
                if (m) {
                    const int64_t p = base_off[1 + l] + wcnt[warp][1 + l] + __popc(b & lt);
                    a.slab_atoms[p] = (int32_t)i;
                    a.slab_side[p] = ((sides >> l) & 1ull) ? 1 : -1;
                }
            }
            __syncthreads();
        }
    }
}

// One CTA: interstitial copies in loop order then slab order (Code/main.cpp:
// 651-654), copies of removed atoms dropped and sources renumbered (:676-679).
__global__ void __launch_bounds__(1024) slab_copies_kernel(const SlabArgs a, disco_copy* copies,
                                                           int64_t copy_capacity)
{
    __shared__ int warp_sum[32];
    __shared__ int64_t carry;
    const int C = a.nl + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int l = 0; l < a.nl; ++l) {
        if (a.loops[l].type != DISCO_MATTER_INTERSTITIAL) continue;
        const int64_t b0 = a.totals[C + l], cnt = a.totals[1 + l];
        const disco_slab_loop& g = a.loops[l].L;
        for (int64_t e0 = 0; e0 < cnt; e0 += blockDim.x) {
            const int64_t e = e0 + threadIdx.x;
            int32_t src = -1;
            int8_t side = 1;
            if (e < cnt) {
                const int32_t atom = a.slab_atoms[b0 + e];
                side = a.slab_side[b0 + e];
                src = a.new_index[atom];
            }
            const bool keep = src >= 0;
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) warp_sum[warp] = __popc(bal);
            __syncthreads();
            if (warp == 0) {
                int s = lane < (int)(blockDim.x >> 5) ? warp_sum[lane] : 0;
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, s, o);
                    if (lane >= o) s += y;
                }
                warp_sum[lane] = s;
            }
            __syncthreads();
            if (keep) {
                const int64_t p = carry + (warp > 0 ? warp_sum[warp - 1] : 0) + __popc(bal & ((1u << lane) - 1u));
                if (p < copy_capacity) {
                    disco_copy cp;
                    cp.atom = src;
                    cp.reserved = 0;
                    const double* sh = side > 0 ? g.shift_pos : g.shift_neg;
                    cp.shift[0] = sh[0]; cp.shift[1] = sh[1]; cp.shift[2] = sh[2];
                    copies[p] = cp;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) carry += warp_sum[(blockDim.x >> 5) - 1];
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) a.totals[2 * C - 1] = carry;   // slot after the loop bases
}

// Code/main.cpp:733-743 + 797-818: copies appended with u(src) + shift, then
// r = x + u folded once into [-L/2, L/2] and shifted by +L/2.
__global__ void finalize_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                const double* __restrict__ z, const double* __restrict__ ux,
                                const double* __restrict__ uy, const double* __restrict__ uz, int64_t n,
                                const disco_copy* __restrict__ copies, int64_t ncopies,
                                double Lx, double Ly, double Lz,
                                double* fx, double* fy, double* fz, double* uxo, double* uyo, double* uzo)
{
    const double hx = Lx / 2., hy = Ly / 2., hz = Lz / 2.;
    const int64_t total = n + ncopies;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        double px, py, pz, qx, qy, qz;
        if (k < n) {
            px = x[k]; py = y[k]; pz = z[k];
            qx = ux[k]; qy = uy[k]; qz = uz[k];
        } else {
            const disco_copy c = copies[k - n];
            px = x[c.atom]; py = y[c.atom]; pz = z[c.atom];
            qx = __dadd_rn(ux[c.atom], c.shift[0]);
            qy = __dadd_rn(uy[c.atom], c.shift[1]);
            qz = __dadd_rn(uz[c.atom], c.shift[2]);
        }
        double rx = __dadd_rn(px, qx), ry = __dadd_rn(py, qy), rz = __dadd_rn(pz, qz);
        if (rx > hx) rx = __dsub_rn(rx, Lx); else if (rx < -hx) rx = __dadd_rn(rx, Lx);
        if (ry > hy) ry = __dsub_rn(ry, Ly); else if (ry < -hy) ry = __dadd_rn(ry, Ly);
        if (rz > hz) rz = __dsub_rn(rz, Lz); else if (rz < -hz) rz = __dadd_rn(rz, Lz);
        fx[k] = __dadd_rn(rx, hx); fy[k] = __dadd_rn(ry, hy); fz[k] = __dadd_rn(rz, hz);
        if (uxo) { uxo[k] = qx; uyo[k] = qy; uzo[k] = qz; }
    }
}

} // namespace disco

// ---- host ------------------------------------------------------------------------------

namespace {

int cfail(cudaError_t e, const char* what)
{
    disco::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? DISCO_ENOMEM : DISCO_ECUDA;
}

int efail(int code, const std::string& msg)
{
    disco::set_last_error(msg);
    return code;
}

// Grid of the tile kernels: one CTA per tile (a persistent grid of 4 CTAs
// per SM measured 25 % slower: the per-round barriers of a tile want as many
// CTAs in flight as the GPU holds).
unsigned slab_grid(int64_t ntiles)
{
    return (unsigned)ntiles;
}

// One loop's SlabResult scalars (Code/prismatic.cpp:42-57) and, when it is
// active (b.n != 0 and apply), its device record.  Never allocates.
int slab_loop_record(const disco_slab_loop& g, int l, const double box[3], disco_slab_info& in,
                     disco::SlabLoopDev& d, bool& active)
{
    std::memset(&in, 0, sizeof(in));
    active = false;
    // host code of this library is built with -ffp-contract=off: these sums
    // round like the contract-off oracle
    const double mn = g.m[0] * g.n[0] + g.m[1] * g.n[1] + g.m[2] * g.n[2];
    int type = DISCO_MATTER_NONE;
    if (!(std::fabs(mn) < 1e-6)) type = mn > 0. ? DISCO_MATTER_VACANCY : DISCO_MATTER_INTERSTITIAL;
    if (!g.apply || type == DISCO_MATTER_NONE) return DISCO_OK;
    if (g.shape < 0 || g.shape > DISCO_SHAPE_POLYGON || g.n_poly < 0 || g.n_poly > DISCO_MAX_POLY ||
        !(g.spacing > 0.)) {
        (void)l;
        disco::set_last_error("bad slab loop: shape, polygon size or spacing out of range");
        return DISCO_EINVAL;
    }
    in.type = type;
    for (int i = 0; i < 3; ++i) in.b[i] = g.bmag * g.m[i];
    in.height = std::fabs(in.b[0] * g.n[0] + in.b[1] * g.n[1] + in.b[2] * g.n[2]);
    in.spacing = g.spacing;
    const double ratio = in.height / g.spacing;
    in.planes = (int)std::lround(ratio);
    if (in.planes < 1 || std::fabs(ratio - in.planes) > 1e-6) {
        disco::set_last_error("|b.n| is not a whole number of plane spacings");
        return DISCO_EPLANES;
    }
    std::memset(&d, 0, sizeof(d));
    d.L = g;
    d.tLo = -std::floor(in.planes / 2.);
    d.tHi = std::ceil(in.planes / 2.);
    const double c = g.u[0] * g.v[0] + g.u[1] * g.v[1] + g.u[2] * g.v[2];
    d.cuv = c;
    d.det = 1.0 - c * c;
    for (int k = 0; k < 3; ++k) {
        d.nf[k] = (float)g.n[k];
        d.cf[k] = (float)g.c[k];
    }
    d.inv_df = (float)(1.0 / in.spacing);
    d.margin = (float)(1e-5 * (box[0] + box[1] + box[2]) / in.spacing + 1e-3);
    d.type = type;
    active = true;
    return DISCO_OK;
}

// Active loops in caller order.
int prepare_loops(const disco_slab_loop* loops, int nloops, const double box[3], disco_slab_info* info,
                  std::vector<disco::SlabLoopDev>& act, std::vector<int>& act_index)
{
    for (int l = 0; l < nloops; ++l) {
        disco::SlabLoopDev d;
        bool active = false;
        const int st = slab_loop_record(loops[l], l, box, info[l], d, active);
        if (st) return st;
        if (!active) continue;
        if ((int)act.size() >= disco::kMaxSlabLoops) {
            disco::set_last_error("more than 64 prismatic loops in one call");
            return DISCO_ELIMIT;
        }
        act.push_back(d);
        act_index.push_back(l);
    }
    return DISCO_OK;
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    template <class T> T* as() { return static_cast<T*>(p); }
};

} // namespace

extern "C" {

int disco_b200_prismatic(const double* x, const double* y, const double* z, int64_t n,
                         const disco_slab_loop* loops, int32_t nloops, const double box[3],
                         double* x_out, double* y_out, double* z_out, int32_t* new_index,
                         disco_slab_info* info,
                         int32_t* slab_atoms, int8_t* slab_side, int64_t slab_capacity,
                         disco_copy* copies, int64_t copy_capacity, int64_t counts[3])
{
    using namespace disco;
    if (n < 0 || nloops < 0 || !box || !counts || (nloops > 0 && (!loops || !info)) ||
        (n > 0 && (!x || !y || !z || !x_out || !y_out || !z_out || !new_index)) ||
        slab_capacity < 0 || copy_capacity < 0 || (slab_capacity > 0 && (!slab_atoms || !slab_side)) ||
        (copy_capacity > 0 && !copies))
        return efail(DISCO_EINVAL, "null or negative argument");
    if (n > 2147483647LL) return efail(DISCO_ELIMIT, "more than 2^31 - 1 atoms");
    if (!(box[0] > 0.) || !(box[1] > 0.) || !(box[2] > 0.)) return efail(DISCO_EINVAL, "box lengths must be positive");
    int dcount = 0;
    if (cudaGetDeviceCount(&dcount) != cudaSuccess || dcount == 0) return efail(DISCO_ENODEV, "no CUDA device");
    std::vector<SlabLoopDev> act;
    std::vector<int> act_index;
    int st = prepare_loops(loops, nloops, box, info, act, act_index);
    if (st) return st;
    const int nl = (int)act.size();
    const int C = nl + 1;
    const int64_t ntiles = (n + kSlabTile - 1) / kSlabTile;

    DevBuf dxyz, dout, didx, dloops, dcnt, doff, dtot, dslab, dside, dcop;
    const size_t nb = (size_t)n * sizeof(double);
    cudaError_t e = cudaSuccess;
    if (n > 0) {
        e = cudaMalloc(&dxyz.p, 3 * nb);
        if (e == cudaSuccess) e = cudaMalloc(&dout.p, 3 * nb);
        if (e == cudaSuccess) e = cudaMalloc(&didx.p, (size_t)n * sizeof(int32_t));
    }
    if (e == cudaSuccess) e = cudaMalloc(&dloops.p, std::max<size_t>(1, act.size()) * sizeof(SlabLoopDev));
    if (e == cudaSuccess) e = cudaMalloc(&dcnt.p, std::max<int64_t>(1, ntiles * C) * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&doff.p, std::max<int64_t>(1, ntiles * C) * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&dtot.p, (size_t)(2 * C + 1) * sizeof(int64_t));
    if (e != cudaSuccess) return cfail(e, "prismatic allocation");
    if (n > 0) {
        e = cudaMemcpy(dxyz.as<double>(), x, nb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dxyz.as<double>() + n, y, nb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dxyz.as<double>() + 2 * n, z, nb, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && nl > 0)
        e = cudaMemcpy(dloops.p, act.data(), act.size() * sizeof(SlabLoopDev), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dtot.p, 0, (size_t)(2 * C + 1) * sizeof(int64_t));
    if (e != cudaSuccess) return cfail(e, "prismatic upload");

    SlabArgs a;
    std::memset(&a, 0, sizeof(a));
    a.x = dxyz.as<double>(); a.y = a.x + n; a.z = a.x + 2 * n;
    a.n = n;
    a.loops = dloops.as<SlabLoopDev>();
    a.nl = nl;
    a.Lx = box[0]; a.Ly = box[1]; a.Lz = box[2];
    a.iLx = (float)(1.0 / box[0]); a.iLy = (float)(1.0 / box[1]); a.iLz = (float)(1.0 / box[2]);
    a.tile_counts = dcnt.as<int32_t>();
    a.tile_offsets = doff.as<int32_t>();
    a.totals = dtot.as<int64_t>();
    a.xo = dout.as<double>(); a.yo = a.xo + n; a.zo = a.xo + 2 * n;
    a.new_index = didx.as<int32_t>();
    const size_t smem = act.size() * sizeof(SlabLoopDev);
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(slab_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(slab_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cfail(e, "prismatic smem");
    }
    if (ntiles > 0) slab_count_kernel<<<slab_grid(ntiles), kSlabThreads, smem>>>(a);
    slab_scan_kernel<<<(unsigned)C, 1024>>>(a, ntiles);
    std::vector<int64_t> tot(2 * C + 1, 0);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(tot.data(), dtot.p, tot.size() * sizeof(int64_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cfail(e, "prismatic count/scan");
    int64_t slab_total = 0, inter_total = 0;
    for (int l = 0; l < nl; ++l) {
        slab_total += tot[1 + l];
        if (act[l].type == DISCO_MATTER_INTERSTITIAL) inter_total += tot[1 + l];
    }
    e = cudaMalloc(&dslab.p, std::max<int64_t>(1, slab_total) * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&dside.p, std::max<int64_t>(1, slab_total));
    if (e == cudaSuccess) e = cudaMalloc(&dcop.p, std::max<int64_t>(1, inter_total) * sizeof(disco_copy));
    if (e != cudaSuccess) return cfail(e, "prismatic slab buffers");
    a.slab_atoms = dslab.as<int32_t>();
    a.slab_side = dside.as<int8_t>();
    if (ntiles > 0) slab_scatter_kernel<<<slab_grid(ntiles), kSlabThreads, smem>>>(a);
    slab_copies_kernel<<<1, 1024>>>(a, dcop.as<disco_copy>(), inter_total);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(tot.data(), dtot.p, tot.size() * sizeof(int64_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cfail(e, "prismatic scatter");
    const int64_t k = tot[0];
    counts[0] = k;
    counts[1] = slab_total;
    counts[2] = tot[2 * C - 1];
    for (int q = 0; q < nl; ++q) {
        disco_slab_info& in = info[act_index[q]];
        in.offset = tot[C + q];
        in.count = tot[1 + q];
    }
    // offsets of inactive loops: where the next active loop starts (empty ranges)
    {
        int64_t next = slab_total;
        for (int l = nloops - 1; l >= 0; --l) {
            if (info[l].type == DISCO_MATTER_NONE) info[l].offset = next;
            else next = info[l].offset;
        }
    }
    if (counts[1] > slab_capacity || counts[2] > copy_capacity)
        return efail(DISCO_ELIMIT, "slab or copy capacity too small (counts hold the sizes needed)");
    if (n > 0) {
        e = cudaMemcpy(new_index, didx.p, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && k > 0) e = cudaMemcpy(x_out, a.xo, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && k > 0) e = cudaMemcpy(y_out, a.yo, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && k > 0) e = cudaMemcpy(z_out, a.zo, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess && slab_total > 0)
        e = cudaMemcpy(slab_atoms, dslab.p, (size_t)slab_total * sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && slab_total > 0)
        e = cudaMemcpy(slab_side, dside.p, (size_t)slab_total, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && counts[2] > 0)
        e = cudaMemcpy(copies, dcop.p, (size_t)counts[2] * sizeof(disco_copy), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cfail(e, "prismatic download");
    return DISCO_OK;
}

int disco_b200_finalize(const double* x, const double* y, const double* z,
                        const double* ux, const double* uy, const double* uz, int64_t n,
                        const disco_copy* copies, int64_t ncopies, const double box[3],
                        double* fx, double* fy, double* fz,
                        double* ux_out, double* uy_out, double* uz_out)
{
    if (n < 0 || ncopies < 0 || !box || (n > 0 && (!x || !y || !z || !ux || !uy || !uz)) ||
        (ncopies > 0 && !copies) || (n + ncopies > 0 && (!fx || !fy || !fz)))
        return efail(DISCO_EINVAL, "null or negative argument");
    const bool want_u = ux_out && uy_out && uz_out;
    if (n + ncopies == 0) return DISCO_OK;
    int dcount = 0;
    if (cudaGetDeviceCount(&dcount) != cudaSuccess || dcount == 0) return efail(DISCO_ENODEV, "no CUDA device");
    for (int64_t j = 0; j < ncopies; ++j)
        if (copies[j].atom < 0 || copies[j].atom >= n) return efail(DISCO_EINVAL, "copy source out of range");
    const int64_t tot = n + ncopies;
    DevBuf din, dcop, dout;
    cudaError_t e = cudaMalloc(&din.p, 6 * std::max<int64_t>(1, n) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dcop.p, std::max<int64_t>(1, ncopies) * sizeof(disco_copy));
    if (e == cudaSuccess) e = cudaMalloc(&dout.p, 6 * tot * sizeof(double));
    if (e != cudaSuccess) return cfail(e, "finalize allocation");
    double* d = din.as<double>();
    const double* src[6] = { x, y, z, ux, uy, uz };
    for (int k = 0; k < 6 && e == cudaSuccess && n > 0; ++k)
        e = cudaMemcpy(d + k * n, src[k], (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ncopies > 0)
        e = cudaMemcpy(dcop.p, copies, (size_t)ncopies * sizeof(disco_copy), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cfail(e, "finalize upload");
    double* o = dout.as<double>();
    const int threads = 256;
    const int64_t blocks = std::min<int64_t>((tot + threads - 1) / threads, 148 * 16);
    disco::finalize_kernel<<<(unsigned)blocks, threads>>>(d, d + n, d + 2 * n, d + 3 * n, d + 4 * n, d + 5 * n, n,
                                                          dcop.as<disco_copy>(), ncopies, box[0], box[1], box[2],
                                                          o, o + tot, o + 2 * tot,
                                                          want_u ? o + 3 * tot : nullptr, o + 4 * tot, o + 5 * tot);
    e = cudaGetLastError();
    double* dst[6] = { fx, fy, fz, ux_out, uy_out, uz_out };
    for (int k = 0; k < (want_u ? 6 : 3) && e == cudaSuccess; ++k)
        e = cudaMemcpy(dst[k], o + k * tot, (size_t)tot * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cfail(e, "finalize");
    return DISCO_OK;
}

int disco_b200_finalize_resident(const double* x, const double* y, const double* z,
                                 const double* ux, const double* uy, const double* uz, int64_t n,
                                 const disco_copy* copies, int64_t ncopies, const double box[3],
                                 double* fx, double* fy, double* fz,
                                 double* ux_out, double* uy_out, double* uz_out, void* stream)
{
    if (n < 0 || ncopies < 0 || !box || (n > 0 && (!x || !y || !z || !ux || !uy || !uz)) ||
        (ncopies > 0 && (!copies || n == 0)) || (n + ncopies > 0 && (!fx || !fy || !fz)))
        return efail(DISCO_EINVAL, "null or negative argument");
    const bool want_u = ux_out && uy_out && uz_out;
    const int64_t tot = n + ncopies;
    if (tot == 0) return DISCO_OK;
    const int threads = 256;
    const int64_t blocks = std::min<int64_t>((tot + threads - 1) / threads, 148 * 16);
    disco::finalize_kernel<<<(unsigned)blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(
        x, y, z, ux, uy, uz, n, copies, ncopies, box[0], box[1], box[2], fx, fy, fz,
        want_u ? ux_out : nullptr, uy_out, uz_out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DISCO_OK : cfail(e, "finalize launch");
}

} // extern "C"

// ---- matter step without allocation ---------------------------------------------------
//
// Callers that own all device memory themselves (a framework with its own
// memory pool, a code that may not synchronise the device the way cudaFree
// does, a process with a fixed memory budget) cannot let the library call
// cudaMalloc.  disco_b200_prismatic_noalloc takes device inputs and outputs
// from the caller and keeps its scratch (active loop table, per-tile counts
// and offsets, totals) in the file-scope array below: 1.25 MiB that every GPU
// loading this library holds until the process exits.

namespace {

constexpr int64_t kNoAllocMaxAtoms = int64_t(1) << 22;                  // 4 194 304 atoms
constexpr int64_t kNoAllocMaxTiles = kNoAllocMaxAtoms / disco::kSlabTile;
constexpr size_t kNoAllocLoopBytes = disco::kMaxSlabLoops * sizeof(disco::SlabLoopDev);
constexpr size_t kNoAllocTotalsBytes = (2 * (disco::kMaxSlabLoops + 1) + 1) * sizeof(int64_t);
constexpr size_t kNoAllocTileBytes = kNoAllocMaxTiles * (disco::kMaxSlabLoops + 1) * sizeof(int32_t);
constexpr size_t kNoAllocScratchBytes = 1280 * 1024;
static_assert(((kNoAllocLoopBytes + 255) & ~size_t(255)) + ((kNoAllocTotalsBytes + 255) & ~size_t(255)) +
                  2 * kNoAllocTileBytes <= kNoAllocScratchBytes,
              "no-alloc scratch layout");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device.  In host code the
// array's name is a host-side stand-in, not a device address: the address is
// looked up once per device with that device current and cached.
int noalloc_scratch(unsigned char** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cfail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return efail(DISCO_ELIMIT, "device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return cfail(e, "cudaGetSymbolAddress of the scratch array");
        g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_addr[dev];
    return DISCO_OK;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

} // namespace

extern "C" {

int disco_b200_prismatic_noalloc(const double* x, const double* y, const double* z, int64_t n,
                                 const disco_slab_loop* loops, int32_t nloops, const double box[3],
                                 double* x_out, double* y_out, double* z_out, int32_t* new_index,
                                 disco_slab_info* info,
                                 int32_t* slab_atoms, int8_t* slab_side, int64_t slab_capacity,
                                 disco_copy* copies, int64_t copy_capacity,
                                 int64_t counts[3], void* stream)
{
    using namespace disco;
    if (n < 0 || nloops < 0 || !box || !counts || (nloops > 0 && (!loops || !info)) ||
        (n > 0 && (!x || !y || !z || !x_out || !y_out || !z_out || !new_index)) ||
        slab_capacity < 0 || copy_capacity < 0 || (slab_capacity > 0 && (!slab_atoms || !slab_side)) ||
        (copy_capacity > 0 && !copies))
        return efail(DISCO_EINVAL, "null or negative argument");
    if (!(box[0] > 0.) || !(box[1] > 0.) || !(box[2] > 0.)) return efail(DISCO_EINVAL, "box lengths must be positive");
    if (n > kNoAllocMaxAtoms)
        return efail(DISCO_ELIMIT, "disco_b200_prismatic_noalloc takes at most 4194304 atoms (its scratch array is fixed)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* base = nullptr;
    int st = noalloc_scratch(&base);
    if (st) return st;
    SlabLoopDev* d_loops = reinterpret_cast<SlabLoopDev*>(base);
    int64_t* d_tot = reinterpret_cast<int64_t*>(base + align256(kNoAllocLoopBytes));
    int32_t* d_cnt = reinterpret_cast<int32_t*>(base + align256(kNoAllocLoopBytes) + align256(kNoAllocTotalsBytes));
    int32_t* d_off = d_cnt + kNoAllocMaxTiles * (kMaxSlabLoops + 1);

    // active loops, one record at a time from the stack (no host allocation)
    int nl = 0;
    int act_index[kMaxSlabLoops];
    cudaError_t e = cudaSuccess;
    for (int l = 0; l < nloops; ++l) {
        SlabLoopDev d;
        bool active = false;
        st = slab_loop_record(loops[l], l, box, info[l], d, active);
        if (st) return st;
        if (!active) continue;
        if (nl >= kMaxSlabLoops) return efail(DISCO_ELIMIT, "more than 64 prismatic loops in one call");
        e = cudaMemcpyAsync(d_loops + nl, &d, sizeof(d), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cfail(e, "loop table upload");
        act_index[nl++] = l;
    }
    const int C = nl + 1;
    const int64_t ntiles = (n + kSlabTile - 1) / kSlabTile;
    // the array keeps the previous call's contents: the totals must start at zero
    e = cudaMemsetAsync(d_tot, 0, kNoAllocTotalsBytes, s);
    if (e != cudaSuccess) return cfail(e, "totals reset");

    SlabArgs a;
    std::memset(&a, 0, sizeof(a));
    a.x = x; a.y = y; a.z = z;
    a.n = n;
    a.loops = d_loops;
    a.nl = nl;
    a.Lx = box[0]; a.Ly = box[1]; a.Lz = box[2];
    a.iLx = (float)(1.0 / box[0]); a.iLy = (float)(1.0 / box[1]); a.iLz = (float)(1.0 / box[2]);
    a.tile_counts = d_cnt;
    a.tile_offsets = d_off;
    a.totals = d_tot;
    a.xo = x_out; a.yo = y_out; a.zo = z_out;
    a.new_index = new_index;
    a.slab_atoms = slab_atoms;
    a.slab_side = slab_side;
    const size_t smem = (size_t)nl * sizeof(SlabLoopDev);
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(slab_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(slab_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cfail(e, "prismatic smem");
    }
    if (ntiles > 0) slab_count_kernel<<<slab_grid(ntiles), kSlabThreads, smem, s>>>(a);
    slab_scan_kernel<<<(unsigned)C, 1024, 0, s>>>(a, ntiles);
    int64_t tot[2 * (kMaxSlabLoops + 1) + 1];
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(tot, d_tot, (size_t)(2 * C) * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cfail(e, "prismatic count/scan");
    int64_t slab_total = 0, inter_total = 0;
    for (int q = 0; q < nl; ++q) {
        slab_total += tot[1 + q];
        // copies can only come from interstitial slabs
        disco_slab_info& in = info[act_index[q]];
        if (in.type == DISCO_MATTER_INTERSTITIAL) inter_total += tot[1 + q];
        in.offset = tot[C + q];
        in.count = tot[1 + q];
    }
    {
        int64_t next = slab_total;
        for (int l = nloops - 1; l >= 0; --l) {
            if (info[l].type == DISCO_MATTER_NONE) info[l].offset = next;
            else next = info[l].offset;
        }
    }
    counts[0] = tot[0];
    counts[1] = slab_total;
    counts[2] = inter_total;         // upper bound until the copies pass has run
    if (slab_total > slab_capacity)
        return efail(DISCO_ELIMIT, "slab capacity too small (counts[1] holds the size needed)");
    if (ntiles > 0) slab_scatter_kernel<<<slab_grid(ntiles), kSlabThreads, smem, s>>>(a);
    slab_copies_kernel<<<1, 1024, 0, s>>>(a, copies, copy_capacity);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&tot[2 * C - 1], d_tot + (2 * C - 1), sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cfail(e, "prismatic scatter");
    counts[2] = tot[2 * C - 1];
    if (counts[2] > copy_capacity)
        return efail(DISCO_ELIMIT, "copy capacity too small (counts[2] holds the size needed)");
    return DISCO_OK;
}

} // extern "C"
