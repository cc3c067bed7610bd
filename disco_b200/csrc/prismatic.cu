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
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace disco {

constexpr int kMaxSlabLoops = 64;                       // active slab loops per call

struct SlabLoopDev {
    disco_slab_loop L;
    double tLo, tHi;       // slab bounds in units of d (Code/prismatic.cpp:58-59)
    double cuv, det;       // u.v and 1 - (u.v)^2 (Code/loop.cpp:327-328)
    double inv_sp;         // 1 / d, rounded (the division's fast path)
    double pad;
};

// ---- the predicate, FP64 round-to-nearest, reference operation order -------------------

// r - L * floor(r / L + 0.5)   (Code/prismatic.cpp:31-34).  The image index
// comes from r times the rounded 1/L unless r/L + 1/2 lies within 1e-9 of an
// integer: the product and the exact quotient differ by under 4e-16 |r/L|
// (|r/L| < 1e6 here), so away from that margin both give the same floor;
// near it (or farther out) the exact quotient is taken.  The result is then
// formed exactly as the reference forms it.
__device__ __forceinline__ double min_image(double r, double L, double invL)
{
    const double q = r * invL;
    const double h = q + 0.5;
    const double f = floor(h);
    const double fr = h - f;
    const double m = (fabs(q) < 1e6 && fr > 1e-9 && fr < 1.0 - 1e-9)
                         ? f : floor(__dadd_rn(__ddiv_rn(r, L), 0.5));
    return __dsub_rn(r, __dmul_rn(L, m));
}

__device__ __forceinline__ double dot3_rn(double a0, double a1, double a2, double b0, double b1, double b2)
{
    return __dadd_rn(__dadd_rn(__dmul_rn(a0, b0), __dmul_rn(a1, b1)), __dmul_rn(a2, b2));
}

// Code/loop.cpp:281-316
__device__ bool inside_uv_rn(const disco_slab_loop& g, double u, double v)
{
    const double eps = 1e-9;
    if (g.shape == DISCO_SHAPE_CIRCLE) {
        // sqrt(x) < y without the square root unless x is within 1e-14 of y^2
        const double x = __dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), y = __dsub_rn(g.radius, eps);
        const double y2 = y * y;
        if (y > 0.0 && x < y2 * (1.0 - 1e-14)) return true;
        if (y > 0.0 && x > y2 * (1.0 + 1e-14)) return false;
        return __dsqrt_rn(x) < y;
    }
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

// Slab membership of one atom (Code/prismatic.cpp:61-72); side = sign of s.
// Every value that decides it is the reference's, rounded as the reference
// rounds it; divisions are skipped only where the decision provably does not
// depend on them: t = s / d against the slab bounds from s times the rounded
// 1/d unless that lies within 1e-9 planes of a bound, and the in-plane
// coordinates' division by det = 1 - (u.v)^2 when det is exactly 1.
__device__ __noinline__ bool slab_member(const SlabLoopDev& S, double x, double y, double z,
                                         double Lx, double Ly, double Lz, double iLx, double iLy, double iLz,
                                         bool& pos_side)
{
    const disco_slab_loop& g = S.L;
    const double r0 = min_image(__dsub_rn(x, g.c[0]), Lx, iLx);
    const double r1 = min_image(__dsub_rn(y, g.c[1]), Ly, iLy);
    const double r2 = min_image(__dsub_rn(z, g.c[2]), Lz, iLz);
    const double s = dot3_rn(r0, r1, r2, g.n[0], g.n[1], g.n[2]);
    const double tf = s * S.inv_sp;
    const double dlt = 1e-9 * (fabs(tf) + 1.0);
    if (tf < S.tLo - dlt || tf >= S.tHi + dlt) return false;
    if (!(tf >= S.tLo + dlt && tf < S.tHi - dlt)) {
        const double t = __ddiv_rn(s, g.spacing);
        if (t < S.tLo || t >= S.tHi) return false;
    }
    const double ru = dot3_rn(r0, r1, r2, g.u[0], g.u[1], g.u[2]);
    const double rv = dot3_rn(r0, r1, r2, g.v[0], g.v[1], g.v[2]);
    const double nu = __dsub_rn(ru, __dmul_rn(S.cuv, rv));
    const double nv = __dsub_rn(rv, __dmul_rn(S.cuv, ru));
    const double uu = S.det == 1.0 ? nu : __ddiv_rn(nu, S.det);
    const double vv = S.det == 1.0 ? nv : __ddiv_rn(nv, S.det);
    if (!inside_uv_rn(g, uu, vv)) return false;
    pos_side = s > 0.;
    return true;
}

// Per-loop header staged in shared memory: what the tile culling and the FP32
// pre-test read for every atom (the full record stays in global memory and is
// read only for the exact test).
struct SlabHead {
    double cx, cy, cz;     // centre (FP64)
    double bound;          // |r| of every slab member is below this (A)
    float nf[3], cf[3];    // pre-test: n, c
    float inv_df, margin;  // 1 / spacing, margin in planes
    float tlo, thi;        // slab bounds in planes
    int32_t type;          // DISCO_MATTER_VACANCY or DISCO_MATTER_INTERSTITIAL
    int32_t pad;
};
static_assert(sizeof(SlabHead) == 80, "slab header layout");

// One slab-member atom, in atom order: which loops' slabs it is in and on
// which side, and whether a vacancy slab removes it.
struct MemberRec {
    int32_t atom;
    int32_t removed;
    uint64_t mask, sides;
};

constexpr int kMatterThreads = 256;
constexpr int kMatterAtoms = 8;                                // per thread
constexpr int kMatterTile = kMatterThreads * kMatterAtoms;     // 2048 atoms per tile
constexpr int kMatterWarps = kMatterThreads / 32;
constexpr int kMaxCats = 2 + 2 * kMaxSlabLoops;                // look-back categories
constexpr int kWarpQueue = 128;                                // exact tests queued per warp
constexpr size_t kMatterSmem = 2 * kMatterTile * sizeof(uint64_t); // masks and sides of a tile

// Tile flags of the look-back: 0 not yet published, 1 the tile's counts
// (agg) are published, 2 its inclusive prefixes (inc) are too.
constexpr int kFlagAgg = 1;
constexpr int kFlagInc = 2;

struct MatterArgs {
    const double *x, *y, *z;
    int64_t n;
    const SlabHead* heads;        // [nl]
    const SlabLoopDev* loops;     // [nl]
    int32_t nl, C;                // C = 2 + 2 nl categories: survivors, members, slab of
                                  // loop l (2 + l), kept copies of loop l (2 + nl + l)
    double Lx, Ly, Lz;
    float iLx, iLy, iLz;          // 1 / box lengths in FP32 (the pre-test only)
    int32_t pad_;
    double idLx, idLy, idLz;      // 1 / box lengths, rounded (the exact test's fast path)
    int* flags;                   // [ntiles] look-back flags, zeroed per call
    unsigned int* ticket;         // tile counter, zeroed per call
    int32_t* agg;                 // [ntiles][C] the tile's counts
    int32_t* inc;                 // [ntiles][C] inclusive prefixes (exclusive = inc - agg)
    MemberRec* members;
    int64_t member_cap;
    double *xo, *yo, *zo;
    int32_t* new_index;
    int32_t* slab_atoms;
    int8_t* slab_side;
    int64_t slab_cap;
    disco_copy* copies;
    int64_t copy_cap;
    int64_t* totals;              // [C] category totals (written by the tail)
    int* err;
};

__device__ __forceinline__ void st_release(int* p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Cheap pre-test in FP32: true only if the atom's t is outside [tLo, tHi) by
// more than `margin` planes.  With the atom and the centre within 2 L of the
// origin and rounded to FP32, and the nearest image unambiguous (r/L + 1/2 at
// least 1e-5 from an integer and |r/L| < 2; else it returns false), the FP32
// t differs from the exactly rounded t of slab_member by less than
// 1.5e-6 (Lx + Ly + Lz) / d + 1e-6 planes; the margin is
// 1e-5 (Lx + Ly + Lz) / d + 1e-3.  So it never rejects a member: the exact
// test decides every atom it passes, and atom sets stay bit-exact.
__device__ __forceinline__ bool clearly_outside(const SlabHead& S, const float (&p)[3], const float (&L)[3],
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
        sure = sure && fabsf(q) < 2.0f && fr >= 1e-5f && fr <= 1.0f - 1e-5f &&
               fabsf(p[k]) < 2.0f * L[k] && fabsf(S.cf[k]) < 2.0f * L[k];
        s = fmaf(S.nf[k], fmaf(-L[k], f, r), s);
    }
    const float t = s * S.inv_df;
    return sure && (t < S.tlo - S.margin || t >= S.thi + S.margin);
}

// Smallest |p - c - m L| over p in [lo, hi] and integers m, less a rounding
// allowance (never above the true value).
__device__ __forceinline__ double periodic_gap(double lo, double hi, double c, double L)
{
    const double a = lo - c, b = hi - c;
    if (!(b - a < L)) return 0.0;
    const double m1 = floor(a / L);
    if ((m1 + 1.0) * L <= b) return 0.0;
    const double d = fmin(a - m1 * L, (m1 + 1.0) * L - b);
    return fmax(0.0, d - 1e-9 * L - 1e-6);
}

// The loops among `cand` (loops whose slab can reach the atom's warp) that the
// FP32 pre-test cannot exclude for this atom: its exact-test candidates.
__device__ __forceinline__ uint64_t pretest(const SlabHead* sh, uint64_t cand, double x, double y, double z,
                                            const MatterArgs& a)
{
    const float L[3] = { (float)a.Lx, (float)a.Ly, (float)a.Lz };
    const float iL[3] = { a.iLx, a.iLy, a.iLz };
    const float p[3] = { (float)x, (float)y, (float)z };
    uint64_t c2 = 0;
    for (uint64_t c = cand; c; c &= c - 1) {
        const int l = __ffsll((long long)c) - 1;
        if (!clearly_outside(sh[l], p, L, iL)) c2 |= 1ull << l;
    }
    return c2;
}

// The matter step's single pass over the atoms.  Each CTA takes the next tile
// of 2048 atoms (a ticket, so that every tile it looks back on belongs to a
// CTA already running); each warp owns 256 consecutive atoms of it (8 rounds
// of 32, coalesced), reads them once, takes their bounding box and skips every
// loop whose slab cannot reach it, and computes each atom's slab mask once
// (kept in shared memory for the ranked writes).  Per category the tile's
// count is published and its exclusive prefix obtained by decoupled
// look-back over the preceding tiles' published counts; survivors (x, y, z,
// new index) and the slab members' records are then written at their final
// ranks.  Bounded waits: a look-back that finds no count for 2 s records
// DISCO_ETIMEOUT and publishes anyway, so no tile waits forever.
// Dynamic shared memory: kMatterTile masks and sides (32 KB); four CTAs per
// SM, so that one CTA's barriers and look-back overlap the others' loads.
__global__ void __launch_bounds__(kMatterThreads, 4) matter_pass_kernel(const MatterArgs a)
{
    extern __shared__ __align__(16) unsigned char dyn[];
    uint64_t* smask = reinterpret_cast<uint64_t*>(dyn);
    uint64_t* ssides = smask + kMatterTile;
    __shared__ SlabHead sh[kMaxSlabLoops];
    __shared__ int cnt_s[kMatterWarps * kMatterAtoms];         // survivors per (warp, round), then prefixes
    __shared__ int cnt_m[kMatterWarps * kMatterAtoms];         // members per (warp, round), then prefixes
    __shared__ int cnt_c[2 * kMaxSlabLoops];                   // slab and kept-copy counts per loop
    __shared__ int64_t excl[kMaxCats];
    __shared__ int aggv[2];
    __shared__ int s_k;
    __shared__ int wq[kMatterWarps][kWarpQueue];                // per warp: (slot, loop) pairs to test
    __shared__ int wq_n[kMatterWarps];
    __shared__ unsigned long long vac_s;
    __shared__ int tile_s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nl = a.nl, C = a.C;
    if (tid == 0) { tile_s = (int)atomicAdd(a.ticket, 1u); vac_s = 0ull; }
    {
        const int words = nl * (int)(sizeof(SlabHead) / 8);
        const uint64_t* src = reinterpret_cast<const uint64_t*>(a.heads);
        uint64_t* dst = reinterpret_cast<uint64_t*>(sh);
        for (int i = tid; i < words; i += kMatterThreads) dst[i] = src[i];
        for (int i = tid; i < 2 * nl; i += kMatterThreads) cnt_c[i] = 0;
    }
    __syncthreads();
    if (tid < nl && sh[tid].type == DISCO_MATTER_VACANCY) atomicOr(&vac_s, 1ull << tid);
    const int64_t tile = tile_s;
    const int64_t wbase = tile * kMatterTile + (int64_t)warp * (32 * kMatterAtoms);   // this warp's atoms

    // the warp's bounding box (its atoms come from HBM here; the later reads
    // of the same 6 KB hit L1/L2) and the loops whose slab can reach it
    double lo[3] = { 1e300, 1e300, 1e300 }, hi[3] = { -1e300, -1e300, -1e300 };
#pragma unroll
    for (int r = 0; r < kMatterAtoms; ++r) {
        const int64_t i = wbase + r * 32 + lane;
        if (i < a.n) {
            const double px = a.x[i], py = a.y[i], pz = a.z[i];
            lo[0] = fmin(lo[0], px); hi[0] = fmax(hi[0], px);
            lo[1] = fmin(lo[1], py); hi[1] = fmax(hi[1], py);
            lo[2] = fmin(lo[2], pz); hi[2] = fmax(hi[2], pz);
        }
    }
    uint64_t wmask = 0;
    if (nl > 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
            for (int o = 16; o > 0; o >>= 1) {
                lo[k] = fmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
                hi[k] = fmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
            }
        for (int half = 0; half < 2; ++half) {
            const int l = lane + 32 * half;
            bool reach = false;
            if (l < nl && lo[0] <= hi[0]) {
                const SlabHead& S = sh[l];
                const double gx = periodic_gap(lo[0], hi[0], S.cx, a.Lx);
                const double gy = periodic_gap(lo[1], hi[1], S.cy, a.Ly);
                const double gz = periodic_gap(lo[2], hi[2], S.cz, a.Lz);
                reach = !(gx * gx + gy * gy + gz * gz > S.bound * S.bound);
            }
            wmask |= (uint64_t)__ballot_sync(0xffffffffu, reach) << (32 * half);
        }
    }
    __syncthreads();                                        // vac_s
    const uint64_t vac = vac_s;

    // every atom's mask, once: the FP32 pre-test per atom, its candidate
    // (atom, loop) pairs queued per warp, the exact FP64 tests of the queue
    // spread over the warp's lanes (one latency chain per 32 pairs rather than
    // one per round and loop), then the counts per (warp, round) and per loop
    const int wt = warp * (32 * kMatterAtoms);              // the warp's first atom in the tile
    if (lane == 0) wq_n[warp] = 0;
    __syncwarp();
#pragma unroll 1
    for (int r = 0; r < kMatterAtoms; ++r) {
        const int64_t i = wbase + r * 32 + lane;
        uint64_t cand = 0;
        if (i < a.n && wmask) cand = pretest(sh, wmask, a.x[i], a.y[i], a.z[i], a);
        smask[wt + r * 32 + lane] = 0;
        ssides[wt + r * 32 + lane] = 0;
        for (uint64_t c = cand; c; c &= c - 1) {
            const int l = __ffsll((long long)c) - 1;
            const int q = atomicAdd(&wq_n[warp], 1);
            if (q < kWarpQueue) {
                wq[warp][q] = (r * 32 + lane) | (l << 16);
            } else {                                         // a full queue: test here
                bool ps = false;
                if (slab_member(a.loops[l], a.x[i], a.y[i], a.z[i], a.Lx, a.Ly, a.Lz, a.idLx, a.idLy, a.idLz, ps)) {
                    smask[wt + r * 32 + lane] |= 1ull << l;
                    if (ps) ssides[wt + r * 32 + lane] |= 1ull << l;
                }
            }
        }
    }
    __syncwarp();
    {
        const int nq = min(wq_n[warp], kWarpQueue);
        for (int q = lane; q < nq; q += 32) {
            const int slot = wq[warp][q] & 0xffff, l = wq[warp][q] >> 16;
            const int64_t i = wbase + slot;
            bool ps = false;
            if (slab_member(a.loops[l], a.x[i], a.y[i], a.z[i], a.Lx, a.Ly, a.Lz, a.idLx, a.idLy, a.idLz, ps)) {
                atomicOr(reinterpret_cast<unsigned long long*>(&smask[wt + slot]), 1ull << l);
                if (ps) atomicOr(reinterpret_cast<unsigned long long*>(&ssides[wt + slot]), 1ull << l);
            }
        }
    }
    __syncwarp();
#pragma unroll 1
    for (int r = 0; r < kMatterAtoms; ++r) {
        const int64_t i = wbase + r * 32 + lane;
        const uint64_t mask = smask[wt + r * 32 + lane];
        const bool removed = (mask & vac) != 0;
        const unsigned bs = __ballot_sync(0xffffffffu, i < a.n && !removed);
        const unsigned bm = __ballot_sync(0xffffffffu, mask != 0);
        if (lane == 0) { cnt_s[warp * kMatterAtoms + r] = __popc(bs); cnt_m[warp * kMatterAtoms + r] = __popc(bm); }
        for (uint64_t m = mask; m; m &= m - 1) {             // members are rare
            const int l = __ffsll((long long)m) - 1;
            atomicAdd(&cnt_c[l], 1);
            if (sh[l].type == DISCO_MATTER_INTERSTITIAL && !removed) atomicAdd(&cnt_c[nl + l], 1);
        }
    }
    __syncthreads();

    // warps 0 and 1: prefixes over (warp, round) in atom order and the tile's
    // survivor and member counts
    if (warp < 2) {
        int* cnt = warp == 0 ? cnt_s : cnt_m;
        constexpr int kPer = kMatterAtoms * kMatterWarps / 32;  // 2 entries per lane
        int v[kPer], tot = 0;
#pragma unroll
        for (int j = 0; j < kPer; ++j) { v[j] = cnt[lane * kPer + j]; tot += v[j]; }
        int incl = tot;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        int run = incl - tot;
#pragma unroll
        for (int j = 0; j < kPer; ++j) { cnt[lane * kPer + j] = run; run += v[j]; }
        if (lane == 31) aggv[warp] = incl;
    }
    __syncthreads();

    // decoupled look-back: publish the tile's counts, then one warp scans the
    // flags of the 32 preceding tiles at a time for the nearest published
    // inclusive prefix (every tile between must have published its counts),
    // and every category's thread sums that window's values
    const int32_t my_agg = tid < C ? (tid < 2 ? aggv[tid] : cnt_c[tid - 2]) : 0;
    if (tid < C) {
        a.agg[tile * C + tid] = my_agg;
        if (tile == 0) a.inc[tid] = my_agg;
        __threadfence();
    }
    __syncthreads();
    if (tid == 0) st_release(a.flags + tile, tile == 0 ? kFlagInc : kFlagAgg);
    int64_t pre = 0;
    if (tile > 0) {
        int64_t jhi = tile - 1;                                 // top of the window
        while (true) {
            if (warp == 0) {
                unsigned long long t0 = 0;
                int k;
                while (true) {
                    const int64_t j = jhi - lane;
                    const int f = j >= 0 ? ld_acquire(a.flags + j) : kFlagAgg;
                    const unsigned bi = __ballot_sync(0xffffffffu, f == kFlagInc);
                    const unsigned br = __ballot_sync(0xffffffffu, f >= kFlagAgg);
                    k = bi ? __ffs(bi) - 1 : 32;                 // nearest inclusive prefix
                    const unsigned need = k == 32 ? 0xffffffffu : ((1u << k) - 1u);
                    if ((br & need) == need) break;
                    if (t0 == 0) t0 = global_ns();
                    else if (global_ns() - t0 > kWaitLimitNs) {
                        if (lane == 0) report(a.err, DISCO_ETIMEOUT);
                        k = -1;
                        break;
                    }
                }
                if (lane == 0) s_k = k;
            }
            __syncthreads();
            const int k = s_k;
            if (k < 0) break;                                   // gave up: publish anyway
            if (tid < C) {
                for (int q = 0; q < k; ++q) pre += __ldcg(a.agg + (jhi - q) * C + tid);
                if (k < 32) pre += __ldcg(a.inc + (jhi - k) * C + tid);
            }
            if (k < 32) break;
            jhi -= 32;
            __syncthreads();                                    // s_k is rewritten
        }
    }
    if (tid < C) {
        if (tile > 0) a.inc[tile * C + tid] = (int32_t)(pre + my_agg);
        excl[tid] = pre;
        __threadfence();
    }
    __syncthreads();
    if (tid == 0 && tile > 0) st_release(a.flags + tile, kFlagInc);

    // survivors at their final ranks, the new-index map, member records
    const unsigned ltm = (1u << lane) - 1u;
#pragma unroll 2
    for (int r = 0; r < kMatterAtoms; ++r) {
        const int64_t i = wbase + r * 32 + lane;
        const bool valid = i < a.n;
        const uint64_t mask = smask[wt + r * 32 + lane];
        const bool surv = valid && !(mask & vac);
        const unsigned bs = __ballot_sync(0xffffffffu, surv);
        const unsigned bm = __ballot_sync(0xffffffffu, mask != 0);
        if (valid) {
            if (surv) {
                const int64_t q = excl[0] + cnt_s[warp * kMatterAtoms + r] + __popc(bs & ltm);
                if (q < a.n) { a.xo[q] = a.x[i]; a.yo[q] = a.y[i]; a.zo[q] = a.z[i]; }
                a.new_index[i] = (int32_t)q;
            } else {
                a.new_index[i] = -1;
            }
        }
        if (mask) {
            const int64_t q = excl[1] + cnt_m[warp * kMatterAtoms + r] + __popc(bm & ltm);
            if (q < a.member_cap) {
                MemberRec m;
                m.atom = (int32_t)i;
                m.removed = (mask & vac) != 0;
                m.mask = mask;
                m.sides = ssides[wt + r * 32 + lane];
                a.members[q] = m;
            }
        }
    }
}

// The slab entries and the interstitial copies, from the member records of
// each tile (tiles spread over the CTAs, after the pass): entry of loop l
// at loop base + the tile's exclusive count of loop l + its rank among the
// tile's members in l (ascending atom order, Code/prismatic.cpp:61-72); a copy
// of an interstitial loop's entry whose atom survives at copy base + the tile's
// exclusive kept count + its rank (loop order, then slab order; sources
// renumbered, Code/main.cpp:651-654,676-679).  CTA 0 also writes the totals.
__global__ void __launch_bounds__(256) matter_tail_kernel(const MatterArgs a, int64_t ntiles)
{
    __shared__ int64_t tot[kMaxCats];
    __shared__ int64_t lbase[kMaxSlabLoops], cbase[kMaxSlabLoops];
    __shared__ int run[2 * kMaxSlabLoops];
    __shared__ int wc[8][2];
    __shared__ unsigned long long umask;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nl = a.nl, C = a.C;
    // totals = the last tile's inclusive counts; loop and copy bases
    for (int c = tid; c < C; c += 256) tot[c] = a.inc[(ntiles - 1) * C + c];
    __syncthreads();
    if (tid == 0) {
        int64_t sb = 0, cb = 0;
        for (int l = 0; l < nl; ++l) {
            lbase[l] = sb; sb += tot[2 + l];
            cbase[l] = cb; cb += tot[2 + nl + l];
        }
        if (blockIdx.x == 0) {
            for (int c = 0; c < C; ++c) a.totals[c] = tot[c];
            a.totals[C] = *a.err;                              // the pass's error word
            *a.err = 0;                                        // ticket and error word cleared
            *a.ticket = 0;                                     // for the next call
        }
    }
    // this CTA's tiles (grid-stride): each tile's flag cleared for the next
    // call (the pass is over), its member records turned into entries
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        if (tid == 0) a.flags[t] = 0;
        const int64_t mend = a.inc[t * C + 1];                           // this tile's member records
        const int64_t m0 = mend - a.agg[t * C + 1];
        if (mend == m0) continue;
        __syncthreads();                                    // run / umask of the previous tile
        if (tid == 0) umask = 0ull;
        for (int i = tid; i < 2 * nl; i += 256) run[i] = 0;
        __syncthreads();
        for (int64_t e0 = m0; e0 < mend; e0 += 256) {
            const int64_t e = e0 + tid;
            MemberRec m;
            m.atom = 0; m.removed = 1; m.mask = 0; m.sides = 0;
            if (e < mend && e < a.member_cap) m = a.members[e];
            if (m.mask) atomicOr(&umask, m.mask);
            __syncthreads();
            const uint64_t um = umask;
            for (uint64_t u = um; u; u &= u - 1) {
                const int l = __ffsll((long long)u) - 1;
                const bool in = (m.mask >> l) & 1ull;
                const bool keep = in && !m.removed && a.heads[l].type == DISCO_MATTER_INTERSTITIAL;
                const unsigned bi = __ballot_sync(0xffffffffu, in);
                const unsigned bk = __ballot_sync(0xffffffffu, keep);
                if (lane == 0) { wc[warp][0] = __popc(bi); wc[warp][1] = __popc(bk); }
                __syncthreads();
                int pi = run[l], pk = run[nl + l];
                for (int w = 0; w < warp; ++w) { pi += wc[w][0]; pk += wc[w][1]; }
                const unsigned ltm = (1u << lane) - 1u;
                if (in) {
                    const int64_t q = lbase[l] + (a.inc[t * C + 2 + l] - a.agg[t * C + 2 + l]) + pi +
                                      __popc(bi & ltm);
                    if (q < a.slab_cap) {
                        a.slab_atoms[q] = m.atom;
                        a.slab_side[q] = ((m.sides >> l) & 1ull) ? 1 : -1;
                    }
                }
                if (keep) {
                    const int64_t q = cbase[l] + (a.inc[t * C + 2 + nl + l] - a.agg[t * C + 2 + nl + l]) + pk +
                                      __popc(bk & ltm);
                    if (q < a.copy_cap) {
                        const disco_slab_loop& g = a.loops[l].L;
                        const double* sh = ((m.sides >> l) & 1ull) ? g.shift_pos : g.shift_neg;
                        disco_copy cp;
                        cp.atom = a.new_index[m.atom];
                        cp.reserved = 0;
                        cp.shift[0] = sh[0]; cp.shift[1] = sh[1]; cp.shift[2] = sh[2];
                        a.copies[q] = cp;
                    }
                }
                __syncthreads();
                if (tid == 0) {
                    for (int w = 0; w < 8; ++w) { run[l] += wc[w][0]; run[nl + l] += wc[w][1]; }
                }
                __syncthreads();
            }
            if (tid == 0) umask = 0ull;
            __syncthreads();
        }
    }
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

// One loop's SlabResult scalars (Code/prismatic.cpp:42-57) and, when it is
// active (b.n != 0 and apply), its device header and record.  Never allocates.
int slab_loop_record(const disco_slab_loop& g, const double box[3], disco_slab_info& in,
                     disco::SlabHead& h, disco::SlabLoopDev& d, bool& active)
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
    d.inv_sp = 1.0 / g.spacing;

    std::memset(&h, 0, sizeof(h));
    h.cx = g.c[0]; h.cy = g.c[1]; h.cz = g.c[2];
    for (int k = 0; k < 3; ++k) {
        h.nf[k] = (float)g.n[k];
        h.cf[k] = (float)g.c[k];
    }
    h.inv_df = (float)(1.0 / in.spacing);
    h.margin = (float)(1e-5 * (box[0] + box[1] + box[2]) / in.spacing + 1e-3);
    h.tlo = (float)d.tLo;
    h.thi = (float)d.tHi;
    h.type = type;
    // Bound on |r| (minimum image) of a member: the in-plane test holds for
    // (uu, vv) within rho of the origin (Code/loop.cpp:281-316), r = uu u + vv v
    // + s n with |s| <= max(|tLo|, tHi) d when u, v are unit vectors orthogonal
    // to n, and |uu u + vv v| <= rho sqrt(1 + |u.v|).  Any other frame: no bound.
    double rho;
    if (g.shape == DISCO_SHAPE_CIRCLE) {
        rho = g.radius;
    } else if (g.shape == DISCO_SHAPE_POLYGON) {
        rho = 0.0;
        for (int i = 0; i < g.n_poly; ++i)
            rho = std::max(rho, std::max(std::hypot(g.pu[i], g.pv[i]), std::hypot(g.qu[i], g.qv[i])));
        rho += std::max(g.r_corner, 0.0);
    } else {
        rho = std::hypot(g.half_m, g.half_p) + std::max(g.r_corner, 0.0);
    }
    const double uu = g.u[0] * g.u[0] + g.u[1] * g.u[1] + g.u[2] * g.u[2];
    const double vv = g.v[0] * g.v[0] + g.v[1] * g.v[1] + g.v[2] * g.v[2];
    const double nn = g.n[0] * g.n[0] + g.n[1] * g.n[1] + g.n[2] * g.n[2];
    const double un = g.u[0] * g.n[0] + g.u[1] * g.n[1] + g.u[2] * g.n[2];
    const double vn = g.v[0] * g.n[0] + g.v[1] * g.n[1] + g.v[2] * g.n[2];
    const bool frame = std::fabs(uu - 1.0) < 1e-9 && std::fabs(vv - 1.0) < 1e-9 && std::fabs(nn - 1.0) < 1e-9 &&
                       std::fabs(un) < 1e-9 && std::fabs(vn) < 1e-9 && std::isfinite(rho);
    const double smax = std::max(std::fabs(d.tLo), std::fabs(d.tHi)) * in.spacing;
    h.bound = frame ? (rho * std::sqrt(1.0 + std::fabs(c)) + smax) * (1.0 + 1e-9) + 1e-6 +
                      1e-9 * (box[0] + box[1] + box[2])
                    : HUGE_VAL;
    active = true;
    return DISCO_OK;
}

// Active loops in caller order into heads[] / recs[] (capacity kMaxSlabLoops).
int prepare_loops(const disco_slab_loop* loops, int nloops, const double box[3], disco_slab_info* info,
                  disco::SlabHead* heads, disco::SlabLoopDev* recs, int* act_index, int& nl)
{
    nl = 0;
    for (int l = 0; l < nloops; ++l) {
        bool active = false;
        disco::SlabHead h;
        disco::SlabLoopDev d;
        const int st = slab_loop_record(loops[l], box, info[l], h, d, active);
        if (st) return st;
        if (!active) continue;
        if (nl >= disco::kMaxSlabLoops) {
            disco::set_last_error("more than 64 prismatic loops in one call");
            return DISCO_ELIMIT;
        }
        heads[nl] = h;
        recs[nl] = d;
        act_index[nl++] = l;
    }
    return DISCO_OK;
}

// Host staging of the loop headers and records of one call: headers, then the
// records at recs_offset(nl), filled and uploaded with a single copy while
// g_stage_mutex is held (never from the stack).
struct LoopStage {
    disco::SlabHead heads[disco::kMaxSlabLoops];
    disco::SlabLoopDev recs[disco::kMaxSlabLoops];
};
std::mutex g_stage_mutex;
LoopStage g_stage_parts;
unsigned char g_stage_bytes[sizeof(LoopStage)];

size_t recs_offset(int nl) { return ((size_t)nl * sizeof(disco::SlabHead) + 15) & ~size_t(15); }

// What the last upload into the no-alloc scratch held (device, context,
// bytes): a call with the same loops on the same device skips the upload,
// since every call waits for its own work before it returns.
struct StageCache {
    unsigned char* dst = nullptr;
    unsigned long long ctx = 0;
    size_t bytes = 0;
    unsigned char data[sizeof(LoopStage)];
};
StageCache g_stage_cache;

void stage_cache_drop()
{
    std::lock_guard<std::mutex> lock(g_stage_mutex);
    g_stage_cache.dst = nullptr;
}

// prepare_loops into the staging buffer, then one upload of its used bytes
// to dst on stream s (skipped when `ctx` is non-zero and the same bytes were
// the last ones uploaded to dst in that context).
int stage_loops(const disco_slab_loop* loops, int nloops, const double box[3], disco_slab_info* info,
                int* act_index, int& nl, unsigned char* dst, cudaStream_t s, unsigned long long ctx = 0)
{
    std::lock_guard<std::mutex> lock(g_stage_mutex);
    int st = prepare_loops(loops, nloops, box, info, g_stage_parts.heads, g_stage_parts.recs, act_index, nl);
    if (st || nl == 0) return st;
    const size_t hb = (size_t)nl * sizeof(disco::SlabHead), off = recs_offset(nl);
    const size_t bytes = off + (size_t)nl * sizeof(disco::SlabLoopDev);
    std::memcpy(g_stage_bytes, g_stage_parts.heads, hb);
    std::memset(g_stage_bytes + hb, 0, off - hb);
    std::memcpy(g_stage_bytes + off, g_stage_parts.recs, (size_t)nl * sizeof(disco::SlabLoopDev));
    if (ctx && g_stage_cache.dst == dst && g_stage_cache.ctx == ctx && g_stage_cache.bytes == bytes &&
        std::memcmp(g_stage_cache.data, g_stage_bytes, bytes) == 0)
        return DISCO_OK;
    g_stage_cache.dst = nullptr;
    const cudaError_t e = cudaMemcpyAsync(dst, g_stage_bytes, bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cfail(e, "loop table upload");
    if (ctx) {
        g_stage_cache.dst = dst;
        g_stage_cache.ctx = ctx;
        g_stage_cache.bytes = bytes;
        std::memcpy(g_stage_cache.data, g_stage_bytes, bytes);
    }
    return DISCO_OK;
}

// Bytes of the look-back flags (ticket and error word first), cleared per call.
size_t status_bytes(int64_t ntiles) { return 16 + (size_t)ntiles * sizeof(int); }

struct MatterScratch {
    unsigned char* loops;        // heads then records (sizeof(LoopStage))
    unsigned char* status;       // status_bytes(ntiles)
    int32_t* agg;                // ntiles * C
    int32_t* inc;                // ntiles * C
    disco::MemberRec* members;
    int64_t member_cap;
    int64_t* totals;             // C + 1 (the last: the kernels' error word)
};

// Queues the matter step on stream s after stage_loops (no host wait): the
// look-back words cleared, the single pass, the tail.
int matter_queue(disco::MatterArgs& a, const MatterScratch& m, int nl, const int64_t ntiles, cudaStream_t s,
                 size_t clear_bytes)
{
    using namespace disco;
    cudaError_t e = cudaSuccess;
    a.heads = reinterpret_cast<const SlabHead*>(m.loops);
    a.loops = reinterpret_cast<const SlabLoopDev*>(m.loops + recs_offset(nl));
    a.nl = nl;
    a.C = 2 + 2 * nl;
    a.flags = reinterpret_cast<int*>(m.status + 16);
    a.ticket = reinterpret_cast<unsigned int*>(m.status);
    a.err = reinterpret_cast<int*>(m.status + 4);
    a.agg = m.agg;
    a.inc = m.inc;
    a.members = m.members;
    a.member_cap = m.member_cap;
    a.totals = m.totals;
    // the tail of every completed call leaves the flags, ticket and error word
    // at zero; a caller that cannot rely on that (fresh memory, a call that
    // failed half-way) clears them here
    if (clear_bytes) {
        e = cudaMemsetAsync(m.status, 0, clear_bytes, s);
        if (e != cudaSuccess) return cfail(e, "look-back reset");
    }
    if (kMatterSmem > 48 * 1024) {
        e = cudaFuncSetAttribute(matter_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMatterSmem);
        if (e != cudaSuccess) return cfail(e, "matter step shared memory");
    }
    if (ntiles > 0) {
        matter_pass_kernel<<<(unsigned)ntiles, kMatterThreads, kMatterSmem, s>>>(a);
        matter_tail_kernel<<<(unsigned)std::min<int64_t>(ntiles, 512), 256, 0, s>>>(a, ntiles);
    } else {
        e = cudaMemsetAsync(m.totals, 0, (size_t)(a.C + 1) * sizeof(int64_t), s);
        if (e != cudaSuccess) return cfail(e, "totals reset");
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cfail(e, "matter step launch");
    return DISCO_OK;
}

// After the stream has reached the end of the step: counts, info offsets and
// the capacity checks from the totals (host copy tot[0..C], tot[C] = error).
int matter_finish(const int64_t* tot, int nl, const int* act_index, int nloops, disco_slab_info* info,
                  int64_t slab_capacity, int64_t copy_capacity, int64_t member_cap, int64_t counts[3])
{
    if (tot[2 + 2 * nl]) return efail(DISCO_ETIMEOUT, "matter step: a bounded device wait gave up");
    int64_t slab_total = 0, copy_total = 0;
    for (int q = 0; q < nl; ++q) {
        disco_slab_info& in = info[act_index[q]];
        in.offset = slab_total;
        in.count = tot[2 + q];
        slab_total += tot[2 + q];
        copy_total += tot[2 + nl + q];
    }
    {
        int64_t next = slab_total;       // inactive loops: empty range where the next active one starts
        for (int l = nloops - 1; l >= 0; --l) {
            if (info[l].type == DISCO_MATTER_NONE) info[l].offset = next;
            else next = info[l].offset;
        }
    }
    counts[0] = tot[0];
    counts[1] = slab_total;
    counts[2] = copy_total;
    if (slab_total > slab_capacity || copy_total > copy_capacity)
        return efail(DISCO_ELIMIT, "slab or copy capacity too small (counts hold the sizes needed)");
    if (tot[1] > member_cap)
        return efail(DISCO_ELIMIT, "more atoms in slabs than the member list holds");
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
    int act_index[kMaxSlabLoops];
    int nl = 0;
    for (int l = 0; l < nloops; ++l) {                  // count the active loops first (sizes)
        disco_slab_info in;
        SlabHead h;
        SlabLoopDev d;
        bool active = false;
        const int st0 = slab_loop_record(loops[l], box, in, h, d, active);
        if (st0) return st0;
        nl += active;
    }
    if (nl > kMaxSlabLoops) return efail(DISCO_ELIMIT, "more than 64 prismatic loops in one call");
    const int C = 2 + 2 * nl;
    const int64_t ntiles = (n + kMatterTile - 1) / kMatterTile;
    const int64_t member_cap = std::max<int64_t>(1, std::min<int64_t>(n, slab_capacity));
    const int64_t scap = std::max<int64_t>(1, slab_capacity), ccap = std::max<int64_t>(1, copy_capacity);

    DevBuf dxyz, dout, didx, dloops, dstat, dagg, dmem, dtot, dslab, dside, dcop;
    const size_t nb = (size_t)n * sizeof(double);
    cudaError_t e = cudaSuccess;
    if (n > 0) {
        e = cudaMalloc(&dxyz.p, 3 * nb);
        if (e == cudaSuccess) e = cudaMalloc(&dout.p, 3 * nb);
        if (e == cudaSuccess) e = cudaMalloc(&didx.p, (size_t)n * sizeof(int32_t));
    }
    if (e == cudaSuccess) e = cudaMalloc(&dloops.p, sizeof(LoopStage));
    if (e == cudaSuccess) e = cudaMalloc(&dstat.p, status_bytes(ntiles));
    if (e == cudaSuccess) e = cudaMalloc(&dagg.p, 2 * std::max<int64_t>(1, ntiles * C) * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&dmem.p, (size_t)member_cap * sizeof(MemberRec));
    if (e == cudaSuccess) e = cudaMalloc(&dtot.p, (size_t)(C + 1) * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&dslab.p, (size_t)scap * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&dside.p, (size_t)scap);
    if (e == cudaSuccess) e = cudaMalloc(&dcop.p, (size_t)ccap * sizeof(disco_copy));
    if (e != cudaSuccess) return cfail(e, "prismatic allocation");
    if (n > 0) {
        e = cudaMemcpy(dxyz.as<double>(), x, nb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dxyz.as<double>() + n, y, nb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dxyz.as<double>() + 2 * n, z, nb, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) return cfail(e, "prismatic upload");
    int st = stage_loops(loops, nloops, box, info, act_index, nl, dloops.as<unsigned char>(), nullptr);
    if (st) return st;

    MatterArgs a;
    std::memset(&a, 0, sizeof(a));
    a.x = dxyz.as<double>(); a.y = a.x + n; a.z = a.x + 2 * n;
    a.n = n;
    a.Lx = box[0]; a.Ly = box[1]; a.Lz = box[2];
    a.iLx = (float)(1.0 / box[0]); a.iLy = (float)(1.0 / box[1]); a.iLz = (float)(1.0 / box[2]);
    a.idLx = 1.0 / box[0]; a.idLy = 1.0 / box[1]; a.idLz = 1.0 / box[2];
    a.xo = dout.as<double>(); a.yo = a.xo + n; a.zo = a.xo + 2 * n;
    a.new_index = didx.as<int32_t>();
    a.slab_atoms = dslab.as<int32_t>();
    a.slab_side = dside.as<int8_t>();
    a.slab_cap = slab_capacity;
    a.copies = dcop.as<disco_copy>();
    a.copy_cap = copy_capacity;
    MatterScratch m;
    m.loops = dloops.as<unsigned char>();
    m.status = dstat.as<unsigned char>();
    m.agg = dagg.as<int32_t>();
    m.inc = m.agg + std::max<int64_t>(1, ntiles * C);
    m.members = dmem.as<MemberRec>();
    m.member_cap = member_cap;
    m.totals = dtot.as<int64_t>();
    st = matter_queue(a, m, nl, ntiles, nullptr, status_bytes(ntiles));
    if (st) return st;
    int64_t tot[kMaxCats + 1];
    e = cudaMemcpy(tot, m.totals, (size_t)(C + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cfail(e, "prismatic totals");
    st = matter_finish(tot, nl, act_index, nloops, info, slab_capacity, copy_capacity, member_cap, counts);
    if (st) return st;
    const int64_t k = counts[0];
    if (n > 0) {
        e = cudaMemcpy(new_index, didx.p, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && k > 0) e = cudaMemcpy(x_out, a.xo, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && k > 0) e = cudaMemcpy(y_out, a.yo, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && k > 0) e = cudaMemcpy(z_out, a.zo, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess && counts[1] > 0)
        e = cudaMemcpy(slab_atoms, dslab.p, (size_t)counts[1] * sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && counts[1] > 0)
        e = cudaMemcpy(slab_side, dside.p, (size_t)counts[1], cudaMemcpyDeviceToHost);
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
// from the caller and keeps its scratch (loop table, look-back words, per-tile
// prefixes, member records, totals) in the file-scope array below: 4 MiB
// that every GPU loading this library holds until the process exits.

namespace {

constexpr int64_t kNoAllocMaxAtoms = int64_t(1) << 22;                  // 4 194 304 atoms
constexpr int64_t kNoAllocMaxTiles = kNoAllocMaxAtoms / disco::kMatterTile;
constexpr int64_t kNoAllocMaxMembers = int64_t(1) << 16;                // atoms in slabs
constexpr size_t align256c(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t kNoAllocLoopOff = 0;
constexpr size_t kNoAllocStatusOff = kNoAllocLoopOff + align256c(sizeof(LoopStage));
constexpr size_t kNoAllocAggOff = kNoAllocStatusOff + align256c(16 + (size_t)kNoAllocMaxTiles * sizeof(int));
constexpr size_t kNoAllocIncOff =
    kNoAllocAggOff + align256c((size_t)kNoAllocMaxTiles * disco::kMaxCats * sizeof(int32_t));
constexpr size_t kNoAllocMemberOff =
    kNoAllocIncOff + align256c((size_t)kNoAllocMaxTiles * disco::kMaxCats * sizeof(int32_t));
constexpr size_t kNoAllocTotalsOff =
    kNoAllocMemberOff + align256c((size_t)kNoAllocMaxMembers * sizeof(disco::MemberRec));
constexpr size_t kNoAllocScratchBytes = 4 * 1024 * 1024;
static_assert(kNoAllocTotalsOff + (disco::kMaxCats + 1) * sizeof(int64_t) <= kNoAllocScratchBytes,
              "no-alloc scratch layout");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_addr[kMaxDevices] = {};
unsigned long long g_noalloc_ctx[kMaxDevices] = {};
bool g_noalloc_dirty[kMaxDevices] = {};     // the look-back flags may not be zero

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique identifier of the calling thread's current context (the driver's
// cuCtxGetId, reached through the runtime without linking libcuda), 0 when
// it cannot be read.
unsigned long long current_context_id()
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
    });
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS) return id;
    return 0;
}

// Device address of g_noalloc_scratch on the current device.  In host code the
// array's name is a host-side stand-in, not a device address: the address is
// looked up with that device current and cached with the identifier of the
// context it belongs to; a new context on that device (after a device reset,
// which reloads the module) gets a fresh lookup.
int noalloc_scratch(unsigned char** out, unsigned long long* ctx_out, int* dev_out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cfail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return efail(DISCO_ELIMIT, "device ordinal above 63");
    // make the primary context current before its identifier is read
    e = cudaFree(nullptr);
    if (e != cudaSuccess) return cfail(e, "device context");
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev] || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return cfail(e, "cudaGetSymbolAddress of the scratch array");
        g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
        g_noalloc_ctx[dev] = ctx;
        g_noalloc_dirty[dev] = true;
    }
    *dev_out = dev;
    *out = g_noalloc_addr[dev];
    *ctx_out = ctx;
    return DISCO_OK;
}

// Reads (and with `take`, clears) or sets a device's dirty flag.
bool noalloc_dirty(int dev, bool take, bool set)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    const bool was = g_noalloc_dirty[dev];
    if (take) g_noalloc_dirty[dev] = false;
    if (set) g_noalloc_dirty[dev] = true;
    return was;
}

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
    int dcount = 0;
    if (cudaGetDeviceCount(&dcount) != cudaSuccess || dcount == 0) return efail(DISCO_ENODEV, "no CUDA device");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* base = nullptr;
    unsigned long long ctx = 0;
    int dev = 0;
    int st = noalloc_scratch(&base, &ctx, &dev);
    if (st) return st;

    int act_index[kMaxSlabLoops];
    int nl = 0;
    st = stage_loops(loops, nloops, box, info, act_index, nl, base + kNoAllocLoopOff, s, ctx);
    if (st) return st;
    const int C = 2 + 2 * nl;
    const int64_t ntiles = (n + kMatterTile - 1) / kMatterTile;
    const int64_t member_cap = std::min<int64_t>(kNoAllocMaxMembers, std::max<int64_t>(0, slab_capacity));

    MatterArgs a;
    std::memset(&a, 0, sizeof(a));
    a.x = x; a.y = y; a.z = z;
    a.n = n;
    a.Lx = box[0]; a.Ly = box[1]; a.Lz = box[2];
    a.iLx = (float)(1.0 / box[0]); a.iLy = (float)(1.0 / box[1]); a.iLz = (float)(1.0 / box[2]);
    a.idLx = 1.0 / box[0]; a.idLy = 1.0 / box[1]; a.idLz = 1.0 / box[2];
    a.xo = x_out; a.yo = y_out; a.zo = z_out;
    a.new_index = new_index;
    a.slab_atoms = slab_atoms;
    a.slab_side = slab_side;
    a.slab_cap = slab_capacity;
    a.copies = copies;
    a.copy_cap = copy_capacity;
    MatterScratch m;
    m.loops = base + kNoAllocLoopOff;
    m.status = base + kNoAllocStatusOff;
    m.agg = reinterpret_cast<int32_t*>(base + kNoAllocAggOff);
    m.inc = reinterpret_cast<int32_t*>(base + kNoAllocIncOff);
    m.members = reinterpret_cast<MemberRec*>(base + kNoAllocMemberOff);
    m.member_cap = member_cap;
    m.totals = reinterpret_cast<int64_t*>(base + kNoAllocTotalsOff);
    const bool dirty = noalloc_dirty(dev, true, false);
    st = matter_queue(a, m, nl, ntiles, s, dirty ? status_bytes(kNoAllocMaxTiles) : 0);
    if (st) { stage_cache_drop(); noalloc_dirty(dev, false, true); return st; }
    int64_t tot[kMaxCats + 1];
    cudaError_t e = cudaMemcpyAsync(tot, m.totals, (size_t)(C + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { stage_cache_drop(); noalloc_dirty(dev, false, true); return cfail(e, "prismatic totals"); }
    st = matter_finish(tot, nl, act_index, nloops, info, slab_capacity, copy_capacity, member_cap, counts);
    if (st == DISCO_ELIMIT && tot[1] > member_cap && counts[1] <= slab_capacity && counts[2] <= copy_capacity)
        return efail(DISCO_ELIMIT, "disco_b200_prismatic_noalloc takes at most 65536 atoms in slabs "
                                   "(its scratch array is fixed)");
    return st;
}

} // extern "C"
