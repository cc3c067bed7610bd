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
// The step is one cooperative kernel (matter_kernel): a first phase computes
// every atom's slab mask once (FP32 bounding-box culling per 128-atom
// segment, an FP32 pre-test, the exact FP64 predicate for the rest, segments
// handed to the grid's warps in chunks from a ticket); after a grid barrier each CTA
// counts its contiguous range, after a second the CTAs' counts are scanned
// per category, and after a third the survivors are compacted in order (x, y,
// z and the new-index map; the positions come back from L2) and the slab
// entries and interstitial copies written in loop order, then atom order,
// with copies of removed atoms dropped and their sources renumbered.
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
    float boundf;          // bound in FP32, rounded up (the culling)
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
constexpr int kMatterWarps = kMatterThreads / 32;
constexpr int kSegRounds = 4;                                  // rounds of 32 atoms per segment
constexpr int kSegAtoms = 32 * kSegRounds;                     // 128 atoms: one warp's unit of work
constexpr int kGroupSegs = 32;                                 // segments per warp between two flushes
constexpr int kSegRow = 2 * kMaxSlabLoops;                     // per-loop slab and copy counts
constexpr int kMaxCats = 2 + 2 * kMaxSlabLoops;                // categories counted per CTA
constexpr int kWarpQueue = 512;                                // exact tests queued per warp
constexpr int kMaxGrid = 8 * 148;                              // CTAs of one call at most
constexpr int kCtlWords = 8;                                   // control words before the per-loop totals
constexpr int kGrab = 2;                                       // segments per ticket of the first phase
constexpr int kFlushAt = 32;                                   // queued exact tests that start a flush
constexpr int kSmallGrid = 64;                                 // grids scanned by one CTA
// dynamic shared memory: per warp the masks and sides of one segment
constexpr size_t kMatterSmem = kMatterWarps * 2 * kSegAtoms * sizeof(uint64_t);

struct MatterArgs {
    const double *x, *y, *z;
    int64_t n;
    const SlabHead* heads;        // [nl]
    const SlabLoopDev* loops;     // [nl]
    int32_t nl, C;                // C = 2 + 2 nl categories: survivors, members, slab of
                                  // loop l (2 + l), kept copies of loop l (2 + nl + l)
    double Lx, Ly, Lz;
    float iLx, iLy, iLz;          // 1 / box lengths in FP32 (culling and pre-test)
    int32_t G;                    // CTAs, all resident at once (cooperative launch)
    double idLx, idLy, idLz;      // 1 / box lengths, rounded (the exact test's fast path)
    int64_t S;                    // segments of kSegAtoms atoms
    int32_t* seg_removed;         // [S] atoms a vacancy slab removes
    int32_t* seg_members;         // [S] slab-member atoms
    int32_t* seg_off;             // [S] first member record of the segment
    int32_t* cta_tot;             // [G][C] counts per CTA
    int32_t* cta_pre;             // [G][C] exclusive prefixes over the CTAs
    unsigned int* ctl;            // [kCtlWords] barrier arrivals, exits, member records taken, error
                                  // word, segment ticket, then [2 nl] per-loop slab and kept-copy
                                  // totals; zero at entry, left zero by the last CTA to leave
    MemberRec* members;
    int64_t member_cap;
    double *xo, *yo, *zo;
    int32_t* new_index;
    int32_t* slab_atoms;
    int8_t* slab_side;
    int64_t slab_cap;
    disco_copy* copies;
    int64_t copy_cap;
    int64_t* totals;              // [C + 1] category totals, then the error word
    int32_t vec_in;               // x, y, z 16-byte aligned: pairs of atoms per 16-byte load
    int32_t vec_out;              // x_out, y_out, z_out 16-byte and new_index 8-byte aligned
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// L2 policies: the first phase's reads of the positions stay in L2 for the
// second phase's (evict-last); the second phase reads them for the last time
// (evict-first).  The positions are never written during the kernel, so these
// loads carry no ordering constraint.
__device__ __forceinline__ uint64_t l2_policy_keep()
{
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint64_t l2_policy_last_use()
{
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ double ld_hint(const double* p, uint64_t pol)
{
    double v;
    asm("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ void ld2_hint(const double* p, uint64_t pol, double& v0, double& v1)
{
    asm("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v0), "=d"(v1) : "l"(p), "l"(pol));
}

// L2 prefetch of one line (the first phase's reads follow within a few
// microseconds; evict-last like those reads).
__device__ __forceinline__ void prefetch_l2_keep(const void* p)
{
    asm volatile("prefetch.global.L2::evict_last [%0];" :: "l"(p));
}

// All CTAs of the launch arrive, then wait until `target` arrivals are
// counted (the launch is cooperative, so every CTA is resident).  Bounded: a
// wait that sees no progress for 2 s records DISCO_ETIMEOUT and goes on.
__device__ __forceinline__ void grid_sync(unsigned* arrive, unsigned target, int* err)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(arrive, 1u);
        unsigned long long t0 = 0;
        unsigned sleep = 32;
        while (ld_acquire_u32(arrive) < target) {
            if (t0 == 0) {
                t0 = global_ns();
            } else if (global_ns() - t0 > kWaitLimitNs) {
                report(err, DISCO_ETIMEOUT);
                break;
            }
            __nanosleep(sleep);
            if (sleep < 256) sleep *= 2;
        }
        __threadfence();
    }
    __syncthreads();
}

// Smallest |p - c - m L| over p in [lo, hi] and integers m, in FP32 for the
// culling: lo, hi are the FP32 roundings of a segment's extreme coordinates,
// c and L those of the loop centre and the box.  Every rounding is covered by
// subtracting 1e-5 (|a| + |b| + L) + 1e-3 A (above ten times the worst
// accumulated error of these few operations at |a| <= 1e5 L); a nearest-image
// index off by one only lowers the result or gives 0, and beyond
// |a| = 1e5 L (or NaN) the answer is 0.  Never above the true gap, so culling
// with it never drops a member.
__device__ __forceinline__ float periodic_gap_f(float lo, float hi, float c, float L, float iL)
{
    const float a = lo - c, b = hi - c;
    if (!(b - a < L) || !(fabsf(a) < 1e5f * L)) return 0.0f;
    const float m1 = floorf(a * iL);
    if ((m1 + 1.0f) * L <= b) return 0.0f;
    const float d = fminf(a - m1 * L, (m1 + 1.0f) * L - b);
    return fmaxf(0.0f, d - (1e-5f * (fabsf(a) + fabsf(b) + L) + 1e-3f));
}

// The FP32 pre-test of the lane's four atoms of a segment (f*[q], their
// positions rounded to FP32) against the loops in `cand` (loops whose slab can
// reach the segment): per atom the loops it cannot exclude, its exact-test
// candidates.  A loop is excluded only if the atom's t is outside [tLo, tHi)
// by more than `margin` planes.  With the atom and the centre within 2 L of
// the origin and rounded to FP32, and the nearest image unambiguous (r/L + 1/2
// at least 1e-5 from an integer and |r/L| < 2; else the loop stays a
// candidate), the FP32 t differs from the exactly rounded t of slab_member by
// less than 1.5e-6 (Lx + Ly + Lz) / d + 1e-6 planes; the margin is
// 1e-5 (Lx + Ly + Lz) / d + 1e-3.  So it never rejects a member: the exact
// test decides every atom it passes, and atom sets stay bit-exact.
__device__ __forceinline__ void pretest_segment(const SlabHead* sh, uint64_t cand, const float (&fx)[kSegRounds],
                                                const float (&fy)[kSegRounds], const float (&fz)[kSegRounds],
                                                const bool (&valid)[kSegRounds], const float (&L)[3],
                                                const float (&iL)[3], uint64_t (&out)[kSegRounds])
{
    bool pin[kSegRounds];
#pragma unroll
    for (int q = 0; q < kSegRounds; ++q) {
        pin[q] = fabsf(fx[q]) < 2.0f * L[0] && fabsf(fy[q]) < 2.0f * L[1] && fabsf(fz[q]) < 2.0f * L[2];
        out[q] = 0ull;
    }
    for (uint64_t c = cand; c; c &= c - 1) {
        const int l = __ffsll((long long)c) - 1;
        const SlabHead& S = sh[l];
        const float cx = S.cf[0], cy = S.cf[1], cz = S.cf[2];
        const float nx = S.nf[0], ny = S.nf[1], nz = S.nf[2];
        const float tlo = S.tlo - S.margin, thi = S.thi + S.margin, idf = S.inv_df;
        const bool cin = fabsf(cx) < 2.0f * L[0] && fabsf(cy) < 2.0f * L[1] && fabsf(cz) < 2.0f * L[2];
#pragma unroll
        for (int q = 0; q < kSegRounds; ++q) {
            const float p[3] = { fx[q], fy[q], fz[q] };
            const float cc[3] = { cx, cy, cz }, nn[3] = { nx, ny, nz };
            float s = 0.0f;
            bool sure = pin[q] && cin;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float r = p[k] - cc[k];
                const float qd = r * iL[k];
                const float h = qd + 0.5f;
                const float f = floorf(h);
                const float fr = h - f;
                sure = sure && fabsf(qd) < 2.0f && fr >= 1e-5f && fr <= 1.0f - 1e-5f;
                s = fmaf(nn[k], fmaf(-L[k], f, r), s);
            }
            const float t = s * idf;
            const bool outside = sure && (t < tlo || t >= thi);
            if (valid[q] && !outside) out[q] |= 1ull << l;
        }
    }
}

// Warp-wide minimum / maximum of a float through the integer reduction unit:
// the bit pattern, its magnitude bits flipped for negative values, orders as a
// signed integer exactly as the floats order (NaN aside, which no member has).
__device__ __forceinline__ int float_order(float f)
{
    const int i = __float_as_int(f);
    return i ^ ((i >> 31) & 0x7fffffff);
}

__device__ __forceinline__ float order_float(int i) { return __int_as_float(i ^ ((i >> 31) & 0x7fffffff)); }

__device__ __forceinline__ float warp_min_f(float v)
{
    return order_float(__reduce_min_sync(0xffffffffu, float_order(v)));
}

__device__ __forceinline__ float warp_max_f(float v)
{
    return order_float(__reduce_max_sync(0xffffffffu, float_order(v)));
}

// Streaming layout of a segment: lane t holds the atoms 64 (q / 2) + 2 t + q % 2,
// q = 0..3 (two 16-byte loads of pairs per coordinate).
__device__ __forceinline__ int slot_of(int q, int lane) { return 64 * (q >> 1) + 2 * lane + (q & 1); }

// 16-byte streaming store of two doubles.
__device__ __forceinline__ void st2_cs(double* p, double v0, double v1)
{
    __stcs(reinterpret_cast<double2*>(p), make_double2(v0, v1));
}

// One coordinate of a member-free segment in the slot_of layout (v[0..3])
// stored at out + sb + slot with 16-byte stores; for an odd sb each lane
// stores its second atom with the next lane's first (the pair after lane 31
// of the first half is lane 0's first atom of the second half), lane 0 the
// segment's first atom and lane 31 its last alone.
__device__ __forceinline__ void store_shifted(double* out, int64_t sb, const double (&v)[kSegRounds], int lane)
{
    if ((sb & 1) == 0) {
        st2_cs(out + sb + 2 * lane, v[0], v[1]);
        st2_cs(out + sb + 64 + 2 * lane, v[2], v[3]);
        return;
    }
    const double n0 = __shfl_down_sync(0xffffffffu, v[0], 1);
    const double n2 = __shfl_down_sync(0xffffffffu, v[2], 1);
    const double h2 = __shfl_sync(0xffffffffu, v[2], 0);
    st2_cs(out + sb + 2 * lane + 1, v[1], lane == 31 ? h2 : n0);
    if (lane < 31) st2_cs(out + sb + 64 + 2 * lane + 1, v[3], n2);
    else __stcs(out + sb + kSegAtoms - 1, v[3]);
    if (lane == 0) __stcs(out + sb, v[0]);
}

// Member-free segment: every atom survives, the survivors are the segment
// shifted to `sb` (survivors before it).  Whole segments with aligned arrays
// move in 16-byte loads and stores.
__device__ __forceinline__ void copy_plain(const MatterArgs& a, int64_t s, int64_t sb, uint64_t pol, int lane)
{
    const int64_t i0 = s * kSegAtoms;
    if (a.vec_in && a.vec_out && i0 + kSegAtoms <= a.n && sb >= 0 && sb + kSegAtoms <= a.n) {
        double x[kSegRounds], y[kSegRounds], z[kSegRounds];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t i = i0 + 64 * h + 2 * lane;
            ld2_hint(a.x + i, pol, x[2 * h], x[2 * h + 1]);
            ld2_hint(a.y + i, pol, y[2 * h], y[2 * h + 1]);
            ld2_hint(a.z + i, pol, z[2 * h], z[2 * h + 1]);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int32_t q = (int32_t)(sb + 64 * h + 2 * lane);
            __stcs(reinterpret_cast<int2*>(a.new_index + i0 + 64 * h + 2 * lane), make_int2(q, q + 1));
        }
        store_shifted(a.xo, sb, x, lane);
        store_shifted(a.yo, sb, y, lane);
        store_shifted(a.zo, sb, z, lane);
        return;
    }
    double px[kSegRounds], py[kSegRounds], pz[kSegRounds];
#pragma unroll
    for (int r = 0; r < kSegRounds; ++r) {
        const int64_t i = i0 + r * 32 + lane;
        px[r] = py[r] = pz[r] = 0.0;
        if (i < a.n) { px[r] = ld_hint(a.x + i, pol); py[r] = ld_hint(a.y + i, pol); pz[r] = ld_hint(a.z + i, pol); }
    }
#pragma unroll
    for (int r = 0; r < kSegRounds; ++r) {
        const int64_t i = i0 + r * 32 + lane;
        const int64_t q = sb + r * 32 + lane;
        if (i < a.n && q >= 0 && q < a.n) {
            __stcs(a.xo + q, px[r]); __stcs(a.yo + q, py[r]); __stcs(a.zo + q, pz[r]);
            __stcs(a.new_index + i, (int32_t)q);
        }
    }
}

// Segment with slab members (its m records at `rec`): the records' masks and
// sides go back into the warp's per-slot table (smask / ssides), then per
// loop its slab entries and interstitial copies at the warp's running
// positions wrun[l] / wrun[nl + l] (ascending atom order within the loop;
// copies of removed atoms dropped, sources renumbered), then the survivors,
// the removed atoms skipped.
__device__ __forceinline__ void copy_members(const MatterArgs& a, const SlabHead* sh, uint64_t vac, int64_t s,
                                             int64_t sb, const MemberRec* rec, int m, uint64_t* smask,
                                             uint64_t* ssides, int64_t* wrun, uint64_t pol, int lane)
{
    const int64_t i0 = s * kSegAtoms;
    const int nl = a.nl;
    const unsigned ltm = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kSegRounds; ++r) { smask[r * 32 + lane] = 0; ssides[r * 32 + lane] = 0; }
    __syncwarp();
    for (int e = lane; e < m; e += 32) {
        const int slot = __ldcg(&rec[e].atom) - (int)i0;
        if (slot >= 0 && slot < kSegAtoms) {
            smask[slot] = __ldcg(reinterpret_cast<const unsigned long long*>(&rec[e].mask));
            ssides[slot] = __ldcg(reinterpret_cast<const unsigned long long*>(&rec[e].sides));
        }
    }
    __syncwarp();
    unsigned rb[kSegRounds];
    uint64_t un = 0;
#pragma unroll
    for (int r = 0; r < kSegRounds; ++r) {
        const uint64_t mk = smask[r * 32 + lane];
        rb[r] = __ballot_sync(0xffffffffu, (mk & vac) != 0);
        un |= mk;
    }
    un = ((uint64_t)__reduce_or_sync(0xffffffffu, (unsigned)(un >> 32)) << 32) |
         __reduce_or_sync(0xffffffffu, (unsigned)un);
    for (uint64_t u = un; u; u &= u - 1) {
        const int l = __ffsll((long long)u) - 1;
        const bool inter = sh[l].type == DISCO_MATTER_INTERSTITIAL;
        int64_t qs = wrun[l], qc = wrun[nl + l];
        int rem_before = 0;
#pragma unroll
        for (int r = 0; r < kSegRounds; ++r) {
            const uint64_t mk = smask[r * 32 + lane];
            const bool in = (mk >> l) & 1ull;
            const bool removed = (rb[r] >> lane) & 1u;
            const bool kp = in && inter && !removed;
            const bool pos = (ssides[r * 32 + lane] >> l) & 1ull;
            const unsigned bi = __ballot_sync(0xffffffffu, in);
            const unsigned bk = __ballot_sync(0xffffffffu, kp);
            if (in) {
                const int64_t q = qs + __popc(bi & ltm);
                if (q >= 0 && q < a.slab_cap) {
                    a.slab_atoms[q] = (int32_t)(i0 + r * 32 + lane);
                    a.slab_side[q] = pos ? 1 : -1;
                }
            }
            if (kp) {
                const int64_t q = qc + __popc(bk & ltm);
                if (q >= 0 && q < a.copy_cap) {
                    const disco_slab_loop& g = a.loops[l].L;
                    const double* shf = pos ? g.shift_pos : g.shift_neg;
                    disco_copy cp;
                    cp.atom = (int32_t)(sb + r * 32 + lane - (rem_before + __popc(rb[r] & ltm)));
                    cp.reserved = 0;
                    cp.shift[0] = shf[0]; cp.shift[1] = shf[1]; cp.shift[2] = shf[2];
                    a.copies[q] = cp;
                }
            }
            qs += __popc(bi);
            qc += __popc(bk);
            rem_before += __popc(rb[r]);
        }
        __syncwarp();
        if (lane == 0) { wrun[l] = qs; wrun[nl + l] = qc; }
        __syncwarp();
    }
    double px[kSegRounds], py[kSegRounds], pz[kSegRounds];
#pragma unroll
    for (int r = 0; r < kSegRounds; ++r) {
        const int64_t i = i0 + r * 32 + lane;
        px[r] = py[r] = pz[r] = 0.0;
        if (i < a.n) { px[r] = ld_hint(a.x + i, pol); py[r] = ld_hint(a.y + i, pol); pz[r] = ld_hint(a.z + i, pol); }
    }
    int before = 0;
#pragma unroll
    for (int r = 0; r < kSegRounds; ++r) {
        const int64_t i = i0 + r * 32 + lane;
        if (i < a.n) {
            if (!((rb[r] >> lane) & 1u)) {
                const int64_t q = sb + r * 32 + lane - before - __popc(rb[r] & ltm);
                if (q >= 0 && q < a.n) { __stcs(a.xo + q, px[r]); __stcs(a.yo + q, py[r]); __stcs(a.zo + q, pz[r]); }
                __stcs(a.new_index + i, (int32_t)q);
            } else {
                __stcs(a.new_index + i, -1);
            }
        }
        before += __popc(rb[r]);
    }
    __syncwarp();                                               // the table is rewritten
}

// From the masks and sides of segment s in the warp's shared-memory buffer:
// its removed and member counts, the per-loop slab and kept-copy counts
// (added to wcnt), and its member records in atom order at `off` (taken here
// from the global record counter when off < 0).
__device__ __forceinline__ void aggregate_segment(const MatterArgs& a, const SlabHead* sh, uint64_t vac, int64_t s,
                                                  const uint64_t* smask, const uint64_t* ssides, int* wcnt,
                                                  int& rc, int& mc, int& off, int lane)
{
    const int64_t i0 = s * kSegAtoms;
    const int nl = a.nl;
    const unsigned ltm = (1u << lane) - 1u;
    unsigned bm[kSegRounds];
    rc = 0;
    mc = 0;
#pragma unroll
    for (int r = 0; r < kSegRounds; ++r) {
        const uint64_t mask = smask[r * 32 + lane];
        const bool removed = (mask & vac) != 0;
        bm[r] = __ballot_sync(0xffffffffu, mask != 0);
        rc += __popc(__ballot_sync(0xffffffffu, removed));
        mc += __popc(bm[r]);
        for (uint64_t u = mask; u; u &= u - 1) {             // members are rare
            const int l = __ffsll((long long)u) - 1;
            atomicAdd(&wcnt[l], 1);
            if (sh[l].type == DISCO_MATTER_INTERSTITIAL && !removed) atomicAdd(&wcnt[nl + l], 1);
        }
    }
    if (off < 0) {
        int o = 0;
        if (lane == 0 && mc > 0) o = (int)atomicAdd(a.ctl + 2, (unsigned)mc);
        off = __shfl_sync(0xffffffffu, o, 0);
    }
    int e = off;
#pragma unroll
    for (int r = 0; r < kSegRounds; ++r) {
        const uint64_t mask = smask[r * 32 + lane];
        if (mask) {
            const int64_t q = (int64_t)e + __popc(bm[r] & ltm);
            if (q < a.member_cap) {
                MemberRec rec;
                rec.atom = (int32_t)(i0 + r * 32 + lane);
                rec.removed = (mask & vac) != 0;
                rec.mask = mask;
                rec.sides = ssides[r * 32 + lane];
                a.members[q] = rec;
            }
        }
        e += __popc(bm[r]);
    }
}

// A segment whose candidates do not fit the warp's queue: its exact tests
// lane by lane, then its counts and records (out of line: a rare path that
// would otherwise raise the register count of the streaming loop; `a` lives
// in shared memory).  Returns (removed, members, first record).
__device__ __noinline__ int3 direct_segment(const MatterArgs& a, const SlabHead* sh, uint64_t vac, int64_t s,
                                           uint64_t c0, uint64_t c1, uint64_t c2, uint64_t c3, uint64_t* smask,
                                           uint64_t* ssides, int* wcnt, int lane)
{
    const int64_t i0 = s * kSegAtoms;
    const uint64_t cand[kSegRounds] = { c0, c1, c2, c3 };
#pragma unroll
    for (int r = 0; r < kSegRounds; ++r) { smask[r * 32 + lane] = 0; ssides[r * 32 + lane] = 0; }
    __syncwarp();
#pragma unroll 1
    for (int q = 0; q < kSegRounds; ++q) {
        const int slot = slot_of(q, lane);
        const int64_t i = i0 + slot;
        for (uint64_t c = cand[q]; c; c &= c - 1) {
            const int l = __ffsll((long long)c) - 1;
            bool ps = false;
            if (slab_member(a.loops[l], a.x[i], a.y[i], a.z[i], a.Lx, a.Ly, a.Lz, a.idLx, a.idLy, a.idLz, ps)) {
                smask[slot] |= 1ull << l;
                if (ps) ssides[slot] |= 1ull << l;
            }
        }
    }
    __syncwarp();
    int rc = 0, mc = 0, off = -1;
    aggregate_segment(a, sh, vac, s, smask, ssides, wcnt, rc, mc, off, lane);
    __syncwarp();
    return make_int3(rc, mc, mc > 0 ? off : 0);
}

// The matter step in one cooperative launch.
//   Phase 1, masks.  The grid's warps take the 128-atom segments in chunks
//     of two from a ticket, so that the warps whose chunks cross slabs take
//     fewer.  Per segment: the positions (16-byte loads, prefetched two
//     segments ahead, kept in L2 for phase 2) rounded to FP32 for a bounding
//     box and a per-loop cull; for the few segments a loop can reach, the
//     FP32 pre-test per atom, its candidate (atom, loop) pairs queued per
//     warp.  Once 32 tests are queued (or 32 segments listed) the warp runs
//     the exact FP64 tests of its queue spread over its lanes, then per listed
//     segment the masks, counts and member records (atom order, one block of
//     records per flush).  Per segment: removed and member counts, first record; per
//     call: the per-loop slab and kept-copy totals.
//   Barrier; per CTA, its counts from the per-segment results, per warp of
//     its contiguous range; barrier; CTA c scans category c over the CTAs;
//     barrier.
//   Phase 2, ordered writes.  CTA k owns a contiguous range of segments, cut
//     into eight contiguous warp ranges; each warp walks its range with the
//     running survivor rank: a member-free segment is a shifted copy; a
//     segment with members writes their slab entries and copies at the warp's
//     running per-loop positions (loop base + CTA prefix + earlier warps'
//     counts), in atom order (Code/prismatic.cpp:61-72,
//     Code/main.cpp:651-654,676-679), then its survivors.
// No look-back and no second kernel: the only waits are the three barriers.
// The outputs must not overlap the positions.
__global__ void __launch_bounds__(kMatterThreads, 3) matter_kernel(const MatterArgs a)
{
    extern __shared__ __align__(16) unsigned char dyn[];       // per warp: masks and sides of one segment
    __shared__ SlabHead sh[kMaxSlabLoops];
    __shared__ __align__(16) unsigned char wq_raw[kMatterWarps * kWarpQueue * 4];   // phase 1 queues, phase 2 wrun
    __shared__ int wl_seg[kMatterWarps][kGroupSegs];           // listed segments of a group (index in the group)
    __shared__ int wl_q[kMatterWarps][kGroupSegs];             // their first queue entry | count << 16
    __shared__ int wl_mr[kMatterWarps][kGroupSegs];            // their member count | removed count << 16
    __shared__ int wcnt[kMatterWarps][kSegRow];                // per warp: slab / kept-copy counts per loop
    __shared__ int wrem[kMatterWarps], wmem[kMatterWarps];
    __shared__ int64_t run[kSegRow];                           // CTA's first slab entry / copy per loop
    __shared__ int64_t scan_w[kMatterWarps];
    __shared__ unsigned long long vac_s;
    __shared__ MatterArgs sa;                                  // for the out-of-line rare path
    static_assert(kMatterWarps * kSegRow * sizeof(int64_t) <= sizeof(wq_raw), "phase 2 positions fit the queues");
    static_assert(sizeof(MatterArgs) % 8 == 0, "argument block copied in words");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nl = a.nl, C = a.C, G = a.G;
    const int64_t k = blockIdx.x;
    const int64_t seg_lo = k * a.S / G, seg_hi = (k + 1) * a.S / G;
    const int64_t nseg = seg_hi - seg_lo;
    const int64_t wlo = seg_lo + nseg * warp / kMatterWarps, whi = seg_lo + nseg * (warp + 1) / kMatterWarps;
    int* err = reinterpret_cast<int*>(a.ctl + 3);
    {
        const int words = nl * (int)(sizeof(SlabHead) / 8);
        const uint64_t* src = reinterpret_cast<const uint64_t*>(a.heads);
        uint64_t* dst = reinterpret_cast<uint64_t*>(sh);
        for (int i = tid; i < words; i += kMatterThreads) dst[i] = src[i];
        for (int i = lane; i < 2 * nl; i += 32) wcnt[warp][i] = 0;
        const uint64_t* as = reinterpret_cast<const uint64_t*>(&a);
        for (int i = tid; i < (int)(sizeof(MatterArgs) / 8); i += kMatterThreads) reinterpret_cast<uint64_t*>(&sa)[i] = as[i];
        if (tid == 0) vac_s = 0ull;
    }
    __syncthreads();
    if (tid < nl && sh[tid].type == DISCO_MATTER_VACANCY) atomicOr(&vac_s, 1ull << tid);
    __syncthreads();
    const uint64_t vac = vac_s;

    // ---- phase 1: masks --------------------------------------------------------------
    {
        const uint64_t keep = l2_policy_keep();
        uint32_t* wq = reinterpret_cast<uint32_t*>(wq_raw) + warp * kWarpQueue;
        uint64_t* smask = reinterpret_cast<uint64_t*>(dyn) + warp * (2 * kSegAtoms);
        uint64_t* ssides = smask + kSegAtoms;
        const double* pf_base = lane < 8 ? a.x : lane < 16 ? a.y : a.z;
        const float Lf[3] = { (float)a.Lx, (float)a.Ly, (float)a.Lz };
        const float iLf[3] = { a.iLx, a.iLy, a.iLz };
        // segments in chunks of kGrab from the call's ticket, the next chunk
        // taken one ahead: warps that meet slabs take fewer segments
        unsigned tk = 0;
        if (lane == 0) tk = atomicAdd(a.ctl + 4, (unsigned)kGrab);
        int64_t cur = __shfl_sync(0xffffffffu, tk, 0);
        if (lane == 0) tk = atomicAdd(a.ctl + 4, (unsigned)kGrab);
        int64_t nxt = __shfl_sync(0xffffffffu, tk, 0);
        int64_t s = cur;                                        // the next segment
        while (true) {
            int nq = 0, nlst = 0;
            while (nlst < kGroupSegs && nq < kFlushAt && s < a.S) {
                const int64_t cend = cur + kGrab < a.S ? cur + kGrab : a.S;
                {
                    const int64_t p2 = s + 2 < cend ? s + 2 : nxt + (s + 2 - cend);   // two segments ahead
                    if (lane < 24 && p2 < a.S) {
                        const int64_t pi = p2 * kSegAtoms + (lane & 7) * 16;
                        if (pi < a.n) prefetch_l2_keep(pf_base + pi);
                    }
                }
                const int64_t i0 = s * kSegAtoms;
                // the segment's positions rounded to FP32 (slot_of layout); an
                // atom past n repeats the segment's first atom
                float fx[kSegRounds], fy[kSegRounds], fz[kSegRounds];
                bool valid[kSegRounds];
                if (a.vec_in && i0 + kSegAtoms <= a.n) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int64_t i = i0 + 64 * h + 2 * lane;
                        double x0, x1, y0, y1, z0, z1;
                        ld2_hint(a.x + i, keep, x0, x1);
                        ld2_hint(a.y + i, keep, y0, y1);
                        ld2_hint(a.z + i, keep, z0, z1);
                        fx[2 * h] = (float)x0; fx[2 * h + 1] = (float)x1;
                        fy[2 * h] = (float)y0; fy[2 * h + 1] = (float)y1;
                        fz[2 * h] = (float)z0; fz[2 * h + 1] = (float)z1;
                    }
#pragma unroll
                    for (int q = 0; q < kSegRounds; ++q) valid[q] = true;
                } else {
#pragma unroll
                    for (int q = 0; q < kSegRounds; ++q) {
                        int64_t i = i0 + slot_of(q, lane);
                        valid[q] = i < a.n;
                        if (!valid[q]) i = i0;
                        fx[q] = (float)ld_hint(a.x + i, keep);
                        fy[q] = (float)ld_hint(a.y + i, keep);
                        fz[q] = (float)ld_hint(a.z + i, keep);
                    }
                }
                // the loops whose slab can reach the segment's bounding box
                uint64_t wmask = 0;
                if (nl > 0) {
                    float lo[3] = { fminf(fminf(fx[0], fx[1]), fminf(fx[2], fx[3])),
                                    fminf(fminf(fy[0], fy[1]), fminf(fy[2], fy[3])),
                                    fminf(fminf(fz[0], fz[1]), fminf(fz[2], fz[3])) };
                    float hi[3] = { fmaxf(fmaxf(fx[0], fx[1]), fmaxf(fx[2], fx[3])),
                                    fmaxf(fmaxf(fy[0], fy[1]), fmaxf(fy[2], fy[3])),
                                    fmaxf(fmaxf(fz[0], fz[1]), fmaxf(fz[2], fz[3])) };
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        lo[d] = warp_min_f(lo[d]);
                        hi[d] = warp_max_f(hi[d]);
                    }
                    for (int half = 0; half * 32 < nl; ++half) {
                        const int l = lane + 32 * half;
                        bool reach = false;
                        if (l < nl) {
                            const SlabHead& S = sh[l];
                            const float gx = periodic_gap_f(lo[0], hi[0], S.cf[0], Lf[0], iLf[0]);
                            const float gy = periodic_gap_f(lo[1], hi[1], S.cf[1], Lf[1], iLf[1]);
                            const float gz = periodic_gap_f(lo[2], hi[2], S.cf[2], Lf[2], iLf[2]);
                            reach = !(gx * gx + gy * gy + gz * gz > S.boundf * S.boundf);
                        }
                        wmask |= (uint64_t)__ballot_sync(0xffffffffu, reach) << (32 * half);
                    }
                }
                int rc = 0, mc = 0, off = 0;
                bool listed = false;
                if (wmask) {
                    // the FP32 pre-test per atom: its exact-test candidates
                    uint64_t cand[kSegRounds];
                    pretest_segment(sh, wmask, fx, fy, fz, valid, Lf, iLf, cand);
                    int cnt = 0;
#pragma unroll
                    for (int q = 0; q < kSegRounds; ++q) cnt += __popcll(cand[q]);
                    int pre = cnt;
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, pre, o);
                        if (lane >= o) pre += y;
                    }
                    const int T = __shfl_sync(0xffffffffu, pre, 31);
                    pre -= cnt;
                    if (T > 0 && nq + T <= kWarpQueue) {
                        // queued: (loop, slot, list entry), tested at the flush
                        int q = nq + pre;
#pragma unroll
                        for (int r = 0; r < kSegRounds; ++r)
                            for (uint64_t c = cand[r]; c; c &= c - 1)
                                wq[q++] = (uint32_t)(__ffsll((long long)c) - 1) | ((uint32_t)slot_of(r, lane) << 6) |
                                          ((uint32_t)nlst << 13);
                        if (lane == 0) {
                            wl_seg[warp][nlst] = (int)s;
                            wl_q[warp][nlst] = nq | (T << 16);
                        }
                        nq += T;
                        ++nlst;
                        listed = true;
                    } else if (T > 0) {
                        // the queue is full: this segment's exact tests here, lane by lane
                        const int3 res = direct_segment(sa, sh, vac, s, cand[0], cand[1], cand[2], cand[3], smask,
                                                        ssides, wcnt[warp], lane);
                        rc = res.x;
                        mc = res.y;
                        off = res.z;
                    }
                }
                if (!listed && lane == 0) { a.seg_removed[s] = rc; a.seg_members[s] = mc; a.seg_off[s] = off; }
                if (++s >= cend) {                              // the next chunk
                    cur = nxt;
                    s = cur;
                    if (cur < a.S) {
                        if (lane == 0) tk = atomicAdd(a.ctl + 4, (unsigned)kGrab);
                        nxt = __shfl_sync(0xffffffffu, tk, 0);
                    }
                }
            }
            if (nq > 0) {
                // flush: the exact tests of the queue spread over the lanes, the
                // result in bits 29 (member) and 30 (positive side) of each entry
                __syncwarp();
                for (int q = lane; q < nq; q += 32) {
                    const uint32_t e = wq[q];
                    const int l = e & 63, slot = (e >> 6) & 127;
                    const int64_t i = (int64_t)wl_seg[warp][(e >> 13) & 31] * kSegAtoms + slot;
                    bool ps = false;
                    const bool in = slab_member(a.loops[l], a.x[i], a.y[i], a.z[i], a.Lx, a.Ly, a.Lz, a.idLx,
                                                a.idLy, a.idLz, ps);
                    wq[q] = e | (in ? 1u << 29 : 0u) | (ps ? 1u << 30 : 0u);
                }
                __syncwarp();
                // member and removed counts per listed segment, then one block of records
                int tot = 0;
                for (int jj = 0; jj < nlst; ++jj) {
                    const int qo = wl_q[warp][jj] & 0xffff, qn = wl_q[warp][jj] >> 16;
                    unsigned mb[kSegRounds], rbm[kSegRounds];
#pragma unroll
                    for (int r = 0; r < kSegRounds; ++r) { mb[r] = 0u; rbm[r] = 0u; }
                    for (int q0 = 0; q0 < qn; q0 += 32) {
                        unsigned slot = 0xffffffffu;
                        bool rmv = false;
                        if (q0 + lane < qn) {
                            const uint32_t e = wq[qo + q0 + lane];
                            if (e & (1u << 29)) {
                                slot = (e >> 6) & 127;
                                rmv = (vac >> (e & 63)) & 1ull;
                            }
                        }
#pragma unroll
                        for (int r = 0; r < kSegRounds; ++r) {
                            const unsigned bit = (slot >> 5) == (unsigned)r ? 1u << (slot & 31u) : 0u;
                            mb[r] |= __reduce_or_sync(0xffffffffu, bit);
                            rbm[r] |= __reduce_or_sync(0xffffffffu, rmv ? bit : 0u);
                        }
                    }
                    int m = 0, rm = 0;
#pragma unroll
                    for (int r = 0; r < kSegRounds; ++r) { m += __popc(mb[r]); rm += __popc(rbm[r]); }
                    if (lane == 0) wl_mr[warp][jj] = m | (rm << 16);
                    tot += m;
                }
                int base = 0;
                if (lane == 0 && tot > 0) base = (int)atomicAdd(a.ctl + 2, (unsigned)tot);
                base = __shfl_sync(0xffffffffu, base, 0);
                __syncwarp();
                for (int jj = 0; jj < nlst; ++jj) {
                    const int64_t sj = wl_seg[warp][jj];
                    const int m = wl_mr[warp][jj] & 0xffff, rm = wl_mr[warp][jj] >> 16;
                    if (m > 0) {
                        const int qo = wl_q[warp][jj] & 0xffff, qn = wl_q[warp][jj] >> 16;
#pragma unroll
                        for (int r = 0; r < kSegRounds; ++r) { smask[r * 32 + lane] = 0; ssides[r * 32 + lane] = 0; }
                        __syncwarp();
                        for (int q = lane; q < qn; q += 32) {
                            const uint32_t e = wq[qo + q];
                            if (e & (1u << 29)) {
                                const int slot = (e >> 6) & 127;
                                atomicOr(reinterpret_cast<unsigned long long*>(&smask[slot]), 1ull << (e & 63));
                                if (e & (1u << 30))
                                    atomicOr(reinterpret_cast<unsigned long long*>(&ssides[slot]), 1ull << (e & 63));
                            }
                        }
                        __syncwarp();
                        int rc2 = 0, mc2 = 0, off2 = base;
                        aggregate_segment(a, sh, vac, sj, smask, ssides, wcnt[warp], rc2, mc2, off2, lane);
                        __syncwarp();
                    }
                    if (lane == 0) { a.seg_removed[sj] = rm; a.seg_members[sj] = m; a.seg_off[sj] = m > 0 ? base : 0; }
                    base += m;
                }
                __syncwarp();                                   // the queue and the list are rewritten
            }
            if (s >= a.S) break;
        }
        // the warp's per-loop counts into the call's per-loop totals (exact
        // whether or not every member record found room)
        __syncwarp();
        for (int c = lane; c < 2 * nl; c += 32)
            if (wcnt[warp][c]) atomicAdd(a.ctl + kCtlWords + c, (unsigned)wcnt[warp][c]);
    }
    grid_sync(a.ctl, (unsigned)G, err);

    // ---- this CTA's counts: per warp of its contiguous range (the second
    // phase's order) the removed and member atoms and, from the member
    // records, the slab entries and kept copies of every loop
    {
        int rem = 0, mem = 0;
        for (int i = lane; i < 2 * nl; i += 32) wcnt[warp][i] = 0;
        __syncwarp();
        for (int64_t c0 = wlo; c0 < whi; c0 += 32) {
            const int cn = (int)(whi - c0 < 32 ? whi - c0 : 32);
            const int v_rem = lane < cn ? __ldcg(a.seg_removed + c0 + lane) : 0;
            const int v_mem = lane < cn ? __ldcg(a.seg_members + c0 + lane) : 0;
            const int v_off = lane < cn ? __ldcg(a.seg_off + c0 + lane) : 0;
            rem += __reduce_add_sync(0xffffffffu, v_rem);
            mem += __reduce_add_sync(0xffffffffu, v_mem);
            // the batch's member records as one list spread over the lanes
            const int mm = v_mem > 0 && (int64_t)v_off + v_mem <= a.member_cap ? v_mem : 0;
            int incl = mm;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int ex = incl - mm, tot = __shfl_sync(0xffffffffu, incl, 31);
            for (int e0 = 0; e0 < tot; e0 += 32) {
                const int e = e0 + lane;
                int j = 0;                                      // the last segment whose records start at or before e
#pragma unroll
                for (int step = 16; step > 0; step >>= 1)
                    if (__shfl_sync(0xffffffffu, ex, j + step) <= e) j += step;
                const int oj = __shfl_sync(0xffffffffu, v_off, j), exj = __shfl_sync(0xffffffffu, ex, j);
                if (e < tot) {
                    const MemberRec* rec = a.members + oj + (e - exj);
                    const uint64_t mk = __ldcg(reinterpret_cast<const unsigned long long*>(&rec->mask));
                    const bool removed = __ldcg(&rec->removed) != 0;
                    for (uint64_t u = mk; u; u &= u - 1) {
                        const int l = __ffsll((long long)u) - 1;
                        atomicAdd(&wcnt[warp][l], 1);
                        if (sh[l].type == DISCO_MATTER_INTERSTITIAL && !removed) atomicAdd(&wcnt[warp][nl + l], 1);
                    }
                }
            }
        }
        if (lane == 0) { wrem[warp] = rem; wmem[warp] = mem; }
    }
    __syncthreads();
    {
        const int64_t e_hi = seg_hi * kSegAtoms < a.n ? seg_hi * kSegAtoms : a.n;
        const int64_t atoms_k = seg_hi > seg_lo ? e_hi - seg_lo * kSegAtoms : 0;
        for (int c = tid; c < C; c += kMatterThreads) {
            int v = 0;
            for (int w = 0; w < kMatterWarps; ++w)
                v += c == 0 ? wrem[w] : c == 1 ? wmem[w] : wcnt[w][c - 2];
            a.cta_tot[k * C + c] = c == 0 ? (int32_t)(atoms_k - v) : v;
        }
    }
    grid_sync(a.ctl, 2u * (unsigned)G, err);

    // ---- scan: exclusive prefixes over the CTAs per category.  A small grid
    // (small boxes) is scanned by CTA 0 alone, one category per thread; a
    // large one by CTA c for category c.
    if (G <= kSmallGrid) {
        if (blockIdx.x == 0)
            for (int c = tid; c < C; c += kMatterThreads) {
                int64_t runv = 0;
                for (int q = 0; q < G; ++q) {
                    const int32_t v = __ldcg(a.cta_tot + (int64_t)q * C + c);
                    a.cta_pre[(int64_t)q * C + c] = (int32_t)runv;
                    runv += v;
                }
                a.totals[c] = c < 2 ? runv : (int64_t)__ldcg(a.ctl + kCtlWords + (c - 2));
            }
    } else
    for (int c = blockIdx.x; c < C; c += G) {
        const int per = (G + kMatterThreads - 1) / kMatterThreads;
        const int k0 = tid * per;
        int64_t sum = 0;
        for (int q = 0; q < per; ++q)
            if (k0 + q < G) sum += __ldcg(a.cta_tot + (int64_t)(k0 + q) * C + c);
        int64_t incl = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) scan_w[warp] = incl;
        __syncthreads();
        int64_t runv = incl - sum, total = 0;
        for (int w = 0; w < kMatterWarps; ++w) {
            if (w < warp) runv += scan_w[w];
            total += scan_w[w];
        }
        for (int q = 0; q < per; ++q)
            if (k0 + q < G) {
                const int32_t v = __ldcg(a.cta_tot + (int64_t)(k0 + q) * C + c);
                a.cta_pre[(int64_t)(k0 + q) * C + c] = (int32_t)runv;
                runv += v;
            }
        // per-loop totals from the masks (the records may have run out of room)
        if (tid == 0) a.totals[c] = c < 2 ? total : (int64_t)__ldcg(a.ctl + kCtlWords + (c - 2));
        __syncthreads();                                        // scan_w is rewritten
    }
    grid_sync(a.ctl, 3u * (unsigned)G, err);

    // ---- phase 2: survivors, slab entries, copies -------------------------------------
    if (warp == 0) {
        // loop bases (exclusive scans over the loops' totals) plus this CTA's prefix
        int64_t sb = 0, cb = 0;
        for (int l0 = 0; l0 < nl; l0 += 32) {
            const int l = l0 + lane;
            const int64_t ts = l < nl ? __ldcg(a.totals + 2 + l) : 0;
            const int64_t tc = l < nl ? __ldcg(a.totals + 2 + nl + l) : 0;
            int64_t is = ts, ic = tc;
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t ys = __shfl_up_sync(0xffffffffu, is, o);
                const int64_t yc = __shfl_up_sync(0xffffffffu, ic, o);
                if (lane >= o) { is += ys; ic += yc; }
            }
            if (l < nl) {
                run[l] = sb + is - ts + __ldcg(a.cta_pre + k * C + 2 + l);
                run[nl + l] = cb + ic - tc + __ldcg(a.cta_pre + k * C + 2 + nl + l);
            }
            sb += __shfl_sync(0xffffffffu, is, 31);
            cb += __shfl_sync(0xffffffffu, ic, 31);
        }
    }
    __syncthreads();
    {
        const uint64_t last = l2_policy_last_use();
        int64_t* wrun = reinterpret_cast<int64_t*>(wq_raw) + warp * kSegRow;   // this warp's next entry per loop
        uint64_t* smask = reinterpret_cast<uint64_t*>(dyn) + warp * (2 * kSegAtoms);
        uint64_t* ssides = smask + kSegAtoms;
        for (int c = lane; c < 2 * nl; c += 32) {
            int64_t v = run[c];
            for (int w = 0; w < warp; ++w) v += wcnt[w][c];
            wrun[c] = v;
        }
        // survivors before this warp's first segment (earlier warps' segments are full)
        int64_t surv = __ldcg(a.cta_pre + k * C);
        for (int w = 0; w < warp; ++w) {
            const int64_t lo_w = seg_lo + nseg * w / kMatterWarps, hi_w = seg_lo + nseg * (w + 1) / kMatterWarps;
            surv += (hi_w - lo_w) * kSegAtoms - wrem[w];
        }
        __syncwarp();
        int64_t rem_run = 0;                                    // removed atoms of the warp's earlier batches
        for (int64_t c0 = wlo; c0 < whi; c0 += 32) {
            const int cn = (int)(whi - c0 < 32 ? whi - c0 : 32);
            const int v_rem = lane < cn ? __ldcg(a.seg_removed + c0 + lane) : 0;
            const int v_mem = lane < cn ? __ldcg(a.seg_members + c0 + lane) : 0;
            const int v_off = lane < cn ? __ldcg(a.seg_off + c0 + lane) : 0;
            int incl = v_rem;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int ex_rem = incl - v_rem;
            const int64_t base = surv + (c0 - wlo) * kSegAtoms - rem_run;      // survivors before the batch
#pragma unroll 1
            for (int j = 0; j < cn; ++j) {
                const int64_t sbj = base + (int64_t)j * kSegAtoms - __shfl_sync(0xffffffffu, ex_rem, j);
                const int m = __shfl_sync(0xffffffffu, v_mem, j), off = __shfl_sync(0xffffffffu, v_off, j);
                if (m > 0 && (int64_t)off + m <= a.member_cap)
                    copy_members(a, sh, vac, c0 + j, sbj, a.members + off, m, smask, ssides, wrun, last, lane);
                else
                    copy_plain(a, c0 + j, sbj, last, lane);
            }
            rem_run += __shfl_sync(0xffffffffu, incl, 31);
        }
    }

    // the last CTA to leave hands the error word over and clears the control words
    if (tid == 0) {
        __threadfence();
        const unsigned done = atomicAdd(a.ctl + 1, 1u);
        if (done == (unsigned)G - 1u) {
            a.totals[C] = atomicExch(err, 0);
            for (int c = 0; c < 2 * nl; ++c) atomicExch(a.ctl + kCtlWords + c, 0u);
            atomicExch(a.ctl + 0, 0u);
            atomicExch(a.ctl + 2, 0u);
            atomicExch(a.ctl + 4, 0u);
            atomicExch(a.ctl + 1, 0u);
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
    {
        const float bf = (float)h.bound;               // rounded up to the next float
        h.boundf = std::isfinite(bf) && (double)bf < h.bound ? std::nextafter(bf, INFINITY) : bf;
    }
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

// Bytes of the control words (barrier arrivals, exits, member records taken,
// error word, per-loop totals); the last CTA of every completed call leaves
// them at zero.
constexpr size_t kCtlBytes = (disco::kCtlWords + 2 * disco::kMaxSlabLoops) * sizeof(unsigned int);

// CTAs of the cooperative launch on the current device: resident CTAs per SM
// times the SM count, at most kMaxGrid (cached per device; no allocation).
int matter_grid_max(int& out)
{
    static std::mutex mu;
    static int cached[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cfail(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && cached[dev] > 0) { out = cached[dev]; return DISCO_OK; }
    int coop = 0, sms = 0, per_sm = 0;
    e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, disco::matter_kernel, disco::kMatterThreads,
                                                          disco::kMatterSmem);
    if (e != cudaSuccess) return cfail(e, "matter step occupancy");
    if (!coop || per_sm < 1 || sms < 1) return efail(DISCO_ENODEV, "the device takes no cooperative launch of the matter step");
    out = std::min(per_sm * sms, disco::kMaxGrid);
    if (dev >= 0 && dev < 64) cached[dev] = out;
    return DISCO_OK;
}

// Whether the positions and the outputs take 16-byte accesses.
void set_vec_flags(disco::MatterArgs& a)
{
    const uintptr_t in = reinterpret_cast<uintptr_t>(a.x) | reinterpret_cast<uintptr_t>(a.y) |
                         reinterpret_cast<uintptr_t>(a.z);
    const uintptr_t out = reinterpret_cast<uintptr_t>(a.xo) | reinterpret_cast<uintptr_t>(a.yo) |
                          reinterpret_cast<uintptr_t>(a.zo);
    a.vec_in = (in & 15) == 0;
    a.vec_out = (out & 15) == 0 && (reinterpret_cast<uintptr_t>(a.new_index) & 7) == 0;
}

// Segments and CTAs of a call on n atoms.
void matter_shape(int64_t n, int grid_max, int64_t& S, int& G)
{
    S = (n + disco::kSegAtoms - 1) / disco::kSegAtoms;
    const int64_t want = (S + disco::kMatterWarps - 1) / disco::kMatterWarps;   // a segment per warp at least
    G = (int)std::max<int64_t>(1, std::min<int64_t>(grid_max, want));
}

struct MatterScratch {
    unsigned char* loops;        // heads then records (sizeof(LoopStage))
    unsigned int* ctl;           // kCtlBytes
    int32_t* seg;                // 3 S: removed, members, first record per segment
    int32_t* cta;                // 2 G C: counts and prefixes per CTA
    disco::MemberRec* members;
    int64_t member_cap;
    int64_t* totals;             // C + 1 (the last: the kernel's error word)
};

// Queues the matter step on stream s after stage_loops (no host wait): the
// control words cleared when `clear`, then one cooperative launch of G CTAs.
int matter_queue(disco::MatterArgs& a, const MatterScratch& m, int nl, int64_t S, int G, cudaStream_t s, bool clear)
{
    using namespace disco;
    cudaError_t e = cudaSuccess;
    a.heads = reinterpret_cast<const SlabHead*>(m.loops);
    a.loops = reinterpret_cast<const SlabLoopDev*>(m.loops + recs_offset(nl));
    a.nl = nl;
    a.C = 2 + 2 * nl;
    a.G = G;
    a.S = S;
    a.seg_removed = m.seg;
    a.seg_members = m.seg + S;
    a.seg_off = m.seg + 2 * S;
    a.cta_tot = m.cta;
    a.cta_pre = m.cta + (int64_t)G * a.C;
    a.ctl = m.ctl;
    a.members = m.members;
    a.member_cap = m.member_cap;
    a.totals = m.totals;
    // a caller that cannot rely on the previous call's exit (fresh memory, a
    // call that failed half-way) clears the control words here
    if (clear) {
        e = cudaMemsetAsync(m.ctl, 0, kCtlBytes, s);
        if (e != cudaSuccess) return cfail(e, "matter step control words");
    }
    if (S > 0) {
        void* params[] = { &a };
        e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(matter_kernel), dim3((unsigned)G),
                                        dim3(kMatterThreads), params, kMatterSmem, s);
    } else {
        e = cudaMemsetAsync(m.totals, 0, (size_t)(a.C + 1) * sizeof(int64_t), s);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
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
    int grid_max = 0;
    int st = matter_grid_max(grid_max);
    if (st) return st;
    int64_t S = 0;
    int G = 1;
    matter_shape(n, grid_max, S, G);
    const int64_t member_cap = std::max<int64_t>(1, std::min<int64_t>(n, slab_capacity));
    const int64_t scap = std::max<int64_t>(1, slab_capacity), ccap = std::max<int64_t>(1, copy_capacity);

    DevBuf dxyz, dout, didx, dloops, dctl, dseg, dcta, dmem, dtot, dslab, dside, dcop;
    const size_t nb = (size_t)n * sizeof(double);
    const int64_t ns = (n + 1) & ~int64_t(1);           // array stride: every array 16-byte aligned
    cudaError_t e = cudaSuccess;
    if (n > 0) {
        e = cudaMalloc(&dxyz.p, 3 * (size_t)ns * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&dout.p, 3 * (size_t)ns * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&didx.p, (size_t)n * sizeof(int32_t));
    }
    if (e == cudaSuccess) e = cudaMalloc(&dloops.p, sizeof(LoopStage));
    if (e == cudaSuccess) e = cudaMalloc(&dctl.p, kCtlBytes);
    if (e == cudaSuccess) e = cudaMalloc(&dseg.p, 3 * std::max<int64_t>(1, S) * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&dcta.p, 2 * (size_t)G * C * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&dmem.p, (size_t)member_cap * sizeof(MemberRec));
    if (e == cudaSuccess) e = cudaMalloc(&dtot.p, (size_t)(C + 1) * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&dslab.p, (size_t)scap * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&dside.p, (size_t)scap);
    if (e == cudaSuccess) e = cudaMalloc(&dcop.p, (size_t)ccap * sizeof(disco_copy));
    if (e != cudaSuccess) return cfail(e, "prismatic allocation");
    if (n > 0) {
        e = cudaMemcpy(dxyz.as<double>(), x, nb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dxyz.as<double>() + ns, y, nb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dxyz.as<double>() + 2 * ns, z, nb, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) return cfail(e, "prismatic upload");
    st = stage_loops(loops, nloops, box, info, act_index, nl, dloops.as<unsigned char>(), nullptr);
    if (st) return st;

    MatterArgs a;
    std::memset(&a, 0, sizeof(a));
    a.x = dxyz.as<double>(); a.y = a.x + ns; a.z = a.x + 2 * ns;
    a.n = n;
    a.Lx = box[0]; a.Ly = box[1]; a.Lz = box[2];
    a.iLx = (float)(1.0 / box[0]); a.iLy = (float)(1.0 / box[1]); a.iLz = (float)(1.0 / box[2]);
    a.idLx = 1.0 / box[0]; a.idLy = 1.0 / box[1]; a.idLz = 1.0 / box[2];
    a.xo = dout.as<double>(); a.yo = a.xo + ns; a.zo = a.xo + 2 * ns;
    a.new_index = didx.as<int32_t>();
    set_vec_flags(a);
    a.slab_atoms = dslab.as<int32_t>();
    a.slab_side = dside.as<int8_t>();
    a.slab_cap = slab_capacity;
    a.copies = dcop.as<disco_copy>();
    a.copy_cap = copy_capacity;
    MatterScratch m;
    m.loops = dloops.as<unsigned char>();
    m.ctl = dctl.as<unsigned int>();
    m.seg = dseg.as<int32_t>();
    m.cta = dcta.as<int32_t>();
    m.members = dmem.as<MemberRec>();
    m.member_cap = member_cap;
    m.totals = dtot.as<int64_t>();
    st = matter_queue(a, m, nl, S, G, nullptr, true);
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
// from the caller and keeps its scratch (loop table, control words, per-segment
// and per-CTA counts and prefixes, member records, totals) in the file-scope
// array below: 8 MiB
// that every GPU loading this library holds until the process exits.

namespace {

constexpr int64_t kNoAllocMaxAtoms = int64_t(1) << 24;                  // 16 777 216 atoms
constexpr int64_t kNoAllocMaxSegs = kNoAllocMaxAtoms / disco::kSegAtoms;
constexpr int64_t kNoAllocMaxMembers = int64_t(1) << 16;                // atoms in slabs
constexpr size_t align256c(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t kNoAllocLoopOff = 0;
constexpr size_t kNoAllocCtlOff = kNoAllocLoopOff + align256c(sizeof(LoopStage));
constexpr size_t kNoAllocSegOff = kNoAllocCtlOff + align256c(kCtlBytes);
constexpr size_t kNoAllocCtaOff = kNoAllocSegOff + align256c(3 * (size_t)kNoAllocMaxSegs * sizeof(int32_t));
constexpr size_t kNoAllocMemberOff =
    kNoAllocCtaOff + align256c(2 * (size_t)disco::kMaxGrid * disco::kMaxCats * sizeof(int32_t));
constexpr size_t kNoAllocTotalsOff =
    kNoAllocMemberOff + align256c((size_t)kNoAllocMaxMembers * sizeof(disco::MemberRec));
constexpr size_t kNoAllocScratchBytes = 8 * 1024 * 1024;
static_assert(kNoAllocTotalsOff + (disco::kMaxCats + 1) * sizeof(int64_t) <= kNoAllocScratchBytes,
              "no-alloc scratch layout");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_addr[kMaxDevices] = {};
unsigned long long g_noalloc_ctx[kMaxDevices] = {};
bool g_noalloc_dirty[kMaxDevices] = {};     // the control words may not be zero

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
        return efail(DISCO_ELIMIT, "disco_b200_prismatic_noalloc takes at most 16777216 atoms (its scratch array is fixed)");
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
    int grid_max = 0;
    st = matter_grid_max(grid_max);
    if (st) return st;
    int64_t S = 0;
    int G = 1;
    matter_shape(n, grid_max, S, G);
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
    set_vec_flags(a);
    a.slab_atoms = slab_atoms;
    a.slab_side = slab_side;
    a.slab_cap = slab_capacity;
    a.copies = copies;
    a.copy_cap = copy_capacity;
    MatterScratch m;
    m.loops = base + kNoAllocLoopOff;
    m.ctl = reinterpret_cast<unsigned int*>(base + kNoAllocCtlOff);
    m.seg = reinterpret_cast<int32_t*>(base + kNoAllocSegOff);
    m.cta = reinterpret_cast<int32_t*>(base + kNoAllocCtaOff);
    m.members = reinterpret_cast<MemberRec*>(base + kNoAllocMemberOff);
    m.member_cap = member_cap;
    m.totals = reinterpret_cast<int64_t*>(base + kNoAllocTotalsOff);
    const bool dirty = noalloc_dirty(dev, true, false);
    st = matter_queue(a, m, nl, S, G, s, dirty);
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
