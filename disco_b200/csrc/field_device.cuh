// Device building blocks of the displacement kernels (FP64 piece fields,
// image enumeration) and the host helper that packs pieces into chunks.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "field.cuh"

namespace disco {

constexpr int kThreads = 256;
constexpr int kMaxLinePiece = 256;         // segments per piece
constexpr int kMaxLooponPiece = 960;       // loopons per piece (fits a 48 KB stage)
constexpr uint32_t kResidentMax = 110u * 1024u;
constexpr uint32_t kStageMax = 48u * 1024u;
constexpr uint32_t kSmemHeader = 128;      // mbarriers at the start of shared memory

// Image img of the (2 images + 1)^3 cube, kk fastest (Code/backend_cpu.cpp:51-53).
// Returns false for an image inside the inner cube max(|i|,|j|,|k|) < image_min
// (image_min = 2 keeps only the far shells 2 <= max|n| <= images).
__device__ __forceinline__ bool image_shift(int img, int images, int image_min, double Lx, double Ly,
                                            double Lz, double& sx, double& sy, double& sz)
{
    const int W = 2 * images + 1;
    const int ii = img / (W * W) - images;
    const int r = img % (W * W);
    const int jj = r / W - images;
    const int kk = r % W - images;
    sx = Lx * ii;
    sy = Ly * jj;
    sz = Lz * kk;
    const int m = max(abs(ii), max(abs(jj), abs(kk)));
    return m >= image_min;
}

// 1/y for a positive normal y: the hardware approximation (rcp.approx.ftz.f64)
// refined by one cubic Newton-Raphson step r = r0 (1 + e + e^2), e = 1 - y r0,
// which takes its ~2^-22 relative error below the double rounding.
__device__ __forceinline__ double rcp_nr(double y)
{
    double r0;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r0) : "d"(y));
    const double e = fma(-y, r0, 1.0);
    return fma(r0, fma(e, e, e), r0);
}

// 1/sqrt(x) for a positive normal x: the hardware approximation
// (rsqrt.approx.ftz.f64) refined by one cubic Householder step of
// f(r) = 1/r^2 - x:  r = r0 (1 + e/2 + 3 e^2/8), e = 1 - x r0^2.
__device__ __forceinline__ double rsqrt_nr(double x)
{
    double r0;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r0) : "d"(x));
    const double e = fma(-(x * r0), r0, 1.0);
    return fma(r0 * e, fma(0.375, e, 0.5), r0);
}

// J0 = ln((S+L)/(S-L)) = 2 atanh(t), t = L/S, as the series
// 2 t (1 + t^2/3 + ... + t^(2N-2)/(2N-1)); line_terms<N> returns the half,
// t (1 + ...).  Its remainder relative to the sum is below t^(2N)/(2N+1), under
// 2^-53 for t <= 0.012 (N = 4), 0.054 (N = 6), 0.11 (N = 8).
template <int N>
__device__ __forceinline__ double half_j0_series(double t)
{
    const double t2 = t * t;
    double p = 1.0 / (2 * N - 1);
#pragma unroll
    for (int k = N - 2; k >= 0; --k) p = fma(p, t2, 1.0 / (2 * k + 1));
    return t * p;
}

// Series tiers: the warp takes the shortest series valid for all its lanes;
// tier 0 is the logarithm.
constexpr double kSeriesT4 = 0.012, kSeriesT6 = 0.054, kSeriesT8 = 0.11;

// Tier of a lane whose segments all have t <= lmax / gap2 (gap2 > 0).
__device__ __forceinline__ unsigned series_tier(double lmax, double gap2)
{
    return lmax <= kSeriesT4 * gap2 ? 3u : lmax <= kSeriesT6 * gap2 ? 2u : lmax <= kSeriesT8 * gap2 ? 1u : 0u;
}

// The segment loop of one line piece.  NS = 0: J0 from the logarithm; NS > 0:
// every segment is far enough from P (for every lane of the warp) that the
// NS-term series is exact.  The solid angle accumulates as the argument of
// the product of (la lb)(1 + e.ha + e.hb + ha.hb) + i (la lb) e.(ha x hb) over
// the fan triangles (Van Oosterom-Strackee on unnormalised vectors; the
// positive factor la lb does not change the argument), renormalised every 16
// segments.  With d = a - sA t: |d|^2 = |a|^2 - sA^2 and d.w = a.w (w = b x t
// is orthogonal to t), so d is never formed; its term -al d enters as
// -al a + al sA t.  The table holds w' = cK w, so a.w' is cK d.w, and the J0
// term takes cJ / cK (cJK; 2 cJK for the half series).  The K0 term's d^2 > 0
// test reads the sign and zero of d^2 from its bits (integer pipe).
template <int NS>
__device__ __forceinline__ void line_segments(const LineSeg* seg, int nseg, double rx, double ry, double rz,
                                              double ex, double ey, double ez, double ax, double ay, double az,
                                              double cJK, double& zr, double& zi,
                                              double& lx, double& ly, double& lz)
{
    const double c2J = 2.0 * cJK;
    double la2 = ax * ax + ay * ay + az * az;
    double ila = rsqrt_nr(la2);
    double la = la2 * ila;
    double ea = ex * ax + ey * ay + ez * az;                            // e . a
#pragma unroll 4
    for (int k = 0; k < nseg; ++k) {
        const LineSeg s = seg[k];
        const double bx = s.vx + rx, by = s.vy + ry, bz = s.vz + rz;    // B - P
        const double lb2 = bx * bx + by * by + bz * bz;
        const double ilb = rsqrt_nr(lb2);
        const double lb = lb2 * ilb;
        const double eb = ex * bx + ey * by + ez * bz;

        // solid angle of triangle (apex, A, B), Code/barnett.hpp:69-72 times l1 la lb;
        // e.(a x b) = e.((A - apex) x (B - apex)) as e is along apex - P
        const double den = fma(ea, lb, fma(eb, la, fma(la, lb, fma(0.5, la2 + lb2, -s.hl2))));   // a.b = (|a|^2 + |b|^2 - L^2) / 2
        const double num = ex * s.nx + ey * s.ny + ez * s.nz;
        const double nzr = zr * den - zi * num;
        zi = zr * num + zi * den;
        zr = nzr;

        // segment A -> B (Code/barnett.hpp:75-100)
        const double sA = ax * s.tx + ay * s.ty + az * s.tz;
        const double sB = sA + s.len;
        const double d2 = fma(-sA, sA, la2);
        const double dw = ax * s.wx + ay * s.wy + az * s.wz;             // cK d.w
        const double sum = la + lb;
        double ga;
        if (NS > 0) ga = c2J * half_j0_series<NS>(s.len * rcp_nr(sum));
        else        ga = cJK * log((sum + s.len) * rcp_nr(sum - s.len));
        const double g = sB * ilb - sA * ila;                           // d^2 K0
        const double al = __double_as_longlong(d2) > 0 ? dw * rcp_nr(d2) * g : 0.0;
        const double be = dw * (ila - ilb);                             // cK d.w K1
        const double c = fma(al, sA, -be);
        lx = fma(c, s.tx, fma(-al, ax, fma(ga, s.wx, lx)));
        ly = fma(c, s.ty, fma(-al, ay, fma(ga, s.wy, ly)));
        lz = fma(c, s.tz, fma(-al, az, fma(ga, s.wz, lz)));

        ax = bx; ay = by; az = bz;
        la2 = lb2; la = lb; ila = ilb;
        ea = eb;
        if ((k & 15) == 15) {                                           // keep |z| in range
            const double sc = rcp_nr(fabs(zr) + fabs(zi));
            zr *= sc; zi *= sc;
        }
    }
}

// Solid angle of a piece's fan seen from P as Code/barnett.hpp:56-72 computes
// it: per triangle (apex, A, B), 2 atan2(num, den) with num = r1.(a x b),
// den = l1 la lb + (r1.a) lb + (r1.b) la + (a.b) l1, from r1 = apex - P,
// a = A - P, b = B - P formed from the input vertices, every operation in the
// source's order and rounded on its own (no contraction).  For an atom on the
// loop's plane inside the contour, num is a rounding residue (or a signed
// zero) and its sign is the branch that puts the atom on one side of the cut
// (Omega = +-2 pi); for an atom on a fan edge or at the apex the per-triangle
// arguments are residues too.  Evaluating the reference's expressions
// operation for operation reproduces its choice in every such case.
static __device__ __noinline__ double fan_solid_angle_ref(const double* __restrict__ v, int nseg, double cx, double cy,
                                                   double cz, double px, double py, double pz)
{
    const double r1x = __dsub_rn(cx, px), r1y = __dsub_rn(cy, py), r1z = __dsub_rn(cz, pz);
    const double l1 = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(r1x, r1x), __dmul_rn(r1y, r1y)),
                                           __dmul_rn(r1z, r1z)));
    double ax = __dsub_rn(__ldg(v), px), ay = __dsub_rn(__ldg(v + 1), py), az = __dsub_rn(__ldg(v + 2), pz);
    double la = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay)), __dmul_rn(az, az)));
    double omega = 0.0;
    for (int k = 1; k <= nseg; ++k) {
        const double bx = __dsub_rn(__ldg(v + 3 * k), px), by = __dsub_rn(__ldg(v + 3 * k + 1), py),
                     bz = __dsub_rn(__ldg(v + 3 * k + 2), pz);
        const double lb = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(bx, bx), __dmul_rn(by, by)), __dmul_rn(bz, bz)));
        const double cxx = __dsub_rn(__dmul_rn(ay, bz), __dmul_rn(az, by));
        const double cyy = __dsub_rn(__dmul_rn(az, bx), __dmul_rn(ax, bz));
        const double czz = __dsub_rn(__dmul_rn(ax, by), __dmul_rn(ay, bx));
        const double num = __dadd_rn(__dadd_rn(__dmul_rn(r1x, cxx), __dmul_rn(r1y, cyy)), __dmul_rn(r1z, czz));
        const double ra = __dadd_rn(__dadd_rn(__dmul_rn(r1x, ax), __dmul_rn(r1y, ay)), __dmul_rn(r1z, az));
        const double rb = __dadd_rn(__dadd_rn(__dmul_rn(r1x, bx), __dmul_rn(r1y, by)), __dmul_rn(r1z, bz));
        const double ab = __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
        const double den = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(l1, la), lb), __dmul_rn(ra, lb)),
                                               __dmul_rn(rb, la)), __dmul_rn(ab, l1));
        omega = __dadd_rn(omega, __dmul_rn(2.0, atan2(num, den)));
        ax = bx; ay = by; az = bz; la = lb;
    }
    return omega;
}

// Field at P (an atom moved by minus an image shift) of one line piece.
// Follows Code/barnett.hpp:55-106 term by term (see field.cu's header for the
// reformulations); adds b Omega/(4 pi) + the line terms to (ux, uy, uz).
// Vertices are stored relative to the apex; r = apex - P.  For every segment,
// RA + RB >= 2 (l1 - rho) with l1 = |apex - P| and rho the piece's largest
// vertex radius, so t = L/(RA+RB) <= lmax / (2 (l1 - rho)).
// For an atom within hband of the loop's plane (a little more than the
// plane's own rounding) the solid angle is left out and `plane` is set: the
// caller adds it from fan_solid_angle_ref (line_piece_plane) in a second pass,
// since on the plane the running product's sign is a rounding residue of
// other operations than the reference's.  Outside the band the product's
// argument is at least about pi hband / rho away from the branch cut, far
// above its rounding.
__device__ __forceinline__ void line_piece_fp64(const LinePiece& pc, const LineSeg* seg,
                                                double Px, double Py, double Pz, double cJK,
                                                double& ux, double& uy, double& uz, bool& plane)
{
    // unit vector from P to the fan apex
    const double rx = pc.cx - Px, ry = pc.cy - Py, rz = pc.cz - Pz;
    const bool on_plane = fabs(pc.nx * rx + pc.ny * ry + pc.nz * rz) <= pc.hband;
    const double l1sq = rx * rx + ry * ry + rz * rz;
    const double il1 = rsqrt_nr(l1sq);
    const double ex = rx * il1, ey = ry * il1, ez = rz * il1;
    const double gap = l1sq * il1 - pc.rho;
    const unsigned mine = gap > 0.0 ? series_tier(pc.lmax, 2.0 * gap) : 0u;
    const unsigned tier = __reduce_min_sync(__activemask(), mine);

    double zr = 1.0, zi = 0.0, lx = 0.0, ly = 0.0, lz = 0.0;
    const double ax = pc.ax + rx, ay = pc.ay + ry, az = pc.az + rz;
    switch (tier) {
    case 3:  line_segments<4>(seg, pc.nseg, rx, ry, rz, ex, ey, ez, ax, ay, az, cJK, zr, zi, lx, ly, lz); break;
    case 2:  line_segments<6>(seg, pc.nseg, rx, ry, rz, ex, ey, ez, ax, ay, az, cJK, zr, zi, lx, ly, lz); break;
    case 1:  line_segments<8>(seg, pc.nseg, rx, ry, rz, ex, ey, ez, ax, ay, az, cJK, zr, zi, lx, ly, lz); break;
    default: line_segments<0>(seg, pc.nseg, rx, ry, rz, ex, ey, ez, ax, ay, az, cJK, zr, zi, lx, ly, lz); break;
    }
    double f = atan2(zi, zr) * (1.0 / 6.283185307179586476925286766559);   // Omega / (4 pi)
    if (on_plane) { f = 0.0; plane = true; }
    ux += pc.bx * f + lx;
    uy += pc.by * f + ly;
    uz += pc.bz * f + lz;
}

// The solid-angle term b Omega/(4 pi) of one line piece for an atom in its
// plane band (the part line_piece_fp64 leaves out there); nothing otherwise.
__device__ __forceinline__ void line_piece_plane(const LinePiece& pc, const double* raw, double Px, double Py,
                                                 double Pz, double& ux, double& uy, double& uz)
{
    const double rx = pc.cx - Px, ry = pc.cy - Py, rz = pc.cz - Pz;
    if (!(fabs(pc.nx * rx + pc.ny * ry + pc.nz * rz) <= pc.hband)) return;
    const double f = fan_solid_angle_ref(raw + 3 * (size_t)pc.raw, pc.nseg, pc.cx, pc.cy, pc.cz, Px, Py, Pz) *
                     (1.0 / 12.566370614359172953850573533118);                 // Omega / (4 pi)
    ux += pc.bx * f;
    uy += pc.by * f;
    uz += pc.bz * f;
}

// Field at P (atom - reference point - image shift) of one loopon piece:
// Code/kroupa.hpp:52-73 regrouped.  With ir = 1/rho, mr = m.rho, nr = n.rho:
//   du = fac fb (k2 (n mr + m nr - rho b_n) + tail rho),  k2 = c2 ir,
//   tail = 3 mr nr ir^3,  fac = ir^2 (0 for rho < 1e-10)
// is fac fb (alpha n + beta m + gamma rho) with alpha = c2 ir mr,
// beta = c2 ir nr, gamma = ir (3 mr nr ir^2 - c2 b_n); fb factors out of the
// sum over the piece's loopons.  1/rho from the kernels' own rsqrt.
__device__ __forceinline__ void loopon_piece_fp64(const LooponPiece& pc, const LooponRec* __restrict__ rec,
                                                  double Px, double Py, double Pz, double c2,
                                                  double& ux, double& uy, double& uz)
{
    const double mP = pc.mx * Px + pc.my * Py + pc.mz * Pz;
    const double nP = pc.nx * Px + pc.ny * Py + pc.nz * Pz;
    const double c2bn = c2 * pc.b_n;
    double dx = 0.0, dy = 0.0, dz = 0.0;
    const int n = pc.n;
#pragma unroll 2
    for (int k = 0; k < n; ++k) {
        const LooponRec l = rec[k];
        const double rx = Px - l.x, ry = Py - l.y, rz = Pz - l.z;
        const double r2 = rx * rx + ry * ry + rz * rz;
        const bool keep = r2 >= 1e-20;                           // rho >= 1e-10 (kroupa.hpp:55)
        const double ir = rsqrt_nr(keep ? r2 : 1.0);
        const double ir2 = ir * ir;
        const double mr = mP - l.ml, nr = nP - l.nl;
        const double cir = c2 * ir;
        const double al = cir * mr, be = cir * nr;
        const double ga = ir * fma(3.0 * mr * nr, ir2, -c2bn);
        const double fac = keep ? ir2 : 0.0;
        dx = fma(fac, fma(al, pc.nx, fma(be, pc.mx, ga * rx)), dx);
        dy = fma(fac, fma(al, pc.ny, fma(be, pc.my, ga * ry)), dy);
        dz = fma(fac, fma(al, pc.nz, fma(be, pc.mz, ga * rz)), dz);
    }
    ux = fma(pc.fbx, dx, ux);
    uy = fma(pc.fby, dy, uy);
    uz = fma(pc.fbz, dz, uz);
}

// ---- the two FP64 policies ----------------------------------------------------------------

struct AccF64 {
    double x, y, z;
    __device__ void clear() { x = y = z = 0.0; }
    __device__ void total(double& ux, double& uy, double& uz) const { ux = x; uy = y; uz = z; }
};

struct LineFp64 {
    using Acc = AccF64;
    static constexpr int kMinBlocks = 2;
    static constexpr bool kAppendsNear = false;
    template <int S>
    static __device__ __forceinline__ void chunk(const FieldArgs& a, const unsigned char* st, int npieces,
                                                 int split, double px, double py, double pz, Acc& acc)
    {
        const LinePiece* pieces = reinterpret_cast<const LinePiece*>(st);
        const LineSeg* recs = reinterpret_cast<const LineSeg*>(st + (size_t)npieces * sizeof(LinePiece));
        const double cJK = a.cJ / a.cK;
        bool plane = false;
        for (int p = 0; p < npieces; ++p) {
            const LinePiece& pc = pieces[p];
            for (int img = split; img < a.nimg; img += S) {
                double sx, sy, sz;
                if (!image_shift(img, a.images, a.image_min, a.Lx, a.Ly, a.Lz, sx, sy, sz)) continue;
                line_piece_fp64(pc, recs + pc.rec, px - sx, py - sy, pz - sz, cJK, acc.x, acc.y, acc.z, plane);
            }
        }
        if (plane) {                        // an atom in a loop's plane band: the reference's solid angle
            for (int p = 0; p < npieces; ++p) {
                const LinePiece& pc = pieces[p];
                for (int img = split; img < a.nimg; img += S) {
                    double sx, sy, sz;
                    if (!image_shift(img, a.images, a.image_min, a.Lx, a.Ly, a.Lz, sx, sy, sz)) continue;
                    line_piece_plane(pc, a.raw, px - sx, py - sy, pz - sz, acc.x, acc.y, acc.z);
                }
            }
        }
    }
};

struct LooponFp64 {
    using Acc = AccF64;
    static constexpr int kMinBlocks = 2;
    static constexpr bool kAppendsNear = false;
    template <int S>
    static __device__ __forceinline__ void chunk(const FieldArgs& a, const unsigned char* st, int npieces,
                                                 int split, double px, double py, double pz, Acc& acc)
    {
        const LooponPiece* pieces = reinterpret_cast<const LooponPiece*>(st);
        const LooponRec* recs = reinterpret_cast<const LooponRec*>(st + (size_t)npieces * sizeof(LooponPiece));
        for (int p = 0; p < npieces; ++p) {
            const LooponPiece& pc = pieces[p];
            const double qx = px - pc.cx, qy = py - pc.cy, qz = pz - pc.cz;
            for (int img = split; img < a.nimg; img += S) {
                double sx, sy, sz;
                if (!image_shift(img, a.images, a.image_min, a.Lx, a.Ly, a.Lz, sx, sy, sz)) continue;
                loopon_piece_fp64(pc, recs + pc.rec, qx - sx, qy - sy, qz - sz, a.c2, acc.x, acc.y, acc.z);
            }
        }
    }
};

// Persistent kernel: CTA b takes atom tiles b, b + grid, ...; for each tile it
// walks the chunks of the table (staged in shared memory) and, per piece, the
// images of its lane's share.
template <class Policy, int S>
__global__ void __launch_bounds__(kThreads, Policy::kMinBlocks) field_kernel(const FieldArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    unsigned char* const stage0 = smem + kSmemHeader;
    const int tid = threadIdx.x;
    constexpr int kAtomsPerCta = kThreads / S;
    // the atoms: all of them, or (FP64 near pass) those the FP32 pass listed
    int64_t n = a.n;
    const int32_t* list = nullptr;
    if (a.near_mode == 2 && a.near_list) {
        const unsigned c = *a.near_count;
        if (c <= (unsigned)a.near_cap) { n = c; list = a.near_list; }
    }
    const int64_t ntiles = (n + kAtomsPerCta - 1) / kAtomsPerCta;
    if ((int64_t)blockIdx.x >= ntiles) return;
    const int nch = a.nchunks;
    const bool resident = a.resident != 0;
    const int64_t my_tiles = (ntiles - 1 - (int64_t)blockIdx.x) / gridDim.x + 1;
    const int64_t nunits = resident ? my_tiles : my_tiles * nch;

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int64_t u) {
        const int ch = resident ? 0 : (int)(u % nch);
        const int buf = resident ? 0 : (int)(u & 1);
        const Chunk c = a.chunks[ch];
        stage_load(stage0 + (size_t)buf * a.stage_bytes, a.table + c.offset, c.bytes, &bar[buf]);
    };
    if (tid == 0) {
        issue(0);
        if (!resident && nunits > 1) issue(1);
    }

    const int split = tid % S;
    double px = 0.0, py = 0.0, pz = 0.0;
    typename Policy::Acc acc;
    int64_t atom = 0;
    bool valid = false;
    for (int64_t u = 0; u < nunits; ++u) {
        const int64_t tk = resident ? u : u / nch;
        const int ch = resident ? 0 : (int)(u % nch);
        const int buf = resident ? 0 : (int)(u & 1);
        if (ch == 0) {
            const int64_t tile = (int64_t)blockIdx.x + tk * gridDim.x;
            const int64_t k = tile * kAtomsPerCta + tid / S;
            valid = k < n;
            const int64_t ik = valid ? k : n - 1;
            atom = list ? (int64_t)list[ik] : ik;
            px = a.x[atom]; py = a.y[atom]; pz = a.z[atom];
            acc.clear();
        }
        if (!resident || u == 0) {
            const uint32_t parity = resident ? 0u : (uint32_t)((u >> 1) & 1);
            const bool ok = mbar_wait_bounded(&bar[buf], parity);
            if (__syncthreads_or(!ok)) {
                // give up: record it, let the copies still in flight land, return
                if (tid == 0) {
                    report(a.status, DISCO_ETIMEOUT);
                    mbar_wait_bounded(&bar[buf], parity);
                    if (!resident && u + 1 < nunits)
                        mbar_wait_bounded(&bar[buf ^ 1], (uint32_t)(((u + 1) >> 1) & 1));
                }
                __syncthreads();
                return;
            }
        }
        const unsigned char* st = stage0 + (size_t)buf * a.stage_bytes;
        Policy::template chunk<S>(a, st, a.chunks[ch].npieces, split, px, py, pz, acc);
        if (resident || ch == nch - 1) {
            double ux, uy, uz;
            acc.total(ux, uy, uz);
#pragma unroll
            for (int o = S / 2; o > 0; o >>= 1) {
                ux += __shfl_xor_sync(0xffffffffu, ux, o);
                uy += __shfl_xor_sync(0xffffffffu, uy, o);
                uz += __shfl_xor_sync(0xffffffffu, uz, o);
            }
            if (valid && split == 0) {
                a.ux[atom] += ux;
                a.uy[atom] += uy;
                a.uz[atom] += uz;
            }
            if constexpr (Policy::kAppendsNear) {
                if (a.near_mode == 1) {
                    // list the atom if any of its S lanes met a near-cut pair
                    const int lane = tid & 31;
                    const unsigned b = __ballot_sync(0xffffffffu, acc.near);
                    const unsigned grp = S == 32 ? 0xffffffffu : (((1u << S) - 1u) << (lane & ~(S - 1)));
                    const bool app = valid && split == 0 && (b & grp) != 0u;
                    const unsigned ba = __ballot_sync(0xffffffffu, app);
                    if (ba) {
                        const int leader = __ffs(ba) - 1;
                        unsigned q0 = 0;
                        if (lane == leader) q0 = atomicAdd(a.near_count, (unsigned)__popc(ba));
                        q0 = __shfl_sync(0xffffffffu, q0, leader);
                        const unsigned q = q0 + (unsigned)__popc(ba & ((1u << lane) - 1u));
                        if (app && q < (unsigned)a.near_cap) a.near_list[q] = (int32_t)atom;
                    }
                }
            }
        }
        if (!resident) {
            __syncthreads();                       // every warp is done with stage[buf]
            if (tid == 0 && u + 2 < nunits) {
                fence_proxy_async_smem();
                issue(u + 2);
            }
        }
    }
}


// ---- host: tables -----------------------------------------------------------------------


// One FP64 line piece: segments k0..k1e-1 of loop lp (segment k runs from
// vertex k-1 to vertex k; Code/barnett.hpp:62-65), with everything that does
// not depend on the atom precomputed; w is stored times cK = 1/(8 pi (1 - nu)).
// rec is left to the chunk packer.  The piece's input vertices (A of its
// first segment, then every B) are appended to raw as x, y, z triplets; the
// loop's mean plane (unit area vector n) and the largest distance of a vertex
// from it give the band |n.(apex - P)| <= hband in which the kernel takes the
// solid angle per triangle (a zero-area loop: everywhere).
inline void make_line_piece(const disco_loop& lp, int k0, int k1e, double bx, double by, double bz,
                            double cK, LinePiece& p, std::vector<LineSeg>& recs, std::vector<double>& raw)
{
    const int nv = lp.n_vertices;
    std::memset(&p, 0, sizeof(p));
    const int a = (k0 + nv - 1) % nv;
    const double c[3] = { lp.cx, lp.cy, lp.cz };
    {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int k = 0; k < nv; ++k) {
            const int km = (k + nv - 1) % nv;
            const double ux = lp.vx[km] - c[0], uy = lp.vy[km] - c[1], uz = lp.vz[km] - c[2];
            const double vx = lp.vx[k] - c[0], vy = lp.vy[k] - c[1], vz = lp.vz[k] - c[2];
            sx += uy * vz - uz * vy;
            sy += uz * vx - ux * vz;
            sz += ux * vy - uy * vx;
        }
        const double s = std::sqrt(sx * sx + sy * sy + sz * sz);
        if (s > 0.0 && std::isfinite(s)) {
            p.nx = sx / s; p.ny = sy / s; p.nz = sz / s;
            double dev = 0.0;
            for (int k = 0; k < nv; ++k)
                dev = std::max(dev, std::fabs(p.nx * (lp.vx[k] - c[0]) + p.ny * (lp.vy[k] - c[1]) +
                                              p.nz * (lp.vz[k] - c[2])));
            p.hband = 2.0 * dev + 1e-8;
        } else {
            p.hband = HUGE_VAL;
        }
    }
    p.raw = (int32_t)(raw.size() / 3);
    raw.push_back(lp.vx[a]); raw.push_back(lp.vy[a]); raw.push_back(lp.vz[a]);
    for (int k = k0; k < k1e; ++k) { raw.push_back(lp.vx[k]); raw.push_back(lp.vy[k]); raw.push_back(lp.vz[k]); }
    p.ax = lp.vx[a] - c[0]; p.ay = lp.vy[a] - c[1]; p.az = lp.vz[a] - c[2];
    p.cx = c[0]; p.cy = c[1]; p.cz = c[2];
    p.bx = bx; p.by = by; p.bz = bz;
    p.nseg = k1e - k0;
    auto radius = [&](int k) {
        const double dx = lp.vx[k] - c[0], dy = lp.vy[k] - c[1], dz = lp.vz[k] - c[2];
        return std::sqrt(dx * dx + dy * dy + dz * dz);
    };
    p.rho = radius(a);
    recs.clear();
    for (int k = k0; k < k1e; ++k) {
        const int km = (k + nv - 1) % nv;
        LineSeg s;
        std::memset(&s, 0, sizeof(s));
        s.vx = lp.vx[k] - c[0]; s.vy = lp.vy[k] - c[1]; s.vz = lp.vz[k] - c[2];
        const double ux = lp.vx[km] - c[0], uy = lp.vy[km] - c[1], uz = lp.vz[km] - c[2];
        s.nx = uy * s.vz - uz * s.vy;
        s.ny = uz * s.vx - ux * s.vz;
        s.nz = ux * s.vy - uy * s.vx;
        const double tx = lp.vx[k] - lp.vx[km], ty = lp.vy[k] - lp.vy[km], tz = lp.vz[k] - lp.vz[km];
        const double L = std::sqrt(tx * tx + ty * ty + tz * tz);
        if (L > 0.0) {
            s.len = L;
            s.tx = tx / L; s.ty = ty / L; s.tz = tz / L;
            s.wx = cK * (by * s.tz - bz * s.ty);
            s.wy = cK * (bz * s.tx - bx * s.tz);
            s.wz = cK * (bx * s.ty - by * s.tx);
        }
        s.hl2 = 0.5 * L * L;
        p.rho = std::max(p.rho, radius(k));
        p.lmax = std::max(p.lmax, L);
        recs.push_back(s);
    }
    // a little slack so that rounding in the kernel's bound never matters
    p.rho *= 1.0 + 1e-12;
    p.lmax *= 1.0 + 1e-12;
}

template <class Piece, class Rec>
struct PieceList {
    std::vector<Piece> pieces;
    std::vector<std::vector<Rec>> recs;
};

// Packs the pieces into chunks.  stage_cap == 0: one resident chunk when the
// table fits in kResidentMax, else stages of kStageMax; stage_cap > 0: stages
// of at most stage_cap bytes (never resident, as the batched kernel needs).
template <class Piece, class Rec>
void pack_chunks(PieceList<Piece, Rec>& L, HostTable& T, uint32_t stage_cap = 0)
{
    size_t total = 0;
    for (size_t i = 0; i < L.pieces.size(); ++i) total += sizeof(Piece) + L.recs[i].size() * sizeof(Rec);
    const bool resident = stage_cap == 0 && total <= kResidentMax;
    const uint32_t cap = resident ? kResidentMax : (stage_cap ? stage_cap : kStageMax);
    T.resident = resident;
    T.bytes.clear();
    T.chunks.clear();
    size_t i = 0;
    uint32_t max_bytes = 16;
    while (i < L.pieces.size()) {
        // the longest run of pieces that fits in one stage
        size_t j = i, bytes = 0;
        while (j < L.pieces.size()) {
            const size_t add = sizeof(Piece) + L.recs[j].size() * sizeof(Rec);
            if (j > i && bytes + add > cap) break;
            bytes += add;
            ++j;
        }
        Chunk c;
        c.offset = T.bytes.size();
        c.bytes = (uint32_t)((bytes + 15) & ~size_t(15));
        c.npieces = (int32_t)(j - i);
        std::vector<unsigned char> blob(c.bytes, 0);
        int32_t rec = 0;
        for (size_t k = i; k < j; ++k) {
            Piece p = L.pieces[k];
            p.rec = rec;
            std::memcpy(blob.data() + (k - i) * sizeof(Piece), &p, sizeof(Piece));
            rec += (int32_t)L.recs[k].size();
        }
        size_t off = (j - i) * sizeof(Piece);
        for (size_t k = i; k < j; ++k) {
            std::memcpy(blob.data() + off, L.recs[k].data(), L.recs[k].size() * sizeof(Rec));
            off += L.recs[k].size() * sizeof(Rec);
        }
        T.bytes.insert(T.bytes.end(), blob.begin(), blob.end());
        T.chunks.push_back(c);
        max_bytes = std::max(max_bytes, c.bytes);
        i = j;
    }
    if (T.chunks.size() <= 1 && stage_cap == 0) T.resident = true;
    T.stage_bytes = max_bytes;
}



} // namespace disco
