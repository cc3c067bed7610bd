// Device side of the FP32 compensated form (DISCO_FP32C): Kahan accumulator,
// FP32 piece fields, the near-cut test and the three policies of the
// persistent kernel skeleton (field_device.cuh).
#pragma once

#include "field_device.cuh"

namespace disco {

constexpr float kNearPlane = 3.0f;   // A from the loop plane
constexpr float kNearRim = 3.0f;     // A beyond the largest vertex radius

// Kahan-compensated FP32 sums plus an FP64 part (near-cut evaluations).
struct AccF32K {
    float sx, sy, sz, cx, cy, cz;
    double dx, dy, dz;
    bool near;                 // a near-cut pair was skipped (left to the FP64 pass)
    __device__ void clear()
    {
        sx = sy = sz = cx = cy = cz = 0.0f;
        dx = dy = dz = 0.0;
        near = false;
    }
    __device__ __forceinline__ static void kahan(float& s, float& c, float v)
    {
        const float y = __fsub_rn(v, c);
        const float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    __device__ __forceinline__ void add(float x, float y, float z)
    {
        kahan(sx, cx, x);
        kahan(sy, cy, y);
        kahan(sz, cz, z);
    }
    __device__ void total(double& ux, double& uy, double& uz) const
    {
        ux = ((double)sx - (double)cx) + dx;
        uy = ((double)sy - (double)cy) + dy;
        uz = ((double)sz - (double)cz) + dz;
    }
};

// The hardware approximations with denormals flushed (single MUFU
// operations; every argument here is a normal number: the near cut keeps an
// atom at least near_h from the loop plane or near_r beyond its rim, and a
// loopon's rho^2 is at least 1e-20).
__device__ __forceinline__ float rsqrt_ftz(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float rcp_ftz(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float lg2_ftz(float x)
{
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Code/barnett.hpp:44-107 in FP32 on centre-relative coordinates, with the
// same reformulation as line_piece_fp64: the solid angle as the argument of
// the product of unnormalised Van Oosterom-Strackee factors (renormalised
// every 4 segments, well inside the FP32 range), e.(a x b) from the segment's
// precomputed (A - apex) x (B - apex), |d|^2 = |a|^2 - sA^2 and d.w = a.w
// without forming d.  In FP32 |a|^2 - sA^2 loses digits for an atom near the
// extension of a segment, but the term it enters carries d^2 through
// d^2 K0 = sB/RB - sA/RA, so its absolute error stays below
// cK |w| 2^-23 per segment.  The table holds w' = cK w, so d.w' is cK d.w and
// the J0 term takes cJ ln2 / cK (cJK2, with J0 from the base-2 logarithm).
// The solid-angle renormalisation only needs some positive scale, so an
// approximate reciprocal serves.
__device__ __forceinline__ void line_piece_fp32(const LinePieceF& pc, const LineSegF* seg, float Px,
                                                float Py, float Pz, float cJK2,
                                                float& ux, float& uy, float& uz)
{
    // apex = centre = origin of these coordinates
    const float il1 = rsqrt_ftz(Px * Px + Py * Py + Pz * Pz);
    const float ex = -Px * il1, ey = -Py * il1, ez = -Pz * il1;
    float ax = pc.ax - Px, ay = pc.ay - Py, az = pc.az - Pz;
    float la2 = ax * ax + ay * ay + az * az;
    float ila = rsqrt_ftz(la2);
    float la = la2 * ila;
    float ea = ex * ax + ey * ay + ez * az;
    float zr = 1.0f, zi = 0.0f, lx = 0.0f, ly = 0.0f, lz = 0.0f;
    const int nseg = pc.nseg;
#pragma unroll 8
    for (int k = 0; k < nseg; ++k) {
        const LineSegF s = seg[k];
        const float bx = s.vx - Px, by = s.vy - Py, bz = s.vz - Pz;
        const float lb2 = bx * bx + by * by + bz * bz;
        const float ilb = rsqrt_ftz(lb2);
        const float lb = lb2 * ilb;
        const float eb = ex * bx + ey * by + ez * bz;
        const float den = fmaf(ea, lb, fmaf(eb, la, fmaf(la, lb, fmaf(0.5f, la2 + lb2, -s.hl2))));   // a.b
        const float num = ex * s.nx + ey * s.ny + ez * s.nz;
        const float nzr = zr * den - zi * num;
        zi = zr * num + zi * den;
        zr = nzr;
        const float sA = ax * s.tx + ay * s.ty + az * s.tz;
        const float sB = sA + s.len;
        const float d2 = fmaf(-sA, sA, la2);
        const float dw = ax * s.wx + ay * s.wy + az * s.wz;          // cK d.w
        const float sum = la + lb;
        const float ga = cJK2 * lg2_ftz((sum + s.len) * rcp_ftz(sum - s.len));
        const float g = sB * ilb - sA * ila;
        const float al = d2 > 0.0f ? dw * rcp_ftz(d2) * g : 0.0f;
        const float be = dw * (ila - ilb);
        const float c = fmaf(al, sA, -be);
        lx = fmaf(c, s.tx, fmaf(-al, ax, fmaf(ga, s.wx, lx)));
        ly = fmaf(c, s.ty, fmaf(-al, ay, fmaf(ga, s.wy, ly)));
        lz = fmaf(c, s.tz, fmaf(-al, az, fmaf(ga, s.wz, lz)));
        ax = bx; ay = by; az = bz;
        la2 = lb2; la = lb; ila = ilb;
        ea = eb;
        if ((k & 3) == 3) {
            const float sc = rcp_ftz(fabsf(zr) + fabsf(zi));
            zr *= sc; zi *= sc;
        }
    }
    const float f = atan2f(zi, zr) * 0.15915494309189533577f;    // Omega / (4 pi)
    ux += pc.bx * f + lx;
    uy += pc.by * f + ly;
    uz += pc.bz * f + lz;
}

// Code/kroupa.hpp:52-73 in FP32 on centre-relative coordinates.
__device__ __forceinline__ void loopon_piece_fp32(const LooponPieceF& pc, const LooponRecF* rec, float Px,
                                                  float Py, float Pz, float c2, float& ux, float& uy,
                                                  float& uz)
{
    // regrouped as loopon_piece_fp64: fb (alpha n + beta m + gamma rho) fac
    const float mP = pc.mx * Px + pc.my * Py + pc.mz * Pz;
    const float nP = pc.nx * Px + pc.ny * Py + pc.nz * Pz;
    const float c2bn = c2 * pc.b_n;
    float dx = 0.0f, dy = 0.0f, dz = 0.0f;
    const int n = pc.n;
#pragma unroll 2
    for (int k = 0; k < n; ++k) {
        const LooponRecF l = rec[k];
        const float rx = Px - l.x, ry = Py - l.y, rz = Pz - l.z;
        const float r2 = rx * rx + ry * ry + rz * rz;
        const bool keep = r2 >= 1e-20f;
        const float ir = rsqrt_ftz(keep ? r2 : 1.0f);
        const float ir2 = ir * ir;
        const float mr = mP - l.ml, nr = nP - l.nl;
        const float cir = c2 * ir;
        const float al = cir * mr, be = cir * nr;
        const float ga = ir * fmaf(3.0f * mr * nr, ir2, -c2bn);
        const float fac = keep ? ir2 : 0.0f;
        dx = fmaf(fac, fmaf(al, pc.nx, fmaf(be, pc.mx, ga * rx)), dx);
        dy = fmaf(fac, fmaf(al, pc.ny, fmaf(be, pc.my, ga * ry)), dy);
        dz = fmaf(fac, fmaf(al, pc.nz, fmaf(be, pc.mz, ga * rz)), dz);
    }
    ux += pc.fbx * dx; uy += pc.fby * dy; uz += pc.fbz * dz;
}

// The near-cut test, shared by the FP32 pass (which skips what it selects)
// and the FP64 pass (which evaluates only that): the same FP32 arithmetic on
// the same inputs, so every (atom, piece, image) is counted exactly once.
__device__ __forceinline__ bool near_cut(const LinePieceF& pc, float Px, float Py, float Pz, float near_h,
                                         float near_r)
{
    const float h = pc.nx * Px + pc.ny * Py + pc.nz * Pz;
    const float r2 = Px * Px + Py * Py + Pz * Pz - h * h;
    const float rim = pc.rmax + near_r;
    return fabsf(h) < near_h && r2 < rim * rim;
}

struct LineFp32 {
    using Acc = AccF32K;
    static constexpr int kMinBlocks = 2;
    static constexpr bool kAppendsNear = true;
    template <int S>
    static __device__ __forceinline__ void chunk(const FieldArgs& a, const unsigned char* st, int npieces,
                                                 int split, double px, double py, double pz, Acc& acc)
    {
        const LinePieceF* pieces = reinterpret_cast<const LinePieceF*>(st);
        const LineSegF* recs = reinterpret_cast<const LineSegF*>(st + (size_t)npieces * sizeof(LinePieceF));
        const float cJK2 = (float)(a.cJ / a.cK * 0.69314718055994530942);
        for (int p = 0; p < npieces; ++p) {
            const LinePieceF& pc = pieces[p];
            const double qx = px - pc.cx, qy = py - pc.cy, qz = pz - pc.cz;
            for (int img = split; img < a.nimg; img += S) {
                double sx, sy, sz;
                if (!image_shift(img, a.images, a.image_min, a.Lx, a.Ly, a.Lz, sx, sy, sz)) continue;
                const float Px = (float)(qx - sx), Py = (float)(qy - sy), Pz = (float)(qz - sz);
                if (near_cut(pc, Px, Py, Pz, a.near_h, a.near_r)) { acc.near = true; continue; }
                float fx = 0.0f, fy = 0.0f, fz = 0.0f;
                line_piece_fp32(pc, recs + pc.rec, Px, Py, Pz, cJK2, fx, fy, fz);
                acc.add(fx, fy, fz);
            }
        }
    }
};

// Second pass of the FP32 line form: the near-cut pairs, in FP64.
struct LineNearFp64 {
    using Acc = AccF64;
    static constexpr int kMinBlocks = 2;
    static constexpr bool kAppendsNear = false;
    template <int S>
    static __device__ __forceinline__ void chunk(const FieldArgs& a, const unsigned char* st, int npieces,
                                                 int split, double px, double py, double pz, Acc& acc)
    {
        const LinePieceF* pieces = reinterpret_cast<const LinePieceF*>(st);
        const double cJK = a.cJ / a.cK;
        bool plane = false;
        for (int p = 0; p < npieces; ++p) {
            const LinePieceF& pc = pieces[p];
            const double qx = px - pc.cx, qy = py - pc.cy, qz = pz - pc.cz;
            for (int img = split; img < a.nimg; img += S) {
                double sx, sy, sz;
                if (!image_shift(img, a.images, a.image_min, a.Lx, a.Ly, a.Lz, sx, sy, sz)) continue;
                const float Px = (float)(qx - sx), Py = (float)(qy - sy), Pz = (float)(qz - sz);
                if (!near_cut(pc, Px, Py, Pz, a.near_h, a.near_r)) continue;
                const LinePiece& p64 = a.pieces64[pc.piece64];
                line_piece_fp64(p64, a.segs64 + p64.rec, px - sx, py - sy, pz - sz, cJK,
                                acc.x, acc.y, acc.z, plane);
            }
        }
        if (plane) {                        // an atom in a loop's plane band: the reference's solid angle
            for (int p = 0; p < npieces; ++p) {
                const LinePieceF& pc = pieces[p];
                const double qx = px - pc.cx, qy = py - pc.cy, qz = pz - pc.cz;
                for (int img = split; img < a.nimg; img += S) {
                    double sx, sy, sz;
                    if (!image_shift(img, a.images, a.image_min, a.Lx, a.Ly, a.Lz, sx, sy, sz)) continue;
                    const float Px = (float)(qx - sx), Py = (float)(qy - sy), Pz = (float)(qz - sz);
                    if (!near_cut(pc, Px, Py, Pz, a.near_h, a.near_r)) continue;
                    line_piece_plane(a.pieces64[pc.piece64], a.raw, px - sx, py - sy, pz - sz,
                                     acc.x, acc.y, acc.z);
                }
            }
        }
    }
};

struct LooponFp32 {
    using Acc = AccF32K;
    static constexpr int kMinBlocks = 2;
    static constexpr bool kAppendsNear = false;
    template <int S>
    static __device__ __forceinline__ void chunk(const FieldArgs& a, const unsigned char* st, int npieces,
                                                 int split, double px, double py, double pz, Acc& acc)
    {
        const LooponPieceF* pieces = reinterpret_cast<const LooponPieceF*>(st);
        const LooponRecF* recs = reinterpret_cast<const LooponRecF*>(st + (size_t)npieces * sizeof(LooponPieceF));
        const float c2 = (float)a.c2;
        for (int p = 0; p < npieces; ++p) {
            const LooponPieceF& pc = pieces[p];
            const double qx = px - pc.cx, qy = py - pc.cy, qz = pz - pc.cz;
            for (int img = split; img < a.nimg; img += S) {
                double sx, sy, sz;
                if (!image_shift(img, a.images, a.image_min, a.Lx, a.Ly, a.Lz, sx, sy, sz)) continue;
                float fx = 0.0f, fy = 0.0f, fz = 0.0f;
                loopon_piece_fp32(pc, recs + pc.rec, (float)(qx - sx), (float)(qy - sy), (float)(qz - sz),
                                  c2, fx, fy, fz);
                acc.add(fx, fy, fz);
            }
        }
    }
};

} // namespace disco
