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

// Largest t = L/(RA+RB) for which the 8-term series of 2 atanh(t) is exact to
// the double rounding: its remainder relative to the sum is below t^16/17.
constexpr double kSeriesTau = 0.11;

// J0 = ln((S+L)/(S-L)) = 2 atanh(t), t = L/S:  2 t (1 + t^2/3 + ... + t^14/15).
__device__ __forceinline__ double j0_series(double t)
{
    const double t2 = t * t;
    double p = 1.0 / 15.0;
    p = fma(p, t2, 1.0 / 13.0);
    p = fma(p, t2, 1.0 / 11.0);
    p = fma(p, t2, 1.0 / 9.0);
    p = fma(p, t2, 1.0 / 7.0);
    p = fma(p, t2, 1.0 / 5.0);
    p = fma(p, t2, 1.0 / 3.0);
    p = fma(p, t2, 1.0);
    return 2.0 * t * p;
}

// The segment loop of one line piece.  FAR: every segment of the piece is far
// enough from P (for every lane of the warp) that J0 comes from the series.
template <bool FAR>
__device__ __forceinline__ void line_segments(const LineSeg* seg, int nseg, double Px, double Py, double Pz,
                                              double ex, double ey, double ez, double ax, double ay, double az,
                                              double cJ, double cK, double& zr, double& zi,
                                              double& lx, double& ly, double& lz)
{
    const double la2 = ax * ax + ay * ay + az * az;
    double ila = rsqrt(la2);
    double la = la2 * ila;
    double hax = ax * ila, hay = ay * ila, haz = az * ila;
    double ca = ex * hax + ey * hay + ez * haz;                 // e . a-hat
    double qx = ey * haz - ez * hay, qy = ez * hax - ex * haz, qz = ex * hay - ey * hax;   // e x a-hat
    for (int k = 0; k < nseg; ++k) {
        const LineSeg s = seg[k];
        const double bx = s.vx - Px, by = s.vy - Py, bz = s.vz - Pz;
        const double lb2 = bx * bx + by * by + bz * bz;
        const double ilb = rsqrt(lb2);
        const double lb = lb2 * ilb;
        const double hbx = bx * ilb, hby = by * ilb, hbz = bz * ilb;
        const double cb = ex * hbx + ey * hby + ez * hbz;

        // solid angle of triangle (apex, A, B): tan(Omega/2) = num / den on unit
        // vectors (Code/barnett.hpp:69-72 divided by l1 la lb > 0)
        const double den = 1.0 + ca + cb + (hax * hbx + hay * hby + haz * hbz);
        const double num = qx * hbx + qy * hby + qz * hbz;
        const double nzr = zr * den - zi * num;
        zi = zr * num + zi * den;
        zr = nzr;

        // segment A -> B (Code/barnett.hpp:75-100)
        const double sA = ax * s.tx + ay * s.ty + az * s.tz;
        const double sB = sA + s.len;
        const double dx = ax - sA * s.tx, dy = ay - sA * s.ty, dz = az - sA * s.tz;
        const double d2 = dx * dx + dy * dy + dz * dz;
        const double dw = dx * s.wx + dy * s.wy + dz * s.wz;
        const double sum = la + lb;
        double J0;
        if (FAR) J0 = j0_series(s.len * rcp_nr(sum));
        else     J0 = log((sum + s.len) * rcp_nr(sum - s.len));
        const double g = sB * ilb - sA * ila;                   // d^2 K0
        const double q = d2 > 0.0 ? dw * rcp_nr(d2) : 0.0;
        const double K1 = ila - ilb;
        const double al = cK * q * g, be = cK * dw * K1, ga = cJ * J0;
        lx += ga * s.wx - al * dx - be * s.tx;
        ly += ga * s.wy - al * dy - be * s.ty;
        lz += ga * s.wz - al * dz - be * s.tz;

        ax = bx; ay = by; az = bz;
        la = lb; ila = ilb;
        hax = hbx; hay = hby; haz = hbz;
        ca = cb;
        qx = ey * hbz - ez * hby; qy = ez * hbx - ex * hbz; qz = ex * hby - ey * hbx;
        if ((k & 63) == 63) {                                   // keep |z| near 1
            const double sc = rcp_nr(fabs(zr) + fabs(zi));
            zr *= sc; zi *= sc;
        }
    }
}

// Field at P (an atom moved by minus an image shift) of one line piece.
// Follows Code/barnett.hpp:55-106 term by term (see field.cu's header for the
// reformulations); adds b Omega/(4 pi) + the line terms to (ux, uy, uz).
// For every segment, RA + RB >= 2 (l1 - rho) with l1 = |apex - P| and rho the
// piece's largest vertex radius, so t = L/(RA+RB) <= lmax / (2 (l1 - rho)).
__device__ __forceinline__ void line_piece_fp64(const LinePiece& pc, const LineSeg* seg,
                                                double Px, double Py, double Pz, double cJ, double cK,
                                                double& ux, double& uy, double& uz)
{
    // unit vector from P to the fan apex
    const double r1x = pc.cx - Px, r1y = pc.cy - Py, r1z = pc.cz - Pz;
    const double l1sq = r1x * r1x + r1y * r1y + r1z * r1z;
    const double il1 = rsqrt(l1sq);
    const double ex = r1x * il1, ey = r1y * il1, ez = r1z * il1;
    const double gap = l1sq * il1 - pc.rho;
    const bool far_lane = gap > 0.0 && pc.lmax <= 2.0 * kSeriesTau * gap;
    const bool far = __all_sync(__activemask(), far_lane);

    double zr = 1.0, zi = 0.0, lx = 0.0, ly = 0.0, lz = 0.0;
    const double ax = pc.ax - Px, ay = pc.ay - Py, az = pc.az - Pz;
    if (far) line_segments<true>(seg, pc.nseg, Px, Py, Pz, ex, ey, ez, ax, ay, az, cJ, cK, zr, zi, lx, ly, lz);
    else     line_segments<false>(seg, pc.nseg, Px, Py, Pz, ex, ey, ez, ax, ay, az, cJ, cK, zr, zi, lx, ly, lz);
    const double f = atan2(zi, zr) * (1.0 / 6.283185307179586476925286766559);   // Omega / (4 pi)
    ux += pc.bx * f + lx;
    uy += pc.by * f + ly;
    uz += pc.bz * f + lz;
}

// Field at P (atom - reference point - image shift) of one loopon piece:
// Code/kroupa.hpp:52-73 with 1/rho from one rsqrt and m.rho, n.rho from
// per-loopon projections.
__device__ __forceinline__ void loopon_piece_fp64(const LooponPiece& pc, const LooponRec* __restrict__ rec,
                                                  double Px, double Py, double Pz, double c2,
                                                  double& ux, double& uy, double& uz)
{
    const double mP = pc.mx * Px + pc.my * Py + pc.mz * Pz;
    const double nP = pc.nx * Px + pc.ny * Py + pc.nz * Pz;
    double dx = 0.0, dy = 0.0, dz = 0.0;
    const int n = pc.n;
    for (int k = 0; k < n; ++k) {
        const LooponRec l = rec[k];
        const double rx = Px - l.x, ry = Py - l.y, rz = Pz - l.z;
        const double r2 = rx * rx + ry * ry + rz * rz;
        const bool keep = r2 >= 1e-20;                           // rho >= 1e-10 (kroupa.hpp:55)
        const double ir = rsqrt(keep ? r2 : 1.0);
        const double ir2 = ir * ir;
        const double mr = mP - l.ml, nr = nP - l.nl;
        const double k2 = c2 * ir;
        const double tail = 3.0 * mr * nr * (ir2 * ir);
        const double fac = keep ? ir2 : 0.0;
        const double ex = pc.nx * mr + pc.mx * nr - rx * pc.b_n;
        const double ey = pc.ny * mr + pc.my * nr - ry * pc.b_n;
        const double ez = pc.nz * mr + pc.mz * nr - rz * pc.b_n;
        dx += fac * (pc.fbx * (k2 * ex + tail * rx));
        dy += fac * (pc.fby * (k2 * ey + tail * ry));
        dz += fac * (pc.fbz * (k2 * ez + tail * rz));
    }
    ux += dx; uy += dy; uz += dz;
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
    template <int S>
    static __device__ __forceinline__ void chunk(const FieldArgs& a, const unsigned char* st, int npieces,
                                                 int split, double px, double py, double pz, Acc& acc)
    {
        const LinePiece* pieces = reinterpret_cast<const LinePiece*>(st);
        const LineSeg* recs = reinterpret_cast<const LineSeg*>(st + (size_t)npieces * sizeof(LinePiece));
        for (int p = 0; p < npieces; ++p) {
            const LinePiece& pc = pieces[p];
            for (int img = split; img < a.nimg; img += S) {
                double sx, sy, sz;
                if (!image_shift(img, a.images, a.image_min, a.Lx, a.Ly, a.Lz, sx, sy, sz)) continue;
                line_piece_fp64(pc, recs + pc.rec, px - sx, py - sy, pz - sz, a.cJ, a.cK, acc.x, acc.y, acc.z);
            }
        }
    }
};

struct LooponFp64 {
    using Acc = AccF64;
    static constexpr int kMinBlocks = 2;
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
    const int64_t ntiles = (a.n + kAtomsPerCta - 1) / kAtomsPerCta;
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
            atom = tile * kAtomsPerCta + tid / S;
            valid = atom < a.n;
            const int64_t ia = valid ? atom : a.n - 1;
            px = a.x[ia]; py = a.y[ia]; pz = a.z[ia];
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
// not depend on the atom precomputed.  rec is left to the chunk packer.
inline void make_line_piece(const disco_loop& lp, int k0, int k1e, double bx, double by, double bz,
                            LinePiece& p, std::vector<LineSeg>& recs)
{
    const int nv = lp.n_vertices;
    std::memset(&p, 0, sizeof(p));
    const int a = (k0 + nv - 1) % nv;
    p.ax = lp.vx[a]; p.ay = lp.vy[a]; p.az = lp.vz[a];
    p.cx = lp.cx; p.cy = lp.cy; p.cz = lp.cz;
    p.bx = bx; p.by = by; p.bz = bz;
    p.nseg = k1e - k0;
    auto radius = [&](int k) {
        const double dx = lp.vx[k] - lp.cx, dy = lp.vy[k] - lp.cy, dz = lp.vz[k] - lp.cz;
        return std::sqrt(dx * dx + dy * dy + dz * dz);
    };
    p.rho = radius(a);
    recs.clear();
    for (int k = k0; k < k1e; ++k) {
        const int km = (k + nv - 1) % nv;
        LineSeg s;
        std::memset(&s, 0, sizeof(s));
        s.vx = lp.vx[k]; s.vy = lp.vy[k]; s.vz = lp.vz[k];
        const double tx = lp.vx[k] - lp.vx[km], ty = lp.vy[k] - lp.vy[km], tz = lp.vz[k] - lp.vz[km];
        const double L = std::sqrt(tx * tx + ty * ty + tz * tz);
        if (L > 0.0) {
            s.len = L;
            s.tx = tx / L; s.ty = ty / L; s.tz = tz / L;
            s.wx = by * s.tz - bz * s.ty;
            s.wy = bz * s.tx - bx * s.tz;
            s.wz = bx * s.ty - by * s.tx;
        }
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
