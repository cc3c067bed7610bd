// FP32 compensated form of the displacement sum (DISCO_FP32C).
//
// Same loop nest, staging and image split as the FP64 kernels; what changes:
//   - every table coordinate is stored relative to its loop's centre (FP32),
//     and the atom enters as (atom - centre - image shift) computed in FP64
//     and rounded once to FP32, so the numbers the FP32 arithmetic sees are
//     distances to the loop, not box coordinates;
//   - the per-segment (per-loopon) arithmetic is FP32 with hardware
//     approximations (rsqrt, reciprocal, log2) where their error (a few ulp)
//     is far below the form's 1e-3 A budget;
//   - each (piece, image) contribution is added to a Kahan-compensated FP32
//     sum (over images and loops), converted to FP64 once at the end;
//   - line method: for an atom within near_h of a loop's plane and within
//     rmax + near_r of its centre in the plane, that (piece, image) is skipped
//     by the FP32 kernel and evaluated by a second, FP64 kernel (the solid
//     angle's branch and the cut surface are decided in FP64 there); one
//     shared FP32 test selects the pairs for both.  The reference's own --fp32 kernels
//     (Code/backend_cuda.cu:197-291, 335-373) centre coordinates the same way
//     but sum the images in FP64 and have no near-cut path.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "common.cuh"
#include "field.cuh"
#include "field_device.cuh"

namespace disco {

constexpr float kNearPlane = 3.0f;   // A from the loop plane
constexpr float kNearRim = 3.0f;     // A beyond the largest vertex radius

// Kahan-compensated FP32 sums plus an FP64 part (near-cut evaluations).
struct AccF32K {
    float sx, sy, sz, cx, cy, cz;
    double dx, dy, dz;
    __device__ void clear()
    {
        sx = sy = sz = cx = cy = cz = 0.0f;
        dx = dy = dz = 0.0;
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

// Code/barnett.hpp:44-107 in FP32 on centre-relative coordinates, with the
// same reformulation as line_piece_fp64.
__device__ __forceinline__ void line_piece_fp32(const LinePieceF& pc, const LineSegF* seg, float Px,
                                                float Py, float Pz, float cJ, float cK,
                                                float& ux, float& uy, float& uz)
{
    // apex = centre = origin of these coordinates
    const float il1 = rsqrtf(Px * Px + Py * Py + Pz * Pz);
    const float ex = -Px * il1, ey = -Py * il1, ez = -Pz * il1;
    float ax = pc.ax - Px, ay = pc.ay - Py, az = pc.az - Pz;
    float la2 = ax * ax + ay * ay + az * az;
    float ila = rsqrtf(la2);
    float la = la2 * ila;
    float hax = ax * ila, hay = ay * ila, haz = az * ila;
    float ca = ex * hax + ey * hay + ez * haz;
    float qx = ey * haz - ez * hay, qy = ez * hax - ex * haz, qz = ex * hay - ey * hax;
    float zr = 1.0f, zi = 0.0f, lx = 0.0f, ly = 0.0f, lz = 0.0f;
    const int nseg = pc.nseg;
    for (int k = 0; k < nseg; ++k) {
        const LineSegF s = seg[k];
        const float bx = s.vx - Px, by = s.vy - Py, bz = s.vz - Pz;
        const float lb2 = bx * bx + by * by + bz * bz;
        const float ilb = rsqrtf(lb2);
        const float lb = lb2 * ilb;
        const float hbx = bx * ilb, hby = by * ilb, hbz = bz * ilb;
        const float cb = ex * hbx + ey * hby + ez * hbz;
        const float den = 1.0f + ca + cb + (hax * hbx + hay * hby + haz * hbz);
        const float num = qx * hbx + qy * hby + qz * hbz;
        const float nzr = zr * den - zi * num;
        zi = zr * num + zi * den;
        zr = nzr;
        const float sA = ax * s.tx + ay * s.ty + az * s.tz;
        const float sB = sA + s.len;
        const float dx = ax - sA * s.tx, dy = ay - sA * s.ty, dz = az - sA * s.tz;
        const float d2 = dx * dx + dy * dy + dz * dz;
        const float dw = dx * s.wx + dy * s.wy + dz * s.wz;
        const float sum = la + lb;
        const float J0 = __logf(__fdividef(sum + s.len, sum - s.len));
        const float g = sB * ilb - sA * ila;
        const float q = d2 > 0.0f ? __fdividef(dw, d2) : 0.0f;
        const float K1 = ila - ilb;
        const float al = cK * q * g, be = cK * dw * K1, ga = cJ * J0;
        lx += ga * s.wx - al * dx - be * s.tx;
        ly += ga * s.wy - al * dy - be * s.ty;
        lz += ga * s.wz - al * dz - be * s.tz;
        ax = bx; ay = by; az = bz;
        la = lb; ila = ilb;
        hax = hbx; hay = hby; haz = hbz;
        ca = cb;
        qx = ey * hbz - ez * hby; qy = ez * hbx - ex * hbz; qz = ex * hby - ey * hbx;
        if ((k & 15) == 15) {
            const float sc = __frcp_rn(fabsf(zr) + fabsf(zi));
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
    const float mP = pc.mx * Px + pc.my * Py + pc.mz * Pz;
    const float nP = pc.nx * Px + pc.ny * Py + pc.nz * Pz;
    float dx = 0.0f, dy = 0.0f, dz = 0.0f;
    const int n = pc.n;
    for (int k = 0; k < n; ++k) {
        const LooponRecF l = rec[k];
        const float rx = Px - l.x, ry = Py - l.y, rz = Pz - l.z;
        const float r2 = rx * rx + ry * ry + rz * rz;
        const bool keep = r2 >= 1e-20f;
        const float ir = rsqrtf(keep ? r2 : 1.0f);
        const float ir2 = ir * ir;
        const float mr = mP - l.ml, nr = nP - l.nl;
        const float k2 = c2 * ir;
        const float tail = 3.0f * mr * nr * (ir2 * ir);
        const float fac = keep ? ir2 : 0.0f;
        const float ex = pc.nx * mr + pc.mx * nr - rx * pc.b_n;
        const float ey = pc.ny * mr + pc.my * nr - ry * pc.b_n;
        const float ez = pc.nz * mr + pc.mz * nr - rz * pc.b_n;
        dx += fac * (pc.fbx * (k2 * ex + tail * rx));
        dy += fac * (pc.fby * (k2 * ey + tail * ry));
        dz += fac * (pc.fbz * (k2 * ez + tail * rz));
    }
    ux += dx; uy += dy; uz += dz;
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
    template <int S>
    static __device__ __forceinline__ void chunk(const FieldArgs& a, const unsigned char* st, int npieces,
                                                 int split, double px, double py, double pz, Acc& acc)
    {
        const LinePieceF* pieces = reinterpret_cast<const LinePieceF*>(st);
        const LineSegF* recs = reinterpret_cast<const LineSegF*>(st + (size_t)npieces * sizeof(LinePieceF));
        const float cJ = (float)a.cJ, cK = (float)a.cK;
        for (int p = 0; p < npieces; ++p) {
            const LinePieceF& pc = pieces[p];
            const double qx = px - pc.cx, qy = py - pc.cy, qz = pz - pc.cz;
            for (int img = split; img < a.nimg; img += S) {
                double sx, sy, sz;
                image_shift(img, a.images, a.Lx, a.Ly, a.Lz, sx, sy, sz);
                const float Px = (float)(qx - sx), Py = (float)(qy - sy), Pz = (float)(qz - sz);
                if (near_cut(pc, Px, Py, Pz, a.near_h, a.near_r)) continue;
                float fx = 0.0f, fy = 0.0f, fz = 0.0f;
                line_piece_fp32(pc, recs + pc.rec, Px, Py, Pz, cJ, cK, fx, fy, fz);
                acc.add(fx, fy, fz);
            }
        }
    }
};

// Second pass of the FP32 line form: the near-cut pairs, in FP64.
struct LineNearFp64 {
    using Acc = AccF64;
    static constexpr int kMinBlocks = 2;
    template <int S>
    static __device__ __forceinline__ void chunk(const FieldArgs& a, const unsigned char* st, int npieces,
                                                 int split, double px, double py, double pz, Acc& acc)
    {
        const LinePieceF* pieces = reinterpret_cast<const LinePieceF*>(st);
        for (int p = 0; p < npieces; ++p) {
            const LinePieceF& pc = pieces[p];
            const double qx = px - pc.cx, qy = py - pc.cy, qz = pz - pc.cz;
            for (int img = split; img < a.nimg; img += S) {
                double sx, sy, sz;
                image_shift(img, a.images, a.Lx, a.Ly, a.Lz, sx, sy, sz);
                const float Px = (float)(qx - sx), Py = (float)(qy - sy), Pz = (float)(qz - sz);
                if (!near_cut(pc, Px, Py, Pz, a.near_h, a.near_r)) continue;
                const LinePiece& p64 = a.pieces64[pc.piece64];
                line_piece_fp64(p64, a.segs64 + p64.rec, px - sx, py - sy, pz - sz, a.cJ, a.cK,
                                acc.x, acc.y, acc.z);
            }
        }
    }
};

struct LooponFp32 {
    using Acc = AccF32K;
    static constexpr int kMinBlocks = 2;
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
                image_shift(img, a.images, a.Lx, a.Ly, a.Lz, sx, sy, sz);
                float fx = 0.0f, fy = 0.0f, fz = 0.0f;
                loopon_piece_fp32(pc, recs + pc.rec, (float)(qx - sx), (float)(qy - sy), (float)(qz - sz),
                                  c2, fx, fy, fz);
                acc.add(fx, fy, fz);
            }
        }
    }
};

// ---- host -------------------------------------------------------------------------------

namespace {

void append_aligned(std::vector<unsigned char>& b, const void* src, size_t n)
{
    while (b.size() % 16) b.push_back(0);
    const unsigned char* s = static_cast<const unsigned char*>(src);
    b.insert(b.end(), s, s + n);
}

} // namespace

int build_table_fp32(const disco_loop* loops, int nloops, int kind, double nu, HostTable& T,
                     std::string& err)
{
    T = HostTable();
    T.kind = kind;
    T.fp32 = true;
    T.loop_evals.assign((size_t)nloops, 0.0);
    const double k1 = 1.0 / (8.0 * M_PI * (1.0 - nu));
    if (kind == kLineKind) {
        PieceList<LinePieceF, LineSegF> L;
        std::vector<LinePiece> p64;
        std::vector<LineSeg> s64;
        for (int l = 0; l < nloops; ++l) {
            const disco_loop& lp = loops[l];
            if (!lp.line) continue;
            const int nv = lp.n_vertices;
            if (nv <= 0) continue;
            if (!lp.vx || !lp.vy || !lp.vz) { err = "line loop without vertices"; return DISCO_EINVAL; }
            const double bx = lp.phys.bx * lp.phys.mx, by = lp.phys.by * lp.phys.my,
                         bz = lp.phys.bz * lp.phys.mz;
            const double c[3] = { lp.cx, lp.cy, lp.cz };
            double rmax = 0.0;
            for (int k = 0; k < nv; ++k) {
                const double dx = lp.vx[k] - c[0], dy = lp.vy[k] - c[1], dz = lp.vz[k] - c[2];
                rmax = std::max(rmax, std::sqrt(dx * dx + dy * dy + dz * dz));
            }
            T.loop_evals[l] = nv;
            T.n_segments += nv;
            for (int k0 = 0; k0 < nv; k0 += kMaxLinePiece) {
                const int k1e = std::min(nv, k0 + kMaxLinePiece);
                const int a = (k0 + nv - 1) % nv;
                LinePiece q;
                std::memset(&q, 0, sizeof(q));
                q.ax = lp.vx[a]; q.ay = lp.vy[a]; q.az = lp.vz[a];
                q.cx = c[0]; q.cy = c[1]; q.cz = c[2];
                q.bx = bx; q.by = by; q.bz = bz;
                q.nseg = k1e - k0;
                q.rec = (int32_t)s64.size();
                LinePieceF p;
                std::memset(&p, 0, sizeof(p));
                p.cx = c[0]; p.cy = c[1]; p.cz = c[2];
                p.ax = (float)(lp.vx[a] - c[0]); p.ay = (float)(lp.vy[a] - c[1]); p.az = (float)(lp.vz[a] - c[2]);
                p.bx = (float)bx; p.by = (float)by; p.bz = (float)bz;
                p.nx = (float)lp.phys.nx; p.ny = (float)lp.phys.ny; p.nz = (float)lp.phys.nz;
                p.rmax = (float)rmax;
                p.nseg = k1e - k0;
                p.piece64 = (int32_t)p64.size();
                std::vector<LineSegF> recs;
                for (int k = k0; k < k1e; ++k) {
                    const int km = (k + nv - 1) % nv;
                    LineSeg s;
                    std::memset(&s, 0, sizeof(s));
                    s.vx = lp.vx[k]; s.vy = lp.vy[k]; s.vz = lp.vz[k];
                    const double tx = lp.vx[k] - lp.vx[km], ty = lp.vy[k] - lp.vy[km], tz = lp.vz[k] - lp.vz[km];
                    const double Ls = std::sqrt(tx * tx + ty * ty + tz * tz);
                    if (Ls > 0.0) {
                        s.len = Ls;
                        s.tx = tx / Ls; s.ty = ty / Ls; s.tz = tz / Ls;
                        s.wx = by * s.tz - bz * s.ty;
                        s.wy = bz * s.tx - bx * s.tz;
                        s.wz = bx * s.ty - by * s.tx;
                    }
                    s64.push_back(s);
                    LineSegF f;
                    std::memset(&f, 0, sizeof(f));
                    f.vx = (float)(s.vx - c[0]); f.vy = (float)(s.vy - c[1]); f.vz = (float)(s.vz - c[2]);
                    f.len = (float)s.len;
                    f.tx = (float)s.tx; f.ty = (float)s.ty; f.tz = (float)s.tz;
                    f.wx = (float)s.wx; f.wy = (float)s.wy; f.wz = (float)s.wz;
                    recs.push_back(f);
                }
                p64.push_back(q);
                L.pieces.push_back(p);
                L.recs.push_back(std::move(recs));
            }
        }
        pack_chunks(L, T);
        if (!T.chunks.empty()) {
            append_aligned(T.bytes, p64.data(), p64.size() * sizeof(LinePiece));
            T.aux_pieces = T.bytes.size() - p64.size() * sizeof(LinePiece);
            append_aligned(T.bytes, s64.data(), s64.size() * sizeof(LineSeg));
            T.aux_segs = T.bytes.size() - s64.size() * sizeof(LineSeg);
        }
    } else {
        PieceList<LooponPieceF, LooponRecF> L;
        for (int l = 0; l < nloops; ++l) {
            const disco_loop& lp = loops[l];
            if (lp.line) continue;
            const int np = lp.n_loopons;
            if (np <= 0) continue;
            if (!lp.x || !lp.y || !lp.z) { err = "loopon loop without loopons"; return DISCO_EINVAL; }
            const disco_loop_phys& ph = lp.phys;
            T.loop_evals[l] = np;
            T.n_loopons += np;
            double cx = 0.0, cy = 0.0, cz = 0.0;
            for (int k = 0; k < np; ++k) { cx += lp.x[k]; cy += lp.y[k]; cz += lp.z[k]; }
            cx /= np; cy /= np; cz /= np;
            for (int k0 = 0; k0 < np; k0 += kMaxLooponPiece) {
                const int k1e = std::min(np, k0 + kMaxLooponPiece);
                LooponPieceF p;
                std::memset(&p, 0, sizeof(p));
                p.cx = cx; p.cy = cy; p.cz = cz;
                p.fbx = (float)(-k1 * ph.dS * ph.bx);
                p.fby = (float)(-k1 * ph.dS * ph.by);
                p.fbz = (float)(-k1 * ph.dS * ph.bz);
                p.mx = (float)ph.mx; p.my = (float)ph.my; p.mz = (float)ph.mz;
                p.nx = (float)ph.nx; p.ny = (float)ph.ny; p.nz = (float)ph.nz;
                p.b_n = (float)(ph.mx * ph.nx + ph.my * ph.ny + ph.mz * ph.nz);
                p.n = k1e - k0;
                std::vector<LooponRecF> recs;
                for (int k = k0; k < k1e; ++k) {
                    const double x = lp.x[k] - cx, y = lp.y[k] - cy, z = lp.z[k] - cz;
                    LooponRecF r;
                    std::memset(&r, 0, sizeof(r));
                    r.x = (float)x; r.y = (float)y; r.z = (float)z;
                    r.ml = (float)(ph.mx * x + ph.my * y + ph.mz * z);
                    r.nl = (float)(ph.nx * x + ph.ny * y + ph.nz * z);
                    recs.push_back(r);
                }
                L.pieces.push_back(p);
                L.recs.push_back(std::move(recs));
            }
        }
        pack_chunks(L, T);
    }
    return DISCO_OK;
}

namespace {

template <class Policy, int S>
int launch_one_f(const FieldArgs& a, int sm_count, size_t smem, cudaStream_t stream, std::string& err)
{
    auto kern = field_kernel<Policy, S>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) { err = cudaGetErrorString(e); return DISCO_ECUDA; }
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
    if (e != cudaSuccess || per_sm < 1) { err = "kernel does not fit on an SM"; return DISCO_ECUDA; }
    const int64_t atoms_per_cta = kThreads / S;
    const int64_t ntiles = (a.n + atoms_per_cta - 1) / atoms_per_cta;
    const int64_t grid = std::min<int64_t>(ntiles, (int64_t)sm_count * per_sm);
    kern<<<(unsigned)grid, kThreads, smem, stream>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) { err = cudaGetErrorString(e); return DISCO_ECUDA; }
    return DISCO_OK;
}

template <class Policy>
int launch_kind_f(const FieldArgs& a, int S, int sm_count, size_t smem, cudaStream_t stream, std::string& err)
{
    switch (S) {
    case 1:  return launch_one_f<Policy, 1>(a, sm_count, smem, stream, err);
    case 2:  return launch_one_f<Policy, 2>(a, sm_count, smem, stream, err);
    case 4:  return launch_one_f<Policy, 4>(a, sm_count, smem, stream, err);
    case 8:  return launch_one_f<Policy, 8>(a, sm_count, smem, stream, err);
    case 16: return launch_one_f<Policy, 16>(a, sm_count, smem, stream, err);
    default: return launch_one_f<Policy, 32>(a, sm_count, smem, stream, err);
    }
}

} // namespace

int choose_split(int64_t n, int nimg, int resident_ctas);

int launch_field_fp32(const FieldArgs& a0, int kind, int sm_count, int split_hint, cudaStream_t stream,
                      std::string& err)
{
    if (a0.n <= 0 || a0.nchunks <= 0) return DISCO_OK;
    FieldArgs a = a0;
    if (a.near_h <= 0.0f) a.near_h = kNearPlane;
    if (a.near_r <= 0.0f) a.near_r = kNearRim;
    const size_t smem = kSmemHeader + (size_t)a.stage_bytes * (a.resident ? 1 : 2);
    const int S = split_hint > 0 ? split_hint : choose_split(a.n, a.nimg, sm_count * 2);
    if (kind != kLineKind) return launch_kind_f<LooponFp32>(a, S, sm_count, smem, stream, err);
    const int st = launch_kind_f<LineFp32>(a, S, sm_count, smem, stream, err);
    if (st) return st;
    return launch_kind_f<LineNearFp64>(a, S, sm_count, smem, stream, err);
}

} // namespace disco
