// Displacement-sum kernels (sm_100a) and their table builder / launcher.
//
// What is summed is the reference's: for every atom, every loop, every periodic
// image and every segment (Barnett line integral, Code/barnett.hpp:44-107) or
// loopon (Kroupa pair term, Code/kroupa.hpp:52-73); Code/backend_cpu.cpp:28-99
// is the loop nest.  How it is summed is B200-specific:
//   - one launch covers all loops and all images (the reference launches and
//     synchronises once per loop, Code/backend_cuda.cu:646-704);
//   - persistent CTAs walk atom tiles; the loop table is cut into chunks that a
//     single thread stages into shared memory with bulk async copies completed
//     on an mbarrier (double-buffered when the table does not fit at once), and
//     every warp reads each record as a shared-memory broadcast;
//   - image shifts are enumerated in registers; when there are too few atoms
//     to fill the GPU, S consecutive lanes share an atom and split its images,
//     and a fixed-order warp butterfly sums their parts;
//   - everything that does not depend on the atom (unit tangent, length,
//     w = b x t per segment; m.l, n.l per loopon; Kroupa prefactors) is
//     computed once on the host;
//   - line method: the solid angle of the fan is the argument of the running
//     complex product of the Van Oosterom-Strackee terms (one atan2 per atom,
//     piece and image instead of one per segment); the line integrals use one
//     rsqrt per vertex, J0 = ln((RA+RB+L)/(RA+RB-L)) and K0 d^2 = sB/RB - sA/RA,
//     all cancellation-free in the product that enters u.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "common.cuh"
#include "field.cuh"

namespace disco {

constexpr int kThreads = 256;
constexpr int kMaxLinePiece = 256;         // segments per piece
constexpr int kMaxLooponPiece = 960;       // loopons per piece (fits a 48 KB stage)
constexpr uint32_t kResidentMax = 110u * 1024u;
constexpr uint32_t kStageMax = 48u * 1024u;
constexpr uint32_t kSmemHeader = 128;      // mbarriers at the start of shared memory

__device__ __forceinline__ void image_shift(int img, int images, double Lx, double Ly, double Lz,
                                            double& sx, double& sy, double& sz)
{
    const int W = 2 * images + 1;
    const int ii = img / (W * W) - images;
    const int r = img % (W * W);
    const int jj = r / W - images;
    const int kk = r % W - images;
    sx = Lx * ii;
    sy = Ly * jj;
    sz = Lz * kk;
}

// Field at P (an atom moved by minus an image shift) of one line piece.
// Follows Code/barnett.hpp:55-106 term by term (see the file header for the
// reformulations); adds b Omega/(4 pi) + the line terms to (ux, uy, uz).
__device__ __forceinline__ void line_piece_fp64(const LinePiece& pc, const LineSeg* seg,
                                                double Px, double Py, double Pz, double cJ, double cK,
                                                double& ux, double& uy, double& uz)
{
    // unit vector from P to the fan apex
    const double r1x = pc.cx - Px, r1y = pc.cy - Py, r1z = pc.cz - Pz;
    const double il1 = rsqrt(r1x * r1x + r1y * r1y + r1z * r1z);
    const double ex = r1x * il1, ey = r1y * il1, ez = r1z * il1;

    // vertex A (start of the current segment) relative to P
    double ax = pc.ax - Px, ay = pc.ay - Py, az = pc.az - Pz;
    double ila = rsqrt(ax * ax + ay * ay + az * az);
    double la = (ax * ax + ay * ay + az * az) * ila;
    double hax = ax * ila, hay = ay * ila, haz = az * ila;
    double ca = ex * hax + ey * hay + ez * haz;                 // e . a-hat
    double qx = ey * haz - ez * hay, qy = ez * hax - ex * haz, qz = ex * hay - ey * hax;   // e x a-hat

    double zr = 1.0, zi = 0.0;                                   // running product
    double lx = 0.0, ly = 0.0, lz = 0.0;
    const int nseg = pc.nseg;
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
        const double J0 = log((sum + s.len) / (sum - s.len));
        const double g = sB * ilb - sA * ila;                   // d^2 K0
        const double q = d2 > 0.0 ? dw / d2 : 0.0;
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
            const double sc = 1.0 / (fabs(zr) + fabs(zi));
            zr *= sc; zi *= sc;
        }
    }
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

// Persistent kernel: CTA b takes atom tiles b, b + grid, ...; for each tile it
// walks the chunks of the table (staged in shared memory) and, per piece, the
// images of its lane's share.
template <int KIND, int S>
__global__ void __launch_bounds__(kThreads, 2) field_fp64_kernel(const FieldArgs a)
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
    double px = 0.0, py = 0.0, pz = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
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
            ux = uy = uz = 0.0;
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
        const int npieces = a.chunks[ch].npieces;
        if (KIND == kLineKind) {
            const LinePiece* pieces = reinterpret_cast<const LinePiece*>(st);
            const LineSeg* recs = reinterpret_cast<const LineSeg*>(st + (size_t)npieces * sizeof(LinePiece));
            for (int p = 0; p < npieces; ++p) {
                const LinePiece& pc = pieces[p];
                for (int img = split; img < a.nimg; img += S) {
                    double sx, sy, sz;
                    image_shift(img, a.images, a.Lx, a.Ly, a.Lz, sx, sy, sz);
                    line_piece_fp64(pc, recs + pc.rec, px - sx, py - sy, pz - sz, a.cJ, a.cK, ux, uy, uz);
                }
            }
        } else {
            const LooponPiece* pieces = reinterpret_cast<const LooponPiece*>(st);
            const LooponRec* recs = reinterpret_cast<const LooponRec*>(st + (size_t)npieces * sizeof(LooponPiece));
            for (int p = 0; p < npieces; ++p) {
                const LooponPiece& pc = pieces[p];
                const double qx = px - pc.cx, qy = py - pc.cy, qz = pz - pc.cz;
                for (int img = split; img < a.nimg; img += S) {
                    double sx, sy, sz;
                    image_shift(img, a.images, a.Lx, a.Ly, a.Lz, sx, sy, sz);
                    loopon_piece_fp64(pc, recs + pc.rec, qx - sx, qy - sy, qz - sz, a.c2, ux, uy, uz);
                }
            }
        }
        if (resident || ch == nch - 1) {
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

namespace {

template <class Piece, class Rec>
struct PieceList {
    std::vector<Piece> pieces;
    std::vector<std::vector<Rec>> recs;
};

template <class Piece, class Rec>
void pack_chunks(PieceList<Piece, Rec>& L, HostTable& T)
{
    size_t total = 0;
    for (size_t i = 0; i < L.pieces.size(); ++i) total += sizeof(Piece) + L.recs[i].size() * sizeof(Rec);
    const uint32_t cap = total <= kResidentMax ? kResidentMax : kStageMax;
    T.resident = total <= kResidentMax;
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
    if (T.chunks.size() <= 1) T.resident = true;
    T.stage_bytes = max_bytes;
}

} // namespace

int build_table(const disco_loop* loops, int nloops, int kind, int precision, double nu,
                HostTable& T, std::string& err)
{
    T = HostTable();
    T.kind = kind;
    T.fp32 = precision == DISCO_FP32C;
    T.loop_evals.assign((size_t)nloops, 0.0);
    if (T.fp32) { err = "FP32 tables are built by build_table_fp32"; return DISCO_EINVAL; }
    const double k1 = 1.0 / (8.0 * M_PI * (1.0 - nu));          // Code/kroupa.hpp:38-41
    if (kind == kLineKind) {
        PieceList<LinePiece, LineSeg> L;
        for (int l = 0; l < nloops; ++l) {
            const disco_loop& lp = loops[l];
            if (!lp.line) continue;
            const int nv = lp.n_vertices;
            if (nv <= 0) continue;
            if (!lp.vx || !lp.vy || !lp.vz) { err = "line loop without vertices"; return DISCO_EINVAL; }
            // b = (|b|_x m_x, |b|_y m_y, |b|_z m_z): Code/backend_cpu.cpp:44-45
            const double bx = lp.phys.bx * lp.phys.mx, by = lp.phys.by * lp.phys.my,
                         bz = lp.phys.bz * lp.phys.mz;
            T.loop_evals[l] = nv;
            T.n_segments += nv;
            for (int k0 = 0; k0 < nv; k0 += kMaxLinePiece) {
                const int k1e = std::min(nv, k0 + kMaxLinePiece);
                LinePiece p;
                std::memset(&p, 0, sizeof(p));
                const int a = (k0 + nv - 1) % nv;
                p.ax = lp.vx[a]; p.ay = lp.vy[a]; p.az = lp.vz[a];
                p.cx = lp.cx; p.cy = lp.cy; p.cz = lp.cz;
                p.bx = bx; p.by = by; p.bz = bz;
                p.nseg = k1e - k0;
                std::vector<LineSeg> recs;
                for (int k = k0; k < k1e; ++k) {
                    const int km = (k + nv - 1) % nv;
                    LineSeg s;
                    std::memset(&s, 0, sizeof(s));
                    s.vx = lp.vx[k]; s.vy = lp.vy[k]; s.vz = lp.vz[k];
                    const double tx = lp.vx[k] - lp.vx[km], ty = lp.vy[k] - lp.vy[km],
                                 tz = lp.vz[k] - lp.vz[km];
                    const double L = std::sqrt(tx * tx + ty * ty + tz * tz);
                    if (L > 0.0) {
                        s.len = L;
                        s.tx = tx / L; s.ty = ty / L; s.tz = tz / L;
                        s.wx = by * s.tz - bz * s.ty;
                        s.wy = bz * s.tx - bx * s.tz;
                        s.wz = bx * s.ty - by * s.tx;
                    }
                    recs.push_back(s);
                }
                L.pieces.push_back(p);
                L.recs.push_back(std::move(recs));
            }
        }
        pack_chunks(L, T);
    } else {
        PieceList<LooponPiece, LooponRec> L;
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
                LooponPiece p;
                std::memset(&p, 0, sizeof(p));
                p.cx = cx; p.cy = cy; p.cz = cz;
                p.fbx = -k1 * ph.dS * ph.bx;
                p.fby = -k1 * ph.dS * ph.by;
                p.fbz = -k1 * ph.dS * ph.bz;
                p.mx = ph.mx; p.my = ph.my; p.mz = ph.mz;
                p.nx = ph.nx; p.ny = ph.ny; p.nz = ph.nz;
                p.b_n = ph.mx * ph.nx + ph.my * ph.ny + ph.mz * ph.nz;
                p.n = k1e - k0;
                std::vector<LooponRec> recs;
                for (int k = k0; k < k1e; ++k) {
                    LooponRec r;
                    r.x = lp.x[k] - cx; r.y = lp.y[k] - cy; r.z = lp.z[k] - cz;
                    r.ml = ph.mx * r.x + ph.my * r.y + ph.mz * r.z;
                    r.nl = ph.nx * r.x + ph.ny * r.y + ph.nz * r.z;
                    r.pad = 0.0;
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

// ---- host: launch ------------------------------------------------------------------------

namespace {

template <int KIND, int S>
int launch_one(const FieldArgs& a, int sm_count, size_t smem, cudaStream_t stream, std::string& err)
{
    auto kern = field_fp64_kernel<KIND, S>;
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

template <int KIND>
int launch_kind(const FieldArgs& a, int S, int sm_count, size_t smem, cudaStream_t stream, std::string& err)
{
    switch (S) {
    case 1:  return launch_one<KIND, 1>(a, sm_count, smem, stream, err);
    case 2:  return launch_one<KIND, 2>(a, sm_count, smem, stream, err);
    case 4:  return launch_one<KIND, 4>(a, sm_count, smem, stream, err);
    case 8:  return launch_one<KIND, 8>(a, sm_count, smem, stream, err);
    case 16: return launch_one<KIND, 16>(a, sm_count, smem, stream, err);
    default: return launch_one<KIND, 32>(a, sm_count, smem, stream, err);
    }
}

} // namespace

// Image split S: the power of two (<= 32, <= images) that minimises
// rounds x images-per-lane, with rounds = ceil(tiles / resident CTAs).
int choose_split(int64_t n, int nimg, int resident_ctas)
{
    int best = 1;
    double best_cost = 1e300;
    for (int S = 1; S <= 32; S *= 2) {
        if (S > 1 && S > nimg) break;
        const int64_t ntiles = (n * S + kThreads - 1) / kThreads;
        const double rounds = std::ceil((double)ntiles / resident_ctas);
        const double cost = rounds * std::ceil((double)nimg / S);
        if (cost < best_cost * (1.0 - 1e-9)) { best_cost = cost; best = S; }
    }
    return best;
}

int launch_field(const FieldArgs& a, int kind, bool fp32, int sm_count, int threads_hint,
                 int split_hint, cudaStream_t stream, std::string& err)
{
    (void)threads_hint;
    if (a.n <= 0 || a.nchunks <= 0) return DISCO_OK;
    if (fp32) { err = "FP32 launch goes through launch_field_fp32"; return DISCO_EINVAL; }
    const size_t smem = kSmemHeader + (size_t)a.stage_bytes * (a.resident ? 1 : 2);
    const int S = split_hint > 0 ? split_hint : choose_split(a.n, a.nimg, sm_count * 2);
    return kind == kLineKind ? launch_kind<kLineKind>(a, S, sm_count, smem, stream, err)
                             : launch_kind<kLooponKind>(a, S, sm_count, smem, stream, err);
}

} // namespace disco
