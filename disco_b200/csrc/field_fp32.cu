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
#include "field_fp32.cuh"

namespace disco {

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
                     std::string& err, uint32_t stage_cap)
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
        std::vector<double> raw;
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
                std::vector<LineSeg> segs;
                make_line_piece(lp, k0, k1e, bx, by, bz, k1, q, segs, raw);
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
                for (const LineSeg& sg : segs) {
                    s64.push_back(sg);
                    LineSegF f;
                    std::memset(&f, 0, sizeof(f));
                    f.vx = (float)sg.vx; f.vy = (float)sg.vy; f.vz = (float)sg.vz;     // apex-relative
                    f.len = (float)sg.len;
                    f.tx = (float)sg.tx; f.ty = (float)sg.ty; f.tz = (float)sg.tz;
                    f.wx = (float)sg.wx; f.wy = (float)sg.wy; f.wz = (float)sg.wz;      // cK w
                    f.nx = (float)sg.nx; f.ny = (float)sg.ny; f.nz = (float)sg.nz;
                    f.hl2 = (float)sg.hl2;
                    recs.push_back(f);
                }
                p64.push_back(q);
                L.pieces.push_back(p);
                L.recs.push_back(std::move(recs));
            }
        }
        pack_chunks(L, T, stage_cap);
        if (!T.chunks.empty()) {
            append_aligned(T.bytes, p64.data(), p64.size() * sizeof(LinePiece));
            T.aux_pieces = T.bytes.size() - p64.size() * sizeof(LinePiece);
            append_aligned(T.bytes, s64.data(), s64.size() * sizeof(LineSeg));
            T.aux_segs = T.bytes.size() - s64.size() * sizeof(LineSeg);
            append_raw(T, raw);
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
        pack_chunks(L, T, stage_cap);
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
    if (!a.near_list) {
        a.near_mode = 0;
        const int st = launch_kind_f<LineFp32>(a, S, sm_count, smem, stream, err);
        if (st) return st;
        return launch_kind_f<LineNearFp64>(a, S, sm_count, smem, stream, err);
    }
    // the FP32 pass lists the atoms with near-cut pairs; the FP64 pass visits
    // only those (every atom if the list overflowed), with its images split
    // over 8 lanes since they are few
    const cudaError_t e = cudaMemsetAsync(a.near_count, 0, sizeof(unsigned int), stream);
    if (e != cudaSuccess) { err = cudaGetErrorString(e); return DISCO_ECUDA; }
    a.near_mode = 1;
    const int st = launch_kind_f<LineFp32>(a, S, sm_count, smem, stream, err);
    if (st) return st;
    a.near_mode = 2;
    int Sn = 1;
    while (Sn < 8 && 2 * Sn <= a.nimg) Sn *= 2;
    return launch_kind_f<LineNearFp64>(a, split_hint > 0 ? S : Sn, sm_count, smem, stream, err);
}

} // namespace disco
