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
#include "field_device.cuh"

namespace disco {

// Appends the raw vertex triplets to the table bytes (16-byte aligned).
void append_raw(HostTable& T, const std::vector<double>& raw)
{
    while (T.bytes.size() % 16) T.bytes.push_back(0);
    T.aux_raw = T.bytes.size();
    const unsigned char* s = reinterpret_cast<const unsigned char*>(raw.data());
    T.bytes.insert(T.bytes.end(), s, s + raw.size() * sizeof(double));
}

int build_table(const disco_loop* loops, int nloops, int kind, int precision, double nu,
                HostTable& T, std::string& err, uint32_t stage_cap)
{
    T = HostTable();
    T.kind = kind;
    T.fp32 = precision == DISCO_FP32C;
    T.loop_evals.assign((size_t)nloops, 0.0);
    if (T.fp32) { err = "FP32 tables are built by build_table_fp32"; return DISCO_EINVAL; }
    const double k1 = 1.0 / (8.0 * M_PI * (1.0 - nu));          // Code/kroupa.hpp:38-41
    if (kind == kLineKind) {
        PieceList<LinePiece, LineSeg> L;
        std::vector<double> raw;
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
                std::vector<LineSeg> recs;
                make_line_piece(lp, k0, k1e, bx, by, bz, k1, p, recs, raw);
                L.pieces.push_back(p);
                L.recs.push_back(std::move(recs));
            }
        }
        pack_chunks(L, T, stage_cap);
        if (!T.chunks.empty()) append_raw(T, raw);
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
        pack_chunks(L, T, stage_cap);
    }
    return DISCO_OK;
}

// ---- host: launch ------------------------------------------------------------------------

namespace {

template <class Policy, int S>
int launch_one(const FieldArgs& a, int sm_count, size_t smem, cudaStream_t stream, std::string& err)
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
int launch_kind(const FieldArgs& a, int S, int sm_count, size_t smem, cudaStream_t stream, std::string& err)
{
    switch (S) {
    case 1:  return launch_one<Policy, 1>(a, sm_count, smem, stream, err);
    case 2:  return launch_one<Policy, 2>(a, sm_count, smem, stream, err);
    case 4:  return launch_one<Policy, 4>(a, sm_count, smem, stream, err);
    case 8:  return launch_one<Policy, 8>(a, sm_count, smem, stream, err);
    case 16: return launch_one<Policy, 16>(a, sm_count, smem, stream, err);
    default: return launch_one<Policy, 32>(a, sm_count, smem, stream, err);
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
    return kind == kLineKind ? launch_kind<LineFp64>(a, S, sm_count, smem, stream, err)
                             : launch_kind<LooponFp64>(a, S, sm_count, smem, stream, err);
}

} // namespace disco

// ---- self-test of the kernels' own FP64 math routines -------------------------------------

namespace {

__global__ void math_check_kernel(int fn, const double* x, double* y, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = x[i];
        double r;
        switch (fn) {
        case 0: r = disco::rsqrt_nr(v); break;
        case 1: r = disco::rcp_nr(v); break;
        case 2: r = 2.0 * disco::half_j0_series<8>(v); break;
        case 3: r = 2.0 * disco::half_j0_series<6>(v); break;
        default: r = 2.0 * disco::half_j0_series<4>(v); break;
        }
        y[i] = r;
    }
}

} // namespace

extern "C" int disco_b200_math_check(int32_t fn, const double* x, double* y, int64_t n, void* stream)
{
    if (fn < 0 || fn > 4 || n < 0 || (n > 0 && (!x || !y))) {
        disco::set_last_error("math_check: bad argument");
        return DISCO_EINVAL;
    }
    if (n == 0) return DISCO_OK;
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 4096);
    math_check_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(fn, x, y, n);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        disco::set_last_error(std::string("math_check: ") + cudaGetErrorString(e));
        return DISCO_ECUDA;
    }
    return DISCO_OK;
}
