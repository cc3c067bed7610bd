// Batched form: many independent samples (own atoms, loops, box, image range)
// in one persistent launch per loop kind.
//
// Work unit = (sample, atom tile, table chunk).  The host knows every unit's
// exact cost (tile atoms x chunk segments or loopons x images), sorts the
// (sample, tile) items by cost and hands them greedily to the least-loaded
// CTA; each CTA then walks its own unit list, staging each unit's chunk with a
// bulk async copy into one of two shared-memory buffers while the other is
// computed.  Per-atom sums persist across the chunks of one item and are added
// to u at the item's last chunk, so no two CTAs ever touch the same atom.
// The launches of a plan are captured once in a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <queue>
#include <string>
#include <vector>

#include "common.cuh"
#include "field.cuh"
#include "field_device.cuh"
#include "field_fp32.cuh"

namespace disco {

struct SampleDev {
    const double *x, *y, *z;
    double *ux, *uy, *uz;
    int64_t n;
    const unsigned char* table;     // this sample's chunks (device)
    const Chunk* chunks;
    const LinePiece* pieces64;      // FP32 line form: FP64 pieces for the near-cut pass
    const LineSeg* segs64;
    const double* raw;              // line method: input vertex triplets
    int32_t nchunks, images, nimg, image_min;
    double Lx, Ly, Lz;
};

struct UnitDev {
    int32_t sample;
    int32_t tile;
    int16_t chunk;
    int8_t first, last;             // first / last chunk of this (sample, tile) item
    int32_t pad;
};

constexpr int kMaxStages = 4;

struct BatchArgs {
    const SampleDev* samples;
    const UnitDev* units;
    const int32_t* cta_first;       // units of CTA b: [cta_first[b], cta_first[b + 1])
    uint32_t stage_bytes;
    int32_t stages;                 // table stages in flight (2..kMaxStages)
    double cJ, cK, c2;
    float near_h, near_r;
    int* status;
    // FP32 line form: (sample, atom) pairs with near-cut pairs, listed by the
    // FP32 pass (near_mode 1); the unit-schedule FP64 pass (near_mode 2) runs
    // only when the list overflowed (*near_count > near_cap)
    int2* near_list;
    unsigned int* near_count;
    int32_t near_cap, near_mode;
};

constexpr int kBatchThreads = 256;

template <class Policy, int S>
__global__ void __launch_bounds__(kBatchThreads, Policy::kMinBlocks) batch_kernel(const BatchArgs b)
{
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    unsigned char* const stage0 = smem + kSmemHeader;
    const int tid = threadIdx.x;
    const int u0 = b.cta_first[blockIdx.x];
    const int nunits = b.cta_first[blockIdx.x + 1] - u0;
    if (nunits <= 0) return;
    if (b.near_mode == 2 && *b.near_count <= (unsigned)b.near_cap) return;   // the listed pass ran
    const int D = b.stages;
    if (tid == 0) {
        for (int j = 0; j < D; ++j) mbar_init(&bar[j], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int u) {
        const UnitDev un = b.units[u0 + u];
        const SampleDev& sd = b.samples[un.sample];
        const Chunk c = sd.chunks[un.chunk];
        stage_load(stage0 + (size_t)(u % D) * b.stage_bytes, sd.table + c.offset, c.bytes, &bar[u % D]);
    };
    if (tid == 0)
        for (int j = 0; j < D && j < nunits; ++j) issue(j);
    constexpr int kAtomsPerTile = kBatchThreads / S;
    const int split = tid % S;
    double px = 0.0, py = 0.0, pz = 0.0;
    int64_t atom = 0;
    bool valid = false;
    typename Policy::Acc acc;
    FieldArgs fa;
    for (int u = 0; u < nunits; ++u) {
        const UnitDev un = b.units[u0 + u];
        const SampleDev& sd = b.samples[un.sample];
        if (un.first) {
            atom = (int64_t)un.tile * kAtomsPerTile + tid / S;
            valid = atom < sd.n;
            const int64_t ia = valid ? atom : sd.n - 1;
            px = sd.x[ia]; py = sd.y[ia]; pz = sd.z[ia];
            acc.clear();
        }
        const int buf = u % D;
        const uint32_t parity = (uint32_t)((u / D) & 1);
        const bool ok = mbar_wait_bounded(&bar[buf], parity);
        if (__syncthreads_or(!ok)) {
            // give up: record it, let every copy still in flight land (bounded), return
            if (tid == 0) {
                report(b.status, DISCO_ETIMEOUT);
                for (int j = u; j < u + D && j < nunits; ++j) mbar_wait_bounded(&bar[j % D], (uint32_t)((j / D) & 1));
            }
            __syncthreads();
            return;
        }
        fa.images = sd.images;
        fa.nimg = sd.nimg;
        fa.image_min = sd.image_min;
        fa.Lx = sd.Lx; fa.Ly = sd.Ly; fa.Lz = sd.Lz;
        fa.cJ = b.cJ; fa.cK = b.cK; fa.c2 = b.c2;
        fa.near_h = b.near_h; fa.near_r = b.near_r;
        fa.pieces64 = sd.pieces64; fa.segs64 = sd.segs64; fa.raw = sd.raw;
        fa.near_list = nullptr; fa.near_count = nullptr; fa.near_cap = 0; fa.near_mode = 0;
        const unsigned char* st = stage0 + (size_t)buf * b.stage_bytes;
        Policy::template chunk<S>(fa, st, sd.chunks[un.chunk].npieces, split, px, py, pz, acc);
        if (un.last) {
            double ux, uy, uz;
            acc.total(ux, uy, uz);
#pragma unroll
            for (int o = S / 2; o > 0; o >>= 1) {
                ux += __shfl_xor_sync(0xffffffffu, ux, o);
                uy += __shfl_xor_sync(0xffffffffu, uy, o);
                uz += __shfl_xor_sync(0xffffffffu, uz, o);
            }
            if (valid && split == 0) {
                sd.ux[atom] += ux;
                sd.uy[atom] += uy;
                sd.uz[atom] += uz;
            }
            if constexpr (Policy::kAppendsNear) {
                if (b.near_mode == 1) {
                    const int lane = tid & 31;
                    const unsigned bn = __ballot_sync(0xffffffffu, acc.near);
                    const unsigned grp = S == 32 ? 0xffffffffu : (((1u << S) - 1u) << (lane & ~(S - 1)));
                    const bool app = valid && split == 0 && (bn & grp) != 0u;
                    const unsigned ba = __ballot_sync(0xffffffffu, app);
                    if (ba) {
                        const int leader = __ffs(ba) - 1;
                        unsigned q0 = 0;
                        if (lane == leader) q0 = atomicAdd(b.near_count, (unsigned)__popc(ba));
                        q0 = __shfl_sync(0xffffffffu, q0, leader);
                        const unsigned q = q0 + (unsigned)__popc(ba & ((1u << lane) - 1u));
                        if (app && q < (unsigned)b.near_cap) b.near_list[q] = make_int2(un.sample, (int)atom);
                    }
                }
            }
        }
        __syncthreads();                           // every warp is done with stage[buf]
        if (tid == 0 && u + D < nunits) {
            fence_proxy_async_smem();
            issue(u + D);
        }
    }
}

// FP64 pass of the FP32 line form over the listed (sample, atom) pairs: S
// lanes per pair split its images and walk the sample's chunks straight from
// global memory (the few near atoms do not pay for staging); a fixed-order
// butterfly sums the lanes, so each atom's result does not depend on the
// list's order.  Returns at once when the list overflowed (the unit-schedule
// pass runs instead).
template <int S>
__global__ void __launch_bounds__(kBatchThreads, 2) batch_near_list_kernel(const BatchArgs b)
{
    const unsigned cnt = *b.near_count;
    if (cnt > (unsigned)b.near_cap) return;
    const int tid = threadIdx.x;
    const int split = tid % S;
    constexpr int kPerCta = kBatchThreads / S;
    FieldArgs fa;
    fa.cJ = b.cJ; fa.cK = b.cK; fa.c2 = b.c2;
    fa.near_h = b.near_h; fa.near_r = b.near_r;
    fa.near_list = nullptr; fa.near_count = nullptr; fa.near_cap = 0; fa.near_mode = 0;
    for (int64_t e0 = (int64_t)blockIdx.x * kPerCta; e0 < (int64_t)cnt; e0 += (int64_t)gridDim.x * kPerCta) {
        const int64_t e = e0 + tid / S;
        const bool valid = e < (int64_t)cnt;
        const int2 pr = b.near_list[valid ? e : (int64_t)cnt - 1];
        const SampleDev& sd = b.samples[pr.x];
        const int64_t atom = pr.y;
        fa.images = sd.images; fa.nimg = sd.nimg; fa.image_min = sd.image_min;
        fa.Lx = sd.Lx; fa.Ly = sd.Ly; fa.Lz = sd.Lz;
        fa.pieces64 = sd.pieces64; fa.segs64 = sd.segs64; fa.raw = sd.raw;
        const double px = sd.x[atom], py = sd.y[atom], pz = sd.z[atom];
        LineNearFp64::Acc acc;
        acc.clear();
        for (int c = 0; c < sd.nchunks; ++c) {
            const Chunk ch = sd.chunks[c];
            LineNearFp64::template chunk<S>(fa, sd.table + ch.offset, ch.npieces, split, px, py, pz, acc);
        }
        double ux, uy, uz;
        acc.total(ux, uy, uz);
#pragma unroll
        for (int o = S / 2; o > 0; o >>= 1) {
            ux += __shfl_xor_sync(0xffffffffu, ux, o);
            uy += __shfl_xor_sync(0xffffffffu, uy, o);
            uz += __shfl_xor_sync(0xffffffffu, uz, o);
        }
        if (valid && split == 0) {
            sd.ux[atom] += ux;
            sd.uy[atom] += uy;
            sd.uz[atom] += uz;
        }
    }
}

} // namespace disco

// ---- host ----------------------------------------------------------------------------------

struct disco_batch_plan {
    int device = 0, sm_count = 0;
    disco_options opt;
    int nsamples = 0;
    int split = 1;
    int stages = 2;
    uint32_t stage_bytes = 0;
    // per kind (0 line, 1 loopon)
    unsigned char* d_table[2] = { nullptr, nullptr };
    disco::SampleDev* d_samples[2] = { nullptr, nullptr };
    disco::UnitDev* d_units[2] = { nullptr, nullptr };
    int32_t* d_cta_first[2] = { nullptr, nullptr };
    int grid[2] = { 0, 0 };
    bool fp32 = false;
    int* d_status = nullptr;
    int2* d_near = nullptr;                 // FP32 line form: (sample, atom) pairs with near-cut pairs
    unsigned int* d_near_count = nullptr;
    int32_t near_cap = 0;
    int near_grid = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t captured_on = nullptr;
    disco_plan_stats stats;
};

namespace {

int bfail(int code, const std::string& msg)
{
    disco::set_last_error(msg);
    return code;
}

int bcuda(cudaError_t e, const char* what)
{
    disco::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? DISCO_ENOMEM : DISCO_ECUDA;
}

void free_batch(disco_batch_plan* p)
{
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    for (int k = 0; k < 2; ++k) {
        if (p->d_table[k]) cudaFree(p->d_table[k]);
        if (p->d_samples[k]) cudaFree(p->d_samples[k]);
        if (p->d_units[k]) cudaFree(p->d_units[k]);
        if (p->d_cta_first[k]) cudaFree(p->d_cta_first[k]);
    }
    if (p->d_status) cudaFree(p->d_status);
    if (p->d_near) cudaFree(p->d_near);
    if (p->d_near_count) cudaFree(p->d_near_count);
    delete p;
}

template <class Policy>
int launch_batch_policy(const disco::BatchArgs& a, int grid, int split, cudaStream_t s, std::string& err)
{
    using namespace disco;
    const size_t smem = kSmemHeader + (size_t)a.stages * a.stage_bytes;
    void (*kern)(BatchArgs) = nullptr;
    switch (split) {
    case 1: kern = batch_kernel<Policy, 1>; break;
    case 2: kern = batch_kernel<Policy, 2>; break;
    case 4: kern = batch_kernel<Policy, 4>; break;
    default: kern = batch_kernel<Policy, 8>; break;
    }
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) { err = cudaGetErrorString(e); return DISCO_ECUDA; }
    kern<<<grid, kBatchThreads, smem, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) { err = cudaGetErrorString(e); return DISCO_ECUDA; }
    return DISCO_OK;
}

// Resident CTAs per SM of the batch kernel(s) of one loop kind at `smem` bytes.
template <class Policy>
int occupancy_of(int split, size_t smem)
{
    using namespace disco;
    void (*kern)(BatchArgs) = nullptr;
    switch (split) {
    case 1: kern = batch_kernel<Policy, 1>; break;
    case 2: kern = batch_kernel<Policy, 2>; break;
    case 4: kern = batch_kernel<Policy, 4>; break;
    default: kern = batch_kernel<Policy, 8>; break;
    }
    int per_sm = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBatchThreads, smem) != cudaSuccess)
        return 0;
    return per_sm;
}

int occupancy(int kind, bool fp32, int split, size_t smem)
{
    using namespace disco;
    if (kind == kLineKind)
        return fp32 ? std::min(occupancy_of<LineFp32>(split, smem), occupancy_of<LineNearFp64>(split, smem))
                    : occupancy_of<LineFp64>(split, smem);
    return fp32 ? occupancy_of<LooponFp32>(split, smem) : occupancy_of<LooponFp64>(split, smem);
}

// Launches every kernel of the plan on stream s (used once, under capture).
int launch_all(disco_batch_plan* p, cudaStream_t s)
{
    using namespace disco;
    const double pi = 3.14159265358979323846;
    const double c3 = 1.0 / (8.0 * pi * (1.0 - p->opt.nu));
    for (int k = 0; k < 2; ++k) {
        if (!p->grid[k]) continue;
        BatchArgs a;
        std::memset(&a, 0, sizeof(a));
        a.samples = p->d_samples[k];
        a.units = p->d_units[k];
        a.cta_first = p->d_cta_first[k];
        a.stage_bytes = p->stage_bytes;
        a.stages = p->stages;
        a.cJ = c3 - 1.0 / (4.0 * pi);
        a.cK = c3;
        a.c2 = 1.0 - 2.0 * p->opt.nu;
        a.near_h = p->opt.near_plane > 0.0 ? (float)p->opt.near_plane : kNearPlane;
        a.near_r = p->opt.near_rim > 0.0 ? (float)p->opt.near_rim : kNearRim;
        a.status = p->d_status;
        a.near_list = p->d_near;
        a.near_count = p->d_near_count;
        a.near_cap = p->near_cap;
        std::string err;
        int st;
        if (k == 0) {
            if (p->fp32) {
                // FP32 pass listing the near atoms, the listed FP64 pass, and the
                // unit-schedule FP64 pass that runs only if the list overflowed
                cudaError_t e = cudaMemsetAsync(p->d_near_count, 0, sizeof(unsigned int), s);
                if (e != cudaSuccess) return bfail(DISCO_ECUDA, cudaGetErrorString(e));
                a.near_mode = 1;
                st = launch_batch_policy<LineFp32>(a, p->grid[k], p->split, s, err);
                if (!st) {
                    batch_near_list_kernel<8><<<p->near_grid, kBatchThreads, 0, s>>>(a);
                    e = cudaGetLastError();
                    if (e != cudaSuccess) { err = cudaGetErrorString(e); st = DISCO_ECUDA; }
                }
                a.near_mode = 2;
                if (!st) st = launch_batch_policy<LineNearFp64>(a, p->grid[k], p->split, s, err);
            } else {
                st = launch_batch_policy<LineFp64>(a, p->grid[k], p->split, s, err);
            }
        } else {
            st = p->fp32 ? launch_batch_policy<LooponFp32>(a, p->grid[k], p->split, s, err)
                         : launch_batch_policy<LooponFp64>(a, p->grid[k], p->split, s, err);
        }
        if (st) return bfail(st, err);
    }
    return DISCO_OK;
}

} // namespace

extern "C" {

int disco_b200_batch_plan_create(const disco_sample* samples, int32_t nsamples, const disco_options* opt,
                                 disco_batch_plan** out)
{
    using namespace disco;
    if (!out) return bfail(DISCO_EINVAL, "null plan pointer");
    *out = nullptr;
    if (nsamples < 0 || (nsamples > 0 && !samples)) return bfail(DISCO_EINVAL, "bad sample array");
    disco_options o;
    if (opt) o = *opt; else disco_b200_options_default(&o);
    if (o.precision != DISCO_FP64 && o.precision != DISCO_FP32C) return bfail(DISCO_EINVAL, "bad precision");
    if (!(o.nu > -1.0 && o.nu < 0.5)) return bfail(DISCO_EINVAL, "nu must be in (-1, 0.5)");
    const int split = o.image_split > 0 ? o.image_split : 1;
    if (split != 1 && split != 2 && split != 4 && split != 8)
        return bfail(DISCO_EINVAL, "batched image_split must be 1, 2, 4 or 8");
    const uint32_t stage = (uint32_t)(o.stage_kb > 0 ? o.stage_kb : 48) * 1024u;
    if (stage < 16 * 1024u || stage > 100 * 1024u) return bfail(DISCO_EINVAL, "stage_kb must be in 16..100");
    const int stages = o.stages > 0 ? o.stages : 2;
    if (stages < 2 || stages > kMaxStages) return bfail(DISCO_EINVAL, "stages must be in 2..4");
    if (kSmemHeader + (size_t)stages * stage > 227u * 1024u)
        return bfail(DISCO_EINVAL, "stages x stage_kb exceeds the 227 KB of shared memory of a CTA");
    for (int s = 0; s < nsamples; ++s) {
        const disco_sample& sm = samples[s];
        if (sm.images < 0 || sm.images > 8) return bfail(DISCO_EINVAL, "sample images must be in 0..8");
        if (sm.image_min < 0 || sm.image_min > sm.images) return bfail(DISCO_EINVAL, "sample image_min out of range");
        if (!(sm.box[0] > 0.) || !(sm.box[1] > 0.) || !(sm.box[2] > 0.)) return bfail(DISCO_EINVAL, "bad box");
        if (sm.atoms.n < 0 || (sm.atoms.n > 0 && (!sm.atoms.x || !sm.atoms.y || !sm.atoms.z ||
                                                  !sm.atoms.ux || !sm.atoms.uy || !sm.atoms.uz)))
            return bfail(DISCO_EINVAL, "bad sample atoms");
        if (sm.nloops < 0 || (sm.nloops > 0 && !sm.loops)) return bfail(DISCO_EINVAL, "bad sample loops");
    }
    if (!disco_b200_available()) return bfail(DISCO_ENODEV, "no CUDA device");
    disco_batch_plan* p = new disco_batch_plan();
    p->opt = o;
    p->nsamples = nsamples;
    p->split = split;
    p->stages = stages;
    p->fp32 = o.precision == DISCO_FP32C;
    std::memset(&p->stats, 0, sizeof(p->stats));
    cudaError_t e = cudaGetDevice(&p->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&p->sm_count, cudaDevAttrMultiProcessorCount, p->device);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->d_status, 0, sizeof(int));
    if (e != cudaSuccess) { free_batch(p); return bcuda(e, "device setup"); }
    const int atoms_per_tile = kBatchThreads / split;
    uint32_t max_stage = 16;
    double evals = 0.0;
    for (int k = 0; k < 2; ++k) {
        const int kind = k == 0 ? kLineKind : kLooponKind;
        std::vector<unsigned char> bytes;
        std::vector<SampleDev> sdev(nsamples);
        std::vector<uint64_t> chunk_off(nsamples, 0), aux_off(nsamples, 0), aux_segs(nsamples, 0),
            aux_raw(nsamples, 0);
        std::vector<std::vector<Chunk>> chunks(nsamples);
        std::vector<double> work(nsamples, 0.0);        // evaluations per atom of each sample
        bool any = false;
        for (int s = 0; s < nsamples; ++s) {
            const disco_sample& sm = samples[s];
            HostTable T;
            std::string err;
            const int st = p->fp32 ? build_table_fp32(sm.loops, sm.nloops, kind, o.nu, T, err, stage)
                                   : build_table(sm.loops, sm.nloops, kind, o.precision, o.nu, T, err, stage);
            if (st) { free_batch(p); return bfail(st, err); }
            std::memset(&sdev[s], 0, sizeof(SampleDev));
            const int W = 2 * sm.images + 1;
            sdev[s].x = sm.atoms.x; sdev[s].y = sm.atoms.y; sdev[s].z = sm.atoms.z;
            sdev[s].ux = sm.atoms.ux; sdev[s].uy = sm.atoms.uy; sdev[s].uz = sm.atoms.uz;
            sdev[s].n = sm.atoms.n;
            sdev[s].images = sm.images;
            sdev[s].nimg = W * W * W;
            sdev[s].image_min = sm.image_min;
            sdev[s].Lx = sm.box[0]; sdev[s].Ly = sm.box[1]; sdev[s].Lz = sm.box[2];
            sdev[s].nchunks = (int32_t)T.chunks.size();
            if (T.chunks.empty()) continue;
            any = true;
            while (bytes.size() % 256) bytes.push_back(0);
            const uint64_t base = bytes.size();
            chunk_off[s] = base;
            bytes.insert(bytes.end(), T.bytes.begin(), T.bytes.end());
            chunks[s] = T.chunks;
            aux_off[s] = T.aux_pieces ? base + T.aux_pieces : 0;
            aux_segs[s] = T.aux_segs ? base + T.aux_segs : 0;
            aux_raw[s] = T.aux_raw ? base + T.aux_raw : 0;
            for (const Chunk& c : T.chunks) max_stage = std::max(max_stage, c.bytes);
            const int inner = sm.image_min > 0 ? 2 * sm.image_min - 1 : 0;
            work[s] = (double)(T.n_segments + T.n_loopons) * (sdev[s].nimg - inner * inner * inner);
            p->stats.n_segments += T.n_segments;
            p->stats.n_loopons += T.n_loopons;
            evals += work[s] * (double)sm.atoms.n;
        }
        if (!any) continue;
        // device copies of the tables, the chunk lists and the sample records
        std::vector<Chunk> all_chunks;
        std::vector<size_t> chunk_base(nsamples, 0);
        for (int s = 0; s < nsamples; ++s) {
            chunk_base[s] = all_chunks.size();
            all_chunks.insert(all_chunks.end(), chunks[s].begin(), chunks[s].end());
        }
        Chunk* d_chunks = nullptr;
        e = cudaMalloc(&p->d_table[k], bytes.size() + all_chunks.size() * sizeof(Chunk) + 256);
        if (e == cudaSuccess) e = cudaMemcpy(p->d_table[k], bytes.data(), bytes.size(), cudaMemcpyHostToDevice);
        const size_t chunks_at = (bytes.size() + 255) & ~size_t(255);
        d_chunks = reinterpret_cast<Chunk*>(p->d_table[k] + chunks_at);
        if (e == cudaSuccess && !all_chunks.empty())
            e = cudaMemcpy(d_chunks, all_chunks.data(), all_chunks.size() * sizeof(Chunk), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { free_batch(p); return bcuda(e, "batch table upload"); }
        for (int s = 0; s < nsamples; ++s) {
            if (chunks[s].empty()) continue;
            // chunk offsets are relative to the sample's own table
            sdev[s].table = p->d_table[k] + chunk_off[s];
            sdev[s].chunks = d_chunks + chunk_base[s];
            if (aux_raw[s]) sdev[s].raw = reinterpret_cast<const double*>(p->d_table[k] + aux_raw[s]);
            if (aux_off[s]) {
                sdev[s].pieces64 = reinterpret_cast<const LinePiece*>(p->d_table[k] + aux_off[s]);
                sdev[s].segs64 = reinterpret_cast<const LineSeg*>(p->d_table[k] + aux_segs[s]);
            }
        }
        // items (sample, tile) with their cost, longest first, greedy to the least-loaded CTA
        struct Item { double cost; int32_t sample, tile; };
        std::vector<Item> items;
        for (int s = 0; s < nsamples; ++s) {
            if (chunks[s].empty() || sdev[s].n == 0) continue;
            const int64_t ntiles = (sdev[s].n + atoms_per_tile - 1) / atoms_per_tile;
            for (int64_t t = 0; t < ntiles; ++t) {
                const int64_t na = std::min<int64_t>(atoms_per_tile, sdev[s].n - t * atoms_per_tile);
                // a partial tile costs what its warps run: whole warps
                const int64_t nw = (na * split + 31) / 32;
                items.push_back({ work[s] * (double)nw, s, (int32_t)t });
            }
        }
        std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) { return a.cost > b.cost; });
        // as many CTAs as fit on the GPU at once, so that the greedy balance holds
        const int per_sm = occupancy(kind, p->fp32, split, kSmemHeader + (size_t)stages * stage);
        if (per_sm < 1) { free_batch(p); return bfail(DISCO_ECUDA, "batch kernel does not fit on an SM"); }
        const int grid_max = p->sm_count * per_sm;
        const int grid = (int)std::min<size_t>(std::max<size_t>(items.size(), 1), (size_t)grid_max);
        std::vector<std::vector<int>> per_cta(grid);
        using Load = std::pair<double, int>;
        std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
        for (int c = 0; c < grid; ++c) heap.push({ 0.0, c });
        for (size_t i = 0; i < items.size(); ++i) {
            Load l = heap.top();
            heap.pop();
            per_cta[l.second].push_back((int)i);
            l.first += items[i].cost;
            heap.push(l);
        }
        std::vector<UnitDev> units;
        std::vector<int32_t> first(grid + 1, 0);
        for (int c = 0; c < grid; ++c) {
            first[c] = (int32_t)units.size();
            for (int i : per_cta[c]) {
                const Item& it = items[i];
                const int nch = (int)chunks[it.sample].size();
                for (int ch = 0; ch < nch; ++ch) {
                    UnitDev u;
                    std::memset(&u, 0, sizeof(u));
                    u.sample = it.sample;
                    u.tile = it.tile;
                    u.chunk = (int16_t)ch;
                    u.first = ch == 0;
                    u.last = ch == nch - 1;
                    units.push_back(u);
                }
            }
        }
        first[grid] = (int32_t)units.size();
        if (units.size() > 2147483647u) { free_batch(p); return bfail(DISCO_ELIMIT, "too many work units"); }
        e = cudaMalloc(&p->d_samples[k], std::max<size_t>(1, sdev.size()) * sizeof(SampleDev));
        if (e == cudaSuccess && nsamples > 0)
            e = cudaMemcpy(p->d_samples[k], sdev.data(), sdev.size() * sizeof(SampleDev), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc(&p->d_units[k], std::max<size_t>(1, units.size()) * sizeof(UnitDev));
        if (e == cudaSuccess && !units.empty())
            e = cudaMemcpy(p->d_units[k], units.data(), units.size() * sizeof(UnitDev), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc(&p->d_cta_first[k], first.size() * sizeof(int32_t));
        if (e == cudaSuccess)
            e = cudaMemcpy(p->d_cta_first[k], first.data(), first.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { free_batch(p); return bcuda(e, "batch queue upload"); }
        p->grid[k] = items.empty() ? 0 : grid;
        if (k == 0) p->stats.n_line_loops = 1; else p->stats.n_loopon_loops = 1;
    }
    if (p->fp32 && p->grid[0]) {
        int64_t total = 0;
        for (int s = 0; s < nsamples; ++s) total += samples[s].atoms.n;
        p->near_cap = (int32_t)std::min<int64_t>(std::max<int64_t>(total, 1), 1 << 21);
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_near_list_kernel<8>, kBatchThreads, 0);
        p->near_grid = std::max(1, p->sm_count * std::max(per_sm, 1));
        if (e == cudaSuccess) e = cudaMalloc(&p->d_near, (size_t)p->near_cap * sizeof(int2));
        if (e == cudaSuccess) e = cudaMalloc(&p->d_near_count, sizeof(unsigned int));
        if (e != cudaSuccess) { free_batch(p); return bcuda(e, "near-cut list"); }
    }
    p->stage_bytes = (max_stage + 15) & ~15u;
    p->stats.n_loops = nsamples;
    p->stats.evals_per_atom = evals;        // for a batch: total evaluations of one execute
    *out = p;
    return DISCO_OK;
}

int disco_b200_batch_plan_execute(disco_batch_plan* p, void* stream)
{
    if (!p) return bfail(DISCO_EINVAL, "null plan");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (!p->exec) {
        // capture the launches once on a private stream, then replay the graph
        cudaStream_t cap = nullptr;
        e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
        if (e != cudaSuccess) return bcuda(e, "capture stream");
        e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) { cudaStreamDestroy(cap); return bcuda(e, "begin capture"); }
        const int st = launch_all(p, cap);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (st) { if (g) cudaGraphDestroy(g); return st; }
        if (e != cudaSuccess) return bcuda(e, "end capture");
        p->graph = g;
        e = cudaGraphInstantiate(&p->exec, g, 0);
        if (e != cudaSuccess) { p->exec = nullptr; return bcuda(e, "graph instantiate"); }
    }
    e = cudaGraphLaunch(p->exec, s);
    if (e != cudaSuccess) return bcuda(e, "graph launch");
    return DISCO_OK;
}

int disco_b200_batch_plan_sync(disco_batch_plan* p, void* stream)
{
    if (!p) return bfail(DISCO_EINVAL, "null plan");
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return bcuda(e, "stream synchronize");
    int st = 0;
    e = cudaMemcpy(&st, p->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return bcuda(e, "status read");
    if (st) {
        cudaMemset(p->d_status, 0, sizeof(int));
        return bfail(st, "a batched kernel reported a bounded wait that gave up");
    }
    return DISCO_OK;
}

int disco_b200_batch_plan_stats(const disco_batch_plan* p, disco_plan_stats* s)
{
    if (!p || !s) return bfail(DISCO_EINVAL, "null argument");
    *s = p->stats;
    return DISCO_OK;
}

int disco_b200_batch_plan_destroy(disco_batch_plan* p)
{
    free_batch(p);
    return DISCO_OK;
}

// Host buffers: one device allocation holds every sample's atoms.
int disco_b200_batch(const disco_sample* samples, int32_t nsamples, const disco_options* opt,
                     disco_timing* timing)
{
    if (nsamples < 0 || (nsamples > 0 && !samples)) return bfail(DISCO_EINVAL, "bad sample array");
    int64_t total = 0;
    for (int s = 0; s < nsamples; ++s) {
        if (samples[s].atoms.n < 0) return bfail(DISCO_EINVAL, "negative atom count");
        total += samples[s].atoms.n;
    }
    if (!disco_b200_available()) return bfail(DISCO_ENODEV, "no CUDA device");
    cudaEvent_t ev[2] = { nullptr, nullptr };
    double* d = nullptr;
    disco_batch_plan* plan = nullptr;
    auto cleanup = [&]() {
        if (plan) disco_b200_batch_plan_destroy(plan);
        if (d) cudaFree(d);
        for (auto& x : ev) if (x) cudaEventDestroy(x);
    };
    cudaError_t e = cudaMalloc(&d, 6 * (size_t)std::max<int64_t>(total, 1) * sizeof(double));
    if (e != cudaSuccess) { cleanup(); return bcuda(e, "batch allocation"); }
    std::vector<disco_sample> dev(samples, samples + nsamples);
    int64_t off = 0;
    for (int s = 0; s < nsamples && e == cudaSuccess; ++s) {
        const int64_t n = samples[s].atoms.n;
        double* base = d + 6 * off;
        const double* src[6] = { samples[s].atoms.x, samples[s].atoms.y, samples[s].atoms.z,
                                 samples[s].atoms.ux, samples[s].atoms.uy, samples[s].atoms.uz };
        for (int k = 0; k < 6 && e == cudaSuccess && n > 0; ++k)
            e = cudaMemcpy(base + k * n, src[k], (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
        dev[s].atoms.x = base; dev[s].atoms.y = base + n; dev[s].atoms.z = base + 2 * n;
        dev[s].atoms.ux = base + 3 * n; dev[s].atoms.uy = base + 4 * n; dev[s].atoms.uz = base + 5 * n;
        off += n;
    }
    if (e != cudaSuccess) { cleanup(); return bcuda(e, "batch upload"); }
    int st = disco_b200_batch_plan_create(dev.data(), nsamples, opt, &plan);
    if (st) { cleanup(); return st; }
    e = cudaEventCreate(&ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&ev[1]);
    if (e == cudaSuccess) e = cudaEventRecord(ev[0], 0);
    if (e != cudaSuccess) { cleanup(); return bcuda(e, "events"); }
    st = disco_b200_batch_plan_execute(plan, nullptr);
    if (!st) {
        e = cudaEventRecord(ev[1], 0);
        st = e == cudaSuccess ? disco_b200_batch_plan_sync(plan, nullptr) : bcuda(e, "event");
    }
    if (st) { std::string m = disco_b200_last_error(); cleanup(); return bfail(st, m); }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    off = 0;
    for (int s = 0; s < nsamples && e == cudaSuccess; ++s) {
        const int64_t n = samples[s].atoms.n;
        double* base = d + 6 * off;
        double* dst[3] = { samples[s].atoms.ux, samples[s].atoms.uy, samples[s].atoms.uz };
        for (int k = 0; k < 3 && e == cudaSuccess && n > 0; ++k)
            e = cudaMemcpy(dst[k], base + (3 + k) * n, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
        off += n;
    }
    cleanup();
    if (e != cudaSuccess) return bcuda(e, "batch download");
    if (timing) { timing->upload = 0.0; timing->kernels = ms * 1e-3; timing->download = 0.0; }
    return DISCO_OK;
}

} // extern "C"
