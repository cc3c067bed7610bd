// extern "C" entry points of the displacement backend (include/disco_b200.h):
// device queries, plans (tables built and uploaded once), the resident
// execute and the host-buffer drop-in that replaces kroupaGPU
// (Code/backend_cuda.cu:568-722).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "common.cuh"
#include "field.cuh"

namespace disco {
int choose_split(int64_t n, int nimg, int resident_ctas);
int launch_field_fp32(const FieldArgs& a, int kind, int sm_count, int split_hint,
                      cudaStream_t stream, std::string& err);
}

struct disco_plan {
    int device = 0;
    int sm_count = 0;
    double box[3] = { 0., 0., 0. };
    disco_options opt;
    int nimg = 1;
    int nloops = 0;
    disco::HostTable tables[2];              // line, loopon
    unsigned char* d_table[2] = { nullptr, nullptr };
    disco::Chunk* d_chunks[2] = { nullptr, nullptr };
    int* d_status = nullptr;
    int32_t* d_near = nullptr;               // FP32 line form: atoms with near-cut pairs
    unsigned int* d_near_count = nullptr;
    int32_t near_cap = 0;
    std::vector<double> loop_evals;          // per input loop: segments or loopons
    disco_plan_stats stats;
};

namespace {

// Last error message of the calling thread: a fixed buffer, so that setting it
// never allocates.
thread_local char g_last_error[512];

void store_error(const char* msg)
{
    std::snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
}

int fail(int code, const std::string& msg)
{
    store_error(msg.c_str());
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    return fail(e == cudaErrorMemoryAllocation ? DISCO_ENOMEM : DISCO_ECUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define DISCO_TRY_CUDA(call, what)                     \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

int check_options(const disco_options& o)
{
    if (o.precision != DISCO_FP64 && o.precision != DISCO_FP32C)
        return fail(DISCO_EINVAL, "precision must be DISCO_FP64 or DISCO_FP32C");
    if (o.images < 0 || o.images > 8) return fail(DISCO_EINVAL, "images must be in 0..8");
    if (o.image_min < 0 || o.image_min > o.images) return fail(DISCO_EINVAL, "image_min must be in 0..images");
    if (!(o.nu > -1.0 && o.nu < 0.5)) return fail(DISCO_EINVAL, "nu must be in (-1, 0.5)");
    if (!(o.near_plane >= 0.0) || !(o.near_rim >= 0.0))
        return fail(DISCO_EINVAL, "near_plane and near_rim must be >= 0");
    if (o.stage_kb != 0 && (o.stage_kb < 16 || o.stage_kb > 100))
        return fail(DISCO_EINVAL, "stage_kb must be 0 or in 16..100");
    if (o.image_split != 0 && (o.image_split < 1 || o.image_split > 32 ||
                               (o.image_split & (o.image_split - 1))))
        return fail(DISCO_EINVAL, "image_split must be 0 or a power of two up to 32");
    return DISCO_OK;
}

void free_plan(disco_plan* p)
{
    if (!p) return;
    for (int k = 0; k < 2; ++k) {
        if (p->d_table[k]) cudaFree(p->d_table[k]);
        if (p->d_chunks[k]) cudaFree(p->d_chunks[k]);
    }
    if (p->d_status) cudaFree(p->d_status);
    if (p->d_near) cudaFree(p->d_near);
    if (p->d_near_count) cudaFree(p->d_near_count);
    delete p;
}

double now_s()
{
    using C = std::chrono::steady_clock;
    return std::chrono::duration<double>(C::now().time_since_epoch()).count();
}

} // namespace

void disco::set_last_error(const std::string& msg) { store_error(msg.c_str()); }
void disco::set_last_error(const char* msg) { store_error(msg); }

extern "C" {

const char* disco_b200_last_error(void) { return g_last_error; }

const char* disco_b200_strerror(int s)
{
    switch (s) {
    case DISCO_OK:       return "ok";
    case DISCO_EINVAL:   return "invalid argument";
    case DISCO_ENODEV:   return "no usable CUDA device";
    case DISCO_ECUDA:    return "CUDA error";
    case DISCO_ENOMEM:   return "out of memory";
    case DISCO_ELIMIT:   return "size above a limit or capacity";
    case DISCO_ETIMEOUT: return "bounded device wait gave up";
    case DISCO_EPLANES:  return "|b.n| is not a whole number of plane spacings";
    default:             return "unknown status";
    }
}

int disco_b200_available(void)
{
    int count = 0;
    return (cudaGetDeviceCount(&count) == cudaSuccess && count > 0) ? 1 : 0;
}

int disco_b200_line_fp64(void) { return 1; }

// printGpuInfo (Code/backend_cuda.cu:543-553): same banner lines.
int disco_b200_device_info(char* buf, size_t len)
{
    if (!buf || len == 0) return fail(DISCO_EINVAL, "null buffer");
    if (!disco_b200_available()) return fail(DISCO_ENODEV, "no CUDA device");
    int dev = 0;
    DISCO_TRY_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    cudaDeviceProp p;
    DISCO_TRY_CUDA(cudaGetDeviceProperties(&p, dev), "cudaGetDeviceProperties");
    std::snprintf(buf, len,
                  "\n--- GPU: %s ---\n  SMs              : %d\n  Global memory    : %zu MB\n"
                  "  Shared mem/block : %zu KB\n\n",
                  p.name, p.multiProcessorCount, (size_t)(p.totalGlobalMem >> 20),
                  (size_t)(p.sharedMemPerBlock / 1024));
    return DISCO_OK;
}

void disco_b200_options_default(disco_options* o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = DISCO_FP64;
    o->images = 1;                // Code/backend_cpu.cpp:51-53
    o->nu = 0.35;                 // Code/kroupa.hpp:24
    o->chunk_pairs = -1.0;        // GpuOptions default (Code/backend.hpp:55)
}

int disco_b200_plan_create(const disco_loop* loops, int32_t nloops, const double box[3],
                           const disco_options* opt, int64_t max_atoms, disco_plan** out)
{
    if (!out) return fail(DISCO_EINVAL, "null plan pointer");
    *out = nullptr;
    if (nloops < 0 || (nloops > 0 && !loops)) return fail(DISCO_EINVAL, "bad loop array");
    if (!box || !(box[0] > 0.) || !(box[1] > 0.) || !(box[2] > 0.))
        return fail(DISCO_EINVAL, "box lengths must be positive");
    disco_options o;
    if (opt) o = *opt; else disco_b200_options_default(&o);
    int st = check_options(o);
    if (st) return st;
    if (max_atoms < 0) return fail(DISCO_EINVAL, "max_atoms < 0");
    if (!disco_b200_available()) return fail(DISCO_ENODEV, "no CUDA device");

    disco_plan* p = new disco_plan();
    p->opt = o;
    p->nloops = nloops;
    for (int i = 0; i < 3; ++i) p->box[i] = box[i];
    const int W = 2 * o.images + 1;
    p->nimg = W * W * W;
    cudaError_t e = cudaGetDevice(&p->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&p->sm_count, cudaDevAttrMultiProcessorCount, p->device);
    if (e != cudaSuccess) { free_plan(p); return cuda_fail(e, "device query"); }

    std::memset(&p->stats, 0, sizeof(p->stats));
    p->stats.n_loops = nloops;
    p->stats.n_images = p->nimg;
    p->loop_evals.assign((size_t)nloops, 0.0);
    for (int l = 0; l < nloops; ++l) {
        if (loops[l].line) p->stats.n_line_loops++; else p->stats.n_loopon_loops++;
    }
    for (int k = 0; k < 2; ++k) {
        std::string err;
        const int kind = k == 0 ? disco::kLineKind : disco::kLooponKind;
        const uint32_t cap = o.stage_kb > 0 ? (uint32_t)o.stage_kb * 1024u : 0u;
        st = o.precision == DISCO_FP32C
                 ? disco::build_table_fp32(loops, nloops, kind, o.nu, p->tables[k], err, cap)
                 : disco::build_table(loops, nloops, kind, o.precision, o.nu, p->tables[k], err, cap);
        if (st) { free_plan(p); return fail(st, err); }
        const disco::HostTable& T = p->tables[k];
        for (int l = 0; l < nloops; ++l) p->loop_evals[l] += T.loop_evals[l];
        p->stats.n_segments += T.n_segments;
        p->stats.n_loopons += T.n_loopons;
        if (T.chunks.empty()) continue;
        e = cudaMalloc(&p->d_table[k], T.bytes.size());
        if (e == cudaSuccess) e = cudaMemcpy(p->d_table[k], T.bytes.data(), T.bytes.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc(&p->d_chunks[k], T.chunks.size() * sizeof(disco::Chunk));
        if (e == cudaSuccess)
            e = cudaMemcpy(p->d_chunks[k], T.chunks.data(), T.chunks.size() * sizeof(disco::Chunk),
                           cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { free_plan(p); return cuda_fail(e, "loop table upload"); }
    }
    {
        const int inner = o.image_min > 0 ? 2 * o.image_min - 1 : 0;
        p->stats.n_images = p->nimg - inner * inner * inner;
    }
    p->stats.evals_per_atom = (double)(p->stats.n_segments + p->stats.n_loopons) * p->stats.n_images;
    e = cudaMalloc(&p->d_status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->d_status, 0, sizeof(int));
    if (e != cudaSuccess) { free_plan(p); return cuda_fail(e, "status word"); }
    if (o.precision == DISCO_FP32C && !p->tables[0].chunks.empty()) {
        // the list of atoms with near-cut pairs: up to 2^21 (a longer list
        // overflows and the FP64 pass visits every atom)
        p->near_cap = (int32_t)std::min<int64_t>(std::max<int64_t>(max_atoms, 1 << 16), 1 << 21);
        e = cudaMalloc(&p->d_near, (size_t)p->near_cap * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMalloc(&p->d_near_count, sizeof(unsigned int));
        if (e != cudaSuccess) { free_plan(p); return cuda_fail(e, "near-cut list"); }
    }
    *out = p;
    return DISCO_OK;
}

int disco_b200_plan_execute(disco_plan* p, const disco_atoms* a, void* stream)
{
    if (!p || !a) return fail(DISCO_EINVAL, "null plan or atoms");
    if (a->n < 0) return fail(DISCO_EINVAL, "negative atom count");
    if (a->n == 0) return DISCO_OK;
    if (!a->x || !a->y || !a->z || !a->ux || !a->uy || !a->uz) return fail(DISCO_EINVAL, "null atom array");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (int k = 0; k < 2; ++k) {
        const disco::HostTable& T = p->tables[k];
        if (T.chunks.empty()) continue;
        disco::FieldArgs fa;
        std::memset(&fa, 0, sizeof(fa));
        fa.x = a->x; fa.y = a->y; fa.z = a->z;
        fa.ux = a->ux; fa.uy = a->uy; fa.uz = a->uz;
        fa.n = a->n;
        fa.table = p->d_table[k];
        fa.chunks = p->d_chunks[k];
        fa.nchunks = (int32_t)T.chunks.size();
        fa.stage_bytes = T.stage_bytes;
        fa.resident = T.resident ? 1 : 0;
        fa.images = p->opt.images;
        fa.nimg = p->nimg;
        fa.image_min = p->opt.image_min;
        fa.Lx = p->box[0]; fa.Ly = p->box[1]; fa.Lz = p->box[2];
        const double pi = 3.14159265358979323846;
        const double c3 = 1.0 / (8.0 * pi * (1.0 - p->opt.nu));      // Code/barnett.hpp:51
        fa.cJ = c3 - 1.0 / (4.0 * pi);
        fa.cK = c3;
        fa.c2 = 1.0 - 2.0 * p->opt.nu;                              // Code/kroupa.hpp:66
        fa.status = p->d_status;
        fa.near_h = (float)p->opt.near_plane;
        fa.near_r = (float)p->opt.near_rim;
        if (k == 0 && T.aux_raw)
            fa.raw = reinterpret_cast<const double*>(p->d_table[k] + T.aux_raw);
        if (T.fp32 && k == 0 && T.aux_pieces) {
            fa.pieces64 = reinterpret_cast<const disco::LinePiece*>(p->d_table[k] + T.aux_pieces);
            fa.segs64 = reinterpret_cast<const disco::LineSeg*>(p->d_table[k] + T.aux_segs);
            fa.near_list = p->d_near;
            fa.near_count = p->d_near_count;
            fa.near_cap = p->near_cap;
        }
        std::string err;
        const int kind = k == 0 ? disco::kLineKind : disco::kLooponKind;
        const int st = T.fp32
            ? disco::launch_field_fp32(fa, kind, p->sm_count, p->opt.image_split, s, err)
            : disco::launch_field(fa, kind, false, p->sm_count, p->opt.threads_per_block,
                                  p->opt.image_split, s, err);
        if (st) return fail(st, err);
    }
    return DISCO_OK;
}

int disco_b200_plan_sync(disco_plan* p, void* stream)
{
    if (!p) return fail(DISCO_EINVAL, "null plan");
    DISCO_TRY_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "stream synchronize");
    int st = 0;
    DISCO_TRY_CUDA(cudaMemcpy(&st, p->d_status, sizeof(int), cudaMemcpyDeviceToHost), "status read");
    if (st) {
        cudaMemset(p->d_status, 0, sizeof(int));
        return fail(st, "a kernel reported: " + std::string(disco_b200_strerror(st)));
    }
    return DISCO_OK;
}

int disco_b200_plan_stats(const disco_plan* p, disco_plan_stats* s)
{
    if (!p || !s) return fail(DISCO_EINVAL, "null argument");
    *s = p->stats;
    return DISCO_OK;
}

int disco_b200_plan_destroy(disco_plan* p)
{
    free_plan(p);
    return DISCO_OK;
}

// kroupaGPU on host buffers (Code/backend_cuda.cu:568-722): allocate, upload,
// one launch per loop kind, download, free.  The displacement arrays are
// uploaded too, so the call accumulates into them exactly like the CPU backend.
int disco_b200_displace(const disco_atoms* atoms, const disco_loop* loops, int32_t nloops,
                        const double box[3], const disco_options* opt, disco_timing* timing)
{
    if (!atoms) return fail(DISCO_EINVAL, "null atoms");
    const int64_t n = atoms->n;
    if (n < 0) return fail(DISCO_EINVAL, "negative atom count");
    if (n > 0 && (!atoms->x || !atoms->y || !atoms->z || !atoms->ux || !atoms->uy || !atoms->uz))
        return fail(DISCO_EINVAL, "null atom array");
    disco_options o;
    if (opt) o = *opt; else disco_b200_options_default(&o);

    const double t0 = now_s();
    disco_plan* plan = nullptr;
    int st = disco_b200_plan_create(loops, nloops, box, &o, n, &plan);
    if (st) return st;
    if (o.verbose) {
        std::printf("Precision: %s\n", o.precision == DISCO_FP32C
                    ? "single (fp32 pair term, compensated sums)" : "double");
    }
    double* d = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t ev[2] = { nullptr, nullptr };
    auto cleanup = [&]() {
        if (d) cudaFree(d);
        if (s) cudaStreamDestroy(s);
        for (auto& x : ev) if (x) cudaEventDestroy(x);
        disco_b200_plan_destroy(plan);
    };
    const size_t bytes = (size_t)n * sizeof(double);
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&ev[1]);
    if (e == cudaSuccess && n > 0) e = cudaMalloc(&d, 6 * bytes);
    const double* src[6] = { atoms->x, atoms->y, atoms->z, atoms->ux, atoms->uy, atoms->uz };
    for (int k = 0; k < 6 && e == cudaSuccess && n > 0; ++k)
        e = cudaMemcpyAsync(d + (size_t)k * n, src[k], bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { cleanup(); return cuda_fail(e, "atom upload"); }
    const double t1 = now_s();

    if (o.verbose) std::printf("Running GPU kernels...\n");
    disco_atoms da;
    da.x = d; da.y = d + n; da.z = d + 2 * n;
    da.ux = d + 3 * n; da.uy = d + 4 * n; da.uz = d + 5 * n;
    da.n = n;
    e = cudaEventRecord(ev[0], s);
    if (e != cudaSuccess) { cleanup(); return cuda_fail(e, "event"); }
    st = disco_b200_plan_execute(plan, &da, s);
    if (st) { cleanup(); return st; }
    e = cudaEventRecord(ev[1], s);
    if (e != cudaSuccess) { cleanup(); return cuda_fail(e, "event"); }
    st = disco_b200_plan_sync(plan, s);
    if (st) { std::string m = g_last_error; cleanup(); return fail(st, m); }  // keep the kernel's message
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    const double t2 = now_s();
    if (o.verbose) std::printf("\nGPU kernel time: %g ms\n\n", (double)ms);

    double* dst[3] = { atoms->ux, atoms->uy, atoms->uz };
    for (int k = 0; k < 3 && e == cudaSuccess && n > 0; ++k)
        e = cudaMemcpyAsync(dst[k], d + (size_t)(3 + k) * n, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { cleanup(); return cuda_fail(e, "displacement download"); }
    std::vector<double> evals = plan->loop_evals;
    cleanup();
    const double t3 = now_s();
    if (timing) {
        timing->upload = t1 - t0;
        timing->kernels = t2 - t1;
        timing->download = t3 - t2;
        if (timing->loop_sec) {
            double tot = 0.0;
            for (double v : evals) tot += v;
            for (int l = 0; l < nloops; ++l)
                timing->loop_sec[l] = tot > 0.0 ? (ms * 1e-3) * evals[l] / tot : 0.0;
        }
    }
    return DISCO_OK;
}

} // extern "C"
