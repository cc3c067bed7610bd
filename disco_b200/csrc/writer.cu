// Text output of the final positions on the device: the atom lines of the
// reference's XYZ writer (Code/main.cpp:826-831) and LAMMPS writer
// (Code/main.cpp:86-92, orthorhombic box), formatted as the C++ stream does
// with `fixed << setprecision(8)`: each coordinate rounded to 8 decimals from
// its exact binary value, ties to even, sign kept for negative values that
// round to zero.
//
// Rounding: a = m 2^k (m the 53-bit significand), so a 1e8 = m 1e8 2^k exactly,
// with m 1e8 < 2^80 held in a 128-bit integer; shifting by -k with round-half-
// even gives the 8-decimal integer R exactly (64 bits: |v| below 1.8e11).
//
// Three kernels: per tile of 1024 atoms the line lengths are summed
// (len_kernel); one CTA turns the tile sums into offsets (offsets_kernel);
// each tile recomputes its lengths, scans them and writes its lines
// (write_kernel).  Only the tile sums are kept between the passes.
#include <algorithm>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 4;
constexpr int kTile = kThreads * kPerThread;
constexpr int kMaxPrefix = 64;            // bytes of the XYZ element name

struct Fixed8 {
    unsigned long long R;                 // round(|v| 1e8)
    bool neg, ok;
};

__device__ __forceinline__ Fixed8 fixed8(double v)
{
    Fixed8 f;
    const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
    f.neg = (bits >> 63) != 0;
    const int ex = (int)((bits >> 52) & 0x7FF);
    const unsigned long long mant = bits & ((1ull << 52) - 1);
    f.ok = ex != 0x7FF;
    f.R = 0;
    if (!f.ok) return f;
    const unsigned long long m = ex == 0 ? mant : (mant | (1ull << 52));
    const int k = ex == 0 ? -1074 : ex - 1075;
    const unsigned __int128 P = (unsigned __int128)m * 100000000ull;
    if (k >= 0) {
        if (k > 10 || (P << k) >> 64) { f.ok = false; return f; }
        f.R = (unsigned long long)(P << k);
        return f;
    }
    const int s = -k;
    if (s > 100) return f;                // |v| 1e8 < 2^-20: rounds to 0
    const unsigned __int128 q = P >> s;
    const unsigned __int128 r = P - (q << s);
    const unsigned __int128 half = (unsigned __int128)1 << (s - 1);
    unsigned __int128 R = q;
    if (r > half || (r == half && (q & 1))) R += 1;
    if (R >> 64) { f.ok = false; return f; }
    f.R = (unsigned long long)R;
    return f;
}

__device__ __forceinline__ int ndigits(unsigned long long v)
{
    int d = 1;
    while (v >= 10) { v /= 10; ++d; }
    return d;
}

__device__ __forceinline__ int fixed8_len(const Fixed8& f)
{
    return (f.neg ? 1 : 0) + ndigits(f.R / 100000000ull) + 9;
}

__device__ __forceinline__ char* put_uint(char* o, unsigned long long v)
{
    const int d = ndigits(v);
    for (int i = d - 1; i >= 0; --i) { o[i] = (char)('0' + v % 10); v /= 10; }
    return o + d;
}

__device__ __forceinline__ char* put_fixed8(char* o, const Fixed8& f)
{
    if (f.neg) *o++ = '-';
    o = put_uint(o, f.R / 100000000ull);
    *o++ = '.';
    unsigned long long fr = f.R % 100000000ull;
    for (int i = 7; i >= 0; --i) { o[i] = (char)('0' + fr % 10); fr /= 10; }
    return o + 8;
}

struct WriterArgs {
    const double *x, *y, *z;
    int64_t n;
    int32_t lammps;                       // 0: "<element> x y z", 1: "<k+1> 1 x y z"
    int32_t plen;
    char prefix[kMaxPrefix];
    int64_t* tile_len;                    // per tile, then exclusive offsets
    int* bad;
    char* out;
};

__device__ __forceinline__ int line_len(const WriterArgs& a, int64_t i, Fixed8 (&c)[3])
{
    c[0] = fixed8(a.x[i]);
    c[1] = fixed8(a.y[i]);
    c[2] = fixed8(a.z[i]);
    if (!(c[0].ok && c[1].ok && c[2].ok)) atomicExch(a.bad, 1);
    const int head = a.lammps ? ndigits((unsigned long long)(i + 1)) + 3 : a.plen + 1;
    return head + fixed8_len(c[0]) + 1 + fixed8_len(c[1]) + 1 + fixed8_len(c[2]) + 1;
}

// Exclusive scan of one value per thread over the CTA; returns the CTA total.
__device__ __forceinline__ long long cta_scan(long long v, long long& excl)
{
    __shared__ long long warp_tot[kThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_tot[w] = inc;
    __syncthreads();
    long long base = 0, tot = 0;
    for (int k = 0; k < kThreads / 32; ++k) {
        if (k < w) base += warp_tot[k];
        tot += warp_tot[k];
    }
    __syncthreads();
    excl = base + inc - v;
    return tot;
}

__global__ void __launch_bounds__(kThreads) len_kernel(const WriterArgs a)
{
    const int64_t t0 = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kPerThread;
    long long mine = 0;
    for (int j = 0; j < kPerThread; ++j) {
        const int64_t i = t0 + j;
        if (i < a.n) {
            Fixed8 c[3];
            mine += line_len(a, i, c);
        }
    }
    long long excl;
    const long long tot = cta_scan(mine, excl);
    if (threadIdx.x == 0) a.tile_len[blockIdx.x] = tot;
}

// tile_len[b] -> exclusive offsets, total in tile_len[ntiles]
__global__ void __launch_bounds__(kThreads) offsets_kernel(int64_t* tile_len, int64_t ntiles)
{
    long long carry = 0;
    for (int64_t b0 = 0; b0 < ntiles; b0 += kThreads) {
        const int64_t b = b0 + threadIdx.x;
        const long long v = b < ntiles ? tile_len[b] : 0;
        long long excl;
        const long long tot = cta_scan(v, excl);
        if (b < ntiles) tile_len[b] = carry + excl;
        carry += tot;
    }
    if (threadIdx.x == 0) tile_len[ntiles] = carry;
}

__global__ void __launch_bounds__(kThreads) write_kernel(const WriterArgs a)
{
    const int64_t t0 = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kPerThread;
    Fixed8 c[kPerThread][3];
    int len[kPerThread];
    long long mine = 0;
    for (int j = 0; j < kPerThread; ++j) {
        const int64_t i = t0 + j;
        len[j] = i < a.n ? line_len(a, i, c[j]) : 0;
        mine += len[j];
    }
    long long excl;
    cta_scan(mine, excl);
    char* o = a.out + a.tile_len[blockIdx.x] + excl;
    for (int j = 0; j < kPerThread; ++j) {
        const int64_t i = t0 + j;
        if (i >= a.n) break;
        if (a.lammps) {
            o = put_uint(o, (unsigned long long)(i + 1));
            *o++ = ' '; *o++ = '1'; *o++ = ' ';
        } else {
            for (int p = 0; p < a.plen; ++p) *o++ = a.prefix[p];
            *o++ = ' ';
        }
        o = put_fixed8(o, c[j][0]);
        *o++ = ' ';
        o = put_fixed8(o, c[j][1]);
        *o++ = ' ';
        o = put_fixed8(o, c[j][2]);
        *o++ = '\n';
    }
}

int wfail(int code, const std::string& msg)
{
    disco::set_last_error(msg);
    return code;
}

} // namespace

extern "C" int disco_b200_format_atoms(int32_t format, const char* element, const double* x, const double* y,
                                       const double* z, int64_t n, char* out, int64_t capacity,
                                       int64_t* bytes, void* stream)
{
    if (!bytes || n < 0 || (format != 0 && format != 1) || (n > 0 && (!x || !y || !z)))
        return wfail(DISCO_EINVAL, "format_atoms: bad argument");
    *bytes = 0;
    WriterArgs a;
    std::memset(&a, 0, sizeof(a));
    a.lammps = format;
    if (format == 0) {
        const size_t L = element ? std::strlen(element) : 0;
        if (L == 0 || L > (size_t)kMaxPrefix) return wfail(DISCO_EINVAL, "format_atoms: element name of 1..64 bytes");
        std::memcpy(a.prefix, element, L);
        a.plen = (int32_t)L;
    }
    if (n == 0) return DISCO_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t ntiles = (n + kTile - 1) / kTile;
    a.x = x; a.y = y; a.z = z; a.n = n;
    void* scratch = nullptr;
    cudaError_t e = cudaMallocAsync(&scratch, (size_t)(ntiles + 2) * sizeof(int64_t), s);
    if (e != cudaSuccess) return wfail(DISCO_ENOMEM, std::string("format_atoms: ") + cudaGetErrorString(e));
    a.tile_len = static_cast<int64_t*>(scratch);
    a.bad = reinterpret_cast<int*>(a.tile_len + ntiles + 1);
    int64_t total = 0;
    int bad = 0;
    e = cudaMemsetAsync(a.bad, 0, sizeof(int), s);
    if (e == cudaSuccess) {
        len_kernel<<<(unsigned)ntiles, kThreads, 0, s>>>(a);
        offsets_kernel<<<1, kThreads, 0, s>>>(a.tile_len, ntiles);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, a.tile_len + ntiles, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, a.bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    int st = DISCO_OK;
    if (e != cudaSuccess) {
        st = wfail(DISCO_ECUDA, std::string("format_atoms: ") + cudaGetErrorString(e));
    } else if (bad) {
        st = wfail(DISCO_EINVAL, "format_atoms: a coordinate is not finite or |v| >= 1.8e11");
    } else {
        *bytes = total;
        if (total > capacity || !out) {
            st = wfail(DISCO_ELIMIT, "format_atoms: output buffer too small (*bytes holds the size needed)");
        } else {
            a.out = out;
            write_kernel<<<(unsigned)ntiles, kThreads, 0, s>>>(a);
            e = cudaGetLastError();
            if (e != cudaSuccess) st = wfail(DISCO_ECUDA, std::string("format_atoms: ") + cudaGetErrorString(e));
        }
    }
    cudaFreeAsync(scratch, s);
    return st;
}
