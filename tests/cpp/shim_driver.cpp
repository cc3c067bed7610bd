// Test driver of the C++ shim (disco_b200/csrc/backend_shim.cpp): a stand-in
// for the reference driver's call site (Code/main.cpp:713-730), compiled
// against include/backend.hpp and linked with libdisco_backend.so exactly as a
// reference build would be.  It reads atoms and loops from a binary file,
// calls gpuAvailable / printGpuInfo / gpuLineFp64 / kroupaGPU and writes the
// displacements and timings.
//
// input:  int64 n, int64 nloops, double box[3], int32 fp32, int32 pad,
//         double x[n], y[n], z[n], then per loop: int32 line, int32 count,
//         double phys[10], double cx, cy, cz, and count x/y/z triplets of
//         doubles (vertices of a line loop, loopons otherwise), SoA
// output: double ux[n], uy[n], uz[n], double kernels, double loopSec[nloops]
#include <cstdint>
#include <cstdio>
#include <vector>

#include "backend.hpp"

template <class T>
static bool get(FILE* f, T* p, size_t k)
{
    return std::fread(p, sizeof(T), k, f) == k;
}

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int64_t n = 0, nl = 0;
    double box[3];
    int32_t fp32 = 0, pad = 0;
    if (!get(f, &n, 1) || !get(f, &nl, 1) || !get(f, box, 3) || !get(f, &fp32, 1) || !get(f, &pad, 1)) return 3;
    std::vector<double> x(n), y(n), z(n), ux(n, 0.0), uy(n, 0.0), uz(n, 0.0);
    if (!get(f, x.data(), n) || !get(f, y.data(), n) || !get(f, z.data(), n)) return 3;
    std::vector<LoopData> loops((size_t)nl);
    for (auto& L : loops) {
        int32_t line = 0, count = 0;
        double phys[10], c[3];
        if (!get(f, &line, 1) || !get(f, &count, 1) || !get(f, phys, 10) || !get(f, c, 3)) return 3;
        L.phys = LoopPhys{ phys[0], phys[1], phys[2], phys[3], phys[4], phys[5], phys[6], phys[7], phys[8], phys[9] };
        L.line = line != 0;
        L.cx = c[0]; L.cy = c[1]; L.cz = c[2];
        std::vector<double>& a = L.line ? L.vx : L.x;
        std::vector<double>& b = L.line ? L.vy : L.y;
        std::vector<double>& d = L.line ? L.vz : L.z;
        a.resize(count); b.resize(count); d.resize(count);
        if (!get(f, a.data(), count) || !get(f, b.data(), count) || !get(f, d.data(), count)) return 3;
    }
    std::fclose(f);

    if (!gpuAvailable()) return 4;
    printGpuInfo();
    if (!gpuLineFp64()) return 5;
    AtomArrays atoms{ x.data(), y.data(), z.data(), ux.data(), uy.data(), uz.data(), (int)n };
    GpuOptions opt;
    opt.fp32 = fp32 != 0;
    BackendTiming t;
    kroupaGPU(atoms, loops, box[0], box[1], box[2], opt, t);

    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    std::fwrite(ux.data(), sizeof(double), n, o);
    std::fwrite(uy.data(), sizeof(double), n, o);
    std::fwrite(uz.data(), sizeof(double), n, o);
    std::fwrite(&t.kernels, sizeof(double), 1, o);
    std::vector<double> ls(t.loopSec);
    ls.resize((size_t)nl, 0.0);
    std::fwrite(ls.data(), sizeof(double), nl, o);
    std::fclose(o);
    return 0;
}
