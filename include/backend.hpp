#pragma once
// =============================================================================
// Source-compatible stand-in for the reference's backend interface
// (Code/backend.hpp:1-63, with LoopPhysT from Code/kroupa.hpp:24-41), so that
// disco_b200/csrc/backend_shim.cpp builds where the reference tree is absent.
// The declarations, field names, types and order are the reference's, because
// the reference driver (Code/main.cpp:689-730) fills and reads these types:
// any difference would break the drop-in.  In a reference build the shim is
// compiled against the reference's own backend.hpp instead of this file.
// =============================================================================

#include <string>
#include <vector>

constexpr double KROUPA_NU = 0.35;   // the reference's compile-time Poisson ratio

template <typename R>
struct LoopPhysT {
    R bx, by, bz;      // Burgers vector components (|b| per axis)
    R mx, my, mz;      // normalised glide direction m
    R nx, ny, nz;      // normalised loop normal n
    R dS;              // loopon surface element
};
using LoopPhys  = LoopPhysT<double>;
using LoopPhysF = LoopPhysT<float>;

struct LoopData {
    std::vector<double> x, y, z;       // loopon positions
    LoopPhys phys;
    bool line = false;
    std::vector<double> vx, vy, vz;    // polyline vertices, counter-clockwise about n
    double cx = 0., cy = 0., cz = 0.;  // fan apex (loop centre)
};

struct AtomArrays {
    const double *x, *y, *z;
    double *ux, *uy, *uz;
    int n;
};

struct BackendTiming {
    double upload = 0., kernels = 0., download = 0.;
    std::vector<double> loopSec;
};

int  cpuThreads();
void kroupaCPU(const AtomArrays& atoms, const std::vector<LoopData>& loops,
               double dx, double dy, double dz, BackendTiming& t);

struct GpuOptions {
    bool   fp32       = false;
    double chunkPairs = -1.;
};
#ifdef WITH_CUDA
bool gpuAvailable();
void printGpuInfo();
bool gpuLineFp64();
void kroupaGPU(const AtomArrays& atoms, const std::vector<LoopData>& loops,
               double dx, double dy, double dz, const GpuOptions& opt, BackendTiming& t);
#endif
