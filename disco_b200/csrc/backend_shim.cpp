// =============================================================================
// The reference's GPU backend functions (Code/backend.hpp:57-62) on top of the
// C-ABI of libdisco_b200.so.  A reference build links this file and the
// library in place of Code/backend_cuda.cu; Code/main.cpp then selects the
// B200 backend exactly as before (gpuAvailable -> printGpuInfo -> kroupaGPU).
//
// Behaviour kept from the reference:
//   - errors print "CUDA error at <file>:<line>  <message>" and exit(EXIT_FAILURE)
//     (Code/backend_cuda.cu:45-53);
//   - BackendTiming is filled (upload, kernels, download, one loopSec per loop);
//   - GpuOptions::fp32 selects the single-precision form, chunkPairs is accepted
//     (B200 has no watchdog to chunk around);
//   - images +-1 and nu = KROUPA_NU, the reference's fixed values.
// =============================================================================
#define WITH_CUDA 1
#include "backend.hpp"

#include <cstdlib>
#include <iostream>
#include <vector>

#include "disco_b200.h"

namespace {

[[noreturn]] void die(int line)
{
    std::cerr << "CUDA error at " << __FILE__ << ":" << line << "  " << disco_b200_last_error() << "\n";
    std::exit(EXIT_FAILURE);
}

} // namespace

bool gpuAvailable()
{
    return disco_b200_available() != 0;
}

void printGpuInfo()
{
    char buf[512];
    if (disco_b200_device_info(buf, sizeof(buf)) != DISCO_OK) die(__LINE__);
    std::cout << buf;
}

bool gpuLineFp64()
{
    return disco_b200_line_fp64() != 0;
}

void kroupaGPU(const AtomArrays& atoms, const std::vector<LoopData>& loops,
               double dx, double dy, double dz, const GpuOptions& opt, BackendTiming& t)
{
    std::vector<disco_loop> L(loops.size());
    for (size_t l = 0; l < loops.size(); ++l) {
        const LoopData& s = loops[l];
        disco_loop& d = L[l];
        d.x = s.x.data(); d.y = s.y.data(); d.z = s.z.data();
        d.n_loopons = (int32_t)s.x.size();
        d.line = s.line ? 1 : 0;
        d.phys.bx = s.phys.bx; d.phys.by = s.phys.by; d.phys.bz = s.phys.bz;
        d.phys.mx = s.phys.mx; d.phys.my = s.phys.my; d.phys.mz = s.phys.mz;
        d.phys.nx = s.phys.nx; d.phys.ny = s.phys.ny; d.phys.nz = s.phys.nz;
        d.phys.dS = s.phys.dS;
        d.vx = s.vx.data(); d.vy = s.vy.data(); d.vz = s.vz.data();
        d.n_vertices = (int32_t)s.vx.size();
        d.reserved = 0;
        d.cx = s.cx; d.cy = s.cy; d.cz = s.cz;
    }
    disco_atoms a;
    a.x = atoms.x; a.y = atoms.y; a.z = atoms.z;
    a.ux = atoms.ux; a.uy = atoms.uy; a.uz = atoms.uz;
    a.n = atoms.n;
    disco_options o;
    disco_b200_options_default(&o);
    o.precision = opt.fp32 ? DISCO_FP32C : DISCO_FP64;
    o.chunk_pairs = opt.chunkPairs;
    o.images = 1;
    o.nu = KROUPA_NU;
    o.verbose = 1;
    t.loopSec.assign(loops.size(), 0.);
    disco_timing tm;
    tm.upload = tm.kernels = tm.download = 0.;
    tm.loop_sec = t.loopSec.data();
    const double box[3] = { dx, dy, dz };
    if (disco_b200_displace(&a, L.data(), (int32_t)L.size(), box, &o, &tm) != DISCO_OK) die(__LINE__);
    t.upload = tm.upload;
    t.kernels = tm.kernels;
    t.download = tm.download;
}
