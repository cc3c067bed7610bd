// =============================================================================
// ORACLE — test infrastructure only.  A thin extern "C" harness around the
// reference's OWN CUDA backend, Code/backend_cuda.cu, compiled where it lies
// for sm_100a by oracle/build_oracle.py into oracle/_ref/libdisco_ref_cuda.so.
// Nothing of the reference is copied: this file only marshals flat arrays
// into the reference's LoopData / AtomArrays / GpuOptions and calls
//
//   ref_kroupa_gpu   -> kroupaGPU   Code/backend_cuda.cu:568-722
//
// so that the reference's GPU kernels (line_kernel, line_kernel_f,
// kroupa_kernel[_tiled][_f], Code/backend_cuda.cu:63-373) can be timed on the
// same B200 as this library's.  Images +-1 and nu = 0.35 are fixed there.
// =============================================================================

#include <vector>

#include "backend.hpp"

#include "../include/disco_b200.h"

using std::vector;

extern "C" {

int ref_gpu_available(void) { return gpuAvailable() ? 1 : 0; }

// kroupaGPU on flat arrays.  timing[0..2] = upload, kernels, download (s),
// as the reference measures them (host clock, a device wait after each loop).
int ref_kroupa_gpu(const disco_atoms* atoms, const disco_loop* loops, int nloops,
                   const double box[3], int fp32, double* timing)
{
    vector<LoopData> ld((size_t)nloops);
    for (int l = 0; l < nloops; l++) {
        const disco_loop& s = loops[l];
        LoopData& d = ld[l];
        d.x.assign(s.x, s.x + (s.n_loopons > 0 ? s.n_loopons : 0));
        d.y.assign(s.y, s.y + (s.n_loopons > 0 ? s.n_loopons : 0));
        d.z.assign(s.z, s.z + (s.n_loopons > 0 ? s.n_loopons : 0));
        d.phys = { s.phys.bx, s.phys.by, s.phys.bz, s.phys.mx, s.phys.my, s.phys.mz,
                   s.phys.nx, s.phys.ny, s.phys.nz, s.phys.dS };
        d.line = s.line != 0;
        if (d.line) {
            d.vx.assign(s.vx, s.vx + s.n_vertices);
            d.vy.assign(s.vy, s.vy + s.n_vertices);
            d.vz.assign(s.vz, s.vz + s.n_vertices);
            d.cx = s.cx; d.cy = s.cy; d.cz = s.cz;
        }
    }
    const AtomArrays a = { atoms->x, atoms->y, atoms->z, atoms->ux, atoms->uy, atoms->uz,
                           (int)atoms->n };
    GpuOptions opt;
    opt.fp32 = fp32 != 0;
    BackendTiming t;
    kroupaGPU(a, ld, box[0], box[1], box[2], opt, t);
    if (timing) { timing[0] = t.upload; timing[1] = t.kernels; timing[2] = t.download; }
    return 0;
}

} // extern "C"
