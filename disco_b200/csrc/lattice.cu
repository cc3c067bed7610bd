// Perfect-lattice sites on the device: Code/lattice.hpp:35-51 (generateLattice)
// without the host build and the host-to-device copy of the positions.  Same
// order (cells i, j, k with k fastest, then the basis sites) and the same
// arithmetic, each operation rounded as the host code rounds it
// ((i a0 + f a0) - L/2 with f a0 exact), so the sites are bit-identical.
#include <algorithm>
#include <string>

#include <cuda_runtime.h>

#include "common.cuh"
#include "../../include/disco_geometry.h"

namespace {

__constant__ double c_basis_bcc[2][3] = { { 0, 0, 0 }, { 0.5, 0.5, 0.5 } };
__constant__ double c_basis_fcc[4][3] = { { 0, 0, 0 }, { 0.5, 0.5, 0 }, { 0.5, 0, 0.5 }, { 0, 0.5, 0.5 } };

__global__ void lattice_kernel(int fcc, int nx, int ny, int nz, double a0, double hx, double hy, double hz,
                               double* __restrict__ x, double* __restrict__ y, double* __restrict__ z)
{
    const int nb = fcc ? 4 : 2;
    const int64_t total = (int64_t)nb * nx * ny * nz;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(q % nb);
        const int64_t cell = q / nb;
        const int k = (int)(cell % nz);
        const int64_t ij = cell / nz;
        const int j = (int)(ij % ny);
        const int i = (int)(ij / ny);
        const double* f = fcc ? c_basis_fcc[b] : c_basis_bcc[b];
        x[q] = __dsub_rn(__dadd_rn(__dmul_rn((double)i, a0), __dmul_rn(f[0], a0)), hx);
        y[q] = __dsub_rn(__dadd_rn(__dmul_rn((double)j, a0), __dmul_rn(f[1], a0)), hy);
        z[q] = __dsub_rn(__dadd_rn(__dmul_rn((double)k, a0), __dmul_rn(f[2], a0)), hz);
    }
}

} // namespace

extern "C" int disco_b200_lattice(int32_t lattice, int32_t nx, int32_t ny, int32_t nz, double a0, double* x,
                                  double* y, double* z, void* stream)
{
    if ((lattice != DISCO_LATTICE_BCC && lattice != DISCO_LATTICE_FCC) || nx < 0 || ny < 0 || nz < 0 ||
        !(a0 > 0.0)) {
        disco::set_last_error("lattice: bad argument");
        return DISCO_EINVAL;
    }
    const int nb = lattice == DISCO_LATTICE_FCC ? 4 : 2;
    const int64_t total = (int64_t)nb * nx * ny * nz;
    if (total == 0) return DISCO_OK;
    if (!x || !y || !z) {
        disco::set_last_error("lattice: null output array");
        return DISCO_EINVAL;
    }
    const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
    lattice_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        lattice == DISCO_LATTICE_FCC, nx, ny, nz, a0, nx * a0 / 2., ny * a0 / 2., nz * a0 / 2., x, y, z);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        disco::set_last_error(std::string("lattice: ") + cudaGetErrorString(e));
        return DISCO_ECUDA;
    }
    return DISCO_OK;
}
