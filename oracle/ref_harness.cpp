// =============================================================================
// ORACLE — test infrastructure only.  A thin extern "C" harness around the
// reference's OWN sources, compiled where they lie (include path
// <reference>/Code, sources backend_cpu.cpp, loop.cpp, prismatic.cpp) by
// oracle/build_oracle.py into oracle/_ref/libdisco_ref.so.  Nothing of the
// reference is copied here: these functions only marshal flat arrays into the
// reference's types and call its functions.
//
//   ref_kroupa_cpu        -> kroupaCPU           Code/backend_cpu.cpp:28-99
//   ref_loop_*            -> class loop          Code/loop.hpp:15-117
//   ref_snap              -> snapToMidPlane      Code/loop.cpp:342-374
//   ref_regular_polygon   -> regularPolygon      Code/loop.cpp:585-608
//   ref_lattice           -> generateLattice     Code/lattice.hpp:35-51
//   ref_prismatic_step    -> prismaticSlab (Code/prismatic.cpp:36-74) driven as
//                            Code/main.cpp:586-687 drives it; that driver code is
//                            inline in main() and cannot be called, so its steps
//                            (removed flags, copies with side*b or the Frank
//                            shift, stable compaction, remap) are restated here.
// =============================================================================

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "backend.hpp"
#include "barnett.hpp"
#include "lattice.hpp"
#include "loop.hpp"
#include "prismatic.hpp"

#include "../include/disco_b200.h"

using std::vector;

extern "C" {

int ref_threads(void) { return cpuThreads(); }

// barnettLoop<double> (Code/barnett.hpp:44-107) at one point, added to u[3]
void ref_barnett_loop(double px, double py, double pz, const double* vx, const double* vy,
                      const double* vz, int nv, double cx, double cy, double cz, double bx,
                      double by, double bz, double* u)
{
    barnettLoop<double>(px, py, pz, vx, vy, vz, nv, cx, cy, cz, bx, by, bz, u[0], u[1], u[2]);
}

// kroupaPair (Code/kroupa.hpp:75-80) for one separation, added to du[3]
void ref_kroupa_pair(double rx, double ry, double rz, const disco_loop_phys* P, double* du)
{
    const LoopPhys L = { P->bx, P->by, P->bz, P->mx, P->my, P->mz, P->nx, P->ny, P->nz, P->dS };
    const double b_n = L.mx*L.nx + L.my*L.ny + L.mz*L.nz;
    kroupaPair(rx, ry, rz, L, kroupaK1(), b_n, du[0], du[1], du[2]);
}

// kroupaCPU on flat arrays (images +-1, nu = 0.35: both fixed in the reference).
int ref_kroupa_cpu(const disco_atoms* atoms, const disco_loop* loops, int nloops,
                   const double box[3], double* loop_sec)
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
    BackendTiming t;
    kroupaCPU(a, ld, box[0], box[1], box[2], t);
    if (loop_sec)
        for (int l = 0; l < nloops; l++) loop_sec[l] = t.loopSec[l];
    return 0;
}

// shape: 0 circle, 1 rectangle, 2 parallelogram, 3 polygon (explicit vertices)
void* ref_loop_new(int shape, double da, double radius, double half_m, double half_p,
                   double corner_r, const double* center, const double* m, const double* n,
                   double a0, const double* side, const double* verts, int nverts,
                   const double* dir1, const double* dir2)
{
    const vector<double> c(center, center + 3), mm(m, m + 3), nn(n, n + 3);
    const vector<double> compress = { 1., 1., 1. };
    vector<double> sd;
    if (side) sd.assign(side, side + 3);
    switch (shape) {
        case 0: return new loop(da, radius, c, mm, nn, a0, compress);
        case 1: return new loop(da, half_m, half_p, corner_r, c, mm, nn, a0, compress, sd);
        case 2: return new loop(da, half_m, half_p, vector<double>(dir1, dir1 + 3),
                                vector<double>(dir2, dir2 + 3), c, mm, nn, a0, compress);
        default: {
            vector<vector<double>> v;
            for (int i = 0; i < nverts; i++) v.push_back({ verts[3*i], verts[3*i+1], verts[3*i+2] });
            return new loop(da, v, corner_r, c, mm, nn, a0, compress, sd);
        }
    }
}

void ref_loop_free(void* h) { delete static_cast<loop*>(h); }

int ref_loop_polyline(void* h, double eps, double* out, int cap)
{
    const vector<vector<double>> P = static_cast<loop*>(h)->polyline(eps);
    const int np = (int)P.size();
    for (int k = 0; k < np && k < cap; k++)
        for (int i = 0; i < 3; i++) out[3*k + i] = P[k][i];
    return np;
}

// generateSurface + generateLoopons (Code/main.cpp:515-516), then the positions
int ref_loop_loopons(void* h, double* out, int cap, double* dS)
{
    loop* lp = static_cast<loop*>(h);
    lp->generateSurface();
    if (lp->getNumberOfLoopons() == 0) lp->generateLoopons();
    const int np = lp->getNumberOfLoopons();
    for (int k = 0; k < np && k < cap; k++) {
        const vector<double> q = lp->getOneLoopon(k);
        for (int i = 0; i < 3; i++) out[3*k + i] = q[i];
    }
    *dS = lp->getSurface();
    return np;
}

// centre, m, n, |b| per axis, contour area
void ref_loop_info(void* h, double* out)
{
    const loop* lp = static_cast<loop*>(h);
    const vector<double> c = lp->getCenter(), m = lp->getM(), n = lp->getN(), b = lp->getBurgers();
    for (int i = 0; i < 3; i++) { out[i] = c[i]; out[3+i] = m[i]; out[6+i] = n[i]; out[9+i] = b[i]; }
    out[12] = lp->getContourArea();
    out[13] = lp->getCornerRadius();
}

int ref_loop_contains(void* h, const double* rel)
{
    return static_cast<loop*>(h)->contains(rel) ? 1 : 0;
}

void ref_snap(const double* center, const double* n, double a0, int nx, int ny, int nz,
              int lattice, double* out, double* spacing)
{
    const vector<double> r = snapToMidPlane(vector<double>(center, center + 3),
                                            vector<double>(n, n + 3), a0, nx, ny, nz, *spacing,
                                            lattice == 1 ? Lattice::FCC : Lattice::BCC);
    for (int i = 0; i < 3; i++) out[i] = r[i];
}

void ref_regular_polygon(int sides, double R, const double* vertexDir, const double* m,
                         const double* n, double* out)
{
    vector<double> vd;
    if (vertexDir) vd.assign(vertexDir, vertexDir + 3);
    const vector<vector<double>> v = regularPolygon(sides, R, vd, vector<double>(m, m + 3),
                                                    vector<double>(n, n + 3));
    for (int k = 0; k < sides; k++)
        for (int i = 0; i < 3; i++) out[3*k + i] = v[k][i];
}

int64_t ref_lattice(int lattice, int nx, int ny, int nz, double a0, double* x, double* y, double* z)
{
    const vector<vector<double>> a = generateLattice(lattice == 1 ? Lattice::FCC : Lattice::BCC,
                                                     nx, ny, nz, a0);
    for (size_t i = 0; i < a.size(); i++) { x[i] = a[i][0]; y[i] = a[i][1]; z[i] = a[i][2]; }
    return (int64_t)a.size();
}

// Matter step of Code/main.cpp:586-687 over reference loop objects.  frank[l]:
// the loop is an FCC Frank loop (its copies get frankCopyShift, main.cpp:636-644;
// box axes = crystal axes).  Outputs as disco_b200_prismatic.
int ref_prismatic_step(void* const* handles, const double* spacing, const int* apply,
                       const int* frank, double a0, int nloops,
                       const double* x, const double* y, const double* z, int64_t n,
                       const double box[3],
                       double* x_out, double* y_out, double* z_out, int32_t* new_index,
                       disco_slab_info* info, int32_t* slab_atoms, int8_t* slab_side,
                       int64_t slab_capacity, disco_copy* copies, int64_t copy_capacity,
                       int64_t counts[3])
{
    const vector<double> X(x, x + n), Y(y, y + n), Z(z, z + n);
    vector<char> removed((size_t)n, 0);
    vector<disco_copy> cps;
    int64_t total = 0;
    for (int l = 0; l < nloops; l++) {
        const loop& lp = *static_cast<const loop*>(handles[l]);
        disco_slab_info inf;
        std::memset(&inf, 0, sizeof(inf));
        inf.offset = total;
        if (matterType(lp) == MatterType::NONE || !apply[l]) { info[l] = inf; continue; }
        const SlabResult sl = prismaticSlab(lp, spacing[l], X, Y, Z, box[0], box[1], box[2]);
        inf.type = sl.type == MatterType::VACANCY ? DISCO_MATTER_VACANCY : DISCO_MATTER_INTERSTITIAL;
        inf.planes = sl.planes; inf.height = sl.height; inf.spacing = sl.spacing;
        for (int i = 0; i < 3; i++) inf.b[i] = sl.b[i];
        inf.count = (int64_t)sl.atoms.size();
        info[l] = inf;
        for (size_t q = 0; q < sl.atoms.size(); q++) {
            if (total + (int64_t)q < slab_capacity) {
                slab_atoms[total + q] = sl.atoms[q];
                slab_side[total + q] = (int8_t)sl.side[q];
            }
        }
        total += (int64_t)sl.atoms.size();
        if (sl.type == MatterType::VACANCY) {
            for (int a : sl.atoms) removed[a] = 1;
        } else {
            double shift[2][3];
            for (int sd = 0; sd < 2; sd++) {
                const double sign = sd == 0 ? 1. : -1.;
                const double v[3] = { sign*sl.b[0], sign*sl.b[1], sign*sl.b[2] };
                if (frank[l]) {
                    const vector<double> nv = lp.getN();
                    const double nhat[3] = { nv[0], nv[1], nv[2] };
                    frankCopyShift(v, nhat, a0, shift[sd]);
                } else {
                    for (int c = 0; c < 3; c++) shift[sd][c] = v[c];
                }
            }
            for (size_t k = 0; k < sl.atoms.size(); k++) {
                const double* sh = shift[sl.side[k] > 0 ? 0 : 1];
                disco_copy c;
                c.atom = sl.atoms[k]; c.reserved = 0;
                c.shift[0] = sh[0]; c.shift[1] = sh[1]; c.shift[2] = sh[2];
                cps.push_back(c);
            }
        }
    }
    int64_t k = 0;
    for (int64_t a = 0; a < n; a++) {
        if (removed[a]) { new_index[a] = -1; continue; }
        new_index[a] = (int32_t)k;
        x_out[k] = x[a]; y_out[k] = y[a]; z_out[k] = z[a];
        k++;
    }
    int64_t nc = 0;
    for (disco_copy c : cps)
        if (new_index[c.atom] >= 0) {
            c.atom = new_index[c.atom];
            if (nc < copy_capacity) copies[nc] = c;
            nc++;
        }
    counts[0] = k; counts[1] = total; counts[2] = nc;
    return (total > slab_capacity || nc > copy_capacity) ? DISCO_ELIMIT : DISCO_OK;
}

// classifyBurgers (Code/lattice.hpp:189-213): 0 perfect, 1 Frank, 2 Shockley, 3 other
int ref_classify_burgers(int lattice, const double* m, const double* n)
{
    return (int)classifyBurgers(lattice == 1 ? Lattice::FCC : Lattice::BCC,
                                vector<double>(m, m + 3), vector<double>(n, n + 3));
}

double ref_plane_spacing(int lattice, const long* h, double a0)
{
    return latticePlaneSpacing(lattice == 1 ? Lattice::FCC : Lattice::BCC, h, a0);
}

} // extern "C"
