// =============================================================================
// ORACLE — test infrastructure only, never shipped and never on the product path.
//
// A CPU restatement of DISCO's displacement hot path, written operation for
// operation after the reference so that it can be compared bit for bit with the
// reference where the reference can run (nu = 0.35, images +-1), and used as the
// checker where it cannot (any nu, any image range).  Only tests/, the smoke
// check of __graft_entry__.py and bench.py's CPU-baseline leg load it.
//
//   oracle_barnett_loop   Code/barnett.hpp:44-107   (nu a parameter)
//   oracle_kroupa_pair    Code/kroupa.hpp:52-73     (nu a parameter)
//   oracle_displace       Code/backend_cpu.cpp:28-99 (images, nu parameters)
//   oracle_prismatic      Code/prismatic.cpp:13-19,31-74 + Code/loop.cpp:281-330
//                         + Code/main.cpp:586-687 (slabs, removal, copies)
//   oracle_finalize       Code/main.cpp:733-743 and 797-818
//
// Built twice by oracle/build_oracle.py: with the reference's own flags
// (-O3 -fopenmp, FMA contraction left to the compiler as in Code/Makefile:66)
// and with -ffp-contract=off, the build the atom-set comparisons use.
// =============================================================================

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>
#include <omp.h>

#include "../include/disco_b200.h"

namespace {

const double kPi = 3.14159265358979323846;

// Code/barnett.hpp:44-107.  Same statements in the same order; the constants
// c3 and cJ are built from nu at run time with the same operations the
// reference folds at compile time (Code/barnett.hpp:50-53).
inline void barnett_loop(double px, double py, double pz,
                         const double* vx, const double* vy, const double* vz, int nv,
                         double cx, double cy, double cz, double bx, double by, double bz,
                         double c3, double cJ, double cK,
                         double& ux, double& uy, double& uz)
{
    const double PI = kPi;
    const double r1x = cx - px, r1y = cy - py, r1z = cz - pz;
    const double l1  = sqrt(r1x*r1x + r1y*r1y + r1z*r1z);

    double omega = 0.0;
    double lx = 0.0, ly = 0.0, lz = 0.0;

    double ax = vx[nv-1] - px, ay = vy[nv-1] - py, az = vz[nv-1] - pz;
    double la = sqrt(ax*ax + ay*ay + az*az);
    for (int k = 0; k < nv; k++) {
        const double bxp = vx[k] - px, byp = vy[k] - py, bzp = vz[k] - pz;
        const double lb  = sqrt(bxp*bxp + byp*byp + bzp*bzp);

        const double num = r1x*(ay*bzp - az*byp) + r1y*(az*bxp - ax*bzp) + r1z*(ax*byp - ay*bxp);
        const double den = l1*la*lb + (r1x*ax + r1y*ay + r1z*az)*lb
                         + (r1x*bxp + r1y*byp + r1z*bzp)*la + (ax*bxp + ay*byp + az*bzp)*l1;
        omega += 2.0 * atan2(num, den);

        double tx = bxp - ax, ty = byp - ay, tz = bzp - az;
        const double L = sqrt(tx*tx + ty*ty + tz*tz);
        if (L > 0.0) {
            tx /= L; ty /= L; tz /= L;
            const double sA = ax*tx + ay*ty + az*tz;
            const double sB = sA + L;
            const double dx = ax - sA*tx, dy = ay - sA*ty, dz = az - sA*tz;
            const double d2 = dx*dx + dy*dy + dz*dz;
            const double RA = la, RB = lb;
            const double fA = sA >= 0.0 ? RA + sA : d2 / (RA - sA);
            const double fB = sB >= 0.0 ? RB + sB : d2 / (RB - sB);
            const double J0 = log(fB / fA);
            double K0;
            if (sA >= 0.0)      K0 = 1.0 / (RA*(RA + sA)) - 1.0 / (RB*(RB + sB));
            else if (sB <= 0.0) K0 = 1.0 / (RB*(RB - sB)) - 1.0 / (RA*(RA - sA));
            else                K0 = (sB/RB - sA/RA) / d2;
            const double K1 = 1.0 / RA - 1.0 / RB;
            const double wx = by*tz - bz*ty, wy = bz*tx - bx*tz, wz = bx*ty - by*tx;
            const double dw = dx*wx + dy*wy + dz*wz;
            lx += wx*J0*cJ - cK*dw*(dx*K0 + tx*K1);
            ly += wy*J0*cJ - cK*dw*(dy*K0 + ty*K1);
            lz += wz*J0*cJ - cK*dw*(dz*K0 + tz*K1);
        }
        ax = bxp; ay = byp; az = bzp; la = lb;
    }
    const double fo = omega / (4.0 * PI);
    ux += bx*fo + lx;
    uy += by*fo + ly;
    uz += bz*fo + lz;
}

// Code/kroupa.hpp:52-73 with (1 - 2 nu) a parameter c2.
inline void kroupa_pair(double rho_x, double rho_y, double rho_z, const disco_loop_phys& L,
                        double k1, double b_n, double c2,
                        double& dux, double& duy, double& duz)
{
    const double rho2 = rho_x*rho_x + rho_y*rho_y + rho_z*rho_z;
    const double rho0 = sqrt(rho2);
    const bool keep = !(rho0 < 1e-10);
    const double rho  = keep ? rho0 : 1.0;
    const double r2   = keep ? rho2 : 1.0;
    const double rho3 = r2 * rho;

    const double b_rho = L.mx*rho_x + L.my*rho_y + L.mz*rho_z;
    const double n_rho = L.nx*rho_x + L.ny*rho_y + L.nz*rho_z;
    const double k2    = c2 / rho;
    const double fac   = keep ? -k1 * L.dS / r2 : 0.0;
    const double tail  = 3.0 * b_rho * n_rho / rho3;

    dux += fac * L.bx * (k2*(L.nx*b_rho + L.mx*n_rho - rho_x*b_n) + tail*rho_x);
    duy += fac * L.by * (k2*(L.ny*b_rho + L.my*n_rho - rho_y*b_n) + tail*rho_y);
    duz += fac * L.bz * (k2*(L.nz*b_rho + L.mz*n_rho - rho_z*b_n) + tail*rho_z);
}

// ---- slab predicate (FP64, operation order of the reference) -----------------

// Code/prismatic.cpp:31-34
inline double min_image(double r, double L) { return r - L * floor(r / L + 0.5); }

// Code/loop.cpp:281-316
bool inside_uv(const disco_slab_loop& lp, double u, double v)
{
    const double eps = 1e-9;
    if (lp.shape == DISCO_SHAPE_CIRCLE)
        return sqrt(u*u + v*v) < lp.radius - eps;
    if (lp.shape == DISCO_SHAPE_POLYGON) {
        const int N = lp.n_poly;
        bool inQ = true;
        for (int i = 0; i < N && inQ; i++)
            if (lp.nu[i]*(u - lp.pu[i]) + lp.nv[i]*(v - lp.pv[i]) < lp.r_corner - eps) inQ = false;
        if (inQ) return true;
        if (lp.r_corner <= 0.) return false;
        double d2 = 1e300;
        for (int i = 0; i < N; i++) {
            const int j = (i + 1) % N;
            const double eu = lp.qu[j] - lp.qu[i], ev = lp.qv[j] - lp.qv[i];
            const double l2 = eu*eu + ev*ev;
            double t = l2 > 0. ? ((u - lp.qu[i])*eu + (v - lp.qv[i])*ev) / l2 : 0.;
            t = fmin(fmax(t, 0.), 1.);
            const double wu = u - lp.qu[i] - t*eu, wv = v - lp.qv[i] - t*ev;
            d2 = fmin(d2, wu*wu + wv*wv);
        }
        return d2 <= lp.r_corner*lp.r_corner + eps;
    }
    const double du = fmax(fabs(u) - fmax(lp.half_m - lp.r_corner, 0.0), 0.0);
    const double dv = fmax(fabs(v) - fmax(lp.half_p - lp.r_corner, 0.0), 0.0);
    return du*du + dv*dv <= lp.r_corner*lp.r_corner + eps;
}

// Code/loop.cpp:323-330
bool contains(const disco_slab_loop& lp, const double rel[3])
{
    const double ru = rel[0]*lp.u[0] + rel[1]*lp.u[1] + rel[2]*lp.u[2];
    const double rv = rel[0]*lp.v[0] + rel[1]*lp.v[1] + rel[2]*lp.v[2];
    const double c = lp.u[0]*lp.v[0] + lp.u[1]*lp.v[1] + lp.u[2]*lp.v[2];
    const double det = 1.0 - c*c;
    return inside_uv(lp, (ru - c*rv) / det, (rv - c*ru) / det);
}

// Code/prismatic.cpp:13-19
int matter_type(const disco_slab_loop& lp)
{
    const double mn = lp.m[0]*lp.n[0] + lp.m[1]*lp.n[1] + lp.m[2]*lp.n[2];
    if (fabs(mn) < 1e-6) return DISCO_MATTER_NONE;
    return mn > 0. ? DISCO_MATTER_VACANCY : DISCO_MATTER_INTERSTITIAL;
}

} // namespace

extern "C" {

int oracle_threads(void) { return omp_get_max_threads(); }

void oracle_barnett_loop(double px, double py, double pz,
                         const double* vx, const double* vy, const double* vz, int nv,
                         double cx, double cy, double cz, double bx, double by, double bz,
                         double nu, double* u)
{
    const double c3 = 1.0 / (8.0 * kPi * (1.0 - nu));
    const double cJ = c3 - 1.0 / (4.0 * kPi);
    barnett_loop(px, py, pz, vx, vy, vz, nv, cx, cy, cz, bx, by, bz, c3, cJ, c3, u[0], u[1], u[2]);
}

void oracle_kroupa_pair(double rx, double ry, double rz, const disco_loop_phys* L,
                        double nu, double* du)
{
    const double k1 = 1.0 / (8.0 * M_PI * (1.0 - nu));       // Code/kroupa.hpp:38-41
    const double b_n = L->mx*L->nx + L->my*L->ny + L->mz*L->nz;
    kroupa_pair(rx, ry, rz, *L, k1, b_n, 1.0 - 2.0*nu, du[0], du[1], du[2]);
}

// Code/backend_cpu.cpp:28-99: loop by loop; per loop an OpenMP loop over atoms,
// images ii, jj, kk in -images..images (kk fastest), each loop's partial added
// to the atom.  threads <= 0 keeps the OpenMP default.  Images with
// max(|ii|,|jj|,|kk|) < image_min are skipped (image_min 0: the reference's sum).
int oracle_displace_shells(const disco_atoms* atoms, const disco_loop* loops, int nloops,
                           const double box[3], int images, int image_min, double nu, int threads,
                           double* loop_sec)
{
    if (threads > 0) omp_set_num_threads(threads);
    const int64_t nbAtoms = atoms->n;
    const double dx = box[0], dy = box[1], dz = box[2];
    const double c3 = 1.0 / (8.0 * kPi * (1.0 - nu));
    const double cJ = c3 - 1.0 / (4.0 * kPi);
    const double k1 = 1.0 / (8.0 * M_PI * (1.0 - nu));
    const double c2 = 1.0 - 2.0*nu;
    const int I = images;
    // The reference's chunk of 256 atoms; smaller on samples too small to give
    // every thread a chunk (scheduling only: the arithmetic per atom is fixed).
    const int nthr = omp_get_max_threads();
    const int chunk = nbAtoms >= (int64_t)256 * 4 * nthr ? 256
                    : (int)std::max<int64_t>(1, nbAtoms / (4 * (int64_t)nthr));
    for (int l = 0; l < nloops; l++) {
        const disco_loop& lp = loops[l];
        const double t0 = omp_get_wtime();
        if (lp.line) {
            const int nv = lp.n_vertices;
            const double bx = lp.phys.bx * lp.phys.mx, by = lp.phys.by * lp.phys.my,
                         bz = lp.phys.bz * lp.phys.mz;
#pragma omp parallel for schedule(dynamic, chunk)
            for (int64_t a = 0; a < nbAtoms; a++) {
                double dux = 0., duy = 0., duz = 0.;
                for (int ii = -I; ii <= I; ii++)
                for (int jj = -I; jj <= I; jj++)
                for (int kk = -I; kk <= I; kk++)
                    if (std::max(std::abs(ii), std::max(std::abs(jj), std::abs(kk))) >= image_min)
                    barnett_loop(atoms->x[a] - dx*ii, atoms->y[a] - dy*jj, atoms->z[a] - dz*kk,
                                 lp.vx, lp.vy, lp.vz, nv, lp.cx, lp.cy, lp.cz, bx, by, bz,
                                 c3, cJ, c3, dux, duy, duz);
                atoms->ux[a] += dux;
                atoms->uy[a] += duy;
                atoms->uz[a] += duz;
            }
        } else {
            const disco_loop_phys L = lp.phys;
            const int nLp = lp.n_loopons;
            const double* lx = lp.x;
            const double* ly = lp.y;
            const double* lz = lp.z;
            const double b_n = L.mx*L.nx + L.my*L.ny + L.mz*L.nz;
#pragma omp parallel for schedule(dynamic, chunk)
            for (int64_t a = 0; a < nbAtoms; a++) {
                const double ax = atoms->x[a], ay = atoms->y[a], az = atoms->z[a];
                double dux = 0., duy = 0., duz = 0.;
                for (int ii = -I; ii <= I; ii++) {
                for (int jj = -I; jj <= I; jj++) {
                for (int kk = -I; kk <= I; kk++) {
                    if (std::max(std::abs(ii), std::max(std::abs(jj), std::abs(kk))) < image_min) continue;
                    const double delta_x = dx * ii;
                    const double delta_y = dy * jj;
                    const double delta_z = dz * kk;
#pragma omp simd reduction(+:dux,duy,duz)
                    for (int p = 0; p < nLp; p++)
                        kroupa_pair(ax - (lx[p] + delta_x), ay - (ly[p] + delta_y), az - (lz[p] + delta_z),
                                    L, k1, b_n, c2, dux, duy, duz);
                }}}
                atoms->ux[a] += dux;
                atoms->uy[a] += duy;
                atoms->uz[a] += duz;
            }
        }
        if (loop_sec) loop_sec[l] = omp_get_wtime() - t0;
    }
    return DISCO_OK;
}

int oracle_displace(const disco_atoms* atoms, const disco_loop* loops, int nloops,
                    const double box[3], int images, double nu, int threads, double* loop_sec)
{
    return oracle_displace_shells(atoms, loops, nloops, box, images, 0, nu, threads, loop_sec);
}

// One slab (Code/prismatic.cpp:36-74): fills info and appends atoms/side.
static int slab_of(const disco_slab_loop& lp, const double* x, const double* y, const double* z,
                   int64_t n, const double box[3], disco_slab_info& info,
                   std::vector<int32_t>& atoms, std::vector<int8_t>& side)
{
    std::memset(&info, 0, sizeof(info));
    info.type = matter_type(lp);
    if (info.type == DISCO_MATTER_NONE) return DISCO_OK;
    for (int i = 0; i < 3; i++) info.b[i] = lp.bmag * lp.m[i];
    info.height  = fabs(info.b[0]*lp.n[0] + info.b[1]*lp.n[1] + info.b[2]*lp.n[2]);
    info.spacing = lp.spacing;
    const double ratio = info.height / lp.spacing;
    info.planes = (int)lround(ratio);
    if (info.planes < 1 || fabs(ratio - info.planes) > 1e-6) return DISCO_EPLANES;
    const double tLo = -floor(info.planes / 2.);
    const double tHi =  ceil(info.planes / 2.);
    for (int64_t a = 0; a < n; a++) {
        const double rel[3] = { min_image(x[a] - lp.c[0], box[0]),
                                min_image(y[a] - lp.c[1], box[1]),
                                min_image(z[a] - lp.c[2], box[2]) };
        const double s = rel[0]*lp.n[0] + rel[1]*lp.n[1] + rel[2]*lp.n[2];
        const double t = s / lp.spacing;
        if (t < tLo || t >= tHi) continue;
        if (!contains(lp, rel)) continue;
        atoms.push_back((int32_t)a);
        side.push_back(s > 0. ? 1 : -1);
    }
    return DISCO_OK;
}

// Code/main.cpp:586-687 (without the polycrystal / twin grain filter): slabs on
// the perfect lattice, vacancy slabs removed, interstitial slabs copied with the
// shift of their side, survivors compacted in order, copies of removed atoms
// dropped and the others renumbered.  Same signature as disco_b200_prismatic.
int oracle_prismatic(const double* x, const double* y, const double* z, int64_t n,
                     const disco_slab_loop* loops, int32_t nloops, const double box[3],
                     double* x_out, double* y_out, double* z_out, int32_t* new_index,
                     disco_slab_info* info,
                     int32_t* slab_atoms, int8_t* slab_side, int64_t slab_capacity,
                     disco_copy* copies, int64_t copy_capacity, int64_t counts[3])
{
    std::vector<char> removed((size_t)n, 0);
    std::vector<int32_t> all_atoms;
    std::vector<int8_t> all_side;
    std::vector<disco_copy> cps;
    for (int l = 0; l < nloops; l++) {
        const disco_slab_loop& lp = loops[l];
        std::vector<int32_t> at;
        std::vector<int8_t> sd;
        disco_slab_info inf;
        std::memset(&inf, 0, sizeof(inf));
        if (lp.apply && matter_type(lp) != DISCO_MATTER_NONE) {
            const int st = slab_of(lp, x, y, z, n, box, inf, at, sd);
            if (st != DISCO_OK) return st;
        } else {
            inf.type = DISCO_MATTER_NONE;
        }
        inf.offset = (int64_t)all_atoms.size();
        inf.count = (int64_t)at.size();
        info[l] = inf;
        if (inf.type == DISCO_MATTER_VACANCY) {
            for (int32_t a : at) removed[a] = 1;
        } else if (inf.type == DISCO_MATTER_INTERSTITIAL) {
            for (size_t k = 0; k < at.size(); k++) {
                const double* sh = sd[k] > 0 ? lp.shift_pos : lp.shift_neg;
                disco_copy c;
                c.atom = at[k]; c.reserved = 0;
                c.shift[0] = sh[0]; c.shift[1] = sh[1]; c.shift[2] = sh[2];
                cps.push_back(c);
            }
        }
        all_atoms.insert(all_atoms.end(), at.begin(), at.end());
        all_side.insert(all_side.end(), sd.begin(), sd.end());
    }
    int64_t k = 0;
    for (int64_t a = 0; a < n; a++) {
        if (removed[a]) { new_index[a] = -1; continue; }
        new_index[a] = (int32_t)k;
        x_out[k] = x[a]; y_out[k] = y[a]; z_out[k] = z[a];
        k++;
    }
    std::vector<disco_copy> kept;
    for (disco_copy c : cps)
        if (new_index[c.atom] >= 0) { c.atom = new_index[c.atom]; kept.push_back(c); }
    counts[0] = k;
    counts[1] = (int64_t)all_atoms.size();
    counts[2] = (int64_t)kept.size();
    if (counts[1] > slab_capacity || counts[2] > copy_capacity) return DISCO_ELIMIT;
    for (size_t i = 0; i < all_atoms.size(); i++) { slab_atoms[i] = all_atoms[i]; slab_side[i] = all_side[i]; }
    for (size_t i = 0; i < kept.size(); i++) copies[i] = kept[i];
    return DISCO_OK;
}

// Code/main.cpp:733-743 (copies appended with u(src) + shift) and 797-818
// (r = x + u, one fold into [-L/2, L/2], shift by +L/2; U = I).
int oracle_finalize(const double* x, const double* y, const double* z,
                    const double* ux, const double* uy, const double* uz, int64_t n,
                    const disco_copy* copies, int64_t ncopies, const double box[3],
                    double* fx, double* fy, double* fz,
                    double* ux_out, double* uy_out, double* uz_out)
{
    const double dx = box[0], dy = box[1], dz = box[2];
    const double dx2 = dx/2., dy2 = dy/2., dz2 = dz/2.;
    for (int64_t k = 0; k < n + ncopies; k++) {
        double px, py, pz, qx, qy, qz;
        if (k < n) {
            px = x[k]; py = y[k]; pz = z[k]; qx = ux[k]; qy = uy[k]; qz = uz[k];
        } else {
            const disco_copy& c = copies[k - n];
            px = x[c.atom]; py = y[c.atom]; pz = z[c.atom];
            qx = ux[c.atom] + c.shift[0]; qy = uy[c.atom] + c.shift[1]; qz = uz[c.atom] + c.shift[2];
        }
        double rx = px + qx, ry = py + qy, rz = pz + qz;
        if      (rx >  dx2) rx -= dx;  else if (rx < -dx2) rx += dx;
        if      (ry >  dy2) ry -= dy;  else if (ry < -dy2) ry += dy;
        if      (rz >  dz2) rz -= dz;  else if (rz < -dz2) rz += dz;
        fx[k] = rx + dx2; fy[k] = ry + dy2; fz[k] = rz + dz2;
        if (ux_out) { ux_out[k] = qx; uy_out[k] = qy; uz_out[k] = qz; }
    }
    return DISCO_OK;
}

// Smallest distance, over all atoms and slab loops, of each of the reference's
// FP64 slab comparisons from its threshold: |t - tLo|, |t - tHi| for atoms whose
// in-plane test decides, and the in-plane margin (circle: |sqrt(u^2+v^2) - (R -
// eps)|; other shapes: the distance of the final comparison).  A margin far
// above the rounding of the predicate means no FMA contraction difference can
// change the atom sets.  Writes {min slab margin, min in-plane margin}.
int oracle_slab_margins(const double* x, const double* y, const double* z, int64_t n,
                        const disco_slab_loop* loops, int32_t nloops, const double box[3],
                        double out[2])
{
    double mt = 1e300, mc = 1e300;
    for (int l = 0; l < nloops; l++) {
        const disco_slab_loop& lp = loops[l];
        if (!lp.apply || matter_type(lp) == DISCO_MATTER_NONE) continue;
        const double b[3] = { lp.bmag*lp.m[0], lp.bmag*lp.m[1], lp.bmag*lp.m[2] };
        const double height = fabs(b[0]*lp.n[0] + b[1]*lp.n[1] + b[2]*lp.n[2]);
        const int planes = (int)lround(height / lp.spacing);
        const double tLo = -floor(planes / 2.), tHi = ceil(planes / 2.);
        for (int64_t a = 0; a < n; a++) {
            const double rel[3] = { min_image(x[a] - lp.c[0], box[0]),
                                    min_image(y[a] - lp.c[1], box[1]),
                                    min_image(z[a] - lp.c[2], box[2]) };
            const double s = rel[0]*lp.n[0] + rel[1]*lp.n[1] + rel[2]*lp.n[2];
            const double t = s / lp.spacing;
            mt = fmin(mt, fmin(fabs(t - tLo), fabs(t - tHi)));
            if (t < tLo || t >= tHi) continue;
            const double ru = rel[0]*lp.u[0] + rel[1]*lp.u[1] + rel[2]*lp.u[2];
            const double rv = rel[0]*lp.v[0] + rel[1]*lp.v[1] + rel[2]*lp.v[2];
            const double c = lp.u[0]*lp.v[0] + lp.u[1]*lp.v[1] + lp.u[2]*lp.v[2];
            const double det = 1.0 - c*c;
            const double uu = (ru - c*rv) / det, vv = (rv - c*ru) / det;
            double m;
            if (lp.shape == DISCO_SHAPE_CIRCLE) {
                m = fabs(sqrt(uu*uu + vv*vv) - (lp.radius - 1e-9));
            } else if (lp.shape == DISCO_SHAPE_POLYGON) {
                m = 1e300;
                for (int i = 0; i < lp.n_poly; i++)
                    m = fmin(m, fabs(lp.nu[i]*(uu - lp.pu[i]) + lp.nv[i]*(vv - lp.pv[i])
                                     - (lp.r_corner - 1e-9)));
            } else {
                const double du = fmax(fabs(uu) - fmax(lp.half_m - lp.r_corner, 0.0), 0.0);
                const double dv = fmax(fabs(vv) - fmax(lp.half_p - lp.r_corner, 0.0), 0.0);
                m = fabs(du*du + dv*dv - (lp.r_corner*lp.r_corner + 1e-9));
            }
            mc = fmin(mc, m);
        }
    }
    out[0] = mt; out[1] = mc;
    return DISCO_OK;
}

} // extern "C"

// The atom lines of the reference's writers, through the same C++ stream
// formatting: XYZ (format 0, Code/main.cpp:826-831) and LAMMPS atomic
// (format 1, Code/main.cpp:86-92, with e1, e2, e3 the unit axes of an
// orthorhombic box).  Returns the byte count; writes at most cap bytes.
extern "C" int64_t oracle_format_atoms(int format, const char* element, const double* x, const double* y, const double* z,
                            int64_t n, char* out, int64_t cap)
{
    std::ostringstream os;
    os << std::fixed << std::setprecision(8);
    const double e1[3] = { 1., 0., 0. }, e2[3] = { 0., 1., 0. }, e3[3] = { 0., 0., 1. };
    for (int64_t k = 0; k < n; k++) {
        if (format == 0) {
            os << element << " " << x[k] << " " << y[k] << " " << z[k] << "\n";
        } else {
            os << k+1 << " 1 "
               << e1[0]*x[k] + e1[1]*y[k] + e1[2]*z[k] << " "
               << e2[0]*x[k] + e2[1]*y[k] + e2[2]*z[k] << " "
               << e3[0]*x[k] + e3[1]*y[k] + e3[2]*z[k] << "\n";
        }
    }
    const std::string s = os.str();
    if ((int64_t)s.size() <= cap && out) std::memcpy(out, s.data(), s.size());
    return (int64_t)s.size();
}
