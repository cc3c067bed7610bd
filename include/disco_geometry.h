/*
 * disco_geometry.h — host-side input synthesis for the displacement backend.
 *
 * These functions are not part of the backend boundary: in the reference the
 * same inputs are produced by host C++ upstream of the backend (the loop class,
 * Code/loop.hpp/.cpp, and the lattice helpers, Code/lattice.hpp), which stays
 * as it is.  They exist so that seeded synthetic workloads (lattices, loops,
 * polylines, loopon grids, slab loops) can be built where the reference tree is
 * absent, with the reference's algorithms restated; the tests compare them with
 * the reference's own functions.  Library: disco_b200/_lib/libdisco_geom.so.
 */
#ifndef DISCO_GEOMETRY_H
#define DISCO_GEOMETRY_H

#include <stdint.h>
#include "disco_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define DISCO_LATTICE_BCC 0
#define DISCO_LATTICE_FCC 1

/* A loop's geometry, the state of the reference's loop class
 * (Code/loop.hpp:19-45) with compress = (1, 1, 1) as Code/main.cpp:232 sets it. */
typedef struct {
    int32_t shape;                 /* DISCO_SHAPE_*                               */
    int32_t n_poly;
    double c[3];                   /* centre (on a mid-plane)                     */
    double m[3], n[3], p[3];       /* unit m, unit n, p = m x n                   */
    double u[3], v[3];             /* loopon grid axes                            */
    double bmag;                   /* |b| = a0 |m| / 2                            */
    double radius, half_m, half_p, r_corner;
    double da, dS;                 /* loopon step and cell area                   */
    double pu[DISCO_MAX_POLY], pv[DISCO_MAX_POLY];
    double qu[DISCO_MAX_POLY], qv[DISCO_MAX_POLY];
    double nu[DISCO_MAX_POLY], nv[DISCO_MAX_POLY];
} disco_geom_loop;

/* Constructors, Code/loop.cpp:58-238.  m and n need not be unit vectors.
 * side / axis / vertex_dir may be NULL (default in-plane axis).  Return
 * DISCO_OK or DISCO_EINVAL (the reference aborts on the same inputs). */
int disco_geom_circle(double da, double radius, const double c[3], const double m[3],
                      const double n[3], double a0, disco_geom_loop *out);
int disco_geom_rectangle(double da, double half_m, double half_p, double corner_r,
                         const double c[3], const double m[3], const double n[3], double a0,
                         const double *side, disco_geom_loop *out);
int disco_geom_parallelogram(double da, double half1, double half2, const double dir1[3],
                             const double dir2[3], const double c[3], const double m[3],
                             const double n[3], double a0, disco_geom_loop *out);
int disco_geom_polygon(double da, const double *verts, int32_t nverts, double corner_r,
                       const double c[3], const double m[3], const double n[3], double a0,
                       const double *axis, disco_geom_loop *out);

/* regularPolygon, Code/loop.cpp:585-608: sides x 3 in-plane offsets. */
int disco_geom_regular_polygon(int32_t sides, double R, const double *vertex_dir,
                               const double m[3], const double n[3], double *out);

/* loop::polyline, Code/loop.cpp:536-580: vertices into out[3*k..], returns the
 * vertex count (out may be NULL to size it). */
int32_t disco_geom_polyline(const disco_geom_loop *lp, double eps, double *out, int32_t cap);

/* generateSurface + generateLoopons, Code/loop.cpp:253-273,426-435: loopon
 * positions into out[3*k..] (NULL to count), returns the count. */
int64_t disco_geom_loopons(const disco_geom_loop *lp, double *out, int64_t cap);

/* loop::getContourArea, Code/loop.cpp:461-484. */
double disco_geom_area(const disco_geom_loop *lp);

/* loop::contains, Code/loop.cpp:323-330 (rel = point - centre, minimum image). */
int disco_geom_contains(const disco_geom_loop *lp, const double rel[3]);

/* snapToMidPlane, Code/loop.cpp:342-374. */
int disco_geom_snap(const double c[3], const double n[3], double a0, int32_t nx, int32_t ny,
                    int32_t nz, int32_t lattice, double out[3], double *spacing);

/* generateLattice, Code/lattice.hpp:35-51: writes nb*nx*ny*nz sites. */
int64_t disco_geom_lattice(int32_t lattice, int32_t nx, int32_t ny, int32_t nz, double a0,
                           double *x, double *y, double *z);

/* classifyBurgers, Code/lattice.hpp:189-213 (m, n crystal frame, m in units
 * of a0/2): 0 perfect, 1 Frank, 2 Shockley, 3 other. */
int32_t disco_geom_classify_burgers(int32_t lattice, const double m[3], const double n[3]);

/* A slab loop for disco_b200_prismatic from a geometry loop: matter type,
 * shifts side*b (Code/main.cpp:630-650), plus frankCopyShift
 * (Code/lattice.hpp:239-256) when frank != 0. */
int disco_geom_slab_loop(const disco_geom_loop *lp, double spacing, int32_t apply,
                         int32_t frank, double a0, disco_slab_loop *out);

#ifdef __cplusplus
}
#endif

#endif /* DISCO_GEOMETRY_H */
