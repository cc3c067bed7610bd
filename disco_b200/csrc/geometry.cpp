// =============================================================================
// Host-side input synthesis: lattices, mid-plane snapping, loop shapes, contour
// polylines, loopon grids and slab loops (include/disco_geometry.h).
//
// The reference builds these inputs in host C++ upstream of its backend (class
// loop, Code/loop.cpp; lattice helpers, Code/lattice.hpp).  The algorithms are
// restated here, formula by formula in the reference's arithmetic order so that
// the same inputs give the same doubles (tests compare them with the reference's
// own functions), so that workloads can be synthesised where the reference
// tree does not exist.  compress is (1, 1, 1) throughout (Code/main.cpp:232).
// =============================================================================

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/disco_geometry.h"

namespace {

struct V3 { double x, y, z; };

inline V3 load(const double* a) { return { a[0], a[1], a[2] }; }
inline void store(double* a, V3 v) { a[0] = v.x; a[1] = v.y; a[2] = v.z; }
inline double dot(V3 a, V3 b) { return a.x*b.x + a.y*b.y + a.z*b.z; }
inline V3 cross(V3 a, V3 b) { return { a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x }; }
inline double norm(V3 a) { return std::sqrt(a.x*a.x + a.y*a.y + a.z*a.z); }

// Unit m and n, |b| = a0 |m| / 2 and p = m x n (Code/loop.cpp:13-35).
void set_frame(disco_geom_loop& g, const double* m, const double* n, double a0)
{
    const double lm = std::sqrt(m[0]*m[0] + m[1]*m[1] + m[2]*m[2]);
    const double ln = std::sqrt(n[0]*n[0] + n[1]*n[1] + n[2]*n[2]);
    for (int i = 0; i < 3; i++) { g.m[i] = m[i] / lm; g.n[i] = n[i] / ln; }
    g.bmag = a0 * 0.5 * lm;
    store(g.p, cross(load(g.m), load(g.n)));
}

// Default in-plane axes (Code/loop.cpp:37-58): u = m projected on the plane or,
// for m parallel to n, n x e_k with e_k the axis of smallest |n_k|; v = u x n.
void default_axes(const double* m, const double* n, double* u, double* v)
{
    const double mn = m[0]*n[0] + m[1]*n[1] + m[2]*n[2];
    V3 a = { m[0] - mn*n[0], m[1] - mn*n[1], m[2] - mn*n[2] };
    double l = norm(a);
    if (l < 1e-6) {
        int k = 0;
        for (int i = 1; i < 3; i++) if (std::fabs(n[i]) < std::fabs(n[k])) k = i;
        double e[3] = { 0., 0., 0. };
        e[k] = 1.;
        a = cross(load(n), load(e));
        l = norm(a);
    }
    a.x /= l; a.y /= l; a.z /= l;
    store(u, a);
    store(v, cross(a, load(n)));
}

// u from a given in-plane direction: projected on the plane when `project`
// (polygon axis, vertex direction), else only normalised (rectangle side).
void axes_from(const double* dir, const double* n, bool project, double* u, double* v)
{
    V3 a = load(dir);
    if (project) {
        const double an = dot(a, load(n));
        a = { dir[0] - an*n[0], dir[1] - an*n[1], dir[2] - an*n[2] };
    }
    const double l = norm(a);
    a.x /= l; a.y /= l; a.z /= l;
    store(u, a);
    store(v, cross(a, load(n)));
}

void init_loop(disco_geom_loop& g, int shape, double da, const double* c, const double* m,
               const double* n, double a0)
{
    std::memset(&g, 0, sizeof(g));
    g.shape = shape;
    g.da = da;
    for (int i = 0; i < 3; i++) g.c[i] = c[i];
    set_frame(g, m, n, a0);
    // generateSurface (Code/loop.cpp:426-435); the parallelogram factor is set by
    // its constructor below
    g.dS = da * da;
}

// Chords of sagitta <= eps for an arc of angle th, radius r (Code/loop.cpp:487-493)
int arc_chords(double th, double r, double eps)
{
    if (r <= 0. || th <= 0.) return 0;
    const double c = 1. - eps / r;
    const double step = (c <= -1.) ? M_PI : 2. * std::acos(std::max(c, -1.));
    return std::max(1, (int)std::ceil(th / step - 1e-12));
}

// Rounded convex polygon in 2D, counter-clockwise (Code/loop.cpp:498-534): each
// corner i becomes an arc of radius r about the inner vertex, from the outward
// normal of side i-1 to that of side i; consecutive duplicates are dropped.
void rounded_outline(const double* pu, const double* pv, int N, double r, double eps,
                     std::vector<double>& ou, std::vector<double>& ov)
{
    auto add = [&](double a, double b) {
        if (!ou.empty() && std::fabs(ou.back() - a) < 1e-12 && std::fabs(ov.back() - b) < 1e-12) return;
        ou.push_back(a); ov.push_back(b);
    };
    if (r <= 0.) {
        for (int i = 0; i < N; i++) add(pu[i], pv[i]);
    } else {
        std::vector<double> on(N), om(N);   // outward unit normal (u, v) of side i
        for (int i = 0; i < N; i++) {
            const int j = (i + 1) % N;
            const double eu = pu[j] - pu[i], ev = pv[j] - pv[i], l = std::sqrt(eu*eu + ev*ev);
            on[i] = ev / l; om[i] = -eu / l;
        }
        for (int i = 0; i < N; i++) {
            const int k = (i + N - 1) % N;
            const double f = r / (1. + on[k]*on[i] + om[k]*om[i]);
            const double cu = pu[i] - f * (on[k] + on[i]), cv = pv[i] - f * (om[k] + om[i]);
            const double a0 = std::atan2(om[k], on[k]);
            double th = std::atan2(om[i], on[i]) - a0;
            while (th < 0.)        th += 2. * M_PI;
            while (th >= 2. * M_PI) th -= 2. * M_PI;
            const int nc = arc_chords(th, r, eps);
            for (int q = 0; q <= nc; q++) {
                const double a = a0 + th * q / std::max(nc, 1);
                add(cu + r * std::cos(a), cv + r * std::sin(a));
            }
        }
    }
    if (ou.size() > 1 && std::fabs(ou.back() - ou[0]) < 1e-12 && std::fabs(ov.back() - ov[0]) < 1e-12) {
        ou.pop_back(); ov.pop_back();
    }
}

// Code/loop.cpp:281-316
bool inside_uv(const disco_geom_loop& g, double u, double v)
{
    const double eps = 1e-9;
    switch (g.shape) {
    case DISCO_SHAPE_CIRCLE:
        return std::sqrt(u*u + v*v) < g.radius - eps;
    case DISCO_SHAPE_POLYGON: {
        const int N = g.n_poly;
        bool inner = true;
        for (int i = 0; i < N && inner; i++)
            if (g.nu[i]*(u - g.pu[i]) + g.nv[i]*(v - g.pv[i]) < g.r_corner - eps) inner = false;
        if (inner) return true;
        if (g.r_corner <= 0.) return false;
        double d2 = 1e300;
        for (int i = 0; i < N; i++) {
            const int j = (i + 1) % N;
            const double eu = g.qu[j] - g.qu[i], ev = g.qv[j] - g.qv[i];
            const double l2 = eu*eu + ev*ev;
            double t = l2 > 0. ? ((u - g.qu[i])*eu + (v - g.qv[i])*ev) / l2 : 0.;
            t = std::min(std::max(t, 0.), 1.);
            const double wu = u - g.qu[i] - t*eu, wv = v - g.qv[i] - t*ev;
            d2 = std::min(d2, wu*wu + wv*wv);
        }
        return d2 <= g.r_corner*g.r_corner + eps;
    }
    default: {
        const double du = std::max(std::fabs(u) - std::max(g.half_m - g.r_corner, 0.0), 0.0);
        const double dv = std::max(std::fabs(v) - std::max(g.half_p - g.r_corner, 0.0), 0.0);
        return du*du + dv*dv <= g.r_corner*g.r_corner + eps;
    }
    }
}

// isLatticeTranslation, Code/lattice.hpp:160-170 (m in units of a0/2)
bool lattice_translation(int lattice, const double* m)
{
    long h[3];
    for (int i = 0; i < 3; i++) {
        h[i] = std::lround(m[i]);
        if (std::fabs(m[i] - h[i]) > 1e-9) return false;
    }
    if (lattice == DISCO_LATTICE_FCC) return labs(h[0] + h[1] + h[2]) % 2 == 0;
    return (labs(h[0]) % 2 == labs(h[1]) % 2) && (labs(h[1]) % 2 == labs(h[2]) % 2);
}

// frankCopyShift, Code/lattice.hpp:239-256: v plus the in-plane a0/6<112>
// vector s (first in permutation x sign order with s.n = 0) for which v + s is
// not an FCC translation.
void frank_shift(const double* v, const double* nhat, double a0, double* out)
{
    static const int perm[3][3] = { {0, 1, 2}, {1, 2, 0}, {2, 0, 1} };
    const double base[3] = { 1., 1., 2. };
    for (int p = 0; p < 3; p++)
        for (int sg = 0; sg < 8; sg++) {
            double s[3];
            for (int i = 0; i < 3; i++)
                s[perm[p][i]] = ((sg >> i) & 1 ? -1. : 1.) * base[i] * a0 / 6.;
            if (std::fabs(s[0]*nhat[0] + s[1]*nhat[1] + s[2]*nhat[2]) > 1e-9 * a0) continue;
            const double w[3] = { 2. * (v[0] + s[0]) / a0, 2. * (v[1] + s[1]) / a0,
                                  2. * (v[2] + s[2]) / a0 };
            if (lattice_translation(DISCO_LATTICE_FCC, w)) continue;
            for (int i = 0; i < 3; i++) out[i] = v[i] + s[i];
            return;
        }
    for (int i = 0; i < 3; i++) out[i] = v[i];
}

} // namespace

extern "C" {

int disco_geom_circle(double da, double radius, const double c[3], const double m[3],
                      const double n[3], double a0, disco_geom_loop* out)
{
    if (!out || !c || !m || !n || !(radius > 0.)) return DISCO_EINVAL;
    init_loop(*out, DISCO_SHAPE_CIRCLE, da, c, m, n, a0);
    out->radius = radius;
    default_axes(out->m, out->n, out->u, out->v);
    return DISCO_OK;
}

int disco_geom_rectangle(double da, double half_m, double half_p, double corner_r,
                         const double c[3], const double m[3], const double n[3], double a0,
                         const double* side, disco_geom_loop* out)
{
    if (!out || !c || !m || !n || !(half_m > 0.) || !(half_p > 0.)) return DISCO_EINVAL;
    init_loop(*out, DISCO_SHAPE_RECTANGLE, da, c, m, n, a0);
    out->half_m = half_m;
    out->half_p = half_p;
    if (side) axes_from(side, out->n, false, out->u, out->v);
    else      default_axes(out->m, out->n, out->u, out->v);
    out->r_corner = std::min(corner_r, std::min(half_m, half_p));   // Code/loop.cpp:104-110
    return DISCO_OK;
}

int disco_geom_parallelogram(double da, double half1, double half2, const double dir1[3],
                             const double dir2[3], const double c[3], const double m[3],
                             const double n[3], double a0, disco_geom_loop* out)
{
    if (!out || !c || !m || !n || !dir1 || !dir2) return DISCO_EINVAL;
    init_loop(*out, DISCO_SHAPE_PARALLELOGRAM, da, c, m, n, a0);
    out->half_m = half1;
    out->half_p = half2;
    const double l1 = std::sqrt(dir1[0]*dir1[0] + dir1[1]*dir1[1] + dir1[2]*dir1[2]);
    const double l2 = std::sqrt(dir2[0]*dir2[0] + dir2[1]*dir2[1] + dir2[2]*dir2[2]);
    for (int i = 0; i < 3; i++) { out->u[i] = dir1[i] / l1; out->v[i] = dir2[i] / l2; }
    out->dS *= norm(cross(load(out->u), load(out->v)));          // Code/loop.cpp:429-433
    return DISCO_OK;
}

// Code/loop.cpp:150-244: project, orient counter-clockwise, check strict
// convexity, clamp the corner radius, inward normals and inner polygon.
int disco_geom_polygon(double da, const double* verts, int32_t nverts, double corner_r,
                       const double c[3], const double m[3], const double n[3], double a0,
                       const double* axis, disco_geom_loop* out)
{
    if (!out || !verts || !c || !m || !n) return DISCO_EINVAL;
    const int N = nverts;
    if (N < 3 || N > DISCO_MAX_POLY || corner_r < 0.) return DISCO_EINVAL;
    init_loop(*out, DISCO_SHAPE_POLYGON, da, c, m, n, a0);
    disco_geom_loop& g = *out;
    if (axis) axes_from(axis, g.n, true, g.u, g.v);
    else      default_axes(g.m, g.n, g.u, g.v);
    g.n_poly = N;
    for (int i = 0; i < N; i++) {
        const double* x = verts + 3*i;
        g.pu[i] = x[0]*g.u[0] + x[1]*g.u[1] + x[2]*g.u[2];
        g.pv[i] = x[0]*g.v[0] + x[1]*g.v[1] + x[2]*g.v[2];
    }
    double area2 = 0.;
    for (int i = 0; i < N; i++) {
        const int j = (i + 1) % N;
        area2 += g.pu[i]*g.pv[j] - g.pu[j]*g.pv[i];
    }
    if (std::fabs(area2) < 1e-12) return DISCO_EINVAL;
    if (area2 < 0.) { std::reverse(g.pu, g.pu + N); std::reverse(g.pv, g.pv + N); }

    double du[DISCO_MAX_POLY], dv[DISCO_MAX_POLY], len[DISCO_MAX_POLY], cot_half[DISCO_MAX_POLY];
    for (int i = 0; i < N; i++) {
        const int j = (i + 1) % N;
        const double eu = g.pu[j] - g.pu[i], ev = g.pv[j] - g.pv[i];
        len[i] = std::sqrt(eu*eu + ev*ev);
        if (len[i] < 1e-9) return DISCO_EINVAL;
        du[i] = eu / len[i];
        dv[i] = ev / len[i];
    }
    double turn = 0.;
    for (int i = 0; i < N; i++) {
        const int k = (i + N - 1) % N;
        const double sn = du[k]*dv[i] - dv[k]*du[i];
        const double cs = du[k]*du[i] + dv[k]*dv[i];
        if (sn < 1e-9) return DISCO_EINVAL;              // not strictly convex
        turn += std::atan2(sn, cs);
        cot_half[i] = (1. - cs) / sn;
    }
    if (std::fabs(turn - 2.*M_PI) > 1e-6) return DISCO_EINVAL;   // self-intersecting
    double rmax = 1e300;
    for (int i = 0; i < N; i++) rmax = std::min(rmax, len[i] / (cot_half[i] + cot_half[(i + 1) % N]));
    g.r_corner = std::min(corner_r, rmax);
    for (int i = 0; i < N; i++) { g.nu[i] = -dv[i]; g.nv[i] = du[i]; }
    for (int i = 0; i < N; i++) {
        const int k = (i + N - 1) % N;
        const double n1u = -dv[k], n1v = du[k], n2u = -dv[i], n2v = du[i];
        const double f = g.r_corner / (1. + n1u*n2u + n1v*n2v);
        g.qu[i] = g.pu[i] + f * (n1u + n2u);
        g.qv[i] = g.pv[i] + f * (n1v + n2v);
    }
    for (int i = 0; i < N; i++) {
        g.half_m = std::max(g.half_m, std::fabs(g.pu[i]));
        g.half_p = std::max(g.half_p, std::fabs(g.pv[i]));
    }
    return DISCO_OK;
}

int disco_geom_regular_polygon(int32_t sides, double R, const double* vertex_dir,
                               const double m[3], const double n[3], double* out)
{
    if (sides < 3 || !out || !m || !n) return DISCO_EINVAL;
    const double lm = std::sqrt(m[0]*m[0] + m[1]*m[1] + m[2]*m[2]);
    const double ln = std::sqrt(n[0]*n[0] + n[1]*n[1] + n[2]*n[2]);
    const double mh[3] = { m[0]/lm, m[1]/lm, m[2]/lm }, nh[3] = { n[0]/ln, n[1]/ln, n[2]/ln };
    double u[3], v[3];
    if (vertex_dir) axes_from(vertex_dir, nh, true, u, v);
    else            default_axes(mh, nh, u, v);
    for (int k = 0; k < sides; k++) {
        const double th = 2. * M_PI * k / sides;
        for (int i = 0; i < 3; i++) out[3*k + i] = R * (std::cos(th) * u[i] + std::sin(th) * v[i]);
    }
    return DISCO_OK;
}

int32_t disco_geom_polyline(const disco_geom_loop* lp, double eps, double* out, int32_t cap)
{
    if (!lp) return -DISCO_EINVAL;
    const disco_geom_loop& g = *lp;
    std::vector<double> a, b;
    switch (g.shape) {
    case DISCO_SHAPE_CIRCLE: {
        // n chords of sagitta <= eps on the equal-area radius (Code/loop.cpp:540-548)
        const int nch = std::max(8, arc_chords(2. * M_PI, g.radius, eps));
        const double Rp = g.radius * std::sqrt(2. * M_PI / (nch * std::sin(2. * M_PI / nch)));
        for (int k = 0; k < nch; k++) {
            a.push_back(Rp * std::cos(2. * M_PI * k / nch));
            b.push_back(Rp * std::sin(2. * M_PI * k / nch));
        }
        break;
    }
    case DISCO_SHAPE_RECTANGLE:
    case DISCO_SHAPE_PARALLELOGRAM: {
        const double pu[4] = { g.half_m, -g.half_m, -g.half_m,  g.half_m };
        const double pv[4] = { g.half_p,  g.half_p, -g.half_p, -g.half_p };
        if (g.shape == DISCO_SHAPE_PARALLELOGRAM) { a.assign(pu, pu + 4); b.assign(pv, pv + 4); }
        else rounded_outline(pu, pv, 4, g.r_corner, eps, a, b);
        break;
    }
    default:
        rounded_outline(g.pu, g.pv, g.n_poly, g.r_corner, eps, a, b);
    }
    const int N = (int)a.size();
    std::vector<double> P(3 * (size_t)N);
    for (int k = 0; k < N; k++)
        for (int i = 0; i < 3; i++)
            P[3*k + i] = 1.0 * (g.u[i]*a[k] + g.v[i]*b[k]) + g.c[i];
    // counter-clockwise about n (Code/loop.cpp:566-578)
    double s = 0.;
    for (int k = 0; k < N; k++) {
        const double* p = &P[3*k];
        const double* q = &P[3*((k + 1) % N)];
        const double r1[3] = { p[0]-g.c[0], p[1]-g.c[1], p[2]-g.c[2] };
        const double r2[3] = { q[0]-g.c[0], q[1]-g.c[1], q[2]-g.c[2] };
        s += (r1[1]*r2[2] - r1[2]*r2[1]) * g.n[0] + (r1[2]*r2[0] - r1[0]*r2[2]) * g.n[1]
           + (r1[0]*r2[1] - r1[1]*r2[0]) * g.n[2];
    }
    if (out) {
        for (int k = 0; k < N && k < cap; k++) {
            const int src = s < 0. ? N - 1 - k : k;
            for (int i = 0; i < 3; i++) out[3*k + i] = P[3*src + i];
        }
    }
    return N;
}

int64_t disco_geom_loopons(const disco_geom_loop* lp, double* out, int64_t cap)
{
    if (!lp) return -DISCO_EINVAL;
    const disco_geom_loop& g = *lp;
    const double ext_m = g.shape == DISCO_SHAPE_CIRCLE ? g.radius : g.half_m;
    const double ext_p = g.shape == DISCO_SHAPE_CIRCLE ? g.radius : g.half_p;
    const int steps_m = (int)std::ceil(ext_m / g.da) + 1;
    const int steps_p = (int)std::ceil(ext_p / g.da) + 1;
    int64_t cnt = 0;
    for (int xi = -steps_m; xi <= steps_m; xi++)
        for (int yi = -steps_p; yi <= steps_p; yi++) {
            const double u = xi * g.da;
            const double v = yi * g.da;
            if (!inside_uv(g, u, v)) continue;
            if (out && cnt < cap)
                for (int i = 0; i < 3; i++)
                    out[3*cnt + i] = 1.0 * (g.u[i]*u + g.v[i]*v) + g.c[i];
            cnt++;
        }
    return cnt;
}

double disco_geom_area(const disco_geom_loop* lp)
{
    const disco_geom_loop& g = *lp;
    const double r = g.r_corner;
    switch (g.shape) {
    case DISCO_SHAPE_CIRCLE:    return M_PI * g.radius * g.radius;
    case DISCO_SHAPE_RECTANGLE: return 4. * g.half_m * g.half_p - (4. - M_PI) * r * r;
    case DISCO_SHAPE_PARALLELOGRAM: {
        const double c = g.u[0]*g.v[0] + g.u[1]*g.v[1] + g.u[2]*g.v[2];
        return 4. * g.half_m * g.half_p * std::sqrt(std::max(1. - c*c, 0.));
    }
    default: {
        const int N = g.n_poly;
        double a2 = 0., per = 0.;
        for (int i = 0; i < N; i++) {
            const int j = (i + 1) % N;
            a2  += g.qu[i]*g.qv[j] - g.qu[j]*g.qv[i];
            per += std::sqrt((g.qu[j]-g.qu[i])*(g.qu[j]-g.qu[i]) + (g.qv[j]-g.qv[i])*(g.qv[j]-g.qv[i]));
        }
        return 0.5 * a2 + per * r + M_PI * r * r;
    }
    }
}

int disco_geom_contains(const disco_geom_loop* lp, const double rel[3])
{
    const disco_geom_loop& g = *lp;
    const double ru = rel[0]*g.u[0] + rel[1]*g.u[1] + rel[2]*g.u[2];
    const double rv = rel[0]*g.v[0] + rel[1]*g.v[1] + rel[2]*g.v[2];
    const double c = g.u[0]*g.v[0] + g.u[1]*g.v[1] + g.u[2]*g.v[2];
    const double det = 1.0 - c*c;
    return inside_uv(g, (ru - c*rv) / det, (rv - c*ru) / det) ? 1 : 0;
}

// latticePlaneSpacing (Code/lattice.hpp:146-153) and snapToMidPlane
// (Code/loop.cpp:342-374): reduce n to coprime Miller indices, project the
// centre on n-hat and move it to the nearest mid-plane at or above it.
int disco_geom_snap(const double c[3], const double n[3], double a0, int32_t nx, int32_t ny,
                    int32_t nz, int32_t lattice, double out[3], double* spacing)
{
    long h[3];
    for (int i = 0; i < 3; i++) {
        h[i] = std::lround(n[i]);
        if (std::fabs(n[i] - h[i]) > 1e-9) return DISCO_EINVAL;
    }
    long g = 0;
    for (int i = 0; i < 3; i++) {
        long a = labs(h[i]);
        while (a) { const long t = g % a; g = a; a = t; }
    }
    if (g == 0) return DISCO_EINVAL;
    for (int i = 0; i < 3; i++) h[i] /= g;
    const double nrm = std::sqrt(double(h[0]*h[0] + h[1]*h[1] + h[2]*h[2]));
    const double nh[3] = { h[0]/nrm, h[1]/nrm, h[2]/nrm };
    const bool full = lattice == DISCO_LATTICE_FCC
        ? ((labs(h[0]) % 2) && (labs(h[1]) % 2) && (labs(h[2]) % 2))
        : (labs(h[0] + h[1] + h[2]) % 2 == 0);
    const double d = full ? a0 / nrm : a0 / (2. * nrm);
    *spacing = d;
    const double o[3] = { -0.5*a0*nx, -0.5*a0*ny, -0.5*a0*nz };
    const double s0 = o[0]*nh[0] + o[1]*nh[1] + o[2]*nh[2];
    const double s = c[0]*nh[0] + c[1]*nh[1] + c[2]*nh[2];
    const double s_mid = s0 + (std::floor((s - s0) / d + 1e-9) + 0.5) * d;
    for (int i = 0; i < 3; i++) out[i] = c[i] + (s_mid - s) * nh[i];
    return DISCO_OK;
}

// generateLattice (Code/lattice.hpp:35-51): cells (i, j, k), k fastest, then
// the basis sites in table order.
int64_t disco_geom_lattice(int32_t lattice, int32_t nx, int32_t ny, int32_t nz, double a0,
                           double* x, double* y, double* z)
{
    static const double bcc[2][3] = { {0, 0, 0}, {0.5, 0.5, 0.5} };
    static const double fcc[4][3] = { {0, 0, 0}, {0.5, 0.5, 0}, {0.5, 0, 0.5}, {0, 0.5, 0.5} };
    const double (*f)[3] = lattice == DISCO_LATTICE_FCC ? fcc : bcc;
    const int nb = lattice == DISCO_LATTICE_FCC ? 4 : 2;
    const double hx = nx * a0 / 2., hy = ny * a0 / 2., hz = nz * a0 / 2.;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; i++) {
        int64_t q = (int64_t)i * ny * nz * nb;
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++)
                for (int b = 0; b < nb; b++, q++) {
                    x[q] = i*a0 + f[b][0]*a0 - hx;
                    y[q] = j*a0 + f[b][1]*a0 - hy;
                    z[q] = k*a0 + f[b][2]*a0 - hz;
                }
    }
    return (int64_t)nb * nx * ny * nz;
}

int32_t disco_geom_classify_burgers(int32_t lattice, const double m[3], const double n[3])
{
    if (lattice_translation(lattice, m)) return 0;
    if (lattice != DISCO_LATTICE_FCC) return 3;
    long k[3];
    for (int i = 0; i < 3; i++) {
        k[i] = std::lround(3. * m[i]);
        if (std::fabs(3. * m[i] - k[i]) > 1e-6) return 3;
    }
    const long a = labs(k[0]), b = labs(k[1]), c = labs(k[2]);
    if (a == 2 && b == 2 && c == 2) {
        const double x[3] = { m[1]*n[2] - m[2]*n[1], m[2]*n[0] - m[0]*n[2], m[0]*n[1] - m[1]*n[0] };
        const double cn = std::sqrt(x[0]*x[0] + x[1]*x[1] + x[2]*x[2]);
        const double nn = std::sqrt(n[0]*n[0] + n[1]*n[1] + n[2]*n[2]);
        return cn < 1e-6 * nn ? 1 : 3;
    }
    const long lo = std::min(a, std::min(b, c)), hi = std::max(a, std::max(b, c));
    if (lo == 1 && hi == 2 && a + b + c == 4) {
        const bool n111 = std::fabs(n[0]) > 0. && std::fabs(std::fabs(n[0]) - std::fabs(n[1])) < 1e-9
                          && std::fabs(std::fabs(n[0]) - std::fabs(n[2])) < 1e-9;
        const double mn = m[0]*n[0] + m[1]*n[1] + m[2]*n[2];
        return (n111 && std::fabs(mn) < 1e-6) ? 2 : 3;
    }
    return 3;
}

int disco_geom_slab_loop(const disco_geom_loop* lp, double spacing, int32_t apply,
                         int32_t frank, double a0, disco_slab_loop* out)
{
    if (!lp || !out) return DISCO_EINVAL;
    const disco_geom_loop& g = *lp;
    std::memset(out, 0, sizeof(*out));
    for (int i = 0; i < 3; i++) {
        out->c[i] = g.c[i]; out->m[i] = g.m[i]; out->n[i] = g.n[i];
        out->u[i] = g.u[i]; out->v[i] = g.v[i];
    }
    out->bmag = g.bmag;
    out->spacing = spacing;
    out->shape = g.shape;
    out->n_poly = g.n_poly;
    out->radius = g.radius; out->half_m = g.half_m; out->half_p = g.half_p;
    out->r_corner = g.r_corner;
    for (int i = 0; i < g.n_poly; i++) {
        out->pu[i] = g.pu[i]; out->pv[i] = g.pv[i];
        out->qu[i] = g.qu[i]; out->qv[i] = g.qv[i];
        out->nu[i] = g.nu[i]; out->nv[i] = g.nv[i];
    }
    out->apply = apply;
    // copy shift per side (Code/main.cpp:630-650): +-b, plus the Shockley shift of
    // an FCC Frank loop (box axes = crystal axes)
    const double b[3] = { g.bmag*g.m[0], g.bmag*g.m[1], g.bmag*g.m[2] };
    for (int sd = 0; sd < 2; sd++) {
        const double sign = sd == 0 ? 1. : -1.;
        const double v[3] = { sign*b[0], sign*b[1], sign*b[2] };
        double* dst = sd == 0 ? out->shift_pos : out->shift_neg;
        if (frank) frank_shift(v, g.n, a0, dst);
        else for (int i = 0; i < 3; i++) dst[i] = v[i];
    }
    return DISCO_OK;
}

} // extern "C"
