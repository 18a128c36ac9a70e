// ab_forbild.cu -- exact analytic projection of FORBILD quadric phantoms.
//
// Replaces project_CB_FORBILD_shapes<float,FORBILD_Shape>
// (src/aprict/data/cusrc/CB_project_texture_chunked.cu:415-593) with
// FORBILD_clip_line_segment (FORBILD_volumes.h:1723-1811) and
// exact_line_integral_prioritise_last (:1889-1954).
//
// Design:
//   * Shapes are reduced on the host, in FP64, to an affine map onto one of
//     four canonical solids plus <= 3 half-spaces (aprict_b200_forbild_compile).
//   * A CTA owns a 16x16 (or 256x1) detector tile of one view. It projects
//     every shape's world bounding box onto the detector (FP64), keeps the
//     shapes whose footprint meets the tile -- in order -- and writes their
//     per-view ray coefficients to shared memory. The reference instead tests
//     every shape on every ray and stages them 4 at a time behind two
//     barriers each (:500-525).
//   * Per ray and kept shape, the entry/exit parameters along the
//     source->pixel segment are solved in FP64 (clip planes, then the
//     quadric), so tangent and grazing rays keep their accuracy.
//   * "Later shapes win" is resolved by visiting the kept shapes from last to
//     first and charging each only for the part of its interval not yet
//     covered (a short list of disjoint covered intervals per ray); the
//     reference stores up to 1000 intervals per thread (12 KB of local memory)
//     and sweeps them in O(k^2).
#include <cuda_runtime.h>

#include <math.h>
#include <string.h>

#include "ab_common.cuh"
#include "ab_host.h"

static_assert(sizeof(aprict_forbild_shape) == 156, "FORBILD_Shape is 156 bytes in the reference");

namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 128;  // shapes per shared-memory chunk (one chunk, one barrier round, up to 128 shapes)
constexpr int kMaxU = 16;   // disjoint covered intervals tracked per ray

struct QView {
    double o[3], d0[3], du[3], dv[3];  // local(t) = o + t (d0 + du fu + dv fv)
    double cq;                         // canonical constant (see kind)
    double g0[3], gd0[3], gdu[3], gdv[3];
    double h, alpha, beta;
    double rho;
    int kind, n_clip;
};

// ------------------------------------------------------------------ host
void nrm3(const double a[3], double o[3]) {
    const double n = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    o[0] = a[0] / n;
    o[1] = a[1] / n;
    o[2] = a[2] / n;
}

// Orthonormal e1, e2 completing the unit vector a.
void perp_basis(const double a[3], double e1[3], double e2[3]) {
    const double t[3] = {fabs(a[0]) < 0.9 ? 1.0 : 0.0, fabs(a[0]) < 0.9 ? 0.0 : 1.0, 0.0};
    double c[3] = {a[1] * t[2] - a[2] * t[1], a[2] * t[0] - a[0] * t[2], a[0] * t[1] - a[1] * t[0]};
    nrm3(c, e1);
    e2[0] = a[1] * e1[2] - a[2] * e1[1];
    e2[1] = a[2] * e1[0] - a[0] * e1[2];
    e2[2] = a[0] * e1[1] - a[1] * e1[0];
}

bool inv3(const double m[9], double o[9]) {
    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                       m[2] * (m[3] * m[7] - m[4] * m[6]);
    if (!(fabs(det) > 0.0) || !isfinite(det)) return false;
    const double id = 1.0 / det;
    o[0] = (m[4] * m[8] - m[5] * m[7]) * id;
    o[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    o[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    o[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    o[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    o[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    o[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    o[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    o[8] = (m[0] * m[4] - m[1] * m[3]) * id;
    return true;
}

void set_rows(double M[9], const double r0[3], const double r1[3], const double r2[3]) {
    for (int i = 0; i < 3; ++i) {
        M[i] = r0[i];
        M[3 + i] = r1[i];
        M[6 + i] = r2[i];
    }
}

}  // namespace

extern "C" int aprict_b200_forbild_compile(const aprict_forbild_shape *sh, int64_t n, aprict_quadric *out) {
    if (n < 0) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "forbild_compile: negative count");
    if (n > 0 && (sh == nullptr || out == nullptr)) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "forbild_compile: null");
    for (int64_t i = 0; i < n; ++i) {
        const aprict_forbild_shape &s = sh[i];
        aprict_quadric q;
        memset(&q, 0, sizeof(q));
        q.rho = s.rho;
        q.c[0] = s.x;
        q.c[1] = s.y;
        q.c[2] = s.z;
        double M[9] = {0};
        const double ex[3] = {1, 0, 0}, ey[3] = {0, 1, 0}, ez[3] = {0, 0, 1};
        auto scaled = [](const double v[3], double f, double o[3]) {
            o[0] = v[0] * f;
            o[1] = v[1] * f;
            o[2] = v[2] * f;
        };
        auto unit = [](aprict_fvec3 v, double o[3]) {
            const double a[3] = {v.x, v.y, v.z};
            nrm3(a, o);
        };
        double r0[3], r1[3], r2[3], ax[3], e1[3], e2[3];
        bool bad = false;
        switch (s.type) {
            case 0:
                q.kind = 0;
                break;
            case 10:  // Ellipsoid (FORBILD_volumes.h:976-1033)
                bad = !(s.dx > 0 && s.dy > 0 && s.dz > 0);
                scaled(ex, 1.0 / s.dx, r0);
                scaled(ey, 1.0 / s.dy, r1);
                scaled(ez, 1.0 / s.dz, r2);
                set_rows(M, r0, r1, r2);
                q.kind = 1;
                break;
            case 11:  // Ellipsoid_free (:1036-1117)
                bad = !(s.dx > 0 && s.dy > 0 && s.dz > 0);
                unit(s.a_x, r0);
                unit(s.a_y, r1);
                unit(s.a_z, r2);
                scaled(r0, 1.0 / s.dx, r0);
                scaled(r1, 1.0 / s.dy, r1);
                scaled(r2, 1.0 / s.dz, r2);
                set_rows(M, r0, r1, r2);
                q.kind = 1;
                break;
            case 13:  // Sphere (:887-973)
                bad = !(s.r > 0);
                scaled(ex, 1.0 / s.r, r0);
                scaled(ey, 1.0 / s.r, r1);
                scaled(ez, 1.0 / s.r, r2);
                set_rows(M, r0, r1, r2);
                q.kind = 1;
                break;
            case 12:  // Ellipt_Cyl (:1120-1203)
                bad = !(s.dx > 0 && s.dy > 0 && s.l > 0);
                unit(s.a_x, r0);
                unit(s.a_y, r1);
                unit(s.axis, r2);
                scaled(r0, 1.0 / s.dx, r0);
                scaled(r1, 1.0 / s.dy, r1);
                set_rows(M, r0, r1, r2);
                q.kind = 2;
                q.h = 0.5 * s.l;
                break;
            case 14:  // Ellipt_Cyl_x: semi-axes dy along y, dz along z, axis x
                bad = !(s.dy > 0 && s.dz > 0 && s.l > 0);
                scaled(ey, 1.0 / s.dy, r0);
                scaled(ez, 1.0 / s.dz, r1);
                set_rows(M, r0, r1, ex);
                q.kind = 2;
                q.h = 0.5 * s.l;
                break;
            case 15:  // Ellipt_Cyl_y: dx along x, dz along z, axis y
                bad = !(s.dx > 0 && s.dz > 0 && s.l > 0);
                scaled(ex, 1.0 / s.dx, r0);
                scaled(ez, 1.0 / s.dz, r1);
                set_rows(M, r0, r1, ey);
                q.kind = 2;
                q.h = 0.5 * s.l;
                break;
            case 16:  // Ellipt_Cyl_z: dx along x, dy along y, axis z
                bad = !(s.dx > 0 && s.dy > 0 && s.l > 0);
                scaled(ex, 1.0 / s.dx, r0);
                scaled(ey, 1.0 / s.dy, r1);
                set_rows(M, r0, r1, ez);
                q.kind = 2;
                q.h = 0.5 * s.l;
                break;
            case 6:  // Cylinder with free axis (:158-287)
            case 7:  // Cylinder_x
            case 8:  // Cylinder_y
            case 9:  // Cylinder_z
                bad = !(s.r > 0 && s.l > 0);
                if (s.type == 6) {
                    unit(s.axis, ax);
                } else {
                    const double *a = s.type == 7 ? ex : (s.type == 8 ? ey : ez);
                    ax[0] = a[0];
                    ax[1] = a[1];
                    ax[2] = a[2];
                }
                perp_basis(ax, e1, e2);
                scaled(e1, 1.0 / s.r, r0);
                scaled(e2, 1.0 / s.r, r1);
                set_rows(M, r0, r1, ax);
                q.kind = 2;
                q.h = 0.5 * s.l;
                break;
            case 2:  // Cone (free axis), radius r1 at -l/2 to r2 at +l/2
            case 3:  // Cone_x
            case 4:  // Cone_y
            case 5:  // Cone_z
                bad = !(s.l > 0 && s.r1 >= 0 && s.r2 >= 0 && (s.r1 > 0 || s.r2 > 0));
                if (s.type == 2) {
                    unit(s.axis, ax);
                } else {
                    const double *a = s.type == 3 ? ex : (s.type == 4 ? ey : ez);
                    ax[0] = a[0];
                    ax[1] = a[1];
                    ax[2] = a[2];
                }
                perp_basis(ax, e1, e2);
                set_rows(M, e1, e2, ax);
                q.kind = 3;
                q.h = 0.5 * s.l;
                q.alpha = 0.5 * ((double)s.r1 + (double)s.r2);
                q.beta = ((double)s.r2 - (double)s.r1) / (double)s.l;
                break;
            case 1:  // Box with full side lengths dx, dy, dz (:1-85)
                bad = !(s.dx > 0 && s.dy > 0 && s.dz > 0);
                scaled(ex, 2.0 / s.dx, r0);
                scaled(ey, 2.0 / s.dy, r1);
                scaled(ez, 2.0 / s.dz, r2);
                set_rows(M, r0, r1, r2);
                q.kind = 4;
                break;
            default:
                return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "forbild_compile: shape %lld has unknown type %u",
                               (long long)i, (unsigned)s.type);
        }
        if (bad || !isfinite(q.rho))
            return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "forbild_compile: shape %lld (type %u) has invalid parameters",
                           (long long)i, (unsigned)s.type);
        memcpy(q.M, M, sizeof(M));
        if (q.kind != 0) {
            double Mi[9];
            if (!inv3(M, Mi))
                return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "forbild_compile: shape %lld has a singular frame",
                               (long long)i);
            // World AABB half extents: support of the canonical solid in the
            // direction of each row of M^-1.
            for (int a = 0; a < 3; ++a) {
                const double w[3] = {Mi[3 * a], Mi[3 * a + 1], Mi[3 * a + 2]};
                double sup;
                switch (q.kind) {
                    case 1: sup = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]); break;
                    case 2: sup = sqrt(w[0] * w[0] + w[1] * w[1]) + q.h * fabs(w[2]); break;
                    case 3: {
                        const double rmax = fmax(fabs(q.alpha - q.beta * q.h), fabs(q.alpha + q.beta * q.h));
                        sup = rmax * sqrt(w[0] * w[0] + w[1] * w[1]) + q.h * fabs(w[2]);
                        break;
                    }
                    default: sup = fabs(w[0]) + fabs(w[1]) + fabs(w[2]); break;
                }
                q.bb_half[a] = sup;
            }
        }
        const aprict_forbild_clip *cs[3] = {&s.cas1, &s.cas2, &s.cas3};
        for (int k = 0; k < 3; ++k) {
            if (cs[k]->mode == 0) continue;
            const double sg = cs[k]->mode == 1 ? 1.0 : -1.0;  // mode 2 keeps a.p > d
            const int kc = q.n_clip & 0xFF;
            q.clip[kc][0] = sg * cs[k]->axis.x;
            q.clip[kc][1] = sg * cs[k]->axis.y;
            q.clip[kc][2] = sg * cs[k]->axis.z;
            q.clip[kc][3] = sg * cs[k]->dotprod;
            if (cs[k]->mode == 2) q.n_clip |= 0x100 << kc;  // strict: a.p > d
            q.n_clip++;
        }
        out[i] = q;
    }
    return APRICT_OK;
}

namespace {

struct ViewGeom {
    ab_d3 s, P, U, V, n, Au, Av, D0;  // D0 = P - s - U hu - V hv
    double s_n;                       // s . n
    double Dn;
};

__device__ void view_geom(const aprict_proj_spec &sp, ViewGeom &g) {
    g.s = ab_d3_of(sp.source_pos);
    g.P = ab_d3_of(sp.det_pos);
    g.U = ab_d3_of(sp.det_u);
    g.V = ab_d3_of(sp.det_v);
    g.n = ab_cross(g.U, g.V);
    const ab_d3 Ps = g.P - g.s;
    g.Dn = ab_dot(Ps, g.n);
    const double hu = ((double)sp.nu - 1.0) * 0.5, hv = ((double)sp.nv - 1.0) * 0.5;
    // pixel index of a point x: (Au.(x-s)) / ((x-s).n), same for v
    g.Au = (g.U * g.Dn - g.n * ab_dot(g.U, Ps)) * (1.0 / ab_dot(g.U, g.U)) + g.n * hu;
    g.Av = (g.V * g.Dn - g.n * ab_dot(g.V, Ps)) * (1.0 / ab_dot(g.V, g.V)) + g.n * hv;
    g.D0 = Ps - g.U * hu - g.V * hv;
    g.s_n = ab_dot(g.s, g.n);
}

// Pixel-index rectangle covering the shape's world AABB in this view;
// false if some corner is not in front of the source (use the whole panel).
__device__ bool footprint(const ViewGeom &g, const aprict_quadric &q, double &u0, double &u1, double &v0,
                          double &v1) {
    u0 = v0 = 1e300;
    u1 = v1 = -1e300;
    for (int c = 0; c < 8; ++c) {
        const ab_d3 x{q.c[0] + ((c & 4) ? q.bb_half[0] : -q.bb_half[0]),
                      q.c[1] + ((c & 2) ? q.bb_half[1] : -q.bb_half[1]),
                      q.c[2] + ((c & 1) ? q.bb_half[2] : -q.bb_half[2])};
        const ab_d3 r = x - g.s;
        const double den = ab_dot(r, g.n) * (g.Dn > 0 ? 1.0 : -1.0);
        if (!(den > 0.0)) return false;
        const double sden = ab_dot(r, g.n);
        const double fu = ab_dot(g.Au, r) / sden, fv = ab_dot(g.Av, r) / sden;
        u0 = fmin(u0, fu);
        u1 = fmax(u1, fu);
        v0 = fmin(v0, fv);
        v1 = fmax(v1, fv);
    }
    return true;
}

__device__ void make_qview(const ViewGeom &g, const aprict_quadric &q, QView &o) {
    const double *M = q.M;
    auto mul = [&](ab_d3 v, double r[3]) {
        r[0] = M[0] * v.x + M[1] * v.y + M[2] * v.z;
        r[1] = M[3] * v.x + M[4] * v.y + M[5] * v.z;
        r[2] = M[6] * v.x + M[7] * v.y + M[8] * v.z;
    };
    mul(g.s - ab_d3{q.c[0], q.c[1], q.c[2]}, o.o);
    mul(g.D0, o.d0);
    mul(g.U, o.du);
    mul(g.V, o.dv);
    o.kind = q.kind;
    o.n_clip = q.n_clip & 0xFF;
    o.rho = q.rho;
    o.h = q.h;
    o.alpha = q.alpha;
    o.beta = q.beta;
    if (q.kind == 1)
        o.cq = o.o[0] * o.o[0] + o.o[1] * o.o[1] + o.o[2] * o.o[2] - 1.0;
    else if (q.kind == 2)
        o.cq = o.o[0] * o.o[0] + o.o[1] * o.o[1] - 1.0;
    else
        o.cq = 0.0;
    for (int k = 0; k < 3; ++k) {
        if (k < (q.n_clip & 0xFF)) {
            const ab_d3 a{q.clip[k][0], q.clip[k][1], q.clip[k][2]};
            o.g0[k] = ab_dot(a, g.s) - q.clip[k][3];
            o.gd0[k] = ab_dot(a, g.D0);
            o.gdu[k] = ab_dot(a, g.U);
            o.gdv[k] = ab_dot(a, g.V);
        } else {
            o.g0[k] = o.gd0[k] = o.gdu[k] = o.gdv[k] = 0.0;
        }
    }
}

// Keep the part of [lo,hi] where a + b t <= 0.
__device__ __forceinline__ void halfline(double a, double b, double &lo, double &hi) {
    if (b == 0.0) {
        if (a > 0.0) hi = lo - 1.0;  // empty
        return;
    }
    const double t = -a / b;
    if (b > 0.0)
        hi = fmin(hi, t);
    else
        lo = fmax(lo, t);
}

// Keep the part of [lo,hi] where |o + t d| <= h.
__device__ __forceinline__ void slab(double o, double d, double h, double &lo, double &hi) {
    if (d == 0.0) {
        if (fabs(o) > h) hi = lo - 1.0;
        return;
    }
    const double inv = 1.0 / d;
    const double t0 = (-h - o) * inv, t1 = (h - o) * inv;
    lo = fmax(lo, fmin(t0, t1));
    hi = fmin(hi, fmax(t0, t1));
}

// Parametric interval of the ray with the clipped shape, within [0, 1].
__device__ bool ray_interval(const QView &q, double fu, double fv, double &lo, double &hi) {
    lo = 0.0;
    hi = 1.0;
    for (int k = 0; k < q.n_clip; ++k) {
        const double sl = fma(q.gdv[k], fv, fma(q.gdu[k], fu, q.gd0[k]));
        halfline(q.g0[k], sl, lo, hi);
    }
    if (!(lo < hi)) return false;
    const double d[3] = {fma(q.dv[0], fv, fma(q.du[0], fu, q.d0[0])), fma(q.dv[1], fv, fma(q.du[1], fu, q.d0[1])),
                         fma(q.dv[2], fv, fma(q.du[2], fu, q.d0[2]))};
    const double *o = q.o;
    if (q.kind == 4) {
        slab(o[0], d[0], 1.0, lo, hi);
        slab(o[1], d[1], 1.0, lo, hi);
        slab(o[2], d[2], 1.0, lo, hi);
        return lo < hi;
    }
    if (q.kind == 2 || q.kind == 3) {
        slab(o[2], d[2], q.h, lo, hi);
        if (!(lo < hi)) return false;
    }
    double A, B, C;  // quadric A t^2 + 2 B t + C <= 0
    if (q.kind == 1) {
        A = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        B = o[0] * d[0] + o[1] * d[1] + o[2] * d[2];
        C = q.cq;
    } else if (q.kind == 2) {
        A = d[0] * d[0] + d[1] * d[1];
        B = o[0] * d[0] + o[1] * d[1];
        C = q.cq;
    } else {
        const double ra = q.alpha + q.beta * o[2], rb = q.beta * d[2];
        A = d[0] * d[0] + d[1] * d[1] - rb * rb;
        B = o[0] * d[0] + o[1] * d[1] - ra * rb;
        C = o[0] * o[0] + o[1] * o[1] - ra * ra;
    }
    if (A == 0.0) {  // linear (or constant) in t
        halfline(C, 2.0 * B, lo, hi);
        return lo < hi;
    }
    const double disc = B * B - A * C;
    if (A > 0.0) {
        if (!(disc > 0.0)) return false;
        const double sq = sqrt(disc);
        // stable roots of A t^2 + 2 B t + C: qq / A and C / qq, both from one
        // reciprocal of A qq (qq != 0 here: disc > 0 makes |qq| >= sq > 0)
        const double qq = -(B + copysign(sq, B));
        const double r = 1.0 / (A * qq);
        double t0 = qq * qq * r, t1 = C * A * r;
        if (t0 > t1) {
            const double tmp = t0;
            t0 = t1;
            t1 = tmp;
        }
        lo = fmax(lo, t0);
        hi = fmin(hi, t1);
        return lo < hi;
    }
    // A < 0 (cone): the solution set is (-inf, t0] U [t1, inf), or all t
    if (!(disc > 0.0)) return lo < hi;
    const double sq = sqrt(disc);
    const double qq = -(B + copysign(sq, B));
    const double r = 1.0 / (A * qq);  // as above: qq != 0
    double t0 = qq * qq * r, t1 = C * A * r;
    if (t0 > t1) {
        const double tmp = t0;
        t0 = t1;
        t1 = tmp;
    }
    const double alo = lo, ahi = fmin(hi, t0);
    const double blo = fmax(lo, t1), bhi = hi;
    const bool a_ok = alo < ahi, b_ok = blo < bhi;
    if (a_ok && b_ok) return lo < hi;  // both nappes within the slab: keep the hull
    if (a_ok) {
        hi = ahi;
        return true;
    }
    if (b_ok) {
        lo = blo;
        return true;
    }
    return false;
}

struct TileMap {
    int tile_u, tile_v, ntu, ntv;
};

// Per view and shape, computed once per view (k_forbild_prep) instead of in
// every detector tile: the pixel rectangle of the shape's bounding box
// (all = 1: some corner is not in front of the source, keep for every tile;
// kind 0 shapes are never kept) and the shape in the view's ray frame.
struct QCull {
    double u0, u1, v0, v1;
    int keep_all, live;
};

__global__ void __launch_bounds__(128) k_forbild_prep(const aprict_proj_spec *__restrict__ specs, uint32_t view0,
                                                      uint32_t nvw, const aprict_quadric *__restrict__ shapes,
                                                      int n_shapes, QCull *cull, QView *qv) {
    const int j = blockIdx.x * 128 + (int)threadIdx.x;
    const uint32_t vi = blockIdx.y;
    if (j >= n_shapes || vi >= nvw) return;
    ViewGeom g;
    view_geom(specs[view0 + vi], g);
    const aprict_quadric &q = shapes[j];
    QCull c{0.0, 0.0, 0.0, 0.0, 0, q.kind != 0};
    const size_t o = (size_t)vi * (size_t)n_shapes + (size_t)j;
    if (c.live) {
        c.keep_all = !footprint(g, q, c.u0, c.u1, c.v0, c.v1);
        make_qview(g, q, qv[o]);
    }
    cull[o] = c;
}

TileMap make_tiles(uint32_t nu, uint32_t nv) {
    TileMap t;
    t.tile_v = nv >= 16 ? 16 : 1;
    t.tile_u = kThreads / t.tile_v;
    t.ntu = (int)((nu + t.tile_u - 1) / t.tile_u);
    t.ntv = (int)((nv + t.tile_v - 1) / t.tile_v);
    return t;
}

// 5 resident CTAs per SM (48 registers, the FP64 root solving spills some to
// L1-resident local memory): the kernel waits on FP64 latencies, and the
// unconstrained 106 registers fit only 2 CTAs. Measured on the 100-shape,
// 720-view workload: 142.9 ms at 2 CTAs, 127.3 at 3, 113.4 at 4, 109.3 at 5,
// 119.8 at 6 (96-shape chunks); 102.7 ms at 5 with 128-shape chunks, which
// hold the 100 shapes in one chunk (warps wait at one barrier round, not two).
// PRE: the per-(view, shape) cull records and ray-frame shapes come from
// k_forbild_prep (85.3 ms with them in the same kernel as the in-tile
// derivation, 70.9 ms in a variant without it: fewer spills; 81.6 ms at 6
// CTAs per SM; 65.2 ms with one reciprocal for both quadric roots).
template <int MODE, bool PRE>
__global__ void __launch_bounds__(kThreads, 5) k_project_forbild(const aprict_proj_spec *__restrict__ specs,
                                                               uint32_t n_views, uint32_t nu, uint32_t nv,
                                                               ab_pstrides ps, float *out,
                                                               const aprict_quadric *__restrict__ shapes,
                                                               int n_shapes, float mba, int ssu, int ssv, TileMap tm,
                                                               uint32_t view0, uint32_t *overflow,
                                                               const QCull *__restrict__ pcull,
                                                               const QView *__restrict__ pqv) {
    extern __shared__ double smem_d[];
    QView *sel = reinterpret_cast<QView *>(smem_d);
    __shared__ int s_count;
    __shared__ int s_warp_pos[kThreads / 32];

    const uint32_t view = view0 + blockIdx.y;
    if (view >= n_views) return;
    const int tu = blockIdx.x % tm.ntu, tv = blockIdx.x / tm.ntu;
    int iu, iv;
    if (tm.tile_v == 1) {
        iu = tu * tm.tile_u + threadIdx.x;
        iv = tv;
    } else {
        iu = tu * tm.tile_u + (threadIdx.x & 15);
        iv = tv * tm.tile_v + (threadIdx.x >> 4);
    }
    const bool active = iu < (int)nu && iv < (int)nv;
    // Pixel-index rectangle of the tile, widened by half a pixel for sub-rays.
    const double tu0 = tu * tm.tile_u - 0.5, tu1 = min((int)nu, (tu + 1) * tm.tile_u) - 0.5;
    const double tv0 = tv * tm.tile_v - 0.5, tv1 = min((int)nv, (tv + 1) * tm.tile_v) - 0.5;

    const aprict_proj_spec sp = specs[view];
    ViewGeom g;
    view_geom(sp, g);

    const int n_chunks = (n_shapes + kChunk - 1) / kChunk;
    const double inv_su = 1.0 / (double)ssu, inv_sv = 1.0 / (double)ssv;
    float totval = 0.f;
    bool ovf = false;
    int cached_chunk = -1;
    for (int ku = 0; ku < ssu; ++ku) {
        float accumulator = 0.f;
        for (int kv = 0; kv < ssv; ++kv) {
            const double fu = (double)iu - 0.5 + inv_su * (ku + 0.5);
            const double fv = (double)iv - 0.5 + inv_sv * (kv + 0.5);
            const ab_d3 dw = g.D0 + g.U * fu + g.V * fv;  // pixel - source (world)
            const double seglen = sqrt(ab_dot(dw, dw));
            double val = 0.0;
            double uL[MODE == 0 ? kMaxU : 1], uR[MODE == 0 ? kMaxU : 1];
            int m = 0;
            for (int cc = 0; cc < n_chunks; ++cc) {
                const int c = MODE == 0 ? n_chunks - 1 - cc : cc;  // later shapes first when they win
                if (c != cached_chunk) {
                    // Cull this chunk's shapes against the tile; keep order.
                    __syncthreads();
                    const int j = c * kChunk + (int)threadIdx.x;
                    bool keep = false;
                    if (PRE) {  // precomputed per view (k_forbild_prep)
                        if (threadIdx.x < kChunk && j < n_shapes) {
                            const QCull cr = pcull[(size_t)blockIdx.y * (size_t)n_shapes + (size_t)j];
                            keep = cr.live && (cr.keep_all || (cr.u1 >= tu0 - 1e-6 && cr.u0 <= tu1 + 1e-6 &&
                                                               cr.v1 >= tv0 - 1e-6 && cr.v0 <= tv1 + 1e-6));
                        }
                    } else if (threadIdx.x < kChunk && j < n_shapes && shapes[j].kind != 0) {  // derived here
                        double u0, u1, v0, v1;
                        keep = !footprint(g, shapes[j], u0, u1, v0, v1) ||
                               (u1 >= tu0 - 1e-6 && u0 <= tu1 + 1e-6 && v1 >= tv0 - 1e-6 && v0 <= tv1 + 1e-6);
                    }
                    const unsigned bal = __ballot_sync(0xffffffffu, keep);
                    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
                    if (lane == 0) s_warp_pos[w] = __popc(bal);
                    __syncthreads();
                    if (threadIdx.x == 0) {
                        int acc = 0;
                        for (int k = 0; k < kThreads / 32; ++k) {
                            const int t = s_warp_pos[k];
                            s_warp_pos[k] = acc;
                            acc += t;
                        }
                        s_count = acc;
                    }
                    __syncthreads();
                    if (keep) {
                        const int pos = s_warp_pos[w] + __popc(bal & ((1u << lane) - 1u));
                        if constexpr (PRE)
                            sel[pos] = pqv[(size_t)blockIdx.y * (size_t)n_shapes + (size_t)j];
                        else
                            make_qview(g, shapes[j], sel[pos]);
                    }
                    __syncthreads();
                    cached_chunk = n_chunks == 1 ? c : -1;
                }
                const int cnt = s_count;
                if (active) {
                    for (int kk = 0; kk < cnt; ++kk) {
                        const QView &q = sel[MODE == 0 ? cnt - 1 - kk : kk];
                        double lo, hi;
                        if (!ray_interval(q, fu, fv, lo, hi)) continue;
                        if (MODE != 0) {
                            val += q.rho * (hi - lo);
                            continue;
                        }
                        double covered = 0.0;
                        for (int i = 0; i < m; ++i) covered += fmax(0.0, fmin(hi, uR[i]) - fmax(lo, uL[i]));
                        val += q.rho * ((hi - lo) - covered);
                        double a = lo, b = hi;
                        int wpos = 0;
                        for (int i = 0; i < m; ++i) {
                            if (uR[i] < a || uL[i] > b) {
                                uL[wpos] = uL[i];
                                uR[wpos] = uR[i];
                                ++wpos;
                            } else {
                                a = fmin(a, uL[i]);
                                b = fmax(b, uR[i]);
                            }
                        }
                        if (wpos < kMaxU) {
                            uL[wpos] = a;
                            uR[wpos] = b;
                            m = wpos + 1;
                        } else {
                            m = wpos;
                            ovf = true;
                        }
                    }
                }
            }
            // priority and line-integral modes are lengths along the segment
            float v = (float)(MODE == 1 ? val : val * seglen);
            v *= mba;
            accumulator += v;
        }
        if (ssv > 1) accumulator /= (float)ssv;
        totval += accumulator;
    }
    if (ssu > 1) totval /= (float)ssu;
    if (!active) return;
    if (ovf && overflow) atomicAdd(overflow, 1u);
    atomicAdd(out + (int64_t)view * ps.view + (int64_t)iu * ps.u + (int64_t)iv * ps.v, totval);
}

}  // namespace

extern "C" int aprict_b200_project_forbild(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                           float *projs_dev, const aprict_quadric *shapes_dev, int64_t n_shapes,
                                           float mba, uint32_t ssu, uint32_t ssv, int mode, uint32_t *overflow_dev,
                                           uint32_t *status_dev, aprict_stream_t stream) {
    (void)status_dev;
    int rc;
    if ((rc = ab_check_projs(pd, projs_dev, "projections")) != APRICT_OK) return rc;
    if (mode < 0 || mode > 2) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "project_forbild: mode must be 0, 1 or 2");
    if (ssu == 0 || ssv == 0 || ssu > 64 || ssv > 64)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ssu/ssv must be in [1, 64]");
    if (!isfinite(mba)) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "non-finite multiply_before_adding");
    if (n_shapes < 0 || n_shapes > (1 << 24)) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "bad shape count");
    if (pd->n_views == 0 || pd->nu == 0 || pd->nv == 0 || n_shapes == 0) return APRICT_OK;
    if (specs_dev == nullptr || shapes_dev == nullptr)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "project_forbild: null pointer");
    const TileMap tm = make_tiles(pd->nu, pd->nv);
    const ab_pstrides ps{pd->stride_view, pd->stride_u, pd->stride_v};
    const size_t smem = (size_t)kChunk * sizeof(QView);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    auto *kd = mode == 0 ? k_project_forbild<0, false>
                         : (mode == 1 ? k_project_forbild<1, false> : k_project_forbild<2, false>);
    auto *kp = mode == 0 ? k_project_forbild<0, true>
                         : (mode == 1 ? k_project_forbild<1, true> : k_project_forbild<2, true>);
    for (auto *kk : {kd, kp}) {
        rc = ab_cuda_check(cudaFuncSetAttribute(kk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                           "project_forbild smem");
        if (rc != APRICT_OK) return rc;
    }
    // Views in groups whose per-(view, shape) records fit 256 MB of
    // stream-ordered scratch; without scratch every tile derives them itself.
    const size_t rec = sizeof(QCull) + sizeof(QView);
    uint64_t per = (256ull << 20) / ((uint64_t)n_shapes * rec);
    per = per < 1 ? 1 : (per > 65535u ? 65535u : per);
    const uint32_t group = (uint32_t)(per < pd->n_views ? per : pd->n_views);
    void *scratch = nullptr;
    if (cudaMallocAsync(&scratch, (size_t)group * (size_t)n_shapes * rec, st) != cudaSuccess) {
        (void)cudaGetLastError();
        scratch = nullptr;
    }
    QCull *cull = static_cast<QCull *>(scratch);
    QView *qv = scratch ? reinterpret_cast<QView *>(cull + (size_t)group * (size_t)n_shapes) : nullptr;
    for (uint32_t v0 = 0; v0 < pd->n_views && rc == APRICT_OK; v0 += group) {
        const uint32_t nvw = pd->n_views - v0 < group ? pd->n_views - v0 : group;
        if (scratch) {
            k_forbild_prep<<<dim3((unsigned)((n_shapes + 127) / 128), nvw), 128, 0, st>>>(
                specs_dev, v0, nvw, shapes_dev, (int)n_shapes, cull, qv);
            rc = ab_cuda_check(cudaGetLastError(), "project_forbild prep launch");
            if (rc != APRICT_OK) break;
        }
        dim3 grid((unsigned)(tm.ntu * tm.ntv), nvw);
        (scratch ? kp : kd)<<<grid, kThreads, smem, st>>>(specs_dev, pd->n_views, pd->nu, pd->nv, ps, projs_dev,
                                                          shapes_dev, (int)n_shapes, mba, (int)ssu, (int)ssv, tm, v0,
                                                          overflow_dev, cull, qv);
        rc = ab_cuda_check(cudaGetLastError(), "project_forbild launch");
    }
    if (scratch) cudaFreeAsync(scratch, st);
    return rc;
}

// ---------------------------------------------------------------------------
// Point sampling ("last shape wins") -- replaces add_FORBILD_sampling
// (src/aprict/data/cusrc/sample_FORBILD_volumes.cu:10-123): per voxel and
// sub-sample the value is the density of the last shape (in order) that
// contains the point, 0 if none; the mean over the sub-samples is added to
// the output. Each CTA (an 8 x 8 x 4 voxel block) first keeps, in order, the
// shapes whose bounding boxes meet its own box, 256 at a time.

namespace {

// Closed solids, as the reference's _in_region (FORBILD_volumes.h); the
// strict clip planes (">") exclude their plane.
__device__ __forceinline__ bool in_quadric(const aprict_quadric &q, double px, double py, double pz) {
    const int nc = q.n_clip & 0xFF;
    for (int k = 0; k < nc; ++k) {
        const double g = q.clip[k][0] * px + q.clip[k][1] * py + q.clip[k][2] * pz - q.clip[k][3];
        if ((q.n_clip >> (8 + k)) & 1 ? !(g < 0.0) : !(g <= 0.0)) return false;
    }
    const double dx = px - q.c[0], dy = py - q.c[1], dz = pz - q.c[2];
    const double lx = q.M[0] * dx + q.M[1] * dy + q.M[2] * dz;
    const double ly = q.M[3] * dx + q.M[4] * dy + q.M[5] * dz;
    const double lz = q.M[6] * dx + q.M[7] * dy + q.M[8] * dz;
    switch (q.kind) {
        case 1: return lx * lx + ly * ly + lz * lz <= 1.0;
        case 2: return fabs(lz) <= q.h && lx * lx + ly * ly <= 1.0;
        case 3: {
            const double r = q.alpha + q.beta * lz;
            return fabs(lz) <= q.h && lx * lx + ly * ly <= r * r;
        }
        case 4: return fabs(lx) <= 1.0 && fabs(ly) <= 1.0 && fabs(lz) <= 1.0;
        default: return false;
    }
}

constexpr int kSampleThreads = 256;  // 8 (x) x 8 (y) x 4 (z) voxels

__global__ void __launch_bounds__(kSampleThreads) k_forbild_sample(const aprict_quadric *__restrict__ shapes, int n,
                                                                    const float *__restrict__ xs,
                                                                    const float *__restrict__ ys,
                                                                    const float *__restrict__ zs, int nx, int ny,
                                                                    int nz, int64_t sx, int64_t sy, int64_t sz,
                                                                    float *out, float ss_wid, int ss) {
    __shared__ int keep[kSampleThreads];
    __shared__ int nkeep;
    __shared__ float box[6];  // CTA box: min x y z, max x y z
    const int t = threadIdx.x;
    const int bx = blockIdx.x * 8, by = blockIdx.y * 8, bz = blockIdx.z * 4;
    const int ix = bx + (t & 7), iy = by + ((t >> 3) & 7), iz = bz + (t >> 6);
    const bool inr = ix < nx && iy < ny && iz < nz;
    // The block's box from its coordinates (grids need not be monotonic).
    if (t < 32) {
        const int lane = t;
        float lo[3], hi[3];
        const float *arr[3] = {xs, ys, zs};
        const int b0[3] = {bx, by, bz}, ext[3] = {8, 8, 4}, nn[3] = {nx, ny, nz};
        for (int a = 0; a < 3; ++a) {
            const int i = b0[a] + (lane % ext[a]);
            const float v = i < nn[a] ? arr[a][i] : arr[a][b0[a]];
            float mn = v, mx = v;
            for (int o = 16; o > 0; o >>= 1) {
                mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            }
            lo[a] = mn;
            hi[a] = mx;
        }
        if (lane == 0) {
            const float hw = 0.5f * ss_wid;
            for (int a = 0; a < 3; ++a) {
                box[a] = lo[a] - hw;
                box[3 + a] = hi[a] + hw;
            }
        }
    }
    const double cx = inr ? (double)xs[ix] : 0.0, cy = inr ? (double)ys[iy] : 0.0, cz = inr ? (double)zs[iz] : 0.0;
    float total = 0.f;
    for (int s = 0; s < ss * ss * ss; ++s) {
        const int ox = s / (ss * ss), oy = (s / ss) % ss, oz = s % ss;
        const double px = cx + ((ox - 0.5 * (ss - 1)) / ss) * (double)ss_wid;
        const double py = cy + ((oy - 0.5 * (ss - 1)) / ss) * (double)ss_wid;
        const double pz = cz + ((oz - 0.5 * (ss - 1)) / ss) * (double)ss_wid;
        float val = 0.f;
        for (int base = 0; base < n; base += kSampleThreads) {
            __syncthreads();  // box ready; the previous chunk's list is consumed
            const int j = base + t;
            bool meet = false;
            if (j < n && shapes[j].kind != 0) {
                const aprict_quadric &q = shapes[j];
                meet = true;
                for (int a = 0; a < 3; ++a)
                    meet = meet && q.c[a] - q.bb_half[a] <= (double)box[3 + a] && q.c[a] + q.bb_half[a] >= (double)box[a];
            }
            // ordered compaction: warp ballots, then warp offsets
            const unsigned bal = __ballot_sync(0xffffffffu, meet);
            __shared__ int wcount[kSampleThreads / 32];
            if ((t & 31) == 0) wcount[t >> 5] = __popc(bal);
            __syncthreads();
            if (meet) {
                int off = __popc(bal & ((1u << (t & 31)) - 1u));
                for (int w = 0; w < (t >> 5); ++w) off += wcount[w];
                keep[off] = j;
            }
            if (t == 0) {
                int c = 0;
                for (int w = 0; w < kSampleThreads / 32; ++w) c += wcount[w];
                nkeep = c;
            }
            __syncthreads();
            if (inr) {
                const int c = nkeep;
                for (int i = 0; i < c; ++i) {
                    const aprict_quadric &q = shapes[keep[i]];
                    if (in_quadric(q, px, py, pz)) val = (float)q.rho;
                }
            }
        }
        total += val;
    }
    if (!inr || total == 0.f) return;
    total /= (float)(ss * ss * ss);
    atomicAdd(out + (int64_t)ix * sx + (int64_t)iy * sy + (int64_t)iz * sz, total);
}

}  // namespace

extern "C" int aprict_b200_forbild_sample(const aprict_quadric *shapes_dev, int64_t n_shapes, const float *xs_dev,
                                          const float *ys_dev, const float *zs_dev, uint32_t nx, uint32_t ny,
                                          uint32_t nz, int64_t stride_x, int64_t stride_y, int64_t stride_z,
                                          float *out_dev, float supersamp_voxwid, uint32_t supersamp_factor,
                                          aprict_stream_t stream) {
    if (n_shapes < 0 || n_shapes > (1 << 24)) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "bad shape count");
    if (supersamp_factor == 0 || supersamp_factor > 8)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "supersamp_factor must be in [1, 8]");
    if (!isfinite(supersamp_voxwid) || supersamp_voxwid < 0.f)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "supersamp_cubic_vox_wid must be finite and >= 0");
    if (nx == 0 || ny == 0 || nz == 0 || n_shapes == 0) return APRICT_OK;
    if (nx > (1u << 30) || ny > (1u << 30) || nz > (1u << 30))
        return ab_fail(APRICT_ERR_TOO_LARGE, "forbild_sample: grid edge exceeds 2^30");
    if (shapes_dev == nullptr || xs_dev == nullptr || ys_dev == nullptr || zs_dev == nullptr || out_dev == nullptr)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "forbild_sample: null pointer");
    if (stride_x < 0 || stride_y < 0 || stride_z < 0)
        return ab_fail(APRICT_ERR_UNSUPPORTED, "forbild_sample: negative strides are not supported");
    const dim3 grid((nx + 7) / 8, (ny + 7) / 8, (nz + 3) / 4);
    if (grid.y > 65535u || grid.z > 65535u) return ab_fail(APRICT_ERR_TOO_LARGE, "forbild_sample: grid too large");
    k_forbild_sample<<<grid, kSampleThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        shapes_dev, (int)n_shapes, xs_dev, ys_dev, zs_dev, (int)nx, (int)ny, (int)nz, stride_x, stride_y, stride_z,
        out_dev, supersamp_voxwid, (int)supersamp_factor);
    return ab_cuda_check(cudaGetLastError(), "forbild_sample launch");
}
