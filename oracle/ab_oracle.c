/* ab_oracle.c -- FP64 CPU restatement of the reference's projection and
 * backprojection arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY. The checker for the CUDA kernels: tests/,
 * __graft_entry__.smoke() and bench.py's CPU baseline load it; the
 * aprict_b200 package never does.
 *
 * The line integral is the one exact_line_integral_unitvoxwid computes
 * (src/aprict/data/cusrc/CB_project_texture_chunked.cu:111-306), restated as
 * Siddon's original parametric form: all voxel-boundary crossings along the
 * source->pixel segment are generated in order, and each piece between two
 * consecutive crossings is charged to the voxel containing its midpoint. Every
 * quantity is double; nothing is stepped incrementally. Tie rules follow the
 * reference: with a zero direction component the voxel along that axis is
 * ceil(c)-1 (reference :189-203, :244-246).
 *
 * The voxel-driven backprojector follows _backproject_CB_getval
 * (src/aprict/data/cusrc/CB_backproject.cu:313-733) for weighting presets 0-6.
 */
#include "ab_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double x, y, z;
} d3;

static d3 d3f(ao_fvec3 v) { return (d3){v.x, v.y, v.z}; }
static d3 add(d3 a, d3 b) { return (d3){a.x + b.x, a.y + b.y, a.z + b.z}; }
static d3 sub(d3 a, d3 b) { return (d3){a.x - b.x, a.y - b.y, a.z - b.z}; }
static d3 scl(d3 a, double s) { return (d3){a.x * s, a.y * s, a.z * s}; }
static double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double nrm(d3 a) { return sqrt(dot(a, a)); }
static d3 cross(d3 a, d3 b) { return (d3){a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

static int64_t vidx(const ao_grid *g, int ix, int iy, int iz) {
    if (g->order == 0) return ((int64_t)ix * g->ny + iy) * g->nz + iz;
    return ((int64_t)iz * g->ny + iy) * g->nx + ix;
}

/* Pixel (fractional index fu, fv) centre in world units. */
static d3 pixel_pos(const ao_proj_spec *sp, double fu, double fv) {
    const double xn = fu - ((double)sp->nu - 1.0) * 0.5;
    const double yn = fv - ((double)sp->nv - 1.0) * 0.5;
    return add(d3f(sp->det_pos), add(scl(d3f(sp->det_u), xn), scl(d3f(sp->det_v), yn)));
}

typedef void (*visit_fn)(void *ctx, double seg, int ix, int iy, int iz);

/* Visits every piece of the ray o + a (e - o), a in [0, a_max], inside the
 * grid [0,n)^3 (voxel units). Returns |e - o| (0 if the ray misses). */
static double traverse(const double o[3], const double e[3], const int n[3], double a_max, visit_fn f, void *ctx) {
    double d[3], a_in = 0.0, a_out = a_max;
    for (int a = 0; a < 3; ++a) {
        d[a] = e[a] - o[a];
        if (d[a] == 0.0) {
            if (!(o[a] > 0.0 && o[a] <= (double)n[a])) return 0.0;
        } else {
            const double t0 = (0.0 - o[a]) / d[a], t1 = ((double)n[a] - o[a]) / d[a];
            const double lo = t0 < t1 ? t0 : t1, hi = t0 < t1 ? t1 : t0;
            if (lo > a_in) a_in = lo;
            if (hi < a_out) a_out = hi;
        }
    }
    const double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (!(a_in < a_out)) return 0.0;
    double nxt[3];
    double bnd[3];
    int fixed[3];
    for (int a = 0; a < 3; ++a) {
        if (d[a] == 0.0) {
            nxt[a] = INFINITY;
            bnd[a] = 0.0;
            fixed[a] = (int)ceil(o[a]) - 1;
        } else {
            const double p = o[a] + a_in * d[a];
            bnd[a] = d[a] > 0.0 ? floor(p) + 1.0 : ceil(p) - 1.0;
            nxt[a] = (bnd[a] - o[a]) / d[a];
            fixed[a] = 0;
        }
    }
    double prev = a_in;
    for (;;) {
        double t = a_out;
        for (int a = 0; a < 3; ++a)
            if (nxt[a] < t) t = nxt[a];
        if (t > prev) {
            const double mid = 0.5 * (prev + t);
            int idx[3];
            for (int a = 0; a < 3; ++a) {
                idx[a] = d[a] == 0.0 ? fixed[a] : (int)floor(o[a] + mid * d[a]);
                if (idx[a] < 0) idx[a] = 0;
                if (idx[a] >= n[a]) idx[a] = n[a] - 1;
            }
            f(ctx, t - prev, idx[0], idx[1], idx[2]);
        }
        if (t >= a_out) break;
        for (int a = 0; a < 3; ++a) {
            if (nxt[a] <= t) {
                bnd[a] += d[a] > 0.0 ? 1.0 : -1.0;
                nxt[a] = (bnd[a] - o[a]) / d[a];
            }
        }
        prev = t;
    }
    return len;
}

typedef struct {
    const float *vol;
    const ao_grid *g;
    double acc;
    int64_t nseg;
} gather_ctx;

static void gather_visit(void *c, double seg, int ix, int iy, int iz) {
    gather_ctx *x = (gather_ctx *)c;
    x->acc += seg * (double)x->vol[vidx(x->g, ix, iy, iz)];
    x->nseg++;
}

static void to_grid(const ao_grid *g, d3 p, double out[3]) {
    out[0] = (p.x - g->corner[0]) / g->voxwid;
    out[1] = (p.y - g->corner[1]) / g->voxwid;
    out[2] = (p.z - g->corner[2]) / g->voxwid;
}

void ao_project_siddon(const ao_proj_spec *specs, int n_views, int nu, int nv, const float *vol, const ao_grid *g,
                       double svf, double mba, int ssu, int ssv, double *out, int64_t *nseg, int nthreads) {
    const int n[3] = {g->nx, g->ny, g->nz};
    int64_t total = 0;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for collapse(2) schedule(dynamic, 4) reduction(+ : total)
    for (int m = 0; m < n_views; ++m) {
        for (int iu = 0; iu < nu; ++iu) {
            const ao_proj_spec *sp = &specs[m];
            double o[3];
            to_grid(g, scl(d3f(sp->source_pos), svf), o);
            for (int iv = 0; iv < nv; ++iv) {
                double tot = 0.0;
                for (int ku = 0; ku < ssu; ++ku) {
                    double accu = 0.0;
                    for (int kv = 0; kv < ssv; ++kv) {
                        const double fu = iu - 0.5 + (ku + 0.5) / ssu, fv = iv - 0.5 + (kv + 0.5) / ssv;
                        double e[3];
                        to_grid(g, scl(pixel_pos(sp, fu, fv), svf), e);
                        gather_ctx c = {vol, g, 0.0, 0};
                        const double len = traverse(o, e, n, 1.0, gather_visit, &c);
                        accu += mba * g->voxwid * len * c.acc;
                        total += c.nseg;
                    }
                    tot += accu / ssv;
                }
                out[((int64_t)m * nu + iu) * nv + iv] += tot / ssu;
            }
        }
    }
    if (nseg) *nseg = total;
}

typedef struct {
    double *vol;
    const ao_grid *g;
    double w;
} scatter_ctx;

static void scatter_visit(void *c, double seg, int ix, int iy, int iz) {
    scatter_ctx *x = (scatter_ctx *)c;
    x->vol[vidx(x->g, ix, iy, iz)] += seg * x->w;
}

static double *alloc_private(int nthr, int64_t nvox) {
    return (double *)calloc((size_t)nthr * (size_t)nvox, sizeof(double));
}

void ao_backproject_transpose(const ao_proj_spec *specs, int n_views, int nu, int nv, const double *projs,
                              const ao_grid *g, double svf, double mba, int ssu, int ssv, double *vol,
                              int nthreads) {
    const int n[3] = {g->nx, g->ny, g->nz};
    const int64_t nvox = (int64_t)g->nx * g->ny * g->nz;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const int nthr = omp_get_max_threads();
    double *priv = alloc_private(nthr, nvox);
#pragma omp parallel
    {
        double *mine = priv + (int64_t)omp_get_thread_num() * nvox;
#pragma omp for collapse(2) schedule(dynamic, 4)
        for (int m = 0; m < n_views; ++m) {
            for (int iu = 0; iu < nu; ++iu) {
                const ao_proj_spec *sp = &specs[m];
                double o[3];
                to_grid(g, scl(d3f(sp->source_pos), svf), o);
                for (int iv = 0; iv < nv; ++iv) {
                    const double p = projs[((int64_t)m * nu + iu) * nv + iv];
                    if (p == 0.0) continue;
                    for (int ku = 0; ku < ssu; ++ku) {
                        for (int kv = 0; kv < ssv; ++kv) {
                            const double fu = iu - 0.5 + (ku + 0.5) / ssu, fv = iv - 0.5 + (kv + 0.5) / ssv;
                            double e[3];
                            to_grid(g, scl(pixel_pos(sp, fu, fv), svf), e);
                            const double dd[3] = {e[0] - o[0], e[1] - o[1], e[2] - o[2]};
                            const double len = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
                            scatter_ctx c = {mine, g, p * mba * g->voxwid * len / (ssu * ssv)};
                            traverse(o, e, n, 1.0, scatter_visit, &c);
                        }
                    }
                }
            }
        }
    }
    for (int t = 0; t < nthr; ++t) {
        const double *src = priv + (int64_t)t * nvox;
        for (int64_t i = 0; i < nvox; ++i) vol[i] += src[i];
    }
    free(priv);
}

/* ---- voxel-driven backprojection (CB_backproject.cu:313-733) ---- */

static double powint(double b, int e) {
    double a = 1.0;
    if (e < 0)
        for (int k = 0; k < -e; ++k) a /= b;
    else
        for (int k = 0; k < e; ++k) a *= b;
    return a;
}

/* get_projected_detector_coords (geometry.h:24-56), FP64: coordinates from the
 * detector centre in pixels. */
static void det_coords(const ao_proj_spec *sp, d3 x, double *cu, double *cv) {
    const d3 s = d3f(sp->source_pos), P = d3f(sp->det_pos), U = d3f(sp->det_u), V = d3f(sp->det_v);
    const d3 n = cross(U, V);
    d3 p = add(s, scl(sub(x, s), dot(sub(P, s), n) / dot(sub(x, s), n)));
    p = sub(p, P);
    *cu = dot(U, p) / dot(U, U);
    *cv = dot(V, p) / dot(V, V);
}

static double get2d(const double *img, int nu, int nv, int i, int j) {
    if (i < 0 || i >= nu || j < 0 || j >= nv) return 0.0;
    return img[(int64_t)i * nv + j];
}

static double taper(double cu, double cv, int nu, int nv, double sep) {
    double ud = fabs(cu) / (nu / 2.0), vd = fabs(cv) / (nv / 2.0);
    ud = fmax(0.0, fmin(1.0, (1.0 - ud) / sep));
    vd = fmax(0.0, fmin(1.0, (1.0 - vd) / sep));
    ud = fmax(0.0, fmin(1.0, (1.0 + cos(M_PI * (1.0 - ud))) / 2.0));
    vd = fmax(0.0, fmin(1.0, (1.0 + cos(M_PI * (1.0 - vd))) / 2.0));
    return ud * vd;
}

static d3 voxel_centre(const ao_grid *g, int ix, int iy, int iz) {
    return (d3){g->corner[0] + (ix + 0.5) * g->voxwid, g->corner[1] + (iy + 0.5) * g->voxwid,
                g->corner[2] + (iz + 0.5) * g->voxwid};
}

/* Cone-cylinder weighting presets of the direct-raycast mode
 * (CB_backproject.cu:530-599), R = config val; x the voxel, s the source,
 * Z = (x - s).L / |L|. */
static double preset_weight(int preset, double R, d3 x, d3 s, double Z) {
    const d3 rs = sub(x, s);
    const double ell = sqrt(rs.x * rs.x + rs.y * rs.y) / R;
    const double zr = Z / R;
    const double c = fmax(0.0, fmin(1.0, fabs(zr / ell)));
    const double d = c - ell;
    const double vy = (s.x * x.y - s.y * x.x) / R / R, vx = (s.x * x.x + s.y * x.y) / R / R;
    const double dc = d / c;
    const double q = (1.0 - dc * dc) / (1.0 + dc * dc);
    switch (preset) {
        case 1: return 1.0 / (c * c * (c * c + d * d));
        case 2: return -2.0 * q * q * (-vy) * (1.0 + vx / zr) / (ell * ell) / R * R;
        case 3: return 1.0 / (zr * c * c);
        case 4: return (vy / zr) / zr;
        case 6: return -2.0 * q * q / (1.0 - dc) * (-vy) * (1.0 + vx / zr) / zr;
        default: return 1.0; /* preset 5 carries no extra factor */
    }
}

/* Value one (sub-)voxel at x receives from view m in fast mode. */
static double fast_value(const ao_proj_spec *sp, const double *img, d3 x, double voxwid, const ao_bp_cfg *c) {
    const d3 s = d3f(sp->source_pos), P = d3f(sp->det_pos), U = d3f(sp->det_u), V = d3f(sp->det_v);
    const int nu = (int)sp->nu, nv = (int)sp->nv;
    double cu, cv;
    det_coords(sp, x, &cu, &cv);
    const double fu = cu + (nu - 1) / 2.0, fv = cv + (nv - 1) / 2.0;
    const d3 L = sub(P, s);
    double mult, value;
    double pv;
    if (c->linear) {
        if (fu <= -1 || fv <= -1 || fu >= nu || fv >= nv) {
            pv = 0.0;
        } else {
            const int i0 = (int)floor(fu), j0 = (int)floor(fv);
            const double fx = fu - i0, fy = fv - j0;
            const double t1 = get2d(img, nu, nv, i0, j0) * (1 - fx) + get2d(img, nu, nv, i0 + 1, j0) * fx;
            const double t2 = get2d(img, nu, nv, i0, j0 + 1) * (1 - fx) + get2d(img, nu, nv, i0 + 1, j0 + 1) * fx;
            pv = t1 * (1 - fy) + t2 * fy;
        }
    } else {
        pv = get2d(img, nu, nv, (int)floor(fu + 0.5), (int)floor(fv + 0.5));
    }
    if (c->raycast) {
        mult = 1.0;
        const double Z = dot(sub(x, s), L) / nrm(L);
        if (c->pL) mult *= powint(Z / nrm(L), c->pL);
        if (c->pV) mult *= powint(Z / c->val, c->pV);
        if (c->preset >= 1 && c->preset <= 6) mult *= preset_weight(c->preset, c->val, x, s, Z);
        value = pv * mult;
    } else {
        const d3 detp = add(P, add(scl(U, cu), scl(V, cv)));
        const double mag = nrm(sub(detp, s)) / nrm(sub(x, s)) * voxwid;
        mult = mag * mag / (nrm(U) * nrm(V));
        if (c->pL) mult *= powint(dot(sub(x, s), L) / dot(L, L), c->pL);
        if (c->pV) mult *= powint(dot(scl(sub(x, s), 1.0 / c->val), L) / nrm(L), c->pV);
        value = voxwid * pv * mult;
    }
    if (c->sep > 0 && value != 0.0) value *= taper(cu, cv, nu, nv, c->sep);
    return value;
}

static int masked(const ao_grid *g, const ao_bp_cfg *c, int ix, int iy, int iz) {
    if (!c->mask) return 0;
    const d3 x = voxel_centre(g, ix, iy, iz);
    return x.x * x.x + x.y * x.y > c->mask_rad * c->mask_rad;
}

/* Nearest-pixel choices that FP64 cannot settle: per voxel, the number of
 * (sub-sample, view) pairs of the fast nearest mode whose detector coordinate
 * (fu or fv, in pixel indices, inside the detector) lies within eps of a
 * half-integer, where floor(f + 1/2) flips with the rounding of the
 * coordinate's evaluation. Symmetric geometries make them exact in real
 * arithmetic (voxel centres projecting onto pixel boundaries); any two FP64
 * evaluations may then pick different neighbours. */
void ao_bp_nearest_ties(const ao_proj_spec *specs, int n_views, const ao_grid *g, const ao_bp_cfg *c, double eps,
                        int32_t *counts, int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for collapse(2) schedule(dynamic, 2)
    for (int ix = 0; ix < g->nx; ++ix) {
        for (int iy = 0; iy < g->ny; ++iy) {
            for (int iz = 0; iz < g->nz; ++iz) {
                const int64_t o = vidx(g, ix, iy, iz);
                counts[o] = 0;
                if (masked(g, c, ix, iy, iz)) continue;
                const d3 xc = voxel_centre(g, ix, iy, iz);
                int cnt = 0;
                for (int si = 0; si < c->ssx; ++si)
                    for (int sj = 0; sj < c->ssy; ++sj)
                        for (int sk = 0; sk < c->ssz; ++sk) {
                            const d3 x = add(xc, scl((d3){-0.5 + (si + 0.5) / c->ssx, -0.5 + (sj + 0.5) / c->ssy,
                                                          -0.5 + (sk + 0.5) / c->ssz},
                                                     g->voxwid));
                            for (int m = 0; m < n_views; ++m) {
                                const int nu = (int)specs[m].nu, nv = (int)specs[m].nv;
                                double cu, cv;
                                det_coords(&specs[m], x, &cu, &cv);
                                const double fu = cu + (nu - 1) / 2.0, fv = cv + (nv - 1) / 2.0;
                                if (!(fu > -1.0 && fu < nu && fv > -1.0 && fv < nv)) continue;
                                const double du = fabs(fu - floor(fu) - 0.5), dv = fabs(fv - floor(fv) - 0.5);
                                if (du < eps || dv < eps) ++cnt;
                            }
                        }
                counts[o] = cnt;
            }
        }
    }
}

void ao_backproject(const ao_proj_spec *specs, int n_views, int nu, int nv, const double *projs,
                    const ao_grid *g, const double *mult, const ao_bp_cfg *c, double *vol, int nthreads) {
    const int64_t nvox = (int64_t)g->nx * g->ny * g->nz;
    const int64_t img = (int64_t)nu * nv;
    const double inv_ss = 1.0 / ((double)c->ssx * c->ssy * c->ssz);
    if (nthreads > 0) omp_set_num_threads(nthreads);
    if (!c->exact) {
#pragma omp parallel for collapse(2) schedule(dynamic, 2)
        for (int ix = 0; ix < g->nx; ++ix) {
            for (int iy = 0; iy < g->ny; ++iy) {
                for (int iz = 0; iz < g->nz; ++iz) {
                    if (masked(g, c, ix, iy, iz)) continue;
                    const d3 xc = voxel_centre(g, ix, iy, iz);
                    double acc = 0.0;
                    for (int si = 0; si < c->ssx; ++si)
                        for (int sj = 0; sj < c->ssy; ++sj)
                            for (int sk = 0; sk < c->ssz; ++sk) {
                                const d3 x = add(xc, scl((d3){-0.5 + (si + 0.5) / c->ssx, -0.5 + (sj + 0.5) / c->ssy,
                                                              -0.5 + (sk + 0.5) / c->ssz},
                                                         g->voxwid));
                                for (int m = 0; m < n_views; ++m)
                                    acc += fast_value(&specs[m], projs + m * img, x, g->voxwid, c);
                            }
                    const int64_t o = vidx(g, ix, iy, iz);
                    vol[o] += acc * inv_ss * (mult ? mult[o] : 1.0);
                }
            }
        }
        return;
    }
    /* Exact mode: sum over footprint pixels of value * chord(pixel-centre ray,
     * voxel cube) (:408-477) == per view, the transpose of a pixel-centre-ray
     * projection over the voxel grid (rays from the source, unbounded past the
     * detector as the reference's chord is), times the per-voxel weights. */
    const int nthr = omp_get_max_threads();
    double *priv = alloc_private(nthr, nvox);
    double *tmp = alloc_private(nthr, nvox);
    const int n[3] = {g->nx, g->ny, g->nz};
#pragma omp parallel
    {
        double *acc = priv + (int64_t)omp_get_thread_num() * nvox;
        double *T = tmp + (int64_t)omp_get_thread_num() * nvox;
#pragma omp for schedule(dynamic, 1)
        for (int m = 0; m < n_views; ++m) {
            const ao_proj_spec *sp = &specs[m];
            const d3 s = d3f(sp->source_pos), L = sub(d3f(sp->det_pos), s);
            for (int si = 0; si < c->ssx; ++si)
                for (int sj = 0; sj < c->ssy; ++sj)
                    for (int sk = 0; sk < c->ssz; ++sk) {
                        const d3 off = scl((d3){-0.5 + (si + 0.5) / c->ssx, -0.5 + (sj + 0.5) / c->ssy,
                                                -0.5 + (sk + 0.5) / c->ssz},
                                           g->voxwid);
                        ao_grid gs = *g;
                        gs.corner[0] += off.x;
                        gs.corner[1] += off.y;
                        gs.corner[2] += off.z;
                        memset(T, 0, sizeof(double) * (size_t)nvox);
                        double o[3];
                        to_grid(&gs, s, o);
                        for (int iu = 0; iu < nu; ++iu)
                            for (int iv = 0; iv < nv; ++iv) {
                                const double p = c->all_ones ? 1.0 : projs[m * img + (int64_t)iu * nv + iv];
                                if (p == 0.0) continue;
                                double e[3];
                                to_grid(&gs, pixel_pos(sp, iu, iv), e);
                                const double dd[3] = {e[0] - o[0], e[1] - o[1], e[2] - o[2]};
                                const double len = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
                                scatter_ctx sc = {T, &gs, p * len * g->voxwid};
                                traverse(o, e, n, INFINITY, scatter_visit, &sc);
                            }
                        for (int ix = 0; ix < g->nx; ++ix)
                            for (int iy = 0; iy < g->ny; ++iy)
                                for (int iz = 0; iz < g->nz; ++iz) {
                                    const int64_t i = vidx(g, ix, iy, iz);
                                    if (T[i] == 0.0 || masked(g, c, ix, iy, iz)) continue;
                                    const d3 x = add(voxel_centre(g, ix, iy, iz), off);
                                    double w = 1.0;
                                    if (c->pL) w *= powint(dot(sub(x, s), L) / dot(L, L), c->pL);
                                    if (c->pV) w *= powint(dot(scl(sub(x, s), 1.0 / c->val), L) / nrm(L), c->pV);
                                    if (c->sep > 0) {
                                        double cu, cv;
                                        det_coords(sp, x, &cu, &cv);
                                        w *= taper(cu, cv, nu, nv, c->sep);
                                    }
                                    acc[i] += T[i] * w * inv_ss;
                                }
                    }
        }
    }
    for (int t = 0; t < nthr; ++t) {
        const double *src = priv + (int64_t)t * nvox;
        for (int64_t i = 0; i < nvox; ++i) vol[i] += src[i] * (mult ? mult[i] : 1.0);
    }
    free(priv);
    free(tmp);
}

/* ---- FORBILD analytic shapes (FORBILD_volumes.h), FP64 ----
 * Each shape type is intersected in its own natural coordinates as the
 * reference structures it: spheres and ellipsoids by a quadratic in the
 * (scaled) frame, cylinders as an axial slab with a radial quadratic, boxes as
 * three slabs, cone frusta as an axial slab with a quadratic for the linearly
 * varying radius; clip planes first (FORBILD_volumes.h:1723-1811). All
 * intervals are parameters along the segment, clamped to [0, 1]. */

typedef struct {
    double lo, hi;
} iv_t;

static void iv_and_lin(iv_t *I, double a, double b) { /* keep a + b t <= 0 */
    if (b == 0.0) {
        if (a > 0.0) I->hi = I->lo - 1.0;
        return;
    }
    const double t = -a / b;
    if (b > 0.0) {
        if (t < I->hi) I->hi = t;
    } else if (t > I->lo) {
        I->lo = t;
    }
}

static void iv_and_slab(iv_t *I, double p, double d, double h) { /* keep |p + t d| <= h */
    iv_and_lin(I, p - h, d);
    iv_and_lin(I, -p - h, -d);
}

/* keep A t^2 + B t + C <= 0 (a convex set for A > 0; for A < 0 the caller's
 * slab keeps one nappe) */
static void iv_and_quad(iv_t *I, double A, double B, double C) {
    if (A == 0.0) {
        iv_and_lin(I, C, B);
        return;
    }
    const double disc = B * B - 4.0 * A * C;
    if (A > 0.0) {
        if (!(disc > 0.0)) {
            I->hi = I->lo - 1.0;
            return;
        }
        const double sq = sqrt(disc);
        const double t0 = (-B - sq) / (2.0 * A), t1 = (-B + sq) / (2.0 * A);
        if (t0 > I->lo) I->lo = t0;
        if (t1 < I->hi) I->hi = t1;
        return;
    }
    if (!(disc > 0.0)) return; /* A < 0, no real roots: q < 0 everywhere */
    const double sq = sqrt(disc);
    double t0 = (-B + sq) / (2.0 * A), t1 = (-B - sq) / (2.0 * A);
    if (t0 > t1) {
        const double x = t0;
        t0 = t1;
        t1 = x;
    }
    /* solution: (-inf, t0] U [t1, inf); within [lo, hi] keep the part that exists */
    const int a_ok = I->lo < fmin(I->hi, t0), b_ok = fmax(I->lo, t1) < I->hi;
    if (a_ok && !b_ok) I->hi = fmin(I->hi, t0);
    if (b_ok && !a_ok) I->lo = fmax(I->lo, t1);
    if (!a_ok && !b_ok) I->hi = I->lo - 1.0;
}

static void unit3(ao_fvec3 v, double o[3]) {
    const double n = sqrt((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
    o[0] = v.x / n;
    o[1] = v.y / n;
    o[2] = v.z / n;
}
static double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* cylinder-like solid: local coords (x, y) scaled to the unit disc, z axial */
static void iv_ecyl(iv_t *I, const double p[3], const double d[3], const double ax[3], double sx, const double ay[3],
                    double sy, const double az[3], double h) {
    const double px = dot3(p, ax) / sx, py = dot3(p, ay) / sy, pz = dot3(p, az);
    const double dx = dot3(d, ax) / sx, dy = dot3(d, ay) / sy, dz = dot3(d, az);
    iv_and_slab(I, pz, dz, h);
    iv_and_quad(I, dx * dx + dy * dy, 2.0 * (px * dx + py * dy), px * px + py * py - 1.0);
}

static void perp2(const double a[3], double e1[3], double e2[3]) {
    const double t[3] = {fabs(a[0]) < 0.9 ? 1.0 : 0.0, fabs(a[0]) < 0.9 ? 0.0 : 1.0, 0.0};
    double c[3] = {a[1] * t[2] - a[2] * t[1], a[2] * t[0] - a[0] * t[2], a[0] * t[1] - a[1] * t[0]};
    const double n = sqrt(dot3(c, c));
    e1[0] = c[0] / n;
    e1[1] = c[1] / n;
    e1[2] = c[2] / n;
    e2[0] = a[1] * e1[2] - a[2] * e1[1];
    e2[1] = a[2] * e1[0] - a[0] * e1[2];
    e2[2] = a[0] * e1[1] - a[1] * e1[0];
}

int ao_forbild_interval(const double v1[3], const double v2[3], const ao_forbild_shape *s, double out2[2]) {
    iv_t I = {0.0, 1.0};
    const double d[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
    out2[0] = out2[1] = 0.0;
    if (s->type == 0) return 0;
    for (int k = 0; k < 3; ++k) {
        const ao_clip *c = &s->cas[k];
        if (c->mode == 0) continue;
        const double a[3] = {c->axis.x, c->axis.y, c->axis.z};
        const double g0 = dot3(a, v1) - c->dotprod, gd = dot3(a, d);
        if (c->mode == 1)
            iv_and_lin(&I, g0, gd);
        else
            iv_and_lin(&I, -g0, -gd);
    }
    if (!(I.lo < I.hi)) return 0;
    const double p[3] = {v1[0] - s->x, v1[1] - s->y, v1[2] - s->z};
    const double ex[3] = {1, 0, 0}, ey[3] = {0, 1, 0}, ez[3] = {0, 0, 1};
    double ax[3], ay[3], az[3];
    switch (s->type) {
        case 13: /* sphere */
            iv_and_quad(&I, dot3(d, d), 2.0 * dot3(p, d), dot3(p, p) - (double)s->r * s->r);
            break;
        case 10: { /* axis-aligned ellipsoid: scale each coordinate */
            const double sc[3] = {s->dx, s->dy, s->dz};
            double pp[3], dd[3];
            for (int i = 0; i < 3; ++i) {
                pp[i] = p[i] / sc[i];
                dd[i] = d[i] / sc[i];
            }
            iv_and_quad(&I, dot3(dd, dd), 2.0 * dot3(pp, dd), dot3(pp, pp) - 1.0);
            break;
        }
        case 11: { /* free ellipsoid */
            unit3(s->a_x, ax);
            unit3(s->a_y, ay);
            unit3(s->a_z, az);
            const double pp[3] = {dot3(p, ax) / s->dx, dot3(p, ay) / s->dy, dot3(p, az) / s->dz};
            const double dd[3] = {dot3(d, ax) / s->dx, dot3(d, ay) / s->dy, dot3(d, az) / s->dz};
            iv_and_quad(&I, dot3(dd, dd), 2.0 * dot3(pp, dd), dot3(pp, pp) - 1.0);
            break;
        }
        case 12:
            unit3(s->a_x, ax);
            unit3(s->a_y, ay);
            unit3(s->axis, az);
            iv_ecyl(&I, p, d, ax, s->dx, ay, s->dy, az, 0.5 * s->l);
            break;
        case 14: iv_ecyl(&I, p, d, ey, s->dy, ez, s->dz, ex, 0.5 * s->l); break;
        case 15: iv_ecyl(&I, p, d, ex, s->dx, ez, s->dz, ey, 0.5 * s->l); break;
        case 16: iv_ecyl(&I, p, d, ex, s->dx, ey, s->dy, ez, 0.5 * s->l); break;
        case 6:
        case 7:
        case 8:
        case 9: { /* circular cylinder: radial distance from the axis */
            double a[3];
            if (s->type == 6)
                unit3(s->axis, a);
            else
                memcpy(a, s->type == 7 ? ex : (s->type == 8 ? ey : ez), sizeof(a));
            const double pz = dot3(p, a), dz = dot3(d, a);
            iv_and_slab(&I, pz, dz, 0.5 * s->l);
            const double pr[3] = {p[0] - pz * a[0], p[1] - pz * a[1], p[2] - pz * a[2]};
            const double dr[3] = {d[0] - dz * a[0], d[1] - dz * a[1], d[2] - dz * a[2]};
            iv_and_quad(&I, dot3(dr, dr), 2.0 * dot3(pr, dr), dot3(pr, pr) - (double)s->r * s->r);
            break;
        }
        case 2:
        case 3:
        case 4:
        case 5: { /* cone frustum, radius r1 at -l/2 .. r2 at +l/2 */
            double a[3], e1[3], e2[3];
            if (s->type == 2)
                unit3(s->axis, a);
            else
                memcpy(a, s->type == 3 ? ex : (s->type == 4 ? ey : ez), sizeof(a));
            perp2(a, e1, e2);
            const double h = 0.5 * s->l;
            const double pz = dot3(p, a), dz = dot3(d, a);
            iv_and_slab(&I, pz, dz, h);
            if (!(I.lo < I.hi)) return 0;
            const double px = dot3(p, e1), py = dot3(p, e2), dx = dot3(d, e1), dy = dot3(d, e2);
            const double al = 0.5 * ((double)s->r1 + s->r2), be = ((double)s->r2 - s->r1) / s->l;
            const double ra = al + be * pz, rb = be * dz;
            iv_and_quad(&I, dx * dx + dy * dy - rb * rb, 2.0 * (px * dx + py * dy - ra * rb), px * px + py * py - ra * ra);
            break;
        }
        case 1: /* box of full side lengths */
            iv_and_slab(&I, p[0], d[0], 0.5 * s->dx);
            iv_and_slab(&I, p[1], d[1], 0.5 * s->dy);
            iv_and_slab(&I, p[2], d[2], 0.5 * s->dz);
            break;
        default: return 0;
    }
    if (!(I.lo < I.hi)) return 0;
    out2[0] = I.lo;
    out2[1] = I.hi;
    return 1;
}

static int cmp_double(const void *a, const void *b) {
    const double x = *(const double *)a, y = *(const double *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

void ao_project_forbild(const ao_proj_spec *specs, int n_views, int nu, int nv, const ao_forbild_shape *shapes,
                        int n_shapes, double mba, int mode, int ssu, int ssv, double *out, int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
    {
        double *lo = (double *)malloc(sizeof(double) * (size_t)(n_shapes + 1));
        double *hi = (double *)malloc(sizeof(double) * (size_t)(n_shapes + 1));
        double *rho = (double *)malloc(sizeof(double) * (size_t)(n_shapes + 1));
        double *ev = (double *)malloc(sizeof(double) * (size_t)(2 * n_shapes + 2));
#pragma omp for collapse(2) schedule(dynamic, 4)
        for (int m = 0; m < n_views; ++m) {
            for (int iu = 0; iu < nu; ++iu) {
                const ao_proj_spec *sp = &specs[m];
                const double s[3] = {sp->source_pos.x, sp->source_pos.y, sp->source_pos.z};
                for (int iv = 0; iv < nv; ++iv) {
                    double tot = 0.0;
                    for (int ku = 0; ku < ssu; ++ku) {
                        double accu = 0.0;
                        for (int kv = 0; kv < ssv; ++kv) {
                            const d3 pp = pixel_pos(sp, iu - 0.5 + (ku + 0.5) / ssu, iv - 0.5 + (kv + 0.5) / ssv);
                            const double e[3] = {pp.x, pp.y, pp.z};
                            const double len = sqrt((e[0] - s[0]) * (e[0] - s[0]) + (e[1] - s[1]) * (e[1] - s[1]) +
                                                    (e[2] - s[2]) * (e[2] - s[2]));
                            int k = 0;
                            for (int j = 0; j < n_shapes; ++j) {
                                double r[2];
                                if (ao_forbild_interval(s, e, &shapes[j], r)) {
                                    lo[k] = r[0];
                                    hi[k] = r[1];
                                    rho[k] = shapes[j].rho;
                                    ++k;
                                }
                            }
                            double val = 0.0;
                            if (mode != 0) {
                                for (int i = 0; i < k; ++i) val += rho[i] * (hi[i] - lo[i]);
                                if (mode == 2) val *= len;
                            } else if (k > 0) {
                                /* elementary segments between all endpoints; each is
                                 * charged to the last shape covering its midpoint */
                                int ne = 0;
                                for (int i = 0; i < k; ++i) {
                                    ev[ne++] = lo[i];
                                    ev[ne++] = hi[i];
                                }
                                qsort(ev, (size_t)ne, sizeof(double), cmp_double);
                                for (int q = 0; q + 1 < ne; ++q) {
                                    const double a = ev[q], b = ev[q + 1];
                                    if (!(b > a)) continue;
                                    const double mid = 0.5 * (a + b);
                                    for (int i = k - 1; i >= 0; --i) {
                                        if (lo[i] <= mid && mid <= hi[i]) {
                                            val += rho[i] * (b - a);
                                            break;
                                        }
                                    }
                                }
                                val *= len;
                            }
                            accu += val * mba;
                        }
                        tot += accu / ssv;
                    }
                    out[((int64_t)m * nu + iu) * nv + iv] += tot / ssu;
                }
            }
        }
        free(lo);
        free(hi);
        free(rho);
        free(ev);
    }
}

/* ---- FORBILD point sampling (FP64), restating add_FORBILD_sampling
 * (src/aprict/data/cusrc/sample_FORBILD_volumes.cu:10-123) with point tests
 * in each shape's natural coordinates: closed solids, clip mode 1 keeps
 * a.p <= d and mode 2 keeps a.p > d (as FORBILD_volumes.h:93-105). */
int ao_forbild_inside(const double pw[3], const ao_forbild_shape *s) {
    if (s->type == 0) return 0;
    for (int k = 0; k < 3; ++k) {
        const ao_clip *c = &s->cas[k];
        if (c->mode == 0) continue;
        const double a[3] = {c->axis.x, c->axis.y, c->axis.z};
        const double g = dot3(a, pw);
        if (c->mode == 1 ? !(g <= c->dotprod) : !(g > c->dotprod)) return 0;
    }
    const double p[3] = {pw[0] - s->x, pw[1] - s->y, pw[2] - s->z};
    const double ex[3] = {1, 0, 0}, ey[3] = {0, 1, 0}, ez[3] = {0, 0, 1};
    double ax[3], ay[3], az[3];
    switch (s->type) {
        case 13: return dot3(p, p) <= (double)s->r * s->r;
        case 10: {
            const double q[3] = {p[0] / s->dx, p[1] / s->dy, p[2] / s->dz};
            return dot3(q, q) <= 1.0;
        }
        case 11: {
            unit3(s->a_x, ax);
            unit3(s->a_y, ay);
            unit3(s->a_z, az);
            const double q[3] = {dot3(p, ax) / s->dx, dot3(p, ay) / s->dy, dot3(p, az) / s->dz};
            return dot3(q, q) <= 1.0;
        }
        case 12:
        case 14:
        case 15:
        case 16: {
            double sx, sy;
            if (s->type == 12) {
                unit3(s->a_x, ax);
                unit3(s->a_y, ay);
                unit3(s->axis, az);
                sx = s->dx;
                sy = s->dy;
            } else {
                const double *A = s->type == 14 ? ey : ex, *B = s->type == 16 ? ey : ez;
                const double *C = s->type == 14 ? ex : (s->type == 15 ? ey : ez);
                memcpy(ax, A, sizeof(ax));
                memcpy(ay, B, sizeof(ay));
                memcpy(az, C, sizeof(az));
                sx = s->type == 14 ? s->dy : s->dx;
                sy = s->type == 16 ? s->dy : s->dz;
            }
            const double u = dot3(p, ax) / sx, v = dot3(p, ay) / sy;
            return fabs(dot3(p, az)) <= 0.5 * s->l && u * u + v * v <= 1.0;
        }
        case 6:
        case 7:
        case 8:
        case 9: {
            double a[3];
            if (s->type == 6)
                unit3(s->axis, a);
            else
                memcpy(a, s->type == 7 ? ex : (s->type == 8 ? ey : ez), sizeof(a));
            const double z = dot3(p, a);
            const double r2 = dot3(p, p) - z * z;
            return fabs(z) <= 0.5 * s->l && r2 <= (double)s->r * s->r;
        }
        case 2:
        case 3:
        case 4:
        case 5: {
            double a[3];
            if (s->type == 2)
                unit3(s->axis, a);
            else
                memcpy(a, s->type == 3 ? ex : (s->type == 4 ? ey : ez), sizeof(a));
            const double z = dot3(p, a);
            if (!(fabs(z) <= 0.5 * s->l)) return 0;
            const double r = 0.5 * ((double)s->r1 + s->r2) + ((double)s->r2 - s->r1) / s->l * z;
            return dot3(p, p) - z * z <= r * r;
        }
        case 1: return fabs(p[0]) <= 0.5 * s->dx && fabs(p[1]) <= 0.5 * s->dy && fabs(p[2]) <= 0.5 * s->dz;
        default: return 0;
    }
}

void ao_forbild_sample(const ao_forbild_shape *shapes, int n, const double *xs, const double *ys, const double *zs,
                       int nx, int ny, int nz, double ss_wid, int ss, double *out, int nthreads) {
#pragma omp parallel for collapse(2) schedule(dynamic, 4) num_threads(nthreads)
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < ny; ++j) {
            for (int k = 0; k < nz; ++k) {
                double tot = 0.0;
                for (int a = 0; a < ss; ++a)
                    for (int b = 0; b < ss; ++b)
                        for (int c = 0; c < ss; ++c) {
                            const double p[3] = {xs[i] + (a - 0.5 * (ss - 1)) / ss * ss_wid,
                                                 ys[j] + (b - 0.5 * (ss - 1)) / ss * ss_wid,
                                                 zs[k] + (c - 0.5 * (ss - 1)) / ss * ss_wid};
                            double val = 0.0;
                            for (int m = 0; m < n; ++m)
                                if (ao_forbild_inside(p, &shapes[m])) val = shapes[m].rho;
                            tot += val;
                        }
                out[((size_t)i * ny + j) * nz + k] = tot / ((double)ss * ss * ss);
            }
        }
    }
}
