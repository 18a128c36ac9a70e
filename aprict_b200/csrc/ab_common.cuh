// ab_common.cuh -- shared device helpers for the aprict_b200 kernels.
//
// Geometry conventions follow the reference (murdock-grewar/aprict 0.1.5):
//   * voxel (i,j,k) of an (X,Y,Z) volume occupies
//     [corner + voxwid*(i,j,k), corner + voxwid*(i+1,j+1,k+1)) in world units
//     (src/aprict/volume/volume.py:133-145, flatpanel.py:1025-1041);
//   * pixel (iu,iv) centre = det_pos + det_u*(iu-(nu-1)/2) + det_v*(iv-(nv-1)/2)
//     (src/aprict/data/cusrc/CB_project_texture_chunked.cu:308-324).
#pragma once

#include <math.h>
#include <stdint.h>

#include "aprict_b200.h"

#if defined(__CUDACC__)
#define AB_HD __host__ __device__ __forceinline__
#define AB_DEV __device__ __forceinline__
// a call, not inlined: for once-per-view set-up inside kernels whose hot loop
// keeps many values in registers
#define AB_HD_CALL __host__ __device__ inline __noinline__
#else
#define AB_HD inline
#define AB_DEV inline
#define AB_HD_CALL inline
#endif

// ---------------------------------------------------------------------------
// Small double-precision vector helpers (ray setup is done in FP64).
struct ab_d3 {
    double x, y, z;
};
AB_HD ab_d3 ab_d3_of(aprict_fvec3 v) { return ab_d3{(double)v.x, (double)v.y, (double)v.z}; }
AB_HD ab_d3 operator+(ab_d3 a, ab_d3 b) { return ab_d3{a.x + b.x, a.y + b.y, a.z + b.z}; }
AB_HD ab_d3 operator-(ab_d3 a, ab_d3 b) { return ab_d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
AB_HD ab_d3 operator*(ab_d3 a, double s) { return ab_d3{a.x * s, a.y * s, a.z * s}; }
AB_HD double ab_dot(ab_d3 a, ab_d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
AB_HD ab_d3 ab_cross(ab_d3 a, ab_d3 b) {
    return ab_d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
AB_HD bool ab_finite3(ab_d3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

// Volume geometry as the traversal sees it: voxel units, corner at the origin.
template <typename Off>
struct ab_grid {
    int n[3];         // X, Y, Z
    Off stride[3];    // element strides of x, y, z
    double corner[3]; // world
    double inv_voxwid;
    float voxwid;
};

template <typename Off>
AB_HD ab_grid<Off> ab_make_grid(const aprict_vol_desc &v) {
    ab_grid<Off> g;
    g.n[0] = (int)v.nx;
    g.n[1] = (int)v.ny;
    g.n[2] = (int)v.nz;
    if (v.order == 0) {  // C order: z fastest
        g.stride[0] = (Off)v.ny * (Off)v.nz;
        g.stride[1] = (Off)v.nz;
        g.stride[2] = 1;
    } else {  // F order: x fastest
        g.stride[0] = 1;
        g.stride[1] = (Off)v.nx;
        g.stride[2] = (Off)v.nx * (Off)v.ny;
    }
    g.corner[0] = v.corner.x;
    g.corner[1] = v.corner.y;
    g.corner[2] = v.corner.z;
    g.voxwid = v.voxwid;
    g.inv_voxwid = 1.0 / (double)v.voxwid;
    return g;
}

// World point -> voxel units relative to the grid corner.
template <typename Off>
AB_HD ab_d3 ab_to_grid(const ab_grid<Off> &g, ab_d3 p) {
    return ab_d3{(p.x - g.corner[0]) * g.inv_voxwid, (p.y - g.corner[1]) * g.inv_voxwid,
                 (p.z - g.corner[2]) * g.inv_voxwid};
}

// ---------------------------------------------------------------------------
// Siddon traversal of the segment o -> e (voxel units, grid corner at 0).
//
// Computes the same quantity as exact_line_integral_unitvoxwid
// (CB_project_texture_chunked.cu:111-272): the exact intersection length of
// the segment with every voxel it crosses. The arithmetic differs on purpose:
//   * entry/exit parameters, the entry voxel and every per-axis crossing
//     origin are computed in FP64;
//   * crossings are stepped in FP32 as tau_a(k) = t0_a + k*dt_a (one fma per
//     step, relative to the entry point), so positions never drift -- the
//     reference adds steps*d to a running position and accumulates error;
//   * the visitor receives (segment length in voxel units, element offset).
// Tie rules mirror the reference: a coordinate exactly on a voxel boundary
// belongs to the voxel the ray moves into; with zero direction along an axis
// the voxel is ceil(c)-1 (reference :189-203, :244-246), so a ray lying in the
// plane c == 0 misses and one in c == n hits the last layer.
//
// ab_siddon_setup prepares the traversal state (in FP64, then rounded to the
// FP32 stepping quantities); ab_siddon runs it with a visitor. Both return
// false when the segment misses the grid or its input is not finite (*bad is
// set for non-finite input).
template <typename Off>
struct ab_ray {
    float t0x, t0y, t0z;  // first crossing along each axis (from the entry point)
    float dtx, dty, dtz;  // crossing spacing along each axis
    float tend;           // exit, clamped to every axis's last in-grid crossing
    Off off;              // element offset of the entry voxel
    Off ox, oy, oz;       // signed element steps
};

template <typename Off>
AB_HD bool ab_siddon_setup(ab_d3 o, ab_d3 e, const int n[3], const Off stride[3], ab_ray<Off> &r, bool *bad) {
    if (!ab_finite3(o) || !ab_finite3(e)) {
        *bad = true;
        return false;
    }
    const double od[3] = {o.x, o.y, o.z};
    const double dd[3] = {e.x - o.x, e.y - o.y, e.z - o.z};
    double a_in = 0.0, a_out = 1.0;
    double inv[3];  // 1 / dd (correctly rounded), reused below instead of divisions
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        inv[a] = 0.0;
        if (dd[a] == 0.0) {
            if (!(od[a] > 0.0 && od[a] <= (double)n[a])) return false;
        } else {
#if defined(__CUDA_ARCH__)
            inv[a] = __drcp_rn(dd[a]);
#else
            inv[a] = 1.0 / dd[a];
#endif
            const double t0 = (0.0 - od[a]) * inv[a];
            const double t1 = ((double)n[a] - od[a]) * inv[a];
            a_in = fmax(a_in, fmin(t0, t1));
            a_out = fmin(a_out, fmax(t0, t1));
        }
    }
    if (!(a_in < a_out)) return false;
    const double len = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);

    int stp[3];
    float t0f[3], dtf[3], texit[3];
    Off off = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double p = od[a] + a_in * dd[a];
        int i;
        if (dd[a] > 0.0) {
            i = (int)floor(p);
        } else {
            i = (int)ceil(p) - 1;
        }
        i = i < 0 ? 0 : (i >= n[a] ? n[a] - 1 : i);
        off += (Off)i * stride[a];
        if (dd[a] == 0.0) {
            stp[a] = 0;
            t0f[a] = INFINITY;
            dtf[a] = 0.f;
            texit[a] = INFINITY;
        } else {
            const bool pos = dd[a] > 0.0;
            stp[a] = pos ? 1 : -1;
            const double b = pos ? (double)(i + 1) : (double)i;
            const double ab = (b - od[a]) * inv[a];
            t0f[a] = (float)((ab - a_in) * len);
            dtf[a] = (float)(len * fabs(inv[a]));
            // Crossings left along this axis until the grid boundary; the last
            // one (k = K-1) is evaluated with the loop's own fma.
            const int K = pos ? n[a] - i : i + 1;
            texit[a] = fmaf((float)(K - 1), dtf[a], t0f[a]);
        }
    }
    // The loop stops at tend. Clamping tend to every axis's boundary crossing,
    // computed by the same fma the loop uses (bitwise identical values), makes
    // a step past the last voxel along any axis impossible: that step would
    // need tm == texit[a] < tend <= texit[a]. No index bookkeeping is needed.
    r.tend = fminf((float)((a_out - a_in) * len), fminf(texit[0], fminf(texit[1], texit[2])));
    r.off = off;
    r.ox = stp[0] > 0 ? stride[0] : (Off)0 - stride[0];
    r.oy = stp[1] > 0 ? stride[1] : (Off)0 - stride[1];
    r.oz = stp[2] > 0 ? stride[2] : (Off)0 - stride[2];
    r.t0x = t0f[0];
    r.t0y = t0f[1];
    r.t0z = t0f[2];
    r.dtx = dtf[0];
    r.dty = dtf[1];
    r.dtz = dtf[2];
    return true;
}

// One traversal step: tm is the next crossing; advances the state past it.
// Branch-free: every lane of a warp runs the same instructions whichever axis
// its ray crosses next. The three crossings are recomputed from their
// counters (an unchanged counter reproduces the same value), so no per-axis
// selects are needed.
#define AB_SIDDON_ADVANCE(R, off, kx, ky, kz, tx, ty, tz, tm) \
    do {                                                      \
        const bool bx_ = (tx) == (tm);                        \
        const bool by_ = !bx_ && ((ty) == (tm));              \
        (off) += bx_ ? (R).ox : (by_ ? (R).oy : (R).oz);      \
        (kx) += bx_ ? 1.f : 0.f;                              \
        (ky) += by_ ? 1.f : 0.f;                              \
        (kz) += (bx_ || by_) ? 0.f : 1.f;                     \
        (tx) = fmaf((kx), (R).dtx, (R).t0x);                  \
        (ty) = fmaf((ky), (R).dty, (R).t0y);                  \
        (tz) = fmaf((kz), (R).dtz, (R).t0z);                  \
    } while (0)

// The same step for 32-bit offsets on the GPU, in PTX: the axis predicates
// drive predicated FP32 counter increments and predicated integer
// multiply-adds (by `one`, a runtime 1 the compiler cannot fold) that advance
// the offset, so the offset update runs on the FMA pipe instead of two selects
// and an add on the ALU pipe, the loop's busiest. Same arithmetic and results
// as AB_SIDDON_ADVANCE (measured bit-identical; 256^3 x 360-view fused
// residual 12.37 -> 10.19 ms, ALU-pipe instructions per step 10.1 -> 5.6).
#if defined(__CUDA_ARCH__)
#define AB_SIDDON_ADVANCE_I32(R, off, kx, ky, kz, tx, ty, tz, tm, one)                    \
    do {                                                                                  \
        asm("{\n\t.reg .pred px, py, pz;\n\t"                                          \
            "setp.eq.f32 px, %4, %6;\n\t"                                              \
            "setp.eq.and.f32 py, %5, %6, !px;\n\t"                                     \
            "or.pred pz, px, py;\n\t"                                                   \
            "@px add.f32 %0, %0, 0f3F800000;\n\t"                                       \
            "@py add.f32 %1, %1, 0f3F800000;\n\t"                                       \
            "@!pz add.f32 %2, %2, 0f3F800000;\n\t"                                      \
            "@px mad.lo.s32 %3, %7, %10, %3;\n\t"                                       \
            "@py mad.lo.s32 %3, %8, %10, %3;\n\t"                                       \
            "@!pz mad.lo.s32 %3, %9, %10, %3;\n\t}"                                     \
            : "+f"(kx), "+f"(ky), "+f"(kz), "+r"(off)                                     \
            : "f"(tx), "f"(ty), "f"(tm), "r"((R).ox), "r"((R).oy), "r"((R).oz), "r"(one)); \
        (tx) = fmaf((kx), (R).dtx, (R).t0x);                                              \
        (ty) = fmaf((ky), (R).dty, (R).t0y);                                              \
        (tz) = fmaf((kz), (R).dtz, (R).t0z);                                              \
    } while (0)
#endif

// Visits every (segment length in voxel units, element offset) of the ray.
template <typename Off, class Visit>
AB_HD bool ab_siddon(ab_d3 o, ab_d3 e, const int n[3], const Off stride[3], Visit &visit, bool *bad) {
    ab_ray<Off> R;
    if (!ab_siddon_setup<Off>(o, e, n, stride, R, bad)) return false;
    Off off = R.off;
    float kx = 0.f, ky = 0.f, kz = 0.f;
    float tx = R.t0x, ty = R.t0y, tz = R.t0z;
    float t = 0.f;
    for (;;) {
        const float tm = fminf(tx, fminf(ty, tz));
        visit(fminf(tm, R.tend) - t, off);
        if (tm >= R.tend) break;
        t = tm;
        AB_SIDDON_ADVANCE(R, off, kx, ky, kz, tx, ty, tz, tm);
    }
    return true;
}

// Number of crossings along one axis before the exit: #{k >= 0 : fma(k, dt, t0) < tend},
// with the traversal's own fma, so the count equals the number of steps the
// exit test would take along this axis. dt >= 1 (a voxel's chord along an
// axis is at least its width) keeps the estimate within a few steps of the
// answer; the two bounded fix-up loops settle it and the final test proves
// it. ok is cleared when the proof fails (never observed; the caller then
// takes no steps and reports the ray).
AB_HD int ab_axis_count(float t0, float dt, float tend, bool &ok) {
    if (!(t0 < tend)) return 0;  // no crossing before the exit (also t0 = +inf)
#if defined(__CUDA_ARCH__)
    const float q = __fdividef(tend - t0, dt);
#else
    const float q = (tend - t0) / dt;
#endif
    int k = q < 1.f ? 1 : (q > 16777216.f ? 16777216 : (int)ceilf(q));
    for (int it = 0; it < 8 && k > 1 && fmaf((float)(k - 1), dt, t0) >= tend; ++it) --k;
    for (int it = 0; it < 8 && fmaf((float)k, dt, t0) < tend; ++it) ++k;
    if (!(fmaf((float)(k - 1), dt, t0) < tend && fmaf((float)k, dt, t0) >= tend)) ok = false;
    return k;
}

// Line integral sum(seg * vol[off]) (voxel units) over the segment o -> e.
//
// The loop runs a precomputed number of steps (the crossings before the exit,
// counted per axis by ab_axis_count), so it needs no exit test per step; each
// step is the same branch-free advance as ab_siddon. Accumulation is
// compensated: the products of kChunk consecutive steps are summed in FP32
// and each partial sum is added to the total with Kahan's compensation (the
// partial sums carry ~sqrt(kChunk) ulp; the total is then as accurate as a
// Kahan sum of the partials). load(off) must be a pure read.
template <typename Off, class Load>
AB_HD bool ab_siddon_gather(ab_d3 o, ab_d3 e, const int n[3], const Off stride[3], Load &load, float &sum,
                            bool *bad, int one = 1) {
    constexpr int kChunk = 16;
    ab_ray<Off> R;
    sum = 0.f;
    if (!ab_siddon_setup<Off>(o, e, n, stride, R, bad)) return false;
    bool ok = true;
    const int N = ab_axis_count(R.t0x, R.dtx, R.tend, ok) + ab_axis_count(R.t0y, R.dty, R.tend, ok) +
                  ab_axis_count(R.t0z, R.dtz, R.tend, ok);
    if (!ok) {
        *bad = true;
        return false;
    }
    Off off = R.off;
    float kx = 0.f, ky = 0.f, kz = 0.f;
    float tx = R.t0x, ty = R.t0y, tz = R.t0z;
    float t = 0.f, s = 0.f, c = 0.f;
    float mu = load(off);
    // Each step: the segment up to the next crossing is accumulated with the
    // current voxel's value, the crossing is passed, and the next voxel's
    // value is loaded (in the grid: the step precedes the exit).
#if defined(__CUDA_ARCH__)
#define AB_GATHER_ADVANCE(tm_)                                                     \
    do {                                                                           \
        if constexpr (sizeof(Off) == 4)                                            \
            AB_SIDDON_ADVANCE_I32(R, off, kx, ky, kz, tx, ty, tz, tm_, one);       \
        else                                                                       \
            AB_SIDDON_ADVANCE(R, off, kx, ky, kz, tx, ty, tz, tm_);                \
    } while (0)
#else
#define AB_GATHER_ADVANCE(tm_) AB_SIDDON_ADVANCE(R, off, kx, ky, kz, tx, ty, tz, tm_)
#endif
#define AB_GATHER_STEP(part)                                   \
    do {                                                       \
        const float tm_ = fminf(tx, fminf(ty, tz));            \
        part = fmaf(tm_ - t, mu, part);                        \
        t = tm_;                                               \
        AB_GATHER_ADVANCE(tm_);                                \
        mu = load(off);                                        \
    } while (0)
    int i = 0;
    for (; i + kChunk <= N; i += kChunk) {
        float part = 0.f;
#pragma unroll
        for (int j = 0; j < kChunk; ++j) AB_GATHER_STEP(part);
        const float y = part - c;
        const float tt = s + y;
        c = (tt - s) - y;
        s = tt;
    }
    float part = 0.f;
    for (; i < N; ++i) AB_GATHER_STEP(part);
#undef AB_GATHER_STEP
#undef AB_GATHER_ADVANCE
    part = fmaf(R.tend - t, mu, part);  // the last segment ends at the exit
    sum = s + (part - c);
    return true;
}

// The transpose of ab_siddon_gather: adds w * seg to vol[off] for every
// segment of the ray (one atomic add per voxel crossed; zero-length segments
// add nothing), with the same counted step loop and per-step arithmetic.
#if defined(__CUDACC__)
template <typename Off>
__device__ __forceinline__ bool ab_siddon_scatter(ab_d3 o, ab_d3 e, const int n[3], const Off stride[3], float *vol,
                                                  float w, bool *bad, int one = 1) {
    ab_ray<Off> R;
    if (!ab_siddon_setup<Off>(o, e, n, stride, R, bad)) return false;
    bool ok = true;
    const int N = ab_axis_count(R.t0x, R.dtx, R.tend, ok) + ab_axis_count(R.t0y, R.dty, R.tend, ok) +
                  ab_axis_count(R.t0z, R.dtz, R.tend, ok);
    if (!ok) {
        *bad = true;
        return false;
    }
    Off off = R.off;
    float kx = 0.f, ky = 0.f, kz = 0.f;
    float tx = R.t0x, ty = R.t0y, tz = R.t0z;
    float t = 0.f;
    for (int i = 0; i < N; ++i) {
        const float tm = fminf(tx, fminf(ty, tz));
        const float seg = tm - t;
        if (seg > 0.f) atomicAdd(vol + off, seg * w);
        t = tm;
        if constexpr (sizeof(Off) == 4)
            AB_SIDDON_ADVANCE_I32(R, off, kx, ky, kz, tx, ty, tz, tm, one);
        else
            AB_SIDDON_ADVANCE(R, off, kx, ky, kz, tx, ty, tz, tm);
    }
    const float seg = R.tend - t;  // the last segment ends at the exit
    if (seg > 0.f) atomicAdd(vol + off, seg * w);
    return true;
}
#endif

// Kahan-compensated FP32 accumulator.
struct ab_kahan {
    float s, c;
    AB_HD void add(float v) {
        const float y = v - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

// Pixel centre (fractional index) in world units, FP64 from the FP32 spec.
AB_HD ab_d3 ab_pixel_pos(const aprict_proj_spec &sp, double fu, double fv) {
    const double xnum = fu - ((double)sp.nu - 1.0) * 0.5;
    const double ynum = fv - ((double)sp.nv - 1.0) * 0.5;
    return ab_d3_of(sp.det_pos) + ab_d3_of(sp.det_u) * xnum + ab_d3_of(sp.det_v) * ynum;
}

// Element offsets into a projection stack.
struct ab_pstrides {
    int64_t view, u, v;
};
