// ab_bpview.cuh -- per-view coefficients for voxel-driven backprojection.
//
// The reference re-derives, for every voxel and view, the detector
// coordinates of a point with get_projected_detector_coords
// (src/aprict/data/cusrc/geometry.h:24-56): a cross product, two norms and
// three divisions in FP32. Here each view is reduced once (in FP64, per CTA,
// into shared memory) to three linear forms of the voxel position x, taken
// relative to the volume centre c0:
//
//   den(x) = (x - s).n                      n = u x v (detector normal)
//   Nu(x)  = A_u.(x - c0) + B_u             u index = Nu(x) / den(x)
//   Nv(x)  = A_v.(x - c0) + B_v             v index = Nv(x) / den(x)
//
// which is the same mapping: with Dn = (P - s).n and lambda = Dn / den(x),
// q = s + (x - s) lambda - P, cu = u.q/|u|^2, so
//   cu * den = [Dn u - (u.(P - s)) n].(x - s) / |u|^2,
// and the pixel index is cu + (nu-1)/2. Shifting the origin to c0 keeps the
// FP32 terms of the dot products small.
#pragma once

#include "ab_common.cuh"

struct ab_bpview {
    float4 nu;   // A_u.xyz, B_u
    float4 nv;   // A_v.xyz, B_v
    float4 den;  // n.xyz,  (c0 - s).n
    float4 zl;   // Lhat.xyz, (c0 - s).Lhat  ->  Z(x) = distance along L = P - s
    float kfast; // voxwid^3 Dn^2 / (|u||v|), already folded into nu, nv, den (fast-mode weight 1 / den^2)
    float invL;  // 1 / |L|
    float halfu; // nu / 2
    float halfv; // nv / 2
    float inv_halfu, inv_halfv;
    // Edge taper: |fu - cu0| <= tap_ru and |fv - cv0| <= tap_rv guarantees a
    // factor of exactly 1 (a margin of 1e-5 keeps it conservative). Without a
    // taper the box is the detector itself (half-widths nu/2, nv/2).
    float cu0, cv0, tap_ru, tap_rv;
    // Nearest-pixel trust thresholds: with |f - round(f)| <= tie the FP32
    // rounding is certain to pick the pixel the exact value picks (see
    // ab_fp32_pixel_error_bound); above it the choice is made in FP64.
    float tie_u, tie_v;
    float sxw, syw;  // source position (world x, y), for the cone-cylinder weighting presets
    // Certainly off the detector: |fu - cu0| > out_ru (or v) puts the nearest
    // pixel out of range in FP32 and in exact arithmetic alike (the half-width
    // plus the FP32 error bound); out_ru + 1/2 does the same for all four
    // bilinear taps.
    float out_ru, out_rv;
};

// A priori bound on the error of the FP32 detector coordinate f = N(x)/D(x)
// as the backprojector evaluates it (coefficients rounded to FP32, a 3-fma
// dot product plus one fma step, an approximate reciprocal and a multiply),
// over a box |x_i - c0_i| <= R_i: with u = 2^-24, S_N = sum |a_i| R_i + |b|
// (and S_D likewise for the denominator), D_min = min |D| over the box,
//   |f32(f) - f| <= 6u (S_N + |f| S_D) / D_min + 4u |f|,   |f| <= max(nu, nv).
// Emulated over circular, helical and short-distance scans the observed
// error stays below 0.3 of this bound. Returns 1 (distrust everything) when
// the box reaches the source plane (D_min <= 0).
AB_HD double ab_fp32_pixel_error_bound(ab_d3 a, double b, ab_d3 n, double bd, const double R[3], double fmax) {
    const double u = 5.9604644775390625e-08;
    const double SN = fabs(a.x) * R[0] + fabs(a.y) * R[1] + fabs(a.z) * R[2] + fabs(b);
    const double nR = fabs(n.x) * R[0] + fabs(n.y) * R[1] + fabs(n.z) * R[2];
    const double SD = nR + fabs(bd);
    const double Dmin = fabs(bd) - nR;
    if (!(Dmin > 0.0)) return 1.0;
    return 6.0 * u * (SN + fmax * SD) / Dmin + 4.0 * u * fmax;
}

// The same three linear forms in FP64 (coefficients before rounding), used to
// settle nearest-pixel choices that the FP32 forms cannot resolve.
struct ab_bpview_d {
    double nu[4], nv[4], den[4];
};

// Exact-mode extras: ray origin and per-pixel direction in world units,
// relative to the volume centre.
struct ab_bpview_exact {
    float4 s;   // s - c0 (xyz), unused
    float4 d0;  // direction to the detector centre pixel origin: P - s - u(nu-1)/2 - v(nv-1)/2
    float4 u;   // det_u
    float4 v;   // det_v
};

// half_ext: the largest |x_i - c0_i| of any point the kernel projects
// (voxel centres with sub-sample offsets), for the nearest-pixel thresholds.
// A call rather than inlined: it runs once per view and chunk in the
// backprojectors, whose voxel loops then keep their accumulators in registers
// (inlined, its FP64 temporaries made the fan-slice kernel spill 324 bytes
// around the loop; out of line, 72 bytes).
AB_HD_CALL bool ab_derive_bpview(const aprict_proj_spec &sp, ab_d3 c0, float voxwid, float sep, const double half_ext[3],
                            ab_bpview &o, ab_bpview_d *od = nullptr) {
    const ab_d3 s = ab_d3_of(sp.source_pos), P = ab_d3_of(sp.det_pos);
    const ab_d3 U = ab_d3_of(sp.det_u), V = ab_d3_of(sp.det_v);
    const ab_d3 n = ab_cross(U, V);
    const double uu = ab_dot(U, U), vv = ab_dot(V, V);
    const ab_d3 Ps = P - s;
    const double Dn = ab_dot(Ps, n);
    const ab_d3 c0s = c0 - s;
    const double Lnorm = sqrt(ab_dot(Ps, Ps));
    bool ok = uu > 0.0 && vv > 0.0 && Dn != 0.0 && Lnorm > 0.0 && ab_finite3(s) && ab_finite3(P) &&
              ab_finite3(U) && ab_finite3(V);
    if (!ok) {
        o = ab_bpview{};
        if (od) *od = ab_bpview_d{};
        return false;
    }
    const double hu = ((double)sp.nu - 1.0) * 0.5, hv = ((double)sp.nv - 1.0) * 0.5;
    // A_u = (Dn U - (U.(P-s)) n) / |U|^2 + hu n ;  B_u = A_u.(c0 - s)
    const ab_d3 Au = (U * Dn - n * ab_dot(U, Ps)) * (1.0 / uu) + n * hu;
    const ab_d3 Av = (V * Dn - n * ab_dot(V, Ps)) * (1.0 / vv) + n * hv;
    const ab_d3 Lh = Ps * (1.0 / Lnorm);
    if (od) {
        *od = ab_bpview_d{{Au.x, Au.y, Au.z, ab_dot(Au, c0s)}, {Av.x, Av.y, Av.z, ab_dot(Av, c0s)},
                          {n.x, n.y, n.z, ab_dot(n, c0s)}};
    }
    // The three forms are scaled by 1 / sqrt(kfast): every ratio (the detector
    // coordinates) is unchanged and the fast-mode weight kfast / D^2 becomes 1 / D'^2.
    const double vw3 = (double)voxwid * (double)voxwid * (double)voxwid;
    const double sc = 1.0 / sqrt(vw3 * Dn * Dn / (sqrt(uu) * sqrt(vv)));
    o.nu = make_float4((float)(Au.x * sc), (float)(Au.y * sc), (float)(Au.z * sc), (float)(ab_dot(Au, c0s) * sc));
    o.nv = make_float4((float)(Av.x * sc), (float)(Av.y * sc), (float)(Av.z * sc), (float)(ab_dot(Av, c0s) * sc));
    o.den = make_float4((float)(n.x * sc), (float)(n.y * sc), (float)(n.z * sc), (float)(ab_dot(n, c0s) * sc));
    o.zl = make_float4((float)Lh.x, (float)Lh.y, (float)Lh.z, (float)ab_dot(Lh, c0s));
    const double vw = (double)voxwid;
    o.kfast = (float)(vw * vw * vw * Dn * Dn / (sqrt(uu) * sqrt(vv)));
    o.invL = (float)(1.0 / Lnorm);
    o.halfu = (float)sp.nu * 0.5f;
    o.halfv = (float)sp.nv * 0.5f;
    o.inv_halfu = (float)(2.0 / (double)sp.nu);
    o.inv_halfv = (float)(2.0 / (double)sp.nv);
    o.cu0 = (float)hu;
    o.cv0 = (float)hv;
    const double keep = sep > 0.f ? (1.0 - (double)sep) * (1.0 - 1e-5) : 1.0;
    o.tap_ru = (float)(0.5 * (double)sp.nu * keep);
    o.tap_rv = (float)(0.5 * (double)sp.nv * keep);
    // Thresholds with a further margin of 1.5 on the bound; never closer to
    // 1/2 than 1e-4, so a trusted pixel is always a valid index.
    const double fmax = (double)(sp.nu > sp.nv ? sp.nu : sp.nv);
    const double bdn = ab_dot(n, c0s);
    const double eu = 1.5 * ab_fp32_pixel_error_bound(Au, ab_dot(Au, c0s), n, bdn, half_ext, fmax);
    const double ev = 1.5 * ab_fp32_pixel_error_bound(Av, ab_dot(Av, c0s), n, bdn, half_ext, fmax);
    o.tie_u = (float)(0.5 - (eu > 1e-4 ? eu : 1e-4));
    o.tie_v = (float)(0.5 - (ev > 1e-4 ? ev : 1e-4));
    o.out_ru = (float)(0.5 * (double)sp.nu + (eu > 1e-4 ? eu : 1e-4) + 1e-3);
    o.out_rv = (float)(0.5 * (double)sp.nv + (ev > 1e-4 ? ev : 1e-4) + 1e-3);
    o.sxw = (float)s.x;
    o.syw = (float)s.y;
    return true;
}

AB_HD void ab_derive_bpview_exact(const aprict_proj_spec &sp, ab_d3 c0, ab_bpview_exact &o) {
    const ab_d3 s = ab_d3_of(sp.source_pos), P = ab_d3_of(sp.det_pos);
    const ab_d3 U = ab_d3_of(sp.det_u), V = ab_d3_of(sp.det_v);
    const double hu = ((double)sp.nu - 1.0) * 0.5, hv = ((double)sp.nv - 1.0) * 0.5;
    const ab_d3 sr = s - c0;
    const ab_d3 d0 = P - s - U * hu - V * hv;
    o.s = make_float4((float)sr.x, (float)sr.y, (float)sr.z, 0.f);
    o.d0 = make_float4((float)d0.x, (float)d0.y, (float)d0.z, 0.f);
    o.u = make_float4((float)U.x, (float)U.y, (float)U.z, 0.f);
    o.v = make_float4((float)V.x, (float)V.y, (float)V.z, 0.f);
}

// FP64 detector index coordinates of world point x (reference formula,
// geometry.h:39-51, in double), used to settle nearest-pixel choices that
// the FP32 path cannot resolve.
AB_HD void ab_project_point_d(const aprict_proj_spec &sp, ab_d3 x, double &fu, double &fv) {
    const ab_d3 s = ab_d3_of(sp.source_pos), P = ab_d3_of(sp.det_pos);
    const ab_d3 U = ab_d3_of(sp.det_u), V = ab_d3_of(sp.det_v);
    const ab_d3 n = ab_cross(U, V);
    const double lam = ab_dot(P - s, n) / ab_dot(x - s, n);
    const ab_d3 q = s + (x - s) * lam - P;
    fu = ab_dot(U, q) / ab_dot(U, U) + ((double)sp.nu - 1.0) * 0.5;
    fv = ab_dot(V, q) / ab_dot(V, V) + ((double)sp.nv - 1.0) * 0.5;
}

// Integer power as in the reference's powint (CB_backproject.cu:21-35).
AB_HD float ab_powint(float b, int e) {
    float a = 1.f;
    if (e < 0) {
        for (int k = 0; k < -e; ++k) a /= b;
    } else {
        for (int k = 0; k < e; ++k) a *= b;
    }
    return a;
}

// One axis's factor of the detector-edge cosine taper (CB_backproject.cu:694-713):
// a = |c|, the distance in pixels from the detector centre along that axis.
// Outside the edge band the clamped argument is 1 and the factor is exactly 1
// (the cosine is only evaluated inside the band).
AB_HD float ab_edge_taper_half(float a, float inv_half, float inv_sep) {
    const float r = a * inv_half;
    const float d = fmaxf(0.f, fminf(1.f, (1.f - r) * inv_sep));
    if (d == 1.f) return 1.f;
    return fmaxf(0.f, fminf(1.f, (1.f + cosf(3.1415926535898f * (1.f - d))) * 0.5f));
}

// The taper's weight at (cu, cv), pixels relative to the detector centre: the
// product of the two axes' factors.
AB_HD float ab_edge_taper(float cu, float cv, float inv_halfu, float inv_halfv, float inv_sep) {
    return ab_edge_taper_half(fabsf(cu), inv_halfu, inv_sep) * ab_edge_taper_half(fabsf(cv), inv_halfv, inv_sep);
}
