// ab_gbc.cu -- the GBC reconstruction's device work: backprojection with the
// cylindrical-locus GBC weights into a volume and a weight-sum volume, the
// expected weight sum over a perfect cylindrical trajectory, the volume-domain
// cone-beam ramp filter's spectral multiplier, and the trilinear low-resolution
// correction.
//
// Reference: backproject_CB_voltex_GBC_cyl / _backproject_CB_getval_GBC_cyl /
// _GBC_weightfun / cossq_soft (src/aprict/data/cusrc/CB_backproject.cu:273-311,
// 736-905, 1030-1105), get_GBC_weight_integ (:1108-1168, driven by
// src/aprict/gbc/weightinteg.py:22-91), ramp_filter_conebeam and
// _conebeam_kfactor_unchunked (src/aprict/gbc/filters.py:59-147, 256-504).
//
// The backprojection launches once for all views (the reference: once per 10
// views, the volume read-modified-written each time). One thread per voxel,
// consecutive threads on consecutive voxels in memory order, per-view
// coefficients staged in shared memory. The weight is evaluated in FP32 from
// reciprocal square roots and one division (the angles' sines and cosines by
// trigonometric identities, the soft windows on squared sines), the detector coordinate
// by the same linear forms as the other backprojection modes, and the
// nearest-pixel choice re-decided in FP64 near ties, so the result follows
// the FP64 restatement. The spectral filter is one pass over the cuFFT
// spectrum with all per-frequency factors (ramp, 1 / k-factor, sinc
// corrections, DC) folded into one FP64 factor; the reference makes about
// ten array passes.
#include <cuda_runtime.h>

#include <cmath>

#include "ab_bpbrick.cuh"

namespace {

constexpr int kGThreads = 256;
constexpr int kGChunk = 64;  // views per shared-memory chunk

// Soft window s(a, b; c) of cossq_soft (CB_backproject.cu:273-311): 0 beyond
// |c| = a, 1 inside |c| = a - b, 3x^2 - 2x^3 between, x = gamma sin|c| - chi,
// gamma = 1 / (sin(a - b) - sin a), chi = gamma sin a. Both angles the weight
// feeds it lie in [0, pi/2], where sin is increasing, so the window is taken
// as a function of s = sin|c| with the comparisons made on sines: no
// transcendental per voxel-view. The constants come from the host in FP64.
struct SoftWin {
    float sa2, sab2, gamma, chi;  // sin^2 a (4 if a >= pi/2), sin^2(a - b) (-1 if a - b <= 0, 4 if >= pi/2), gamma, chi
};

struct GbcSoft {
    SoftWin v, h;  // vertical (elevation) and horizontal windows
};

SoftWin soft_win(double a, double b) {
    const double half_pi = 1.5707963267948966;
    SoftWin w;
    w.sa2 = a >= half_pi ? 4.f : (float)(sin(a) * sin(a));
    w.sab2 = a - b <= 0.0 ? -1.f : (a - b >= half_pi ? 4.f : (float)(sin(a - b) * sin(a - b)));
    const double g = 1.0 / (sin(a - b) - sin(a));
    w.gamma = (float)g;
    w.chi = (float)(g * sin(a));
    return w;
}

// The soft band's cubic at s = sin|angle|.
__device__ __forceinline__ float soft_cubic(float s, const SoftWin &w) {
    const float x = w.gamma * s - w.chi;
    return fmaxf(0.f, fminf(1.f, 3.f * x * x - 2.f * x * x * x));
}

// The window at s = sqrt(s2), s = sin|angle| in [0, 1]: compared on squares,
// a square root only inside the soft band.
__device__ __forceinline__ float soft_of_sin2(float s2, const SoftWin &w) {
    if (s2 > w.sa2) return 0.f;
    if (s2 < w.sab2) return 1.f;
    return soft_cubic(sqrtf(s2), w);
}

// The same window when s itself is at hand (s2 = s * s): no square root.
__device__ __forceinline__ float soft_of_sin(float s, float s2, const SoftWin &w) {
    if (s2 > w.sa2) return 0.f;
    if (s2 < w.sab2) return 1.f;
    return soft_cubic(s, w);
}

// GBC weight (eq. 23 of the GBC method with the soft windows,
// CB_backproject.cu:736-787) of the voxel at world position p for the source
// at s (inv_ls = 1 / |(s_x, s_y)|), on a cylinder of radius R (inv_R = 1/R)
// about the world z axis. With r = p - s, q = r_x^2 + r_y^2:
//   ell = sqrt(q) / R, c = clamp(|Z / R / ell|) = clamp(|r . L| / (|L| sqrt(q))),
//   theta = atan2(r_z / R, ell): cos theta = ell / h, sin|theta| = |r_z / R| / h,
//   h = hypot(ell, r_z / R); phi = acos(c): sin^2 phi = 1 - c^2.
// Reciprocal square roots and one fast division, as the reference's
// fast-math build evaluates its transcendental form; the limits at q = 0 and
// h = 0 are the reference's (c = 1, cos theta = 1).
__device__ float gbc_weight(float inv_R, float px, float py, float pz, float sx, float sy, float sz, float inv_ls,
                            const GbcSoft &S) {
    const float rx = px - sx, ry = py - sy, rz = pz - sz;
    const float q = rx * rx + ry * ry;
    const float rq = rsqrtf(q);
    const float ell = q > 0.f ? q * rq * inv_R : 0.f;
    const float c = fmaxf(0.f, fminf(1.f, fabsf((rx * sx + ry * sy) * inv_ls * rq)));  // NaN at q = 0 -> 1
    const float d = c - ell;
    const float zr = rz * inv_R;
    const float h2 = ell * ell + zr * zr;
    const float ih = rsqrtf(h2);
    const float cos_el = h2 > 0.f ? ell * ih : 1.f;
    const float sin_el = h2 > 0.f ? fabsf(zr) * ih : 0.f;
    const float weight = __fdividef(cos_el * cos_el * cos_el * c, fmaxf(1e-9f, c * c + d * d));
    return weight * soft_of_sin(sin_el, sin_el * sin_el, S.v) * soft_of_sin2(fmaxf(0.f, 1.f - c * c), S.h);
}

struct GbcParams {
    float *vol2;  // weight-sum volume (same layout as the volume)
    float inv_R;  // 1 / R
    GbcSoft soft;
    float pos000[3];  // world centre of voxel (0, 0, 0): corner + voxwid / 2
};

// Resident CTAs per SM: the kernel is bound by the latency of its detector
// gathers, and at the unconstrained ~105 registers only 2 CTAs fit; a few
// registers spilled (view derivation, FP64 tie refinement) cost less than the
// lost occupancy (198^3 x 360 views: bilinear 22.7 -> 17.2 ms at 3 CTAs,
// nearest 19.7 -> 12.9 ms at 4).
template <bool BILIN>
__global__ void __launch_bounds__(kGThreads, BILIN ? 3 : 4) k_backproject_gbc(const ab_bp::BPParams P, const GbcParams G,
                                                               int order_f) {
    using namespace ab_bp;
    __shared__ ab_bpview sv[kGChunk];
    __shared__ ab_bpview_d svd[BILIN ? 1 : kGChunk];
    __shared__ float ssrc[kGChunk][4];  // source x, y, z, 1 / |(x, y)|

    const int64_t nvox = (int64_t)P.n[0] * P.n[1] * P.n[2];
    const int64_t e = (int64_t)blockIdx.x * kGThreads + threadIdx.x;
    const bool live = e < nvox;
    int id[3];
    if (order_f) {  // x fastest
        id[0] = (int)(e % P.n[0]);
        id[1] = (int)((e / P.n[0]) % P.n[1]);
        id[2] = (int)(e / ((int64_t)P.n[0] * P.n[1]));
    } else {  // z fastest
        id[2] = (int)(e % P.n[2]);
        id[1] = (int)((e / P.n[2]) % P.n[1]);
        id[0] = (int)(e / ((int64_t)P.n[1] * P.n[2]));
    }
    const float vw = P.voxwid;
    const float offs[3] = {1.f / (float)P.ssx, 1.f / (float)P.ssy, 1.f / (float)P.ssz};
    const int n_sub = P.ssx * P.ssy * P.ssz;
    float acc = 0.f, acc2 = 0.f;

    for (uint32_t v0 = 0; v0 < P.n_views; v0 += kGChunk) {
        const int cn = (int)min((uint32_t)kGChunk, P.n_views - v0);
        __syncthreads();
        for (int t = threadIdx.x; t < cn; t += kGThreads) {
            const ab_d3 c0d{P.cornerd[0] + 0.5 * P.vwd * P.n[0], P.cornerd[1] + 0.5 * P.vwd * P.n[1],
                            P.cornerd[2] + 0.5 * P.vwd * P.n[2]};
            const aprict_proj_spec sp = P.specs[v0 + t];
            const double hext[3] = {(0.5 * P.n[0] + 1.0) * P.vwd, (0.5 * P.n[1] + 1.0) * P.vwd,
                                    (0.5 * P.n[2] + 1.0) * P.vwd};
            if (!ab_derive_bpview(sp, c0d, vw, 0.f, hext, sv[t], BILIN ? nullptr : &svd[t]) && P.status)
                atomicOr(P.status, APRICT_STATUS_BAD_GEOMETRY);
            ssrc[t][0] = sp.source_pos.x;
            ssrc[t][1] = sp.source_pos.y;
            ssrc[t][2] = sp.source_pos.z;
            ssrc[t][3] = rsqrtf(sp.source_pos.x * sp.source_pos.x + sp.source_pos.y * sp.source_pos.y);
        }
        __syncthreads();
        if (!live) continue;
        for (int isub = 0; isub < n_sub; ++isub) {
            const int sidx[3] = {isub / (P.ssy * P.ssz), (isub / P.ssz) % P.ssy, isub % P.ssz};
            float fsub[3], rel[3], wp[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                fsub[a] = -0.5f + offs[a] * (0.5f + (float)sidx[a]);
                // relative to the volume centre, for the detector coordinate
                rel[a] = ((float)id[a] + 0.5f - 0.5f * (float)P.n[a]) * vw + fsub[a] * vw;
                // world position as the reference forms it (pos_000_c + idx voxwid + offset voxwid)
                wp[a] = (G.pos000[a] + (float)id[a] * vw) + fsub[a] * vw;
            }
            float s = 0.f, s2 = 0.f;
            for (int t = 0; t < cn; ++t) {
                const float w =
                    gbc_weight(G.inv_R, wp[0], wp[1], wp[2], ssrc[t][0], ssrc[t][1], ssrc[t][2], ssrc[t][3], G.soft);
                s2 += w;
                if (w == 0.f) continue;
                const ab_bpview &b = sv[t];
                const float rD = rcp_fast(dot4(b.den, rel[0], rel[1], rel[2]));
                const float fu = dot4(b.nu, rel[0], rel[1], rel[2]) * rD;
                const float fv = dot4(b.nv, rel[0], rel[1], rel[2]) * rD;
                const float *pvw = P.projs + (int64_t)(v0 + t) * P.stride_view;
                float pv;
                if (BILIN) {
                    pv = fetch_bilinear(P, pvw, fu, fv);
                } else {
                    float du, dv;
                    int iu = round_index(fu, -2.f, P.fnu1, du);
                    int iv = round_index(fv, -2.f, P.fnv1, dv);
                    const bool tu = fabsf(du) > b.tie_u, tv = fabsf(dv) > b.tie_v;
                    if (tu || tv) {
                        const VoxRef vr{((double)id[0] + 0.5 + (double)fsub[0] - 0.5 * P.n[0]) * P.vwd,
                                        ((double)id[1] + 0.5 + (double)fsub[1] - 0.5 * P.n[1]) * P.vwd,
                                        ((double)id[2] + 0.5 + (double)fsub[2] - 0.5 * P.n[2]) * P.vwd};
                        const ab_bpview_d &cd = svd[BILIN ? 0 : t];
                        if (tu) iu = refine_index(cd.nu, cd.den, vr, iu, du);
                        if (tv) iv = refine_index(cd.nv, cd.den, vr, iv, dv);
                    }
                    const bool inb = (unsigned)iu < P.nu && (unsigned)iv < P.nv;
                    pv = inb ? __ldg(pvw + (iu * P.su + iv * P.sv)) : 0.f;
                }
                s = fmaf(pv, w, s);
            }
            acc += s;
            acc2 += s2;
        }
    }
    if (!live) return;
    const float value = n_sub == 1 ? acc : acc / (float)n_sub;
    const float value2 = n_sub == 1 ? acc2 : acc2 / (float)n_sub;
    if (value == 0.f && value2 == 0.f) return;  // the reference writes neither (:1068-1075)
    const int64_t o = (int64_t)id[0] * P.vs[0] + (int64_t)id[1] * P.vs[1] + (int64_t)id[2] * P.vs[2];
    const float m = P.mult ? P.mult[o] : 1.f;
    if (value != 0.f) P.vol[o] = value * m + P.vol[o];
    if (value2 != 0.f) G.vol2[o] = value2 * m + G.vol2[o];
}

// Z-column layout for C-order volumes: the 32 lanes of a warp and each
// thread's kGZ voxels lie along z (voxel k of a lane 32 k further), warps
// along y, one x layer per CTA. For a view whose detector u axis and normal
// have no z component (the GBC's cylindrical scans) the thread's voxels share
// x and y, and with them everything horizontal: the depth and its
// reciprocal, u (the pixel column or the bilinear columns and their weight),
// the horizontal distance ell, the horizontal angle's cosine c, its window,
// and the weight's factor c / max(1e-9, c^2 + (c - ell)^2). Per voxel only
// the elevation (its cosine cubed and window) and v remain. Other views take
// the per-voxel formulas of k_backproject_gbc.
constexpr int kGZ = 4;

template <bool BILIN>
__global__ void __launch_bounds__(kGThreads, BILIN ? 3 : 4) k_backproject_gbc_z(const ab_bp::BPParams P, const GbcParams G,
                                                                 int gb0, int gb1) {
    using namespace ab_bp;
    __shared__ ab_bpview sv[kGChunk];
    __shared__ ab_bpview_d svd[BILIN ? 1 : kGChunk];
    __shared__ float ssrc[kGChunk][4];  // source x, y, z, 1 / |(x, y)|
    __shared__ uint8_t szinv[kGChunk];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int b0 = (int)(blockIdx.x % (unsigned)gb0), b1 = (int)((blockIdx.x / (unsigned)gb0) % (unsigned)gb1);
    const int ix = (int)(blockIdx.x / ((unsigned)gb0 * (unsigned)gb1));
    const int iy = b1 * 8 + warp, iz0 = b0 * 32 * kGZ + lane;
    const bool col_live = iy < P.n[1];
    bool live[kGZ];
#pragma unroll
    for (int k = 0; k < kGZ; ++k) live[k] = col_live && iz0 + 32 * k < P.n[2];
    const float vw = P.voxwid;
    const float offs[3] = {1.f / (float)P.ssx, 1.f / (float)P.ssy, 1.f / (float)P.ssz};
    const int n_sub = P.ssx * P.ssy * P.ssz;
    float acc[kGZ], acc2[kGZ];
#pragma unroll
    for (int k = 0; k < kGZ; ++k) acc[k] = acc2[k] = 0.f;

    for (uint32_t v0 = 0; v0 < P.n_views; v0 += kGChunk) {
        const int cn = (int)min((uint32_t)kGChunk, P.n_views - v0);
        __syncthreads();
        for (int t = threadIdx.x; t < cn; t += kGThreads) {
            const ab_d3 c0d{P.cornerd[0] + 0.5 * P.vwd * P.n[0], P.cornerd[1] + 0.5 * P.vwd * P.n[1],
                            P.cornerd[2] + 0.5 * P.vwd * P.n[2]};
            const aprict_proj_spec sp = P.specs[v0 + t];
            const double hext[3] = {(0.5 * P.n[0] + 1.0) * P.vwd, (0.5 * P.n[1] + 1.0) * P.vwd,
                                    (0.5 * P.n[2] + 1.0) * P.vwd};
            if (!ab_derive_bpview(sp, c0d, vw, 0.f, hext, sv[t], BILIN ? nullptr : &svd[t]) && P.status)
                atomicOr(P.status, APRICT_STATUS_BAD_GEOMETRY);
            ssrc[t][0] = sp.source_pos.x;
            ssrc[t][1] = sp.source_pos.y;
            ssrc[t][2] = sp.source_pos.z;
            ssrc[t][3] = rsqrtf(sp.source_pos.x * sp.source_pos.x + sp.source_pos.y * sp.source_pos.y);
            const ab_bpview &bt = sv[t];
            szinv[t] = (uint8_t)(bt.den.z == 0.f && bt.nu.z == 0.f && (BILIN || (svd[t].nu[2] == 0.0 && svd[t].den[2] == 0.0)));
        }
        __syncthreads();
        if (!__any_sync(0xffffffffu, col_live && live[0])) continue;  // warp-uniform
        for (int isub = 0; isub < n_sub; ++isub) {
            const int sidx[3] = {isub / (P.ssy * P.ssz), (isub / P.ssz) % P.ssy, isub % P.ssz};
            float fsub[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) fsub[a] = -0.5f + offs[a] * (0.5f + (float)sidx[a]);
            const int idv[2] = {ix, iy};
            float rel[2], wp[2];
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                rel[a] = ((float)idv[a] + 0.5f - 0.5f * (float)P.n[a]) * vw + fsub[a] * vw;
                wp[a] = (G.pos000[a] + (float)idv[a] * vw) + fsub[a] * vw;
            }
            float relz[kGZ], wpz[kGZ];
#pragma unroll
            for (int k = 0; k < kGZ; ++k) {
                const int iz = iz0 + 32 * k;
                relz[k] = ((float)iz + 0.5f - 0.5f * (float)P.n[2]) * vw + fsub[2] * vw;
                wpz[k] = (G.pos000[2] + (float)iz * vw) + fsub[2] * vw;
            }
            float s[kGZ], s2[kGZ];
#pragma unroll
            for (int k = 0; k < kGZ; ++k) s[k] = s2[k] = 0.f;
            for (int t = 0; t < cn; ++t) {
                const ab_bpview &b = sv[t];
                const float sx = ssrc[t][0], sy = ssrc[t][1], sz = ssrc[t][2], inv_ls = ssrc[t][3];
                const float *pvw = P.projs + (int64_t)(v0 + t) * P.stride_view;
                if (szinv[t]) {
                    // horizontal: shared by the thread's voxels
                    const float rx = wp[0] - sx, ry = wp[1] - sy;
                    const float q = rx * rx + ry * ry;
                    const float rq = rsqrtf(q);
                    const float ell = q > 0.f ? q * rq * G.inv_R : 0.f;
                    const float c = fmaxf(0.f, fminf(1.f, fabsf((rx * sx + ry * sy) * inv_ls * rq)));
                    const float d = c - ell;
                    const float ac = __fdividef(c, fmaxf(1e-9f, c * c + d * d)) *
                                     soft_of_sin2(fmaxf(0.f, 1.f - c * c), G.soft.h);
                    const float rD = rcp_fast(dot4(b.den, rel[0], rel[1], relz[0]));
                    const float fu = dot4(b.nu, rel[0], rel[1], relz[0]) * rD;
                    // u: the pixel column (nearest) or the two columns and their weight (bilinear)
                    int iu = -1, i0 = 0;
                    float fx = 0.f;
                    bool ucol = false;
                    if (BILIN) {
                        ucol = !(fu <= -1.f || fu >= (float)P.nu);
                        i0 = (int)floorf(fu);
                        fx = fu - (float)i0;
                    } else {
                        float du;
                        iu = round_index(fu, -2.f, P.fnu1, du);
                        if (fabsf(du) > b.tie_u) {
                            const VoxRef vr{((double)ix + 0.5 + (double)fsub[0] - 0.5 * P.n[0]) * P.vwd,
                                            ((double)iy + 0.5 + (double)fsub[1] - 0.5 * P.n[1]) * P.vwd, 0.0};
                            iu = refine_index(svd[BILIN ? 0 : t].nu, svd[BILIN ? 0 : t].den, vr, iu, du);
                        }
                        ucol = (unsigned)iu < P.nu;
                    }
#pragma unroll
                    for (int k = 0; k < kGZ; ++k) {
                        const float zr = (wpz[k] - sz) * G.inv_R;
                        const float h2 = ell * ell + zr * zr;
                        const float ih = rsqrtf(h2);
                        const float cos_el = h2 > 0.f ? ell * ih : 1.f;
                        const float sin_el = h2 > 0.f ? fabsf(zr) * ih : 0.f;
                        const float w = cos_el * cos_el * cos_el * ac * soft_of_sin(sin_el, sin_el * sin_el, G.soft.v);
                        s2[k] += w;
                        if (w == 0.f || !ucol) continue;
                        const float fv = dot4(b.nv, rel[0], rel[1], relz[k]) * rD;
                        float pv;
                        if (BILIN) {
                            if (fv <= -1.f || fv >= (float)P.nv) continue;
                            const int j0 = (int)floorf(fv);
                            const float fy = fv - (float)j0;
                            auto get = [&](int i, int j) -> float {
                                if (i < 0 || i >= (int)P.nu || j < 0 || j >= (int)P.nv) return 0.f;
                                return __ldg(pvw + (i * P.su + j * P.sv));
                            };
                            const float v00 = get(i0, j0), v01 = get(i0, j0 + 1), v10 = get(i0 + 1, j0),
                                        v11 = get(i0 + 1, j0 + 1);
                            const float t1 = v00 * (1.f - fx) + v10 * fx;
                            const float t2 = v01 * (1.f - fx) + v11 * fx;
                            pv = t1 * (1.f - fy) + t2 * fy;
                        } else {
                            float dv;
                            int iv = round_index(fv, -2.f, P.fnv1, dv);
                            if (fabsf(dv) > b.tie_v) {
                                const VoxRef vr{((double)ix + 0.5 + (double)fsub[0] - 0.5 * P.n[0]) * P.vwd,
                                                ((double)iy + 0.5 + (double)fsub[1] - 0.5 * P.n[1]) * P.vwd,
                                                ((double)(iz0 + 32 * k) + 0.5 + (double)fsub[2] - 0.5 * P.n[2]) *
                                                    P.vwd};
                                iv = refine_index(svd[BILIN ? 0 : t].nv, svd[BILIN ? 0 : t].den, vr, iv, dv);
                            }
                            pv = (unsigned)iv < P.nv ? __ldg(pvw + (iu * P.su + iv * P.sv)) : 0.f;
                        }
                        s[k] = fmaf(pv, w, s[k]);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < kGZ; ++k) {
                        const float w = gbc_weight(G.inv_R, wp[0], wp[1], wpz[k], sx, sy, sz, inv_ls, G.soft);
                        s2[k] += w;
                        if (w == 0.f) continue;
                        const float rD = rcp_fast(dot4(b.den, rel[0], rel[1], relz[k]));
                        const float fu = dot4(b.nu, rel[0], rel[1], relz[k]) * rD;
                        const float fv = dot4(b.nv, rel[0], rel[1], relz[k]) * rD;
                        float pv;
                        if (BILIN) {
                            pv = fetch_bilinear(P, pvw, fu, fv);
                        } else {
                            float du, dv;
                            int iu = round_index(fu, -2.f, P.fnu1, du);
                            int iv = round_index(fv, -2.f, P.fnv1, dv);
                            const bool tu = fabsf(du) > b.tie_u, tv = fabsf(dv) > b.tie_v;
                            if (tu || tv) {
                                const VoxRef vr{((double)ix + 0.5 + (double)fsub[0] - 0.5 * P.n[0]) * P.vwd,
                                                ((double)iy + 0.5 + (double)fsub[1] - 0.5 * P.n[1]) * P.vwd,
                                                ((double)(iz0 + 32 * k) + 0.5 + (double)fsub[2] - 0.5 * P.n[2]) *
                                                    P.vwd};
                                const ab_bpview_d &cd = svd[BILIN ? 0 : t];
                                if (tu) iu = refine_index(cd.nu, cd.den, vr, iu, du);
                                if (tv) iv = refine_index(cd.nv, cd.den, vr, iv, dv);
                            }
                            const bool inb = (unsigned)iu < P.nu && (unsigned)iv < P.nv;
                            pv = inb ? __ldg(pvw + (iu * P.su + iv * P.sv)) : 0.f;
                        }
                        s[k] = fmaf(pv, w, s[k]);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < kGZ; ++k) {
                acc[k] += s[k];
                acc2[k] += s2[k];
            }
        }
    }
#pragma unroll
    for (int k = 0; k < kGZ; ++k) {
        if (!live[k]) continue;
        const float value = n_sub == 1 ? acc[k] : acc[k] / (float)n_sub;
        const float value2 = n_sub == 1 ? acc2[k] : acc2[k] / (float)n_sub;
        if (value == 0.f && value2 == 0.f) continue;  // the reference writes neither (:1068-1075)
        const int64_t o = (int64_t)ix * P.vs[0] + (int64_t)iy * P.vs[1] + (int64_t)(iz0 + 32 * k) * P.vs[2];
        const float m = P.mult ? P.mult[o] : 1.f;
        if (value != 0.f) P.vol[o] = value * m + P.vol[o];
        if (value2 != 0.f) G.vol2[o] = value2 * m + G.vol2[o];
    }
}

// Expected GBC weight sum at radius r (units of R) over a perfect cylindrical
// source locus: sum over num_z heights z in [0, tan(vartheta_v) (1 + r_max)]
// (the first with weight 1/2) and num_ang source angles t in [0, pi) of the
// weight of the voxel (r, 0, 0) for the source (cos t, sin t, z), times
// 4 z_max pi / (num_z num_ang) (get_GBC_weight_integ, CB_backproject.cu:1108-1168).
//
// The weight factorises: with the voxel at (r, 0, 0) and the source at
// (cos t, sin t, z), ell and the horizontal angle depend on (r, t) only, so
//   w(r, t, z) = A(r, t) cos^3(theta) s_v(sin^2 theta),
//   A = c / max(1e-9, c^2 + (c - ell)^2) s_h(1 - c^2),
//   cos theta = ell / h, sin^2 theta = z^2 / h^2, h^2 = ell^2 + z^2.
// One thread per (radius, angle) evaluates A once and runs the height loop
// (a reciprocal square root and a few multiplies per sample). sin^2 theta
// grows with z, so the loop stops at the first height past the vertical
// window, where the window is 0 (it reaches 0 continuously at its edge).
// Heights are summed in FP32 in runs of 64, the runs in FP64; per radius an
// FP64 block sum over angles and one atomic add.
constexpr int kZRun = 64;  // heights per FP32 partial sum

// sum over heights iz = 0 .. num_z - 1 (iz = 0 with weight 1/2) of
// cos^3(theta) s_v(sin^2 theta), for horizontal distance ell. sin^2 theta
// grows with z, so the heights fall into three ranges: the window's flat part
// (s_v = 1, sin^2 < sin^2(a - b)), its soft band, and beyond (s_v = 0). The
// flat part runs first without the window's test; from the first height
// that leaves it, every sample takes the full rule until the window closes.
__device__ double height_sum(float ell, int num_z, float dz, const SoftWin &v) {
    const float e2 = ell * ell, e3 = e2 * ell;
    double tot = 0.5 * (double)soft_of_sin2(0.f, v);  // z = 0: cos theta = 1, sin theta = 0
    if (e3 == 0.f) return tot;  // ell = 0: cos theta = 0 at every z > 0
    int iz = 1;
    bool flat = true;
    while (flat && iz < num_z) {  // flat part, runs of kZRun summed in FP32
        const int stop = min(num_z, iz + kZRun);
        float part = 0.f;
        for (; iz < stop; ++iz) {
            const float z = (float)iz * dz;
            const float ih = rsqrtf(fmaf(z, z, e2));
            const float s = fabsf(z) * ih;  // sin|theta| (z < 0 when the vertical window passes pi/2)
            if (!(s * s < v.sab2)) {
                flat = false;  // this height starts the band: not consumed here
                break;
            }
            part = fmaf(e3 * ih, ih * ih, part);
        }
        tot += (double)part;
    }
    bool done = false;
    while (!done && iz < num_z) {  // soft band, until the window closes
        const int stop = min(num_z, iz + kZRun);
        float part = 0.f;
        for (; iz < stop; ++iz) {
            const float z = (float)iz * dz;
            const float ih = rsqrtf(fmaf(z, z, e2));
            const float s = fabsf(z) * ih;
            const float s2 = s * s;
            if (s2 > v.sa2) {
                done = true;
                break;
            }
            const float win = s2 < v.sab2 ? 1.f : soft_cubic(s, v);
            part = fmaf(e3 * ih * (ih * ih), win, part);
        }
        tot += (double)part;
    }
    return tot;
}

__global__ void __launch_bounds__(kGThreads) k_gbc_weight_integ(const float *r_on_R, int nr, double *out, int num_z,
                                                                int num_ang, GbcSoft S, float tan_v) {
    __shared__ double warp_sums[kGThreads / 32];
    const float maxz = tan_v * (1.f + r_on_R[nr - 1]);  // tan(soft_vartheta_v) (1 + r_max)
    const float dz = maxz / (float)(num_z - 1);
    const int ia = blockIdx.x * kGThreads + threadIdx.x;
    const bool live = ia < num_ang;
    const float t = (float)(live ? ia : 0) / (float)num_ang * 3.1415926535898f;
    const float ct = cosf(t), st = sinf(t);
    const double mult = (double)((4.f * maxz * 3.1415926535898f) / ((float)num_z * (float)num_ang));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = blockIdx.y; r < nr; r += gridDim.y) {
        double w = 0.0;
        if (live) {
            const float rx = r_on_R[r] - ct, ry = -st;  // voxel minus source, in units of R
            const float q = rx * rx + ry * ry;
            const float rq = rsqrtf(q);
            const float ell = q > 0.f ? q * rq : 0.f;
            const float c = fmaxf(0.f, fminf(1.f, fabsf((rx * ct + ry * st) * rq)));  // NaN at q = 0 -> 1
            const float d = c - ell;
            const float a = __fdividef(c, fmaxf(1e-9f, c * c + d * d)) * soft_of_sin2(fmaxf(0.f, 1.f - c * c), S.h);
            if (a != 0.f) w = (double)a * height_sum(ell, num_z, dz, S.v);
        }
#pragma unroll
        for (int k = 16; k > 0; k >>= 1) w += __shfl_xor_sync(0xffffffffu, w, k);
        if (lane == 0) warp_sums[warp] = w;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = 0.0;
            for (int k = 0; k < kGThreads / 32; ++k) b += warp_sums[k];
            if (b != 0.0) atomicAdd(out + r, b * mult);
        }
        __syncthreads();
    }
}

// k-factor of the softened Colsher window at polar angle th (radians from
// the k_z axis, |th| taken), cone angle `cone` and softening `soft`
// (_conebeam_kfactor_unchunked, gbc/filters.py:59-147): 2 pi outside
// (cone/2 - soft, pi - (cone/2 - soft)), else the cubic in sin(th).
__device__ double conebeam_kfactor(double th, double cone, double soft) {
    th = fabs(th);
    const double h = cone / 2 - soft;
    if (!(h < th && th < M_PI - h)) return 2 * M_PI;
    const double gamma = 1.0 / (sin(cone / 2 - soft) - sin(cone / 2));
    const double chi = gamma * sin(cone / 2);
    const double s = sin(th);
    const double alpha = h <= 0 ? 0.0 : fmax(0.0, fmin(1.0, sin(h) / s));
    const double beta = fmax(0.0, fmin(1.0, sin(cone / 2) >= s ? 1.0 : sin(cone / 2) / s));
    const double t1 = asin(beta) - asin(alpha);
    const double t2 = sqrt(1 - beta * beta);
    const double t3 = sqrt(1 - alpha * alpha);
    double out = t1 * 4 * (chi * chi) * (3 + 2 * chi) + 4 * asin(alpha);
    out += s * (24 * gamma * chi * (1 + chi) * (t2 - t3));
    out += s * s * (6 * gamma * gamma * (1 + 2 * chi) * (t1 - beta * t2 + alpha * t3));
    out += s * s * s * (-2.0 / 3.0 * gamma * gamma * gamma * (-9 * (t2 - t3) + (cos(3 * asin(beta)) - cos(3 * asin(alpha)))));
    return out;
}

__device__ double fftfreq(int k, int n) { return (double)(k < (n + 1) / 2 ? k : k - n) / (double)n; }

__device__ double sinc(double x) {
    if (x == 0.0) return 1.0;
    const double px = M_PI * x;
    return sin(px) / px;
}

struct SpecParams {
    float2 *spec;  // (n0, n1, n2 / 2 + 1) complex, C order
    int n0, n1, n2;
    double multiplier, cone, soft;
};

// One pass over the rfftn spectrum of an (n0, n1, n2) volume (axis 2 = z,
// the cylinder axis): times |k| * multiplier, divided by the k-factor of the
// polar angle (cone > 0; cone = pi gives 2 pi; cone = 0 uses the lateral |k|
// without a k-factor), times sinc(f0) sinc(f1) sinc(f2); the DC term is set
// to 0 (filters.py:340-398).
__global__ void __launch_bounds__(kGThreads) k_conebeam_spectral(const SpecParams P) {
    const int m2 = P.n2 / 2 + 1;
    const int64_t n = (int64_t)P.n0 * P.n1 * m2;
    const int64_t step = (int64_t)gridDim.x * kGThreads;
    for (int64_t e = (int64_t)blockIdx.x * kGThreads + threadIdx.x; e < n; e += step) {
        const int k2 = (int)(e % m2);
        const int64_t r = e / m2;
        const int k1 = (int)(r % P.n1), k0 = (int)(r / P.n1);
        const double f0 = fftfreq(k0, P.n0), f1 = fftfreq(k1, P.n1), f2 = (double)k2 / (double)P.n2;
        const double lat2 = f0 * f0 + f1 * f1;
        double factor;
        if (P.cone == 0.0) {
            factor = sqrt(lat2) * P.multiplier;
        } else {
            factor = sqrt(lat2 + f2 * f2) * P.multiplier;
            const double th = fabs(M_PI / 2 - atan2(f2, sqrt(lat2)));
            factor /= P.cone == M_PI ? 2 * M_PI : conebeam_kfactor(th, P.cone, P.soft);
        }
        factor *= sinc(f0) * sinc(f1) * sinc(f2);
        if (e == 0) factor = 0.0;
        const float2 z = P.spec[e];
        P.spec[e] = make_float2((float)((double)z.x * factor), (float)((double)z.y * factor));
    }
}

// out[x][y][z] += trilinear value of low at (x, y, z) / d - 1/2 + 1/(2d) per
// axis, neighbour indices clamped to the array (scipy.ndimage.map_coordinates
// order 1, mode "nearest", the reference's low-resolution correction,
// filters.py:403-455). Both arrays C order (z fastest).
__global__ void __launch_bounds__(kGThreads) k_add_upsampled(float *out, int n0, int n1, int n2, const float *low,
                                                             int m0, int m1, int m2, int d) {
    const int64_t n = (int64_t)n0 * n1 * n2;
    const int64_t step = (int64_t)gridDim.x * kGThreads;
    for (int64_t e = (int64_t)blockIdx.x * kGThreads + threadIdx.x; e < n; e += step) {
        const int z = (int)(e % n2);
        const int64_t r = e / n2;
        const int y = (int)(r % n1), x = (int)(r / n1);
        const int idx[3] = {x, y, z}, lim[3] = {m0, m1, m2};
        int i0[3], i1[3];
        double t[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double c = (double)idx[a] / d - 0.5 + 1.0 / d / 2;
            const double f = floor(c);
            t[a] = c - f;
            const int fi = (int)f;
            i0[a] = min(max(fi, 0), lim[a] - 1);
            i1[a] = min(max(fi + 1, 0), lim[a] - 1);
        }
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int a = c >> 2 & 1, b = c >> 1 & 1, g = c & 1;
            const double w = (a ? t[0] : 1 - t[0]) * (b ? t[1] : 1 - t[1]) * (g ? t[2] : 1 - t[2]);
            const int ix = a ? i1[0] : i0[0], iy = b ? i1[1] : i0[1], iz = g ? i1[2] : i0[2];
            v += w * (double)low[((int64_t)ix * m1 + iy) * m2 + iz];
        }
        out[e] += (float)v;
    }
}

unsigned grid_for(int64_t n) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 148;
    const int64_t want = (n + kGThreads - 1) / kGThreads, cap = (int64_t)sms * 16;
    return (unsigned)(want < cap ? want : cap);
}

bool finite_soft(const aprict_backproject_config *c) {
    return std::isfinite(c->soft_vartheta_v) && std::isfinite(c->soft_vartheta_v_softspan) &&
           std::isfinite(c->soft_vartheta_h) && std::isfinite(c->soft_vartheta_h_softspan);
}

}  // namespace

extern "C" int aprict_b200_backproject_gbc(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                           const float *projs_dev, const aprict_vol_desc *vd, float *vol_dev,
                                           float *weightsum_dev, const float *multiplier_dev,
                                           const aprict_backproject_config *cfg, uint32_t *status_dev,
                                           aprict_stream_t stream) {
    if (cfg == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null backproject config");
    if (cfg->weighting_preset != 7)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "the GBC backprojection takes weighting preset 7");
    if (cfg->exact) return ab_fail(APRICT_ERR_UNSUPPORTED, "the GBC backprojection is a fast (approximate) mode");
    if (!(cfg->Z_on_val_factor_val > 0.f) || !finite_soft(cfg))
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "GBC needs R > 0 in Z_on_val_factor_val and finite soft windows");
    if (weightsum_dev == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "GBC needs a weight-sum volume");
    if ((reinterpret_cast<uintptr_t>(weightsum_dev) & 3u) != 0)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "weight-sum volume pointer not 4-byte aligned");
    if (weightsum_dev == vol_dev) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "the weight sums need their own volume");
    aprict_backproject_config c = *cfg;
    c.weighting_preset = 0;  // validated here; the shared checks below know presets 0-6
    ab_bp::BPParams P;
    uint64_t units = 0;
    int xb = 2;
    int rc = ab_bp::make_bp_params(specs_dev, pd, projs_dev, vd, vol_dev, multiplier_dev, &c, status_dev, P, units,
                                   xb, 2);
    if (rc != APRICT_OK || units == 0) return rc;
    GbcParams G;
    G.vol2 = weightsum_dev;
    G.inv_R = (float)(1.0 / (double)cfg->Z_on_val_factor_val);
    G.soft = GbcSoft{soft_win(cfg->soft_vartheta_v, cfg->soft_vartheta_v_softspan),
                     soft_win(cfg->soft_vartheta_h, cfg->soft_vartheta_h_softspan)};
    G.pos000[0] = vd->corner.x + 0.5f * vd->voxwid;
    G.pos000[1] = vd->corner.y + 0.5f * vd->voxwid;
    G.pos000[2] = vd->corner.z + 0.5f * vd->voxwid;
    const int64_t nvox = (int64_t)vd->nx * vd->ny * vd->nz;
    const int64_t blocks = (nvox + kGThreads - 1) / kGThreads;
    if (blocks > 0x7fffffffLL) return ab_fail(APRICT_ERR_TOO_LARGE, "volume too large for the grid");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int order_f = vd->order != 0;
    if (!order_f) {  // C order: z columns (see k_backproject_gbc_z)
        const int64_t gb0 = ((int64_t)vd->nz + 32 * kGZ - 1) / (32 * kGZ), gb1 = ((int64_t)vd->ny + 7) / 8;
        const int64_t zblocks = gb0 * gb1 * (int64_t)vd->nx;
        if (zblocks > 0x7fffffffLL) return ab_fail(APRICT_ERR_TOO_LARGE, "volume too large for the grid");
        if (cfg->approx_mode_linear_interpolate)
            k_backproject_gbc_z<true><<<(unsigned)zblocks, kGThreads, 0, st>>>(P, G, (int)gb0, (int)gb1);
        else
            k_backproject_gbc_z<false><<<(unsigned)zblocks, kGThreads, 0, st>>>(P, G, (int)gb0, (int)gb1);
    } else if (cfg->approx_mode_linear_interpolate) {
        k_backproject_gbc<true><<<(unsigned)blocks, kGThreads, 0, st>>>(P, G, order_f);
    } else {
        k_backproject_gbc<false><<<(unsigned)blocks, kGThreads, 0, st>>>(P, G, order_f);
    }
    return ab_cuda_check(cudaGetLastError(), "backproject_gbc launch");
}

extern "C" int aprict_b200_gbc_weight_integral(const float *r_on_R_dev, int32_t n_r, double *out_dev, int32_t num_z,
                                               int32_t num_ang, const aprict_backproject_config *cfg,
                                               aprict_stream_t stream) {
    if (cfg == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null backproject config");
    if (n_r <= 0) return APRICT_OK;
    if (r_on_R_dev == nullptr || out_dev == nullptr)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null radius or output array");
    if (num_z < 2 || num_ang < 1 || (int64_t)num_z * num_ang > (int64_t)1 << 31)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "num_z must be >= 2, num_ang >= 1, num_z * num_ang <= 2^31");
    if (!finite_soft(cfg)) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "non-finite soft windows");
    const GbcSoft S{soft_win(cfg->soft_vartheta_v, cfg->soft_vartheta_v_softspan),
                    soft_win(cfg->soft_vartheta_h, cfg->soft_vartheta_h_softspan)};
    const dim3 grid((unsigned)((num_ang + kGThreads - 1) / kGThreads), (unsigned)min(n_r, 65535));
    k_gbc_weight_integ<<<grid, kGThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        r_on_R_dev, n_r, out_dev, num_z, num_ang, S, (float)tan((double)cfg->soft_vartheta_v));
    return ab_cuda_check(cudaGetLastError(), "gbc_weight_integral launch");
}

extern "C" int aprict_b200_conebeam_spectral(void *spec_dev, int32_t n0, int32_t n1, int32_t n2, double multiplier,
                                             double cone_angle, double theta_soft, aprict_stream_t stream) {
    if (n0 <= 0 || n1 <= 0 || n2 <= 0) return APRICT_OK;
    if (spec_dev == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null spectrum");
    if ((reinterpret_cast<uintptr_t>(spec_dev) & 7u) != 0)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "spectrum pointer not 8-byte aligned");
    if (!(cone_angle >= 0.0 && cone_angle <= M_PI))
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "cone angle must lie in [0, pi]");
    if (!std::isfinite(multiplier) || !std::isfinite(theta_soft))
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "non-finite multiplier or softening");
    SpecParams P{static_cast<float2 *>(spec_dev), n0, n1, n2, multiplier, cone_angle, theta_soft};
    const int64_t n = (int64_t)n0 * n1 * (n2 / 2 + 1);
    k_conebeam_spectral<<<grid_for(n), kGThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(P);
    return ab_cuda_check(cudaGetLastError(), "conebeam_spectral launch");
}

extern "C" int aprict_b200_add_upsampled(float *out_dev, int32_t n0, int32_t n1, int32_t n2, const float *low_dev,
                                         int32_t m0, int32_t m1, int32_t m2, int32_t factor, aprict_stream_t stream) {
    if (n0 <= 0 || n1 <= 0 || n2 <= 0) return APRICT_OK;
    if (out_dev == nullptr || low_dev == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null array");
    if (m0 <= 0 || m1 <= 0 || m2 <= 0 || factor <= 0)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "empty low-resolution array or non-positive factor");
    const int64_t n = (int64_t)n0 * n1 * n2;
    k_add_upsampled<<<grid_for(n), kGThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(out_dev, n0, n1, n2,
                                                                                          low_dev, m0, m1, m2, factor);
    return ab_cuda_check(cudaGetLastError(), "add_upsampled launch");
}
