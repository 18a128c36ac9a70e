// ab_bpbrick.cuh -- the voxel-driven backprojector's work unit, shared by
// the one-scan kernel (ab_backproject.cu) and the persistent multi-scan
// kernel (ab_batch.cu).
//
// Replaces backproject_CB_voltex<float,float>
// (src/aprict/data/cusrc/CB_backproject.cu:952-1027; per-voxel body
// _backproject_CB_getval :313-733) and the host loop that launches it once per
// 10 views with the 640-byte proj_chunk_spec_maxlen10 passed by value
// (src/aprict/cb/flatpanel.py:1192-1278).
//
// B200 layout: a warp covers 32 consecutive voxels along the volume's fastest
// axis, so the final read-modify-write of the volume is one coalesced 128-byte
// line per warp, and for circular scans the 32 voxel centres project onto one
// detector column -- the projection gathers of a warp fall into 2-3 lines.
// Each thread carries XB voxels along the slowest axis (independent
// accumulators for ILP). Per-view coefficients (ab_bpview) are derived once per
// CTA into shared memory and read as uniform broadcasts; the volume is read and
// written exactly once per call instead of once per 10 views. CTAs are issued
// in brick order (all of the fastest axis x a compact block of the other two)
// so that the CTAs resident at one time project onto a small part of each
// view and the projection data they gather stays in L2.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "ab_bpview.cuh"
#include "ab_host.h"

namespace ab_bp {

constexpr int kThreads = 256;  // 32 (fast axis) x 8 (middle axis)
// Views per shared-memory chunk: 128, or 64 with 8 voxels per thread (whose
// per-voxel shared arrays are twice as large; the static 48 KB holds both).
template <int XB>
constexpr int chunk_views() { return XB == 8 ? 64 : 128; }

struct BPParams {
    const aprict_proj_spec *specs;
    uint32_t n_views, nu, nv;
    int64_t stride_view;
    int su, sv;  // u, v element strides (in-view offsets are checked to fit 32 bits)
    // -0x4B400000 (su + sv) mod 2^32: turns the bit patterns of two magic-rounded
    // coordinates into the pixel offset with two multiply-adds
    uint32_t koff;
    float fnu1, fnv1;  // nu + 1, nv + 1: clamp bounds for the rounded pixel index
    const float *projs;
    float *vol;
    const float *mult;
    int n[3];        // volume shape (x, y, z)
    int64_t vs[3];   // element strides (x, y, z)
    float voxwid;
    float c0[3];     // volume centre (world)
    double cornerd[3];
    double vwd;
    // brick-ordered CTA remap
    int gb[3];       // blocks along fastest, middle, slowest axis
    int sb1, sb2;    // super-brick extent in blocks along middle, slowest axis
    int nsb1;        // super-bricks along the middle axis
    // config
    int mask;
    float mask_r2;
    int all_ones;
    float sep, inv_sep;
    int pL, pV;
    float val;
    float inv_val;  // 1 / val
    int preset;     // direct-raycast weighting preset 0-6
    int ssx, ssy, ssz;
    int wide;  // su, sv < 2^30: byte addresses as two 32 x 32 -> 64-bit multiply-adds
    uint32_t *status;
};

// Pixel index with the reference's zero-order rule (get_zero_interp,
// CB_backproject.cu:256-271): floor(f + 0.5). The FP32 estimate of f carries
// an error below a per-view a priori bound (ab_fp32_pixel_error_bound; about
// 5e-4 pixel on a 384-pixel detector, 1e-4 observed). When f lies within 1.5x
// that bound of a half-integer (|f - round(f)| > tie_u / tie_v of the view)
// the choice is made again in FP64 from the voxel's exact position.

// x + 1.5 * 2^23 rounds x to the nearest integer (ties to even), which then
// sits in the low mantissa bits; valid for |x| < 2^22 (the clamp ensures it,
// and sends NaN to lo). frac = x - index, in [-1/2, 1/2]. Round-to-even and
// floor(x + 1/2) differ only at exact half-integers, which the caller always
// refines.
constexpr float kMagic = 12582912.0f;

__device__ __forceinline__ int round_index(float x, float lo, float hi, float &frac) {
    const float xc = fminf(fmaxf(x, lo), hi);
    const float t = __fadd_rn(xc, kMagic);
    frac = __fsub_rn(xc, __fsub_rn(t, kMagic));
    return __float_as_int(t) - 0x4B400000;
}

// FP64 position of a voxel (centre + sub-sample offset) relative to the
// volume centre, from its integer indices: exact in double.
struct VoxRef {
    double x, y, z;
};

// floor(N/D + 1/2) in FP64 given the FP32 estimate i of the rounded value
// and its fraction (f - i): the answer is i or its neighbour on the side of
// frac, decided by the sign of N - (i +- 1/2) D without a division.
__device__ __forceinline__ int refine_index(const double *num, const double *den, const VoxRef &r, int i, float frac) {
    const double N = fma(num[0], r.x, fma(num[1], r.y, fma(num[2], r.z, num[3])));
    const double D = fma(den[0], r.x, fma(den[1], r.y, fma(den[2], r.z, den[3])));
    if (!(D != 0.0) || !(fabs(N) < 1e300)) return -1;
    const double h = frac > 0.f ? (double)i + 0.5 : (double)i - 0.5;
    const double e = fma(-h, D, N);  // (N/D - h) * D
    if (frac > 0.f) return (D > 0.0 ? e >= 0.0 : e <= 0.0) ? i + 1 : i;
    return (D > 0.0 ? e < 0.0 : e > 0.0) ? i - 1 : i;
}

// Bilinear rule of get_bilinear_interp (CB_backproject.cu:221-254), same
// operation order.
__device__ __forceinline__ float fetch_bilinear(const BPParams &P, const float *pvw, float fu, float fv) {
    if (fu <= -1.f || fv <= -1.f || fu >= (float)P.nu || fv >= (float)P.nv) return 0.f;
    const int i0 = (int)floorf(fu), j0 = (int)floorf(fv);
    const float fx = fu - (float)i0, fy = fv - (float)j0;
    auto get = [&](int i, int j) -> float {
        if (i < 0 || i >= (int)P.nu || j < 0 || j >= (int)P.nv) return 0.f;
        return __ldg(pvw + (i * P.su + j * P.sv));
    };
    const float v00 = get(i0, j0), v01 = get(i0, j0 + 1), v10 = get(i0 + 1, j0), v11 = get(i0 + 1, j0 + 1);
    const float t1 = v00 * (1.f - fx) + v10 * fx;
    const float t2 = v01 * (1.f - fx) + v11 * fx;
    return t1 * (1.f - fy) + t2 * fy;
}

__device__ __forceinline__ float dot4(const float4 a, float x, float y, float z) {
    return fmaf(a.x, x, fmaf(a.y, y, fmaf(a.z, z, a.w)));
}

// 1/x with one MUFU op (relative error < 2^-22); nearest-pixel ties are
// settled in FP64 separately.
__device__ __forceinline__ float rcp_fast(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// sqrt with one MUFU op (relative error ~2^-22), for the exact mode's chord
// lengths. The reference builds its kernels with -use_fast_math
// (src/aprict/cuda/header_injection.py:54-59), where sqrtf is this
// approximation as well.
__device__ __forceinline__ float sqrt_fast(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float taper(const ab_bpview &b, float fu, float fv, float inv_sep) {
    if (fabsf(fu - b.cu0) <= b.tap_ru && fabsf(fv - b.cv0) <= b.tap_rv) return 1.f;
    return ab_edge_taper(fu - b.cu0, fv - b.cv0, b.inv_halfu, b.inv_halfv, inv_sep);
}

// True when every point of the box [lo, hi] (relative to the volume centre)
// projects beyond one edge of the detector by more than the view's
// off-detector margin plus `extra` (1/2 for the bilinear taps and the exact
// footprints): its samples are then all 0. The projection of the box is the
// convex hull of its corners' projections when all of them lie in front of
// the source (D > 0); corner coordinates carry the same FP32 error bound as
// the voxels' (within the out_ru / out_rv margin).
__device__ __forceinline__ bool brick_off_detector(const ab_bpview &b, const float lo[3], const float hi[3],
                                                   float extra) {
    float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f;
    bool front = true;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float x = (c & 4) ? hi[0] : lo[0], y = (c & 2) ? hi[1] : lo[1], z = (c & 1) ? hi[2] : lo[2];
        const float D = dot4(b.den, x, y, z);
        front = front && D > 0.f;
        const float rD = rcp_fast(D);
        const float fu = dot4(b.nu, x, y, z) * rD - b.cu0, fv = dot4(b.nv, x, y, z) * rD - b.cv0;
        umin = fminf(umin, fu);
        umax = fmaxf(umax, fu);
        vmin = fminf(vmin, fv);
        vmax = fmaxf(vmax, fv);
    }
    const float eu = b.out_ru + extra, ev = b.out_rv + extra;
    return front && (umin > eu || umax < -eu || vmin > ev || vmax < -ev);
}

// True when every point of the box [lo, hi] (relative to the volume centre)
// projects, in the FP32 evaluation of the fast modes, into the flat box of the
// detector-edge taper (inside the detector, taper weight exactly 1). The exact
// projection of the box lies within the hull of its corners' projections
// when all of them lie in front of the source; the FP32 coordinates of the
// corners and of any voxel each carry at most the view's error bound, which
// is below (1/2 - tie) / 1.5, so two bounds plus 1e-3 pixel are kept free
// (plus `extra`: 1/2 keeps both bilinear taps of every voxel on the detector).
__device__ __forceinline__ bool brick_in_flat_box(const ab_bpview &b, const float lo[3], const float hi[3],
                                                  float extra = 0.f) {
    float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f;
    bool front = true;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float x = (c & 4) ? hi[0] : lo[0], y = (c & 2) ? hi[1] : lo[1], z = (c & 1) ? hi[2] : lo[2];
        const float D = dot4(b.den, x, y, z);
        front = front && D > 0.f;
        const float rD = rcp_fast(D);
        const float fu = dot4(b.nu, x, y, z) * rD - b.cu0, fv = dot4(b.nv, x, y, z) * rD - b.cv0;
        umin = fminf(umin, fu);
        umax = fmaxf(umax, fu);
        vmin = fminf(vmin, fv);
        vmax = fmaxf(vmax, fv);
    }
    const float mu = (0.5f - b.tie_u) * (4.f / 3.f) + 1e-3f + extra, mv = (0.5f - b.tie_v) * (4.f / 3.f) + 1e-3f + extra;
    return front && umin - mu >= -b.tap_ru && umax + mu <= b.tap_ru && vmin - mv >= -b.tap_rv &&
           vmax + mv <= b.tap_rv;
}

// x^e for a small integer e with one approximate reciprocal for e < 0
// (relative error ~1e-6; the reference divides e times, CB_backproject.cu:21-35).
__device__ __forceinline__ float powi_fast(float x, int e) {
    const float r = e < 0 ? rcp_fast(x) : x;
    const int n = e < 0 ? -e : e;
    float a = 1.f;
    for (int k = 0; k < n; ++k) a *= r;
    return a;
}

// Cone-cylinder weighting presets 1-6 of the direct-raycast mode
// (CB_backproject.cu:530-599), R = val: xw, yw the voxel's world x, y; Z its
// distance from the source along the source-detector axis.
__device__ __forceinline__ float preset_weight(int preset, float R, float xw, float yw, float sx, float sy, float Z) {
    const float rx = xw - sx, ry = yw - sy;
    const float ell = sqrtf(rx * rx + ry * ry) / R;
    const float zr = Z / R;
    const float c = fmaxf(0.f, fminf(1.f, fabsf(zr / ell)));
    const float d = c - ell;
    const float vy = (sx * yw - sy * xw) / R / R, vx = (sx * xw + sy * yw) / R / R;
    const float dc = d / c;
    const float q = (1.f - dc * dc) / (1.f + dc * dc);
    switch (preset) {
        case 1: return 1.f / (c * c * (c * c + d * d));
        case 2: return -2.f * q * q * (-vy) * (1.f + vx / zr) / (ell * ell) / R * R;
        case 3: return 1.f / (zr * c * c);
        case 4: return (vy / zr) / zr;
        case 6: return -2.f * q * q / (1.f - dc) * (-vy) * (1.f + vx / zr) / zr;
        default: return 1.f;  // preset 5 carries no extra factor
    }
}

// (Z/L)^pL (Z/val)^pV, the direct-raycast weights (CB_backproject.cu:512-528).
__device__ __forceinline__ float zpow(const BPParams &P, const ab_bpview &b, float Z) {
    float w = 1.f;
    if (P.pL != 0) w *= powi_fast(Z * b.invL, P.pL);
    if (P.pV != 0) w *= powi_fast(Z * P.inv_val, P.pV);
    return w;
}

// EXACT: chord-length footprint (CB_backproject.cu:408-477).
// RAYCAST: fast mode with direct-raycast weights (:512-646, preset 0).
// BILIN: bilinear instead of nearest detector sampling.
// ORD: 0 = C order (fastest axis z, slowest x), 1 = F order (fastest x).
// XB: voxels per thread along the slowest axis (2, 4 or 8: more reuse of each
// view's coefficients against fewer registers per voxel).
// Shared-memory staging of one chunk of per-view coefficients.
// Fast modes also keep, per warp, a queue of deferred voxel-views (see
// bp_brick) and the per-(lane, voxel) sums of their contributions.
constexpr int kWarps = kThreads / 32;
// Queue entry: (view in chunk) << (5 + kbits) | k << 5 | lane, kbits = log2 XB.
template <int XB>
constexpr int q_kbits() { return XB == 2 ? 1 : (XB == 4 ? 2 : 3); }
static_assert((chunk_views<8>() - 1) << (5 + q_kbits<8>()) < 65536, "queue entries are 16 bits");
static_assert((chunk_views<4>() - 1) << (5 + q_kbits<4>()) < 65536, "queue entries are 16 bits");
static_assert(chunk_views<2>() <= 256 && chunk_views<2>() % 32 == 0 && chunk_views<8>() % 32 == 0,
              "chunk views are compacted 32 at a time into 8-bit indices");

// Resident CTAs per SM the kernels are compiled for (launch bounds), by XB
// and mode; also the default number of CTA waves per super-brick. The fast
// modes are bound by the latency of the pixel gathers: more resident warps
// beat the few registers spilled to (L1-resident) local memory at 64
// registers a thread, in the exact mode too.
constexpr int kExactBlocks = 4;
constexpr int bp_min_blocks(int xb, bool exact) { return exact ? kExactBlocks : (xb == 8 ? 3 : 4); }
// Default voxels per thread: 4 in the fast modes, 2 in the exact mode (whose
// per-voxel footprint loop gains nothing from sharing a view's coefficients).
constexpr int default_xb(bool exact) { return exact ? 2 : 4; }

// Whether a kernel variant keeps the per-warp view table (the z-column
// layout's fast nearest mode).
constexpr bool bp_ztable(int ord, bool exact, bool raycast, bool bilin) { return ord == 3 && !exact && !raycast && !bilin; }

template <bool EXACT, bool BILIN, int XB, bool ZT = false>
struct BPSmem {
    static constexpr bool kNear = !EXACT && !BILIN;
    static constexpr int kQCap = 32 + 32 * XB;  // a flush leaves < 32; one view adds <= 32 * XB
    static constexpr int kChunk = chunk_views<XB>();
    ab_bpview sv[kChunk];
    float4 sd[kChunk];  // per view: steps of N_u, N_v, D, Z along the thread's XB axis
    ab_bpview_d svd[kNear ? kChunk : 1];
    ab_bpview_exact sx[EXACT ? kChunk : 1];
    float box[6];             // the brick's box (low corner, high corner) relative to the volume centre
    float boxa[6];            // the box of every thread's voxels (not clipped to the volume)
    uint8_t inner[kChunk];    // per view: every voxel of the CTA projects into the flat box
    int vcount;               // views of the chunk whose brick projection reaches the detector
    uint8_t off_det[kChunk];  // per view: the whole brick projects beyond one detector edge
    uint8_t zinv[kChunk];     // per view: depth and u do not change along z (ORD 3 shares them)
    uint8_t vzero[kChunk];    // per view (slice stacks): one detector row, v form identically zero
    uint8_t vlist[kChunk];    // those views' indices in the chunk, in order
    uint16_t q[EXACT ? 1 : kWarps][EXACT ? 1 : kQCap];
    // Nearest mode, z-column layout: per warp, the warp-uniform part of 32
    // consecutive views of the chunk (rD, weight, and the 64-bit byte address
    // of the column's pixel 0 less 4 * 0x4B400000 * sv, split in two words; rD
    // NaN when the warp's column misses the detector)
    float4 zrec[ZT ? kWarps : 1][ZT ? 32 : 1];
    // Compensated per-voxel totals over the view chunks: sum and Kahan term,
    // [warp][lane * XB + k], each slot owned by one thread.
    float ksum[kWarps][32 * XB];
    float kcomp[kWarps][32 * XB];
};

// One backprojection work unit: brick `brick` (brick order) of the volume,
// all views. Every thread of the CTA calls it with the same brick; it contains
// __syncthreads and returns uniformly.
template <int ORD, bool EXACT, bool RAYCAST, bool BILIN, int XB, bool SKIP = RAYCAST>
__device__ __forceinline__ void bp_brick(const BPParams &P, uint32_t brick,
                                         BPSmem<EXACT, BILIN, XB, bp_ztable(ORD, EXACT, RAYCAST, BILIN)> &sm) {
    static_assert(XB == 2 || XB == 4 || XB == 8, "XB is 2, 4 or 8");
    constexpr int kXB = XB, kKB = q_kbits<XB>();
    constexpr int kChunk = chunk_views<XB>();
    constexpr bool kNear = !EXACT && !BILIN;
    ab_bpview *sv = sm.sv;
    ab_bpview_d *svd = sm.svd;
    ab_bpview_exact *sx = sm.sx;

    // Brick-ordered block coordinates (uniform per CTA).
    const int per_sb = P.gb[0] * P.sb1 * P.sb2;
    const int sb = (int)brick / per_sb;
    int r = (int)brick - sb * per_sb;
    const int b0 = r % P.gb[0];
    r /= P.gb[0];
    const int b1 = (sb % P.nsb1) * P.sb1 + r % P.sb1;
    const int b2 = (sb / P.nsb1) * P.sb2 + r / P.sb1;
    if (b1 >= P.gb[1] || b2 >= P.gb[2]) return;  // the whole CTA returns before any barrier

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // Axes: a0 along the lanes (memory-contiguous), a1 along the warps, a2
    // along each thread's XB voxels. ORD 0: C order (z, y, x); ORD 1: F order
    // (x, y, z); ORD 2: C order with nz == 1 (slices): lanes along y (stride
    // 1), warps and XB both along x, z = 0. ORD 3: C order with the lanes and
    // each thread's XB voxels all along z (voxel k of a lane 32 k further),
    // one x layer per CTA: a thread's voxels then share x and y, so for views
    // whose detector u axis and normal have no z component (circular and
    // helical scans with an upright detector) the voxels share their depth and
    // u coordinate, which are computed once per warp and view (the fast modes)
    // or once per thread and view (the exact mode).
    constexpr bool kZ = ORD == 3;
    constexpr int a0 = ORD == 0 || ORD == 3 ? 2 : (ORD == 1 ? 0 : 1);
    constexpr int a1 = ORD == 2 ? 2 : 1;
    constexpr int a2 = ORD == 1 || ORD == 3 ? 2 : 0;
    constexpr int kStride = kZ ? 32 : 1;  // index step between a thread's voxels along a2
    const int i0 = b0 * 32 * (kZ ? kXB : 1) + lane;
    const int i1 = ORD == 2 ? 0 : b1 * 8 + warp;
    const int i2b = ORD == 2 ? (b1 * 8 + warp) * kXB : (kZ ? i0 : b2 * kXB);
    const bool in01 = i0 < P.n[a0] && i1 < P.n[a1] && (!kZ || b2 < P.n[0]);
    // (x, y, z) indices of voxel k of lane ln of this warp
    auto vox_id = [&](int ln, int k, int id[3]) {
        if constexpr (kZ) {
            id[0] = b2;
            id[1] = i1;
            id[2] = b0 * 32 * kXB + ln + 32 * k;
        } else {
            id[a0] = b0 * 32 + ln;
            id[a1] = i1;
            id[a2] = i2b + k;
        }
    };

    // Voxel-centre coordinates relative to the volume centre, per axis.
    const float vw = P.voxwid;
    float base[3];
    int idx[3];
    vox_id(lane, 0, idx);
#pragma unroll
    for (int a = 0; a < 3; ++a) base[a] = ((float)idx[a] + 0.5f - 0.5f * (float)P.n[a]) * vw;

    // Cylinder mask about world x = y = 0 (CB_backproject.cu:339-343).
    bool live[kXB];
    bool any_live = false;
#pragma unroll
    for (int k = 0; k < kXB; ++k) {
        float c[3] = {base[0], base[1], base[2]};
        c[a2] += (float)(k * kStride) * vw;
        bool ok = in01 && (i2b + k * kStride) < P.n[a2];
        if (ok && P.mask) {
            const float xw = c[0] + P.c0[0], yw = c[1] + P.c0[1];
            ok = !(xw * xw + yw * yw > P.mask_r2);
        }
        live[k] = ok;
        any_live |= ok;
    }

    // SKIP (by default in the direct-raycast mode, the cone-cylinder FBP's,
    // whose views each see only a slab of the volume): skip the views whose
    // projection of the brick misses the detector, and leave voxel-views
    // certainly off the detector out of the second pass. The one-scan kernel's
    // other modes keep the plain loop: measured 3 % slower with the skip on a
    // circular scan that never misses.
    // Slice stacks (ORD 2: fan-beam sinograms on a one-row detector) always see
    // their slice, so they skip nothing and keep the plain loop (the skip's
    // per-view work measured 15 % on 64 fan-beam slices).
    constexpr bool kSkip = SKIP && !EXACT && ORD != 2;
    // Interior bricks (fast and direct-raycast modes, nearest or bilinear): in a
    // view that projects the whole brick into the detector's flat box, only
    // near-tie pixel choices can need the second pass (none with bilinear
    // taps), and the voxels take a predicate-free pass (see the view loop).
    // Not for slice stacks, whose
    // small bricks pay more for the per-view corner projections than the pass
    // saves (64 fan-beam slices: 1953 -> 1830 slices/s with it).
    constexpr bool kInt = !EXACT && ORD != 2;
    // The brick's box relative to the volume centre (voxel faces, clipped to
    // the volume): every sub-sample of its voxels lies inside. Kept in shared
    // memory for the per-view off-detector test (ordered by the chunk loop's
    // first barrier).
    if ((kSkip || kInt) && threadIdx.x == 0) {
        int lo[3], hi[3], ha[3];
        if constexpr (kZ) {
            lo[0] = b2;
            hi[0] = b2 + 1;
            lo[1] = b1 * 8;
            ha[1] = b1 * 8 + 8;
            lo[2] = b0 * 32 * kXB;
            ha[2] = lo[2] + 32 * kXB;
            ha[0] = hi[0];
        } else {
            lo[a0] = b0 * 32;
            ha[a0] = b0 * 32 + 32;
            lo[a1] = ORD == 2 ? 0 : b1 * 8;
            ha[a1] = ORD == 2 ? 1 : b1 * 8 + 8;
            lo[a2] = ORD == 2 ? b1 * 8 * kXB : i2b;
            ha[a2] = lo[a2] + (ORD == 2 ? 8 * kXB : kXB);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (!(kZ && a == 0)) hi[a] = min(ha[a], P.n[a]);
            sm.box[a] = sm.boxa[a] = ((float)lo[a] - 0.5f * (float)P.n[a]) * vw;
            sm.box[3 + a] = ((float)hi[a] - 0.5f * (float)P.n[a]) * vw;
            sm.boxa[3 + a] = ((float)ha[a] - 0.5f * (float)P.n[a]) * vw;
        }
    }

    // One accumulator per voxel over all views and sub-samples; the mean over
    // the ssx*ssy*ssz sub-samples is taken at the end (the reference averages
    // level by level, CB_backproject.cu:717-731 -- the same value up to float
    // rounding, identical when there is no supersampling). Compensated
    // summation: acc holds the plain FP32 sum of at most one chunk of views
    // (kChunk), which is then added to the voxel's total with Kahan's
    // compensation (total and compensation in shared memory, no registers).
    float acc[kXB];
    float *ksum = sm.ksum[warp], *kcomp = sm.kcomp[warp];
#pragma unroll
    for (int k = 0; k < kXB; ++k) {
        acc[k] = 0.f;
        ksum[lane * kXB + k] = 0.f;
        kcomp[lane * kXB + k] = 0.f;
    }
    // Nearest-pixel modes add each view's product one view late: the pixel
    // loads of view t are still in flight while view t+1's coordinates are
    // computed (the same additions in the same order as without the delay).
    float pvp[kXB], wp[kXB];
#pragma unroll
    for (int k = 0; k < kXB; ++k) pvp[k] = wp[k] = 0.f;

    // Fast modes: voxel-views the branch-free pass cannot finish (near-tie
    // pixel choices, the detector-edge taper band; ~0.1-1 % of them) are not
    // finished by their own lane -- that would stall the other 31 lanes of
    // the warp -- but queued per warp as (view, voxel, lane) and finished 32
    // at a time, every lane on a different item, whenever 32 are queued and
    // at the end of each view chunk. Their contributions are added to the
    // voxels' totals in shared memory (ksum, shared-memory atomics).
    uint16_t *q = sm.q[EXACT ? 0 : warp];
    int qn = 0;

    const float offx = 1.f / (float)P.ssx, offy = 1.f / (float)P.ssy, offz = 1.f / (float)P.ssz;
    const bool needZ = P.pL != 0 || P.pV != 0 || (RAYCAST && P.preset != 0);
    const int n_sub = P.ssx * P.ssy * P.ssz;
    for (int isub = 0; isub < n_sub; ++isub) {
        const int si = isub / (P.ssy * P.ssz), sj = (isub / P.ssz) % P.ssy, sk = isub % P.ssz;
        {
            {
                const float fsub[3] = {-0.5f + offx * (0.5f + si), -0.5f + offy * (0.5f + sj),
                                       -0.5f + offz * (0.5f + sk)};
                const float X0 = base[0] + fsub[0] * vw, Y0 = base[1] + fsub[1] * vw, Z0 = base[2] + fsub[2] * vw;

                // Finish the first c queued items (lane j takes item j) with the
                // full rule, then drop them from the queue. Warp-uniform call.
                auto flush = [&](int c, uint32_t v0) {
                    if (lane < c) {
                        const unsigned e = q[lane];
                        const int L = (int)(e & 31u), k = (int)((e >> 5) & (kXB - 1u)), tt = (int)(e >> (5 + kKB));
                        // the owner's voxel (same formulas as its own pass)
                        int id[3];
                        vox_id(L, 0, id);
                        float bb[3];
#pragma unroll
                        for (int a = 0; a < 3; ++a) bb[a] = ((float)id[a] + 0.5f - 0.5f * (float)P.n[a]) * vw;
                        const float X = bb[0] + fsub[0] * vw, Y = bb[1] + fsub[1] * vw, Z = bb[2] + fsub[2] * vw;
                        const ab_bpview bq = sv[tt];
                        const float *pvq = P.projs + (int64_t)(v0 + tt) * P.stride_view;
                        const float kf = (float)k;
                        const float vws = vw * (float)kStride;
                        const float D = fmaf(kf, (a2 == 0 ? bq.den.x : (a2 == 1 ? bq.den.y : bq.den.z)) * vws,
                                             dot4(bq.den, X, Y, Z));
                        const float rD = rcp_fast(D);
                        const float fu = fmaf(kf, (a2 == 0 ? bq.nu.x : (a2 == 1 ? bq.nu.y : bq.nu.z)) * vws,
                                              dot4(bq.nu, X, Y, Z)) * rD;
                        const float fv = fmaf(kf, (a2 == 0 ? bq.nv.x : (a2 == 1 ? bq.nv.y : bq.nv.z)) * vws,
                                              dot4(bq.nv, X, Y, Z)) * rD;
                        float w = RAYCAST ? 1.f : rD * rD;
                        if (needZ) {
                            const float Zk = fmaf(kf, (a2 == 0 ? bq.zl.x : (a2 == 1 ? bq.zl.y : bq.zl.z)) * vws,
                                                  dot4(bq.zl, X, Y, Z));
                            w *= zpow(P, bq, Zk);
                            if (RAYCAST && P.preset != 0)
                                w *= preset_weight(P.preset, P.val, X + (a2 == 0 ? kf * vw : 0.f) + P.c0[0],
                                                   Y + P.c0[1], bq.sxw, bq.syw, Zk);
                        }
                        float pv;
                        if (BILIN) {
                            pv = fetch_bilinear(P, pvq, fu, fv);
                        } else {
                            float du, dv;
                            int iu = round_index(fu, -2.f, P.fnu1, du);
                            int iv = round_index(fv, -2.f, P.fnv1, dv);
                            const bool tu = fabsf(du) > bq.tie_u, tv = fabsf(dv) > bq.tie_v;
                            if (tu || tv) {
                                vox_id(L, k, id);
                                const VoxRef vr{((double)id[0] + 0.5 + (double)fsub[0] - 0.5 * P.n[0]) * P.vwd,
                                                ((double)id[1] + 0.5 + (double)fsub[1] - 0.5 * P.n[1]) * P.vwd,
                                                ((double)id[2] + 0.5 + (double)fsub[2] - 0.5 * P.n[2]) * P.vwd};
                                const ab_bpview_d &cd = svd[kNear ? tt : 0];
                                if (tu) iu = refine_index(cd.nu, cd.den, vr, iu, du);
                                if (tv) iv = refine_index(cd.nv, cd.den, vr, iv, dv);
                            }
                            const bool inb = (unsigned)iu < P.nu && (unsigned)iv < P.nv;
                            pv = inb ? __ldg(pvq + (iu * P.su + iv * P.sv)) : 0.f;
                        }
                        float s = pv * w;
                        if (P.sep > 0.f && s != 0.f) s *= taper(bq, fu, fv, P.inv_sep);
                        atomicAdd(&ksum[L * kXB + k], s);
                    }
                    __syncwarp();
                    const int rem = qn - c;
                    for (int i0q = 0; i0q < rem; i0q += 32) {
                        const int i = i0q + lane;
                        const uint16_t v = i < rem ? q[i + c] : (uint16_t)0;
                        __syncwarp();
                        if (i < rem) q[i] = v;
                        __syncwarp();
                    }
                    qn = rem;
                };

                for (uint32_t v0 = 0; v0 < P.n_views; v0 += kChunk) {
                    const int cn = (int)min((uint32_t)kChunk, P.n_views - v0);
                    __syncthreads();
                    for (int t = threadIdx.x; t < cn; t += kThreads) {
                        // Volume centre in FP64 (exact: corner and voxwid are floats, n an integer).
                        const ab_d3 c0d{P.cornerd[0] + 0.5 * P.vwd * P.n[0], P.cornerd[1] + 0.5 * P.vwd * P.n[1],
                                        P.cornerd[2] + 0.5 * P.vwd * P.n[2]};
                        const aprict_proj_spec sp = P.specs[v0 + t];
                        // every projected point lies within n/2 + 1 voxels of the centre
                        const double hext[3] = {(0.5 * P.n[0] + 1.0) * P.vwd, (0.5 * P.n[1] + 1.0) * P.vwd,
                                                (0.5 * P.n[2] + 1.0) * P.vwd};
                        if (!ab_derive_bpview(sp, c0d, vw, P.sep, hext, sv[t], kNear ? &svd[t] : nullptr) && P.status)
                            atomicOr(P.status, APRICT_STATUS_BAD_GEOMETRY);
                        if (EXACT) ab_derive_bpview_exact(sp, c0d, sx[t]);
                        const ab_bpview &bt = sv[t];
                        if (kSkip) sm.off_det[t] = brick_off_detector(bt, sm.box, sm.box + 3, BILIN ? 0.5f : 0.f);
                        if (kInt)
                            sm.inner[t] = (uint8_t)(P.wide && bt.tie_u >= 0.25f && bt.tie_v >= 0.25f &&
                                                    brick_in_flat_box(bt, sm.boxa, sm.boxa + 3, BILIN ? 0.5f : 0.f));
                        const float vws = vw * (float)kStride;
                        sm.sd[t] = make_float4((a2 == 0 ? bt.nu.x : (a2 == 1 ? bt.nu.y : bt.nu.z)) * vws,
                                               (a2 == 0 ? bt.nv.x : (a2 == 1 ? bt.nv.y : bt.nv.z)) * vws,
                                               (a2 == 0 ? bt.den.x : (a2 == 1 ? bt.den.y : bt.den.z)) * vws,
                                               (a2 == 0 ? bt.zl.x : (a2 == 1 ? bt.zl.y : bt.zl.z)) * vws);
                        // exact zeros in the z coefficients, FP32 and FP64 alike (ORD 3 only)
                        if constexpr (EXACT)  // and the detector's v axis has no x-y component
                            sm.zinv[t] = (uint8_t)(kZ && bt.den.z == 0.f && bt.nu.z == 0.f &&
                                                   (!needZ || bt.zl.z == 0.f) && sx[t].v.x == 0.f &&
                                                   sx[t].v.y == 0.f);
                        else
                            sm.zinv[t] = (uint8_t)(kZ && kNear && bt.den.z == 0.f && bt.nu.z == 0.f &&
                                                   (!needZ || bt.zl.z == 0.f) && svd[t].nu[2] == 0.0 &&
                                                   svd[t].den[2] == 0.0);
                        // A fan-beam slice: the v form vanishes in the slice plane (its x, y
                        // and constant coefficients are exact zeros), and with one z layer
                        // and no z sub-samples every sample lies in that plane (z = 0
                        // relative to the volume centre, exactly): every voxel projects
                        // onto row 0 of the one-row detector exactly.
                        if constexpr (ORD == 2)
                            sm.vzero[t] = (uint8_t)(P.nv == 1u && P.n[2] == 1 && P.ssz == 1 && bt.nv.x == 0.f &&
                                                    bt.nv.y == 0.f && bt.nv.w == 0.f);
                    }
                    __syncthreads();
                    // The chunk's views whose projection of the brick reaches the
                    // detector, in view order (warp 0 compacts; the others read the list
                    // after the barrier). Views that miss it add only zeros.
                    if (kSkip && warp == 0) {
                        const unsigned lt = (1u << lane) - 1u;
                        int base_j = 0;
#pragma unroll
                        for (int g = 0; g < kChunk / 32; ++g) {
                            const int tv = g * 32 + lane;
                            const bool keep = tv < cn && !sm.off_det[tv];
                            const unsigned m = __ballot_sync(0xffffffffu, keep);
                            if (keep) sm.vlist[base_j + __popc(m & lt)] = (uint8_t)tv;
                            base_j += __popc(m);
                        }
                        if (lane == 0) sm.vcount = base_j;
                    }
                    if (kSkip) __syncthreads();
                    // warp-uniform skip (the fast modes' queue uses whole-warp votes)
                    if (!__any_sync(0xffffffffu, any_live)) continue;
                    const int n_list = kSkip ? sm.vcount : cn;
                    for (int j = 0; j < n_list; ++j) {
                        if constexpr (kZ && kNear && !RAYCAST) {
                            if ((j & 31) == 0) {
                                // The warp's table for views j .. j + 31: every lane of
                                // the warp has this x and y, so for a view whose depth and
                                // u coordinate do not change along z (zinv) everything
                                // that depends on u is warp-uniform -- the reciprocal
                                // depth, the weight, the u half of the pixel choice (FP64
                                // for a near tie), the u half of the edge taper and
                                // whether the column lies on the detector. Lane L settles
                                // view j + L once for the warp's 32 x XB voxels.
                                const int jj = j + lane;
                                const int tt = jj < n_list ? (kSkip ? (int)sm.vlist[jj] : jj) : 0;
                                if (jj < n_list && sm.zinv[tt]) {
                                    const ab_bpview bq = sv[tt];
                                    const float rDq = rcp_fast(dot4(bq.den, X0, Y0, Z0));
                                    const float fu = dot4(bq.nu, X0, Y0, Z0) * rDq;
                                    float w = rDq * rDq;
                                    if (needZ) w *= zpow(P, bq, dot4(bq.zl, X0, Y0, Z0));
                                    float du;
                                    int iu = round_index(fu, -2.f, P.fnu1, du);
                                    if (fabsf(du) > bq.tie_u) {
                                        const VoxRef vr{((double)b2 + 0.5 + (double)fsub[0] - 0.5 * P.n[0]) * P.vwd,
                                                        ((double)i1 + 0.5 + (double)fsub[1] - 0.5 * P.n[1]) * P.vwd,
                                                        0.0};
                                        iu = refine_index(svd[tt].nu, svd[tt].den, vr, iu, du);
                                    }
                                    float4 rec = make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
                                    if ((unsigned)iu < P.nu) {
                                        const float cu = fu - bq.cu0;
                                        if (P.sep > 0.f && fabsf(cu) > bq.tap_ru)
                                            w *= ab_edge_taper_half(fabsf(cu), bq.inv_halfu, P.inv_sep);
                                        // + 4 sv bits(tv) is then the byte address of row round(fv)
                                        const uint64_t col =
                                            (uint64_t)(uintptr_t)(P.projs + (int64_t)(v0 + tt) * P.stride_view +
                                                                  (int64_t)iu * P.su) -
                                            4ull * 0x4B400000ull * (uint64_t)(uint32_t)P.sv;
                                        rec = make_float4(rDq, w, __uint_as_float((uint32_t)col),
                                                          __uint_as_float((uint32_t)(col >> 32)));
                                    }
                                    sm.zrec[warp][lane] = rec;
                                }
                                __syncwarp();
                            }
                        }
                        const int t = kSkip ? (int)sm.vlist[j] : j;
                        const int view = (int)v0 + t;
                        const ab_bpview b = sv[t];
                        const float *pvw = P.projs + (int64_t)view * P.stride_view;
                        const float Nu0 = dot4(b.nu, X0, Y0, Z0), Nv0 = dot4(b.nv, X0, Y0, Z0);
                        const float D0 = dot4(b.den, X0, Y0, Z0);
                        const float4 steps = sm.sd[t];
                        const float dNu = steps.x, dNv = steps.y, dD = steps.z;
                        float Zb = 0.f, dZ = 0.f;
                        if (needZ) {
                            Zb = dot4(b.zl, X0, Y0, Z0);
                            dZ = steps.w;
                        }
                        if constexpr (EXACT) {
                            if (kZ && sm.zinv[t]) {
                                // Upright detector in the z-column layout: the thread's voxels
                                // share x and y, so the depth and u of the column's four
                                // vertical edges, the footprint's pixel columns and, per pixel
                                // column, the x-y slab of its rays (whose x and y do not depend
                                // on the row) are computed once per thread and view; per voxel
                                // only the v extent and, per pixel, the z slab remain, each by
                                // the per-voxel path's formulas.
                                const ab_bpview_exact e = sx[t];
                                const float h = 0.5f * vw;
                                const float hd0 = b.den.x * h, hd1 = b.den.y * h;
                                const float hu0 = b.nu.x * h, hu1 = b.nu.y * h;
                                const float hv0 = b.nv.x * h, hv1 = b.nv.y * h, hv2 = b.nv.z * h;
                                float rr[4], bv[4];
                                float umin = 3.0e38f, umax = -3.0e38f;
#pragma unroll
                                for (int c = 0; c < 4; ++c) {
                                    const float sx_ = (c & 2) ? 1.f : -1.f, sy_ = (c & 1) ? 1.f : -1.f;
                                    rr[c] = rcp_fast(D0 + sx_ * hd0 + sy_ * hd1);
                                    const float uu = (Nu0 + sx_ * hu0 + sy_ * hu1) * rr[c];
                                    umin = fminf(umin, uu);
                                    umax = fmaxf(umax, uu);
                                    bv[c] = sx_ * hv0 + sy_ * hv1;
                                }
                                const int ulo = max(0, (int)ceilf(umin - 1e-3f));
                                const int uhi = min((int)P.nu - 1, (int)floorf(umax + 1e-3f));
                                int vlo[kXB], vhi[kXB];
                                float sk[kXB], zlo[kXB], zhi[kXB];
#pragma unroll
                                for (int k = 0; k < kXB; ++k) {
                                    const float Nv = fmaf((float)k, dNv, Nv0);
                                    float vmin = 3.0e38f, vmax = -3.0e38f;
#pragma unroll
                                    for (int c = 0; c < 4; ++c) {
                                        const float v1 = (Nv + bv[c] - hv2) * rr[c], v2 = (Nv + bv[c] + hv2) * rr[c];
                                        vmin = fminf(vmin, fminf(v1, v2));
                                        vmax = fmaxf(vmax, fmaxf(v1, v2));
                                    }
                                    vlo[k] = live[k] ? max(0, (int)ceilf(vmin - 1e-3f)) : 1;
                                    vhi[k] = live[k] ? min((int)P.nv - 1, (int)floorf(vmax + 1e-3f)) : 0;
                                    // ray origin relative to the voxel's centre, z part: the slab's
                                    // bounds -h - r0z and h - r0z
                                    const float r0z = e.s.z - (Z0 + (float)k * vw * (float)kStride);
                                    zlo[k] = -h - r0z;
                                    zhi[k] = h - r0z;
                                    sk[k] = 0.f;
                                }
                                const float r0x = e.s.x - X0, r0y = e.s.y - Y0;
                                for (int iu = ulo; iu <= uhi; ++iu) {
                                    const float dx = fmaf(e.u.x, (float)iu, e.d0.x);
                                    const float dy = fmaf(e.u.y, (float)iu, e.d0.y);
                                    const float duz = fmaf(e.u.z, (float)iu, e.d0.z);
                                    float a_lo = 0.f, a_hi = 3.0e38f;
                                    bool miss = false;
                                    if (dx != 0.f) {
                                        const float inv = rcp_fast(dx);
                                        const float t1 = (-h - r0x) * inv, t2 = (h - r0x) * inv;
                                        a_lo = fmaxf(a_lo, fminf(t1, t2));
                                        a_hi = fminf(a_hi, fmaxf(t1, t2));
                                    } else {
                                        miss |= fabsf(r0x) > h;
                                    }
                                    if (dy != 0.f) {
                                        const float inv = rcp_fast(dy);
                                        const float t1 = (-h - r0y) * inv, t2 = (h - r0y) * inv;
                                        a_lo = fmaxf(a_lo, fminf(t1, t2));
                                        a_hi = fminf(a_hi, fmaxf(t1, t2));
                                    } else {
                                        miss |= fabsf(r0y) > h;
                                    }
                                    if (miss || !(a_hi > a_lo)) continue;  // the column's rays miss the voxels
                                    const float dxy2 = dx * dx + dy * dy;
                                    const float *pcol = pvw + iu * P.su;
#pragma unroll
                                    for (int k = 0; k < kXB; ++k) {
                                        for (int iv = vlo[k]; iv <= vhi[k]; ++iv) {
                                            const float dz = fmaf(e.v.z, (float)iv, duz);
                                            float lo = a_lo, hi = a_hi;
                                            if (dz != 0.f) {
                                                const float inv = rcp_fast(dz);
                                                const float t1 = zlo[k] * inv, t2 = zhi[k] * inv;
                                                lo = fmaxf(lo, fminf(t1, t2));
                                                hi = fminf(hi, fmaxf(t1, t2));
                                            } else if (zlo[k] > 0.f || zhi[k] < 0.f) {
                                                continue;  // |r0z| > h
                                            }
                                            if (!(hi > lo)) continue;
                                            const float chord = (hi - lo) * sqrt_fast(dxy2 + dz * dz);
                                            const float pv = P.all_ones ? 1.f : __ldg(pcol + iv * P.sv);
                                            sk[k] = fmaf(pv, chord, sk[k]);
                                        }
                                    }
                                }
                                const float rD = rcp_fast(D0);
                                const float fu = Nu0 * rD;
#pragma unroll
                                for (int k = 0; k < kXB; ++k) {
                                    if (!live[k]) continue;
                                    float s = sk[k];
                                    if (needZ) s *= zpow(P, b, fmaf((float)k, dZ, Zb));
                                    const float fv = fmaf((float)k, dNv, Nv0) * rD;
                                    if (P.sep > 0.f && s != 0.f) s *= taper(b, fu, fv, P.inv_sep);
                                    acc[k] += s;
                                }
                            } else {
#pragma unroll
                            for (int k = 0; k < kXB; ++k) {
                                if (!live[k]) continue;
                                const float kf = (float)k;
                                const float D = fmaf(kf, dD, D0);
                                const float rD = rcp_fast(D);
                                const float fu = fmaf(kf, dNu, Nu0) * rD;
                                const float fv = fmaf(kf, dNv, Nv0) * rD;
                                float s;
                                {
                                    // Footprint: bounding box of the 8 projected corners.
                                    const ab_bpview_exact e = sx[t];
                                    const float h = 0.5f * vw;
                                    const float hu[3] = {b.nu.x * h, b.nu.y * h, b.nu.z * h};
                                    const float hv[3] = {b.nv.x * h, b.nv.y * h, b.nv.z * h};
                                    const float hd[3] = {b.den.x * h, b.den.y * h, b.den.z * h};
                                    const float Nu = fmaf(kf, dNu, Nu0), Nv = fmaf(kf, dNv, Nv0);
                                    float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f;
#pragma unroll
                                    for (int c = 0; c < 8; ++c) {
                                        const float sx_ = (c & 4) ? 1.f : -1.f, sy_ = (c & 2) ? 1.f : -1.f,
                                                    sz_ = (c & 1) ? 1.f : -1.f;
                                        const float dd = D + sx_ * hd[0] + sy_ * hd[1] + sz_ * hd[2];
                                        const float rr = rcp_fast(dd);
                                        const float uu = (Nu + sx_ * hu[0] + sy_ * hu[1] + sz_ * hu[2]) * rr;
                                        const float vv = (Nv + sx_ * hv[0] + sy_ * hv[1] + sz_ * hv[2]) * rr;
                                        umin = fminf(umin, uu);
                                        umax = fmaxf(umax, uu);
                                        vmin = fminf(vmin, vv);
                                        vmax = fmaxf(vmax, vv);
                                    }
                                    const int ulo = max(0, (int)ceilf(umin - 1e-3f));
                                    const int uhi = min((int)P.nu - 1, (int)floorf(umax + 1e-3f));
                                    const int vlo = max(0, (int)ceilf(vmin - 1e-3f));
                                    const int vhi = min((int)P.nv - 1, (int)floorf(vmax + 1e-3f));
                                    // Ray origin relative to this voxel's centre.
                                    float cx[3] = {X0, Y0, Z0};
                                    cx[a2] += kf * vw * (float)kStride;
                                    const float r0x = e.s.x - cx[0], r0y = e.s.y - cx[1], r0z = e.s.z - cx[2];
                                    s = 0.f;
                                    for (int iu = ulo; iu <= uhi; ++iu) {
                                        const float dux = fmaf(e.u.x, (float)iu, e.d0.x);
                                        const float duy = fmaf(e.u.y, (float)iu, e.d0.y);
                                        const float duz = fmaf(e.u.z, (float)iu, e.d0.z);
                                        for (int iv = vlo; iv <= vhi; ++iv) {
                                            const float dx = fmaf(e.v.x, (float)iv, dux);
                                            const float dy = fmaf(e.v.y, (float)iv, duy);
                                            const float dz = fmaf(e.v.z, (float)iv, duz);
                                            float a_lo = 0.f, a_hi = 3.0e38f;
                                            bool miss = false;
                                            if (dx != 0.f) {
                                                const float inv = rcp_fast(dx);
                                                const float t1 = (-h - r0x) * inv, t2 = (h - r0x) * inv;
                                                a_lo = fmaxf(a_lo, fminf(t1, t2));
                                                a_hi = fminf(a_hi, fmaxf(t1, t2));
                                            } else {
                                                miss |= fabsf(r0x) > h;
                                            }
                                            if (dy != 0.f) {
                                                const float inv = rcp_fast(dy);
                                                const float t1 = (-h - r0y) * inv, t2 = (h - r0y) * inv;
                                                a_lo = fmaxf(a_lo, fminf(t1, t2));
                                                a_hi = fminf(a_hi, fmaxf(t1, t2));
                                            } else {
                                                miss |= fabsf(r0y) > h;
                                            }
                                            if (dz != 0.f) {
                                                const float inv = rcp_fast(dz);
                                                const float t1 = (-h - r0z) * inv, t2 = (h - r0z) * inv;
                                                a_lo = fmaxf(a_lo, fminf(t1, t2));
                                                a_hi = fminf(a_hi, fmaxf(t1, t2));
                                            } else {
                                                miss |= fabsf(r0z) > h;
                                            }
                                            if (miss || !(a_hi > a_lo)) continue;
                                            const float chord = (a_hi - a_lo) * sqrt_fast(dx * dx + dy * dy + dz * dz);
                                            const float pv = P.all_ones ? 1.f : __ldg(pvw + (iu * P.su + iv * P.sv));
                                            s = fmaf(pv, chord, s);
                                        }
                                    }
                                    if (needZ) s *= zpow(P, b, fmaf(kf, dZ, Zb));
                                }
                                if (P.sep > 0.f && s != 0.f) s *= taper(b, fu, fv, P.inv_sep);
                                acc[k] += s;
                            }
                            }
                        } else {
                            // Fast modes: one branch-free pass over the thread's voxels;
                            // voxel-views that need more (a near-tie pixel choice, the
                            // detector-edge taper band) are flagged and finished in a rare
                            // second pass, so the common path has no divergent branches.
                            unsigned pending = 0;
                            // ORD 3 on a view whose depth, u coordinate and distance along
                            // the axis do not change along z (exact zeros in the per-view
                            // steps; warp-uniform): the thread's voxels share rD, fu, the
                            // weight and the u half of the pixel choice, computed once.
                            const bool zinv = kZ && kNear && !RAYCAST && sm.zinv[t];
                            if (zinv) {
                                // the warp-uniform part from the warp's table (filled above)
                                const float4 rec = sm.zrec[warp][j & 31];
                                const float rD = rec.x;
                                if (rD == rD) {  // else the column is off the detector: zeros
                                    const float w = rec.y;
                                    const uint64_t col = ((uint64_t)__float_as_uint(rec.w) << 32) | __float_as_uint(rec.z);
                                    const uint32_t sv4 = 4u * (uint32_t)P.sv;
                                    // Interior column: fv is monotone in k, so when the first and
                                    // last voxel of every lane lie in the flat box, all of the
                                    // warp's rows are on the detector with taper weight 1 and only
                                    // a near-tie row choice remains. That pass has no predicates:
                                    // it loads every voxel's FP32-rounded pixel (live or not; dead
                                    // voxels are never written) and turns the tie test into an
                                    // FMA-pipe value slow = 0 or 1 that zeroes the weight and sets
                                    // the voxel's bit of the fix-up mask.
                                    const float fvf = fmaf(0.f, dNv, Nv0) * rD;
                                    const float fvl = fmaf((float)(kXB - 1), dNv, Nv0) * rD;
                                    const bool inbox = fabsf(fvf - b.cv0) <= b.tap_rv && fabsf(fvl - b.cv0) <= b.tap_rv;
                                    if (__all_sync(0xffffffffu, inbox) && b.tie_v >= 0.25f) {
                                        // |dv| and tie_v lie in [0, 1/2] and tie_v >= 1/4: |dv| > tie_v
                                        // means |dv| - tie_v >= 2^-25, so 2^40 (|dv| - tie_v)
                                        // saturates to exactly 1, and to 0 otherwise
                                        const float ntie = -b.tie_v * 0x1p40f;
                                        float pendf = 0.f;
#pragma unroll
                                        for (int k = 0; k < kXB; ++k) {
                                            const float fv = fmaf((float)k, dNv, Nv0) * rD;
                                            const float tv = __fadd_rn(fv, kMagic);
                                            const float dv = __fsub_rn(fv, __fsub_rn(tv, kMagic));
                                            const float slow = __saturatef(fmaf(fabsf(dv), 0x1p40f, ntie));
                                            const float pv = __ldg(reinterpret_cast<const float *>(
                                                col + (uint64_t)(uint32_t)__float_as_int(tv) * sv4));
                                            acc[k] = fmaf(pvp[k], wp[k], acc[k]);
                                            pvp[k] = pv;
                                            wp[k] = fmaf(-slow, w, w);
                                            pendf = fmaf(slow, (float)(1u << k), pendf);
                                        }
                                        pending = (unsigned)pendf;
                                    } else {
#pragma unroll
                                    for (int k = 0; k < kXB; ++k) {
                                        const float fv = fmaf((float)k, dNv, Nv0) * rD;
                                        const float av = fabsf(fv - b.cv0);
                                        const bool outside = kSkip && av > b.out_rv;
                                        const float tv = __fadd_rn(fv, kMagic);
                                        const float dv = __fsub_rn(fv, __fsub_rn(tv, kMagic));
                                        const bool fast = av <= b.tap_rv && fabsf(dv) <= b.tie_v;
                                        float pv = 0.f;
                                        if (live[k] && fast)
                                            pv = __ldg(reinterpret_cast<const float *>(
                                                col + (uint64_t)(uint32_t)__float_as_int(tv) * sv4));
                                        acc[k] = fmaf(pvp[k], wp[k], acc[k]);
                                        pvp[k] = pv;
                                        wp[k] = w;
                                        pending |= (live[k] && !fast && !outside) ? 1u << k : 0u;
                                    }
                                    }
                                }
                            } else if (ORD == 2 && !BILIN && sm.vzero[t]) {
                                // Fan-beam slice: one detector row and a v form that is zero
                                // at every point, so every voxel projects onto row 0 exactly
                                // (v = 0 = the row centre, no tie, inside the flat box in v);
                                // only u is computed, by the same steps as the general loop.
                                const uint32_t offu0 = 0u - 0x4B400000u * (uint32_t)P.su;
#pragma unroll
                                for (int k = 0; k < kXB; ++k) {
                                    const float kf = (float)k;
                                    const float D = fmaf(kf, dD, D0);
                                    const float rD = rcp_fast(D);
                                    const float fu = fmaf(kf, dNu, Nu0) * rD;
                                    float w = RAYCAST ? 1.f : rD * rD;
                                    if (needZ) {
                                        const float Zk = fmaf(kf, dZ, Zb);
                                        w *= zpow(P, b, Zk);
                                        if (RAYCAST && P.preset != 0)
                                            w *= preset_weight(P.preset, P.val, X0 + (a2 == 0 ? kf * vw : 0.f) + P.c0[0],
                                                               Y0 + P.c0[1], b.sxw, b.syw, Zk);
                                    }
                                    const float au = fabsf(fu - b.cu0);
                                    const bool outside = kSkip && au > b.out_ru;
                                    const float tu = __fadd_rn(fu, kMagic);
                                    const float du = __fsub_rn(fu, __fsub_rn(tu, kMagic));
                                    const bool fast = au <= b.tap_ru && fabsf(du) <= b.tie_u;
                                    const int off = (int)((uint32_t)__float_as_int(tu) * (uint32_t)P.su + offu0);
                                    float pv = 0.f;
                                    if (live[k] && fast) pv = __ldg(pvw + off);
                                    acc[k] = fmaf(pvp[k], wp[k], acc[k]);
                                    pvp[k] = pv;
                                    wp[k] = w;
                                    pending |= (live[k] && !fast && !outside) ? 1u << k : 0u;
                                }
                            } else if (kInt && BILIN && sm.inner[t]) {
                                // Interior brick, bilinear: every voxel's four taps are on the
                                // detector with taper weight 1 (the flat box less 1/2 pixel), so
                                // they are loaded without bounds checks and nothing is deferred;
                                // the interpolation is fetch_bilinear's, in the same order.
                                const uint64_t vb = (uint64_t)(uintptr_t)pvw;
                                const uint32_t su4 = 4u * (uint32_t)P.su, sv4 = 4u * (uint32_t)P.sv;
#pragma unroll
                                for (int k = 0; k < kXB; ++k) {
                                    const float kf = (float)k;
                                    const float D = fmaf(kf, dD, D0);
                                    const float rD = rcp_fast(D);
                                    const float fu = fmaf(kf, dNu, Nu0) * rD;
                                    const float fv = fmaf(kf, dNv, Nv0) * rD;
                                    float w = RAYCAST ? 1.f : rD * rD;
                                    if (needZ) {
                                        const float Zk = fmaf(kf, dZ, Zb);
                                        w *= zpow(P, b, Zk);
                                        if (RAYCAST && P.preset != 0)
                                            w *= preset_weight(P.preset, P.val, X0 + (a2 == 0 ? kf * vw : 0.f) + P.c0[0],
                                                               Y0 + P.c0[1], b.sxw, b.syw, Zk);
                                    }
                                    const float flu = floorf(fu), flv = floorf(fv);
                                    const float fx = fu - flu, fy = fv - flv;
                                    const float *p00 = reinterpret_cast<const float *>(
                                        vb + (uint64_t)(uint32_t)(int)flu * su4 + (uint64_t)(uint32_t)(int)flv * sv4);
                                    const float *p10 = reinterpret_cast<const float *>(reinterpret_cast<uintptr_t>(p00) + su4);
                                    const float v00 = __ldg(p00), v01 = __ldg(reinterpret_cast<const float *>(
                                                                      reinterpret_cast<uintptr_t>(p00) + sv4));
                                    const float v10 = __ldg(p10), v11 = __ldg(reinterpret_cast<const float *>(
                                                                      reinterpret_cast<uintptr_t>(p10) + sv4));
                                    const float t1 = v00 * (1.f - fx) + v10 * fx;
                                    const float t2 = v01 * (1.f - fx) + v11 * fx;
                                    acc[k] = fmaf(t1 * (1.f - fy) + t2 * fy, w, acc[k]);
                                }
                            } else if (kInt && !BILIN && sm.inner[t]) {
                                // Interior brick: every voxel's pixel is on the detector with
                                // taper weight 1, so the pass has no predicates; it loads every
                                // voxel's FP32-rounded pixel (dead voxels are never written) and
                                // turns the u and v near-tie tests into an FMA-pipe value slow =
                                // 0 or 1 (as in the z-column interior columns) that zeroes the
                                // weight and sets the voxel's bit of the fix-up mask. Byte
                                // addresses: two 32 x 32 -> 64-bit multiply-adds of the rounded
                                // indices' bit patterns onto the view's base less the magic bias.
                                const float ntu = -b.tie_u * 0x1p40f, ntv = -b.tie_v * 0x1p40f;
                                const uint64_t vb = (uint64_t)(uintptr_t)pvw -
                                                    4ull * 0x4B400000ull *
                                                        ((uint64_t)(uint32_t)P.su + (uint64_t)(uint32_t)P.sv);
                                const uint32_t su4 = 4u * (uint32_t)P.su, sv4 = 4u * (uint32_t)P.sv;
                                float pendf = 0.f;
#pragma unroll
                                for (int k = 0; k < kXB; ++k) {
                                    const float kf = (float)k;
                                    const float D = fmaf(kf, dD, D0);
                                    const float rD = rcp_fast(D);
                                    const float fu = fmaf(kf, dNu, Nu0) * rD;
                                    const float fv = fmaf(kf, dNv, Nv0) * rD;
                                    float w = RAYCAST ? 1.f : rD * rD;
                                    if (needZ) {
                                        const float Zk = fmaf(kf, dZ, Zb);
                                        w *= zpow(P, b, Zk);
                                        if (RAYCAST && P.preset != 0)
                                            w *= preset_weight(P.preset, P.val, X0 + (a2 == 0 ? kf * vw : 0.f) + P.c0[0],
                                                               Y0 + P.c0[1], b.sxw, b.syw, Zk);
                                    }
                                    const float tu = __fadd_rn(fu, kMagic), tv = __fadd_rn(fv, kMagic);
                                    const float du = __fsub_rn(fu, __fsub_rn(tu, kMagic));
                                    const float dv = __fsub_rn(fv, __fsub_rn(tv, kMagic));
                                    const float slow = __saturatef(__saturatef(fmaf(fabsf(du), 0x1p40f, ntu)) +
                                                                   __saturatef(fmaf(fabsf(dv), 0x1p40f, ntv)));
                                    const float pv = __ldg(reinterpret_cast<const float *>(
                                        vb + (uint64_t)(uint32_t)__float_as_int(tu) * su4 +
                                        (uint64_t)(uint32_t)__float_as_int(tv) * sv4));
                                    acc[k] = fmaf(pvp[k], wp[k], acc[k]);
                                    pvp[k] = pv;
                                    wp[k] = fmaf(-slow, w, w);
                                    pendf = fmaf(slow, (float)(1u << k), pendf);
                                }
                                pending = (unsigned)pendf;
                            } else {
#pragma unroll
                            for (int k = 0; k < kXB; ++k) {
                                const float kf = (float)k;
                                const float D = fmaf(kf, dD, D0);
                                const float rD = rcp_fast(D);
                                const float fu = fmaf(kf, dNu, Nu0) * rD;
                                const float fv = fmaf(kf, dNv, Nv0) * rD;
                                float w = RAYCAST ? 1.f : rD * rD;
                                if (needZ) {
                                    const float Zk = fmaf(kf, dZ, Zb);
                                    w *= zpow(P, b, Zk);
                                    if (RAYCAST && P.preset != 0)
                                        w *= preset_weight(P.preset, P.val, X0 + (a2 == 0 ? kf * vw : 0.f) + P.c0[0],
                                                           Y0 + P.c0[1], b.sxw, b.syw, Zk);
                                }
                                // inner: inside the taper's flat box, which lies inside the
                                // detector (|f - c| <= n/2 without a taper); outside: certainly
                                // off the detector (contributes 0: neither loaded nor queued)
                                const float au = fabsf(fu - b.cu0), av = fabsf(fv - b.cv0);
                                const bool inner = au <= b.tap_ru && av <= b.tap_rv;
                                const bool outside = kSkip && (au > b.out_ru + (BILIN ? 0.5f : 0.f) ||
                                                               av > b.out_rv + (BILIN ? 0.5f : 0.f));
                                float pv = 0.f;
                                bool fast;
                                if (BILIN) {
                                    fast = inner;
                                    pv = fetch_bilinear(P, pvw, fu, fv);
                                    pv = live[k] && fast ? pv : 0.f;
                                } else {
                                    // Inside the detector box |f| < 2^22, so the rounding trick
                                    // needs no clamp; a pixel at most 1/2 - refine from f is
                                    // then a valid index (the box edges are half-integers).
                                    const float tu = __fadd_rn(fu, kMagic), tv = __fadd_rn(fv, kMagic);
                                    const float du = __fsub_rn(fu, __fsub_rn(tu, kMagic));
                                    const float dv = __fsub_rn(fv, __fsub_rn(tv, kMagic));
                                    fast = inner && fabsf(du) <= b.tie_u && fabsf(dv) <= b.tie_v;
                                    // pixel offset from the rounded indices (bits - magic)
                                    // (bits(tu) - 0x4B400000) su + (bits(tv) - 0x4B400000) sv, in
                                    // wrapping unsigned arithmetic (the in-view offset fits 31 bits)
                                    const int off = (int)((uint32_t)__float_as_int(tu) * (uint32_t)P.su +
                                                          ((uint32_t)__float_as_int(tv) * (uint32_t)P.sv + P.koff));
                                    if (live[k] && fast) pv = __ldg(pvw + off);
                                }
                                if (BILIN) {
                                    acc[k] = fmaf(pv, w, acc[k]);
                                } else {
                                    acc[k] = fmaf(pvp[k], wp[k], acc[k]);
                                    pvp[k] = pv;
                                    wp[k] = w;
                                }
                                pending |= (live[k] && !fast && !outside) ? 1u << k : 0u;
                            }
                            }
                            if (__any_sync(0xffffffffu, pending != 0u)) {
                                // each lane's deferred voxel-views go to consecutive queue
                                // slots after those of the lower lanes (warp prefix sum)
                                const int cnt = __popc(pending);
                                int incl = cnt;
#pragma unroll
                                for (int o = 1; o < 32; o <<= 1) {
                                    const int y = __shfl_up_sync(0xffffffffu, incl, o);
                                    if (lane >= o) incl += y;
                                }
                                int pos = qn + incl - cnt;
                                for (unsigned pm = pending; pm != 0u; pm &= pm - 1u) {
                                    const int k = __ffs(pm) - 1;
                                    q[pos++] = (uint16_t)((t << (5 + kKB)) | (k << 5) | lane);
                                }
                                qn += __shfl_sync(0xffffffffu, incl, 31);
                                __syncwarp();
                                while (qn >= 32) flush(32, v0);
                            }
                        }
                    }
                    // the queue refers to this chunk's coefficients: finish it now
                    if constexpr (!EXACT) {
                        if (qn > 0) flush(qn, v0);
                    }
                    // the chunk's partial sums into the compensated totals; the
                    // delayed product of the chunk's last view is folded in first, so a
                    // partial holds exactly its own views' products whichever views a
                    // kernel skips (the batch kernel skips views off the detector)
#pragma unroll
                    for (int k = 0; k < kXB; ++k) {
                        if constexpr (!EXACT && !BILIN) {
                            acc[k] = fmaf(pvp[k], wp[k], acc[k]);
                            pvp[k] = 0.f;
                        }
                        const int i = lane * kXB + k;
                        const float sk = ksum[i];
                        const float y = acc[k] - kcomp[i];
                        const float tk = sk + y;
                        kcomp[i] = (tk - sk) - y;
                        ksum[i] = tk;
                        acc[k] = 0.f;
                    }
                }
            }
        }
    }

    if constexpr (!EXACT && !BILIN) {  // the last view's delayed products
#pragma unroll
        for (int k = 0; k < kXB; ++k) acc[k] = fmaf(pvp[k], wp[k], acc[k]);
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < kXB; ++k) acc[k] = ksum[lane * kXB + k] + (acc[k] - kcomp[lane * kXB + k]);

#pragma unroll
    for (int k = 0; k < kXB; ++k) {
        if (!live[k]) continue;
        const float value = n_sub == 1 ? acc[k] : acc[k] / (float)n_sub;
        if (value == 0.f) continue;  // the reference skips the write (:1010)
        int id[3];
        vox_id(lane, k, id);
        const int64_t o = (int64_t)id[0] * P.vs[0] + (int64_t)id[1] * P.vs[1] + (int64_t)id[2] * P.vs[2];
        const float m = P.mult ? __ldcs(P.mult + o) : 1.f;
        __stcs(P.vol + o, value * m + __ldcs(P.vol + o));
    }
}

// Host: the kernel's axis assignment for a volume (see bp_brick): 0 C order,
// 1 F order, 2 C order with one z layer (slice stacks of fan-beam scans),
// where lanes run along y instead of the single z layer.
inline int bp_ord(const aprict_vol_desc *vd) { return vd->order == 0 ? (vd->nz == 1 && vd->ny > 1 ? 2 : 0) : 1; }

// Host: whether ORD 3 (lanes and a thread's voxels along z) applies: the
// fast nearest mode, or the exact mode where exact_ok (one-scan calls), on a
// C-order volume tall enough to fill the 32 XB voxels of a thread column,
// unless tuning knob 7 is 1, with a v stride below 2^30 elements (the gathers
// form their byte address as a 32 x 32-bit product). Measured on a 256^3
// volume with 360 views: nearest 9.82 -> 8.68 ms; on 128^3 with 180 views,
// exact 10.0 -> 7.1 ms (the column's x-y quantities shared); bilinear (27.4 vs
// 28.1 ms) keeps ORD 0.
inline bool bp_zlanes_ok(const aprict_vol_desc *vd, const aprict_proj_desc *pd, int xb,
                         const aprict_backproject_config *cfg, bool exact_ok = false) {
    return bp_ord(vd) == 0 && ab_tuning_get(AB_TUNE_BP_ZLANES) != 1 && vd->nz >= 32u * (uint32_t)xb &&
           pd->stride_v < (int64_t)1 << 30 && (!cfg->exact || exact_ok) && !cfg->approx_mode_direct_raycast &&
           !cfg->approx_mode_linear_interpolate;
}

// Host: validate one backprojection call and fill its parameters; units is
// the number of work units (bricks, 0 when empty), xb the voxels per thread
// (force_xb 2, 4 or 8, or 0 for the tuning knob's choice). With ord_out the
// caller accepts ORD 3 where bp_zlanes_ok holds and learns the layout chosen;
// without it the layout is bp_ord's.
inline int make_bp_params(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd, const float *projs_dev,
                          const aprict_vol_desc *vd, float *vol_dev, const float *multiplier_dev,
                          const aprict_backproject_config *cfg, uint32_t *status_dev, BPParams &P,
                          uint64_t &units, int &xb, int force_xb = 0, int *ord_out = nullptr) {
    units = 0;
    int rc;
    if ((rc = ab_check_projs(pd, projs_dev, "projections")) != APRICT_OK) return rc;
    if ((rc = ab_check_vol(vd, vol_dev, "volume")) != APRICT_OK) return rc;
    if (cfg == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null backproject config");
    if (cfg->apply_summand_multiplier != (multiplier_dev != nullptr ? 1u : 0u))
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT,
                       "apply_summand_multiplier must be set if and only if a multiplier is given");
    if (cfg->weighting_preset > 6)
        return ab_fail(APRICT_ERR_UNSUPPORTED,
                       "backprojection weighting preset %u: presets 0-6 here, 7 (GBC) through "
                       "aprict_b200_backproject_gbc",
                       cfg->weighting_preset);
    if (cfg->ssx == 0 || cfg->ssy == 0 || cfg->ssz == 0 || cfg->ssx > 16 || cfg->ssy > 16 || cfg->ssz > 16)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ssx/ssy/ssz must be in [1, 16]");
    if (cfg->Z_on_val_factor_power != 0 && !(cfg->Z_on_val_factor_val != 0.f))
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "Z_on_val_factor_val must be nonzero");
    if (pd->n_views == 0 || pd->nu == 0 || pd->nv == 0) return APRICT_OK;
    if (specs_dev == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null view specs");
    if (multiplier_dev && (reinterpret_cast<uintptr_t>(multiplier_dev) & 3u))
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "multiplier pointer not 4-byte aligned");
    if (pd->nu > (1u << 21) || pd->nv > (1u << 21))
        return ab_fail(APRICT_ERR_TOO_LARGE, "backprojection supports at most 2^21 detector pixels per axis");
    if ((int64_t)(pd->nu - 1) * pd->stride_u + (int64_t)(pd->nv - 1) * pd->stride_v + 1 > 0x7fffffffLL)
        return ab_fail(APRICT_ERR_TOO_LARGE, "one projection image spans more than 2^31 elements");

    P = BPParams{};
    P.specs = specs_dev;
    P.n_views = pd->n_views;
    P.nu = pd->nu;
    P.nv = pd->nv;
    P.stride_view = pd->stride_view;
    P.su = (int)pd->stride_u;
    P.sv = (int)pd->stride_v;
    P.koff = 0u - 0x4B400000u * (uint32_t)P.su - 0x4B400000u * (uint32_t)P.sv;
    P.wide = pd->stride_u < ((int64_t)1 << 30) && pd->stride_v < ((int64_t)1 << 30);
    P.fnu1 = (float)pd->nu + 1.f;
    P.fnv1 = (float)pd->nv + 1.f;
    P.projs = projs_dev;
    P.vol = vol_dev;
    P.mult = multiplier_dev;
    P.n[0] = (int)vd->nx;
    P.n[1] = (int)vd->ny;
    P.n[2] = (int)vd->nz;
    if (vd->order == 0) {
        P.vs[0] = (int64_t)vd->ny * vd->nz;
        P.vs[1] = vd->nz;
        P.vs[2] = 1;
    } else {
        P.vs[0] = 1;
        P.vs[1] = vd->nx;
        P.vs[2] = (int64_t)vd->nx * vd->ny;
    }
    P.voxwid = vd->voxwid;
    P.vwd = (double)vd->voxwid;
    P.cornerd[0] = vd->corner.x;
    P.cornerd[1] = vd->corner.y;
    P.cornerd[2] = vd->corner.z;
    P.c0[0] = vd->corner.x + 0.5f * vd->voxwid * (float)vd->nx;
    P.c0[1] = vd->corner.y + 0.5f * vd->voxwid * (float)vd->ny;
    P.c0[2] = vd->corner.z + 0.5f * vd->voxwid * (float)vd->nz;
    P.mask = cfg->mask_to_cylinder ? 1 : 0;
    P.mask_r2 = cfg->mask_to_cyl_rad * cfg->mask_to_cyl_rad;
    P.all_ones = cfg->backproject_all_1s ? 1 : 0;
    P.sep = cfg->soften_edge_proportion;
    P.inv_sep = P.sep > 0.f ? 1.f / P.sep : 0.f;
    P.pL = cfg->Z_on_L_factor_power;
    P.pV = cfg->Z_on_val_factor_power;
    P.val = cfg->Z_on_val_factor_val;
    P.inv_val = P.val != 0.f ? (float)(1.0 / (double)P.val) : 0.f;
    P.preset = (int)cfg->weighting_preset;
    P.ssx = (int)cfg->ssx;
    P.ssy = (int)cfg->ssy;
    P.ssz = (int)cfg->ssz;
    P.status = status_dev;

    const int knob = ab_tuning_get(AB_TUNE_BP_XB);
    const bool forced = force_xb == 2 || force_xb == 4 || force_xb == 8;
    xb = forced ? force_xb : (knob == 2 || knob == 4 || knob == 8 ? knob : default_xb(cfg->exact != 0));
    const int ord = ord_out && bp_zlanes_ok(vd, pd, xb, cfg, true) ? 3 : bp_ord(vd);
    if (ord_out) *ord_out = ord;
    // z columns of 8 voxels per thread where the volume is tall enough (the
    // per-view work of a thread is shared by twice as many voxels: sirt256
    // 8.66 -> 8.35 ms), unless the caller or the knob chose
    if (ord == 3 && !forced && knob == 0 && vd->nz >= 256u && !cfg->exact) xb = 8;
    const int kXB = xb;
    if (ord == 2) {  // slices: lanes along y, warps x XB along x
        P.gb[0] = (P.n[1] + 31) / 32;
        P.gb[1] = (P.n[0] + 8 * kXB - 1) / (8 * kXB);
        P.gb[2] = 1;
    } else if (ord == 3) {  // z columns of 32 XB voxels, warps along y, one x layer
        P.gb[0] = (P.n[2] + 32 * kXB - 1) / (32 * kXB);
        P.gb[1] = (P.n[1] + 7) / 8;
        P.gb[2] = P.n[0];
    } else {
        const int n0 = ord == 0 ? P.n[2] : P.n[0], n1 = P.n[1], n2 = ord == 0 ? P.n[0] : P.n[2];
        P.gb[0] = (n0 + 31) / 32;
        P.gb[1] = (n1 + 7) / 8;
        P.gb[2] = (n2 + kXB - 1) / kXB;
    }
    // Super-brick: all blocks of the fastest axis x sb1 x sb2 blocks (8 and
    // kXB voxels each; 8 and 1 for ORD 3), about one wave of resident CTAs,
    // with equal extents in voxels along the middle and slowest axes.
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    const int wave = ab_tuning_get(AB_TUNE_BP_WAVE) > 0 ? ab_tuning_get(AB_TUNE_BP_WAVE) : bp_min_blocks(xb, cfg->exact != 0);
    const double target = (double)wave * sms / (double)P.gb[0];  // blocks of the (middle x slowest) plane per wave
    const int ext2 = ord == 3 ? 1 : kXB;  // voxels of a block along the slowest axis
    int sb1 = (int)floor(sqrt(target * ext2 / 8.0) + 0.5);
    sb1 = sb1 < 1 ? 1 : (sb1 > P.gb[1] ? P.gb[1] : sb1);
    int sb2 = (int)floor(target / sb1 + 0.5);
    sb2 = sb2 < 1 ? 1 : (sb2 > P.gb[2] ? P.gb[2] : sb2);
    P.sb1 = sb1;
    P.sb2 = sb2;
    P.nsb1 = (P.gb[1] + sb1 - 1) / sb1;
    const int64_t nsb = (int64_t)P.nsb1 * ((P.gb[2] + sb2 - 1) / sb2);
    const int64_t grid = nsb * P.gb[0] * sb1 * sb2;
    if (grid > 0x7fffffffLL) return ab_fail(APRICT_ERR_TOO_LARGE, "volume too large for the grid");
    units = (uint64_t)grid;
    return APRICT_OK;
}

}  // namespace ab_bp
