// ab_rotate.cu -- rotated bilinear resampling of projection stacks for the
// cone-cylinder FBP filter.
//
// FBPFilterer.filter_bulk_axis1_stream (src/aprict/cb/ramp_filter.py:577-842)
// filters every cone-beam projection along tilted lines: it zero-pads the
// projection to a wider frame (:651), rotates it with
// cupyx.scipy.ndimage.rotate(order=1, mode="grid-constant", reshape=False,
// prefilter=False) (:662-683), multiplies by a weight mask (:685-689) and a
// per-view letterbox of detector columns (:690-749), ramp-filters along u,
// rotates the result back (:790-806) and crops the padding (:836-842) -- one
// library call and several array passes per projection. Here the rotation,
// padding, mask, letterbox and crop of a whole stack are one launch each way.
//
// The resampling is the published scipy.ndimage definition that the cupyx
// call follows: output index o maps to input coordinate
//     q = M (o - c) + c,   M = [[cos a, sin a], [-sin a, cos a]],
// a the rotate() angle and c = (n - 1) / 2 per axis of the (padded) frame,
// and the value is the bilinear interpolation of the four neighbours of q,
// neighbours outside the array counting as 0 (mode "grid-constant"). The
// coordinates and weights are FP64, the result is rounded to FP32 as the
// library stores it; the mask product is FP64 rounded to FP32 (an FP32 array
// times an FP64 mask) and so is the letterbox product.
#include <cuda_runtime.h>

#include <cmath>

#include "ab_host.h"

namespace {

constexpr int kThreads = 256;

struct RotParams {
    const float *in;
    float *out;
    const double *cs;     // (cos a, sin a) per view
    const double *mask;   // (nu_out, nv_out) dense, or null
    const double *colw;   // (n_views, nv_out) dense, or null
    int nu_in, nv_in, nu_out, nv_out;
    int64_t is_view, is_u, is_v, os_view, os_u, os_v;
    double cu, cv;        // rotation centre in the padded frame
    double in_u0, in_v0;  // position of in[0][0] in the padded frame
    int out_u0, out_v0;   // position of out[0][0] in the padded frame
};

__global__ void __launch_bounds__(kThreads) k_rotate(const RotParams P, int64_t n) {
    const int64_t step = (int64_t)gridDim.x * kThreads;
    for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n; e += step) {
        const int j = (int)(e % P.nv_out);
        const int64_t r = e / P.nv_out;
        const int i = (int)(r % P.nu_out);
        const int m = (int)(r / P.nu_out);
        const double c = P.cs[2 * m], s = P.cs[2 * m + 1];
        const double pu = (double)(i + P.out_u0) - P.cu, pv = (double)(j + P.out_v0) - P.cv;
        // input coordinate, relative to in[0][0]
        const double qu = (c * pu + s * pv + P.cu) - P.in_u0;
        const double qv = (-s * pu + c * pv + P.cv) - P.in_v0;
        double val = 0.0;
        // Only coordinates with a neighbour inside the array contribute (this
        // also keeps non-finite coordinates away from the integer conversion).
        if (qu > -1.0 && qu < (double)P.nu_in && qv > -1.0 && qv < (double)P.nv_in) {
            const double fu = floor(qu), fv = floor(qv);
            const double tu = qu - fu, tv = qv - fv;
            const int iu = (int)fu, iv = (int)fv;
            const float *src = P.in + (int64_t)m * P.is_view;
            const bool u0 = iu >= 0, u1 = iu + 1 < P.nu_in, v0 = iv >= 0, v1 = iv + 1 < P.nv_in;
            const double a00 = u0 && v0 ? (double)__ldg(src + (int64_t)iu * P.is_u + (int64_t)iv * P.is_v) : 0.0;
            const double a01 = u0 && v1 ? (double)__ldg(src + (int64_t)iu * P.is_u + (int64_t)(iv + 1) * P.is_v) : 0.0;
            const double a10 = u1 && v0 ? (double)__ldg(src + (int64_t)(iu + 1) * P.is_u + (int64_t)iv * P.is_v) : 0.0;
            const double a11 = u1 && v1 ? (double)__ldg(src + (int64_t)(iu + 1) * P.is_u + (int64_t)(iv + 1) * P.is_v) : 0.0;
            val = (1.0 - tu) * ((1.0 - tv) * a00 + tv * a01) + tu * ((1.0 - tv) * a10 + tv * a11);
        }
        float x = (float)val;
        if (P.mask) x = (float)((double)x * P.mask[(int64_t)i * P.nv_out + j]);
        if (P.colw) x = (float)((double)x * P.colw[(int64_t)m * P.nv_out + j]);
        P.out[(int64_t)m * P.os_view + (int64_t)i * P.os_u + (int64_t)j * P.os_v] = x;
    }
}

}  // namespace

extern "C" int aprict_b200_rotate_projections(const aprict_proj_desc *in_desc, const float *in_dev,
                                              const aprict_proj_desc *out_desc, float *out_dev, const double *cs_dev,
                                              double centre_u, double centre_v, int32_t in_off_u, int32_t in_off_v,
                                              int32_t out_off_u, int32_t out_off_v, const double *mask_dev,
                                              const double *colw_dev, aprict_stream_t stream) {
    int rc;
    if ((rc = ab_check_projs(in_desc, in_dev, "rotate input")) != APRICT_OK) return rc;
    if ((rc = ab_check_projs(out_desc, out_dev, "rotate output")) != APRICT_OK) return rc;
    if (in_desc->n_views != out_desc->n_views)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "rotate: input and output view counts differ");
    if (out_desc->n_views == 0 || out_desc->nu == 0 || out_desc->nv == 0) return APRICT_OK;
    if (cs_dev == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "rotate: null rotation table");
    if (in_dev == out_dev) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "rotate: in-place resampling is not supported");
    if (!std::isfinite(centre_u) || !std::isfinite(centre_v))
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "rotate: non-finite rotation centre");
    const int32_t lim = 1 << 24;
    if (in_off_u < -lim || in_off_u > lim || in_off_v < -lim || in_off_v > lim || out_off_u < -lim ||
        out_off_u > lim || out_off_v < -lim || out_off_v > lim)
        return ab_fail(APRICT_ERR_TOO_LARGE, "rotate: frame offsets exceed 2^24");
    RotParams P;
    P.in = in_dev;
    P.out = out_dev;
    P.cs = cs_dev;
    P.mask = mask_dev;
    P.colw = colw_dev;
    P.nu_in = (int)in_desc->nu;
    P.nv_in = (int)in_desc->nv;
    P.nu_out = (int)out_desc->nu;
    P.nv_out = (int)out_desc->nv;
    P.is_view = in_desc->stride_view;
    P.is_u = in_desc->stride_u;
    P.is_v = in_desc->stride_v;
    P.os_view = out_desc->stride_view;
    P.os_u = out_desc->stride_u;
    P.os_v = out_desc->stride_v;
    P.cu = centre_u;
    P.cv = centre_v;
    P.in_u0 = (double)in_off_u;
    P.in_v0 = (double)in_off_v;
    P.out_u0 = out_off_u;
    P.out_v0 = out_off_v;
    // An empty input leaves an all-zero output: point the (never read) source
    // at the output so that no null pointer reaches the kernel.
    if (in_desc->nu == 0 || in_desc->nv == 0) {
        P.in = out_dev;
        P.nu_in = P.nv_in = 0;
    }
    const int64_t n = (int64_t)out_desc->n_views * out_desc->nu * out_desc->nv;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 148;
    const int64_t want = (n + kThreads - 1) / kThreads;
    const int64_t cap = (int64_t)sms * 8;  // 8 CTAs of 256 threads per SM, grid-stride beyond
    k_rotate<<<(unsigned)(want < cap ? want : cap), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(P, n);
    return ab_cuda_check(cudaGetLastError(), "rotate_projections launch");
}
