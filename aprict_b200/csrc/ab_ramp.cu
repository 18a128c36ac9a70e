// ab_ramp.cu -- weighted 1-D convolution along the detector u axis (ramp /
// Hilbert filtering for FBP), as a shared-memory direct convolution.
//
// Replaces RampFilterer._filter_chunk_axis1 (src/aprict/cb/ramp_filter.py:139-240):
// zero-pad each detector row to next_fast_len(2 nu - 1), cuFFT rfft, multiply
// by the kernel spectrum, irfft, crop -- i.e. an exact linear convolution of
// the (cosine-weighted, :685-689) row with taps h[n], |n| <= nu-1. Here the
// same linear convolution is evaluated directly:
//     out[row][m] = scale * sum_j h[m - j] * w[j][v] * in[row][j].
//
// B200 layout: a CTA stages R rows (times the weights; R = 8 while the Q x R
// accumulators fit, else 4) and all 2 nu - 1 taps in shared memory with
// coalesced loads, then each thread produces Q outputs per row (m = t, t+T,
// ...), reading the weighted rows as R/4 float4 broadcasts and the taps
// conflict-free: each tap read feeds R multiply-adds. Pure Ram-Lak taps vanish at even
// nonzero offsets (src/aprict/ramp_kernels.py:43-59), so in ODD mode only
// taps of odd offset are visited plus the centre tap: half the FMAs.
#include <cuda_runtime.h>

#include "ab_common.cuh"
#include "ab_host.h"

namespace {

constexpr int kThreads = 256;
constexpr int kR = 4;  // rows per CTA for Q >= 8 (one float4 of a column)

struct RampParams {
    const float *in;
    float *out;
    const float *taps;     // 2*nu-1, centre at nu-1
    const float *weights;  // (nu, nv) element strides (wsu, wsv), or null
    int64_t wsu, wsv;
    int n_views, nu, nv;
    int64_t is_view, is_u, is_v;  // input strides (elements)
    int64_t os_view, os_u, os_v;  // output strides
    float scale;
    int odd;  // taps at even nonzero offsets are all zero
};

__device__ __forceinline__ void row_of(const RampParams &P, int64_t r, int &m, int &v) {
    m = (int)(r / P.nv);
    v = (int)(r % P.nv);
}

template <int Q, int R>
__global__ void __launch_bounds__(kThreads) k_ramp(RampParams P, int64_t n_rows) {
    constexpr int kG = R / 4;  // float4 groups of rows
    extern __shared__ float4 smem4[];
    float4 *xs = smem4;                                      // [nu][kG] x 4 rows
    float *hs = reinterpret_cast<float *>(smem4 + (size_t)P.nu * kG);  // [2 nu - 1]
    const int64_t r0 = (int64_t)blockIdx.x * R;
    const int nu = P.nu;

    for (int k = threadIdx.x; k < 2 * nu - 1; k += kThreads) hs[k] = P.taps[k];
    // Stage the weighted rows. Rows of a CTA are consecutive row indices
    // (view-major, v fastest): when the v stride is 1 the R rows of one u are
    // adjacent in memory, otherwise each row is contiguous along u.
    float *xf = reinterpret_cast<float *>(xs);
    const bool v_contig = P.is_v == 1 && P.nv >= R;
    for (int e = threadIdx.x; e < R * nu; e += kThreads) {
        int q, j;
        if (v_contig) {
            q = e % R;
            j = e / R;
        } else {
            q = e / nu;
            j = e % nu;
        }
        const int64_t r = r0 + q;
        float val = 0.f;
        if (r < n_rows) {
            int m, v;
            row_of(P, r, m, v);
            val = P.in[(int64_t)m * P.is_view + (int64_t)j * P.is_u + (int64_t)v * P.is_v];
            if (P.weights) val *= P.weights[(int64_t)j * P.wsu + (int64_t)v * P.wsv];
        }
        xf[j * R + q] = val;
    }
    __syncthreads();

    float acc[Q][R];
#pragma unroll
    for (int a = 0; a < Q; ++a)
#pragma unroll
        for (int q = 0; q < R; ++q) acc[a][q] = 0.f;

    const int t = threadIdx.x;
    // Taps index: h[m - j] lives at hs[m - j + nu - 1].
    if (P.odd) {
        // m shares the parity of t (kThreads is even); visit j of the other parity.
        const int j0 = 1 - (t & 1);
        for (int j = j0; j < nu; j += 2) {
            float4 x[kG];
#pragma unroll
            for (int g = 0; g < kG; ++g) x[g] = xs[j * kG + g];
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                const int m = t + a * kThreads;
                const float h = (m < nu) ? hs[m - j + nu - 1] : 0.f;
#pragma unroll
                for (int g = 0; g < kG; ++g) {
                    acc[a][4 * g + 0] = fmaf(h, x[g].x, acc[a][4 * g + 0]);
                    acc[a][4 * g + 1] = fmaf(h, x[g].y, acc[a][4 * g + 1]);
                    acc[a][4 * g + 2] = fmaf(h, x[g].z, acc[a][4 * g + 2]);
                    acc[a][4 * g + 3] = fmaf(h, x[g].w, acc[a][4 * g + 3]);
                }
            }
        }
        const float hc = hs[nu - 1];
#pragma unroll
        for (int a = 0; a < Q; ++a) {
            const int m = t + a * kThreads;
            if (m < nu) {
#pragma unroll
                for (int g = 0; g < kG; ++g) {
                    const float4 x = xs[m * kG + g];
                    acc[a][4 * g + 0] = fmaf(hc, x.x, acc[a][4 * g + 0]);
                    acc[a][4 * g + 1] = fmaf(hc, x.y, acc[a][4 * g + 1]);
                    acc[a][4 * g + 2] = fmaf(hc, x.z, acc[a][4 * g + 2]);
                    acc[a][4 * g + 3] = fmaf(hc, x.w, acc[a][4 * g + 3]);
                }
            }
        }
    } else {
        for (int j = 0; j < nu; ++j) {
            float4 x[kG];
#pragma unroll
            for (int g = 0; g < kG; ++g) x[g] = xs[j * kG + g];
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                const int m = t + a * kThreads;
                const float h = (m < nu) ? hs[m - j + nu - 1] : 0.f;
#pragma unroll
                for (int g = 0; g < kG; ++g) {
                    acc[a][4 * g + 0] = fmaf(h, x[g].x, acc[a][4 * g + 0]);
                    acc[a][4 * g + 1] = fmaf(h, x[g].y, acc[a][4 * g + 1]);
                    acc[a][4 * g + 2] = fmaf(h, x[g].z, acc[a][4 * g + 2]);
                    acc[a][4 * g + 3] = fmaf(h, x[g].w, acc[a][4 * g + 3]);
                }
            }
        }
    }

#pragma unroll
    for (int a = 0; a < Q; ++a) {
        const int mo = t + a * kThreads;
        if (mo >= nu) continue;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const int64_t r = r0 + q;
            if (r >= n_rows) continue;
            int m, v;
            row_of(P, r, m, v);
            P.out[(int64_t)m * P.os_view + (int64_t)mo * P.os_u + (int64_t)v * P.os_v] = acc[a][q] * P.scale;
        }
    }
}

}  // namespace

extern "C" int aprict_b200_ramp_filter(const aprict_proj_desc *in_desc, const float *in_dev,
                                       const aprict_proj_desc *out_desc, float *out_dev, const float *taps_dev,
                                       int odd_taps_only, const float *weights_dev, int64_t w_stride_u,
                                       int64_t w_stride_v, float scale, aprict_stream_t stream) {
    int rc;
    if ((rc = ab_check_projs(in_desc, in_dev, "ramp input")) != APRICT_OK) return rc;
    if ((rc = ab_check_projs(out_desc, out_dev, "ramp output")) != APRICT_OK) return rc;
    if (in_desc->n_views != out_desc->n_views || in_desc->nu != out_desc->nu || in_desc->nv != out_desc->nv)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ramp filter: input and output shapes differ");
    if (in_desc->n_views == 0 || in_desc->nu == 0 || in_desc->nv == 0) return APRICT_OK;
    if (taps_dev == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ramp filter: null taps");
    if (in_dev == out_dev) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ramp filter: in-place filtering is not supported");
    const int nu = (int)in_desc->nu;
    const int q = (nu + kThreads - 1) / kThreads;
    // rows per CTA: 8 while the accumulators fit (Q <= 4), else 4
    const int rows = q <= 4 ? 8 : kR;
    const size_t smem = (size_t)nu * rows * sizeof(float) + (size_t)(2 * nu - 1) * sizeof(float);
    if (smem > 200 * 1024) return ab_fail(APRICT_ERR_TOO_LARGE, "ramp filter: nu = %d exceeds shared memory", nu);
    RampParams P;
    P.in = in_dev;
    P.out = out_dev;
    P.taps = taps_dev;
    P.weights = weights_dev;
    P.wsu = w_stride_u;
    P.wsv = w_stride_v;
    P.n_views = (int)in_desc->n_views;
    P.nu = nu;
    P.nv = (int)in_desc->nv;
    P.is_view = in_desc->stride_view;
    P.is_u = in_desc->stride_u;
    P.is_v = in_desc->stride_v;
    P.os_view = out_desc->stride_view;
    P.os_u = out_desc->stride_u;
    P.os_v = out_desc->stride_v;
    P.scale = scale;
    P.odd = odd_taps_only ? 1 : 0;
    const int64_t n_rows = (int64_t)in_desc->n_views * in_desc->nv;
    const int64_t blocks = (n_rows + rows - 1) / rows;
    if (blocks > 0x7fffffff) return ab_fail(APRICT_ERR_TOO_LARGE, "ramp filter: too many rows");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
#define AB_RAMP_LAUNCH(QQ, RR)                                                                                \
    do {                                                                                                      \
        if (smem > 48 * 1024) cudaFuncSetAttribute(k_ramp<QQ, RR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        k_ramp<QQ, RR><<<(unsigned)blocks, kThreads, smem, st>>>(P, n_rows);                                  \
    } while (0)
    if (q <= 1)
        AB_RAMP_LAUNCH(1, 8);
    else if (q <= 2)
        AB_RAMP_LAUNCH(2, 8);
    else if (q <= 4)
        AB_RAMP_LAUNCH(4, 8);
    else if (q <= 8)
        AB_RAMP_LAUNCH(8, 4);
    else if (q <= 16)
        AB_RAMP_LAUNCH(16, 4);
    else
        return ab_fail(APRICT_ERR_TOO_LARGE, "ramp filter: nu = %d exceeds 4096", nu);
#undef AB_RAMP_LAUNCH
    return ab_cuda_check(cudaGetLastError(), "ramp_filter launch");
}
