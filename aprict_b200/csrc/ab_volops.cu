// ab_volops.cu -- element-wise volume operations.
//
// Replaces the surface kernels of src/aprict/data/cusrc/texture_operations.cu
// (fill_surface :124-135, softmask_surface_to_cylinder_xy :137-162,
// multiplicatively_invert_surface :164-185, multiply_surface :187-199,
// inner_product_3D_surfaces :284-307, multiply_surfaces :309-...) driven by
// src/aprict/lib/texture_tools/operations.py. Volumes here are linear
// buffers, so every op except the cylinder mask is a flat vectorised sweep:
// float4 loads/stores when the pointer and length allow, grid-stride loops
// sized to a multiple of the SM count.
#include <cuda_runtime.h>

#include "ab_common.cuh"
#include "ab_host.h"

namespace {

constexpr int kThreads = 256;

int grid_for(int64_t n4) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    int64_t want = (n4 + kThreads - 1) / kThreads;
    const int64_t cap = (int64_t)sms * 8;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return (int)want;
}

template <class F>
__global__ void k_map(float *__restrict__ v, int64_t n, F f) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool vec = (reinterpret_cast<uintptr_t>(v) & 15u) == 0;
    if (vec) {
        const int64_t n4 = n >> 2;
        float4 *v4 = reinterpret_cast<float4 *>(v);
        for (int64_t j = i; j < n4; j += stride) {
            float4 x = v4[j];
            x.x = f(x.x);
            x.y = f(x.y);
            x.z = f(x.z);
            x.w = f(x.w);
            v4[j] = x;
        }
        for (int64_t j = (n4 << 2) + i; j < n; j += stride) v[j] = f(v[j]);
    } else {
        for (int64_t j = i; j < n; j += stride) v[j] = f(v[j]);
    }
}

struct FillOp {
    float c;
    __device__ float operator()(float) const { return c; }
};
struct ScaleOp {
    float c;
    __device__ float operator()(float x) const { return c * x; }
};
// multiplicatively_invert_surface: v <- 1 / (v + eps exp(-v/eps)), zeros
// optionally left alone.
struct InvertOp {
    float eps;
    int ignore_zeros;
    __device__ float operator()(float x) const {
        if (ignore_zeros && x == 0.f) return x;
        if (eps > 0.f) x = x + eps * expf(-x / eps);
        return 1.f / x;
    }
};

template <class F>
int launch_map(float *v, int64_t n, F f, aprict_stream_t stream, const char *what) {
    if (n < 0) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: negative length", what);
    if (n == 0) return APRICT_OK;
    if (v == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: null pointer", what);
    k_map<<<grid_for(n / 4 + 1), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(v, n, f);
    return ab_cuda_check(cudaGetLastError(), what);
}

// softmask_surface_to_cylinder_xy (texture_operations.cu:137-162): the radius
// is measured in voxel indices about the volume centre, relative to the
// inscribed circle of the xy cross-section.
__global__ void k_softmask(float *__restrict__ v, int nx, int ny, int nz, int64_t sx, int64_t sy, int64_t sz,
                           float r0) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const float cx = (nx - 1) / 2.f, cy = (ny - 1) / 2.f;
    const float inv = 2.f / (float)min(nx, ny);
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        // e enumerates (x, y, z) with z fastest; offsets follow the strides.
        const int z = (int)(e % nz);
        const int64_t r = e / nz;
        const int y = (int)(r % ny);
        const int x = (int)(r / ny);
        const float dx = (float)x - cx, dy = (float)y - cy;
        float rr = sqrtf(dx * dx + dy * dy) * inv;
        if (rr < r0) continue;
        float m;
        if (r0 >= 1.f) {
            m = 0.f;
        } else {
            rr = fminf((rr - r0) / (1.f - r0), 1.f);
            m = fminf(1.f, fmaxf(0.f, (1.f + cospif(rr)) * 0.5f));
        }
        const int64_t o = (int64_t)x * sx + (int64_t)y * sy + (int64_t)z * sz;
        v[o] *= m;
    }
}

// <a, b> in double: per-thread double partials, warp shuffle, one atomic per
// block (inner_product_3D_surfaces reduces with a shared cuda::atomic<double>,
// texture_operations.cu:284-307).
__global__ void k_dot(const float *__restrict__ a, const float *__restrict__ b, int64_t n, double *out) {
    double s = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        s += (double)a[i] * (double)b[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ double red[kThreads / 32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < kThreads / 32 ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) atomicAdd(out, s);
    }
}

__global__ void k_mul(float *__restrict__ out, const float *__restrict__ a, const float *__restrict__ b,
                      int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = a[i] * b[i];
}

// out = a + alpha * b
__global__ void k_axpy(float *__restrict__ out, const float *a, float alpha, const float *__restrict__ b,
                       int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = fmaf(alpha, b[i], a[i]);
}

// out = a / (w + eps exp(-w / eps)) (divide_surfaces_softzero,
// texture_operations.cu:333-351): the reciprocal of the softened divisor,
// then the product, in the reference's order; eps <= 0 divides plainly.
__global__ void k_div_softzero(float *out, const float *a, const float *__restrict__ w, int64_t n, float eps) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float d = w[i];
        if (eps > 0.f) d = d + eps * expf(-d / eps);
        out[i] = a[i] * (1.f / d);
    }
}

// v[x][y][z] *= g[x * ny + y] for every z (multiply_surfaces with the second
// surface broadcast over z, texture_operations.cu:309-331).
__global__ void k_mul_xygrid(float *v, int nx, int ny, int nz, int64_t sx, int64_t sy, int64_t sz, int order_f,
                             const float *__restrict__ g) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        int x, y, z;
        if (order_f) {  // x fastest
            x = (int)(e % nx);
            y = (int)((e / nx) % ny);
            z = (int)(e / ((int64_t)nx * ny));
        } else {  // z fastest
            z = (int)(e % nz);
            y = (int)((e / nz) % ny);
            x = (int)(e / ((int64_t)ny * nz));
        }
        v[(int64_t)x * sx + (int64_t)y * sy + (int64_t)z * sz] *= g[(int64_t)x * ny + y];
    }
}

}  // namespace

extern "C" int aprict_b200_vol_div_softzero(float *out_dev, const float *a_dev, const float *w_dev, int64_t n,
                                            float eps, aprict_stream_t stream) {
    if (n < 0) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "vol_div_softzero: negative length");
    if (n == 0) return APRICT_OK;
    if (!a_dev || !w_dev || !out_dev) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "vol_div_softzero: null pointer");
    if (!(eps == eps)) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "vol_div_softzero: eps is NaN");
    k_div_softzero<<<grid_for(n), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(out_dev, a_dev, w_dev, n,
                                                                                         eps);
    return ab_cuda_check(cudaGetLastError(), "vol_div_softzero");
}

extern "C" int aprict_b200_vol_mul_xygrid(float *v_dev, const aprict_vol_desc *vd, const float *grid_dev,
                                          aprict_stream_t stream) {
    int rc = ab_check_vol(vd, v_dev, "vol_mul_xygrid");
    if (rc != APRICT_OK) return rc;
    const int64_t n = (int64_t)vd->nx * vd->ny * vd->nz;
    if (n == 0) return APRICT_OK;
    if (grid_dev == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "vol_mul_xygrid: null grid");
    int64_t sx, sy, sz;
    if (vd->order == 0) {
        sx = (int64_t)vd->ny * vd->nz;
        sy = vd->nz;
        sz = 1;
    } else {
        sx = 1;
        sy = vd->nx;
        sz = (int64_t)vd->nx * vd->ny;
    }
    k_mul_xygrid<<<grid_for(n), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        v_dev, (int)vd->nx, (int)vd->ny, (int)vd->nz, sx, sy, sz, vd->order != 0, grid_dev);
    return ab_cuda_check(cudaGetLastError(), "vol_mul_xygrid");
}

extern "C" int aprict_b200_vol_fill(float *v_dev, int64_t n, float value, aprict_stream_t stream) {
    return launch_map(v_dev, n, FillOp{value}, stream, "vol_fill");
}

extern "C" int aprict_b200_vol_scale(float *v_dev, int64_t n, float factor, aprict_stream_t stream) {
    return launch_map(v_dev, n, ScaleOp{factor}, stream, "vol_scale");
}

extern "C" int aprict_b200_vol_invert(float *v_dev, int64_t n, int ignore_zeros, float eps,
                                      aprict_stream_t stream) {
    return launch_map(v_dev, n, InvertOp{eps, ignore_zeros}, stream, "vol_invert");
}

extern "C" int aprict_b200_vol_softmask_cylinder(float *v_dev, const aprict_vol_desc *vd, float relrad_start,
                                                 aprict_stream_t stream) {
    int rc = ab_check_vol(vd, v_dev, "vol_softmask_cylinder");
    if (rc != APRICT_OK) return rc;
    if (!(relrad_start >= 0.f && relrad_start <= 1.f))
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "relrad_start must be in [0, 1]");
    int64_t sx, sy, sz;
    if (vd->order == 0) {
        sx = (int64_t)vd->ny * vd->nz;
        sy = vd->nz;
        sz = 1;
    } else {
        sx = 1;
        sy = vd->nx;
        sz = (int64_t)vd->nx * vd->ny;
    }
    const int64_t n = (int64_t)vd->nx * vd->ny * vd->nz;
    k_softmask<<<grid_for(n), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        v_dev, (int)vd->nx, (int)vd->ny, (int)vd->nz, sx, sy, sz, relrad_start);
    return ab_cuda_check(cudaGetLastError(), "vol_softmask_cylinder");
}

extern "C" int aprict_b200_vol_dot(const float *a_dev, const float *b_dev, int64_t n, double *out_dev,
                                   aprict_stream_t stream) {
    if (n < 0) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "vol_dot: negative length");
    if (n == 0) return APRICT_OK;
    if (!a_dev || !b_dev || !out_dev) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "vol_dot: null pointer");
    k_dot<<<grid_for(n), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a_dev, b_dev, n, out_dev);
    return ab_cuda_check(cudaGetLastError(), "vol_dot");
}

extern "C" int aprict_b200_vol_mul(float *out_dev, const float *a_dev, const float *b_dev, int64_t n,
                                   aprict_stream_t stream) {
    if (n < 0) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "vol_mul: negative length");
    if (n == 0) return APRICT_OK;
    if (!a_dev || !b_dev || !out_dev) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "vol_mul: null pointer");
    k_mul<<<grid_for(n), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(out_dev, a_dev, b_dev, n);
    return ab_cuda_check(cudaGetLastError(), "vol_mul");
}

extern "C" int aprict_b200_vol_axpy(float *out_dev, const float *a_dev, float alpha, const float *b_dev,
                                    int64_t n, aprict_stream_t stream) {
    if (n < 0) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "vol_axpy: negative length");
    if (n == 0) return APRICT_OK;
    if (!a_dev || !b_dev || !out_dev) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "vol_axpy: null pointer");
    k_axpy<<<grid_for(n), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(out_dev, a_dev, alpha, b_dev, n);
    return ab_cuda_check(cudaGetLastError(), "vol_axpy");
}
