// ref_gpu_project.cu -- the reference's projector kernel on the GPU, and the
// volume arrays both reference kernels read (see ref_gpu.h).
//
// TEST INFRASTRUCTURE ONLY. Includes src/aprict/data/cusrc/CB_project_texture_chunked.cu
// in place from the reference checkout. That file builds a uint3 from a braced
// list of ints (:257), which the reference's NVRTC build accepts and nvcc's
// front end does not; the reference's uint3 is therefore read as a small
// struct with an (int, int, int) constructor for the duration of the include
// (only its x, y, z members are used).
#include <cstdio>
#include <cuda/atomic>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "ref_gpu.h"

struct refgpu_u3 {
    unsigned int x, y, z;
    __host__ __device__ refgpu_u3() {}
    __host__ __device__ refgpu_u3(int a, int b, int c) : x((unsigned)a), y((unsigned)b), z((unsigned)c) {}
};
#define uint3 refgpu_u3
namespace refp {
#include "CB_project_texture_chunked.cu"
}
#undef uint3

static_assert(sizeof(refp::proj_spec) == 60, "proj_spec is the 60-byte record");

struct refgpu_vol {
    cudaArray_t arr;
    cudaSurfaceObject_t surf;
    int nx, ny, nz;
};

static cudaMemcpy3DParms copy_params(const refgpu_vol *v) {
    cudaMemcpy3DParms p{};
    p.extent = make_cudaExtent((size_t)v->nz, (size_t)v->ny, (size_t)v->nx);
    p.kind = cudaMemcpyDeviceToDevice;
    return p;
}

extern "C" int refgpu_vol_create(const float *src_dev, int nx, int ny, int nz, refgpu_vol **out) {
    *out = nullptr;
    if (nx <= 0 || ny <= 0 || nz <= 0) return (int)cudaErrorInvalidValue;
    refgpu_vol *v = new refgpu_vol{};
    v->nx = nx;
    v->ny = ny;
    v->nz = nz;
    const cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    cudaError_t e = cudaMalloc3DArray(&v->arr, &cd, make_cudaExtent((size_t)nz, (size_t)ny, (size_t)nx),
                                      cudaArraySurfaceLoadStore);
    if (e != cudaSuccess) {
        delete v;
        return (int)e;
    }
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = v->arr;
    e = cudaCreateSurfaceObject(&v->surf, &rd);
    if (e == cudaSuccess && src_dev) {
        cudaMemcpy3DParms p = copy_params(v);
        p.srcPtr = make_cudaPitchedPtr((void *)src_dev, (size_t)nz * sizeof(float), (size_t)nz, (size_t)ny);
        p.dstArray = v->arr;
        e = cudaMemcpy3D(&p);
    }
    if (e != cudaSuccess) {
        refgpu_vol_destroy(v);
        return (int)e;
    }
    *out = v;
    return 0;
}

extern "C" int refgpu_vol_read(const refgpu_vol *v, float *dst_dev, cudaStream_t st) {
    cudaMemcpy3DParms p = copy_params(v);
    p.srcArray = v->arr;
    p.dstPtr = make_cudaPitchedPtr(dst_dev, (size_t)v->nz * sizeof(float), (size_t)v->nz, (size_t)v->ny);
    return (int)cudaMemcpy3DAsync(&p, st);
}

extern "C" int refgpu_vol_write(refgpu_vol *v, const float *src_dev, cudaStream_t st) {
    cudaMemcpy3DParms p = copy_params(v);
    p.srcPtr = make_cudaPitchedPtr((void *)src_dev, (size_t)v->nz * sizeof(float), (size_t)v->nz, (size_t)v->ny);
    p.dstArray = v->arr;
    return (int)cudaMemcpy3DAsync(&p, st);
}

extern "C" void refgpu_vol_destroy(refgpu_vol *v) {
    if (!v) return;
    if (v->surf) cudaDestroySurfaceObject(v->surf);
    if (v->arr) cudaFreeArray(v->arr);
    delete v;
}

// The reference's surface object of a volume (used by ref_gpu_backproject.cu).
extern "C" cudaSurfaceObject_t refgpu_vol_surface(const refgpu_vol *v) { return v ? v->surf : 0; }
extern "C" void refgpu_vol_shape(const refgpu_vol *v, int *n) {
    n[0] = v->nx;
    n[1] = v->ny;
    n[2] = v->nz;
}

extern "C" int refgpu_project(const refgpu_vol *v, float voxwid, const float *texpos, const void *specs_dev,
                              unsigned n_views, unsigned nu, unsigned nv, float *out_dev, float svf, float mba,
                              unsigned ssu, unsigned ssv, cudaStream_t st) {
    if (n_views == 0 || nu == 0 || nv == 0) return 0;
    if (n_views > 65535u) return (int)cudaErrorInvalidValue;
    refp::config_CB_project cfg;
    cfg.shrink_volume_factor = svf;
    cfg.multiply_before_adding = mba;
    cfg.ssu = ssu;
    cfg.ssv = ssv;
    refp::vol_tex_chunk_spec tcs;
    tcs.voxwid = voxwid;
    tcs.offsets.x = tcs.offsets.y = tcs.offsets.z = 0;
    tcs.shape.x = (unsigned)v->nx;
    tcs.shape.y = (unsigned)v->ny;
    tcs.shape.z = (unsigned)v->nz;
    tcs.texpos.x = texpos[0];
    tcs.texpos.y = texpos[1];
    tcs.texpos.z = texpos[2];
    // strides in bytes of the (view, u, v) output, as the reference passes them
    refp::ulvec3 strides;
    strides.x = (unsigned long)nu * nv * sizeof(float);
    strides.y = (unsigned long)nv * sizeof(float);
    strides.z = sizeof(float);
    // flatpanel.py:1012-1022: 32 x 20 x 1 threads (fewer on a smaller detector)
    const unsigned bx = nu < 32u ? nu : 32u, by = nv < 20u ? nv : 20u;
    const dim3 block(bx, by, 1), grid((nu + bx - 1) / bx, (nv + by - 1) / by, n_views);
    refp::project_CB_texture_chunked<float, float><<<grid, block, 0, st>>>(
        cfg, static_cast<const refp::proj_spec *>(specs_dev), n_views, tcs, v->surf, false, strides, out_dev);
    return (int)cudaGetLastError();
}
