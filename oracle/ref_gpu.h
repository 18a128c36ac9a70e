// ref_gpu.h -- the reference's own GPU kernels, launched as the reference launches them.
//
// TEST INFRASTRUCTURE ONLY (the reference's GPU path, timed beside ours; never
// shipped): ref_gpu_project.cu and ref_gpu_backproject.cu #include the
// reference's src/aprict/data/cusrc/CB_project_texture_chunked.cu and
// CB_backproject.cu in place from the reference checkout (see oracle/Makefile)
// and compile them with nvcc for sm_100a into oracle/_ref/libaprict_refgpu.so.
// The host functions below reproduce the reference's launches
// (src/aprict/cb/flatpanel.py:997-1125 for the projection, :1128-1281 for the
// backprojection: 32 x 20 x 1 threads per block over (u, v, view); 8 x 8 x 8
// over the volume, one launch per 10 views with the chunk passed by value) and
// keep the volume, as the reference's Texture does, in a 3-D CUDA array behind
// a surface object (width = the fastest, z, axis of a C-order volume).
#pragma once

#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

// A C-order float volume (nx, ny, nz) in a CUDA array with a surface object.
typedef struct refgpu_vol refgpu_vol;

// Allocates the array and copies the C-order device buffer src (nx*ny*nz
// floats) into it; 0 on success, else a cudaError_t value.
int refgpu_vol_create(const float *src_dev, int nx, int ny, int nz, refgpu_vol **out);
// Copies the array back into / in from a C-order device buffer.
int refgpu_vol_read(const refgpu_vol *v, float *dst_dev, cudaStream_t st);
int refgpu_vol_write(refgpu_vol *v, const float *src_dev, cudaStream_t st);
void refgpu_vol_destroy(refgpu_vol *v);

// project_CB_texture_chunked<float,float> over n_views views of nu x nv pixels
// (specs_dev: 60-byte proj_spec records in device memory), accumulated
// atomically into out_dev (n_views, nu, nv) float, C order. texpos: the
// volume's corner (world). Returns the launch's cudaError_t.
int refgpu_project(const refgpu_vol *v, float voxwid, const float *texpos, const void *specs_dev,
                   unsigned n_views, unsigned nu, unsigned nv, float *out_dev, float svf, float mba,
                   unsigned ssu, unsigned ssv, cudaStream_t st);

// backproject_CB_voltex<float,float> in chunks of 10 views (the last spec
// repeated to fill a chunk), adding into the volume's surface; mult (nullable)
// is the summand multiplier's volume. specs_host: the proj_spec records in
// host memory (each chunk is passed by value). projs_dev: (n_views, nu, nv)
// float, C order. The configuration fields are the reference's
// config_CB_backproject fields. Returns the first launch error.
int refgpu_backproject(refgpu_vol *v, const refgpu_vol *mult, float voxwid, const float *texpos,
                       const void *specs_host, unsigned n_views, unsigned nu, unsigned nv, const float *projs_dev,
                       int exact, int all_ones, int mask, float mask_rad, float sep, int pL, int pV, float val,
                       int raycast, int linear, unsigned ssx, unsigned ssy, unsigned ssz, cudaStream_t st);

#ifdef __cplusplus
}
#endif
