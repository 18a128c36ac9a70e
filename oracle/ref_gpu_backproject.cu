// ref_gpu_backproject.cu -- the reference's backprojector kernel on the GPU (see ref_gpu.h).
//
// TEST INFRASTRUCTURE ONLY. Includes src/aprict/data/cusrc/CB_backproject.cu in
// place from the reference checkout, with the same reading of uint3 as
// ref_gpu_project.cu. One dead template of that file
// (exact_line_integral_backproject_fast, :133-150, never instantiated) names
// three undeclared variables; the declarations below (never defined or used)
// let it compile unchanged.
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
namespace refg {
struct fvec3;
extern fvec3 relvoxpos, dv2, minstepxyz;
#include "CB_backproject.cu"
}  // namespace refg
#undef uint3

static_assert(sizeof(refg::proj_spec) == 60, "proj_spec is the 60-byte record");

extern "C" cudaSurfaceObject_t refgpu_vol_surface(const refgpu_vol *v);
extern "C" void refgpu_vol_shape(const refgpu_vol *v, int *n);

extern "C" int refgpu_backproject(refgpu_vol *v, const refgpu_vol *mult, float voxwid, const float *texpos,
                                  const void *specs_host, unsigned n_views, unsigned nu, unsigned nv,
                                  const float *projs_dev, int exact, int all_ones, int mask, float mask_rad,
                                  float sep, int pL, int pV, float val, int raycast, int linear, unsigned ssx,
                                  unsigned ssy, unsigned ssz, cudaStream_t st) {
    if (n_views == 0 || nu == 0 || nv == 0) return 0;
    int n[3];
    refgpu_vol_shape(v, n);
    if (mult) {
        int m[3];
        refgpu_vol_shape(mult, m);
        if (m[0] != n[0] || m[1] != n[1] || m[2] != n[2]) return (int)cudaErrorInvalidValue;
    }
    refg::config_CB_backproject cfg{};
    cfg.exact_line_integ_backproj = exact != 0;
    cfg.backproject_all_1s = all_ones != 0;
    cfg.mask_to_cylinder = mask != 0;
    cfg.mask_to_cyl_rad = mask_rad;
    cfg.apply_summand_multiplier = mult != nullptr;
    cfg.soften_edge_proportion = sep;
    cfg.Z_on_L_factor_power = pL;
    cfg.Z_on_val_factor_power = pV;
    cfg.Z_on_val_factor_val = val;
    cfg.approx_mode_direct_raycast = raycast != 0;
    cfg.approx_mode_linear_interpolate = linear != 0;
    cfg.backproj_weighting_preset = 0;
    cfg.ssx = ssx;
    cfg.ssy = ssy;
    cfg.ssz = ssz;
    refg::vol_tex_chunk_spec tcs;
    tcs.voxwid = voxwid;
    tcs.offsets.x = tcs.offsets.y = tcs.offsets.z = 0;
    tcs.shape.x = (unsigned)n[0];
    tcs.shape.y = (unsigned)n[1];
    tcs.shape.z = (unsigned)n[2];
    tcs.texpos.x = texpos[0];
    tcs.texpos.y = texpos[1];
    tcs.texpos.z = texpos[2];
    // flatpanel.py:1162-1170: 8 x 8 x 8 threads over the volume's (x, y, z) indices
    const unsigned bx = n[0] < 8 ? n[0] : 8, by = n[1] < 8 ? n[1] : 8, bz = n[2] < 8 ? n[2] : 8;
    const dim3 block(bx, by, bz), grid((n[0] + bx - 1) / bx, (n[1] + by - 1) / by, (n[2] + bz - 1) / bz);
    const refg::proj_spec *ps = static_cast<const refg::proj_spec *>(specs_host);
    const cudaSurfaceObject_t surf = refgpu_vol_surface(v), msurf = refgpu_vol_surface(mult);
    // flatpanel.py:1192-1278: one launch per 10 views, the last spec repeated to fill the chunk
    for (unsigned c0 = 0; c0 < n_views; c0 += 10) {
        refg::proj_chunk_spec_maxlen10 chunk;
        const unsigned cn = n_views - c0 < 10 ? n_views - c0 : 10;
        for (unsigned k = 0; k < 10; ++k) chunk.projspecs[k] = ps[c0 + (k < cn ? k : cn - 1)];
        chunk.numprojs = (unsigned char)cn;
        chunk.projmemaddr = (unsigned long)(projs_dev + (size_t)c0 * nu * nv);
        chunk.projmemstrides.x = (unsigned long)nu * nv * sizeof(float);
        chunk.projmemstrides.y = (unsigned long)nv * sizeof(float);
        chunk.projmemstrides.z = sizeof(float);
        refg::backproject_CB_voltex<float, float><<<grid, block, 0, st>>>(cfg, tcs, surf, false, msurf, false, chunk,
                                                                          0, false);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return (int)e;
    }
    return 0;
}
