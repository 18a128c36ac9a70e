// ref_backproject.cpp -- the reference's backprojector kernel, compiled for the CPU.
//
// TEST INFRASTRUCTURE ONLY (checker and CPU baseline, never shipped): this
// file #includes src/aprict/data/cusrc/CB_backproject.cu in place from the
// reference checkout (see oracle/Makefile) and calls
// backproject_CB_voltex<float,float> (:952-1027) once per voxel under OpenMP,
// in chunks of 10 views with the last view repeated to fill a chunk, exactly
// as flatpanel.backproject launches it (src/aprict/cb/flatpanel.py:1192-1278).
#include "ab_ref_prelude.h"
#include <cuda/atomic>
#include <cuda_fp16.h>

// exact_line_integral_backproject_fast (CB_backproject.cu:133-150) is dead
// code that names three undeclared variables; these declarations (never
// defined or used) let the file compile unchanged.
namespace refb {
struct fvec3;
extern fvec3 relvoxpos, dv2, minstepxyz;
}  // namespace refb

namespace refb {
#include "CB_backproject.cu"
}

extern "C" {

long long ref_backproject(const void *specs, unsigned n_views, unsigned nu, unsigned nv, const float *projs,
                          float *vol, unsigned nx, unsigned ny, unsigned nz, float voxwid, const float *texpos,
                          const float *mult, int exact, int all_ones, int mask, float mask_rad, float sep, int pL,
                          int pV, float val, int raycast, int linear, unsigned ssx, unsigned ssy, unsigned ssz,
                          int preset, int nthreads) {
    ab_surface surf{(unsigned char *)vol, nz, ny, nx, sizeof(float), 0};
    ab_surface msurf{(unsigned char *)mult, nz, ny, nx, sizeof(float), 0};
    refb::config_CB_backproject cfg{};
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
    cfg.backproj_weighting_preset = (unsigned char)preset;
    cfg.ssx = ssx;
    cfg.ssy = ssy;
    cfg.ssz = ssz;
    refb::vol_tex_chunk_spec tcs;
    tcs.voxwid = voxwid;
    tcs.offsets = refb::uivec3(0, 0, 0);
    tcs.shape = refb::uivec3(nx, ny, nz);
    tcs.texpos = refb::fvec3(texpos[0], texpos[1], texpos[2]);
    const refb::proj_spec *ps = (const refb::proj_spec *)specs;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    for (unsigned c0 = 0; c0 < n_views; c0 += 10) {
        refb::proj_chunk_spec_maxlen10 chunk;
        const unsigned cn = n_views - c0 < 10 ? n_views - c0 : 10;
        for (unsigned k = 0; k < 10; ++k) chunk.projspecs[k] = ps[c0 + (k < cn ? k : cn - 1)];
        chunk.numprojs = (unsigned char)cn;
        chunk.projmemaddr = (unsigned long)(projs + (size_t)c0 * nu * nv);
        chunk.projmemstrides = refb::ulvec3((unsigned long)nu * nv * sizeof(float), (unsigned long)nv * sizeof(float),
                                            sizeof(float));
#pragma omp parallel for collapse(2) schedule(dynamic, 2)
        for (long long x = 0; x < (long long)nx; ++x) {
            for (long long y = 0; y < (long long)ny; ++y) {
                blockDim = ab_dim3{1, 1, 1};
                threadIdx = ab_dim3{0, 0, 0};
                for (unsigned z = 0; z < nz; ++z) {
                    blockIdx = ab_dim3{(unsigned)x, (unsigned)y, z};
                    refb::backproject_CB_voltex<float, float>(cfg, tcs, (cudaSurfaceObject_t)&surf, false,
                                                              (cudaSurfaceObject_t)&msurf, false, chunk, 0, false);
                }
            }
        }
    }
    return surf.oob + msurf.oob;
}

// The reference's GBC kernel backproject_CB_voltex_GBC_cyl<float,float>
// (CB_backproject.cu:1030-1105), launched as flatpanel.backproject launches
// it for weighting preset 7: per chunk of 10 views, per voxel, the volume and
// the weight-sum volume both accumulated.
long long ref_backproject_gbc(const void *specs, unsigned n_views, unsigned nu, unsigned nv, const float *projs,
                              float *vol, float *vol2, unsigned nx, unsigned ny, unsigned nz, float voxwid,
                              const float *texpos, const float *mult, float R, int linear, unsigned ssx,
                              unsigned ssy, unsigned ssz, const float *soft, int nthreads) {
    ab_surface surf{(unsigned char *)vol, nz, ny, nx, sizeof(float), 0};
    ab_surface surf2{(unsigned char *)vol2, nz, ny, nx, sizeof(float), 0};
    ab_surface msurf{(unsigned char *)mult, nz, ny, nx, sizeof(float), 0};
    refb::config_CB_backproject cfg{};
    cfg.apply_summand_multiplier = mult != nullptr;
    cfg.Z_on_val_factor_val = R;
    cfg.approx_mode_direct_raycast = true;
    cfg.approx_mode_linear_interpolate = linear != 0;
    cfg.backproj_weighting_preset = 7;
    cfg.ssx = ssx;
    cfg.ssy = ssy;
    cfg.ssz = ssz;
    cfg.soft_vartheta_v = soft[0];
    cfg.soft_vartheta_v_softspan = soft[1];
    cfg.soft_vartheta_h = soft[2];
    cfg.soft_vartheta_h_softspan = soft[3];
    refb::vol_tex_chunk_spec tcs;
    tcs.voxwid = voxwid;
    tcs.offsets = refb::uivec3(0, 0, 0);
    tcs.shape = refb::uivec3(nx, ny, nz);
    tcs.texpos = refb::fvec3(texpos[0], texpos[1], texpos[2]);
    const refb::proj_spec *ps = (const refb::proj_spec *)specs;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    for (unsigned c0 = 0; c0 < n_views; c0 += 10) {
        refb::proj_chunk_spec_maxlen10 chunk;
        const unsigned cn = n_views - c0 < 10 ? n_views - c0 : 10;
        for (unsigned k = 0; k < 10; ++k) chunk.projspecs[k] = ps[c0 + (k < cn ? k : cn - 1)];
        chunk.numprojs = (unsigned char)cn;
        chunk.projmemaddr = (unsigned long)(projs + (size_t)c0 * nu * nv);
        chunk.projmemstrides = refb::ulvec3((unsigned long)nu * nv * sizeof(float), (unsigned long)nv * sizeof(float),
                                            sizeof(float));
#pragma omp parallel for collapse(2) schedule(dynamic, 2)
        for (long long x = 0; x < (long long)nx; ++x) {
            for (long long y = 0; y < (long long)ny; ++y) {
                blockDim = ab_dim3{1, 1, 1};
                threadIdx = ab_dim3{0, 0, 0};
                for (unsigned z = 0; z < nz; ++z) {
                    blockIdx = ab_dim3{(unsigned)x, (unsigned)y, z};
                    refb::backproject_CB_voltex_GBC_cyl<float, float>(cfg, tcs, (cudaSurfaceObject_t)&surf, false,
                                                                      (cudaSurfaceObject_t)&msurf, false, chunk,
                                                                      (cudaSurfaceObject_t)&surf2, false);
                }
            }
        }
    }
    return surf.oob + surf2.oob + msurf.oob;
}

// The reference's _GBC_weightfun<float> (CB_backproject.cu:736-787) at n points.
void ref_gbc_weight(float R, const float *vox, const float *src, const float *soft, long long n, float *out) {
    for (long long i = 0; i < n; ++i)
        out[i] = refb::_GBC_weightfun<float>(R, refb::fvec3(vox[3 * i], vox[3 * i + 1], vox[3 * i + 2]),
                                             refb::fvec3(src[3 * i], src[3 * i + 1], src[3 * i + 2]), soft[0], soft[2],
                                             soft[1], soft[3]);
}
}
