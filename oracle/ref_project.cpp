// ref_project.cpp -- the reference's projector kernels, compiled for the CPU.
//
// TEST INFRASTRUCTURE ONLY (checker and CPU baseline, never shipped): this
// file #includes src/aprict/data/cusrc/CB_project_texture_chunked.cu in place
// from the reference checkout (see oracle/Makefile) and drives its kernels one
// "thread" at a time under OpenMP:
//   * project_CB_texture_chunked<float,float> (:327-412) is called as is, with
//     blockDim = 1 and blockIdx = (iu, iv, view);
//   * project_CB_FORBILD_shapes needs >= 4 cooperating threads per block to
//     stage shapes (:441-460), so its per-thread body (:479-592) is restated
//     here around the reference's own FORBILD_clip_line_segment (FORBILD_volumes.h:1723-1811)
//     and exact_line_integral_prioritise_last (:1889-1954).
#include "ab_ref_prelude.h"
#include <cuda/atomic>
#include <cuda_fp16.h>

thread_local ab_dim3 threadIdx, blockIdx, blockDim;

namespace refp {
#include "CB_project_texture_chunked.cu"
}

extern "C" {

// Siddon projection of a C-order (X,Y,Z) float volume into out (M,nu,nv),
// contiguous float, accumulating. Returns the number of out-of-bounds surface
// accesses (0 expected).
long long ref_project_siddon(const void *specs, unsigned n_views, unsigned nu, unsigned nv, const float *vol,
                             unsigned nx, unsigned ny, unsigned nz, float voxwid, const float *texpos,
                             float svf, float mba, unsigned ssu, unsigned ssv, float *out, int nthreads) {
    ab_surface surf{(unsigned char *)vol, nz, ny, nx, sizeof(float), 0};
    refp::config_CB_project cfg;
    cfg.shrink_volume_factor = svf;
    cfg.multiply_before_adding = mba;
    cfg.ssu = ssu;
    cfg.ssv = ssv;
    refp::vol_tex_chunk_spec tcs;
    tcs.voxwid = voxwid;
    tcs.offsets = refp::uivec3(0, 0, 0);
    tcs.shape = refp::uivec3(nx, ny, nz);
    tcs.texpos = refp::fvec3(texpos[0], texpos[1], texpos[2]);
    const refp::ulvec3 strides((unsigned long)nu * nv * sizeof(float), (unsigned long)nv * sizeof(float),
                               sizeof(float));
    const refp::proj_spec *ps = (const refp::proj_spec *)specs;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (long long m = 0; m < (long long)n_views; ++m) {
        for (long long iu = 0; iu < (long long)nu; ++iu) {
            blockDim = ab_dim3{1, 1, 1};
            threadIdx = ab_dim3{0, 0, 0};
            for (unsigned iv = 0; iv < nv; ++iv) {
                blockIdx = ab_dim3{(unsigned)iu, iv, (unsigned)m};
                refp::project_CB_texture_chunked<float, float>(cfg, ps, n_views, tcs, (cudaSurfaceObject_t)&surf,
                                                               false, strides, out);
            }
        }
    }
    return surf.oob;
}

// Analytic projection of FORBILD shapes (reference struct layout, 156 bytes
// each) into out (M,nu,nv) float, accumulating. *overflow counts rays whose
// interval list overflowed (the reference's out_of_mem_count).
void ref_project_forbild(const void *specs, unsigned n_views, unsigned nu, unsigned nv, const void *shapes,
                         unsigned n_shapes, float mba, int overlap_addition, unsigned ssu, unsigned ssv, float *out,
                         unsigned *overflow, int nthreads) {
    const refp::proj_spec *ps = (const refp::proj_spec *)specs;
    const refp::FORBILD_Shape *sh = (const refp::FORBILD_Shape *)shapes;
    unsigned ovf = 0;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for collapse(2) schedule(dynamic, 4) reduction(+ : ovf)
    for (long long m = 0; m < (long long)n_views; ++m) {
        for (long long iu = 0; iu < (long long)nu; ++iu) {
            static thread_local refp::fvec2 intervals[MAX_INTERSECTIONS_PER_LINE];
            static thread_local float rhos[MAX_INTERSECTIONS_PER_LINE];
            const refp::proj_spec p = ps[m];
            const refp::fvec3 source_pos = p.sourcepos;
            const float idx_offx = 1 / ((float)ssu), idx_offy = 1 / ((float)ssv);
            for (unsigned iv = 0; iv < nv; ++iv) {
                bool out_of_mem_flag = false;
                float totval = 0;
                for (unsigned du = 0; du < ssu; du++) {
                    float accumulator = 0;
                    for (unsigned dv = 0; dv < ssv; dv++) {
                        const float fx = (float)iu - 0.5f + idx_offx * (du + 0.5f);
                        const float fy = (float)iv - 0.5f + idx_offy * (dv + 0.5f);
                        const refp::fvec3 det_pos = refp::detpos(p.dspec, fx, fy);
                        unsigned j = 0;
                        for (unsigned s = 0; s < n_shapes; ++s) {
                            const refp::fvec2 iv2 = refp::FORBILD_clip_line_segment(source_pos, det_pos, sh[s]);
                            if (iv2.x < iv2.y) {
                                if (j >= MAX_INTERSECTIONS_PER_LINE) {
                                    out_of_mem_flag = true;
                                } else {
                                    intervals[j] = iv2;
                                    rhos[j] = sh[s].rho;
                                    j++;
                                }
                            }
                        }
                        float val = 0;
                        if (overlap_addition) {
                            for (unsigned k = 0; k < j; k++) val += rhos[k] * (intervals[k].y - intervals[k].x);
                        } else {
                            val = refp::exact_line_integral_prioritise_last(source_pos, det_pos, intervals, rhos, j);
                        }
                        val *= mba;
                        accumulator += val;
                    }
                    if (ssv > 1) accumulator /= (float)ssv;
                    totval += accumulator;
                }
                if (ssu > 1) totval /= (float)ssu;
                if (out_of_mem_flag) ovf++;
                out[((size_t)m * nu + iu) * nv + iv] += totval;
            }
        }
    }
    if (overflow) *overflow += ovf;
}

// Interval [t0,t1] of one ray with one shape (FORBILD_clip_line_segment).
void ref_forbild_interval(const float *v1, const float *v2, const void *shape, float *out2) {
    const refp::FORBILD_Shape *s = (const refp::FORBILD_Shape *)shape;
    const refp::fvec2 r = refp::FORBILD_clip_line_segment(refp::fvec3(v1[0], v1[1], v1[2]),
                                                          refp::fvec3(v2[0], v2[1], v2[2]), *s);
    out2[0] = r.x;
    out2[1] = r.y;
}

// Bounding box of one shape (get_bbox(FORBILD_Shape), as used by
// get_bboxes_FORBILD.cu:8-20).
void ref_forbild_bbox(const void *shape, float *out6) {
    const refp::FORBILD_Shape *s = (const refp::FORBILD_Shape *)shape;
    const refp::bbox b = refp::get_bbox(*s);
    out6[0] = b.xyz_min.x;
    out6[1] = b.xyz_min.y;
    out6[2] = b.xyz_min.z;
    out6[3] = b.xyz_max.x;
    out6[4] = b.xyz_max.y;
    out6[5] = b.xyz_max.z;
}

// The per-voxel body of add_FORBILD_sampling (sample_FORBILD_volumes.cu:28-122)
// restated on the CPU around the reference's own _in_region(fvec3,
// FORBILD_Shape) (FORBILD_volumes.h:1626-): for each sub-sample the density
// of the last shape containing the point, the mean over sub-samples (the
// kernel's offsets, including its y <- offz, z <- offy order).
void ref_forbild_sample(const void *shapes, unsigned n, const float *xs, const float *ys, const float *zs,
                        unsigned nx, unsigned ny, unsigned nz, float ss_wid, unsigned ss, float *out, int nthreads) {
    const refp::FORBILD_Shape *sh = (const refp::FORBILD_Shape *)shapes;
#pragma omp parallel for collapse(2) schedule(dynamic, 4) num_threads(nthreads)
    for (unsigned i = 0; i < nx; ++i) {
        for (unsigned j = 0; j < ny; ++j) {
            for (unsigned k = 0; k < nz; ++k) {
                const refp::fvec3 pos_c(xs[i], ys[j], zs[k]);
                float totval = 0.f;
                for (unsigned ox = 0; ox < ss; ++ox)
                    for (unsigned oy = 0; oy < ss; ++oy)
                        for (unsigned oz = 0; oz < ss; ++oz) {
                            const refp::fvec3 pos = pos_c + refp::fvec3((ox - (ss - 1.f) / 2.f) / (float)ss,
                                                                        (oz - (ss - 1.f) / 2.f) / (float)ss,
                                                                        (oy - (ss - 1.f) / 2.f) / (float)ss) *
                                                                ss_wid;
                            float val = 0.f;
                            for (unsigned m = 0; m < n; ++m)
                                if (refp::_in_region(pos, sh[m])) val = sh[m].rho;
                            totval += val;
                        }
                out[((size_t)i * ny + j) * nz + k] = totval == 0.f ? 0.f : totval / (float)(ss * ss * ss);
            }
        }
    }
}

unsigned ref_sizeof_proj_spec(void) { return sizeof(refp::proj_spec); }
unsigned ref_sizeof_forbild_shape(void) { return sizeof(refp::FORBILD_Shape); }
}
