/*
 * aprict_b200.h -- C ABI of the B200 (sm_100a) cone-beam projection /
 * reconstruction kernels.
 *
 * Every entry point:
 *   - takes plain pointers and sizes (device pointers are marked *_dev),
 *   - enqueues work on the given CUDA stream (NULL = legacy default stream)
 *     and returns without synchronising,
 *   - allocates no device memory (the caller owns every buffer),
 *   - returns an aprict_status (0 = OK) after validating its arguments on the
 *     host; nothing is launched when the return value is nonzero.
 *
 * Operators ACCUMULATE into their output, as the reference's do
 * (project: atomicAdd in CB_project_texture_chunked.cu:411; backproject:
 * surface read-modify-write in CB_backproject.cu:1010-1015).
 *
 * Data layout (matches the reference's Python API, flatpanel.py:81-83 and
 * volume.py:133-145):
 *   - volume (X,Y,Z) float32, C order (z fastest) or F order (x fastest);
 *     voxel (i,j,k) centre = corner + voxwid*((i,j,k) + 0.5);
 *   - projections (views, nu, nv) float32 with arbitrary element strides;
 *     pixel (iu,iv) centre = det_pos + det_u*(iu-(nu-1)/2) + det_v*(iv-(nv-1)/2).
 */
#ifndef APRICT_B200_H
#define APRICT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *aprict_stream_t; /* a cudaStream_t */

#if defined(__GNUC__)
#define APRICT_API __attribute__((visibility("default")))
#else
#define APRICT_API
#endif

/* Host-side return codes. */
typedef enum {
    APRICT_OK = 0,
    APRICT_ERR_INVALID_ARGUMENT = 1, /* reference: ValueError (flatpanel.py:1141-1159) */
    APRICT_ERR_UNSUPPORTED = 2,      /* reference: NotImplementedError (flatpanel.py:247-255) */
    APRICT_ERR_CUDA = 3,             /* a CUDA runtime call failed */
    APRICT_ERR_TOO_LARGE = 4,        /* a size exceeds what the kernel indexes */
    APRICT_ERR_NO_DEVICE = 5         /* no usable sm_100 device */
} aprict_status;

/* Bits of the optional device status word (uint32) a kernel ORs into. */
#define APRICT_STATUS_OVERFLOW 0x1u     /* quadric interval list full (reference out_of_mem_count) */
#define APRICT_STATUS_NONFINITE 0x2u    /* a non-finite ray or voxel value was met */
#define APRICT_STATUS_BAD_GEOMETRY 0x4u /* degenerate view (zero-length detector vectors, ...) */
#define APRICT_STATUS_TIMEOUT 0x8u      /* a bounded wait gave up */

typedef struct {
    float x, y, z;
} aprict_fvec3;

/* One cone-beam view. Byte-identical to the reference's proj_spec
 * (geometry.h:1-13: fvec3 sourcepos; det_spec{pos,u,v,nu,nv,type}); 60 bytes. */
typedef struct {
    aprict_fvec3 source_pos;
    aprict_fvec3 det_pos; /* centre of the detector */
    aprict_fvec3 det_u;   /* pixel-centre step along a row (index iu) */
    aprict_fvec3 det_v;   /* pixel-centre step along a column (index iv) */
    uint32_t nu;
    uint32_t nv;
    uint8_t type; /* 0 = flat panel; anything else is rejected */
    uint8_t pad_[3];
} aprict_proj_spec;

/* Voxel grid. Replaces the reference's vol_tex_chunk_spec + surface object
 * (geometry.h:78-83): a linear device buffer instead of a cudaArray. */
typedef struct {
    uint32_t nx, ny, nz;
    uint32_t order; /* 0 = C order (z fastest), 1 = F order (x fastest) */
    float voxwid;
    aprict_fvec3 corner; /* world position of the outer corner of voxel (0,0,0) */
} aprict_vol_desc;

/* Projection stack (views, nu, nv); strides in ELEMENTS (the reference passes
 * byte strides as ulvec3(view,u,v), CB_project_texture_chunked.cu:366-370). */
typedef struct {
    uint32_t n_views, nu, nv, pad_;
    int64_t stride_view, stride_u, stride_v;
} aprict_proj_desc;

/* Same fields and layout as the reference's config_CB_project
 * (config_cb_project.h / geometry.h:94-99). */
typedef struct {
    float shrink_volume_factor;
    float multiply_before_adding;
    uint32_t ssu, ssv;
} aprict_project_config;

/* Fields of the reference's config_CB_backproject (geometry.h:108-128),
 * widened to 32-bit members. */
typedef struct {
    uint32_t exact;              /* exact_line_integ_backproj */
    uint32_t backproject_all_1s; /* exact mode only, as in the reference */
    uint32_t mask_to_cylinder;
    float mask_to_cyl_rad; /* world units, cylinder about world x=y=0 */
    uint32_t apply_summand_multiplier;
    float soften_edge_proportion;
    int32_t Z_on_L_factor_power;
    int32_t Z_on_val_factor_power;
    float Z_on_val_factor_val;
    uint32_t approx_mode_direct_raycast;
    uint32_t approx_mode_linear_interpolate;
    uint32_t weighting_preset; /* 0 plain, 1-6 cone-cylinder FBP weights, 7 GBC (backproject_gbc) */
    uint32_t ssx, ssy, ssz;
    float soft_vartheta_v, soft_vartheta_v_softspan;
    float soft_vartheta_h, soft_vartheta_h_softspan;
} aprict_backproject_config;

/* Human-readable text for an aprict_status code. */
APRICT_API const char *aprict_b200_status_string(int status);

/* Detail of the last nonzero status returned on the calling host thread. */
APRICT_API const char *aprict_b200_last_error(void);

/* Library version as "MAJOR.MINOR.PATCH". */
APRICT_API const char *aprict_b200_version(void);

/* Launch-shape knobs, process-wide (0 = built-in default). Keys:
 *   0 forward-projector tile height in pixels: 8, 16 or 32;
 *   1 backprojector voxels per thread along the slowest axis: 2, 4 or 8 (default 4, 2 in the exact mode);
 *   2 backprojector brick-order wave size in CTAs per SM: 1..16;
 *   3 forward-projector warp patch height (lanes along v): 8, 16 or 32;
 *   4 forward-projector views per detector tile: 1, 2 or 4 (default 4);
 *   5 forward-projector views inside one warp's patch: 1, 2 or 4;
 *   6 one-scan forward projector with one sub-ray per pixel: 0 specialised path (default), 1 general path;
 *   7 one-scan backprojector on C-order volumes: 0 z-column layout when the volume is tall enough (default), 1 never.
 * Set by the autotuner (aprict_b200/autotune.py); results never depend on them. */
APRICT_API int aprict_b200_set_tuning(int key, int value);
APRICT_API int aprict_b200_get_tuning(int key);

/* sizeof() of a struct declared here, by its type name (0 if unknown); lets
 * bindings verify their struct mirrors without a GPU. */
APRICT_API size_t aprict_b200_struct_size(const char *name);

/* Siddon exact line-integral forward projection of a voxel volume.
 * Replaces project_CB_texture_chunked<float,float>
 * (CB_project_texture_chunked.cu:327-412) as launched by
 * flatpanel.project (flatpanel.py:997-1125).
 *   specs_dev : n_views aprict_proj_spec in device memory
 *   base_dev  : NULL  -> projs += mba * A vol   (reference semantics, atomic)
 *               !NULL -> projs  = base + mba * A vol (fused residual; base may
 *                        equal projs_dev; same strides as projs)
 *   status_dev: optional device word (may be NULL)                        */
APRICT_API int aprict_b200_project_siddon(const aprict_proj_spec *specs_dev,
                               const aprict_proj_desc *projs, float *projs_dev,
                               const float *base_dev,
                               const aprict_vol_desc *vol, const float *vol_dev,
                               const aprict_project_config *cfg,
                               uint32_t *status_dev, aprict_stream_t stream);

/* Ray-driven matched adjoint of aprict_b200_project_siddon:
 * vol += A^T projs with exactly the forward projector's intersection lengths
 * (the same traversal code), scattered with atomic adds. No counterpart
 * kernel in the reference; it is the transpose the reference's exact
 * backprojector (CB_backproject.cu:408-477) approximates voxel by voxel. */
APRICT_API int aprict_b200_backproject_scatter(const aprict_proj_spec *specs_dev,
                                    const aprict_proj_desc *projs,
                                    const float *projs_dev,
                                    const aprict_vol_desc *vol, float *vol_dev,
                                    const aprict_project_config *cfg,
                                    uint32_t *status_dev,
                                    aprict_stream_t stream);

/* Voxel-driven backprojection (exact chord-length footprint or fast
 * nearest/bilinear), all views in one launch:
 * vol += multiplier * BP(projs). Replaces backproject_CB_voltex<float,float>
 * (CB_backproject.cu:952-1027, per-voxel body :313-733) and the host loop of
 * 10-view launches in flatpanel.backproject (flatpanel.py:1128-1281).
 *   multiplier_dev: required iff cfg->apply_summand_multiplier (same layout
 *                   as vol)                                               */
APRICT_API int aprict_b200_backproject(const aprict_proj_spec *specs_dev,
                            const aprict_proj_desc *projs,
                            const float *projs_dev,
                            const aprict_vol_desc *vol, float *vol_dev,
                            const float *multiplier_dev,
                            const aprict_backproject_config *cfg,
                            uint32_t *status_dev, aprict_stream_t stream);


/* ---- Element-wise volume operations (linear float32 buffers of n elements).
 * Replace the surface kernels of texture_operations.cu driven by
 * src/aprict/lib/texture_tools/operations.py. ---- */

/* v[:] = value (fill_surface, texture_operations.cu:124-135). */
APRICT_API int aprict_b200_vol_fill(float *v_dev, int64_t n, float value, aprict_stream_t stream);

/* v *= factor (multiply_surface, texture_operations.cu:187-199). */
APRICT_API int aprict_b200_vol_scale(float *v_dev, int64_t n, float factor, aprict_stream_t stream);

/* v <- 1/(v + eps*exp(-v/eps)) (eps > 0) or 1/v (eps == 0), zeros kept when
 * ignore_zeros (multiplicatively_invert_surface, texture_operations.cu:164-185). */
APRICT_API int aprict_b200_vol_invert(float *v_dev, int64_t n, int ignore_zeros, float eps,
                                      aprict_stream_t stream);

/* Cosine taper outside relrad_start of the inscribed xy circle about the
 * volume centre; relrad_start == 1 zeroes everything outside the circle
 * (softmask_surface_to_cylinder_xy, texture_operations.cu:137-162). */
APRICT_API int aprict_b200_vol_softmask_cylinder(float *v_dev, const aprict_vol_desc *vol,
                                                 float relrad_start, aprict_stream_t stream);

/* *out_dev += sum(a*b), accumulated in double (inner_product_3D_surfaces,
 * texture_operations.cu:284-307). The caller zeroes *out_dev. */
APRICT_API int aprict_b200_vol_dot(const float *a_dev, const float *b_dev, int64_t n, double *out_dev,
                                   aprict_stream_t stream);

/* out = a * b element-wise (multiply_surfaces, texture_operations.cu:309-). */
APRICT_API int aprict_b200_vol_mul(float *out_dev, const float *a_dev, const float *b_dev, int64_t n,
                                   aprict_stream_t stream);

/* out = a + alpha * b element-wise (out may alias a). */
APRICT_API int aprict_b200_vol_axpy(float *out_dev, const float *a_dev, float alpha, const float *b_dev,
                                    int64_t n, aprict_stream_t stream);

/* out = a / (w + eps exp(-w / eps)), the reciprocal taken first
 * (divide_surfaces_softzero, texture_operations.cu:333-351); eps <= 0 divides
 * plainly. out may alias a. */
APRICT_API int aprict_b200_vol_div_softzero(float *out_dev, const float *a_dev, const float *w_dev, int64_t n,
                                            float eps, aprict_stream_t stream);

/* v[x][y][z] *= grid[x * ny + y] for every z (Volume.multiply_by_xygrid,
 * volume.py:170-190). */
APRICT_API int aprict_b200_vol_mul_xygrid(float *v_dev, const aprict_vol_desc *vd, const float *grid_dev,
                                          aprict_stream_t stream);

/* ---- Ramp filtering ----
 * out[view][m][v] = scale * sum_j taps[m - j + nu - 1] * w[j][v] * in[view][j][v]
 * for m, j in [0, nu): the linear convolution the reference evaluates by
 * zero-padded cuFFT (RampFilterer._filter_chunk_axis1, ramp_filter.py:139-240)
 * after the cosine weighting of FBPFilterer (ramp_filter.py:407-449, :685-689).
 *   taps_dev      : 2*nu-1 floats, h[-(nu-1)] .. h[nu-1]
 *   odd_taps_only : nonzero if taps at even nonzero offsets are all zero (pure
 *                   Ram-Lak); halves the work
 *   weights_dev   : (nu, nv) per-pixel weights with element strides
 *                   (w_stride_u, w_stride_v), or NULL for none
 * in and out must not alias; nu <= 4096. */
APRICT_API int aprict_b200_ramp_filter(const aprict_proj_desc *in, const float *in_dev,
                                       const aprict_proj_desc *out, float *out_dev, const float *taps_dev,
                                       int odd_taps_only, const float *weights_dev, int64_t w_stride_u,
                                       int64_t w_stride_v, float scale, aprict_stream_t stream);

/* The same convolution by FFT, from tables built once per filter (the
 * reference's RampFilterer keeps the kernel spectrum, ramp_filter.py:83-137):
 * rows zero-padded to N = 2^p >= 2 nu - 1, two rows per complex transform,
 * forward transform in FP64, inverse in FP32. For 128 <= nu <= 2048.
 *   aprict_b200_ramp_fft_tables_bytes: bytes of the tables for rows of nu
 *       samples (32 N), 0 where nu is outside the FFT range
 *   aprict_b200_ramp_fft_tables: builds them from taps_dev (2*nu-1 floats)
 *       into tables_dev (16-byte aligned), enqueued on stream
 *   aprict_b200_ramp_filter_fft: aprict_b200_ramp_filter with the filter
 *       given by tables built for the same nu; same arguments otherwise */
APRICT_API int64_t aprict_b200_ramp_fft_tables_bytes(int64_t nu);
APRICT_API int aprict_b200_ramp_fft_tables(const float *taps_dev, int64_t nu, void *tables_dev,
                                           aprict_stream_t stream);
APRICT_API int aprict_b200_ramp_filter_fft(const aprict_proj_desc *in, const float *in_dev,
                                           const aprict_proj_desc *out, float *out_dev, const void *tables_dev,
                                           const float *weights_dev, int64_t w_stride_u, int64_t w_stride_v,
                                           float scale, aprict_stream_t stream);

/* Rotated bilinear resampling of a projection stack: the per-projection
 * rotations of the cone-cylinder FBP filter with its padding, weight mask,
 * letterbox and crop (FBPFilterer.filter_bulk_axis1_stream,
 * cb/ramp_filter.py:651-749 forward, :790-842 back; the rotations are
 * cupyx.scipy.ndimage.rotate(order=1, mode="grid-constant", reshape=False,
 * prefilter=False)). Both arrays live in one padded frame with rotation
 * centre (centre_u, centre_v); in[0][0] sits at (in_off_u, in_off_v) and
 * out[0][0] at (out_off_u, out_off_v). For view m and output pixel (i, j),
 * with p = (i + out_off_u, j + out_off_v) - centre and (c, s) = cs_dev[2m],
 * cs_dev[2m+1] (cosine and sine of the rotate() angle):
 *   q   = (c p_u + s p_v, -s p_u + c p_v) + centre - (in_off_u, in_off_v)
 *   x   = (float) bilinear(in[m], q)      FP64, neighbours outside in are 0
 *   x   = (float)(x * mask_dev[i * nv_out + j])      if mask_dev (FP64)
 *   out = (float)(x * colw_dev[m * nv_out + j])      if colw_dev (FP64)
 * cs_dev, mask_dev and colw_dev are device arrays; in and out must not alias. */
APRICT_API int aprict_b200_rotate_projections(const aprict_proj_desc *in, const float *in_dev,
                                              const aprict_proj_desc *out, float *out_dev, const double *cs_dev,
                                              double centre_u, double centre_v, int32_t in_off_u, int32_t in_off_v,
                                              int32_t out_off_u, int32_t out_off_v, const double *mask_dev,
                                              const double *colw_dev, aprict_stream_t stream);

/* ---- GBC reconstruction ---- */

/* GBC backprojection with a cylindrical source locus
 * (backproject_CB_voltex_GBC_cyl, CB_backproject.cu:736-905, 1030-1105; chosen
 * by flatpanel.backproject for weighting preset 7, flatpanel.py:216-232).
 * For every voxel and view: the weight w of _GBC_weightfun (R =
 * cfg->Z_on_val_factor_val, about the world z axis; soft windows from the
 * soft_vartheta_* fields), weightsum += w and, where w != 0, vol += w times
 * the nearest or bilinear detector value; both sums averaged over the
 * ssx*ssy*ssz sub-samples and multiplied by the summand multiplier. No
 * cylinder mask, taper or Z factors. cfg->weighting_preset must be 7;
 * weightsum_dev has the volume's layout and must not alias it. */
APRICT_API int aprict_b200_backproject_gbc(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                           const float *projs_dev, const aprict_vol_desc *vd, float *vol_dev,
                                           float *weightsum_dev, const float *multiplier_dev,
                                           const aprict_backproject_config *cfg, uint32_t *status_dev,
                                           aprict_stream_t stream);

/* out_dev[r] += the expected GBC weight sum at radius r_on_R_dev[r] (units of
 * R, increasing) over a perfect cylindrical locus sampled by num_z heights and
 * num_ang angles (get_GBC_weight_integ, CB_backproject.cu:1108-1168;
 * gbc/weightinteg.py:22-57). The caller zeroes out_dev (FP64). */
APRICT_API int aprict_b200_gbc_weight_integral(const float *r_on_R_dev, int32_t n_r, double *out_dev, int32_t num_z,
                                               int32_t num_ang, const aprict_backproject_config *cfg,
                                               aprict_stream_t stream);

/* In place on the (n0, n1, n2/2+1) complex64 rfftn spectrum of an (n0, n1,
 * n2) volume (axis 2 the cylinder axis): times multiplier * |k|, divided by
 * the softened Colsher k-factor of the polar angle (cone_angle in (0, pi);
 * 2 pi at cone_angle = pi; lateral |k| and no k-factor at cone_angle = 0),
 * times sinc(f0) sinc(f1) sinc(f2), DC set to 0 (ramp_filter_conebeam,
 * gbc/filters.py:59-147, 340-398). */
APRICT_API int aprict_b200_conebeam_spectral(void *spec_dev, int32_t n0, int32_t n1, int32_t n2, double multiplier,
                                             double cone_angle, double theta_soft, aprict_stream_t stream);

/* out[x][y][z] += order-1 interpolation of low (m0, m1, m2) at
 * (x, y, z) / factor - 1/2 + 1/(2 factor), neighbour indices clamped
 * (map_coordinates mode "nearest"; the low-resolution correction of
 * ramp_filter_conebeam, gbc/filters.py:403-455). Both C order. */
APRICT_API int aprict_b200_add_upsampled(float *out_dev, int32_t n0, int32_t n1, int32_t n2, const float *low_dev,
                                         int32_t m0, int32_t m1, int32_t m2, int32_t factor, aprict_stream_t stream);

/* ---- Analytic (FORBILD) phantoms ---- */

/* One clipping half-space (FORBILD_ClipAxisSpec, FORBILD_volumes.h:89-155):
 * mode 0 = off, 1 = keep p.axis <= dotprod, 2 = keep p.axis > dotprod. */
typedef struct {
    aprict_fvec3 axis;
    float dotprod;
    uint8_t mode;
    uint8_t pad_[3];
} aprict_forbild_clip;

/* One FORBILD shape, byte-identical to the reference's FORBILD_Shape
 * (FORBILD_volumes.h:1395-1415; type map src/aprict/cuda/structs/FORBILD_volumes.py:517-534):
 * 1 Box, 2-5 Cone/_x/_y/_z, 6-9 Cylinder/_x/_y/_z, 10 Ellipsoid,
 * 11 Ellipsoid_free, 12 Ellipt_Cyl, 13 Sphere, 14-16 Ellipt_Cyl_x/_y/_z;
 * 0 = no shape. 156 bytes. */
typedef struct {
    uint8_t type;
    uint8_t pad_[3];
    float rho;
    aprict_forbild_clip cas1, cas2, cas3;
    float x, y, z, dx, dy, dz, r, r1, r2, l;
    aprict_fvec3 a_x, a_y, a_z, axis;
} aprict_forbild_shape;

/* A shape reduced (in FP64, on the host) to an affine map onto a canonical
 * solid: local = M (p - c);
 *   kind 1: |local| <= 1                       (ellipsoids, spheres)
 *   kind 2: lx^2+ly^2 <= 1, |lz| <= h           (cylinders)
 *   kind 3: lx^2+ly^2 <= (alpha+beta lz)^2, |lz| <= h   (cone frusta)
 *   kind 4: |lx|,|ly|,|lz| <= 1                 (boxes)
 * clipped by g_k(p) = clip[k].xyz . p - clip[k].w <= 0 for k < (n_clip & 0xFF);
 * bit 8 + k of n_clip marks clip k as strict (< 0: the FORBILD ">" planes). */
typedef struct {
    int32_t kind;
    int32_t n_clip;
    double rho;
    double c[3];
    double M[9]; /* row-major */
    double h, alpha, beta;
    double clip[3][4];
    double bb_half[3]; /* half extents of the world AABB about c */
} aprict_quadric;

/* Host function (no device work): compile n FORBILD shapes into
 * aprict_quadric records. Null shapes (type 0) compile to kind 0. Returns
 * APRICT_ERR_INVALID_ARGUMENT for an unknown type or degenerate parameters. */
APRICT_API int aprict_b200_forbild_compile(const aprict_forbild_shape *shapes_host, int64_t n,
                                           aprict_quadric *out_host);

/* Analytic projection of compiled shapes, accumulated into projs
 * (project_CB_FORBILD_shapes, CB_project_texture_chunked.cu:415-593):
 *   mode 0: later shapes override earlier ones (the reference default,
 *           exact_line_integral_prioritise_last, FORBILD_volumes.h:1889-1954);
 *   mode 1: additive, sum rho * dt with dt the parametric chord on the
 *           source->pixel segment (the reference's overlap_addition, :556-560,
 *           which does not multiply by the segment length);
 *   mode 2: additive line integral, sum rho * dt * |segment|.
 * Entry/exit parameters are solved in FP64. Each CTA culls the shapes against
 * its detector tile first. overflow_dev (optional) counts rays whose covered
 * interval list overflowed in mode 0 (the reference's out_of_mem_count). */
APRICT_API int aprict_b200_project_forbild(const aprict_proj_spec *specs_dev, const aprict_proj_desc *projs,
                                           float *projs_dev, const aprict_quadric *shapes_dev, int64_t n_shapes,
                                           float multiply_before_adding, uint32_t ssu, uint32_t ssv, int mode,
                                           uint32_t *overflow_dev, uint32_t *status_dev, aprict_stream_t stream);

/* ---- SIRT (reference mode) ----
 * One iteration of SIRT_flatpanel (sirt_vram.py:130-152) as two launches on
 * the stream: r = b - A x (fused residual), then x += M (.) B r with cfg_bp
 * (which must apply the summand multiplier M). b, r: projection stacks with
 * the layout of pd; x, M: volumes of vd. */
APRICT_API int aprict_b200_sirt_step(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                     const float *b_dev, float *r_dev, const aprict_vol_desc *vd, float *x_dev,
                                     const float *M_dev, const aprict_backproject_config *cfg_bp,
                                     uint32_t *status_dev, aprict_stream_t stream);

/* n_iter SIRT steps captured once as a CUDA graph (on a private stream) and
 * replayed with aprict_b200_sirt_graph_launch. The graph records the
 * pointers and settings given here. The kernels must already be loaded when
 * it is created: run one aprict_b200_sirt_step (or any projection and
 * backprojection) in the process first. */
typedef struct aprict_sirt_graph aprict_sirt_graph;
APRICT_API int aprict_b200_sirt_graph_create(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                             const float *b_dev, float *r_dev, const aprict_vol_desc *vd,
                                             float *x_dev, const float *M_dev,
                                             const aprict_backproject_config *cfg_bp, uint32_t *status_dev,
                                             int n_iter, aprict_sirt_graph **out);
APRICT_API int aprict_b200_sirt_graph_launch(const aprict_sirt_graph *graph, aprict_stream_t stream);
APRICT_API int aprict_b200_sirt_graph_iterations(const aprict_sirt_graph *graph);
APRICT_API void aprict_b200_sirt_graph_destroy(aprict_sirt_graph *graph);

/* ---- Many scans in one persistent launch ----
 * No reference counterpart (the reference runs one scan per call). A batch is
 * a plan built on the host from per-scan arguments -- exactly the arguments
 * of one aprict_b200_project_siddon / aprict_b200_backproject call each -- and
 * copied by the caller to device memory; aprict_b200_batch_run then performs
 * every scan's operation in one launch whose CTAs pull detector tiles (project)
 * or volume bricks (backproject) of all scans from a counter kept in the plan.
 * Each scan's result equals that of its one-scan call. */
enum { APRICT_BATCH_PROJECT = 0, APRICT_BATCH_BACKPROJECT = 1 };

typedef struct {
    const aprict_proj_spec *specs_dev;
    aprict_proj_desc projs;
    float *projs_dev;            /* project: output; backproject: input */
    const float *base_dev;       /* project only: NULL = accumulate, else fused residual base */
    aprict_vol_desc vol;
    float *vol_dev;              /* project: input; backproject: output */
    const float *multiplier_dev; /* backproject only: iff the scan's config applies one */
    uint32_t *status_dev;        /* optional */
} aprict_scan;

/* Bytes a plan of n_scans needs (0 for an invalid op or count). */
APRICT_API size_t aprict_b200_batch_plan_bytes(int op, int n_scans);

/* Validate the scans (as the one-scan calls would) and write the plan into
 * plan_host (256-byte aligned, plan_capacity >= plan_bytes). Enqueues no
 * device work; it queries the current device (multiprocessor count and
 * occupancy, which also loads the kernels, so a later run inside a stream
 * capture loads nothing).
 * configs points to n_scans aprict_project_config (op PROJECT) or
 * aprict_backproject_config (op BACKPROJECT); a backprojection batch needs
 * the same volume order and mode (exact / fast / raycast, nearest /
 * bilinear) in every scan. The plan records the device pointers given here. */
APRICT_API int aprict_b200_batch_plan(int op, const aprict_scan *scans, int n_scans, const void *configs,
                                      void *plan_host, size_t plan_capacity);

/* Run a plan: plan_dev is a byte copy of plan_host in device memory (256-byte
 * aligned). The work counters in plan_dev must be zero before the first run
 * (they are in a fresh copy); each run leaves them zero again, so the same
 * plan_dev can be run repeatedly or captured in a CUDA graph. Two runs of one
 * plan_dev must not overlap in time (they would share its counters). A batch
 * of more than 96 scans runs as one launch per 96 scans. */
APRICT_API int aprict_b200_batch_run(const void *plan_host, void *plan_dev, aprict_stream_t stream);

/* aprict_b200_batch_run for callers that cannot allocate device memory (no
 * counterpart in the reference). The plan's work counters live in a static
 * 8 KB device array of the library instead of a caller copy of the plan, so
 * the caller passes only the host plan: nothing is allocated, copied from
 * the host, or freed. The counters are cleared (an asynchronous memset on
 * the stream) at every call. Limits: at most 15 launch groups (1440 scans)
 * per plan, else APRICT_ERR_TOO_LARGE; the first call on each device looks
 * the array up (cudaGetSymbolAddress, which may load the module), so make it
 * before any stream capture; calls that overlap in time on one device share
 * the array and race, so serialise them (one stream, or events). After a
 * device reset the cached address is stale: the next call finds its clearing
 * memset refused and looks the array up again. */
APRICT_API int aprict_b200_batch_run_static(const void *plan_host, aprict_stream_t stream);

/* Point-sample compiled shapes onto a grid, "last shape wins"
 * (add_FORBILD_sampling, sample_FORBILD_volumes.cu:10-123): for voxel
 * (i, j, k) at (xs[i], ys[j], zs[k]) and each of supersamp_factor^3
 * sub-samples spaced supersamp_voxwid / supersamp_factor apart around it, the
 * density of the last shape containing the point (0 if none); the mean is
 * added to out[i*stride_x + j*stride_y + k*stride_z]. Entry tests in FP64. */
APRICT_API int aprict_b200_forbild_sample(const aprict_quadric *shapes_dev, int64_t n_shapes, const float *xs_dev,
                                          const float *ys_dev, const float *zs_dev, uint32_t nx, uint32_t ny,
                                          uint32_t nz, int64_t stride_x, int64_t stride_y, int64_t stride_z,
                                          float *out_dev, float supersamp_voxwid, uint32_t supersamp_factor,
                                          aprict_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* APRICT_B200_H */
