/* ab_oracle.h -- FP64 CPU restatement of the reference's projection /
 * backprojection arithmetic. TEST INFRASTRUCTURE ONLY: used by tests/,
 * __graft_entry__.smoke() and bench.py's CPU baseline as the checker; the
 * aprict_b200 package never loads it. */
#ifndef AB_ORACLE_H
#define AB_ORACLE_H
#include <stdint.h>

typedef struct {
    float x, y, z;
} ao_fvec3;

/* Same 60-byte layout as the reference's proj_spec (geometry.h:1-13). */
typedef struct {
    ao_fvec3 source_pos, det_pos, det_u, det_v;
    uint32_t nu, nv;
    uint8_t type, pad_[3];
} ao_proj_spec;

typedef struct {
    int nx, ny, nz;
    int order; /* 0 = C (z fastest), 1 = F (x fastest) */
    double voxwid;
    double corner[3];
} ao_grid;

typedef struct {
    int exact, all_ones, mask;
    double mask_rad, sep;
    int pL, pV;
    double val;
    int raycast, linear;
    int ssx, ssy, ssz;
    int preset; /* direct-raycast weighting preset 0-6 (CB_backproject.cu:530-599) */
} ao_bp_cfg;

/* out[m,iu,iv] += mba * line integrals (ssu x ssv sub-rays averaged),
 * following project_CB_texture_chunked (CB_project_texture_chunked.cu:327-412).
 * nseg (optional) receives the number of positive-length ray/voxel segments. */
void ao_project_siddon(const ao_proj_spec *specs, int n_views, int nu, int nv, const float *vol, const ao_grid *g,
                       double svf, double mba, int ssu, int ssv, double *out, int64_t *nseg, int nthreads);

/* vol += A^T projs for the operator above (exact transpose, FP64). */
void ao_backproject_transpose(const ao_proj_spec *specs, int n_views, int nu, int nv, const double *projs,
                              const ao_grid *g, double svf, double mba, int ssu, int ssv, double *vol,
                              int nthreads);

/* vol += mult * BP(projs), the voxel-driven backprojector of
 * _backproject_CB_getval (CB_backproject.cu:313-733), presets 0-6, in FP64. */
/* Per voxel: fast-nearest (sub-sample, view) pairs whose pixel choice lies within eps of a tie. */
void ao_bp_nearest_ties(const ao_proj_spec *specs, int n_views, const ao_grid *g, const ao_bp_cfg *c, double eps,
                        int32_t *counts, int nthreads);
void ao_backproject(const ao_proj_spec *specs, int n_views, int nu, int nv, const double *projs,
                    const ao_grid *g, const double *mult, const ao_bp_cfg *cfg, double *vol, int nthreads);

/* Reference layout of FORBILD_Shape (FORBILD_volumes.h:1395-1415), 156 bytes. */
typedef struct {
    ao_fvec3 axis;
    float dotprod;
    uint8_t mode, pad_[3];
} ao_clip;
typedef struct {
    uint8_t type, pad_[3];
    float rho;
    ao_clip cas[3];
    float x, y, z, dx, dy, dz, r, r1, r2, l;
    ao_fvec3 a_x, a_y, a_z, axis;
} ao_forbild_shape;

/* out[m,iu,iv] += mba * analytic projection of the shapes (FP64):
 * mode 0 later shapes win (x |segment|), 1 sum rho*dt, 2 sum rho*dt*|segment|
 * (project_CB_FORBILD_shapes, CB_project_texture_chunked.cu:415-593). */
void ao_project_forbild(const ao_proj_spec *specs, int n_views, int nu, int nv, const ao_forbild_shape *shapes,
                        int n_shapes, double mba, int mode, int ssu, int ssv, double *out, int nthreads);

/* Interval [t0,t1] of the segment v1->v2 with one shape (after clipping), FP64. */
int ao_forbild_interval(const double v1[3], const double v2[3], const ao_forbild_shape *s, double out2[2]);
int ao_forbild_inside(const double p[3], const ao_forbild_shape *s);
void ao_forbild_sample(const ao_forbild_shape *shapes, int n, const double *xs, const double *ys, const double *zs,
                       int nx, int ny, int nz, double ss_wid, int ss, double *out, int nthreads);

#endif
