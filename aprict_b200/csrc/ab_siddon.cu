// ab_siddon.cu -- Siddon forward projector and its ray-driven matched adjoint
// (one scan per launch). The forward work unit lives in ab_fptile.cuh.
#include <cuda_runtime.h>

#include "ab_fptile.cuh"

namespace {

using namespace ab_fp;

// Projector kernels over linear tile indices (used when the tile counts do
// not fit a 3-D grid).
template <typename Off, bool SS1>
__global__ void __launch_bounds__(kThreads, 4) k_project_siddon(const FPScan<Off> S) {
    fp_tile<Off, SS1>(S, blockIdx.x);
}

// The same with the tile given by a 3-D grid (x: column tile, y: view group,
// z: row band; the hardware issues blocks in that linear order), which saves
// the per-thread division of a linear block index. With one sub-ray per pixel
// the specialised ray path runs (no spills; 12.35 ms against 13.25 ms for the
// general path on the 256^3 x 360-view fused residual, bit-identical results),
// at 5 resident CTAs per SM (48 registers, no spills: 9.93 against 10.20 ms at
// 4); tuning knob 6 = 1 forces the general path.
template <typename Off, bool SS1>
__global__ void __launch_bounds__(kThreads, fp_min_blocks(SS1)) k_project_siddon_3d(const FPScan<Off> S) {
    int view, iu, iv;
    if (!tile_thread(S.tm, S.n_views, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, view, iu, iv) ||
        iu >= (int)S.nu || iv >= (int)S.nv)
        return;
    fp_ray<Off, SS1>(S, view, iu, iv);
}

template <typename Off>
int launch_project(const FPScan<Off> &S, uint64_t nblocks, cudaStream_t st) {
    const TileMap &tm = S.tm;
    const bool ss1 = S.ssu == 1 && S.ssv == 1;
    if (tm.ntw <= 65535 && tm.ntv <= 65535 && tm.ntu <= 0x7fffffff) {
        const dim3 grid((unsigned)tm.ntu, (unsigned)tm.ntw, (unsigned)tm.ntv);
        if (ss1 && ab_tuning_get(AB_TUNE_FP_SS1) == 0)
            k_project_siddon_3d<Off, true><<<grid, kThreads, 0, st>>>(S);
        else
            k_project_siddon_3d<Off, false><<<grid, kThreads, 0, st>>>(S);
    } else {
        if (nblocks > 0x7fffffffull) return ab_fail(APRICT_ERR_TOO_LARGE, "too many detector tiles");
        k_project_siddon<Off, false><<<(unsigned)nblocks, kThreads, 0, st>>>(S);
    }
    return APRICT_OK;
}

template <typename Off>
__global__ void __launch_bounds__(kThreads, 4)
    k_backproject_scatter(const aprict_proj_spec *__restrict__ specs, uint32_t n_views, uint32_t nu, uint32_t nv,
                          ab_pstrides ps, const float *__restrict__ projs, ab_grid<Off> g, float *vol, float svf,
                          float mba, int ssu, int ssv, TileMap tm, uint32_t *status, int one) {
    int view, iu, iv;
    if (!block_tile(tm, n_views, blockIdx.x, view, iu, iv) || iu >= (int)nu || iv >= (int)nv) return;
    const int64_t o = (int64_t)view * ps.view + (int64_t)iu * ps.u + (int64_t)iv * ps.v;
    const float p = projs[o];
    if (p == 0.f) return;
    const aprict_proj_spec sp = specs[view];
    const ab_d3 src = ab_to_grid(g, ab_d3_of(sp.source_pos) * (double)svf);
    // Transpose of: out = (1/ssu) sum_ku (1/ssv) sum_kv mba * voxwid * sum_seg seg*mu
    const float w = p * mba * g.voxwid / (float)(ssu * ssv);
    bool bad = false;
    const double inv_su = 1.0 / (double)ssu, inv_sv = 1.0 / (double)ssv;
    for (int ku = 0; ku < ssu; ++ku) {
        for (int kv = 0; kv < ssv; ++kv) {
            const double fu = (double)iu - 0.5 + inv_su * (ku + 0.5);
            const double fv = (double)iv - 0.5 + inv_sv * (kv + 0.5);
            const ab_d3 dst = ab_to_grid(g, ab_pixel_pos(sp, fu, fv) * (double)svf);
            ab_siddon_scatter<Off>(src, dst, g.n, g.stride, vol, w, &bad, one);
        }
    }
    if (bad && status) atomicOr(status, APRICT_STATUS_NONFINITE);
}

}  // namespace

extern "C" int aprict_b200_project_siddon(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                          float *projs_dev, const float *base_dev, const aprict_vol_desc *vd,
                                          const float *vol_dev, const aprict_project_config *cfg,
                                          uint32_t *status_dev, aprict_stream_t stream) {
    int rc = fp_check(specs_dev, pd, projs_dev, vd, vol_dev, cfg);
    if (rc != APRICT_OK) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    uint64_t nblocks = 0;
    if (small_volume(vd)) {
        const FPScan<int32_t> S =
            make_fpscan<int32_t>(specs_dev, pd, projs_dev, base_dev, vd, vol_dev, cfg, status_dev, nblocks);
        if (nblocks == 0) return APRICT_OK;
        rc = launch_project<int32_t>(S, nblocks, st);
    } else {
        const FPScan<int64_t> S =
            make_fpscan<int64_t>(specs_dev, pd, projs_dev, base_dev, vd, vol_dev, cfg, status_dev, nblocks);
        if (nblocks == 0) return APRICT_OK;
        rc = launch_project<int64_t>(S, nblocks, st);
    }
    if (rc != APRICT_OK) return rc;
    return ab_cuda_check(cudaGetLastError(), "project_siddon launch");
}

extern "C" int aprict_b200_backproject_scatter(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                               const float *projs_dev, const aprict_vol_desc *vd, float *vol_dev,
                                               const aprict_project_config *cfg, uint32_t *status_dev,
                                               aprict_stream_t stream) {
    int rc = fp_check(specs_dev, pd, projs_dev, vd, vol_dev, cfg);
    if (rc != APRICT_OK) return rc;
    if (pd->n_views == 0 || pd->nu == 0 || pd->nv == 0) return APRICT_OK;
    const TileMap tm = make_tiles(pd->nu, pd->nv, pd->n_views);
    const ab_pstrides ps{pd->stride_view, pd->stride_u, pd->stride_v};
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const uint64_t nblocks = tm.units();
    if (nblocks > 0x7fffffffull) return ab_fail(APRICT_ERR_TOO_LARGE, "too many detector tiles");
    if (small_volume(vd)) {
        k_backproject_scatter<int32_t><<<(unsigned)nblocks, kThreads, 0, st>>>(
            specs_dev, pd->n_views, pd->nu, pd->nv, ps, projs_dev, ab_make_grid<int32_t>(*vd), vol_dev,
            cfg->shrink_volume_factor, cfg->multiply_before_adding, (int)cfg->ssu, (int)cfg->ssv, tm, status_dev, 1);
    } else {
        k_backproject_scatter<int64_t><<<(unsigned)nblocks, kThreads, 0, st>>>(
            specs_dev, pd->n_views, pd->nu, pd->nv, ps, projs_dev, ab_make_grid<int64_t>(*vd), vol_dev,
            cfg->shrink_volume_factor, cfg->multiply_before_adding, (int)cfg->ssu, (int)cfg->ssv, tm, status_dev, 1);
    }
    return ab_cuda_check(cudaGetLastError(), "backproject_scatter launch");
}
