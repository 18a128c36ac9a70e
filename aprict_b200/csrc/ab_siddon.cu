// ab_siddon.cu -- Siddon forward projector and its ray-driven matched adjoint.
//
// Forward: replaces project_CB_texture_chunked<float,float>
// (src/aprict/data/cusrc/CB_project_texture_chunked.cu:327-412). One thread
// per (view, pixel); ssu x ssv sub-rays averaged as in :381-407; result
// scaled by multiply_before_adding (:394) and accumulated (:411).
//
// B200 layout: a CTA covers a 2-D detector tile of one view and each warp a
// 4 (u) x 8 (v) pixel patch (2 x 16 or 1 x 32 as tuned), so the rays of a warp are spatially coherent and
// their voxel gathers hit the same L1 lines; 8 consecutive v per row make the
// output access one 32-byte sector.
#include <cuda_runtime.h>

#include "ab_common.cuh"
#include "ab_host.h"

namespace {

constexpr int kThreads = 256;

struct TileMap {
    int tile_u, tile_v;  // tile extents in pixels
    int warp_v;          // lanes of a warp along v (warp patch: 32/warp_v along u)
    int ntu, ntv;        // number of tiles along u, v
};

// Tile shapes: tv == 1 -> one detector row per tile (used when nv < 8);
// otherwise warps are 4 (u) x 8 (v) patches.
TileMap make_tiles(uint32_t nu, uint32_t nv) {
    TileMap t;
    t.tile_v = nv >= 16 ? 16 : (nv >= 8 ? 8 : 1);
    const int want = ab_tuning_get(AB_TUNE_FP_TILE_V);  // autotuner override: 8, 16 or 32
    if ((want == 8 || want == 16 || want == 32) && nv >= 8) t.tile_v = want;
    // Warp patch: 4 (u) x 8 (v) by default; the autotuner may try 2 x 16 or 1 x 32.
    const int wv = ab_tuning_get(AB_TUNE_FP_WARP_V);
    t.warp_v = (wv == 16 || wv == 32) ? wv : 8;
    if (t.tile_v > 1 && t.warp_v > t.tile_v) t.tile_v = t.warp_v;
    t.tile_u = kThreads / t.tile_v;
    t.ntu = (int)((nu + t.tile_u - 1) / t.tile_u);
    t.ntv = (int)((nv + t.tile_v - 1) / t.tile_v);
    return t;
}

// Blocks are ordered (detector row band, view, column tile) with the band
// slowest: the CTAs resident at one time work on one band of rows of some
// tens of views, whose rays cross only a slab of the volume, so the volume
// data they gather stays in L2 (rather than whole views, which touch all of it).
__device__ __forceinline__ void block_tile(const TileMap &tm, uint32_t n_views, int &view, int &iu, int &iv) {
    const uint32_t b = blockIdx.x;
    const int tu = (int)(b % (uint32_t)tm.ntu);
    const uint32_t rest = b / (uint32_t)tm.ntu;
    view = (int)(rest % n_views);
    const int tv = (int)(rest / n_views);
    const int t = threadIdx.x;
    if (tm.tile_v == 1) {
        iu = tu * tm.tile_u + t;
        iv = tv;
    } else {
        const int lane = t & 31, warp = t >> 5;
        const int wv_per = tm.tile_v / tm.warp_v;  // warps along v in the tile
        const int wu = warp / wv_per, wv = warp % wv_per;
        iu = tu * tm.tile_u + wu * (32 / tm.warp_v) + lane / tm.warp_v;
        iv = tv * tm.tile_v + wv * tm.warp_v + lane % tm.warp_v;
    }
}

// L2 policy for the volume gathers: keep the volume resident (evict_last)
// while the streamed projection reads/writes of the same kernel are marked
// evict-first, so a volume that fits in L2 is fetched from HBM about once.
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ float ldg_keep(const float *p, uint64_t pol) {
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}

template <typename Off>
struct VolLoad {
    const float *__restrict__ vol;
    uint64_t pol;
    __device__ __forceinline__ float operator()(Off off) const { return ldg_keep(vol + off, pol); }
};

template <typename Off>
struct ScatterVisit {
    float *__restrict__ vol;
    float w;
    __device__ __forceinline__ void operator()(float seg, Off off) {
        if (seg > 0.f) atomicAdd(vol + off, seg * w);
    }
};


template <typename Off>
__global__ void __launch_bounds__(kThreads, 4)
    k_project_siddon(const aprict_proj_spec *__restrict__ specs, uint32_t n_views, uint32_t nu, uint32_t nv,
                     ab_pstrides ps, float *__restrict__ out, const float *base, ab_grid<Off> g, const float *vol,
                     float svf, float mba, int ssu, int ssv, TileMap tm, uint32_t *status) {
    int view, iu, iv;
    block_tile(tm, n_views, view, iu, iv);
    if (iu >= (int)nu || iv >= (int)nv) return;
    const aprict_proj_spec sp = specs[view];
    const ab_d3 src = ab_to_grid(g, ab_d3_of(sp.source_pos) * (double)svf);

    bool bad = false;
    float tot = 0.f;
    const uint64_t pol = l2_evict_last_policy();
    const double inv_su = 1.0 / (double)ssu, inv_sv = 1.0 / (double)ssv;
    for (int ku = 0; ku < ssu; ++ku) {
        float accu = 0.f;
        for (int kv = 0; kv < ssv; ++kv) {
            const double fu = (double)iu - 0.5 + inv_su * (ku + 0.5);
            const double fv = (double)iv - 0.5 + inv_sv * (kv + 0.5);
            const ab_d3 dst = ab_to_grid(g, ab_pixel_pos(sp, fu, fv) * (double)svf);
            VolLoad<Off> ld{vol, pol};
            float sum;
            ab_siddon_gather<Off>(src, dst, g.n, g.stride, ld, sum, &bad);
            accu += (sum * g.voxwid) * mba;
        }
        if (ssv > 1) accu /= (float)ssv;
        tot += accu;
    }
    if (ssu > 1) tot /= (float)ssu;
    if (bad && status) atomicOr(status, APRICT_STATUS_NONFINITE);
    const int64_t o = (int64_t)view * ps.view + (int64_t)iu * ps.u + (int64_t)iv * ps.v;
    if (base) {
        __stcs(out + o, __ldcs(base + o) + tot);  // streamed once: evict-first
    } else {
        atomicAdd(out + o, tot);
    }
}

template <typename Off>
__global__ void __launch_bounds__(kThreads, 4)
    k_backproject_scatter(const aprict_proj_spec *__restrict__ specs, uint32_t n_views, uint32_t nu, uint32_t nv,
                          ab_pstrides ps, const float *__restrict__ projs, ab_grid<Off> g, float *vol, float svf,
                          float mba, int ssu, int ssv, TileMap tm, uint32_t *status) {
    int view, iu, iv;
    block_tile(tm, n_views, view, iu, iv);
    if (iu >= (int)nu || iv >= (int)nv) return;
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
            ScatterVisit<Off> vis{vol, w};
            ab_siddon<Off>(src, dst, g.n, g.stride, vis, &bad);
        }
    }
    if (bad && status) atomicOr(status, APRICT_STATUS_NONFINITE);
}

int check_common(const aprict_proj_spec *specs, const aprict_proj_desc *pd, const void *pptr,
                 const aprict_vol_desc *vd, const void *vptr, const aprict_project_config *cfg) {
    int rc;
    if ((rc = ab_check_projs(pd, pptr, "projections")) != APRICT_OK) return rc;
    if ((rc = ab_check_vol(vd, vptr, "volume")) != APRICT_OK) return rc;
    if (cfg == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null project config");
    if (cfg->ssu == 0 || cfg->ssv == 0 || cfg->ssu > 64 || cfg->ssv > 64)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ssu/ssv must be in [1, 64]");
    if (!isfinite(cfg->shrink_volume_factor) || !isfinite(cfg->multiply_before_adding))
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "non-finite project config");
    if (pd->n_views && specs == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null view specs");
    return APRICT_OK;
}

bool small_volume(const aprict_vol_desc *vd) {
    return (uint64_t)vd->nx * vd->ny * vd->nz < (1ull << 31);
}

}  // namespace

extern "C" int aprict_b200_project_siddon(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                          float *projs_dev, const float *base_dev, const aprict_vol_desc *vd,
                                          const float *vol_dev, const aprict_project_config *cfg,
                                          uint32_t *status_dev, aprict_stream_t stream) {
    int rc = check_common(specs_dev, pd, projs_dev, vd, vol_dev, cfg);
    if (rc != APRICT_OK) return rc;
    if (pd->n_views == 0 || pd->nu == 0 || pd->nv == 0) return APRICT_OK;
    const TileMap tm = make_tiles(pd->nu, pd->nv);
    const ab_pstrides ps{pd->stride_view, pd->stride_u, pd->stride_v};
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const uint64_t nblocks = (uint64_t)tm.ntu * tm.ntv * pd->n_views;
    if (nblocks > 0x7fffffffull) return ab_fail(APRICT_ERR_TOO_LARGE, "too many detector tiles");
    if (small_volume(vd)) {
        k_project_siddon<int32_t><<<(unsigned)nblocks, kThreads, 0, st>>>(
            specs_dev, pd->n_views, pd->nu, pd->nv, ps, projs_dev, base_dev, ab_make_grid<int32_t>(*vd), vol_dev,
            cfg->shrink_volume_factor, cfg->multiply_before_adding, (int)cfg->ssu, (int)cfg->ssv, tm, status_dev);
    } else {
        k_project_siddon<int64_t><<<(unsigned)nblocks, kThreads, 0, st>>>(
            specs_dev, pd->n_views, pd->nu, pd->nv, ps, projs_dev, base_dev, ab_make_grid<int64_t>(*vd), vol_dev,
            cfg->shrink_volume_factor, cfg->multiply_before_adding, (int)cfg->ssu, (int)cfg->ssv, tm, status_dev);
    }
    return ab_cuda_check(cudaGetLastError(), "project_siddon launch");
}

extern "C" int aprict_b200_backproject_scatter(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                               const float *projs_dev, const aprict_vol_desc *vd, float *vol_dev,
                                               const aprict_project_config *cfg, uint32_t *status_dev,
                                               aprict_stream_t stream) {
    int rc = check_common(specs_dev, pd, projs_dev, vd, vol_dev, cfg);
    if (rc != APRICT_OK) return rc;
    if (pd->n_views == 0 || pd->nu == 0 || pd->nv == 0) return APRICT_OK;
    const TileMap tm = make_tiles(pd->nu, pd->nv);
    const ab_pstrides ps{pd->stride_view, pd->stride_u, pd->stride_v};
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const uint64_t nblocks = (uint64_t)tm.ntu * tm.ntv * pd->n_views;
    if (nblocks > 0x7fffffffull) return ab_fail(APRICT_ERR_TOO_LARGE, "too many detector tiles");
    if (small_volume(vd)) {
        k_backproject_scatter<int32_t><<<(unsigned)nblocks, kThreads, 0, st>>>(
            specs_dev, pd->n_views, pd->nu, pd->nv, ps, projs_dev, ab_make_grid<int32_t>(*vd), vol_dev,
            cfg->shrink_volume_factor, cfg->multiply_before_adding, (int)cfg->ssu, (int)cfg->ssv, tm, status_dev);
    } else {
        k_backproject_scatter<int64_t><<<(unsigned)nblocks, kThreads, 0, st>>>(
            specs_dev, pd->n_views, pd->nu, pd->nv, ps, projs_dev, ab_make_grid<int64_t>(*vd), vol_dev,
            cfg->shrink_volume_factor, cfg->multiply_before_adding, (int)cfg->ssu, (int)cfg->ssv, tm, status_dev);
    }
    return ab_cuda_check(cudaGetLastError(), "backproject_scatter launch");
}
