// ab_fptile.cuh -- the Siddon forward projector's work unit, shared by the
// one-scan kernel (ab_siddon.cu) and the persistent multi-scan kernel
// (ab_batch.cu).
//
// Replaces project_CB_texture_chunked<float,float>
// (src/aprict/data/cusrc/CB_project_texture_chunked.cu:327-412): one thread
// per (view, pixel); ssu x ssv sub-rays averaged as in :381-407; result
// scaled by multiply_before_adding (:394) and accumulated (:411).
//
// B200 layout: a CTA covers a 2-D detector tile of one view (or of 2 or 4
// neighbouring views, as tuned) and each warp a 4 (u) x 8 (v) pixel patch
// (2 x 16 or 1 x 32 as tuned), so the rays of a warp are spatially coherent
// and their voxel gathers hit the same L1 lines; 8 consecutive v per row make
// the output access one 32-byte sector.
#pragma once

#include <cuda_runtime.h>

#include "ab_common.cuh"
#include "ab_host.h"

namespace ab_fp {


constexpr int kThreads = 256;

// Resident CTAs per SM the projector kernels are compiled for: the
// single-sub-ray ray path fits 48 registers without spilling, the general
// (sub-ray) path keeps 64.
constexpr int fp_min_blocks(bool ss1) { return ss1 ? 5 : 4; }

struct TileMap {
    int tile_w, tile_u, tile_v;  // tile extents: views, pixels along u, pixels along v
    int warp_w, warp_u, warp_v;  // a warp's patch (product 32)
    int ntw, ntu, ntv;           // number of tiles along views, u, v
    // log2 of the power-of-two extents above, for shift/mask decomposition
    int lg_warp_u, lg_warp_v, lg_nwu, lg_nwv, lg_tile_u;
    uint64_t units() const { return (uint64_t)ntw * ntu * ntv; }
};

inline int ilog2_pow2(int x) {
    int l = 0;
    while ((1 << l) < x) ++l;
    return l;
}

// Tile shapes: tv == 1 -> one detector row per tile (used when nv < 8);
// otherwise warps are 1 (view) x 4 (u) x 8 (v) patches of a 4 x 4 x 16
// tile: four neighbouring views, one per pair of warps. Rays of neighbouring
// views cross nearly the same voxels, so more of their gathers hit the same
// L1 lines. The autotuner may change the tile height (8, 16, 32), the warp
// patch height (16, 32), the views per tile (1, 2, 4) and put 2 or 4 views
// inside each warp's patch.
inline TileMap make_tiles(uint32_t nu, uint32_t nv, uint32_t n_views) {
    TileMap t;
    t.tile_v = nv >= 16 ? 16 : (nv >= 8 ? 8 : 1);
    const int want = ab_tuning_get(AB_TUNE_FP_TILE_V);  // autotuner override: 8, 16 or 32
    if ((want == 8 || want == 16 || want == 32) && nv >= 8) t.tile_v = want;
    const int wv = ab_tuning_get(AB_TUNE_FP_WARP_V);
    t.warp_v = (wv == 16 || wv == 32) ? wv : 8;
    const int tw = ab_tuning_get(AB_TUNE_FP_VIEWS), ww = ab_tuning_get(AB_TUNE_FP_WARP_VIEWS);
    t.tile_w = (tw == 1 || tw == 2) ? tw : 4;  // 4 by default: measured 2 % faster than 1 on a 256^3 volume
    t.warp_w = (ww == 2 || ww == 4) ? ww : 1;
    if (t.tile_v == 1) {
        t.tile_w = t.warp_w = 1;
        t.warp_v = 1;
    } else {
        if (t.warp_v > t.tile_v) t.tile_v = t.warp_v;
        if (t.warp_w > t.tile_w) t.warp_w = t.tile_w;
        while (t.warp_w * t.warp_v > 32) t.warp_w /= 2;
        while (t.tile_w * t.tile_v > kThreads / (32 / (t.warp_w * t.warp_v))) t.tile_w /= 2;
        if (t.warp_w > t.tile_w) t.warp_w = t.tile_w;
    }
    t.warp_u = 32 / (t.warp_w * t.warp_v);
    t.tile_u = kThreads / (t.tile_w * t.tile_v);
    t.lg_warp_u = ilog2_pow2(t.warp_u);
    t.lg_warp_v = ilog2_pow2(t.warp_v);
    t.lg_nwu = ilog2_pow2(t.tile_u / t.warp_u);
    t.lg_nwv = ilog2_pow2(t.tile_v / t.warp_v);
    t.lg_tile_u = ilog2_pow2(t.tile_u);
    t.ntu = (int)((nu + t.tile_u - 1) / t.tile_u);
    t.ntv = (int)((nv + t.tile_v - 1) / t.tile_v);
    t.ntw = (int)((n_views + t.tile_w - 1) / t.tile_w);
    return t;
}

// Blocks are ordered (detector row band, view group, column tile) with the
// band slowest: the CTAs resident at one time work on one band of rows of
// some tens of views, whose rays cross only a slab of the volume, so the
// volume data they gather stays in L2 (rather than whole views, which touch
// all of it). tile_thread maps (column tile tu, view group tw, row band tv)
// and the thread to its ray; every extent inside a tile is a power of two, so
// the decomposition is shifts and masks. False when the thread has no ray
// (past the last view).
__device__ __forceinline__ bool tile_thread(const TileMap &tm, uint32_t n_views, int tu, int tw, int tv, int &view,
                                            int &iu, int &iv) {
    const int t = threadIdx.x;
    if (tm.tile_v == 1) {
        view = tw;
        iu = (tu << tm.lg_tile_u) + t;
        iv = tv;
    } else {
        const int lane = t & 31, warp = t >> 5;
        const int lv = lane & (tm.warp_v - 1);
        const int lu = (lane >> tm.lg_warp_v) & (tm.warp_u - 1);
        const int lw = lane >> (tm.lg_warp_v + tm.lg_warp_u);
        const int wv = warp & ((1 << tm.lg_nwv) - 1);
        const int wu = (warp >> tm.lg_nwv) & ((1 << tm.lg_nwu) - 1);
        const int ww = warp >> (tm.lg_nwv + tm.lg_nwu);
        view = tw * tm.tile_w + ww * tm.warp_w + lw;
        iu = (tu << tm.lg_tile_u) + (wu << tm.lg_warp_u) + lu;
        iv = tv * tm.tile_v + (wv << tm.lg_warp_v) + lv;
    }
    return view < (int)n_views;
}

// The same for a linear work-unit index b (column tile fastest, then view
// group, then row band).
__device__ __forceinline__ bool block_tile(const TileMap &tm, uint32_t n_views, uint32_t b, int &view, int &iu,
                                           int &iv) {
    const int tu = (int)(b % (uint32_t)tm.ntu);
    const uint32_t rest = b / (uint32_t)tm.ntu;
    const int tw = (int)(rest % (uint32_t)tm.ntw);
    const int tv = (int)(rest / (uint32_t)tm.ntw);
    return tile_thread(tm, n_views, tu, tw, tv, view, iu, iv);
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



// One forward-projection work unit: a detector tile of one view (kThreads rays).
template <typename Off>
struct FPScan {
    const aprict_proj_spec *specs;
    uint32_t n_views, nu, nv;
    ab_pstrides ps;
    float *out;
    const float *base;  // NULL: out += mba A vol (atomic); else out = base + mba A vol
    ab_grid<Off> g;
    const float *vol;
    float svf, mba;
    int ssu, ssv;
    TileMap tm;
    uint32_t *status;
    int one;  // 1, passed at run time (see AB_SIDDON_ADVANCE_I32)
};

// Rays of work unit b (block_tile order) of scan S; every thread of the CTA
// calls it with the same b. No barriers inside. SS1: one sub-ray per pixel
// (ssu = ssv = 1), which keeps nothing but the sum live across the traversal.
template <typename Off, bool SS1>
__device__ __forceinline__ void fp_ray(const FPScan<Off> &S, int view, int iu, int iv) {
    const uint64_t pol = l2_evict_last_policy();
    bool bad = false;
    float tot;
    if (SS1) {
        const aprict_proj_spec &sp = S.specs[view];
        const ab_d3 src = ab_to_grid(S.g, ab_d3_of(sp.source_pos) * (double)S.svf);
        const ab_d3 dst = ab_to_grid(S.g, ab_pixel_pos(sp, (double)iu, (double)iv) * (double)S.svf);
        VolLoad<Off> ld{S.vol, pol};
        float sum;
        ab_siddon_gather<Off>(src, dst, S.g.n, S.g.stride, ld, sum, &bad, S.one);
        tot = (sum * S.g.voxwid) * S.mba;
    } else {
        const aprict_proj_spec sp = S.specs[view];
        const ab_grid<Off> &g = S.g;
        const ab_d3 src = ab_to_grid(g, ab_d3_of(sp.source_pos) * (double)S.svf);
        tot = 0.f;
        const int ssu = S.ssu, ssv = S.ssv;
        const double inv_su = 1.0 / (double)ssu, inv_sv = 1.0 / (double)ssv;
        for (int ku = 0; ku < ssu; ++ku) {
            float accu = 0.f;
            for (int kv = 0; kv < ssv; ++kv) {
                const double fu = (double)iu - 0.5 + inv_su * (ku + 0.5);
                const double fv = (double)iv - 0.5 + inv_sv * (kv + 0.5);
                const ab_d3 dst = ab_to_grid(g, ab_pixel_pos(sp, fu, fv) * (double)S.svf);
                VolLoad<Off> ld{S.vol, pol};
                float sum;
                ab_siddon_gather<Off>(src, dst, g.n, g.stride, ld, sum, &bad, S.one);
                accu += (sum * g.voxwid) * S.mba;
            }
            if (ssv > 1) accu /= (float)ssv;
            tot += accu;
        }
        if (ssu > 1) tot /= (float)ssu;
    }
    if (bad && S.status) atomicOr(S.status, APRICT_STATUS_NONFINITE);
    const int64_t o = (int64_t)view * S.ps.view + (int64_t)iu * S.ps.u + (int64_t)iv * S.ps.v;
    if (S.base) {
        __stcs(S.out + o, __ldcs(S.base + o) + tot);  // streamed once: evict-first
    } else {
        atomicAdd(S.out + o, tot);
    }
}

// Rays of work unit b (linear tile order) of scan S.
template <typename Off, bool SS1>
__device__ __forceinline__ void fp_tile(const FPScan<Off> &S, uint32_t b) {
    int view, iu, iv;
    if (!block_tile(S.tm, S.n_views, b, view, iu, iv) || iu >= (int)S.nu || iv >= (int)S.nv) return;
    fp_ray<Off, SS1>(S, view, iu, iv);
}

// Host: argument checks shared by the projector and its adjoint.
inline int fp_check(const aprict_proj_spec *specs, const aprict_proj_desc *pd, const void *pptr,
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

inline bool small_volume(const aprict_vol_desc *vd) { return (uint64_t)vd->nx * vd->ny * vd->nz < (1ull << 31); }

// Host: the scan descriptor and its number of work units (0 when empty).
template <typename Off>
inline FPScan<Off> make_fpscan(const aprict_proj_spec *specs, const aprict_proj_desc *pd, float *projs,
                               const float *base, const aprict_vol_desc *vd, const float *vol,
                               const aprict_project_config *cfg, uint32_t *status, uint64_t &units) {
    FPScan<Off> S{};
    S.specs = specs;
    S.n_views = pd->n_views;
    S.nu = pd->nu;
    S.nv = pd->nv;
    S.ps = ab_pstrides{pd->stride_view, pd->stride_u, pd->stride_v};
    S.out = projs;
    S.base = base;
    S.g = ab_make_grid<Off>(*vd);
    S.vol = vol;
    S.svf = cfg->shrink_volume_factor;
    S.mba = cfg->multiply_before_adding;
    S.ssu = (int)cfg->ssu;
    S.ssv = (int)cfg->ssv;
    S.tm = make_tiles(pd->nu, pd->nv, pd->n_views);
    S.status = status;
    S.one = 1;
    units = (pd->n_views == 0 || pd->nu == 0 || pd->nv == 0) ? 0 : S.tm.units();
    return S;
}

}  // namespace ab_fp
