// ab_backproject.cu -- voxel-driven cone-beam backprojection, all views in
// one launch (one scan). The work unit lives in ab_bpbrick.cuh.
#include <cuda_runtime.h>

#include "ab_bpbrick.cuh"

namespace {

using namespace ab_bp;

template <int ORD, bool EXACT, bool RAYCAST, bool BILIN, int XB>
__global__ void __launch_bounds__(kThreads, bp_min_blocks(XB, EXACT)) k_backproject(const BPParams P) {
    __shared__ BPSmem<EXACT, BILIN, XB, bp_ztable(ORD, EXACT, RAYCAST, BILIN)> sm;
    bp_brick<ORD, EXACT, RAYCAST, BILIN, XB>(P, blockIdx.x, sm);
}

template <int ORD, int XB>
void launch_bp(const BPParams &P, const aprict_backproject_config *cfg, bool lin, unsigned grid, cudaStream_t st) {
    if (cfg->exact) {
        k_backproject<ORD, true, false, false, XB><<<grid, kThreads, 0, st>>>(P);
    } else if (cfg->approx_mode_direct_raycast) {
        if (lin)
            k_backproject<ORD, false, true, true, XB><<<grid, kThreads, 0, st>>>(P);
        else
            k_backproject<ORD, false, true, false, XB><<<grid, kThreads, 0, st>>>(P);
    } else {
        if (lin)
            k_backproject<ORD, false, false, true, XB><<<grid, kThreads, 0, st>>>(P);
        else
            k_backproject<ORD, false, false, false, XB><<<grid, kThreads, 0, st>>>(P);
    }
}

}  // namespace

extern "C" int aprict_b200_backproject(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                       const float *projs_dev, const aprict_vol_desc *vd, float *vol_dev,
                                       const float *multiplier_dev, const aprict_backproject_config *cfg,
                                       uint32_t *status_dev, aprict_stream_t stream) {
    BPParams P;
    uint64_t grid = 0;
    int xb = 2;
    int ord = 0;
    // Slice stacks (one z layer) always take two voxels per thread.
    const int rc = make_bp_params(specs_dev, pd, projs_dev, vd, vol_dev, multiplier_dev, cfg, status_dev, P, grid, xb,
                                  vd != nullptr && bp_ord(vd) == 2 ? 2 : 0, &ord);
    if (rc != APRICT_OK || grid == 0) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const bool lin = cfg->approx_mode_linear_interpolate != 0;
    if (ord == 2) {
        launch_bp<2, 2>(P, cfg, lin, (unsigned)grid, st);  // slices (xb forced to 2 above)
    } else if (ord == 3) {  // C order, z columns
        if (xb == 8)
            launch_bp<3, 8>(P, cfg, lin, (unsigned)grid, st);
        else if (xb == 4)
            launch_bp<3, 4>(P, cfg, lin, (unsigned)grid, st);
        else
            launch_bp<3, 2>(P, cfg, lin, (unsigned)grid, st);
    } else if (xb == 8) {
        if (ord == 0)
            launch_bp<0, 8>(P, cfg, lin, (unsigned)grid, st);
        else
            launch_bp<1, 8>(P, cfg, lin, (unsigned)grid, st);
    } else if (xb == 4) {
        if (ord == 0)
            launch_bp<0, 4>(P, cfg, lin, (unsigned)grid, st);
        else
            launch_bp<1, 4>(P, cfg, lin, (unsigned)grid, st);
    } else {
        if (ord == 0)
            launch_bp<0, 2>(P, cfg, lin, (unsigned)grid, st);
        else
            launch_bp<1, 2>(P, cfg, lin, (unsigned)grid, st);
    }
    return ab_cuda_check(cudaGetLastError(), "backproject launch");
}
