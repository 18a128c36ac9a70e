// ab_host.h -- host-side argument validation and error plumbing shared by the
// C-ABI entry points. Mirrors the checks the reference makes in Python before
// a launch (flatpanel.py:235-266, 1141-1159) so that nothing invalid reaches
// the GPU.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "aprict_b200.h"

// Thread-local text of the last error, returned by aprict_b200_last_error().
void ab_set_error(const char *fmt, ...);
int ab_fail(int status, const char *fmt, ...);

// Converts a CUDA runtime error into APRICT_ERR_CUDA (and records its text).
int ab_cuda_check(cudaError_t e, const char *what);

int ab_check_vol(const aprict_vol_desc *v, const void *ptr, const char *name);
int ab_check_projs(const aprict_proj_desc *p, const void *ptr, const char *name);

// Launch-shape knobs (set by the autotuner through aprict_b200_set_tuning).
enum {
    AB_TUNE_FP_TILE_V = 0,  // forward projector tile height in pixels (0 = auto, 8, 16, 32)
    AB_TUNE_BP_XB = 1,      // backprojector voxels per thread (0 = auto = 2, 2, 4)
    AB_TUNE_BP_WAVE = 2,    // backprojector super-brick size in CTAs per SM (0 = auto = 3)
    AB_TUNE_FP_WARP_V = 3,  // forward projector lanes of a warp along v (0 = auto = 8, 8, 16, 32)
    AB_TUNE_FP_VIEWS = 4,   // forward projector views per tile (0 = auto = 4, 1, 2, 4)
    AB_TUNE_FP_WARP_VIEWS = 5,  // forward projector views inside a warp's patch (0 = auto = 1, 1, 2, 4)
    AB_TUNE_FP_SS1 = 6,     // one-scan projector, one sub-ray per pixel: 0 = specialised path, 1 = general path
    AB_TUNE_BP_ZLANES = 7,  // one-scan backprojector on C-order volumes: 0 = z-column layout when tall enough, 1 = never
    AB_TUNE_COUNT = 8
};
int ab_tuning_get(int key);

// Largest element offset reachable in a projection stack (for overflow checks).
int64_t ab_projs_max_offset(const aprict_proj_desc *p);
