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

// Largest element offset reachable in a projection stack (for overflow checks).
int64_t ab_projs_max_offset(const aprict_proj_desc *p);
