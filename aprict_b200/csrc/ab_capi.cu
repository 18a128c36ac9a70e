// ab_capi.cu -- status strings, version and shared host validation.
#include <math.h>
#include <stddef.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "ab_host.h"

static_assert(sizeof(aprict_proj_spec) == 60, "proj_spec must match the reference's 60-byte layout");
static_assert(sizeof(aprict_vol_desc) == 32, "vol_desc layout");
static_assert(sizeof(aprict_proj_desc) == 40, "proj_desc layout");
static_assert(sizeof(aprict_project_config) == 16, "project_config layout");
static_assert(sizeof(aprict_backproject_config) == 76, "backproject_config layout");
static_assert(sizeof(aprict_scan) == 120 && offsetof(aprict_scan, vol) == 64 && offsetof(aprict_scan, vol_dev) == 96,
              "scan layout");

static thread_local char g_last_error[512] = "";
static int g_tuning[AB_TUNE_COUNT] = {0, 0, 0, 0, 0, 0, 0, 0};

int ab_tuning_get(int key) { return key >= 0 && key < AB_TUNE_COUNT ? __atomic_load_n(&g_tuning[key], __ATOMIC_RELAXED) : 0; }

void ab_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

int ab_fail(int status, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

int ab_cuda_check(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return APRICT_OK;
    return ab_fail(APRICT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int ab_check_vol(const aprict_vol_desc *v, const void *ptr, const char *name) {
    if (v == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: null volume descriptor", name);
    if (ptr == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: null volume pointer", name);
    if (v->nx == 0 || v->ny == 0 || v->nz == 0)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: empty volume shape", name);
    if (v->order > 1) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: order must be 0 (C) or 1 (F)", name);
    if (!(v->voxwid > 0.f) || !isfinite(v->voxwid))
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: voxwid must be positive and finite", name);
    if (!isfinite(v->corner.x) || !isfinite(v->corner.y) || !isfinite(v->corner.z))
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: non-finite volume corner", name);
    if (v->nx > (1u << 30) || v->ny > (1u << 30) || v->nz > (1u << 30))
        return ab_fail(APRICT_ERR_TOO_LARGE, "%s: volume edge exceeds 2^30", name);
    if ((reinterpret_cast<uintptr_t>(ptr) & 3u) != 0)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: volume pointer not 4-byte aligned", name);
    return APRICT_OK;
}

int64_t ab_projs_max_offset(const aprict_proj_desc *p) {
    int64_t m = 0;
    if (p->n_views) m += (int64_t)(p->n_views - 1) * (p->stride_view < 0 ? -p->stride_view : p->stride_view);
    if (p->nu) m += (int64_t)(p->nu - 1) * (p->stride_u < 0 ? -p->stride_u : p->stride_u);
    if (p->nv) m += (int64_t)(p->nv - 1) * (p->stride_v < 0 ? -p->stride_v : p->stride_v);
    return m;
}

int ab_check_projs(const aprict_proj_desc *p, const void *ptr, const char *name) {
    if (p == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: null projection descriptor", name);
    if (p->n_views == 0 || p->nu == 0 || p->nv == 0) return APRICT_OK;  // empty: nothing to do
    if (ptr == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: null projection pointer", name);
    if (p->stride_view < 0 || p->stride_u < 0 || p->stride_v < 0)
        return ab_fail(APRICT_ERR_UNSUPPORTED, "%s: negative projection strides are not supported", name);
    if (p->nu > (1u << 24) || p->nv > (1u << 24))
        return ab_fail(APRICT_ERR_TOO_LARGE, "%s: detector edge exceeds 2^24", name);
    if ((reinterpret_cast<uintptr_t>(ptr) & 3u) != 0)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "%s: projection pointer not 4-byte aligned", name);
    return APRICT_OK;
}

extern "C" {

const char *aprict_b200_status_string(int status) {
    switch (status) {
        case APRICT_OK: return "ok";
        case APRICT_ERR_INVALID_ARGUMENT: return "invalid argument";
        case APRICT_ERR_UNSUPPORTED: return "unsupported configuration";
        case APRICT_ERR_CUDA: return "CUDA runtime error";
        case APRICT_ERR_TOO_LARGE: return "size too large";
        case APRICT_ERR_NO_DEVICE: return "no usable device";
        default: return "unknown status";
    }
}

const char *aprict_b200_last_error(void) { return g_last_error; }

const char *aprict_b200_version(void) { return "0.1.0"; }

int aprict_b200_set_tuning(int key, int value) {
    if (key < 0 || key >= AB_TUNE_COUNT) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "unknown tuning key %d", key);
    bool ok;
    switch (key) {
        case AB_TUNE_FP_TILE_V: ok = value == 0 || value == 8 || value == 16 || value == 32; break;
        case AB_TUNE_BP_XB: ok = value == 0 || value == 2 || value == 4 || value == 8; break;
        case AB_TUNE_FP_WARP_V: ok = value == 0 || value == 8 || value == 16 || value == 32; break;
        case AB_TUNE_FP_VIEWS:
        case AB_TUNE_FP_WARP_VIEWS: ok = value == 0 || value == 1 || value == 2 || value == 4; break;
        case AB_TUNE_FP_SS1:
        case AB_TUNE_BP_ZLANES: ok = value == 0 || value == 1; break;
        default: ok = value >= 0 && value <= 16; break;
    }
    if (!ok) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "tuning value %d not allowed for key %d", value, key);
    __atomic_store_n(&g_tuning[key], value, __ATOMIC_RELAXED);
    return APRICT_OK;
}

int aprict_b200_get_tuning(int key) { return ab_tuning_get(key); }

size_t aprict_b200_struct_size(const char *name) {
    if (name == nullptr) return 0;
    if (!strcmp(name, "aprict_proj_spec")) return sizeof(aprict_proj_spec);
    if (!strcmp(name, "aprict_vol_desc")) return sizeof(aprict_vol_desc);
    if (!strcmp(name, "aprict_proj_desc")) return sizeof(aprict_proj_desc);
    if (!strcmp(name, "aprict_project_config")) return sizeof(aprict_project_config);
    if (!strcmp(name, "aprict_backproject_config")) return sizeof(aprict_backproject_config);
    if (!strcmp(name, "aprict_forbild_shape")) return sizeof(aprict_forbild_shape);
    if (!strcmp(name, "aprict_quadric")) return sizeof(aprict_quadric);
    if (!strcmp(name, "aprict_scan")) return sizeof(aprict_scan);
    return 0;
}

}  // extern "C"
