// ab_batch.cu -- many independent scans in one persistent launch.
//
// The reference projects and backprojects one scan per call, each call a
// sequence of launches sized to that scan (flatpanel.py:1047-1122,
// 1161-1278); a workload of many small, uneven scans leaves most of the GPU
// idle at the tail of every launch and pays a launch and a host
// synchronisation per 10 views. Here a batch of scans is one plan: the
// per-scan parameters of the one-scan kernels (FPScan / BPParams) plus the
// prefix sums of their work-unit counts. One persistent launch of
// (SMs x resident CTAs) CTAs then pulls work units from a global counter --
// the detector tiles of every scan for a projection, the volume bricks of
// every scan for a backprojection -- so the whole GPU stays busy across scan
// boundaries. Scans are ordered largest first so that the small ones fill the
// tail. The counter lives in the plan; the last CTA to finish puts it back to
// zero, so a plan is relaunched (or replayed in a CUDA graph) with no host
// work. There are no waits between CTAs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "ab_bpbrick.cuh"
#include "ab_fptile.cuh"

namespace {

constexpr uint32_t kPlanMagic = 0x41424232u;  // "ABB2"
constexpr int kGroup = 96;                    // scans per launch (kernel-parameter space)

// Plan layout (host image; the caller's device copy is used only for the
// per-group counters): header, then n_groups Group records (256 bytes
// apart, so each group's counters own their line), then the per-scan
// parameters in execution order.
struct PlanHeader {
    uint32_t magic;
    int32_t op;       // APRICT_BATCH_PROJECT / APRICT_BATCH_BACKPROJECT
    int32_t n_scans;
    int32_t variant;  // kernel template variant (see the run function)
    int32_t n_groups;
    int32_t pad_;
    uint64_t groups_off, params_off, bytes;
};

struct Group {
    uint32_t counter;  // next work unit; zero between launches (device copy)
    uint32_t exited;   // CTAs finished in the current launch; zero between launches
    uint32_t first;    // first scan (execution order)
    uint32_t count;    // scans in the group
    uint32_t n_units;
    int32_t grid;                 // persistent CTAs (SMs x resident CTAs, at most n_units)
    uint32_t prefix[kGroup + 1];  // cumulative work units of the group's scans
};

// Launch arguments: the group's scans travel in the kernel parameter space
// (constant bank), where the per-scan fields cost no registers to keep.
template <class Params>
struct BatchArgs {
    Group *g;  // device copy of the group record (counters)
    uint32_t count, n_units;
    uint32_t prefix[kGroup + 1];
    Params scans[kGroup];
};
static_assert(sizeof(BatchArgs<ab_bp::BPParams>) <= 32000, "batch arguments exceed the kernel parameter space");
static_assert(sizeof(BatchArgs<ab_fp::FPScan<int64_t>>) <= 32000, "batch arguments exceed the kernel parameter space");

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

size_t params_size(int op) {
    return op == APRICT_BATCH_PROJECT ? std::max(sizeof(ab_fp::FPScan<int64_t>), sizeof(ab_fp::FPScan<int32_t>))
                                      : sizeof(ab_bp::BPParams);
}

int n_groups_of(int n) { return (n + kGroup - 1) / kGroup; }

size_t plan_bytes(int op, int n) {
    return align256(sizeof(PlanHeader)) + (size_t)n_groups_of(n) * align256(sizeof(Group)) +
           align256(params_size(op) * (size_t)n);
}

// Work-unit fetch shared by both kernels: thread 0 takes the next unit and
// finds its scan (binary search over the prefix sums); the CTA reads both
// from shared memory. Returns false when the group is exhausted.
template <class Args>
__device__ __forceinline__ bool next_unit(const Args &A, uint32_t &unit, int &scan) {
    __shared__ uint32_t s_unit;
    __shared__ int s_scan;
    if (threadIdx.x == 0) {
        const uint32_t it = atomicAdd(&A.g->counter, 1u);
        int s = 0;
        if (it < A.n_units) {
            int lo = 0, hi = (int)A.count - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (A.prefix[mid] <= it)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            s = lo;
        }
        s_unit = it;
        s_scan = s;
    }
    __syncthreads();
    unit = s_unit;
    scan = s_scan;
    __syncthreads();  // s_unit is rewritten only after every thread has read it
    if (unit >= A.n_units) return false;
    unit -= A.prefix[scan];
    return true;
}

// The last CTA of a launch puts the counters back to zero for the next one.
// Every CTA has taken its final (out-of-range) unit before it counts itself
// out, so no unit is fetched after the reset.
__device__ __forceinline__ void retire(Group *g) {
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t done = atomicAdd(&g->exited, 1u) + 1u;
        if (done == gridDim.x) {
            g->counter = 0u;
            g->exited = 0u;
            __threadfence();
        }
    }
}

template <typename Off, bool SS1>
__global__ void __launch_bounds__(ab_fp::kThreads, ab_fp::fp_min_blocks(SS1))
    k_batch_project(const __grid_constant__ BatchArgs<ab_fp::FPScan<Off>> A) {
    uint32_t unit;
    int s;
    while (next_unit(A, unit, s)) ab_fp::fp_tile<Off, SS1>(A.scans[s], unit);
    retire(A.g);
}

// Voxels per thread of the batch backprojection kernel: the single-scan
// default, and four for slice stacks, where a batch holds many slices (64
// fan-beam slices 30.7 -> 27.7 ms against two); the single-scan launch keeps
// two there (one slice has too few bricks at four: 68 -> 80 ms for 64 slices
// one by one), so a batched slice equals its one-scan result to FP32 rounding.
constexpr int batch_xb(int ord, bool exact) { return ord == 2 ? 4 : ab_bp::default_xb(exact); }

// The batch kernel skips, in every fast mode, the views whose projection of
// a brick misses the detector: batches mix helical and circular scans, and
// the helical ones leave most of a volume off each view's detector (48
// uneven scans: 326.6 -> 265.3 ms per batched backprojection).
template <int ORD, bool EXACT, bool RAYCAST, bool BILIN, int XB = batch_xb(ORD, EXACT)>
__global__ void __launch_bounds__(ab_bp::kThreads, ab_bp::bp_min_blocks(XB, EXACT))
    k_batch_backproject(const __grid_constant__ BatchArgs<ab_bp::BPParams> A) {
    __shared__ ab_bp::BPSmem<EXACT, BILIN, XB, ab_bp::bp_ztable(ORD, EXACT, RAYCAST, BILIN)> sm;
    uint32_t unit;
    int s;
    while (next_unit(A, unit, s)) ab_bp::bp_brick<ORD, EXACT, RAYCAST, BILIN, XB, true>(A.scans[s], unit, sm);
    retire(A.g);
}

// Backprojection kernel variant code: ORD + 3 * mode (ORD from ab_bp::bp_ord),
// mode 0 fast nearest, 1 fast bilinear, 2 raycast nearest, 3 raycast
// bilinear, 4 exact; 15: fast nearest in the z-column layout (ORD 3) with 4
// voxels per thread, 16: the same with 8 (every scan at least 256 voxels tall).
int bp_variant(const aprict_backproject_config *c, const aprict_vol_desc *vd) {
    const int mode = c->exact ? 4
                              : (c->approx_mode_direct_raycast ? 2 : 0) + (c->approx_mode_linear_interpolate ? 1 : 0);
    return ab_bp::bp_ord(vd) + 3 * mode;
}

// The batch backprojection kernel of a variant code.
template <int V>
auto bp_kernel() {
    if constexpr (V == 16) {
        return k_batch_backproject<3, false, false, false, 8>;
    } else {
        constexpr int ORD = V == 15 ? 3 : V % 3, mode = V == 15 ? 0 : V / 3;
        return k_batch_backproject<ORD, mode == 4, mode == 2 || mode == 3, mode == 1 || mode == 3>;
    }
}

template <class F>
int with_bp_kernel(int variant, F &&f) {
    switch (variant) {
        case 0: return f(bp_kernel<0>());
        case 1: return f(bp_kernel<1>());
        case 2: return f(bp_kernel<2>());
        case 3: return f(bp_kernel<3>());
        case 4: return f(bp_kernel<4>());
        case 5: return f(bp_kernel<5>());
        case 6: return f(bp_kernel<6>());
        case 7: return f(bp_kernel<7>());
        case 8: return f(bp_kernel<8>());
        case 9: return f(bp_kernel<9>());
        case 10: return f(bp_kernel<10>());
        case 11: return f(bp_kernel<11>());
        case 12: return f(bp_kernel<12>());
        case 13: return f(bp_kernel<13>());
        case 14: return f(bp_kernel<14>());
        case 15: return f(bp_kernel<15>());
        case 16: return f(bp_kernel<16>());
        default: return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "corrupt batch plan (variant %d)", variant);
    }
}

// Multiprocessor count of the current device, cached per device ordinal (a
// plan built on another device gets that device's persistent grid).
int sm_count(int &sms) {
    constexpr int kMaxDev = 64;
    static int cached[kMaxDev] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return ab_fail(APRICT_ERR_CUDA, "cannot query the current device");
    int n = (dev >= 0 && dev < kMaxDev) ? __atomic_load_n(&cached[dev], __ATOMIC_RELAXED) : 0;
    if (n == 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            return ab_fail(APRICT_ERR_CUDA, "cannot query the multiprocessor count");
        if (dev >= 0 && dev < kMaxDev) __atomic_store_n(&cached[dev], n, __ATOMIC_RELAXED);
    }
    sms = n;
    return APRICT_OK;
}

// Persistent grid of a kernel: SMs x resident CTAs (the query also loads the
// kernel, so a later launch inside a stream capture loads nothing).
template <class K>
int grid_for(K kernel, uint32_t n_units, int32_t &grid) {
    int sms = 0, per_sm = 0;
    const int rc = sm_count(sms);
    if (rc != APRICT_OK) return rc;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0) != cudaSuccess || per_sm <= 0)
        return ab_fail(APRICT_ERR_CUDA, "occupancy query failed");
    grid = (int32_t)std::min<uint64_t>((uint64_t)sms * per_sm, n_units);
    return APRICT_OK;
}

template <class Params, class K>
int launch_group(K kernel, const PlanHeader *H, const Group &gh, Group *gd, const char *params_host,
                 cudaStream_t st) {
    if (gh.n_units == 0) return APRICT_OK;
    const int grid = gh.grid;
    if (grid <= 0) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "corrupt batch plan (grid)");
    BatchArgs<Params> A;
    A.g = gd;
    A.count = gh.count;
    A.n_units = gh.n_units;
    memcpy(A.prefix, gh.prefix, sizeof(A.prefix));
    memcpy(A.scans, params_host + (size_t)gh.first * sizeof(Params), sizeof(Params) * gh.count);
    (void)H;
    kernel<<<grid, 256, 0, st>>>(A);
    return ab_cuda_check(cudaGetLastError(), "batch launch");
}

int scan_error(int rc, int i) {
    char msg[512];
    snprintf(msg, sizeof(msg), "%s", aprict_b200_last_error());
    return ab_fail(rc, "scan %d: %s", i, msg);
}

}  // namespace

extern "C" size_t aprict_b200_batch_plan_bytes(int op, int n_scans) {
    if ((op != APRICT_BATCH_PROJECT && op != APRICT_BATCH_BACKPROJECT) || n_scans <= 0) return 0;
    return plan_bytes(op, n_scans);
}

extern "C" int aprict_b200_batch_plan(int op, const aprict_scan *scans, int n_scans, const void *configs,
                                      void *plan_host, size_t plan_capacity) {
    if (op != APRICT_BATCH_PROJECT && op != APRICT_BATCH_BACKPROJECT)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "unknown batch operation %d", op);
    if (scans == nullptr || configs == nullptr || plan_host == nullptr || n_scans <= 0)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "batch plan needs scans, configs and a plan buffer");
    const size_t need = plan_bytes(op, n_scans);
    if (plan_capacity < need)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "plan buffer too small: %zu bytes, %zu needed", plan_capacity,
                       need);
    if (reinterpret_cast<uintptr_t>(plan_host) & 255u)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "plan buffer must be 256-byte aligned");

    // Validate every scan and build its parameters with the one-scan code.
    std::vector<uint64_t> units(n_scans, 0);
    std::vector<ab_fp::FPScan<int32_t>> fp32(op == APRICT_BATCH_PROJECT ? n_scans : 0);
    std::vector<ab_fp::FPScan<int64_t>> fp64(op == APRICT_BATCH_PROJECT ? n_scans : 0);
    std::vector<ab_bp::BPParams> bp(op == APRICT_BATCH_BACKPROJECT ? n_scans : 0);
    bool all_small = true, all_ss1 = true;
    int variant = -1;
    // The z-column layout for a backprojection batch only when every scan
    // qualifies (one kernel variant per plan; each scan then gets the layout
    // its one-scan call would take).
    bool zlanes = op == APRICT_BATCH_BACKPROJECT && n_scans > 0;
    bool tall = true;  // every scan at least 256 voxels tall: 8 voxels per thread, as the one-scan call
    for (int i = 0; zlanes && i < n_scans; ++i) {
        const aprict_backproject_config *cfg = static_cast<const aprict_backproject_config *>(configs) + i;
        const int xb = batch_xb(ab_bp::bp_ord(&scans[i].vol), cfg->exact != 0);
        zlanes = ab_bp::bp_zlanes_ok(&scans[i].vol, &scans[i].projs, xb, cfg) && batch_xb(3, cfg->exact != 0) == xb;
        tall = tall && scans[i].vol.nz >= 256u;
    }
    const bool zl8 = zlanes && tall && ab_tuning_get(AB_TUNE_BP_XB) == 0;
    for (int i = 0; i < n_scans; ++i) {
        const aprict_scan &sc = scans[i];
        int rc;
        if (op == APRICT_BATCH_PROJECT) {
            const aprict_project_config *cfg = static_cast<const aprict_project_config *>(configs) + i;
            rc = ab_fp::fp_check(sc.specs_dev, &sc.projs, sc.projs_dev, &sc.vol, sc.vol_dev, cfg);
            if (rc != APRICT_OK) return scan_error(rc, i);
            all_small = all_small && ab_fp::small_volume(&sc.vol);
            all_ss1 = all_ss1 && cfg->ssu == 1 && cfg->ssv == 1;
            uint64_t u = 0;
            fp32[i] = ab_fp::make_fpscan<int32_t>(sc.specs_dev, &sc.projs, sc.projs_dev, sc.base_dev, &sc.vol,
                                                  sc.vol_dev, cfg, sc.status_dev, u);
            fp64[i] = ab_fp::make_fpscan<int64_t>(sc.specs_dev, &sc.projs, sc.projs_dev, sc.base_dev, &sc.vol,
                                                  sc.vol_dev, cfg, sc.status_dev, u);
            units[i] = u;
        } else {
            const aprict_backproject_config *cfg = static_cast<const aprict_backproject_config *>(configs) + i;
            int xb = 0, ord = -1;
            uint64_t u = 0;
            rc = ab_bp::make_bp_params(sc.specs_dev, &sc.projs, sc.projs_dev, &sc.vol, sc.vol_dev, sc.multiplier_dev,
                                       cfg, sc.status_dev, bp[i], u, xb,
                                       zl8 ? 8 : batch_xb(ab_bp::bp_ord(&sc.vol), cfg->exact != 0),
                                       zlanes ? &ord : nullptr);
            if (rc != APRICT_OK) return scan_error(rc, i);
            const int v = ord == 3 ? (xb == 8 ? 16 : 15) : bp_variant(cfg, &sc.vol);
            if (variant >= 0 && v != variant)
                return ab_fail(APRICT_ERR_INVALID_ARGUMENT,
                               "scan %d: every scan of a backprojection batch needs the same volume order, "
                               "slice form (one z layer or more) and backprojection mode (exact / fast / raycast, "
                               "nearest / bilinear)",
                               i);
            variant = v;
            units[i] = u;
        }
    }
    // projection variant: bit 0 = 64-bit offsets, bit 1 = sub-rays (ssu or ssv > 1)
    if (op == APRICT_BATCH_PROJECT) variant = (all_small ? 0 : 1) | (all_ss1 ? 0 : 2);

    // Largest scans first; zero-unit scans are kept (they take no units).
    std::vector<int> order(n_scans);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return units[a] > units[b]; });

    char *base = static_cast<char *>(plan_host);
    memset(base, 0, need);
    PlanHeader *H = reinterpret_cast<PlanHeader *>(base);
    H->magic = kPlanMagic;
    H->op = op;
    H->n_scans = n_scans;
    H->variant = variant;
    H->n_groups = n_groups_of(n_scans);
    H->groups_off = align256(sizeof(PlanHeader));
    H->params_off = H->groups_off + (size_t)H->n_groups * align256(sizeof(Group));
    H->bytes = need;
    for (int gi = 0; gi < H->n_groups; ++gi) {
        Group *G = reinterpret_cast<Group *>(base + H->groups_off + (size_t)gi * align256(sizeof(Group)));
        G->first = (uint32_t)(gi * kGroup);
        G->count = (uint32_t)std::min(kGroup, n_scans - gi * kGroup);
        uint64_t acc = 0;
        for (uint32_t k = 0; k < G->count; ++k) {
            G->prefix[k] = (uint32_t)acc;
            acc += units[order[G->first + k]];
        }
        for (uint32_t k = G->count; k <= (uint32_t)kGroup; ++k) G->prefix[k] = (uint32_t)acc;
        if (acc >= 0x7fffffffull) return ab_fail(APRICT_ERR_TOO_LARGE, "batch has too many work units");
        G->n_units = (uint32_t)acc;
        int rc = APRICT_OK;
        if (G->n_units > 0) {
            if (op == APRICT_BATCH_PROJECT) {
                switch (variant) {
                    case 0: rc = grid_for(k_batch_project<int32_t, true>, G->n_units, G->grid); break;
                    case 1: rc = grid_for(k_batch_project<int64_t, true>, G->n_units, G->grid); break;
                    case 2: rc = grid_for(k_batch_project<int32_t, false>, G->n_units, G->grid); break;
                    default: rc = grid_for(k_batch_project<int64_t, false>, G->n_units, G->grid); break;
                }
            } else {
                rc = with_bp_kernel(variant, [&](auto k) { return grid_for(k, G->n_units, G->grid); });
            }
        }
        if (rc != APRICT_OK) return rc;
    }
    char *params = base + H->params_off;
    for (int k = 0; k < n_scans; ++k) {
        const int i = order[k];
        if (op == APRICT_BATCH_PROJECT) {
            if ((variant & 1) == 0)
                memcpy(params + k * sizeof(ab_fp::FPScan<int32_t>), &fp32[i], sizeof(ab_fp::FPScan<int32_t>));
            else
                memcpy(params + k * sizeof(ab_fp::FPScan<int64_t>), &fp64[i], sizeof(ab_fp::FPScan<int64_t>));
        } else {
            memcpy(params + k * sizeof(ab_bp::BPParams), &bp[i], sizeof(ab_bp::BPParams));
        }
    }
    return APRICT_OK;
}

extern "C" int aprict_b200_batch_run(const void *plan_host, void *plan_dev, aprict_stream_t stream) {
    if (plan_host == nullptr || plan_dev == nullptr)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "batch run needs the host plan and its device copy");
    if (reinterpret_cast<uintptr_t>(plan_dev) & 255u)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "device plan must be 256-byte aligned");
    const PlanHeader *H = static_cast<const PlanHeader *>(plan_host);
    if (H->magic != kPlanMagic) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "not a batch plan");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const char *hb = static_cast<const char *>(plan_host);
    char *db = static_cast<char *>(plan_dev);
    const char *params = hb + H->params_off;
    for (int gi = 0; gi < H->n_groups; ++gi) {
        const size_t off = H->groups_off + (size_t)gi * align256(sizeof(Group));
        const Group &gh = *reinterpret_cast<const Group *>(hb + off);
        Group *gd = reinterpret_cast<Group *>(db + off);
        int rc;
        if (H->op == APRICT_BATCH_PROJECT) {
            using F32 = ab_fp::FPScan<int32_t>;
            using F64 = ab_fp::FPScan<int64_t>;
            switch (H->variant) {
                case 0: rc = launch_group<F32>(k_batch_project<int32_t, true>, H, gh, gd, params, st); break;
                case 1: rc = launch_group<F64>(k_batch_project<int64_t, true>, H, gh, gd, params, st); break;
                case 2: rc = launch_group<F32>(k_batch_project<int32_t, false>, H, gh, gd, params, st); break;
                case 3: rc = launch_group<F64>(k_batch_project<int64_t, false>, H, gh, gd, params, st); break;
                default: return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "corrupt batch plan (variant %d)", H->variant);
            }
        } else {
            rc = with_bp_kernel(H->variant, [&](auto k) {
                return launch_group<ab_bp::BPParams>(k, H, gh, gd, params, st);
            });
        }
        if (rc != APRICT_OK) return rc;
    }
    return APRICT_OK;
}

// ---------------------------------------------------------------------------
// Batch run without a caller-provided device plan: the work counters live in
// a fixed static device array instead (no allocation anywhere on this path).

static constexpr size_t kStaticScratchBytes = 8192;  // header slot + 15 launch groups (1440 scans)
static __device__ __align__(256) unsigned char g_batch_scratch[kStaticScratchBytes];
static constexpr int kMaxDevices = 64;
static void *g_scratch_addr[kMaxDevices] = {};

extern "C" int aprict_b200_batch_run_static(const void *plan_host, aprict_stream_t stream) {
    if (plan_host == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "batch run needs the host plan");
    const PlanHeader *H = static_cast<const PlanHeader *>(plan_host);
    if (H->magic != kPlanMagic) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "not a batch plan");
    // The kernels touch only the Group counters of the device copy, at the
    // offsets the host image gives them.
    const size_t need = H->groups_off + (size_t)H->n_groups * align256(sizeof(Group));
    if (need > kStaticScratchBytes)
        return ab_fail(APRICT_ERR_TOO_LARGE,
                       "plan has %d launch groups (%d scans); the static scratch holds at most %zu groups (%zu scans)",
                       H->n_groups, H->n_scans, (kStaticScratchBytes - H->groups_off) / align256(sizeof(Group)),
                       (kStaticScratchBytes - H->groups_off) / align256(sizeof(Group)) * (size_t)kGroup);
    int dev = 0;
    int rc = ab_cuda_check(cudaGetDevice(&dev), "batch_run_static: cudaGetDevice");
    if (rc != APRICT_OK) return rc;
    if (dev < 0 || dev >= kMaxDevices) return ab_fail(APRICT_ERR_TOO_LARGE, "device ordinal %d out of range", dev);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    void *scratch = __atomic_load_n(&g_scratch_addr[dev], __ATOMIC_ACQUIRE);
    cudaError_t e = cudaErrorInvalidValue;
    // Two tries: a device reset since the address was cached invalidates it,
    // and the memset then fails; look the array up again once.
    for (int attempt = 0; attempt < 2; ++attempt) {
        if (scratch == nullptr) {
            // First call on this device (or after a reset): look up the array's
            // address (this can load the module, so make the first call before
            // any stream capture).
            rc = ab_cuda_check(cudaGetSymbolAddress(&scratch, g_batch_scratch),
                               "batch_run_static: cudaGetSymbolAddress");
            if (rc != APRICT_OK) return rc;
            __atomic_store_n(&g_scratch_addr[dev], scratch, __ATOMIC_RELEASE);
        }
        // Counters start at zero for every call, whatever an earlier call left.
        e = cudaMemsetAsync(scratch, 0, need, st);
        if (e == cudaSuccess || attempt == 1 || (e != cudaErrorInvalidValue && e != cudaErrorContextIsDestroyed))
            break;
        (void)cudaGetLastError();  // the failed memset's (non-sticky) error
        scratch = nullptr;
        __atomic_store_n(&g_scratch_addr[dev], scratch, __ATOMIC_RELEASE);
    }
    rc = ab_cuda_check(e, "batch_run_static: clearing the counters");
    if (rc != APRICT_OK) return rc;
    return aprict_b200_batch_run(plan_host, scratch, stream);
}
