// ab_sirt.cu -- the reference-mode SIRT iteration as C entry points.
//
// Replaces the loop body of SIRT_flatpanel.iterate
// (src/aprict/iterators/sirt_vram.py:130-152): copy b -> r, project with
// multiply_before_adding = -1, backproject r in chunks of 10 views with the
// preconditioner as summand multiplier, two host synchronisations. Here one
// step is two launches on the caller's stream -- the fused residual
// r = b - A x and one all-view backprojection x += M (.) B r -- and a graph
// of n steps is captured once and replayed with one cudaGraphLaunch.
#include <cuda_runtime.h>

#include <new>

#include "ab_host.h"

struct aprict_sirt_graph {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    int n_iter;
};

namespace {

int sirt_check(const aprict_backproject_config *cfg_bp, const float *M_dev) {
    if (cfg_bp == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null backproject config");
    if (M_dev == nullptr || !cfg_bp->apply_summand_multiplier)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT,
                       "a SIRT step needs the preconditioner as summand multiplier (apply_summand_multiplier = 1)");
    return APRICT_OK;
}

int sirt_step(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd, const float *b_dev, float *r_dev,
              const aprict_vol_desc *vd, float *x_dev, const float *M_dev, const aprict_backproject_config *cfg_bp,
              uint32_t *status_dev, aprict_stream_t stream) {
    const aprict_project_config residual{1.f, -1.f, 1, 1};
    int rc = aprict_b200_project_siddon(specs_dev, pd, r_dev, b_dev, vd, x_dev, &residual, status_dev, stream);
    if (rc != APRICT_OK) return rc;
    return aprict_b200_backproject(specs_dev, pd, r_dev, vd, x_dev, M_dev, cfg_bp, status_dev, stream);
}

}  // namespace

extern "C" int aprict_b200_sirt_step(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                     const float *b_dev, float *r_dev, const aprict_vol_desc *vd, float *x_dev,
                                     const float *M_dev, const aprict_backproject_config *cfg_bp,
                                     uint32_t *status_dev, aprict_stream_t stream) {
    const int rc = sirt_check(cfg_bp, M_dev);
    if (rc != APRICT_OK) return rc;
    return sirt_step(specs_dev, pd, b_dev, r_dev, vd, x_dev, M_dev, cfg_bp, status_dev, stream);
}

extern "C" int aprict_b200_sirt_graph_create(const aprict_proj_spec *specs_dev, const aprict_proj_desc *pd,
                                             const float *b_dev, float *r_dev, const aprict_vol_desc *vd,
                                             float *x_dev, const float *M_dev,
                                             const aprict_backproject_config *cfg_bp, uint32_t *status_dev,
                                             int n_iter, aprict_sirt_graph **out) {
    if (out == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null graph handle pointer");
    *out = nullptr;
    if (n_iter <= 0 || n_iter > 100000) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "n_iter must be in [1, 100000]");
    int rc = sirt_check(cfg_bp, M_dev);
    if (rc != APRICT_OK) return rc;
    cudaStream_t cap = nullptr;
    if ((rc = ab_cuda_check(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "sirt graph: stream")) != APRICT_OK)
        return rc;
    cudaGraph_t graph = nullptr;
    rc = ab_cuda_check(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "sirt graph: begin capture");
    if (rc == APRICT_OK) {
        int step_rc = APRICT_OK;
        for (int i = 0; i < n_iter && step_rc == APRICT_OK; ++i)
            step_rc = sirt_step(specs_dev, pd, b_dev, r_dev, vd, x_dev, M_dev, cfg_bp, status_dev, cap);
        const cudaError_t e = cudaStreamEndCapture(cap, &graph);
        rc = step_rc != APRICT_OK ? step_rc : ab_cuda_check(e, "sirt graph: end capture");
    }
    cudaGraphExec_t exec = nullptr;
    if (rc == APRICT_OK) rc = ab_cuda_check(cudaGraphInstantiate(&exec, graph, 0), "sirt graph: instantiate");
    cudaStreamDestroy(cap);
    if (rc != APRICT_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    aprict_sirt_graph *g = new (std::nothrow) aprict_sirt_graph{graph, exec, n_iter};
    if (g == nullptr) {
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        return ab_fail(APRICT_ERR_CUDA, "sirt graph: out of host memory");
    }
    *out = g;
    return APRICT_OK;
}

extern "C" int aprict_b200_sirt_graph_launch(const aprict_sirt_graph *g, aprict_stream_t stream) {
    if (g == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "null graph");
    return ab_cuda_check(cudaGraphLaunch(g->exec, reinterpret_cast<cudaStream_t>(stream)), "sirt graph: launch");
}

extern "C" int aprict_b200_sirt_graph_iterations(const aprict_sirt_graph *g) { return g ? g->n_iter : 0; }

extern "C" void aprict_b200_sirt_graph_destroy(aprict_sirt_graph *g) {
    if (g == nullptr) return;
    cudaGraphExecDestroy(g->exec);
    cudaGraphDestroy(g->graph);
    delete g;
}
