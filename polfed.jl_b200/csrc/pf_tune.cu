// pf_tune.cu -- the step-kernel autotuner.
//
// The Clenshaw / KPM / apply step can give each thread 1..16 columns of a
// row (more columns per thread amortise the per-row basis-state, diagonal
// and flip-rank work; fewer raise occupancy and parallelism), or, for chain
// operators, share each row among s lanes of a warp (width 0, the
// warp-cooperative step).  The best choice depends on the model, s, dtype
// and D, so it is measured: every
// valid width runs the recurrence step (the filter's dominant launch) on
// scratch blocks, timed with CUDA events on the handle's stream, and the
// fastest is cached on the operator for all later launches.
#include "pf_internal.h"

#include <algorithm>
#include <vector>

namespace pf {

template <typename T>
static int tune_typed(pf_op *op, int s, std::vector<std::pair<int, float>> *timings) {
    pf_handle *h = op->h;
    cudaStream_t st = h->stream;
    const int64_t D = op->dim;
    const size_t n = (size_t)D * s;
    T *buf = nullptr;
    PF_CUDA(cudaMalloc(&buf, 3 * n * sizeof(T)));
    T *q = buf, *p = buf + n, *x = buf + 2 * n;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int best = default_width(s, (int)sizeof(T));
    try {
        launch_probes<T>(st, D, s, PF_PROBE_GAUSSIAN, 1, 0, q);
        launch_probes<T>(st, D, s, PF_PROBE_GAUSSIAN, 2, 0, p);
        launch_probes<T>(st, D, s, PF_PROBE_GAUSSIAN, 3, 0, x);
        PF_CUDA(cudaEventCreate(&e0));
        PF_CUDA(cudaEventCreate(&e1));
        const int vmax = 64 / (int)sizeof(T);
        float best_ms = 1e30f;
        const int reps = 20;
        // The recurrence b_k = c X + 2 Ht b_{k+1} - b_{k+2} with a norm-preserving
        // scaling (alpha = 0.5, beta = -0.25) keeps the scratch data bounded.
        std::vector<int> widths;
        for (int V = 1; V <= vmax; V *= 2)
            if (s % V == 0) widths.push_back(V);
        if (coop_eligible(op, s, StepFlags::Q | StepFlags::P | StepFlags::X)) widths.push_back(kCoopWidth);
        for (int V : widths) {
            for (int r = 0; r < 3; ++r)
                launch_step_width<T>(op, st, D, s, q, p, x, p, 0.1, 0.5, -0.25, 0.05, 0.0,
                                     StepFlags::Q | StepFlags::P | StepFlags::X, nullptr, V);
            PF_CUDA(cudaEventRecord(e0, st));
            for (int r = 0; r < reps; ++r)
                launch_step_width<T>(op, st, D, s, q, p, x, p, 0.1, 0.5, -0.25, 0.05, 0.0,
                                     StepFlags::Q | StepFlags::P | StepFlags::X, nullptr, V);
            PF_CUDA(cudaEventRecord(e1, st));
            PF_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            PF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            ms /= reps;
            if (timings) timings->push_back({V, ms});
            if (ms < best_ms) { best_ms = ms; best = V; }
        }
    } catch (...) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaFree(buf);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PF_CUDA(cudaFree(buf));
    std::lock_guard<std::mutex> lock(op->tune_mu);
    op->tuned_width[std::make_pair((int)sizeof(T), s)] = best;
    return best;
}

int autotune_step(pf_op *op, int s, int dtype, std::vector<std::pair<int, float>> *timings) {
    PF_CHECK(s >= 1, PF_ERR_INVALID, "s must be positive");
    PF_CUDA(cudaSetDevice(op->h->device));
    if (dtype == PF_F64) return tune_typed<double>(op, s, timings);
    if (dtype == PF_F32) return tune_typed<float>(op, s, timings);
    throw Error(PF_ERR_INVALID, "dtype must be PF_F64 or PF_F32");
}

}  // namespace pf
