// pf_capi.cu -- the extern "C" boundary of libpolfed_b200.so.
// Every entry point converts C++ exceptions into a status code plus a
// thread-local message (pf_last_error), so nothing but ints and plain
// pointers crosses the ABI.
#include "pf_internal.h"
#include "pf_solver.h"

#include <cstring>
#include <string>

namespace pf {
static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }
// Stream priority for handles created by this thread (the pool and the
// auxiliary handles set it around their pf_handle_create calls).
thread_local int t_new_handle_priority = 0;
}  // namespace pf

// Every entry point leaves the calling thread's current CUDA device as it
// found it (the library switches to a handle's device internally), so a
// caller working on another GPU is not moved.
struct DeviceRestore {
    int dev = -1;
    DeviceRestore() {
        if (cudaGetDevice(&dev) != cudaSuccess) {
            dev = -1;
            cudaGetLastError();
        }
    }
    ~DeviceRestore() {
        if (dev >= 0) cudaSetDevice(dev);
    }
};

#define PF_API_BEGIN      \
    DeviceRestore pf_dev_restore_; \
    try {
#define PF_API_END                                              \
    return PF_OK;                                               \
    }                                                           \
    catch (const pf::Error &e) {                                \
        pf::set_last_error(e.what());                           \
        return e.code;                                          \
    }                                                           \
    catch (const std::bad_alloc &) {                            \
        pf::set_last_error("host allocation failed");           \
        return PF_ERR_NOMEM;                                    \
    }                                                           \
    catch (const std::exception &e) {                           \
        pf::set_last_error(e.what());                           \
        return PF_ERR_CUDA;                                     \
    }

extern "C" {

int pf_abi_version(void) { return PF_ABI_VERSION; }
void pf_abi_sizes(size_t *params, size_t *report, size_t *pool_stats) {
    if (params) *params = sizeof(pf_params);
    if (report) *report = sizeof(pf_report);
    if (pool_stats) *pool_stats = sizeof(pf_pool_stats);
}

const char *pf_last_error(void) { return pf::g_last_error.c_str(); }

int pf_handle_create(int device, pf_handle **out) {
    PF_API_BEGIN
    PF_CHECK(out != nullptr, PF_ERR_INVALID, "null output pointer");
    int ndev = 0;
    PF_CUDA(cudaGetDeviceCount(&ndev));
    PF_CHECK(device >= 0 && device < ndev, PF_ERR_INVALID, "no such CUDA device");
    PF_CUDA(cudaSetDevice(device));
    {
        // solver workspaces are allocated stream-ordered from the device pool;
        // keep freed memory in the pool so later allocations never synchronise
        cudaMemPool_t pool;
        PF_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t keep = UINT64_MAX;
        PF_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    cudaDeviceProp prop;
    PF_CUDA(cudaGetDeviceProperties(&prop, device));
    PF_CHECK(prop.major >= 10, PF_ERR_UNSUPPORTED, "libpolfed_b200 is built for sm_100a (B200) only");
    pf_handle *h = new pf_handle();
    h->device = device;
    h->num_sms = prop.multiProcessorCount;
    try {
        h->priority = pf::t_new_handle_priority;
        PF_CUDA(cudaStreamCreateWithPriority(&h->stream, cudaStreamNonBlocking, h->priority));
        PF_CUBLAS(cublasCreate(&h->blas));
        PF_CUBLAS(cublasSetStream(h->blas, h->stream));
        PF_CUSOLVER(cusolverDnCreate(&h->solver));
        PF_CUSOLVER(cusolverDnSetStream(h->solver, h->stream));
        PF_CUDA(cudaMalloc(&h->red_counter, 64 * sizeof(unsigned int)));
        PF_CUDA(cudaMemset(h->red_counter, 0, 64 * sizeof(unsigned int)));
    } catch (...) {
        if (h->blas) cublasDestroy(h->blas);
        if (h->solver) cusolverDnDestroy(h->solver);
        if (h->stream) cudaStreamDestroy(h->stream);
        delete h;
        throw;
    }
    *out = h;
    PF_API_END
}

int pf_handle_destroy(pf_handle *h) {
    PF_API_BEGIN
    if (!h) return PF_OK;
    if (h->aux) pf_handle_destroy(h->aux);
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->blas) cublasDestroy(h->blas);
    if (h->solver) cusolverDnDestroy(h->solver);
    if (h->scratch) cudaFree(h->scratch);
    if (h->red_partials) cudaFree(h->red_partials);
    if (h->red_counter) cudaFree(h->red_counter);
    if (h->pinned) cudaFreeHost(h->pinned);
    for (cudaEvent_t e : h->timing_events) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    PF_API_END
}

int pf_handle_stream(pf_handle *h, void **stream) {
    PF_API_BEGIN
    PF_CHECK(h && stream, PF_ERR_INVALID, "null argument");
    *stream = (void *)h->stream;
    PF_API_END
}

int pf_handle_synchronize(pf_handle *h) {
    PF_API_BEGIN
    PF_CHECK(h, PF_ERR_INVALID, "null handle");
    PF_CUDA(cudaSetDevice(h->device));
    PF_CUDA(cudaStreamSynchronize(h->stream));
    PF_API_END
}

int pf_handle_set_overlap(pf_handle *h, int on) {
    PF_API_BEGIN
    PF_CHECK(h, PF_ERR_INVALID, "null handle");
    h->overlap = on != 0;
    PF_API_END
}

int pf_op_spin_chain_create(pf_handle *h, int L, int Lup, int nbonds, const int32_t *bonds, const double *J,
                            const double *Delta, const double *fields, pf_op **out) {
    PF_API_BEGIN
    PF_CHECK(out != nullptr, PF_ERR_INVALID, "null output pointer");
    *out = pf::create_spin_chain(h, L, Lup, nbonds, bonds, J, Delta, fields);
    PF_API_END
}

int pf_op_qsun_create(pf_handle *h, int L_loc, int L_grain, double g0, const double *coup, const int32_t *nbr,
                      const double *fields, const double *grain, pf_op **out) {
    PF_API_BEGIN
    PF_CHECK(out != nullptr, PF_ERR_INVALID, "null output pointer");
    *out = pf::create_qsun(h, L_loc, L_grain, g0, coup, nbr, fields, grain);
    PF_API_END
}

int pf_op_qsun_spin_create(pf_handle *h, int L_loc, int L_grain, int two_S, int u1, int two_Sz, double g0,
                           const double *coup, const int32_t *nbr, const double *fields, const double *grain,
                           pf_op **out) {
    PF_API_BEGIN
    PF_CHECK(out != nullptr, PF_ERR_INVALID, "null output pointer");
    *out = pf::create_qsun_spin(h, L_loc, L_grain, two_S, u1, two_Sz, g0, coup, nbr, fields, grain);
    PF_API_END
}

int pf_op_csr_create_hermitian(pf_handle *h, int64_t D, int64_t nnz, const int64_t *indptr,
                               const int32_t *indices, const double *values, pf_op **out) {
    PF_API_BEGIN
    PF_CHECK(out != nullptr, PF_ERR_INVALID, "null output pointer");
    *out = pf::create_csr_hermitian(h, D, nnz, indptr, indices, values);
    PF_API_END
}

int pf_op_csr_create(pf_handle *h, int64_t D, int64_t nnz, const int64_t *indptr, const int32_t *indices,
                     const double *values, pf_op **out) {
    PF_API_BEGIN
    PF_CHECK(out != nullptr, PF_ERR_INVALID, "null output pointer");
    *out = pf::create_csr(h, D, nnz, indptr, indices, values);
    PF_API_END
}

int pf_op_bind(const pf_op *op, pf_handle *h, pf_op **out) {
    PF_API_BEGIN
    PF_CHECK(out != nullptr, PF_ERR_INVALID, "null output pointer");
    *out = pf::bind_op(op, h);
    PF_API_END
}

int pf_op_destroy(pf_op *op) {
    PF_API_BEGIN
    pf::destroy_op(op);
    PF_API_END
}

int64_t pf_op_dim(const pf_op *op) { return op ? op->dim : -1; }

int pf_basis_unrank(pf_op *op, int64_t n, const int64_t *idx, uint64_t *states) {
    PF_API_BEGIN
    PF_CHECK(op && (n == 0 || (idx && states)), PF_ERR_INVALID, "null argument");
    PF_CHECK(op->kind == pf::OP_CHAIN, PF_ERR_UNSUPPORTED, "basis rank/unrank applies to spin-chain operators");
    PF_CUDA(cudaSetDevice(op->h->device));
    pf::launch_unrank(op, op->h->stream, n, idx, states);
    PF_API_END
}

int pf_basis_rank(pf_op *op, int64_t n, const uint64_t *states, int64_t *idx) {
    PF_API_BEGIN
    PF_CHECK(op && (n == 0 || (idx && states)), PF_ERR_INVALID, "null argument");
    PF_CHECK(op->kind == pf::OP_CHAIN, PF_ERR_UNSUPPORTED, "basis rank/unrank applies to spin-chain operators");
    PF_CUDA(cudaSetDevice(op->h->device));
    pf::launch_rank(op, op->h->stream, n, states, idx);
    PF_API_END
}

int pf_apply(pf_op *op, int dtype, double a, double b, int s, const void *X, int64_t ldx, void *Y, int64_t ldy) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    pf::op_apply(op, dtype, a, b, s, X, ldx, Y, ldy);
    PF_API_END
}

int pf_apply_noalloc(pf_op *op, int dtype, double a, double b, int s, const void *X, int64_t ldx, void *Y,
                     int64_t ldy) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    pf::op_apply_noalloc(op, dtype, a, b, s, X, ldx, Y, ldy);
    PF_API_END
}

int pf_clenshaw_recurrence(pf_op *op, int dtype, double a, double b, double c, int s, void *b1, const void *b2,
                           const void *b3, const void *X, int64_t ld) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    pf::op_recurrence(op, dtype, a, b, c, s, b1, b2, b3, X, ld);
    PF_API_END
}

int pf_clenshaw_finalsum(pf_op *op, int dtype, double a, double b, double c0, int s, const void *b1, const void *b2,
                         void *Y, const void *X, int64_t ld) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    pf::op_finalsum(op, dtype, a, b, c0, s, b1, b2, Y, X, ld);
    PF_API_END
}

int pf_filter(pf_op *op, int dtype, double a, double b, int K, const double *coeffs, int s, const void *X,
              int64_t ldx, void *Y, int64_t ldy) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    pf::op_filter(op, dtype, a, b, K, coeffs, s, X, ldx, Y, ldy);
    PF_API_END
}

int pf_kpm_moments(pf_op *op, int dtype, double a, double b, int N, int R, const void *probes, int64_t ldp,
                   int probe_kind, uint64_t seed, double *mu) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    pf::op_kpm(op, dtype, a, b, N, R, probes, ldp, probe_kind, seed, mu);
    PF_API_END
}

int pf_autotune(pf_op *op, int dtype, int s, int *width, float *times_ms) {
    PF_API_BEGIN
    PF_CHECK(op && width, PF_ERR_INVALID, "null argument");
    std::vector<std::pair<int, float>> t;
    const int code = pf::autotune_step(op, s, dtype, &t);
    *width = code == PF_WIDTH_COOP ? PF_WIDTH_COOP : pf::variant_width(code);
    if (times_ms) {
        for (int i = 0; i < 6; ++i) times_ms[i] = 0.f;
        for (auto &pr : t) {
            int idx = 5;  // PF_WIDTH_COOP
            if (pr.first != PF_WIDTH_COOP) {
                const int w = pf::variant_width(pr.first);
                idx = 0;
                while ((1 << idx) < w) ++idx;
            }
            // the fastest profile of each width
            if (idx < 6 && (times_ms[idx] == 0.f || pr.second < times_ms[idx])) times_ms[idx] = pr.second;
        }
    }
    PF_API_END
}

int pf_gram_bf16x3(pf_handle *h, int64_t D, int nB, const double *B, int64_t ldb, const double *r, int s,
                   double *G) {
    PF_API_BEGIN
    pf::op_gram_bf16x3(h, D, nB, B, ldb, r, s, G);
    PF_API_END
}

int pf_gather_peak(pf_handle *h, int log2_rows, double *bytes_per_s) {
    PF_API_BEGIN
    PF_CHECK(h && bytes_per_s, PF_ERR_INVALID, "null argument");
    *bytes_per_s = pf::gather_peak(h, log2_rows);
    PF_API_END
}

int pf_step_variant(pf_op *op, int dtype, int s, int *width, int *gather_batch, int *ctas_per_sm) {
    PF_API_BEGIN
    PF_CHECK(op && width && gather_batch && ctas_per_sm, PF_ERR_INVALID, "null argument");
    PF_CHECK(dtype == PF_F64 || dtype == PF_F32, PF_ERR_INVALID, "dtype must be PF_F64 or PF_F32");
    PF_CHECK(s >= 1, PF_ERR_INVALID, "s must be positive");
    const int elem = dtype == PF_F64 ? 8 : 4;
    int code = pf::default_width(s, elem);
    {
        std::lock_guard<std::mutex> lock(op->tune_mu);
        auto it = op->tuned_width.find(std::make_pair(elem, s));
        if (it != op->tuned_width.end()) code = it->second;
    }
    pf::variant_params(code, elem, width, gather_batch, ctas_per_sm);
    PF_API_END
}

int pf_step_profile(pf_op *op, int dtype, int s, int *profile) {
    PF_API_BEGIN
    PF_CHECK(op && profile, PF_ERR_INVALID, "null argument");
    PF_CHECK(dtype == PF_F64 || dtype == PF_F32, PF_ERR_INVALID, "dtype must be PF_F64 or PF_F32");
    PF_CHECK(s >= 1, PF_ERR_INVALID, "s must be positive");
    const int elem = dtype == PF_F64 ? 8 : 4;
    int code = pf::default_width(s, elem);
    {
        std::lock_guard<std::mutex> lock(op->tune_mu);
        auto it = op->tuned_width.find(std::make_pair(elem, s));
        if (it != op->tuned_width.end()) code = it->second;
    }
    *profile = code == PF_WIDTH_COOP ? 0 : pf::variant_profile(code);
    PF_API_END
}

int pf_set_step_variant(pf_op *op, int dtype, int s, int width, int profile) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    PF_CHECK(profile >= 0 && profile <= pf::kStepProfiles, PF_ERR_INVALID, "profile must be in 0..9");
    PF_CHECK(width != PF_WIDTH_COOP || profile == 0, PF_ERR_INVALID, "the warp-cooperative step has no profiles");
    PF_CHECK(profile != pf::kProfileAsync || pf::qsun_async_eligible(op, s, width, dtype == PF_F64 ? 8 : 4),
             PF_ERR_INVALID,
             "asynchronous gathers (profile 5) need a Quantum Sun operator and 16- or 32-byte column segments");
    PF_CHECK(pf::qsun_tile_ipt(profile) == 0 || pf::qsun_tile_eligible(op, s, width, dtype == PF_F64 ? 8 : 4, profile),
             PF_ERR_INVALID,
             "row tiles (profiles 6, 8, 9) need a Quantum Sun operator with at least one tile of states, a power-of-two "
             "number of column groups and at most 64 KB per tile");
    PF_CHECK(profile != pf::kProfileLocalRank || (op->kind == pf::OP_CHAIN && op->Lup >= 0), PF_ERR_INVALID,
             "local flip-rank updates (profile 7) need a spin-chain operator on an Sz sector");
    const int st = pf_set_step_width(op, dtype, s, width);
    if (st != PF_OK) return st;
    std::lock_guard<std::mutex> lock(op->tune_mu);
    op->tuned_width[std::make_pair(dtype == PF_F64 ? 8 : 4, s)] = pf::variant_code(width, profile);
    PF_API_END
}

int pf_set_filter_slab(pf_op *op, int cols) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    op->slab_cols = cols;
    PF_API_END
}

int pf_set_step_width(pf_op *op, int dtype, int s, int width) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    PF_CHECK(dtype == PF_F64 || dtype == PF_F32, PF_ERR_INVALID, "dtype must be PF_F64 or PF_F32");
    PF_CHECK(s >= 1, PF_ERR_INVALID, "s must be positive");
    const int elem = dtype == PF_F64 ? 8 : 4;
    if (width == PF_WIDTH_COOP) {
        PF_CHECK(pf::coop_eligible(op, s, pf::StepFlags::Q | pf::StepFlags::P | pf::StepFlags::X), PF_ERR_INVALID,
                 "the warp-cooperative step needs a chain operator and s in {4, 8, 16, 32}");
    } else {
        PF_CHECK(width >= 1 && (width & (width - 1)) == 0 && s % width == 0 && width * elem <= 64, PF_ERR_INVALID,
                 "width must be a power of two dividing s with at most 64 bytes of columns");
    }
    std::lock_guard<std::mutex> lock(op->tune_mu);
    op->tuned_width[std::make_pair(elem, s)] = width;
    PF_API_END
}

void pf_params_default(pf_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->target_kind = PF_TARGET_MAXDOS;
    p->target_value = 0.0;
    p->order = 0;
    p->cutoff = 0.17;               // PolfedDefaults.jl:119
    p->normalization = 1.0;         // :126
    p->order_safety_factor = 0.97;  // :133
    p->tol = 1e-14;                 // :177
    p->eigentol = 1e-9;             // :184
    p->overestimate_iters = 1.25;   // :151
    p->which = PF_WHICH_LR;         // :191
    p->dos_N = 250;                 // :210
    p->dos_R = 300;                 // :217
    p->dos_kernel = PF_KERNEL_JACKSON;
    p->probe_kind = PF_PROBE_GAUSSIAN;
    p->seed = 0x5eed5eedULL;
    p->probes = nullptr;
    p->precision = PF_PREC_FP64;
    p->reorth_passes = 1;
    p->extrema_maxdim = 1000;       // Plan.jl:143,160
    p->refine = 4;                  // FP64 refinement passes of the mixed-precision solve
    p->autotune = 1;
    p->host_qr = 0;
}

int pf_solve(pf_op *op, const pf_params *params, int s, int nev, const double *x0, int x0_mem, double *vals,
             double *vecs, int vecs_mem, pf_report *report, int *nconv) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    PF_CHECK(op->complex_dim == 0, PF_ERR_INVALID, "a Hermitian operator is solved with pf_solve_hermitian");
    pf::solve(op, params, s, nev, x0, x0_mem, vals, vecs, vecs_mem, report, nconv);
    PF_API_END
}

int pf_solve_hermitian(pf_op *op, const pf_params *params, int s, int nev, const double *x0, int x0_mem,
                       double *vals, double *vecs, int vecs_mem, pf_report *report, int *nconv) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    pf::solve_hermitian(op, params, s, nev, x0, x0_mem, vals, vecs, vecs_mem, report, nconv);
    PF_API_END
}

int pf_lanczos_extrema(pf_op *op, const double *x0, int maxdim, double tol, double eigentol, double *Emin,
                       double *Emax) {
    PF_API_BEGIN
    PF_CHECK(op, PF_ERR_INVALID, "null operator");
    pf::lanczos_extrema(op, x0, maxdim, tol, eigentol, Emin, Emax);
    PF_API_END
}

// ------------------------------------------------------------- request pool
int pf_pool_create(int device, int workers, double hbm_budget, pf_pool **out) {
    PF_API_BEGIN
    PF_CHECK(out != nullptr, PF_ERR_INVALID, "null output pointer");
    *out = pf::pool_create(device, workers, hbm_budget);
    PF_API_END
}

int pf_pool_destroy(pf_pool *pool) {
    PF_API_BEGIN
    pf::pool_destroy(pool);
    PF_API_END
}

int pf_pool_shutdown(pf_pool *pool) {
    PF_API_BEGIN
    pf::pool_shutdown(pool);
    PF_API_END
}

int pf_pool_stream(pf_pool *pool, int worker, void **stream) {
    PF_API_BEGIN
    PF_CHECK(pool && stream, PF_ERR_INVALID, "null argument");
    *stream = (void *)pf::pool_stream(pool, worker);
    PF_API_END
}

int pf_pool_set_admission(pf_pool *pool, int policy, double max_wait_s) {
    PF_API_BEGIN
    pf::pool_set_admission(pool, policy, max_wait_s);
    PF_API_END
}

int pf_pool_set_batching(pf_pool *pool, int on) {
    PF_API_BEGIN
    pf::pool_set_batching(pool, on);
    PF_API_END
}

int pf_pool_set_priority_dim(pf_pool *pool, int64_t dim) {
    PF_API_BEGIN
    pf::pool_set_priority_dim(pool, dim);
    PF_API_END
}

double pf_solve_footprint(const pf_op *op, const pf_params *params, int s, int nev) {
    if (!op || !params || s < 1 || nev < 1) return -1.0;
    return pf::solve_footprint(op, params, s, nev);
}

int pf_pool_solve_batch(pf_pool *pool, int n, pf_op *const *ops, const pf_params *const *params, const int *s,
                        const int *nev, const double *const *x0, int x0_mem, double *const *vals,
                        double *const *vecs, int vecs_mem, pf_report *reports, int *nconv) {
    PF_API_BEGIN
    std::string err;
    int st = pf::pool_solve_batch(pool, n, ops, params, s, nev, x0, x0_mem, vals, vecs, vecs_mem, reports, nconv, err);
    if (st != PF_OK) throw pf::Error(st, err);
    PF_API_END
}

int pf_pool_submit(pf_pool *pool, pf_op *op, const pf_params *params, int s, int nev, const double *x0,
                   double *vecs_out, int vecs_mem, int64_t *request) {
    PF_API_BEGIN
    PF_CHECK(request != nullptr, PF_ERR_INVALID, "null output pointer");
    *request = pf::pool_submit(pool, op, params, s, nev, x0, vecs_out, vecs_mem);
    PF_API_END
}

int pf_pool_poll(pf_pool *pool, int64_t request, int *state) {
    PF_API_BEGIN
    PF_CHECK(pool && state, PF_ERR_INVALID, "null argument");
    *state = pf::pool_poll(pool, request);
    PF_API_END
}

int pf_pool_fetch(pf_pool *pool, int64_t request, double timeout_s, double *vals, pf_report *report, int *nconv) {
    PF_API_BEGIN
    PF_CHECK(pool, PF_ERR_INVALID, "null pool");
    std::string err;
    int st = pf::pool_fetch(pool, request, timeout_s, vals, report, nconv, err);
    if (st != PF_OK) throw pf::Error(st, err);
    PF_API_END
}

int pf_pool_cancel(pf_pool *pool, int64_t request) {
    PF_API_BEGIN
    PF_CHECK(pool, PF_ERR_INVALID, "null pool");
    pf::pool_cancel(pool, request);
    PF_API_END
}

int pf_pool_wait(pf_pool *pool, int64_t request, double timeout_s, int *state) {
    PF_API_BEGIN
    PF_CHECK(pool && state, PF_ERR_INVALID, "null argument");
    *state = pf::pool_wait(pool, request, timeout_s);
    PF_API_END
}

int pf_pool_request_times(pf_pool *pool, int64_t request, double *times) {
    PF_API_BEGIN
    PF_CHECK(pool && times, PF_ERR_INVALID, "null argument");
    pf::pool_request_times(pool, request, times);
    PF_API_END
}

int pf_pool_get_stats(pf_pool *pool, pf_pool_stats *stats) {
    PF_API_BEGIN
    PF_CHECK(pool && stats, PF_ERR_INVALID, "null argument");
    pf::pool_stats(pool, stats);
    PF_API_END
}

}  // extern "C"
