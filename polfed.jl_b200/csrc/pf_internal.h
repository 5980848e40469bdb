// pf_internal.h -- internal types shared by the kernels, the solver and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>
#include <stdint.h>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include <stdexcept>

#include "../../include/polfed_b200.h"

#define PF_MAX_BONDS 64
#define PF_MAX_SITES 32
#define PF_MAX_GRAIN 16   // dg = 2^L_grain <= 16
#define PF_MAX_LOC   32

namespace pf {

// ---------------------------------------------------------------- errors
struct Error : std::runtime_error {
    int code;
    // set when the request itself cannot be met (a planning bisection has no
    // bracket: no interval around the target holds nev states, or no order
    // meets the cutoff there), as opposed to a failure while solving
    bool infeasible = false;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string &msg);

#define PF_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            throw ::pf::Error(e_ == cudaErrorMemoryAllocation ? PF_ERR_NOMEM : PF_ERR_CUDA, \
                              std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)
#define PF_CUBLAS(call)                                                                 \
    do {                                                                                \
        cublasStatus_t e_ = (call);                                                     \
        if (e_ != CUBLAS_STATUS_SUCCESS)                                                \
            throw ::pf::Error(PF_ERR_CUDA, std::string(#call) + ": cublas status " +    \
                                               std::to_string((int)e_));                \
    } while (0)
#define PF_CUSOLVER(call)                                                               \
    do {                                                                                \
        cusolverStatus_t e_ = (call);                                                   \
        if (e_ != CUSOLVER_STATUS_SUCCESS)                                              \
            throw ::pf::Error(PF_ERR_CUDA, std::string(#call) + ": cusolver status " +  \
                                               std::to_string((int)e_));                \
    } while (0)
#define PF_CHECK(cond, code, msg)                                                       \
    do {                                                                                \
        if (!(cond)) throw ::pf::Error((code), (msg));                                  \
    } while (0)

// ------------------------------------------------------- operator descriptors
// Both descriptors are passed to kernels by value (kernel parameter space), so
// every thread of a warp reads the same bond / flip entry at the same time and
// the access is a broadcast.

// Spin-1/2 chain on an Sz sector (or the full 2^L space when full != 0).
template <typename T>
struct ChainDesc {
    int L, Lup, nb, nchunks, full;
    uint32_t bmask[PF_MAX_BONDS];  // (1 << i) | (1 << j)
    uint8_t bi[PF_MAX_BONDS], bj[PF_MAX_BONDS];
    T jhalf[PF_MAX_BONDS];         // J_b / 2            (off-diagonal element)
    T jdq[PF_MAX_BONDS];           // J_b * Delta_b / 4  (Sz Sz with Sz = +-1/2)
    T hhalf[PF_MAX_SITES];         // h_i / 2            (h Sz with Sz = +-1/2)
    const uint32_t *states;        // D basis states (sector only)
    const uint32_t *rank_tab;      // chunked rank tables (sector only)
    const T *diag;                 // D diagonal elements (k_chain_diag), or null
};

// Spin-1/2 Quantum Sun in the full space; grain = the low L_grain bits.
template <typename T>
struct QSunDesc {
    int L, L_grain, L_loc, dg;
    uint32_t fmask[PF_MAX_LOC];     // (1 << (L_grain + j)) | (1 << nbr[j])
    uint8_t site[PF_MAX_LOC];       // L_grain + j
    T cflip[PF_MAX_LOC];            // g0 * coup[j] / 4
    T hhalf[PF_MAX_LOC];            // h_j / 2
    T grain[PF_MAX_GRAIN * PF_MAX_GRAIN];  // row-major dg x dg
};

// A user-supplied real symmetric sparse matrix in CSR form (row pointers,
// column indices and values per row, any column order; the diagonal is an
// ordinary entry).
template <typename T>
struct CsrDesc {
    const int64_t *indptr;   // D + 1
    const int32_t *indices;  // nnz
    const T *values;         // nnz
};

enum OpKind { OP_CHAIN = 0, OP_QSUN = 1, OP_CSR = 2 };

// Number of entries of the chunked rank table for an L-bit sector:
// chunk c (bits 8c..8c+7) holds (8c+1) x 256 entries.
__host__ __device__ inline int rank_table_entries(int nchunks) {
    int n = 0;
    for (int c = 0; c < nchunks; ++c) n += (8 * c + 1) * 256;
    return n;
}
__host__ __device__ inline int rank_table_offset(int c) {
    int n = 0;
    for (int q = 0; q < c; ++q) n += (8 * q + 1) * 256;
    return n;
}

}  // namespace pf

// ------------------------------------------------------------ opaque handles
struct pf_engine;
struct pf_handle {
    int device = 0;
    int num_sms = 148;
    int priority = 0;                 // CUDA stream priority (lower = more urgent)
    cudaStream_t stream = nullptr;
    cublasHandle_t blas = nullptr;
    cusolverDnHandle_t solver = nullptr;
    // per-handle scratch, grown on demand
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    double *red_partials = nullptr;   // deterministic reduction partials
    size_t red_partials_len = 0;
    unsigned int *red_counter = nullptr;
    // second handle of the same device for work that runs beside this one's
    // (the two extremal Lanczos probes); created on first use
    pf_handle *aux = nullptr;
    std::mutex aux_mu;
    // filter engine of the pool this handle works for (not owned); null: the
    // handle runs its own graph-captured filters
    pf_engine *engine = nullptr;
    // page-locked staging for the solver's small host<->device transfers
    // (pageable copies are staged by the driver synchronously and serialise
    // concurrent solves); grown on demand
    void *pinned = nullptr;
    size_t pinned_bytes = 0;
    // timing events of the solver's stage clocks, kept for reuse (creating
    // events every iteration costs host time that stalls the stream)
    std::vector<cudaEvent_t> timing_events;
    // step kernels launch with programmatic dependent launch (each one's
    // launch and shared-memory set-up overlap its predecessor's tail)
    bool overlap = true;
};

struct pf_op {
    pf_handle *h = nullptr;
    int kind = 0;
    int64_t dim = 0;
    int L = 0, Lup = -1;
    pf::ChainDesc<double> chain64;
    pf::ChainDesc<float> chain32;
    pf::QSunDesc<double> qsun64;
    pf::QSunDesc<float> qsun32;
    pf::CsrDesc<double> csr64{};
    pf::CsrDesc<float> csr32{};
    int64_t nnz = 0;
    // > 0: the real embedding [[A, -B], [B, A]] of a complex Hermitian H = A + iB
    // of this dimension (dim = 2 complex_dim); solved by solve_hermitian
    int64_t complex_dim = 0;
    uint32_t *d_states = nullptr;
    uint32_t *d_rank_tab = nullptr;
    double *d_diag64 = nullptr;       // chain diagonal in each precision (warp-cooperative step)
    float *d_diag32 = nullptr;
    // owns d_states / d_rank_tab; shared with the views pf_op_bind makes on other handles
    std::shared_ptr<void> tables_owner;
    // device copies of the descriptors, read by the multi-instance step kernel
    // of the filter engine; shared with views
    void *d_desc64 = nullptr, *d_desc32 = nullptr;
    std::shared_ptr<void> multi_owner;
    // Quantum Sun: the tiled step's shared-memory tables, ready-made (owned
    // by tables_owner)
    void *d_qtab64 = nullptr, *d_qtab32 = nullptr;
    int smem_bytes = 0;               // dynamic shared memory of the step kernels
    int slab_cols = 0;                // filter column slabs: 0 automatic, > 0 forced width, < 0 never
    // autotuned columns-per-thread of the step kernel, keyed by (element bytes, s)
    std::mutex tune_mu;
    std::map<std::pair<int, int>, int> tuned_width;
    // host copies of the defining parameters (for reports and re-creation)
    std::vector<int32_t> bonds;
    std::vector<double> J, Delta, fields, coup, grain;
    std::vector<int32_t> nbr;
    double g0 = 0.0;
    int L_loc = 0, L_grain = 0;
};

namespace pf {

// ------------------------------------------------------------ kernel API
// A "block" here is row-interleaved (RI): element (row i, column c) at i*s + c.

struct StepFlags {
    enum : int { Q = 1, P = 2, X = 4, DOTS = 8 };
};

// out = cx*X + alpha*Htilde(q) + beta*p   (RI layout, s columns)
//   Htilde q = (H q - shift q) * inva
// flags select which of q / p / X take part; DOTS accumulates per column
// <out,out> and <out,q> into dots[2*s] (deterministic two-stage reduction).
// ld > 0: the blocks' row stride when only s of their columns take part (a
// column slab of a wider RI block); stream != 0: x, p and out move with
// evict-first cache hints.
template <typename T>
void launch_step(pf_op *op, cudaStream_t st, int64_t D, int s, const T *q, const T *p,
                 const T *x, T *out, double cx, double alpha, double beta, double inva,
                 double shift, int flags, double *dots, int ld = 0, int stream = 0);

// Same with an explicit columns-per-thread width V (s % V == 0, V*sizeof(T) <= 64),
// or V == kCoopWidth: the warp-cooperative chain step (coop_eligible).
template <typename T>
void launch_step_width(pf_op *op, cudaStream_t st, int64_t D, int s, const T *q, const T *p, const T *x, T *out,
                       double cx, double alpha, double beta, double inva, double shift, int flags, double *dots,
                       int V, int ld = 0, int stream = 0);
int default_width(int s, int elem_bytes);
constexpr int kCoopWidth = 0;
// A step-kernel variant code: columns per thread V (bits 0-7) and a profile
// (bits 8+; 0 = default gather batch and register cap, 1..4 = the tuned
// (batch, resident CTAs) pairs (8,2) (8,3) (4,4) (8,4), 5 = asynchronous
// gathers, 6 / 8 / 9 = shared-memory row tiles of 1 / 2 / 4 rows per thread,
// all three Quantum Sun only, 7 = local flip-rank updates, sector-basis
// chains only), or kCoopWidth for the warp-cooperative chain step.
constexpr int kStepProfiles = 9;
// Profile 5: the Quantum Sun step with asynchronous (cp.async) row gathers;
// profiles 6, 8, 9: the Quantum Sun step over shared-memory tiles of
// 2^t rows (one, two or four rows per thread); profile 7: the sector-basis
// chain step with local flip-rank updates.
constexpr int kProfileAsync = 5;
constexpr int kProfileTile = 6;
constexpr int kProfileLocalRank = 7;
constexpr int kProfileTile2 = 8;
constexpr int kProfileTile4 = 9;
bool qsun_async_eligible(const pf_op *op, int s, int V, int elem);
// rows per thread of a tiled profile (0: not a tiled profile)
int qsun_tile_ipt(int profile);
bool qsun_tile_eligible(const pf_op *op, int s, int V, int elem, int profile);
// Builds the tiled step's model tables (padded grain block and per-byte
// diagonal sums) in device memory for both precisions.
void build_qsun_tables(pf_op *op);
constexpr int variant_code(int V, int profile) { return V | (profile << 8); }
constexpr int variant_width(int code) { return code & 0xff; }
constexpr int variant_profile(int code) { return code >> 8; }
bool coop_eligible(const pf_op *op, int s, int flags);
// Diagonal of a chain operator in both precisions (same term order as the step kernels).
void build_chain_diag(pf_op *op);
// Times every columns-per-thread width of the Clenshaw step for (s, dtype) on
// scratch blocks and records the fastest in op->tuned_width.  Returns it.
int autotune_step(pf_op *op, int s, int dtype, std::vector<std::pair<int, float>> *timings);
extern thread_local bool t_refuse_spilling;
// Measured throughput (bytes/s) of random 32-byte-per-thread row gathers from
// an L2-resident block of 2^log2_rows 64-byte rows.
double gather_peak(pf_handle *h, int log2_rows);
// Take the variant for (s, dtype) from the persistent tuning cache, if it holds
// one for this device, model and size; returns whether it did.
bool cached_step_variant(pf_op *op, int s, int dtype);
// (gather batch U, resident CTAs per SM) of a variant code for element size elem.
void variant_params(int code, int elem, int *V, int *U, int *MB);

// RI <-> column-major conversion, optional precision change.
template <typename TS, typename TD>
void launch_cm_to_ri(cudaStream_t st, int64_t D, int s, const TS *src, int64_t ld, TD *dst);
template <typename TS, typename TD>
void launch_ri_to_cm(cudaStream_t st, int64_t D, int s, const TS *src, TD *dst, int64_t ld);

// Per-column dot products of RI blocks: out[c] = sum_i A[i,c] * B[i,c] (FP64 result).
template <typename T>
void launch_coldots(pf_handle *h, cudaStream_t st, int64_t D, int s, const T *A, const T *B,
                    double *out);
// out[c] = || HA[:,c] - e[c] A[:,c] ||^2  (RI blocks, FP64)
void launch_colresid(pf_handle *h, cudaStream_t st, int64_t D, int s, const double *HA,
                     const double *A, const double *e, double *out);

// Probe generation (RI, D x R): Gaussian or Rademacher from a counter hash.
template <typename T>
void launch_probes(cudaStream_t st, int64_t D, int R, int kind, uint64_t seed, int col0, T *dst);
template <typename T>
void launch_scale_cols(cudaStream_t st, int64_t D, int s, T *A, const double *scale);

void launch_unrank(pf_op *op, cudaStream_t st, int64_t n, const int64_t *idx, uint64_t *out);
void launch_rank(pf_op *op, cudaStream_t st, int64_t n, const uint64_t *states, int64_t *out);

// grid sizing helper: persistent grid of num_sms * blocks_per_sm CTAs at most
int grid_for(pf_handle *h, int64_t work_items, int threads, int blocks_per_sm);

void ensure_reduction(pf_handle *h, size_t n);

// Launches of this library's kernels issued by the calling host thread (a
// graph replay counts every kernel node).  A solve runs on one host thread, so
// the difference across a solve is exactly that solve's launches.
void count_launches(int64_t n);
int64_t thread_launches();

}  // namespace pf
