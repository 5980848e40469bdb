// pf_solver.h -- host-side orchestration of the POLFED path on one device.
#pragma once
#include <functional>
#include <vector>

#include "pf_internal.h"

namespace pf {

pf_op *create_spin_chain(pf_handle *h, int L, int Lup, int nbonds, const int32_t *bonds, const double *J,
                         const double *Delta, const double *fields);
pf_op *create_qsun(pf_handle *h, int L_loc, int L_grain, double g0, const double *coup, const int32_t *nbr,
                   const double *fields, const double *grain);
pf_op *create_csr(pf_handle *h, int64_t D, int64_t nnz, const int64_t *indptr, const int32_t *indices,
                  const double *values);
// A complex Hermitian CSR matrix (values interleaved re, im) as its real
// embedding (pf_op.complex_dim = D, dim = 2 D).
pf_op *create_csr_hermitian(pf_handle *h, int64_t D, int64_t nnz, const int64_t *indptr, const int32_t *indices,
                            const double *values);
// polfed on a complex Hermitian operator: x0, vecs complex (interleaved)
// column-major; nev eigenpairs of H.
void solve_hermitian(pf_op *op, const pf_params *P, int s, int nev, const double *x0, int x0_mem, double *vals,
                     double *vecs, int vecs_mem, pf_report *rep, int *nconv);
// An OP_CSR operator that takes ownership of device arrays (cudaMalloc'd on
// h's device): row pointers (D + 1), column indices and values in both
// precisions (nnz each).
pf_op *adopt_csr(pf_handle *h, int64_t D, int64_t nnz, int64_t *dptr, int32_t *didx, double *dv64, float *dv32);
// The Quantum Sun for spin S = two_S / 2 (QuantumSun.jl) or its total-S_z
// sector (u1 != 0, S_z = two_Sz / 2; QuantumSun_U1_conserving.jl), built as a
// CSR matrix on the device.  grain: the final dg x dg grain block
// (dg = (two_S + 1)^L_grain, row-major, already normalised and, for the
// sector, masked to equal grain magnetisation).
pf_op *create_qsun_spin(pf_handle *h, int L_loc, int L_grain, int two_S, int u1, int two_Sz, double g0,
                        const double *coup, const int32_t *nbr, const double *fields, const double *grain);
void destroy_op(pf_op *op);
pf_op *bind_op(const pf_op *src, pf_handle *h);
void *handle_scratch(pf_handle *h, size_t bytes);

void op_apply(pf_op *op, int dtype, double a, double b, int s, const void *X, int64_t ldx, void *Y, int64_t ldy);
void op_apply_noalloc(pf_op *op, int dtype, double a, double b, int s, const void *X, int64_t ldx, void *Y,
                      int64_t ldy);
void op_recurrence(pf_op *op, int dtype, double a, double b, double c, int s, void *b1, const void *b2,
                   const void *b3, const void *X, int64_t ld);
void op_finalsum(pf_op *op, int dtype, double a, double b, double c0, int s, const void *b1, const void *b2,
                 void *Y, const void *X, int64_t ld);
void op_filter(pf_op *op, int dtype, double a, double b, int K, const double *coeffs, int s, const void *X,
               int64_t ldx, void *Y, int64_t ldy);
void op_kpm(pf_op *op, int dtype, double a, double b, int N, int R, const void *probes, int64_t ldp,
            int probe_kind, uint64_t seed, double *mu);

void solve(pf_op *op, const pf_params *p, int s, int nev, const double *x0, int x0_mem, double *vals,
           double *vecs, int vecs_mem, pf_report *rep, int *nconv);
void lanczos_extrema(pf_op *op, const double *x0_host, int maxdim, double tol, double eigentol, double *Emin,
                     double *Emax);

extern thread_local int t_new_handle_priority;

// split-BF16 Gram product on the tensor cores (pf_tc.cu)
size_t gram_bf16_workspace(int64_t D, int nB, int s);
void gram_bf16x3(pf_handle *h, cudaStream_t st, int64_t D, int nB, const double *B, int ldb, const double *r, int s,
                 double *G, void *work, int *err);
void op_gram_bf16x3(pf_handle *h, int64_t D, int nB, const double *B, int64_t ldb, const double *r, int s, double *G);

// fused s-column block passes of a Lanczos iteration (pf_blocks.cu)
constexpr int kBlkMaxS = 32;
enum : int { BLK_SOLVE = 1, BLK_GRAM = 2, BLK_APPEND = 4 };
enum : int { EPI_GRAM = 0, EPI_CHOL = 1, EPI_CHOL_BETA = 2, EPI_ALPHA = 3 };
struct BlkPass {
    int64_t D = 0;
    int s = 0, flags = 0, epi = EPI_GRAM;
    double *W = nullptr;               // RI block (D x s); solved in place with BLK_SOLVE
    const double *Y = nullptr;         // Gram W^T Y (overlap); null: W^T W
    const double *Rs = nullptr;        // BLK_SOLVE: R (upper, column-major s x s)
    double *basis = nullptr;           // BLK_APPEND: row-major basis, row stride ldb, at column col
    int64_t ldb = 0;
    int col = 0;
    double *partial = nullptr;         // blk_partial_doubles(D, s)
    unsigned *counter = nullptr;       // blk_counters() counters, zero before the first pass (each pass leaves them zero)
    double *G = nullptr;               // BLK_GRAM: the Gram matrix (full, column-major s x s)
    double *R = nullptr;               // EPI_CHOL*: this pass's Cholesky factor
    const double *rtot_in = nullptr;   // EPI_CHOL*: running product so far (null: I)
    double *rtot_out = nullptr;        // EPI_CHOL*: R * rtot_in
    int *flag = nullptr;               // EPI_CHOL*: set on a rejected pivot (then R = I)
    double *T = nullptr;               // EPI_CHOL_BETA / EPI_ALPHA: T (column-major, ldT)
    int ldT = 0, k = 0;                // beta at rows k, columns k - s (and transpose); alpha at (k, k)
    double *keep = nullptr;            // EPI_CHOL_BETA: beta; EPI_ALPHA: alpha (symmetric)
};
size_t blk_partial_doubles(int64_t D, int s);
int blk_counters();   // the counters a pass needs (all zero before the first pass)
void blk_pass(cudaStream_t st, const BlkPass &p);
void blk_update(cudaStream_t st, int64_t D, int s, double *r, const double *V, const double *Vp, const double *alpha,
                const double *beta);
void small_chol(cudaStream_t st, const double *G, int s, double *R, const double *rtot_in, double *rtot_out,
                int *flag);

// filter engine (pf_engine.cu): one step launch for every filter in flight
void build_multi_tables(pf_op *op);
bool multi_eligible(const pf_op *op, int dtype);
pf_engine *engine_create(int device);
void engine_destroy(pf_engine *eng);
void engine_stats(pf_engine *eng, double *launches, double *seconds, double *bytes, double *instance_steps);
void engine_filter(pf_engine *eng, pf_op *op, cudaStream_t st, int elem, int s, int V,
                   const std::vector<double> &coeffs, double a, double b, void *X, void *Y, void *A, void *B);

// request pool (pf_pool.cpp)
double solve_footprint(const pf_op *op, const pf_params *p, int s, int nev);
pf_pool *pool_create(int device, int workers, double budget);
void pool_destroy(pf_pool *pool);
void pool_shutdown(pf_pool *pool);
void pool_set_batching(pf_pool *pool, int on);
cudaStream_t pool_stream(pf_pool *pool, int worker);
void pool_set_priority_dim(pf_pool *pool, int64_t dim);
void pool_set_admission(pf_pool *pool, int policy, double max_wait);
int64_t pool_submit(pf_pool *pool, pf_op *op, const pf_params *p, int s, int nev, const double *x0,
                    double *vecs_out, int vecs_mem);
int pool_solve_batch(pf_pool *pool, int n, pf_op *const *ops, const pf_params *const *params, const int *s,
                     const int *nev, const double *const *x0, int x0_mem, double *const *vals, double *const *vecs,
                     int vecs_mem, pf_report *reports, int *nconv, std::string &first_error);
int pool_poll(pf_pool *pool, int64_t id);
int pool_fetch(pf_pool *pool, int64_t id, double timeout_s, double *vals, pf_report *rep, int *nconv,
               std::string &error);
void pool_cancel(pf_pool *pool, int64_t id);
void pool_stats(pf_pool *pool, pf_pool_stats *st);
void pool_request_times(pf_pool *pool, int64_t id, double *times);
int pool_wait(pf_pool *pool, int64_t id, double timeout_s);

}  // namespace pf
