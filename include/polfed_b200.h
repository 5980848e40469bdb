/*
 * polfed_b200.h -- C ABI of the B200 (sm_100a) POLFED filter-and-Lanczos library.
 *
 * Every entry point returns an int status (PF_OK == 0).  On failure
 * pf_last_error() returns a thread-local message.  No C++ exception and no
 * torch type crosses this boundary; arrays are plain pointers plus sizes.
 * A handle owns one CUDA stream plus workspaces; handles are independent and
 * may be used from different host threads, but one handle is not re-entrant.
 * Every entry point returns with the calling thread's current CUDA device
 * unchanged (work runs on the handle's device whatever is current).
 *
 * Matrix-shaped arguments are column-major with a leading dimension, like a
 * Julia CuArray / Array.  "device" pointers are CUDA global memory on the
 * handle's device; "host" pointers are ordinary (pageable or pinned) memory.
 *
 * Reference interfaces replaced (Polfed.jl, file:line within that project):
 *   operators          Models/SpinHalfChains.jl:74-99 (xxz_hamiltonian),
 *                      :189-220 (j1j2_hamiltonian), :267-315 (matrix elements);
 *                      QSun/QuantumSun.jl:1-102 (qsun_hamiltonian, S = 1/2)
 *   pf_apply           MappingConfig.f!_rescaled, Polfed/Plan/Plan.jl:173-177
 *                      and the plain operator f!, PolfedCore.jl:172
 *   pf_clenshaw_*      MappingConfig.clenshaw_recurrence / clenshaw_finalsum,
 *                      Polfed/Structs/MappingConfig.jl:35-45; the CUDA.jl
 *                      kernels of Optimization/gpu/vector_dispatch.jl:113-139
 *   pf_filter          the whole Clenshaw loop, Clenshaw/Algorithm/ClenshawAlgorithm.jl:12-29
 *   pf_kpm_moments     dos_moments, DensetiesOfStates/Moments.jl:42-140
 *   pf_solve           polfed(f!, x0, howmany, target; ...), Polfed/PolfedCore.jl:194-263
 *   pf_lanczos_extrema lanczos_extrema, Lanczos/Lanczos.jl:183-212
 */
#ifndef POLFED_B200_H
#define POLFED_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PF_ABI_VERSION 1

/* status codes */
#define PF_OK              0
#define PF_ERR_INVALID     1  /* bad argument (ArgumentError / DimensionMismatch) */
#define PF_ERR_CUDA        2  /* CUDA runtime / cuBLAS / cuSOLVER failure */
#define PF_ERR_NOMEM       3  /* device allocation failed */
#define PF_ERR_NUMERIC     4  /* non-finite values, failed bisection bracket, ... */
#define PF_ERR_UNSUPPORTED 5

/* element types */
#define PF_F64 0
#define PF_F32 1

/* memory spaces */
#define PF_MEM_HOST   0
#define PF_MEM_DEVICE 1

/* target kinds (Polfed/Structs/TargetSpec.jl:26-58) */
#define PF_TARGET_MAXDOS     0  /* :maxdos */
#define PF_TARGET_MIDDLE     1  /* :middle */
#define PF_TARGET_OFFSET     2  /* (:offset, eta) */
#define PF_TARGET_UNRESCALED 3  /* (:unrescaled, E) or a plain number */
#define PF_TARGET_RESCALED   4  /* (:rescaled, eps) */

/* eigenvalue selection (Lanczos/Convergence/EigSorter.jl) */
#define PF_WHICH_SR 0
#define PF_WHICH_LR 1

/* DoS damping kernels (DensetiesOfStates/Kernels.jl:33-72) */
#define PF_KERNEL_JACKSON    0
#define PF_KERNEL_LORENTZ    1
#define PF_KERNEL_FEJER      2
#define PF_KERNEL_LANCZOS    3
#define PF_KERNEL_WANGZUNGER 4
#define PF_KERNEL_DIRICHLET  5

/* KPM probe vectors */
#define PF_PROBE_GAUSSIAN   0  /* randn, normalised per column (Moments.jl:101-102) */
#define PF_PROBE_RADEMACHER 1  /* +-1/sqrt(D) */

/* solve precision */
#define PF_PREC_FP64  0  /* FP64 throughout (the reference's arithmetic) */
#define PF_PREC_MIXED 1  /* FP32 filter and KPM; FP64 Lanczos basis, Ritz vectors,
                             residuals and pf_params.refine FP64 refinement passes */

typedef struct pf_handle pf_handle;
typedef struct pf_op pf_op;

/* ------------------------------------------------------------ library */
int         pf_abi_version(void);
/* sizeof(pf_params), sizeof(pf_report) and sizeof(pf_pool_stats) as this
 * library was compiled, for bindings that mirror the structs (any pointer
 * may be NULL). */
void        pf_abi_sizes(size_t *params, size_t *report, size_t *pool_stats);
const char *pf_last_error(void);

int pf_handle_create(int device, pf_handle **out);
int pf_handle_destroy(pf_handle *h);
/* The handle's cudaStream_t, for callers that order their own work with it. */
int pf_handle_stream(pf_handle *h, void **stream);
int pf_handle_synchronize(pf_handle *h);
/* on != 0 (the default): the handle's step kernels launch with programmatic
 * dependent launch -- a step's launch and shared-memory table set-up overlap
 * the previous step's tail, and it waits for that step's writes before
 * reading any block; 0: plain stream order.  Results are identical. */
int pf_handle_set_overlap(pf_handle *h, int on);

/* ---------------------------------------------------------- operators */
/* Spin-1/2 chain  H = sum_b J_b (S+_i S-_j + h.c.)/2 + J_b Delta_b Sz_i Sz_j
 *                   + sum_i h_i Sz_i
 * on the sector of states with Lup up spins (Lup < 0: the full 2^L space).
 * bonds holds 2*nbonds 0-based sites (i0, j0, i1, j1, ...), as returned by
 * _chain_bonds with 1 subtracted.  Host arrays are copied.  L <= 32, nbonds <= 64.
 * Replaces SpinHalfChains.jl:267-315 (_spin_half_hamiltonian). */
int pf_op_spin_chain_create(pf_handle *h, int L, int Lup, int nbonds, const int32_t *bonds,
                            const double *J, const double *Delta, const double *fields,
                            pf_op **out);
/* Quantum Sun (S = 1/2, full space of L_loc + L_grain spins), QuantumSun.jl:1-102:
 * coup[j] = g0-free couplings alpha^{u_j}, nbr[j] in [0, L_grain), fields[j] = h_j,
 * grain = the dg x dg grain block (row-major, dg = 2^L_grain <= 16), already
 * scaled by gamma / sqrt(dg + 1). */
int pf_op_qsun_create(pf_handle *h, int L_loc, int L_grain, double g0, const double *coup,
                      const int32_t *nbr, const double *fields, const double *grain,
                      pf_op **out);
/* The Quantum Sun for any spin S = two_S / 2 (1/2 .. 15/2; QuantumSun.jl:1-102)
 * in the full space (u1 = 0) or in the total-S_z sector S_z = two_Sz / 2
 * (u1 = 1; QuantumSun_U1_conserving.jl:1-212): localized fields, the S^x S^x
 * (in the sector S^x S^x + S^y S^y) coupling of each localized spin j to grain
 * site nbr[j] with strength g0 * coup[j], and the grain block.  States are
 * indexed as the reference indexes them (sorted packed digit codes: the
 * base-(2S+1) value of the digits, ranked within the sector).  grain is the
 * final dg x dg block (row-major, dg = (2S+1)^L_grain <= 4096): the full space
 * takes gamma GOE / sqrt(dg + 1), the sector the GOE masked to equal grain
 * magnetisation and scaled by gamma / sqrt(tr(R^2) / dim) (R its embedding in
 * the sector).  The matrix is assembled as CSR on the device and applied by
 * the CSR step.  A sector outside [-L S, L S] or off the spin lattice fails
 * with the reference's message. */
int pf_op_qsun_spin_create(pf_handle *h, int L_loc, int L_grain, int two_S, int u1, int two_Sz, double g0,
                           const double *coup, const int32_t *nbr, const double *fields, const double *grain,
                           pf_op **out);
/* A real symmetric sparse matrix (polfed(mat, ...), PolfedCore.jl:153-184,
 * whose operator is mul!(Y, mat, X)): CSR with 0-based row pointers
 * indptr[D + 1] (indptr[0] = 0, indptr[D] = nnz, non-decreasing), column
 * indices in [0, D) and values, host arrays copied.  Symmetry is the
 * caller's contract, as in the reference.  D < 2^31. */
int pf_op_csr_create(pf_handle *h, int64_t D, int64_t nnz, const int64_t *indptr, const int32_t *indices,
                     const double *values, pf_op **out);
/* A complex Hermitian sparse matrix H = A + iB (the reference's CPU path
 * takes complex Hermitian input; its GPU path refuses it, PolfedCore.jl:160-162):
 * CSR as pf_op_csr_create with values[2 nnz] interleaved (re, im) -- the
 * layout of C double _Complex, Julia ComplexF64 and numpy complex128 arrays.
 * Hermiticity is the caller's contract; a diagonal entry with a nonzero
 * imaginary part is refused.  The operator is H's real embedding
 * M = [[A, -B], [B, A]] (pf_op_dim = 2 D; pf_apply applies M to [Re X; Im X])
 * and is solved with pf_solve_hermitian.  D < 2^30. */
int pf_op_csr_create_hermitian(pf_handle *h, int64_t D, int64_t nnz, const int64_t *indptr,
                               const int32_t *indices, const double *values, pf_op **out);
/* A view of op that runs on handle h (same device).  It shares op's device
 * tables, so several host threads can solve concurrently, each on its own
 * handle / stream.  Destroy views and the original in any order; the tables
 * are freed with the last of them.  (No reference counterpart: the reference
 * runs one solve at a time.) */
int     pf_op_bind(const pf_op *op, pf_handle *h, pf_op **out);
int     pf_op_destroy(pf_op *op);
int64_t pf_op_dim(const pf_op *op);

/* Bit-exact basis work (device pointers).  unrank: idx -> basis state;
 * rank: state -> index, or -1 for a state outside the basis. */
int pf_basis_unrank(pf_op *op, int64_t n, const int64_t *idx, uint64_t *states);
int pf_basis_rank(pf_op *op, int64_t n, const uint64_t *states, int64_t *idx);

/* ------------------------------------------- operator-level drop-ins */
/* All block arguments are device pointers, column-major D x s with leading
 * dimension ld >= D, element type dtype (PF_F64 / PF_F32).  Htilde = (H - b)/a;
 * a = 1, b = 0 gives the plain H.  Results are ordered on the handle's stream. */

/* Y = Htilde X                                  (f!_rescaled, Plan.jl:173-177) */
int pf_apply(pf_op *op, int dtype, double a, double b, int s,
             const void *X, int64_t ldx, void *Y, int64_t ldy);
/* b1 = c X + 2 Htilde b2 - b3       (clenshaw_recurrence, vector_dispatch.jl:120-124) */
int pf_clenshaw_recurrence(pf_op *op, int dtype, double a, double b, double c, int s,
                           void *b1, const void *b2, const void *b3, const void *X, int64_t ld);
/* Same result as pf_apply, for callers that cannot let a library allocate
 * device memory (a CuArray / caching-allocator pool that owns the HBM budget,
 * or a loop that cannot absorb cudaMalloc's implicit synchronisation).  This
 * entry point has no counterpart in the reference.  It never allocates: blocks
 * with s > 1 are staged in one fixed 16 MiB device array built into the
 * library (held by every GPU that loads it until exit), so 2*D*s*element_size
 * must not exceed 16 MiB -- larger blocks are rejected with PF_ERR_INVALID.
 * The array's device address is looked up inside the first call on each
 * device; make that first call before any stream capture.  All calls share the
 * array: calls that overlap on the GPU race and must be ordered by the caller. */
int pf_apply_noalloc(pf_op *op, int dtype, double a, double b, int s,
                     const void *X, int64_t ldx, void *Y, int64_t ldy);
/* Y = c0 X + Htilde b1 - b2        (clenshaw_finalsum, vector_dispatch.jl:134-137) */
int pf_clenshaw_finalsum(pf_op *op, int dtype, double a, double b, double c0, int s,
                         const void *b1, const void *b2, void *Y, const void *X, int64_t ld);
/* Y = sum_{k=0}^{K} coeffs[k] T_k(Htilde) X  (ClenshawAlgorithm.jl:12-29); coeffs on host. */
int pf_filter(pf_op *op, int dtype, double a, double b, int K, const double *coeffs,
              int s, const void *X, int64_t ldx, void *Y, int64_t ldy);
/* KPM moments mu[0..N-1] = (D/R) sum_r <r|T_n(Htilde)|r> (Moments.jl:42-140).
 * probes: device D x R column-major with normalised columns, or NULL to draw
 * R probes of probe_kind from seed on the device.  mu is a host array. */
int pf_kpm_moments(pf_op *op, int dtype, double a, double b, int N, int R,
                   const void *probes, int64_t ldp, int probe_kind, uint64_t seed,
                   double *mu);

/* Autotuner (no reference counterpart: the reference has no kernel variants).
 * Times every variant of the Clenshaw step kernel for block width s and dtype
 * on scratch blocks -- 1, 2, 4, 8 or 16 columns per thread, each with five
 * (gather batch, register cap) profiles (and, for the Quantum Sun, the
 * asynchronous-gather and row-tile profiles of pf_set_step_variant; for
 * sector chains the local flip-rank profile), and for chain operators with s in
 * {4, 8, 16, 32} the warp-cooperative step (width PF_WIDTH_COOP: the s lanes
 * of a warp share one row) -- keeps the fastest for this operator and returns
 * its width in *width; times_ms[i] (optional, 6 entries) receives the
 * measured milliseconds per launch of the fastest profile of widths 1, 2, 4,
 * 8, 16 and PF_WIDTH_COOP (0 where not offered).  Every variant computes the
 * same sums in the same order.  The choice is also written to a persistent
 * cache ($POLFED_B200_TUNE_CACHE, else ~/.cache/polfed_b200/step_variants.json)
 * that pf_solve consults before timing. */
#define PF_WIDTH_COOP 0
int pf_autotune(pf_op *op, int dtype, int s, int *width, float *times_ms);
/* G = B^T r on the 5th-generation tensor cores (tcgen05.mma, BF16 inputs,
 * FP32 accumulation) in split BF16: every FP64 value v = hi + lo with
 * hi = bf16(v), lo = bf16(v - hi), and G ~= Bhi^T rhi + Bhi^T rlo + Blo^T rhi,
 * the row chunks' FP32 partial sums added in FP64.  B is row-major D x nB with
 * row stride ldb (the Krylov basis layout), r row-major D x s (s <= 32), G
 * column-major nB x s; all device pointers.  Relative error ~1e-5 of |B| |r|:
 * the first pass of the reorthogonalisation mode reorth_passes = 3 (the
 * Gram contraction of reorthogonalization.jl:77-84).  Synchronises. */
int pf_gram_bf16x3(pf_handle *h, int64_t D, int nB, const double *B, int64_t ldb, const double *r, int s,
                   double *G);
/* Roofline probe (no reference counterpart): the measured throughput, in
 * bytes per second, of random row gathers -- each thread reads 32 bytes of 16
 * rows chosen by a row-XOR pattern, as spin flips do -- from an L2-resident
 * block of 2^log2_rows 64-byte rows (10 <= log2_rows <= 24).  The ceiling of
 * a step kernel whose blocks stay in L2. */
int pf_gather_peak(pf_handle *h, int log2_rows, double *bytes_per_s);
/* The step-kernel variant in use for (dtype, s): columns per thread (0: the
 * warp-cooperative step), gathers issued per batch and the resident CTAs per
 * SM it is compiled for (its register cap). */
int pf_step_variant(pf_op *op, int dtype, int s, int *width, int *gather_batch, int *ctas_per_sm);
/* The profile (0..9, as for pf_set_step_variant) of the variant in use for
 * (dtype, s), so that a variant the autotuner chose can be pinned again with
 * pf_set_step_variant (for instance in another process). */
int pf_step_profile(pf_op *op, int dtype, int s, int *profile);
/* Pin the step-kernel variant for (dtype, s) without timing (a width the
 * autotuner could have chosen); later launches on this operator use it. */
int pf_set_step_width(pf_op *op, int dtype, int s, int width);
/* Same with a profile: 0 = the width's default gather batch and register cap,
 * 1..4 = (8 gathers, 2 CTAs/SM), (8, 3), (4, 4), (8, 4); 5 = Quantum Sun
 * operators only, with 16- or 32-byte column segments: every gather of a row
 * issued at once as an asynchronous global-to-shared copy; 6, 8, 9 = Quantum
 * Sun operators only, contiguous rows, s / width a power of two: each CTA
 * stages a tile of 2^t consecutive rows (every column; 1, 2 or 4 rows per
 * thread, at most 64 KB) in shared memory and serves the grain block and the
 * flips of outer bits below t from it, gathering only the other flips;
 * 7 = spin chains on an Sz sector only: the rank of a state reached by a
 * flip of sites at most two apart is updated from the row's own rank (a few
 * binomial-table reads) instead of re-ranked. */
int pf_set_step_variant(pf_op *op, int dtype, int s, int width, int profile);

/* Column slabs of the filter (no reference counterpart).  cols > 0: filter in
 * slabs of cols columns (a divisor of s), so the block each step gathers from
 * (D x cols) can stay in L2 while the once-touched streams pass with
 * evict-first hints; cols <= 0: whole blocks (the default).  Results are
 * unchanged either way. */
int pf_set_filter_slab(pf_op *op, int cols);

/* ----------------------------------------------------------- solving */
typedef struct pf_params {
    int    target_kind;          /* PF_TARGET_* */
    double target_value;         /* eta, E or eps depending on target_kind */
    int    has_Emin, has_Emax;   /* MappingConfig.Emin / Emax given? */
    double Emin, Emax;
    int    has_left, has_right;  /* TransformConfig.left / right (unrescaled) */
    double left, right;
    int    order;                /* TransformConfig.order, 0 = automatic */
    double cutoff;               /* 0.17 */
    double normalization;        /* 1.0 */
    double order_safety_factor;  /* 0.97 */
    double tol;                  /* 1e-14 */
    double eigentol;             /* 1e-9 */
    double overestimate_iters;   /* 1.25 */
    int    which;                /* PF_WHICH_LR */
    int    dos_N;                /* 250 */
    int    dos_R;                /* 300 */
    int    dos_kernel;           /* PF_KERNEL_JACKSON */
    int    probe_kind;           /* PF_PROBE_GAUSSIAN */
    uint64_t seed;               /* probe seed */
    const double *probes;        /* optional host D x R normalised probes (overrides seed) */
    int    precision;            /* PF_PREC_FP64 */
    int    reorth_passes;        /* 1 = FullRO of the reference; 2 = CGS2 in FP64; 3 = CGS2 whose first
                                    Gram product B^T r runs on the tensor cores in split BF16
                                    (pf_gram_bf16x3), the updates and the second pass in FP64 (s <= 32) */
    int    extrema_maxdim;       /* 1000 (Plan.jl:143,160) */
    int    refine;               /* PF_PREC_MIXED: at most this many FP64 refinement passes (4; 0 = none).
                                    Each applies the FP64 filter to the FP32 run's 2 nev leading Ritz
                                    vectors (nev targets + nev guards, at most the Krylov dimension)
                                    and runs a Rayleigh-Ritz step with the FP64 H on them; passes stop
                                    once all nev targets meet eigentol. */
    int    autotune;             /* 1: time the step-kernel variants once per (op, s, dtype) */
    int    host_qr;              /* 0: the s x s algebra of a Lanczos iteration stays on the device
                                    (a CholQR breakdown restarts the run with the host QR) and each
                                    convergence check runs beside the next iteration; 1: every
                                    iteration reads its Gram matrices back and factors them on the
                                    host (the same R bit for bit; Householder QR on a breakdown) and
                                    checks run in turn.  Both give the same results. */
} pf_params;

#define PF_REPORT_MAX_CHECKS 128

/* Mirrors SpectralTransformReport, FactorizationReport and BenchmarkReport
 * (SpectralTransformReport.jl:30-71, FactorizationReport.jl:48-143,
 * BenchmarkReport.jl:68-129). Times are seconds measured with CUDA events. */
typedef struct pf_report {
    double  Emin, Emax, a, b;
    double  target, left, right;        /* rescaled units */
    int     order;
    double  order_safety_factor;
    int64_t matvecs;                    /* K * s * iters + howmany */
    int64_t kpm_block_matvecs;          /* column-matvecs spent in KPM */
    int     blocksize, howmany;
    int     iters_needed, iters_reserved, krylovdim;
    double  tol, residual;
    int     converged_tol;
    double  eigentol, eigenresidual;
    int     converged_eigentol;
    int     refined;                    /* pairs that met eigentol only after the FP64 refinement
                                           (PF_PREC_MIXED; its time is in stage 5) */
    int     numofchecks;
    int     converged_history[PF_REPORT_MAX_CHECKS];
    int     krylovdim_history[PF_REPORT_MAX_CHECKS];
    double  maxresidual_history[PF_REPORT_MAX_CHECKS];
    /* stage times: 0 tridiagonalization, 1 mapping (filter), 2 overlap,
     * 3 orthogonalization, 4 reorthogonalization, 5 convergence check,
     * 6 Emin/Emax probes, 7 KPM DoS, 8 bounds+order, 9 total */
    double  stage_seconds[10];
    double  basis_bytes_reserved, basis_bytes_used;
    int64_t kernel_launches;            /* this library's kernel launches in the solve */
    int     qr_restarts;                /* Lanczos runs restarted with the host QR: the s x s work of
                                           an iteration runs on the device, and a CholQR pass whose
                                           Gram matrix is not positive definite (a rank-deficient
                                           block) is redone with the host's Householder QR */
} pf_report;

void pf_params_default(pf_params *p);

/* POLFED solve on operator op (PolfedCore.jl:194-263).  x0 is D x s
 * (s == 1: scalar Lanczos), in host or device memory per x0_mem.  Outputs:
 * vals[nev] (host), vecs D x nev column-major (host or device per vecs_mem;
 * may be NULL), report (may be NULL), *nconv = number of returned pairs,
 * sorted ascending (LanczosMethod.jl:74-82). */
int pf_solve(pf_op *op, const pf_params *params, int s, int nev,
             const double *x0, int x0_mem, double *vals, double *vecs, int vecs_mem,
             pf_report *report, int *nconv);
/* POLFED on a complex Hermitian operator (pf_op_csr_create_hermitian).  x0 is
 * D x s complex column-major (interleaved re, im), vecs D x nev complex
 * (interleaved); vals real.  The complex block Lanczos from x0 is run as the
 * real block Lanczos of the embedding from [v, i v] (2s columns, 2 nev pairs:
 * every eigenvalue of H appears twice), and each group of equal eigenvalues
 * is turned back into complex eigenvectors x + iy (one per complex direction,
 * unit norm, arbitrary phase).  The report describes that real run, with
 * blocksize s, howmany nev and converged_eigentol the returned count. */
int pf_solve_hermitian(pf_op *op, const pf_params *params, int s, int nev,
                       const double *x0, int x0_mem, double *vals, double *vecs, int vecs_mem,
                       pf_report *report, int *nconv);

/* ------------------------------------------------ batching and serving */
/* No reference counterpart: the reference solves one problem per call.  A
 * pool owns `workers` handles (one stream each) and a request queue.  Each
 * worker runs one solve at a time; up to `workers` solves are in flight
 * together, so their latency-bound launches and host round trips overlap.
 * A request is admitted when a worker is free and its estimated device
 * footprint fits in what `hbm_budget` (bytes; 0 = 90 % of free memory at
 * creation) leaves; otherwise it waits in FIFO order.  Requests run the
 * same solve as pf_solve and give the same result alone or in a mix.  Each
 * request takes its own view of its operator when it is submitted (device
 * tables and tuned step widths shared), so an operator may be destroyed as
 * soon as the submitting call returns. */
typedef struct pf_pool pf_pool;

typedef struct pf_pool_stats {
    int64_t submitted, completed, failed, queued, running;
    int64_t eigenpairs;            /* converged pairs of completed requests */
    double  bytes_budget, bytes_in_use, bytes_peak;
    double  p50_latency, p99_latency, mean_latency;  /* seconds, submit -> done */
    double  busy_seconds;          /* wall time with at least one request running */
    int64_t rejected;              /* infeasible requests (see PF_REQ_REJECTED) */
    /* the filter engine's batched step launches: number, summed kernel time
     * (CUDA events, seconds), algorithmic bytes moved (streams x D x s x
     * element size per instance-step) and instance-steps served */
    double  filter_launches, filter_seconds, filter_bytes, filter_instance_steps;
} pf_pool_stats;

#define PF_REQ_QUEUED   0
#define PF_REQ_RUNNING  1
#define PF_REQ_DONE     2
#define PF_REQ_FAILED   3
/* The request cannot be met: the density of states holds fewer than nev
 * states within reach of its target, so the interval bisection has no
 * bracket (the reference raises the same error, Bisection.jl:18-40).  It is
 * found in the planning stage, before any Lanczos work; pf_pool_fetch returns
 * PF_ERR_NUMERIC with the reference's message. */
#define PF_REQ_REJECTED 4

int pf_pool_create(int device, int workers, double hbm_budget, pf_pool **out);
/* Stop the pool without freeing it: queued requests fail with
 * PF_ERR_INVALID ("pool destroyed ..."), threads blocked in pf_pool_fetch /
 * pf_pool_wait / pf_pool_solve_batch are woken, running requests finish, and
 * later submissions are refused.  Finished requests can still be fetched. */
int pf_pool_shutdown(pf_pool *pool);
/* pf_pool_shutdown, then free the pool once no thread is inside pf_pool_fetch,
 * pf_pool_wait or pf_pool_solve_batch.  No call may start on the pool once
 * pf_pool_destroy has been called (callers whose threads may still be about
 * to call in use pf_pool_shutdown first and destroy after they are done). */
int pf_pool_destroy(pf_pool *pool);
/* The CUDA streams (cudaStream_t) of the pool: index w < workers is worker
 * w's default-priority stream, workers + w its high-priority stream; for
 * callers that order their own work or timing events against the solves. */
int pf_pool_stream(pf_pool *pool, int worker, void **stream);
/* Batched filtering (default off): the Clenshaw steps of every request in
 * flight run as one multi-instance launch per step on the pool's engine
 * stream (continuous batching: a filter joins at the next step after it is
 * submitted and leaves after its own final sum).  Each instance computes
 * exactly the rows and sums of the per-solve kernel.  Off: every request runs
 * its own graph-captured filter on its worker stream.  Applies to requests
 * that start after the call. */
int pf_pool_set_batching(pf_pool *pool, int on);
/* Requests on operators of dimension <= dim (default 65536; 0: none) run on
 * the workers' high-priority streams, so their short launches are dispatched
 * ahead of the queued launches of larger solves.  Results are unchanged. */
int pf_pool_set_priority_dim(pf_pool *pool, int64_t dim);
/* Admission order.  PF_ADMIT_FIFO (default): arrival order.  PF_ADMIT_SHORTEST:
 * the fitting request of least expected work D^2 (20.427 s + 1.696 nev) / nev
 * first, except that a request queued for max_wait_s seconds goes first in
 * arrival order and nothing overtakes it (no request waits forever). */
#define PF_ADMIT_FIFO     0
#define PF_ADMIT_SHORTEST 1
int pf_pool_set_admission(pf_pool *pool, int policy, double max_wait_s);
/* Estimated device bytes of one solve (what admission charges). */
double pf_solve_footprint(const pf_op *op, const pf_params *params, int s, int nev);
/* Solve n problems concurrently; arrays of length n (params may repeat one
 * struct by passing the same pointer n times).  x0[i] is D x s[i] in x0_mem;
 * vals[i] holds nev[i] doubles; vecs[i] (may be NULL) D x nev[i] in vecs_mem;
 * reports may be NULL.  Returns the first failing status (all are run). */
int pf_pool_solve_batch(pf_pool *pool, int n, pf_op *const *ops, const pf_params *const *params,
                        const int *s, const int *nev, const double *const *x0, int x0_mem,
                        double *const *vals, double *const *vecs, int vecs_mem, pf_report *reports,
                        int *nconv);
/* Queue one solve; x0 (host, D x s) is copied.  vecs_out (may be NULL, host
 * or device per vecs_mem, D x nev) must stay valid until the request is
 * fetched or cancelled. */
int pf_pool_submit(pf_pool *pool, pf_op *op, const pf_params *params, int s, int nev, const double *x0,
                   double *vecs_out, int vecs_mem, int64_t *request);
int pf_pool_poll(pf_pool *pool, int64_t request, int *state);
/* Wait for (timeout_s < 0: indefinitely) and collect a finished request: vals
 * (nev doubles, host), report (may be NULL), *nconv; the request is released.
 * A failed or rejected request returns its error status, and *nconv is then
 * -PF_REQ_FAILED or -PF_REQ_REJECTED. */
int pf_pool_fetch(pf_pool *pool, int64_t request, double timeout_s, double *vals, pf_report *report,
                  int *nconv);
/* Wait (timeout_s < 0: indefinitely) until the request has finished, without
 * collecting it; *state is its PF_REQ_* state when the wait ends. */
int pf_pool_wait(pf_pool *pool, int64_t request, double timeout_s, int *state);
/* Seconds since the pool was created at which the request was submitted,
 * started and finished (times[3]; -1 for what has not happened yet).  Valid
 * until the request is fetched, cancelled or collected. */
int pf_pool_request_times(pf_pool *pool, int64_t request, double *times);
/* Drop a queued request.  A running one finishes and is then discarded: its
 * worker still writes the host output arrays given at submission, which must
 * stay valid until the pool is destroyed. */
int pf_pool_cancel(pf_pool *pool, int64_t request);
int pf_pool_get_stats(pf_pool *pool, pf_pool_stats *stats);

/* (Emin, Emax) from two Lanczos probes on H (Lanczos.jl:183-212); x0 length D (host). */
int pf_lanczos_extrema(pf_op *op, const double *x0, int maxdim, double tol, double eigentol,
                       double *Emin, double *Emax);

#ifdef __cplusplus
}
#endif
#endif /* POLFED_B200_H */
