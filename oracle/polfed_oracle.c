/*
 * polfed_oracle.c -- CPU restatement of the POLFED filter-and-Lanczos hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.  The product (libpolfed_b200.so) never links or calls it.
 *
 * Every routine restates one piece of the reference (Polfed.jl, Julia) in
 * plain C with FP64 arithmetic.  Sites are 0-based here (bit index == site);
 * the reference uses 1-based sites and bit (site-1), which is the same bit.
 *
 *   orc_sector_basis      Models/SpinHalfChains.jl:259-262 (_lup_basis)
 *   orc_sector_rank       Models/SpinHalfChains.jl:278 (Dict state => n)
 *   orc_spin_chain_coo    Models/SpinHalfChains.jl:264-315
 *   orc_qsun_coo          QSun/QuantumSun.jl:1-102, QSun/SpinOperators.jl:147-181
 *   orc_csr_apply         the `mul!(Y, mat, X)` operator of PolfedCore.jl:172
 *   orc_csr_rescaled      Polfed/Plan/Plan.jl:173-177 (f!_rescaled closure)
 *   orc_clenshaw_filter   Clenshaw/Algorithm/ClenshawAlgorithm.jl:12-29 with
 *                         Clenshaw/Clenshaw.jl:69-117,141-153 (Chebyshev)
 *   orc_kpm_trace         DensetiesOfStates/Moments.jl:87-140 (trace!)
 *   orc_bucket_*          the reference's CPU "optimized mapping": off-diagonal
 *                         entries grouped by value (optimization.jl:134-182,
 *                         allocate/pack :229-265), rescaled once
 *                         (optimize_spectral_transform, optimization.jl:75-119),
 *                         applied per bucket (cpu/mapping.jl:27-120,
 *                         single_row_mappings.jl:9-79), the fused Clenshaw row
 *                         kernels (cpu/clenshaw_recurrence_relation.jl:25-134,
 *                         cpu/clenshaw_final_sum.jl:25-137) and the threaded
 *                         KPM over probes (Moments.jl:87-109)
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ basis */

/* Ascending L-bit integers with popcount == Lup (SpinHalfChains.jl:259-262).
 * Lup < 0 selects the full 2^L space (every integer in ascending order).
 * Returns the count; writes states when out != NULL. */
int64_t orc_sector_basis(int L, int Lup, uint64_t *out) {
    int64_t n = 0;
    uint64_t top = (uint64_t)1 << L;
    for (uint64_t st = 0; st < top; ++st) {
        if (Lup >= 0 && __builtin_popcountll(st) != Lup) continue;
        if (out) out[n] = st;
        ++n;
    }
    return n;
}

/* Index of each state in the ascending basis (the Dict lookup of
 * SpinHalfChains.jl:278, 0-based); -1 when the state is not in the basis. */
void orc_sector_rank(int64_t nbasis, const uint64_t *basis, int64_t n,
                     const uint64_t *states, int64_t *idx) {
    for (int64_t q = 0; q < n; ++q) {
        uint64_t key = states[q];
        int64_t lo = 0, hi = nbasis;
        while (lo < hi) {
            int64_t mid = lo + (hi - lo) / 2;
            if (basis[mid] < key) lo = mid + 1; else hi = mid;
        }
        idx[q] = (lo < nbasis && basis[lo] == key) ? lo : -1;
    }
}

static int64_t lookup(int64_t nbasis, const uint64_t *basis, uint64_t key) {
    int64_t r;
    orc_sector_rank(nbasis, basis, 1, &key, &r);
    return r;
}

/* ------------------------------------------------------------- operators */

/* COO triplets of the spin-1/2 chain Hamiltonian, in the order the reference
 * pushes them (SpinHalfChains.jl:284-311): for each column (basis state), one
 * off-diagonal J_b/2 per bond whose two spins differ, then the diagonal
 *   sum_i h_i s^z_i + sum_b J_b Delta_b s^z_i s^z_j.
 * Duplicates are summed later (Julia `sparse` semantics).  Returns the number
 * of triplets; writes them when rows != NULL. */
int64_t orc_spin_chain_coo(int L, int Lup, int nbonds, const int *bi, const int *bj,
                           const double *J, const double *Delta, const double *fields,
                           int64_t *rows, int64_t *cols, double *vals) {
    int64_t D = orc_sector_basis(L, Lup, NULL);
    uint64_t *basis = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(D > 0 ? D : 1));
    orc_sector_basis(L, Lup, basis);
    int64_t nnz = 0;
    for (int64_t col = 0; col < D; ++col) {
        uint64_t st = basis[col];
        double diag = 0.0;
        for (int site = 0; site < L; ++site)
            diag += fields[site] * ((((st >> site) & 1u) == 1u) ? 0.5 : -0.5);
        for (int b = 0; b < nbonds; ++b) {
            double zi = (((st >> bi[b]) & 1u) == 1u) ? 0.5 : -0.5;
            double zj = (((st >> bj[b]) & 1u) == 1u) ? 0.5 : -0.5;
            diag += J[b] * Delta[b] * zi * zj;
            if (zi != zj) {
                uint64_t fl = st ^ ((uint64_t)1 << bi[b]) ^ ((uint64_t)1 << bj[b]);
                if (rows) {
                    rows[nnz] = lookup(D, basis, fl);
                    cols[nnz] = col;
                    vals[nnz] = J[b] / 2;
                }
                ++nnz;
            }
        }
        if (rows) { rows[nnz] = col; cols[nnz] = col; vals[nnz] = diag; }
        ++nnz;
    }
    free(basis);
    return nnz;
}

/* COO triplets of the spin-1/2 Quantum Sun Hamiltonian in the full 2^L space
 * (QuantumSun.jl:1-102 with S = 1/2, so SpinBasis has one bit per site and
 * state_index(state) == state + 1).  Outer spin j (0-based) lives on bit
 * L_grain + j; its field term is h_j s^z; its coupling flips that bit and grain
 * bit nbr[j] with amplitude g0 * coup[j] * (1/2)(1/2) (the sigma_x matrix
 * elements of SpinOperators.jl:167-181 for S = 1/2).  The grain block
 * kron(I, Hg) (QuantumSun.jl:99) adds Hg[g, g'] between states that differ
 * only in their low L_grain bits.  Hg is row-major dg x dg, already scaled by
 * gamma / sqrt(dg + 1). */
int64_t orc_qsun_coo(int L_loc, int L_grain, double g0, const double *coup,
                     const int *nbr, const double *fields, const double *Hg,
                     int64_t *rows, int64_t *cols, double *vals) {
    int L = L_loc + L_grain;
    int64_t D = (int64_t)1 << L;
    int64_t dg = (int64_t)1 << L_grain;
    int64_t nnz = 0;
    for (int64_t k = 0; k < D; ++k) {
        uint64_t st = (uint64_t)k;
        for (int j = 0; j < L_loc; ++j) {
            int site = L_grain + j;
            double m = (double)((st >> site) & 1u) - 0.5;
            if (rows) { rows[nnz] = k; cols[nnz] = k; vals[nnz] = fields[j] * m; }
            ++nnz;
        }
        for (int j = 0; j < L_loc; ++j) {
            int site = L_grain + j;
            /* sigma_x(site) has exactly one branch for S=1/2 (up or down) with
             * coefficient 1/2; so does sigma_x on the grain site. */
            uint64_t s1 = st ^ ((uint64_t)1 << site);
            uint64_t s2 = s1 ^ ((uint64_t)1 << nbr[j]);
            if (rows) { rows[nnz] = (int64_t)s2; cols[nnz] = k; vals[nnz] = g0 * coup[j] * 0.5 * 0.5; }
            ++nnz;
        }
    }
    for (int64_t blk = 0; blk < D / dg; ++blk)
        for (int64_t g = 0; g < dg; ++g)
            for (int64_t h = 0; h < dg; ++h) {
                if (rows) {
                    rows[nnz] = blk * dg + g;
                    cols[nnz] = blk * dg + h;
                    vals[nnz] = Hg[g * dg + h];
                }
                ++nnz;
            }
    return nnz;
}

/* ------------------------------------------------------------ CSR kernels */

/* Y = H X for a CSR matrix and column-major D x s blocks (leading dims ldx,ldy). */
void orc_csr_apply(int64_t D, const int64_t *rowptr, const int64_t *colidx, const double *v,
                   int s, const double *X, int64_t ldx, double *Y, int64_t ldy) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < D; ++i) {
        for (int c = 0; c < s; ++c) {
            double acc = 0.0;
            for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p)
                acc += v[p] * X[colidx[p] + c * ldx];
            Y[i + c * ldy] = acc;
        }
    }
}

/* f!_rescaled of Plan.jl:173-177:  f!(Y, X); Y *= 1/a; Y -= (b/a) * X. */
void orc_csr_rescaled(int64_t D, const int64_t *rowptr, const int64_t *colidx, const double *v,
                      double a, double b, int s, const double *X, int64_t ldx,
                      double *Y, int64_t ldy) {
    double inva = 1.0 / a, boa = b / a;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < D; ++i) {
        for (int c = 0; c < s; ++c) {
            double acc = 0.0;
            for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p)
                acc += v[p] * X[colidx[p] + c * ldx];
            double y = acc * inva;
            Y[i + c * ldy] = y - boa * X[i + c * ldx];
        }
    }
}

/* Chebyshev Clenshaw filter Y = sum_{k=0}^{K} coeffs[k] T_k(Htilde) X.
 * Buffers b[0..2] rotate with the permutation (3,1,2) of
 * ClenshawAlgorithm.jl:2,25:  recurrence writes b[1] = c_k X + 2 Ht b[2] - b[3]
 * (Clenshaw.jl:69-81 with alpha=2, beta=-1), then b <- (b[3], b[1], b[2]).
 * Final sum (Clenshaw.jl:104-117): Y = c_0 X + Ht b[2] - b[3].
 * work holds 3*D*s doubles. */
void orc_clenshaw_filter(int64_t D, const int64_t *rowptr, const int64_t *colidx, const double *v,
                         double a, double b, int K, const double *coeffs, int s,
                         const double *X, double *Y, double *work) {
    int64_t n = D * (int64_t)s;
    double *bb[3] = {work, work + n, work + 2 * n};
    memset(work, 0, sizeof(double) * (size_t)(3 * n));
    for (int k = K; k >= 1; --k) {
        double ck = coeffs[k];
        orc_csr_rescaled(D, rowptr, colidx, v, a, b, s, bb[1], D, bb[0], D);
#pragma omp parallel for schedule(static)
        for (int64_t q = 0; q < n; ++q)
            bb[0][q] = ck * X[q] + 2.0 * bb[0][q] + (-1.0) * bb[2][q];
        double *t0 = bb[0], *t1 = bb[1], *t2 = bb[2];
        bb[0] = t2; bb[1] = t0; bb[2] = t1;
    }
    orc_csr_rescaled(D, rowptr, colidx, v, a, b, s, bb[1], D, Y, D);
    double c0 = coeffs[0];
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; ++q)
        Y[q] = c0 * 1.0 * X[q] + 1.0 * Y[q] + (-1.0) * 1.0 * bb[2][q];
}

/* Serial rescaled apply of one vector (used inside the per-probe trace). */
static void csr_rescaled_vec(int64_t D, const int64_t *rowptr, const int64_t *colidx,
                             const double *v, double inva, double boa,
                             const double *x, double *y) {
    for (int64_t i = 0; i < D; ++i) {
        double acc = 0.0;
        for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p) acc += v[p] * x[colidx[p]];
        y[i] = acc * inva - boa * x[i];
    }
}

/* KPM moments of Moments.jl:87-140: for each probe r (column of `probes`,
 * already normalised), trace! accumulates
 *   mu[0] += <r, r>,  mu[1] += <r, Ht r>,  mu[n] += <r, T_n(Ht) r>
 * with v_{n} = 2 Ht v_{n-1} - v_{n-2}.  Probes are spread over threads and the
 * per-thread sums are reduced at the end, as the threaded CPU path does.
 * mu is NOT scaled by D/R here. */
void orc_kpm_trace(int64_t D, const int64_t *rowptr, const int64_t *colidx, const double *v,
                   double a, double b, int N, int R, const double *probes, double *mu) {
    double inva = 1.0 / a, boa = b / a;
    for (int n = 0; n < N; ++n) mu[n] = 0.0;
#pragma omp parallel
    {
        double *loc = (double *)calloc((size_t)N, sizeof(double));
        double *w = (double *)malloc(sizeof(double) * (size_t)(3 * D));
#pragma omp for schedule(static)
        for (int r = 0; r < R; ++r) {
            const double *al = probes + (int64_t)r * D;
            double *v0 = w, *v1 = w + D, *v2 = w + 2 * D;
            double d = 0.0;
            for (int64_t i = 0; i < D; ++i) { v0[i] = al[i]; d += al[i] * v0[i]; }
            loc[0] += d;
            if (N > 1) {
                csr_rescaled_vec(D, rowptr, colidx, v, inva, boa, v0, v1);
                d = 0.0;
                for (int64_t i = 0; i < D; ++i) d += al[i] * v1[i];
                loc[1] += d;
            }
            for (int n = 2; n < N; ++n) {
                csr_rescaled_vec(D, rowptr, colidx, v, inva, boa, v1, v2);
                d = 0.0;
                for (int64_t i = 0; i < D; ++i) {
                    v2[i] = 2.0 * v2[i];
                    v2[i] = v2[i] - v0[i];
                    d += al[i] * v2[i];
                }
                loc[n] += d;
                double *t = v0; v0 = v1; v1 = v2; v2 = t;
            }
        }
#pragma omp critical
        for (int n = 0; n < N; ++n) mu[n] += loc[n];
        free(loc);
        free(w);
    }
}

/* ------------------------------------------------ bucketed ("optimized") mapping */

/* The packed form of optimization.jl:134-265: a diagonal diag[D] and nb
 * value buckets; bucket k holds value bval[k] and, for every row i, the
 * column indices bflat[boff[k] + bstart[k*(D+1) + i] ... bstart[k*(D+1)+i+1])
 * of its entries equal to that value (0-based).  Diagonal and values are
 * already the rescaled ones when used for Htilde. */
typedef struct {
    int64_t D;
    int nb;
    const double *diag;
    const double *bval;
    const int64_t *bstart;   /* nb x (D+1) */
    const int64_t *boff;     /* nb offsets into bflat */
    const int64_t *bflat;
} orc_buckets;

/* Serial single-vector form used inside the per-probe KPM chains. */
static void bucket_map_vec_serial(const orc_buckets *B, const double *x, double *y) {
    const int64_t D = B->D;
    for (int64_t i = 0; i < D; ++i) y[i] = B->diag[i] * x[i];
    for (int k = 0; k < B->nb; ++k) {
        const int64_t *st = B->bstart + (int64_t)k * (D + 1);
        const int64_t *fl = B->bflat + B->boff[k];
        const double val = B->bval[k];
        for (int64_t i = 0; i < D; ++i) {
            double sum = 0.0;
            for (int64_t p = st[i]; p < st[i + 1]; ++p) sum += x[fl[p]];
            y[i] += val * sum;
        }
    }
}

static orc_buckets mkb(int64_t D, int nb, const double *diag, const double *bval, const int64_t *bstart,
                       const int64_t *boff, const int64_t *bflat) {
    orc_buckets B = {D, nb, diag, bval, bstart, boff, bflat};
    return B;
}

/* mapping! for a vector, multi-bucket method (cpu/mapping.jl:46-64), the
 * reference's default CPU strategy (MulColsParallel(1) -> column by column,
 * each pass threaded over rows): y = diag .* x, then for each bucket in value
 * order y_i += val * sum x[flat]. */
static void bucket_map_vec(const orc_buckets *B, const double *x, double *y) {
    const int64_t D = B->D;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < D; ++i) y[i] = B->diag[i] * x[i];
    for (int k = 0; k < B->nb; ++k) {
        const int64_t *st = B->bstart + (int64_t)k * (D + 1);
        const int64_t *fl = B->bflat + B->boff[k];
        const double val = B->bval[k];
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < D; ++i) {
            double sum = 0.0;
            for (int64_t p = st[i]; p < st[i + 1]; ++p) sum += x[fl[p]];
            y[i] += val * sum;
        }
    }
}

/* Y = Htilde X for a column-major D x s block, column by column
 * (mapping_columnwise!, cpu/mapping.jl:67-95). */
void orc_bucket_apply(int64_t D, int nb, const double *diag, const double *bval, const int64_t *bstart,
                      const int64_t *boff, const int64_t *bflat, int s, const double *X, double *Y) {
    orc_buckets B = mkb(D, nb, diag, bval, bstart, boff, bflat);
    for (int c = 0; c < s; ++c) bucket_map_vec(&B, X + (int64_t)c * D, Y + (int64_t)c * D);
}

/* The Chebyshev filter with the fused row kernels, column by column: the
 * recurrence b1 = c X + 2 Ht b2 - b3 (multi-bucket method: mapping!(b1, b2)
 * then the elementwise update, clenshaw_recurrence_relation.jl:46-64) for
 * k = K..1 with the buffer rotation of ClenshawAlgorithm.jl:2,25, then the
 * final sum Y = c0 X + Ht b1 - b2 (clenshaw_final_sum.jl).  work: 3 D doubles. */
void orc_bucket_filter(int64_t D, int nb, const double *diag, const double *bval, const int64_t *bstart,
                       const int64_t *boff, const int64_t *bflat, int K, const double *coeffs, int s,
                       const double *X, double *Y, double *work) {
    orc_buckets B = mkb(D, nb, diag, bval, bstart, boff, bflat);
    for (int c = 0; c < s; ++c) {
        const double *x = X + (int64_t)c * D;
        double *y = Y + (int64_t)c * D;
        double *bb[3] = {work, work + D, work + 2 * D};
        memset(work, 0, sizeof(double) * (size_t)(3 * D));
        for (int k = K; k >= 1; --k) {
            const double ck = coeffs[k];
            bucket_map_vec(&B, bb[1], bb[0]);
            double *b1 = bb[0], *b3 = bb[2];
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < D; ++i) b1[i] = ck * x[i] + 2.0 * b1[i] - b3[i];
            double *t0 = bb[0], *t1 = bb[1], *t2 = bb[2];
            bb[0] = t2; bb[1] = t0; bb[2] = t1;
        }
        bucket_map_vec(&B, bb[1], y);
        const double c0 = coeffs[0];
        const double *b2 = bb[2];
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < D; ++i) y[i] = c0 * x[i] + y[i] - b2[i];
    }
}

/* KPM moments with the bucketed Htilde (trace!, Moments.jl:87-140): probes
 * spread over threads, each a serial chain v_n = 2 Ht v_{n-1} - v_{n-2}. */
void orc_bucket_kpm_trace(int64_t D, int nb, const double *diag, const double *bval, const int64_t *bstart,
                          const int64_t *boff, const int64_t *bflat, int N, int R, const double *probes,
                          double *mu) {
    orc_buckets B = mkb(D, nb, diag, bval, bstart, boff, bflat);
    for (int n = 0; n < N; ++n) mu[n] = 0.0;
#pragma omp parallel
    {
        double *loc = (double *)calloc((size_t)N, sizeof(double));
        double *w = (double *)malloc(sizeof(double) * (size_t)(3 * D));
#pragma omp for schedule(static)
        for (int r = 0; r < R; ++r) {
            const double *al = probes + (int64_t)r * D;
            double *v0 = w, *v1 = w + D, *v2 = w + 2 * D;
            double d = 0.0;
            for (int64_t i = 0; i < D; ++i) { v0[i] = al[i]; d += al[i] * v0[i]; }
            loc[0] += d;
            if (N > 1) {
                bucket_map_vec_serial(&B, v0, v1);
                d = 0.0;
                for (int64_t i = 0; i < D; ++i) d += al[i] * v1[i];
                loc[1] += d;
            }
            for (int n = 2; n < N; ++n) {
                bucket_map_vec_serial(&B, v1, v2);
                d = 0.0;
                for (int64_t i = 0; i < D; ++i) {
                    v2[i] = 2.0 * v2[i] - v0[i];
                    d += al[i] * v2[i];
                }
                loc[n] += d;
                double *t = v0; v0 = v1; v1 = v2; v2 = t;
            }
        }
#pragma omp critical
        for (int n = 0; n < N; ++n) mu[n] += loc[n];
        free(loc);
        free(w);
    }
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
