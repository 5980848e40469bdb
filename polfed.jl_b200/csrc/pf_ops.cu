// pf_ops.cu -- operator descriptors and the operator-level drop-ins.
//
// Spin chains (SpinHalfChains.jl:267-315) are described by their bonds,
// couplings and fields; the sector basis is enumerated once in ascending order
// (_lup_basis, SpinHalfChains.jl:259-262) and uploaded as 32-bit states, and
// the inverse map (the Dict of SpinHalfChains.jl:278) becomes per-byte
// combinatorial-rank tables.  The Quantum Sun (QuantumSun.jl:1-102, S = 1/2)
// needs no tables: its basis index is the state itself.
#include "pf_internal.h"
#include "pf_solver.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace pf {

static uint64_t binom(int n, int k) {
    if (k < 0 || k > n) return 0;
    uint64_t r = 1;
    for (int i = 1; i <= k; ++i) r = r * (uint64_t)(n - k + i) / (uint64_t)i;
    return r;
}

// Rank tables: chunk c covers bits 8c..8c+7; entry [p][byte] is the part of
// rank(s) = sum_k C(p_k, k) contributed by the set bits of that byte when p
// set bits lie below the chunk.
static std::vector<uint32_t> build_rank_tables(int nchunks) {
    std::vector<uint32_t> tab(rank_table_entries(nchunks));
    for (int c = 0; c < nchunks; ++c) {
        const int off = rank_table_offset(c);
        for (int p = 0; p <= 8 * c; ++p)
            for (int byte = 0; byte < 256; ++byte) {
                uint64_t v = 0;
                int ord = 0;
                for (int t = 0; t < 8; ++t)
                    if (byte & (1 << t)) {
                        ++ord;
                        v += binom(8 * c + t, p + ord);
                    }
                tab[off + p * 256 + byte] = (uint32_t)v;
            }
    }
    return tab;
}

template <typename T>
static void fill_chain(ChainDesc<T> &d, pf_op *op) {
    std::memset(&d, 0, sizeof(d));
    d.L = op->L;
    d.Lup = op->Lup;
    d.full = op->Lup < 0 ? 1 : 0;
    d.nchunks = (op->L + 7) / 8;
    d.nb = (int)op->bonds.size() / 2;
    for (int b = 0; b < d.nb; ++b) {
        const int i = op->bonds[2 * b], j = op->bonds[2 * b + 1];
        d.bi[b] = (uint8_t)i;
        d.bj[b] = (uint8_t)j;
        d.bmask[b] = (1u << i) | (1u << j);
        d.jhalf[b] = (T)(op->J[b] / 2);
        d.jdq[b] = (T)((op->J[b] * op->Delta[b]) * 0.25);
    }
    for (int i = 0; i < op->L; ++i) d.hhalf[i] = (T)(op->fields[i] * 0.5);
    d.states = op->d_states;
    d.rank_tab = op->d_rank_tab;
}

template <typename T>
static void fill_qsun(QSunDesc<T> &d, pf_op *op) {
    std::memset(&d, 0, sizeof(d));
    d.L_grain = op->L_grain;
    d.L_loc = op->L_loc;
    d.L = op->L;
    d.dg = 1 << op->L_grain;
    for (int j = 0; j < op->L_loc; ++j) {
        const int site = op->L_grain + j;
        d.site[j] = (uint8_t)site;
        d.fmask[j] = (1u << site) | (1u << op->nbr[j]);
        d.cflip[j] = (T)(op->g0 * op->coup[j] * 0.5 * 0.5);
        d.hhalf[j] = (T)(op->fields[j] * 0.5);
    }
    for (int q = 0; q < d.dg * d.dg; ++q) d.grain[q] = (T)op->grain[q];
}

pf_op *create_spin_chain(pf_handle *h, int L, int Lup, int nbonds, const int32_t *bonds, const double *J,
                         const double *Delta, const double *fields) {
    PF_CHECK(h != nullptr, PF_ERR_INVALID, "null handle");
    PF_CHECK(L >= 1 && L <= PF_MAX_SITES, PF_ERR_INVALID, "L must satisfy 1 <= L <= 32");
    PF_CHECK(Lup >= -1 && Lup <= L, PF_ERR_INVALID,
             "Lup must satisfy 0 <= Lup <= L (or -1 for the full space)");
    PF_CHECK(nbonds >= 0 && nbonds <= PF_MAX_BONDS, PF_ERR_INVALID, "at most 64 bonds");
    PF_CHECK(nbonds == 0 || (bonds && J && Delta), PF_ERR_INVALID, "null bond arrays");
    PF_CHECK(fields != nullptr, PF_ERR_INVALID, "null fields");
    const uint64_t D = Lup < 0 ? (1ull << L) : binom(L, Lup);
    PF_CHECK(D >= 1 && D < (1ull << 31), PF_ERR_UNSUPPORTED, "basis dimension must be below 2^31");
    for (int b = 0; b < nbonds; ++b) {
        PF_CHECK(bonds[2 * b] >= 0 && bonds[2 * b] < L && bonds[2 * b + 1] >= 0 && bonds[2 * b + 1] < L,
                 PF_ERR_INVALID, "bond site out of range");
        PF_CHECK(bonds[2 * b] != bonds[2 * b + 1], PF_ERR_INVALID, "bond joins a site to itself");
        PF_CHECK(std::isfinite(J[b]) && std::isfinite(Delta[b]), PF_ERR_INVALID, "non-finite coupling");
    }
    for (int i = 0; i < L; ++i) PF_CHECK(std::isfinite(fields[i]), PF_ERR_INVALID, "non-finite field");

    PF_CUDA(cudaSetDevice(h->device));
    pf_op *op = new pf_op();
    op->h = h;
    op->kind = OP_CHAIN;
    op->L = L;
    op->Lup = Lup;
    op->dim = (int64_t)D;
    op->bonds.assign(bonds, bonds + 2 * nbonds);
    op->J.assign(J, J + nbonds);
    op->Delta.assign(Delta, Delta + nbonds);
    op->fields.assign(fields, fields + L);
    try {
        if (Lup >= 0) {
            std::vector<uint32_t> states((size_t)D);
            // ascending states with popcount Lup (Gosper's next-combination step)
            uint64_t st = (Lup == 0) ? 0ull : ((1ull << Lup) - 1ull);
            for (uint64_t n = 0; n < D; ++n) {
                states[n] = (uint32_t)st;
                if (Lup == 0) break;
                const uint64_t c = st & (~st + 1ull);
                const uint64_t r = st + c;
                st = (((r ^ st) >> 2) / c) | r;
            }
            PF_CUDA(cudaMalloc(&op->d_states, D * sizeof(uint32_t)));
            PF_CUDA(cudaMemcpy(op->d_states, states.data(), D * sizeof(uint32_t), cudaMemcpyHostToDevice));
            const int nchunks = (L + 7) / 8;
            std::vector<uint32_t> tab = build_rank_tables(nchunks);
            PF_CUDA(cudaMalloc(&op->d_rank_tab, tab.size() * sizeof(uint32_t)));
            PF_CUDA(cudaMemcpy(op->d_rank_tab, tab.data(), tab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
        }
        fill_chain(op->chain64, op);
        fill_chain(op->chain32, op);
        build_chain_diag(op);
        build_multi_tables(op);
        uint32_t *tst = op->d_states, *trk = op->d_rank_tab;
        double *tdg = op->d_diag64;
        float *tdf = op->d_diag32;
        const int dev = h->device;
        op->tables_owner = std::shared_ptr<void>(nullptr, [tst, trk, tdg, tdf, dev](void *) {
            cudaSetDevice(dev);
            cudaFree(tst);
            cudaFree(trk);
            cudaFree(tdg);
            cudaFree(tdf);
        });
    } catch (...) {
        if (!op->tables_owner) {
            if (op->d_states) cudaFree(op->d_states);
            if (op->d_rank_tab) cudaFree(op->d_rank_tab);
            if (op->d_diag64) cudaFree(op->d_diag64);
            if (op->d_diag32) cudaFree(op->d_diag32);
        }
        delete op;
        throw;
    }
    return op;
}

pf_op *create_qsun(pf_handle *h, int L_loc, int L_grain, double g0, const double *coup, const int32_t *nbr,
                   const double *fields, const double *grain) {
    PF_CHECK(h != nullptr, PF_ERR_INVALID, "null handle");
    PF_CHECK(L_grain >= 1 && (1 << L_grain) <= PF_MAX_GRAIN, PF_ERR_INVALID, "1 <= L_grain <= 4");
    PF_CHECK(L_loc >= 1 && L_loc <= PF_MAX_LOC, PF_ERR_INVALID, "1 <= L_loc <= 32");
    PF_CHECK(L_loc + L_grain <= 30, PF_ERR_UNSUPPORTED, "L_loc + L_grain <= 30");
    PF_CHECK(coup && nbr && fields && grain, PF_ERR_INVALID, "null QSun parameter array");
    PF_CHECK(std::isfinite(g0), PF_ERR_INVALID, "non-finite g0");
    for (int j = 0; j < L_loc; ++j) {
        PF_CHECK(nbr[j] >= 0 && nbr[j] < L_grain, PF_ERR_INVALID, "grain neighbour out of range");
        PF_CHECK(std::isfinite(coup[j]) && std::isfinite(fields[j]), PF_ERR_INVALID, "non-finite parameter");
    }
    const int dg = 1 << L_grain;
    for (int q = 0; q < dg * dg; ++q) PF_CHECK(std::isfinite(grain[q]), PF_ERR_INVALID, "non-finite grain block");
    for (int g = 0; g < dg; ++g)
        for (int k = 0; k < dg; ++k)
            PF_CHECK(grain[g * dg + k] == grain[k * dg + g], PF_ERR_INVALID, "grain block must be symmetric");
    PF_CUDA(cudaSetDevice(h->device));
    pf_op *op = new pf_op();
    op->h = h;
    op->kind = OP_QSUN;
    op->L_loc = L_loc;
    op->L_grain = L_grain;
    op->L = L_loc + L_grain;
    op->dim = (int64_t)1 << op->L;
    op->g0 = g0;
    op->coup.assign(coup, coup + L_loc);
    op->nbr.assign(nbr, nbr + L_loc);
    op->fields.assign(fields, fields + L_loc);
    op->grain.assign(grain, grain + dg * dg);
    fill_qsun(op->qsun64, op);
    fill_qsun(op->qsun32, op);
    try {
        build_qsun_tables(op);
        void *t64 = op->d_qtab64, *t32 = op->d_qtab32;
        const int dev = h->device;
        op->tables_owner = std::shared_ptr<void>(nullptr, [t64, t32, dev](void *) {
            cudaSetDevice(dev);
            cudaFree(t64);
            cudaFree(t32);
        });
        build_multi_tables(op);
    } catch (...) {
        if (!op->tables_owner) {
            if (op->d_qtab64) cudaFree(op->d_qtab64);
            if (op->d_qtab32) cudaFree(op->d_qtab32);
        }
        delete op;
        throw;
    }
    return op;
}

pf_op *create_csr(pf_handle *h, int64_t D, int64_t nnz, const int64_t *indptr, const int32_t *indices,
                  const double *values) {
    PF_CHECK(h != nullptr, PF_ERR_INVALID, "null handle");
    PF_CHECK(D >= 1 && D < ((int64_t)1 << 31), PF_ERR_UNSUPPORTED, "matrix dimension must be in [1, 2^31)");
    PF_CHECK(nnz >= 0 && indptr && (nnz == 0 || (indices && values)), PF_ERR_INVALID, "null CSR array");
    PF_CHECK(indptr[0] == 0 && indptr[D] == nnz, PF_ERR_INVALID, "indptr must start at 0 and end at nnz");
    for (int64_t i = 0; i < D; ++i)
        PF_CHECK(indptr[i + 1] >= indptr[i], PF_ERR_INVALID, "indptr must be non-decreasing");
    for (int64_t p = 0; p < nnz; ++p) {
        PF_CHECK(indices[p] >= 0 && (int64_t)indices[p] < D, PF_ERR_INVALID, "column index out of range");
        PF_CHECK(std::isfinite(values[p]), PF_ERR_INVALID, "non-finite matrix entry");
    }
    PF_CUDA(cudaSetDevice(h->device));
    int64_t *dptr = nullptr;
    int32_t *didx = nullptr;
    double *dv64 = nullptr;
    float *dv32 = nullptr;
    try {
        std::vector<float> v32(values, values + nnz);
        PF_CUDA(cudaMalloc(&dptr, (D + 1) * sizeof(int64_t)));
        PF_CUDA(cudaMalloc(&didx, std::max<int64_t>(nnz, 1) * sizeof(int32_t)));
        PF_CUDA(cudaMalloc(&dv64, std::max<int64_t>(nnz, 1) * sizeof(double)));
        PF_CUDA(cudaMalloc(&dv32, std::max<int64_t>(nnz, 1) * sizeof(float)));
        PF_CUDA(cudaMemcpy(dptr, indptr, (D + 1) * sizeof(int64_t), cudaMemcpyHostToDevice));
        if (nnz > 0) {
            PF_CUDA(cudaMemcpy(didx, indices, nnz * sizeof(int32_t), cudaMemcpyHostToDevice));
            PF_CUDA(cudaMemcpy(dv64, values, nnz * sizeof(double), cudaMemcpyHostToDevice));
            PF_CUDA(cudaMemcpy(dv32, v32.data(), nnz * sizeof(float), cudaMemcpyHostToDevice));
        }
    } catch (...) {
        if (dptr) cudaFree(dptr);
        if (didx) cudaFree(didx);
        if (dv64) cudaFree(dv64);
        if (dv32) cudaFree(dv32);
        throw;
    }
    return adopt_csr(h, D, nnz, dptr, didx, dv64, dv32);
}

// H = A + iB Hermitian (CSR, values interleaved re, im) as the real symmetric
// M = [[A, -B], [B, A]] of twice the dimension: M [x; y] = [Re H(x+iy); Im H(x+iy)].
pf_op *create_csr_hermitian(pf_handle *h, int64_t D, int64_t nnz, const int64_t *indptr, const int32_t *indices,
                            const double *values) {
    PF_CHECK(h != nullptr, PF_ERR_INVALID, "null handle");
    PF_CHECK(D >= 1 && D < ((int64_t)1 << 30), PF_ERR_UNSUPPORTED, "Hermitian matrix dimension must be in [1, 2^30)");
    PF_CHECK(nnz >= 0 && indptr && (nnz == 0 || (indices && values)), PF_ERR_INVALID, "null CSR array");
    PF_CHECK(indptr[0] == 0 && indptr[D] == nnz, PF_ERR_INVALID, "indptr must start at 0 and end at nnz");
    for (int64_t i = 0; i < D; ++i)
        PF_CHECK(indptr[i + 1] >= indptr[i], PF_ERR_INVALID, "indptr must be non-decreasing");
    for (int64_t p = 0; p < nnz; ++p) {
        PF_CHECK(indices[p] >= 0 && (int64_t)indices[p] < D, PF_ERR_INVALID, "column index out of range");
        PF_CHECK(std::isfinite(values[2 * p]) && std::isfinite(values[2 * p + 1]), PF_ERR_INVALID,
                 "non-finite matrix entry");
    }
    for (int64_t i = 0; i < D; ++i)
        for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p)
            PF_CHECK(indices[p] != i || values[2 * p + 1] == 0.0, PF_ERR_INVALID,
                     "a Hermitian matrix has a real diagonal");
    // rows 0..D-1: [A, -B]; rows D..2D-1: [B, A] (entries whose part is zero are left out)
    std::vector<int64_t> ptr((size_t)2 * D + 1, 0);
    std::vector<int32_t> idx;
    std::vector<double> val;
    idx.reserve((size_t)4 * nnz);
    val.reserve((size_t)4 * nnz);
    for (int half = 0; half < 2; ++half)
        for (int64_t i = 0; i < D; ++i) {
            for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
                const double re = values[2 * p], im = values[2 * p + 1];
                const int32_t c = indices[p];
                if (half == 0) {
                    if (re != 0.0) idx.push_back(c), val.push_back(re);
                    if (im != 0.0) idx.push_back((int32_t)(D + c)), val.push_back(-im);
                } else {
                    if (im != 0.0) idx.push_back(c), val.push_back(im);
                    if (re != 0.0) idx.push_back((int32_t)(D + c)), val.push_back(re);
                }
            }
            ptr[(size_t)half * D + i + 1] = (int64_t)idx.size();
        }
    pf_op *op = create_csr(h, 2 * D, (int64_t)idx.size(), ptr.data(), idx.data(), val.data());
    op->complex_dim = D;
    return op;
}

pf_op *adopt_csr(pf_handle *h, int64_t D, int64_t nnz, int64_t *dptr, int32_t *didx, double *dv64, float *dv32) {
    pf_op *op = nullptr;
    const int dev = h->device;
    auto owner = std::shared_ptr<void>(nullptr, [dptr, didx, dv64, dv32, dev](void *) {
        cudaSetDevice(dev);
        cudaFree(dptr);
        cudaFree(didx);
        cudaFree(dv64);
        cudaFree(dv32);
    });
    op = new pf_op();
    op->h = h;
    op->kind = OP_CSR;
    op->dim = D;
    op->nnz = nnz;
    op->tables_owner = owner;
    op->csr64 = {dptr, didx, dv64};
    op->csr32 = {dptr, didx, dv32};
    try {
        build_multi_tables(op);
    } catch (...) {
        delete op;
        throw;
    }
    return op;
}

void destroy_op(pf_op *op) {
    if (!op) return;
    delete op;  // the device tables go with the last operator sharing them
}

pf_op *bind_op(const pf_op *src, pf_handle *h) {
    PF_CHECK(src && h, PF_ERR_INVALID, "null argument");
    PF_CHECK(src->h->device == h->device, PF_ERR_INVALID, "an operator can only be bound to a handle of its device");
    pf_op *op = new pf_op();
    op->h = h;
    op->kind = src->kind;
    op->dim = src->dim;
    op->L = src->L;
    op->Lup = src->Lup;
    op->chain64 = src->chain64;
    op->chain32 = src->chain32;
    op->qsun64 = src->qsun64;
    op->qsun32 = src->qsun32;
    op->csr64 = src->csr64;
    op->csr32 = src->csr32;
    op->nnz = src->nnz;
    op->complex_dim = src->complex_dim;
    op->d_states = src->d_states;
    op->d_rank_tab = src->d_rank_tab;
    op->d_diag64 = src->d_diag64;
    op->d_diag32 = src->d_diag32;
    op->tables_owner = src->tables_owner;
    op->d_desc64 = src->d_desc64;
    op->d_desc32 = src->d_desc32;
    op->d_qtab64 = src->d_qtab64;
    op->d_qtab32 = src->d_qtab32;
    op->multi_owner = src->multi_owner;
    op->smem_bytes = src->smem_bytes;
    op->slab_cols = src->slab_cols;
    {
        std::lock_guard<std::mutex> lock(const_cast<pf_op *>(src)->tune_mu);
        op->tuned_width = src->tuned_width;
    }
    op->bonds = src->bonds;
    op->J = src->J;
    op->Delta = src->Delta;
    op->fields = src->fields;
    op->coup = src->coup;
    op->grain = src->grain;
    op->nbr = src->nbr;
    op->g0 = src->g0;
    op->L_loc = src->L_loc;
    op->L_grain = src->L_grain;
    return op;
}

// ------------------------------------------------------- handle scratch
void *handle_scratch(pf_handle *h, size_t bytes) {
    if (h->scratch_bytes < bytes) {
        if (h->scratch) {
            PF_CUDA(cudaStreamSynchronize(h->stream));
            cudaFree(h->scratch);
        }
        h->scratch = nullptr;
        h->scratch_bytes = 0;
        PF_CUDA(cudaMalloc(&h->scratch, bytes));
        h->scratch_bytes = bytes;
    }
    return h->scratch;
}

// --------------------------------------------------- operator-level API
template <typename T>
static void op_step_cm(pf_op *op, int s, const T *q, const T *p, const T *x, T *out, int64_t ld,
                       int64_t ldout, double cx, double alpha, double beta, double a, double b, int flags) {
    pf_handle *h = op->h;
    const int64_t D = op->dim;
    PF_CHECK(ld >= D && ldout >= D, PF_ERR_INVALID, "leading dimension smaller than the operator dimension");
    PF_CHECK(a != 0.0 && std::isfinite(a) && std::isfinite(b), PF_ERR_INVALID, "rescaling a must be finite and nonzero");
    if (s == 1) {
        launch_step<T>(op, h->stream, D, 1, q, p, x, out, cx, alpha, beta, 1.0 / a, b, flags, nullptr);
        return;
    }
    const size_t n = (size_t)D * s;
    T *base = (T *)handle_scratch(h, 4 * n * sizeof(T));
    T *qr = base, *pr = base + n, *xr = base + 2 * n, *outr = base + 3 * n;
    if (flags & StepFlags::Q) launch_cm_to_ri<T, T>(h->stream, D, s, q, ld, qr);
    if (flags & StepFlags::P) launch_cm_to_ri<T, T>(h->stream, D, s, p, ld, pr);
    if (flags & StepFlags::X) launch_cm_to_ri<T, T>(h->stream, D, s, x, ld, xr);
    launch_step<T>(op, h->stream, D, s, qr, pr, xr, outr, cx, alpha, beta, 1.0 / a, b, flags, nullptr);
    launch_ri_to_cm<T, T>(h->stream, D, s, outr, out, ldout);
}

void op_apply(pf_op *op, int dtype, double a, double b, int s, const void *X, int64_t ldx, void *Y, int64_t ldy) {
    PF_CHECK(X && Y && s >= 1, PF_ERR_INVALID, "invalid apply arguments");
    PF_CUDA(cudaSetDevice(op->h->device));
    if (dtype == PF_F64)
        op_step_cm<double>(op, s, (const double *)X, nullptr, nullptr, (double *)Y, ldx, ldy, 0, 1, 0, a, b, StepFlags::Q);
    else if (dtype == PF_F32)
        op_step_cm<float>(op, s, (const float *)X, nullptr, nullptr, (float *)Y, ldx, ldy, 0, 1, 0, a, b, StepFlags::Q);
    else throw Error(PF_ERR_INVALID, "dtype must be PF_F64 or PF_F32");
}

void op_recurrence(pf_op *op, int dtype, double a, double b, double c, int s, void *b1, const void *b2,
                   const void *b3, const void *X, int64_t ld) {
    PF_CHECK(b1 && b2 && b3 && X && s >= 1, PF_ERR_INVALID, "invalid recurrence arguments");
    PF_CUDA(cudaSetDevice(op->h->device));
    const int fl = StepFlags::Q | StepFlags::P | StepFlags::X;
    if (dtype == PF_F64)
        op_step_cm<double>(op, s, (const double *)b2, (const double *)b3, (const double *)X, (double *)b1, ld, ld,
                           c, 2.0, -1.0, a, b, fl);
    else if (dtype == PF_F32)
        op_step_cm<float>(op, s, (const float *)b2, (const float *)b3, (const float *)X, (float *)b1, ld, ld,
                          c, 2.0, -1.0, a, b, fl);
    else throw Error(PF_ERR_INVALID, "dtype must be PF_F64 or PF_F32");
}

void op_finalsum(pf_op *op, int dtype, double a, double b, double c0, int s, const void *b1, const void *b2,
                 void *Y, const void *X, int64_t ld) {
    PF_CHECK(b1 && b2 && Y && X && s >= 1, PF_ERR_INVALID, "invalid final-sum arguments");
    PF_CUDA(cudaSetDevice(op->h->device));
    const int fl = StepFlags::Q | StepFlags::P | StepFlags::X;
    if (dtype == PF_F64)
        op_step_cm<double>(op, s, (const double *)b1, (const double *)b2, (const double *)X, (double *)Y, ld, ld,
                           c0, 1.0, -1.0, a, b, fl);
    else if (dtype == PF_F32)
        op_step_cm<float>(op, s, (const float *)b1, (const float *)b2, (const float *)X, (float *)Y, ld, ld,
                          c0, 1.0, -1.0, a, b, fl);
    else throw Error(PF_ERR_INVALID, "dtype must be PF_F64 or PF_F32");
}

}  // namespace pf
