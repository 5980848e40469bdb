// pf_rows.cuh -- per-row Hamiltonian evaluation shared by the step kernels.
//
// Each row function returns, for row `row` and columns c0..c0+V-1 of a
// row-interleaved block q (element (i, c) at i*s + c), the off-diagonal
// gather sum in acc[] and the row's diagonal element.  The matrix is never
// stored: the spin-chain and Quantum Sun rows are derived from the operator
// descriptor (SpinHalfChains.jl:267-315, QuantumSun.jl:1-102), a CSR row from
// the user's matrix.
#pragma once
#include "pf_internal.h"

namespace pf {

template <typename T, int V>
struct alignas(sizeof(T) * V) Pack {
    T v[V];
};

template <typename T, int V>
__device__ __forceinline__ Pack<T, V> ldp(const T *p) {
    return *reinterpret_cast<const Pack<T, V> *>(p);
}
template <typename T, int V>
__device__ __forceinline__ void stp(T *p, const Pack<T, V> &v) {
    *reinterpret_cast<Pack<T, V> *>(p) = v;
}

// ------------------------------------------------------------ sector rank
__device__ __forceinline__ uint32_t sector_rank(uint32_t st, const uint32_t *tab, int nchunks) {
    uint32_t r = 0;
    int p = 0;
    int off = 0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        if (c < nchunks) {
            uint32_t byte = (st >> (8 * c)) & 0xffu;
            r += tab[off + p * 256 + (int)byte];
            p += __popc(byte);
            off += (8 * c + 1) * 256;
        }
    }
    return r;
}

// Loads and stores of a row segment with evict-first ("streaming") cache
// hints when `stream` is set, so data touched once per pass does not push the
// gathered block out of L2.  Segments are moved as 8- or 16-byte words.
template <typename T, int V>
__device__ __forceinline__ Pack<T, V> ldp_hint(const T *p, int stream) {
    if (!stream) return ldp<T, V>(p);
    Pack<T, V> r;
    constexpr int bytes = V * (int)sizeof(T);
    if constexpr (bytes % 16 == 0) {
        const double2 *s = reinterpret_cast<const double2 *>(p);
        double2 *d = reinterpret_cast<double2 *>(&r);
#pragma unroll
        for (int i = 0; i < bytes / 16; ++i) d[i] = __ldcs(s + i);
    } else if constexpr (bytes == 8) {
        *reinterpret_cast<double *>(&r) = __ldcs(reinterpret_cast<const double *>(p));
    } else {
        *reinterpret_cast<float *>(&r) = __ldcs(reinterpret_cast<const float *>(p));
    }
    return r;
}
template <typename T, int V>
__device__ __forceinline__ void stp_hint(T *p, const Pack<T, V> &v, int stream) {
    if (!stream) {
        stp<T, V>(p, v);
        return;
    }
    constexpr int bytes = V * (int)sizeof(T);
    if constexpr (bytes % 16 == 0) {
        double2 *d = reinterpret_cast<double2 *>(p);
        const double2 *s = reinterpret_cast<const double2 *>(&v);
#pragma unroll
        for (int i = 0; i < bytes / 16; ++i) __stcs(d + i, s[i]);
    } else if constexpr (bytes == 8) {
        __stcs(reinterpret_cast<double *>(p), *reinterpret_cast<const double *>(&v));
    } else {
        __stcs(reinterpret_cast<float *>(p), *reinterpret_cast<const float *>(&v));
    }
}

// Programmatic dependent launch.  A step kernel lets the next kernel of its
// stream launch as soon as it starts (its CTAs become resident as this grid's
// retire) and, after staging its own read-only tables, waits until its
// predecessor has completed and its writes are visible before it reads any
// block.  Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Explicitly rounded arithmetic.  Every step-kernel variant (any width,
// gather batch or register cap; per-thread, warp-cooperative or
// multi-instance) performs exactly these operations in the same order, so all
// of them give bit-identical results whatever contractions the compiler would
// otherwise choose per instantiation.
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double mul_t(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_t(float a, float b) { return __fmul_rn(a, b); }

// One output element of a step: cx x + alpha ((acc + diag q) / a - (b/a) q) + beta p,
// with the terms that are absent (has_x / has_q / has_p false) left out.
template <typename T>
__device__ __forceinline__ T step_combine(bool has_x, bool has_q, bool has_p, T cx, T x, T alpha, T acc, T diag,
                                          T q, T inva, T boa, T beta, T p) {
    T res = has_x ? mul_t(cx, x) : T(0);
    if (has_q) {
        const T hq = fma_t(-boa, q, mul_t(fma_t(diag, q, acc), inva));
        res = fma_t(alpha, hq, res);
    }
    if (has_p) res = fma_t(beta, p, res);
    return res;
}

// Pull a row's own operand segment toward L1 before its gathers are issued,
// so the later load of it does not add a dependent L2 round trip (no register
// is held meanwhile).
__device__ __forceinline__ void prefetch_l1(const void *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// ------------------------------------------------------------ row models
// Each returns (through acc / diag) the off-diagonal gather sum and the
// diagonal element of row `row` for columns c0..c0+V-1.

// Gathers are issued in unrolled batches of U independent loads so that each
// thread keeps several L2/HBM requests in flight (the loop bodies have no
// load-to-load dependence); accumulation follows the reference's term order.
// U shrinks as the per-thread column count V grows, to bound registers; a
// tuned variant may set it explicitly (template argument UB > 0).
template <typename T, int V>
struct Batch {
    static constexpr int bytes = V * (int)sizeof(T);
    static constexpr int U = bytes >= 64 ? 2 : (bytes >= 16 ? 4 : 8);
};

// Resident CTAs per SM the step kernel is compiled for: caps registers so
// enough warps stay resident to cover L2 latency with independent gathers
// (with no cap the 64-byte-per-thread variants took 170 registers, one CTA
// per SM, 8 warps -- latency-bound).
template <typename T, int V>
struct MinBlocks {
    static constexpr int bytes = V * (int)sizeof(T);
    static constexpr int value = bytes >= 32 ? 2 : 3;
};

// A chain row in two passes: first the diagonal over every bond in bond order
// (fields, then the Sz Sz terms) and the mask of the bonds whose spins differ;
// then the flipping bonds only, U of them per round (lowest bond first), each
// round issuing its U gathers before any is used.  Bonds that do not flip
// (about half of them) take no slot in a round, so a row needs about half
// the dependent gather rounds of a walk over every bond; the gathers are
// still accumulated in bond order.  RANK(b) returns the flipped state's
// index.
template <typename T, int V, bool HASQ, int U, class RankF>
__device__ __forceinline__ void chain_row_walk(const ChainDesc<T> &d, uint32_t st, int s, const T *__restrict__ qc,
                                               T (&acc)[V], T &diag, RankF rank) {
    T dg = T(0);
    for (int i = 0; i < d.L; ++i) dg += ((st >> i) & 1u) ? d.hhalf[i] : -d.hhalf[i];
    uint64_t act = 0ull;
    for (int b = 0; b < d.nb; ++b) {
        const uint32_t bm = d.bmask[b];
        const uint32_t m = st & bm;
        const bool differ = (m != 0u) && (m != bm);
        dg += differ ? -d.jdq[b] : d.jdq[b];
        if (differ) act |= 1ull << b;
    }
    diag = dg;
    if constexpr (HASQ) {
        while (act != 0ull) {
            uint32_t r2[U];
            T jh[U];
            bool on[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                on[u] = act != 0ull;
                r2[u] = 0u;
                jh[u] = T(0);
                if (on[u]) {
                    const int b = __ffsll((long long)act) - 1;
                    act &= act - 1ull;
                    r2[u] = rank(b);
                    jh[u] = d.jhalf[b];
                }
            }
            Pack<T, V> g[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (on[u]) g[u] = ldp<T, V>(qc + (size_t)r2[u] * s);
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (on[u]) {
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[v] = fma_t(jh[u], g[u].v[v], acc[v]);
                }
        }
    }
}

template <typename T, int V, bool HASQ, int UB = 0>
__device__ __forceinline__ void chain_row(const ChainDesc<T> &d, const uint32_t *tab, uint32_t row,
                                          int s, int c0, const T *__restrict__ q, T (&acc)[V],
                                          T &diag) {
    constexpr int U = UB > 0 ? UB : Batch<T, V>::U;
    const uint32_t st = d.full ? row : __ldg(d.states + row);
    chain_row_walk<T, V, HASQ, U>(d, st, s, q + c0, acc, diag, [&](int b) -> uint32_t {
        const uint32_t st2 = st ^ d.bmask[b];
        return d.full ? st2 : sector_rank(st2, tab, d.nchunks);
    });
}

// Rank of the state reached by the flip of bond b from state st of rank row,
// by the local update of the combinatorial number system when the bond joins
// sites at most two apart: moving a particle between sites lo < hi changes
// only the terms of the particles in [lo, hi].  With k0 particles below lo,
// a particle moving up from lo to lo + 1 changes C(lo, k0+1) into
// C(lo+1, k0+1), i.e. by C(lo, k0) (Pascal's rule); moving to lo + 2 past an
// empty site changes C(lo, k0+1) into C(lo+2, k0+1), and past an occupied one
// the middle particle also drops one ordinal.  A move down is the reverse
// move's negative.  Farther bonds (the periodic wrap) use the full table
// rank.  ctab[n * 33 + k] = C(n, k) for n, k <= 32.  Exact integer work: the
// result equals sector_rank(st ^ bmask[b]).
template <typename T>
__device__ __forceinline__ uint32_t flip_rank_local(const ChainDesc<T> &d, const uint32_t *tab, const uint32_t *ctab,
                                                    uint32_t st, uint32_t row, int b) {
    const int i = d.bi[b], j = d.bj[b];
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const int span = hi - lo;
    if (span > 2) return sector_rank(st ^ d.bmask[b], tab, d.nchunks);
    const int k0 = __popc(st & ((1u << lo) - 1u));
    const bool up = (st >> lo) & 1u;   // the particle sits at lo and moves to hi
    uint32_t delta;
    if (span == 1) {
        delta = ctab[lo * 33 + k0];
    } else {
        const bool mid = (st >> (lo + 1)) & 1u;
        if (!mid) delta = ctab[(lo + 2) * 33 + k0 + 1] - ctab[lo * 33 + k0 + 1];
        else
            delta = ctab[(lo + 2) * 33 + k0 + 2] + ctab[(lo + 1) * 33 + k0 + 1] - ctab[lo * 33 + k0 + 1] -
                    ctab[(lo + 1) * 33 + k0 + 2];
    }
    return up ? row + delta : row - delta;
}

// chain_row with flip ranks from flip_rank_local (the rank of the row's own
// state is the row index); identical sums in identical order.
template <typename T, int V, bool HASQ, int UB = 0>
__device__ __forceinline__ void chain_row_local(const ChainDesc<T> &d, const uint32_t *tab, const uint32_t *ctab,
                                                uint32_t row, int s, int c0, const T *__restrict__ q, T (&acc)[V],
                                                T &diag) {
    constexpr int U = UB > 0 ? UB : Batch<T, V>::U;
    const uint32_t st = d.full ? row : __ldg(d.states + row);
    chain_row_walk<T, V, HASQ, U>(d, st, s, q + c0, acc, diag, [&](int b) -> uint32_t {
        return d.full ? (st ^ d.bmask[b]) : flip_rank_local(d, tab, ctab, st, row, b);
    });
}

// Quantum Sun shared-memory layout: the grain block with a padded row stride
// (dg + 1, so the 8 rows of one grain group read different banks), then four
// 256-entry diagonal tables, one per byte of the outer-spin bits.
template <typename T>
struct QSunSmem {
    static __host__ __device__ int grain_stride(int dg) { return dg + 1; }
    static __host__ __device__ int bytes(int dg) { return (dg * (dg + 1) + 4 * 256) * (int)sizeof(T); }
};

template <typename T, int V, bool HASQ, int UB = 0>
__device__ __forceinline__ void qsun_row(const QSunDesc<T> &d, const T *smem_t, uint32_t row,
                                         int s, int c0, const T *__restrict__ q, T (&acc)[V],
                                         T &diag) {
    constexpr int U = UB > 0 ? UB : Batch<T, V>::U;
    const int gs = d.dg + 1;
    const T *dtab = smem_t + d.dg * gs;
    const uint32_t outer = row >> d.L_grain;
    T dg = dtab[outer & 0xffu];
    if (d.L_loc > 8) dg += dtab[256 + ((outer >> 8) & 0xffu)];
    if (d.L_loc > 16) dg += dtab[512 + ((outer >> 16) & 0xffu)];
    if (d.L_loc > 24) dg += dtab[768 + ((outer >> 24) & 0xffu)];
    diag = dg;
    if constexpr (HASQ) {
        const T *qc = q + c0;
        for (int j0 = 0; j0 < d.L_loc; j0 += U) {
            Pack<T, V> g[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (j0 + u < d.L_loc) g[u] = ldp<T, V>(qc + (size_t)(row ^ d.fmask[j0 + u]) * s);
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (j0 + u < d.L_loc) {
                    const T cf = d.cflip[j0 + u];
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[v] = fma_t(cf, g[u].v[v], acc[v]);
                }
        }
        const uint32_t g = row & ((uint32_t)d.dg - 1u);
        const uint32_t base = row - g;
        const T *grow = smem_t + g * gs;
        for (int h0 = 0; h0 < d.dg; h0 += U) {
            Pack<T, V> x[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (h0 + u < d.dg) x[u] = ldp<T, V>(qc + (size_t)(base + h0 + u) * s);
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (h0 + u < d.dg) {
                    const T w = grow[h0 + u];
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[v] = fma_t(w, x[u].v[v], acc[v]);
                }
        }
    }
}

// CSR row (a user matrix): the entries of the row in storage order, gathered
// in unrolled batches of U like the matrix-free rows; the diagonal is an
// ordinary entry, so diag = 0.
template <typename T, int V, bool HASQ, int UB = 0>
__device__ __forceinline__ void csr_row(const CsrDesc<T> &d, uint32_t row, int s, int c0, const T *__restrict__ q,
                                        T (&acc)[V], T &diag) {
    diag = T(0);
    if constexpr (HASQ) {
        constexpr int U = UB > 0 ? UB : Batch<T, V>::U;
        const int64_t b = __ldg(d.indptr + row), e = __ldg(d.indptr + row + 1);
        const T *qc = q + c0;
        for (int64_t p0 = b; p0 < e; p0 += U) {
            int32_t col[U];
            T val[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (p0 + u < e) {
                    col[u] = __ldg(d.indices + p0 + u);
                    val[u] = __ldg(d.values + p0 + u);
                }
            Pack<T, V> g[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (p0 + u < e) g[u] = ldp<T, V>(qc + (size_t)col[u] * s);
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (p0 + u < e) {
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[v] = fma_t(val[u], g[u].v[v], acc[v]);
                }
        }
    }
}


// Quantum Sun row with the grain block read from the descriptor (global
// memory, L1-resident) and the diagonal from a per-row array built by
// k_qsun_diag: the same values and the same order of additions as qsun_row,
// so both produce identical results.  Used where one launch serves several
// operators and per-operator shared-memory tables cannot be staged.
template <typename T, int V, bool HASQ, int UB = 0>
__device__ __forceinline__ void qsun_row_g(const QSunDesc<T> &d, const T *__restrict__ dvec, uint32_t row, int s,
                                           int c0, const T *__restrict__ q, T (&acc)[V], T &diag) {
    constexpr int U = UB > 0 ? UB : Batch<T, V>::U;
    diag = dvec[row];
    if constexpr (HASQ) {
        const T *qc = q + c0;
        for (int j0 = 0; j0 < d.L_loc; j0 += U) {
            Pack<T, V> g[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (j0 + u < d.L_loc) g[u] = ldp<T, V>(qc + (size_t)(row ^ d.fmask[j0 + u]) * s);
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (j0 + u < d.L_loc) {
                    const T cf = d.cflip[j0 + u];
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[v] = fma_t(cf, g[u].v[v], acc[v]);
                }
        }
        const uint32_t g = row & ((uint32_t)d.dg - 1u);
        const uint32_t base = row - g;
        const T *grow = d.grain + g * d.dg;
        for (int h0 = 0; h0 < d.dg; h0 += U) {
            Pack<T, V> x[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (h0 + u < d.dg) x[u] = ldp<T, V>(qc + (size_t)(base + h0 + u) * s);
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (h0 + u < d.dg) {
                    const T w = grow[h0 + u];
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[v] = fma_t(w, x[u].v[v], acc[v]);
                }
        }
    }
}

// Diagonal of a Quantum Sun row, summed exactly as qsun_row sums it: per byte
// of the outer-spin bits the sum over its 8 spins of +-h_j/2 in spin order,
// then the byte sums in byte order.
template <typename T>
__device__ __forceinline__ T qsun_diag(const QSunDesc<T> &d, uint32_t row) {
    const uint32_t outer = row >> d.L_grain;
    T dg = T(0);
    for (int c = 0; c < 4; ++c) {
        if (c > 0 && d.L_loc <= 8 * c) break;
        const uint32_t byte = (outer >> (8 * c)) & 0xffu;
        T acc = T(0);
        for (int t = 0; t < 8; ++t) {
            const int j = 8 * c + t;
            if (j < d.L_loc) acc += ((byte >> t) & 1u) ? d.hhalf[j] : -d.hhalf[j];
        }
        dg = (c == 0) ? acc : dg + acc;
    }
    return dg;
}

}  // namespace pf
