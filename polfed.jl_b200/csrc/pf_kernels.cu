// pf_kernels.cu -- matrix-free Hamiltonian kernels for sm_100a.
//
// One fused row kernel serves every operator application of the path:
//   out = cx*X + alpha*Htilde(q) + beta*p,   Htilde q = (H q)/a - (b/a) q
// which is
//   * the Clenshaw recurrence  b_k = c_k X + 2 Htilde b_{k+1} - b_{k+2}
//     (Clenshaw.jl:69-81, vector_dispatch.jl:120-123) with b_k written in
//     place over b_{k+2} (each element is read then written by one thread);
//   * the final sum            Y = c_0 X + Htilde b_1 - b_2 (Clenshaw.jl:104-117);
//   * the KPM step             v_{n+1} = 2 Htilde v_n - v_{n-1} (Moments.jl:133-139)
//     with per-column <v_{n+1}, v_{n+1}> and <v_{n+1}, v_n> fused in;
//   * the plain / rescaled apply (Plan.jl:173-177, PolfedCore.jl:172).
//
// Blocks are row-interleaved (element (i, c) at i*s + c), so the s values a
// Hamiltonian flip gathers from row j are one contiguous 8*s or 4*s byte run.
// The matrix is never stored: each thread derives its row's basis state,
// diagonal and flipped neighbours from the operator descriptor.
//   * spin chain (SpinHalfChains.jl:267-315): diagonal sum_i h_i Sz_i +
//     sum_b J_b Delta_b Sz_i Sz_j in the reference's summation order (bit-exact
//     in FP64); one flip per bond with unequal spins, value J_b/2; the flipped
//     state's index comes from the combinatorial number system
//     rank(s) = sum_k C(p_k, k) (p_1 < p_2 < ... the set bits) evaluated with
//     per-byte lookup tables held in shared memory.
//   * Quantum Sun (QuantumSun.jl:1-102, S=1/2): index == state; L_loc flips
//     of (outer bit, grain bit) with value g0 c_j / 4, plus the dense grain
//     block on the low L_grain bits (held in shared memory).
#include "pf_internal.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

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

// ------------------------------------------------------------ row models
// Each returns (through acc / diag) the off-diagonal gather sum and the
// diagonal element of row `row` for columns c0..c0+V-1.

// Gathers are issued in unrolled batches of U independent loads so that each
// thread keeps several L2/HBM requests in flight (the loop bodies have no
// load-to-load dependence); accumulation follows the reference's term order.
// U shrinks as the per-thread column count V grows, to bound registers.
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

template <typename T, int V, bool HASQ>
__device__ __forceinline__ void chain_row(const ChainDesc<T> &d, const uint32_t *tab, uint32_t row,
                                          int s, int c0, const T *__restrict__ q, T (&acc)[V],
                                          T &diag) {
    constexpr int U = Batch<T, V>::U;
    const uint32_t st = d.full ? row : __ldg(d.states + row);
    T dg = T(0);
    for (int i = 0; i < d.L; ++i) dg += ((st >> i) & 1u) ? d.hhalf[i] : -d.hhalf[i];
    const T *qc = q + c0;
    for (int b0 = 0; b0 < d.nb; b0 += U) {
        uint32_t r2[U];
        bool act[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int b = b0 + u;
            act[u] = false;
            r2[u] = 0u;
            if (b < d.nb) {
                const uint32_t bm = d.bmask[b];
                const uint32_t m = st & bm;
                const bool differ = (m != 0u) && (m != bm);
                dg += differ ? -d.jdq[b] : d.jdq[b];
                act[u] = differ;
                if (HASQ && differ) {
                    const uint32_t st2 = st ^ bm;
                    r2[u] = d.full ? st2 : sector_rank(st2, tab, d.nchunks);
                }
            }
        }
        if constexpr (HASQ) {
            Pack<T, V> g[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (act[u]) g[u] = ldp<T, V>(qc + (size_t)r2[u] * s);
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (act[u]) {
                    const T jh = d.jhalf[b0 + u];
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[v] += jh * g[u].v[v];
                }
        }
    }
    diag = dg;
}

// Quantum Sun shared-memory layout: the grain block with a padded row stride
// (dg + 1, so the 8 rows of one grain group read different banks), then four
// 256-entry diagonal tables, one per byte of the outer-spin bits.
template <typename T>
struct QSunSmem {
    static __host__ __device__ int grain_stride(int dg) { return dg + 1; }
    static __host__ __device__ int bytes(int dg) { return (dg * (dg + 1) + 4 * 256) * (int)sizeof(T); }
};

template <typename T, int V, bool HASQ>
__device__ __forceinline__ void qsun_row(const QSunDesc<T> &d, const T *smem_t, uint32_t row,
                                         int s, int c0, const T *__restrict__ q, T (&acc)[V],
                                         T &diag) {
    constexpr int U = Batch<T, V>::U;
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
                    for (int v = 0; v < V; ++v) acc[v] += cf * g[u].v[v];
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
                    for (int v = 0; v < V; ++v) acc[v] += w * x[u].v[v];
                }
        }
    }
}

// CSR row (a user matrix): the entries of the row in storage order, gathered
// in unrolled batches of U like the matrix-free rows; the diagonal is an
// ordinary entry, so diag = 0.
template <typename T, int V, bool HASQ>
__device__ __forceinline__ void csr_row(const CsrDesc<T> &d, uint32_t row, int s, int c0, const T *__restrict__ q,
                                        T (&acc)[V], T &diag) {
    diag = T(0);
    if constexpr (HASQ) {
        constexpr int U = Batch<T, V>::U;
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
                    for (int v = 0; v < V; ++v) acc[v] += val[u] * g[u].v[v];
                }
        }
    }
}

template <typename T>
struct StepArgs {
    uint32_t D;
    int s;
    int G;          // column groups per row = s / V
    uint32_t items; // D * G
    const T *q;
    const T *p;     // may alias out (in-place update)
    const T *x;
    T *out;
    T cx, alpha, beta, inva, boa;
    double *partials;
    unsigned int *counter;
    double *dots;
};

template <class Desc>
struct DescTraits;
template <typename T>
struct DescTraits<ChainDesc<T>> {
    static constexpr int kind = OP_CHAIN;
};
template <typename T>
struct DescTraits<QSunDesc<T>> {
    static constexpr int kind = OP_QSUN;
};
template <typename T>
struct DescTraits<CsrDesc<T>> {
    static constexpr int kind = OP_CSR;
};

constexpr int kThreads = 256;

// Deterministic "last block reduces" epilogue: every block writes its
// per-column partials, the block that finishes last sums them in block order.
__device__ void finish_reduction(int nvals, const double *blockvals, double *partials,
                                 unsigned int *counter, double *out) {
    __shared__ bool last;
    for (int c = threadIdx.x; c < nvals; c += blockDim.x)
        partials[(size_t)blockIdx.x * nvals + c] = blockvals[c];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        for (int c = threadIdx.x; c < nvals; c += blockDim.x) {
            double acc = 0.0;
            for (unsigned int b = 0; b < gridDim.x; ++b)
                acc += ((volatile double *)partials)[(size_t)b * nvals + c];
            out[c] = acc;
        }
        if (threadIdx.x == 0) *counter = 0u;
    }
}

template <typename T, int V, class Desc, int FLAGS>
__global__ void __launch_bounds__(kThreads, MinBlocks<T, V>::value) k_step(const Desc d, const StepArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr bool HASQ = (FLAGS & StepFlags::Q) != 0;
    constexpr bool HASP = (FLAGS & StepFlags::P) != 0;
    constexpr bool HASX = (FLAGS & StepFlags::X) != 0;
    constexpr bool DOTS = (FLAGS & StepFlags::DOTS) != 0;
    const uint32_t *tab = reinterpret_cast<const uint32_t *>(smem_raw);
    const T *smem_t = reinterpret_cast<const T *>(smem_raw);
    if constexpr (DescTraits<Desc>::kind == OP_CHAIN) {
        if (HASQ && !d.full) {
            const int n = rank_table_entries(d.nchunks);
            uint32_t *t = reinterpret_cast<uint32_t *>(smem_raw);
            for (int i = threadIdx.x; i < n; i += blockDim.x) t[i] = __ldg(d.rank_tab + i);
        }
    } else if constexpr (DescTraits<Desc>::kind == OP_QSUN) {
        T *sm = reinterpret_cast<T *>(smem_raw);
        const int gs = d.dg + 1;
        for (int i = threadIdx.x; i < d.dg * d.dg; i += blockDim.x) sm[(i / d.dg) * gs + (i % d.dg)] = d.grain[i];
        T *dtab = sm + d.dg * gs;
        // dtab[c*256 + byte] = sum over the 8 outer spins of chunk c of h_j (bit - 1/2)
        for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) {
            const int c = i >> 8, byte = i & 255;
            T acc = T(0);
            for (int t = 0; t < 8; ++t) {
                const int j = 8 * c + t;
                if (j < d.L_loc) acc += ((byte >> t) & 1) ? d.hhalf[j] : -d.hhalf[j];
            }
            dtab[i] = acc;
        }
    }
    __syncthreads();

    double dd1[V], dd2[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dd1[v] = dd2[v] = 0.0;

    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t G = (uint32_t)a.G;
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < a.items; it += stride) {
        const uint32_t row = (G == 1u) ? it : it / G;
        const int c0 = (G == 1u) ? 0 : (int)(it - row * G) * V;
        const size_t off = (size_t)row * a.s + c0;
        T acc[V];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = T(0);
        T diag;
        if constexpr (DescTraits<Desc>::kind == OP_CHAIN)
            chain_row<T, V, HASQ>(d, tab, row, a.s, c0, a.q, acc, diag);
        else if constexpr (DescTraits<Desc>::kind == OP_QSUN)
            qsun_row<T, V, HASQ>(d, smem_t, row, a.s, c0, a.q, acc, diag);
        else
            csr_row<T, V, HASQ>(d, row, a.s, c0, a.q, acc, diag);
        Pack<T, V> res;
#pragma unroll
        for (int v = 0; v < V; ++v) res.v[v] = T(0);
        if constexpr (HASX) {
            const Pack<T, V> xo = ldp<T, V>(a.x + off);
#pragma unroll
            for (int v = 0; v < V; ++v) res.v[v] = a.cx * xo.v[v];
        }
        Pack<T, V> qo;
        if constexpr (HASQ) {
            qo = ldp<T, V>(a.q + off);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const T hq = (acc[v] + diag * qo.v[v]) * a.inva - a.boa * qo.v[v];
                res.v[v] = res.v[v] + a.alpha * hq;
            }
        }
        if constexpr (HASP) {
            const Pack<T, V> po = ldp<T, V>(a.p + off);
#pragma unroll
            for (int v = 0; v < V; ++v) res.v[v] = res.v[v] + a.beta * po.v[v];
        }
        stp<T, V>(a.out + off, res);
        if constexpr (DOTS) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
                dd1[v] += (double)res.v[v] * (double)res.v[v];
                if constexpr (HASQ) dd2[v] += (double)res.v[v] * (double)qo.v[v];
            }
        }
    }

    if constexpr (DOTS) {
        // Every item of a thread has column group threadIdx.x % G (G divides the
        // grid stride; checked on the host).  Lanes of one group are first
        // summed with warp shuffles, then per warp in shared memory.
        const int Gi = a.G;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (Gi < 32) {
#pragma unroll
            for (int v = 0; v < V; ++v)
                for (int o = 16; o >= Gi; o >>= 1) {
                    dd1[v] += __shfl_xor_sync(0xffffffffu, dd1[v], o);
                    dd2[v] += __shfl_xor_sync(0xffffffffu, dd2[v], o);
                }
        }
        const int lanes = Gi < 32 ? Gi : 32;
        __syncthreads();
        double *red = reinterpret_cast<double *>(smem_raw);  // [8 warps][lanes][2V]
        if (lane < lanes)
            for (int v = 0; v < V; ++v) {
                red[(warp * lanes + lane) * 2 * V + v] = dd1[v];
                red[(warp * lanes + lane) * 2 * V + V + v] = dd2[v];
            }
        __syncthreads();
        double *bv = red + (kThreads / 32) * lanes * 2 * V;  // [2 s]
        for (int c = threadIdx.x; c < a.s; c += blockDim.x) {
            const int g = c / V, v = c - g * V;
            double s1 = 0.0, s2 = 0.0;
            if (Gi < 32) {
                for (int w = 0; w < kThreads / 32; ++w) {
                    s1 += red[(w * lanes + g) * 2 * V + v];
                    s2 += red[(w * lanes + g) * 2 * V + V + v];
                }
            } else {
                for (int t = g; t < kThreads; t += Gi) {
                    const int w = t >> 5, l = t & 31;
                    s1 += red[(w * lanes + l) * 2 * V + v];
                    s2 += red[(w * lanes + l) * 2 * V + V + v];
                }
            }
            bv[c] = s1;
            bv[a.s + c] = s2;
        }
        __syncthreads();
        finish_reduction(2 * a.s, bv, a.partials, a.counter, a.dots);
    }
}

// ------------------------------------------------ warp-cooperative chain step
// Diagonal of a chain row: fields in site order, then the Sz Sz term of every
// bond in bond order -- the same sequence of additions chain_row performs, so
// the stored diagonal equals the one the per-thread kernels compute.
template <typename T>
__device__ __forceinline__ T chain_diag(const ChainDesc<T> &d, uint32_t st) {
    T dg = T(0);
    for (int i = 0; i < d.L; ++i) dg += ((st >> i) & 1u) ? d.hhalf[i] : -d.hhalf[i];
    for (int b = 0; b < d.nb; ++b) {
        const uint32_t bm = d.bmask[b];
        const uint32_t m = st & bm;
        const bool differ = (m != 0u) && (m != bm);
        dg += differ ? -d.jdq[b] : d.jdq[b];
    }
    return dg;
}

template <typename T>
__global__ void k_chain_diag(const ChainDesc<T> d, uint32_t D, T *__restrict__ out) {
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < D; row += gridDim.x * blockDim.x) {
        const uint32_t st = d.full ? row : __ldg(d.states + row);
        out[row] = chain_diag<T>(d, st);
    }
}

// One round of the cooperative step: lane lr ranks the flip of bond b0 + lr,
// the ranks are shuffled to every lane of the row (r[j] = rank of bond b0 + j,
// or all ones when that bond does not flip the state) and each lane gathers
// its column of every flipped neighbour.
template <typename T, int S>
__device__ __forceinline__ void coop_round(const ChainDesc<T> &d, const uint32_t *sbm, const uint32_t *tab,
                                           uint32_t st, bool valid, int b0, int lr, int rb, const T *qc,
                                           uint32_t (&r)[S], T (&g)[S]) {
    uint32_t mine = 0xffffffffu;
    const int b = b0 + lr;
    if (valid && b < d.nb) {
        const uint32_t bm = sbm[b];
        const uint32_t m = st & bm;
        if (m != 0u && m != bm) mine = d.full ? (st ^ bm) : sector_rank(st ^ bm, tab, d.nchunks);
    }
#pragma unroll
    for (int j = 0; j < S; ++j) {
        r[j] = __shfl_sync(0xffffffffu, mine, rb + j);
        g[j] = (r[j] != 0xffffffffu) ? __ldg(qc + (size_t)r[j] * S) : T(0);
    }
}

// One row per S lanes (S = s, a power of two <= 32), one column per lane.  The
// lanes of a row split its bonds: lane l ranks the flipped states of bonds
// l, l+S, l+2S, ...; one shuffle per bond hands the rank to every lane of the
// row, and each lane gathers its own column.  A round issues S independent
// gathers per lane with one register each, and the row's rank work is done
// once instead of once per column group.  Gathers are accumulated in bond
// order and the diagonal comes from k_chain_diag, so every output equals the
// per-thread kernel's.  One-column lanes issue 4- or 8-byte gathers, so the
// variant pays where latency, not load-instruction throughput, bounds the
// step: small D.  Shared memory: the bond masks (lane-indexed, so not
// read from the kernel parameters), then the rank tables.
template <typename T, int S, int FLAGS>
__global__ void __launch_bounds__(kThreads) k_step_coop(const ChainDesc<T> d, const StepArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr bool HASQ = (FLAGS & StepFlags::Q) != 0;
    constexpr bool HASP = (FLAGS & StepFlags::P) != 0;
    constexpr bool HASX = (FLAGS & StepFlags::X) != 0;
    uint32_t *sbm = reinterpret_cast<uint32_t *>(smem_raw);
    uint32_t *tab = sbm + PF_MAX_BONDS;
    if constexpr (HASQ) {
        for (int i = threadIdx.x; i < d.nb; i += blockDim.x) sbm[i] = d.bmask[i];
        if (!d.full) {
            const int n = rank_table_entries(d.nchunks);
            for (int i = threadIdx.x; i < n; i += blockDim.x) tab[i] = __ldg(d.rank_tab + i);
        }
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const int lr = lane & (S - 1);   // this lane's column
    const int rb = lane & ~(S - 1);  // first lane of this lane's row
    const uint64_t total = (uint64_t)a.D * S;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // warp-uniform loop: every lane of a warp runs the same iterations (shuffles)
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
        const uint64_t t = base + lane;
        const bool valid = t < total;
        const uint32_t row = valid ? (uint32_t)(t / S) : 0u;
        // the row's own operands, diagonal and basis state are independent
        // loads: issue them together, ahead of the gathers
        T xo = T(0), qo = T(0), po = T(0), dgv = T(0);
        uint32_t st = 0u;
        if (valid) {
            if constexpr (HASX) xo = a.x[t];
            if constexpr (HASQ) {
                qo = a.q[t];
                dgv = d.diag[row];
                st = d.full ? row : __ldg(d.states + row);
            }
            if constexpr (HASP) po = a.p[t];
        }
        T acc = T(0);
        if constexpr (HASQ) {
            const T *qc = a.q + lr;
            for (int b0 = 0; b0 < d.nb; b0 += S) {
                uint32_t r[S];
                T g[S];
                coop_round<T, S>(d, sbm, tab, st, valid, b0, lr, rb, qc, r, g);
#pragma unroll
                for (int j = 0; j < S; ++j)
                    if (r[j] != 0xffffffffu) acc += d.jhalf[b0 + j] * g[j];
            }
        }
        if (valid) {
            T res = T(0);
            if constexpr (HASX) res = a.cx * xo;
            if constexpr (HASQ) {
                const T hq = (acc + dgv * qo) * a.inva - a.boa * qo;
                res = res + a.alpha * hq;
            }
            if constexpr (HASP) res = res + a.beta * po;
            a.out[t] = res;
        }
    }
}


static thread_local int64_t t_launches = 0;
void count_launches(int64_t n) { t_launches += n; }
int64_t thread_launches() { return t_launches; }

int grid_for(pf_handle *h, int64_t work_items, int threads, int blocks_per_sm) {
    int64_t need = (work_items + threads - 1) / threads;
    int64_t cap = (int64_t)h->num_sms * blocks_per_sm;
    if (need < 1) need = 1;
    return (int)std::min(need, cap);
}

void ensure_reduction(pf_handle *h, size_t n) {
    if (h->red_partials_len >= n) return;
    if (h->red_partials) cudaFree(h->red_partials);
    h->red_partials = nullptr;
    h->red_partials_len = 0;
    PF_CUDA(cudaMalloc(&h->red_partials, n * sizeof(double)));
    h->red_partials_len = n;
    if (!h->red_counter) {
        PF_CUDA(cudaMalloc(&h->red_counter, 64 * sizeof(unsigned int)));
        PF_CUDA(cudaMemset(h->red_counter, 0, 64 * sizeof(unsigned int)));
    }
}

// Resident CTAs per SM of a kernel instance (occupancy calculator, cached per
// host thread so concurrent solves do not contend on a lock every launch).
static int blocks_per_sm(const void *kern, int smem) {
    thread_local std::map<std::pair<const void *, int>, int> cache;
    auto key = std::make_pair(kern, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int nb = 0;
    PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, kThreads, smem));
    if (nb < 1) nb = 1;
    cache[key] = nb;
    return nb;
}

template <typename T, int V, class Desc, int FLAGS>
static void launch_one(pf_op *op, cudaStream_t st, const Desc &d, StepArgs<T> a, int smem) {
    auto kern = k_step<T, V, Desc, FLAGS>;
    if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    // one item per thread when the whole block fits on the device at once,
    // otherwise a persistent grid of every resident CTA
    const int grid = grid_for(op->h, a.items, kThreads, blocks_per_sm((const void *)kern, smem));
    if constexpr ((FLAGS & StepFlags::DOTS) != 0) {
        ensure_reduction(op->h, (size_t)grid * 2 * a.s);
        a.partials = op->h->red_partials;
        a.counter = op->h->red_counter;
    }
    kern<<<grid, kThreads, smem, st>>>(d, a);
    PF_CUDA(cudaGetLastError());
    count_launches(1);
}

template <typename T, int V, class Desc>
static void dispatch_flags(pf_op *op, cudaStream_t st, const Desc &d, const StepArgs<T> &a,
                           int flags, int smem) {
    using F = StepFlags;
    switch (flags) {
        case F::X: launch_one<T, V, Desc, F::X>(op, st, d, a, smem); break;
        case F::Q: launch_one<T, V, Desc, F::Q>(op, st, d, a, smem); break;
        case F::Q | F::X: launch_one<T, V, Desc, F::Q | F::X>(op, st, d, a, smem); break;
        case F::Q | F::P: launch_one<T, V, Desc, F::Q | F::P>(op, st, d, a, smem); break;
        case F::Q | F::P | F::X: launch_one<T, V, Desc, F::Q | F::P | F::X>(op, st, d, a, smem); break;
        case F::Q | F::DOTS: launch_one<T, V, Desc, F::Q | F::DOTS>(op, st, d, a, smem); break;
        case F::Q | F::P | F::DOTS:
            launch_one<T, V, Desc, F::Q | F::P | F::DOTS>(op, st, d, a, smem);
            break;
        default: throw Error(PF_ERR_INVALID, "unsupported step flag combination");
    }
}

template <typename T>
static const ChainDesc<T> &chain_of(pf_op *op);
template <>
const ChainDesc<double> &chain_of<double>(pf_op *op) { return op->chain64; }
template <>
const ChainDesc<float> &chain_of<float>(pf_op *op) { return op->chain32; }
template <typename T>
static const QSunDesc<T> &qsun_of(pf_op *op);
template <>
const QSunDesc<double> &qsun_of<double>(pf_op *op) { return op->qsun64; }
template <>
const QSunDesc<float> &qsun_of<float>(pf_op *op) { return op->qsun32; }

template <typename T>
static const CsrDesc<T> &csr_of(pf_op *op);
template <>
const CsrDesc<double> &csr_of<double>(pf_op *op) { return op->csr64; }
template <>
const CsrDesc<float> &csr_of<float>(pf_op *op) { return op->csr32; }

template <typename T, int V>
static void dispatch_op(pf_op *op, cudaStream_t st, const StepArgs<T> &a, int flags) {
    int smem = 0;
    const int lanes = a.G < 32 ? a.G : 32;
    const int dots_smem = (kThreads / 32) * lanes * 2 * V * 8 + 2 * a.s * 8;
    if (op->kind == OP_CHAIN) {
        const ChainDesc<T> &d = chain_of<T>(op);
        if ((flags & StepFlags::Q) && !d.full) smem = rank_table_entries(d.nchunks) * 4;
        if (flags & StepFlags::DOTS) smem = std::max(smem, dots_smem);
        dispatch_flags<T, V>(op, st, d, a, flags, smem);
    } else if (op->kind == OP_QSUN) {
        const QSunDesc<T> &d = qsun_of<T>(op);
        smem = QSunSmem<T>::bytes(d.dg);
        if (flags & StepFlags::DOTS) smem = std::max(smem, dots_smem);
        dispatch_flags<T, V>(op, st, d, a, flags, smem);
    } else {
        const CsrDesc<T> &d = csr_of<T>(op);
        if (flags & StepFlags::DOTS) smem = dots_smem;
        dispatch_flags<T, V>(op, st, d, a, flags, smem);
    }
}

bool coop_eligible(const pf_op *op, int s, int flags) {
    return op->kind == OP_CHAIN && op->d_diag64 != nullptr && op->d_diag32 != nullptr &&
           (s == 4 || s == 8 || s == 16 || s == 32) && (flags & StepFlags::DOTS) == 0;
}

template <typename T, int S, int FLAGS>
static void launch_coop_one(pf_op *op, cudaStream_t st, const ChainDesc<T> &d, const StepArgs<T> &a) {
    auto kern = k_step_coop<T, S, FLAGS>;
    int smem = PF_MAX_BONDS * 4;
    if ((FLAGS & StepFlags::Q) && !d.full) smem += rank_table_entries(d.nchunks) * 4;
    if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int grid = grid_for(op->h, (int64_t)a.D * S, kThreads, blocks_per_sm((const void *)kern, smem));
    kern<<<grid, kThreads, smem, st>>>(d, a);
    PF_CUDA(cudaGetLastError());
    count_launches(1);
}

template <typename T, int S>
static void coop_flags(pf_op *op, cudaStream_t st, const ChainDesc<T> &d, const StepArgs<T> &a, int flags) {
    using F = StepFlags;
    switch (flags) {
        case F::X: launch_coop_one<T, S, F::X>(op, st, d, a); break;
        case F::Q: launch_coop_one<T, S, F::Q>(op, st, d, a); break;
        case F::Q | F::X: launch_coop_one<T, S, F::Q | F::X>(op, st, d, a); break;
        case F::Q | F::P: launch_coop_one<T, S, F::Q | F::P>(op, st, d, a); break;
        case F::Q | F::P | F::X: launch_coop_one<T, S, F::Q | F::P | F::X>(op, st, d, a); break;
        default: throw Error(PF_ERR_INVALID, "unsupported step flag combination");
    }
}

template <typename T>
static void launch_coop(pf_op *op, cudaStream_t st, const StepArgs<T> &a, int flags) {
    const ChainDesc<T> &d = chain_of<T>(op);
    PF_CHECK(d.diag != nullptr, PF_ERR_INVALID, "chain diagonal missing");
    switch (a.s) {
        case 4: coop_flags<T, 4>(op, st, d, a, flags); break;
        case 8: coop_flags<T, 8>(op, st, d, a, flags); break;
        case 16: coop_flags<T, 16>(op, st, d, a, flags); break;
        case 32: coop_flags<T, 32>(op, st, d, a, flags); break;
        default: throw Error(PF_ERR_INVALID, "the warp-cooperative step needs s in {4, 8, 16, 32}");
    }
}

void build_chain_diag(pf_op *op) {
    PF_CHECK(op->kind == OP_CHAIN, PF_ERR_INVALID, "not a chain operator");
    const uint64_t D = (uint64_t)op->dim;
    if ((double)D * 12.0 > 4.0 * (double)(1ull << 30)) return;  // the cooperative step is not offered
    PF_CUDA(cudaMalloc(&op->d_diag64, D * sizeof(double)));
    PF_CUDA(cudaMalloc(&op->d_diag32, D * sizeof(float)));
    cudaStream_t st = op->h->stream;
    const int grid = grid_for(op->h, (int64_t)D, kThreads, 8);
    k_chain_diag<double><<<grid, kThreads, 0, st>>>(op->chain64, (uint32_t)D, op->d_diag64);
    k_chain_diag<float><<<grid, kThreads, 0, st>>>(op->chain32, (uint32_t)D, op->d_diag32);
    PF_CUDA(cudaGetLastError());
    count_launches(2);
    PF_CUDA(cudaStreamSynchronize(st));
    op->chain64.diag = op->d_diag64;
    op->chain32.diag = op->d_diag32;
}

// Columns per thread: the widest power of two dividing s within one 64-byte
// run by default, or the width the autotuner measured fastest for (s, dtype).
int default_width(int s, int elem_bytes) {
    const int vmax = 64 / elem_bytes;
    for (int w = vmax; w >= 1; w /= 2)
        if (s % w == 0) return w;
    return 1;
}

template <typename T>
void launch_step_width(pf_op *op, cudaStream_t st, int64_t D, int s, const T *q, const T *p, const T *x, T *out,
                       double cx, double alpha, double beta, double inva, double shift, int flags, double *dots,
                       int V) {
    PF_CHECK(D == op->dim, PF_ERR_INVALID, "block height does not match the operator dimension");
    PF_CHECK(s >= 1, PF_ERR_INVALID, "block must have at least one column");
    const bool coop = (V == kCoopWidth);
    PF_CHECK(!coop || coop_eligible(op, s, flags), PF_ERR_INVALID,
             "the warp-cooperative step needs a chain operator, s in {4, 8, 16, 32} and no fused dots");
    PF_CHECK(coop || (V >= 1 && s % V == 0 && V * (int)sizeof(T) <= 64), PF_ERR_INVALID,
             "invalid columns-per-thread width");
    StepArgs<T> a;
    a.D = (uint32_t)D;
    a.s = s;
    a.G = coop ? s : s / V;
    PF_CHECK((int64_t)D * a.G < (int64_t)0xffffffffLL, PF_ERR_UNSUPPORTED, "block too large for one launch");
    a.items = (uint32_t)(D * a.G);
    a.q = q; a.p = p; a.x = x; a.out = out;
    a.cx = (T)cx; a.alpha = (T)alpha; a.beta = (T)beta;
    a.inva = (T)inva; a.boa = (T)(shift * inva);
    a.partials = nullptr; a.counter = nullptr; a.dots = dots;
    if (coop) {
        launch_coop<T>(op, st, a, flags);
        return;
    }
    if (flags & StepFlags::DOTS)
        PF_CHECK(kThreads % a.G == 0, PF_ERR_UNSUPPORTED, "fused dots need s/V to divide 256");
    switch (V) {
        case 1: dispatch_op<T, 1>(op, st, a, flags); break;
        case 2: dispatch_op<T, 2>(op, st, a, flags); break;
        case 4: dispatch_op<T, 4>(op, st, a, flags); break;
        case 8: dispatch_op<T, 8>(op, st, a, flags); break;
        case 16:
            if constexpr (sizeof(T) == 4) { dispatch_op<T, 16>(op, st, a, flags); break; }
            [[fallthrough]];
        default: throw Error(PF_ERR_INVALID, "bad vector width");
    }
}

template <typename T>
void launch_step(pf_op *op, cudaStream_t st, int64_t D, int s, const T *q, const T *p,
                 const T *x, T *out, double cx, double alpha, double beta, double inva,
                 double shift, int flags, double *dots) {
    int V = default_width(s, (int)sizeof(T));
    {
        std::lock_guard<std::mutex> lock(op->tune_mu);
        auto it = op->tuned_width.find(std::make_pair((int)sizeof(T), s));
        if (it != op->tuned_width.end()) V = it->second;
    }
    if (flags & StepFlags::DOTS) {
        // the fused dots keep 2V FP64 accumulators per thread: at most 32 bytes of columns
        V = default_width(s, (int)sizeof(T));
        while (V > 1 && (V * (int)sizeof(T) > 32 || kThreads % (s / V) != 0)) V /= 2;
    }
    if (V == kCoopWidth && !coop_eligible(op, s, flags)) V = default_width(s, (int)sizeof(T));
    launch_step_width<T>(op, st, D, s, q, p, x, out, cx, alpha, beta, inva, shift, flags, dots, V);
}

template void launch_step_width<double>(pf_op *, cudaStream_t, int64_t, int, const double *, const double *,
                                        const double *, double *, double, double, double, double, double, int,
                                        double *, int);
template void launch_step_width<float>(pf_op *, cudaStream_t, int64_t, int, const float *, const float *,
                                       const float *, float *, double, double, double, double, double, int,
                                       double *, int);
template void launch_step<double>(pf_op *, cudaStream_t, int64_t, int, const double *, const double *,
                                  const double *, double *, double, double, double, double, double,
                                  int, double *);
template void launch_step<float>(pf_op *, cudaStream_t, int64_t, int, const float *, const float *,
                                 const float *, float *, double, double, double, double, double,
                                 int, double *);

// --------------------------------------------------------- layout changes
template <typename TS, typename TD>
__global__ void k_cm_to_ri(uint32_t D, int s, const TS *__restrict__ src, int64_t ld, TD *__restrict__ dst) {
    // tile 32 rows x 32 cols through shared memory
    __shared__ TD tile[32][33];
    const uint32_t r0 = blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k;
        const uint32_t r = r0 + threadIdx.x;
        if (c < s && r < D) tile[k][threadIdx.x] = (TD)src[(size_t)c * ld + r];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const uint32_t r = r0 + k;
        const int c = c0 + threadIdx.x;
        if (c < s && r < D) dst[(size_t)r * s + c] = tile[threadIdx.x][k];
    }
}

template <typename TS, typename TD>
__global__ void k_ri_to_cm(uint32_t D, int s, const TS *__restrict__ src, TD *__restrict__ dst, int64_t ld) {
    __shared__ TD tile[32][33];
    const uint32_t r0 = blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const uint32_t r = r0 + k;
        const int c = c0 + threadIdx.x;
        if (c < s && r < D) tile[k][threadIdx.x] = (TD)src[(size_t)r * s + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k;
        const uint32_t r = r0 + threadIdx.x;
        if (c < s && r < D) dst[(size_t)c * ld + r] = tile[threadIdx.x][k];
    }
}

template <typename TS, typename TD>
void launch_cm_to_ri(cudaStream_t st, int64_t D, int s, const TS *src, int64_t ld, TD *dst) {
    dim3 grid((unsigned)((D + 31) / 32), (unsigned)((s + 31) / 32));
    k_cm_to_ri<TS, TD><<<grid, dim3(32, 8), 0, st>>>((uint32_t)D, s, src, ld, dst);
    count_launches(1);
    PF_CUDA(cudaGetLastError());
}
template <typename TS, typename TD>
void launch_ri_to_cm(cudaStream_t st, int64_t D, int s, const TS *src, TD *dst, int64_t ld) {
    dim3 grid((unsigned)((D + 31) / 32), (unsigned)((s + 31) / 32));
    k_ri_to_cm<TS, TD><<<grid, dim3(32, 8), 0, st>>>((uint32_t)D, s, src, dst, ld);
    count_launches(1);
    PF_CUDA(cudaGetLastError());
}
template void launch_cm_to_ri<double, double>(cudaStream_t, int64_t, int, const double *, int64_t, double *);
template void launch_cm_to_ri<float, float>(cudaStream_t, int64_t, int, const float *, int64_t, float *);
template void launch_cm_to_ri<double, float>(cudaStream_t, int64_t, int, const double *, int64_t, float *);
template void launch_ri_to_cm<double, double>(cudaStream_t, int64_t, int, const double *, double *, int64_t);
template void launch_ri_to_cm<float, float>(cudaStream_t, int64_t, int, const float *, float *, int64_t);
template void launch_ri_to_cm<float, double>(cudaStream_t, int64_t, int, const float *, double *, int64_t);
template void launch_ri_to_cm<double, float>(cudaStream_t, int64_t, int, const double *, float *, int64_t);
template void launch_cm_to_ri<float, double>(cudaStream_t, int64_t, int, const float *, int64_t, double *);

// ------------------------------------------------------- column reductions
template <typename T>
__global__ void __launch_bounds__(kThreads) k_coldots(uint32_t D, int s, uint32_t rows_per_block,
                                                     const T *__restrict__ A, const T *__restrict__ B,
                                                     double *partials, unsigned int *counter, double *out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *bv = reinterpret_cast<double *>(smem_raw);
    const uint32_t r0 = blockIdx.x * rows_per_block;
    const uint32_t r1 = min(D, r0 + rows_per_block);
    for (int c = threadIdx.x; c < s; c += blockDim.x) {
        double acc = 0.0;
        for (uint32_t r = r0; r < r1; ++r) acc += (double)A[(size_t)r * s + c] * (double)B[(size_t)r * s + c];
        bv[c] = acc;
    }
    __syncthreads();
    finish_reduction(s, bv, partials, counter, out);
}

__global__ void __launch_bounds__(kThreads) k_colresid(uint32_t D, int s, uint32_t rows_per_block,
                                                      const double *__restrict__ HA, const double *__restrict__ A,
                                                      const double *__restrict__ e, double *partials,
                                                      unsigned int *counter, double *out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *bv = reinterpret_cast<double *>(smem_raw);
    const uint32_t r0 = blockIdx.x * rows_per_block;
    const uint32_t r1 = min(D, r0 + rows_per_block);
    for (int c = threadIdx.x; c < s; c += blockDim.x) {
        const double ec = e[c];
        double acc = 0.0;
        for (uint32_t r = r0; r < r1; ++r) {
            const double d = HA[(size_t)r * s + c] - ec * A[(size_t)r * s + c];
            acc += d * d;
        }
        bv[c] = acc;
    }
    __syncthreads();
    finish_reduction(s, bv, partials, counter, out);
}

// For narrow blocks (s < 64) the per-column loops above leave most threads
// idle; this variant gives each thread a strided set of rows of one column.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_coldots_narrow(uint32_t D, int s, const T *__restrict__ A,
                                                            const T *__restrict__ B, double *partials,
                                                            unsigned int *counter, double *out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *red = reinterpret_cast<double *>(smem_raw);  // [kThreads]
    double *bv = red + kThreads;                          // [s]
    // lanes of one row group: threads t with t % s == c handle column c
    const int per = kThreads / s;  // row slots per block iteration
    const int t = threadIdx.x;
    double acc = 0.0;
    if (t < per * s) {
        const int c = t % s, slot = t / s;
        for (uint32_t r = blockIdx.x * per + slot; r < D; r += gridDim.x * per)
            acc += (double)A[(size_t)r * s + c] * (double)B[(size_t)r * s + c];
    }
    red[t] = acc;
    __syncthreads();
    for (int c = t; c < s; c += blockDim.x) {
        double a = 0.0;
        for (int q = c; q < per * s; q += s) a += red[q];
        bv[c] = a;
    }
    __syncthreads();
    finish_reduction(s, bv, partials, counter, out);
}

template <typename T>
void launch_coldots(pf_handle *h, cudaStream_t st, int64_t D, int s, const T *A, const T *B, double *out) {
    if (s < 64) {
        int grid = grid_for(h, D * s, kThreads, 2);
        ensure_reduction(h, (size_t)grid * s);
        size_t smem = (kThreads + s) * sizeof(double);
        k_coldots_narrow<T><<<grid, kThreads, smem, st>>>((uint32_t)D, s, A, B, h->red_partials,
                                                          h->red_counter, out);
        count_launches(1);
    } else {
        uint32_t rpb = 64;
        int grid = (int)((D + rpb - 1) / rpb);
        if (grid > 4 * h->num_sms) {
            rpb = (uint32_t)((D + 4 * h->num_sms - 1) / (4 * h->num_sms));
            grid = (int)((D + rpb - 1) / rpb);
        }
        ensure_reduction(h, (size_t)grid * s);
        size_t smem = s * sizeof(double);
        if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(k_coldots<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_coldots<T><<<grid, kThreads, smem, st>>>((uint32_t)D, s, rpb, A, B, h->red_partials,
                                                   h->red_counter, out);
        count_launches(1);
    }
    PF_CUDA(cudaGetLastError());
}
template void launch_coldots<double>(pf_handle *, cudaStream_t, int64_t, int, const double *, const double *, double *);
template void launch_coldots<float>(pf_handle *, cudaStream_t, int64_t, int, const float *, const float *, double *);

void launch_colresid(pf_handle *h, cudaStream_t st, int64_t D, int s, const double *HA, const double *A,
                     const double *e, double *out) {
    uint32_t rpb = 64;
    int grid = (int)((D + rpb - 1) / rpb);
    if (grid > 4 * h->num_sms) {
        rpb = (uint32_t)((D + 4 * h->num_sms - 1) / (4 * h->num_sms));
        grid = (int)((D + rpb - 1) / rpb);
    }
    ensure_reduction(h, (size_t)grid * s);
    size_t smem = s * sizeof(double);
    if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(k_colresid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_colresid<<<grid, kThreads, smem, st>>>((uint32_t)D, s, rpb, HA, A, e, h->red_partials, h->red_counter, out);
    count_launches(1);
    PF_CUDA(cudaGetLastError());
}

// --------------------------------------------------------------- probes
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    // splitmix64 finaliser (Steele, Lea, Flood 2014)
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

template <typename T>
__global__ void k_probes(uint32_t D, int R, int kind, uint64_t seed, int col0, T *dst) {
    const uint64_t n = (uint64_t)D * R;
    for (uint64_t it = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; it < n;
         it += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t row = it / R;
        const int c = (int)(it - row * R);
        const uint64_t key = ((uint64_t)(col0 + c) << 32) ^ row;
        const uint64_t h1 = mix64(seed ^ mix64(key));
        double val;
        if (kind == PF_PROBE_RADEMACHER) {
            val = (h1 & 1ull) ? 1.0 : -1.0;
        } else {
            // Box-Muller on two 53-bit uniforms in (0, 1]
            const uint64_t h2 = mix64(h1 ^ 0xd1b54a32d192ed03ULL);
            const double u1 = ((double)(h1 >> 11) + 1.0) * (1.0 / 9007199254740992.0);
            const double u2 = (double)(h2 >> 11) * (1.0 / 9007199254740992.0);
            val = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
        }
        dst[it] = (T)val;
    }
}

template <typename T>
void launch_probes(cudaStream_t st, int64_t D, int R, int kind, uint64_t seed, int col0, T *dst) {
    int grid = (int)std::min<int64_t>((D * R + 255) / 256, 148 * 8);
    k_probes<T><<<grid, 256, 0, st>>>((uint32_t)D, R, kind, seed, col0, dst);
    count_launches(1);
    PF_CUDA(cudaGetLastError());
}
template void launch_probes<double>(cudaStream_t, int64_t, int, int, uint64_t, int, double *);
template void launch_probes<float>(cudaStream_t, int64_t, int, int, uint64_t, int, float *);

template <typename T>
__global__ void k_scale_cols(uint32_t D, int s, T *A, const double *scale) {
    const uint64_t n = (uint64_t)D * s;
    for (uint64_t it = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; it < n;
         it += (uint64_t)gridDim.x * blockDim.x) {
        const int c = (int)(it % s);
        A[it] = (T)((double)A[it] * scale[c]);
    }
}
template <typename T>
void launch_scale_cols(cudaStream_t st, int64_t D, int s, T *A, const double *scale) {
    int grid = (int)std::min<int64_t>((D * s + 255) / 256, 148 * 8);
    k_scale_cols<T><<<grid, 256, 0, st>>>((uint32_t)D, s, A, scale);
    count_launches(1);
    PF_CUDA(cudaGetLastError());
}
template void launch_scale_cols<double>(cudaStream_t, int64_t, int, double *, const double *);
template void launch_scale_cols<float>(cudaStream_t, int64_t, int, float *, const double *);

// --------------------------------------------------------------- basis
__global__ void k_unrank(uint64_t n, int full, uint32_t D, const uint32_t *states, const int64_t *idx,
                         uint64_t *out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const int64_t k = idx[i];
        if (k < 0 || (uint64_t)k >= D) out[i] = ~0ull;
        else out[i] = full ? (uint64_t)k : (uint64_t)states[k];
    }
}

__global__ void k_rank(uint64_t n, int L, int Lup, int full, int nchunks, const uint32_t *tab,
                       const uint64_t *states, int64_t *out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t *t = reinterpret_cast<uint32_t *>(smem_raw);
    if (!full) {
        const int ne = rank_table_entries(nchunks);
        for (int i = threadIdx.x; i < ne; i += blockDim.x) t[i] = tab[i];
    }
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t st = states[i];
        if ((L < 64 && (st >> L) != 0ull)) { out[i] = -1; continue; }
        if (full) { out[i] = (int64_t)st; continue; }
        if (__popcll(st) != Lup) { out[i] = -1; continue; }
        out[i] = (int64_t)sector_rank((uint32_t)st, t, nchunks);
    }
}

void launch_unrank(pf_op *op, cudaStream_t st, int64_t n, const int64_t *idx, uint64_t *out) {
    if (n <= 0) return;
    int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    k_unrank<<<grid, 256, 0, st>>>((uint64_t)n, op->chain64.full, (uint32_t)op->dim, op->d_states, idx, out);
    count_launches(1);
    PF_CUDA(cudaGetLastError());
}

void launch_rank(pf_op *op, cudaStream_t st, int64_t n, const uint64_t *states, int64_t *out) {
    if (n <= 0) return;
    const ChainDesc<double> &d = op->chain64;
    int smem = d.full ? 0 : rank_table_entries(d.nchunks) * 4;
    if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(k_rank, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 4);
    k_rank<<<grid, 256, smem, st>>>((uint64_t)n, d.L, d.Lup, d.full, d.nchunks, op->d_rank_tab, states, out);
    count_launches(1);
    PF_CUDA(cudaGetLastError());
}

}  // namespace pf
