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
#include "pf_rows.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

namespace pf {

template <typename T>
struct StepArgs {
    uint32_t D;
    int s;          // columns processed per row
    int ld;         // row stride of the blocks (>= s: a column slab of a wider RI block)
    int stream;     // 1: x, p and out move with evict-first hints (slab passes)
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
// The partials are read through L2 (__ldcg: other blocks wrote them before
// the counter told this block it is last) in unrolled runs, so a run's loads
// are in flight together while the sum keeps block order.
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
        const unsigned int nb = gridDim.x;
        for (int c = threadIdx.x; c < nvals; c += blockDim.x) {
            double acc = 0.0;
            const double *col = partials + c;
#pragma unroll 8
            for (unsigned int b = 0; b < nb; ++b) acc += __ldcg(col + (size_t)b * nvals);
            out[c] = acc;
        }
        if (threadIdx.x == 0) *counter = 0u;
    }
}

// UB > 0 / MB > 0: a tuned variant's gather batch and resident-CTA target
// (register cap); 0 keeps the defaults of Batch / MinBlocks.  RK = 1 (chain
// operators): flip ranks by the local update of flip_rank_local, with the
// binomial table staged after the rank tables.
template <typename T, int V, class Desc, int FLAGS, int UB = 0, int MB = 0, int RK = 0>
__global__ void __launch_bounds__(kThreads, MB > 0 ? MB : MinBlocks<T, V>::value)
    k_step(const Desc d, const StepArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_trigger();
    constexpr bool HASQ = (FLAGS & StepFlags::Q) != 0;
    constexpr bool HASP = (FLAGS & StepFlags::P) != 0;
    constexpr bool HASX = (FLAGS & StepFlags::X) != 0;
    constexpr bool DOTS = (FLAGS & StepFlags::DOTS) != 0;
    const uint32_t *tab = reinterpret_cast<const uint32_t *>(smem_raw);
    const T *smem_t = reinterpret_cast<const T *>(smem_raw);
    const uint32_t *ctab = nullptr;
    if constexpr (DescTraits<Desc>::kind == OP_CHAIN) {
        if (HASQ && !d.full) {
            const int n = rank_table_entries(d.nchunks);
            uint32_t *t = reinterpret_cast<uint32_t *>(smem_raw);
            for (int i = threadIdx.x; i < n; i += blockDim.x) t[i] = __ldg(d.rank_tab + i);
            if constexpr (RK == 1) {
                uint32_t *c = t + n;   // C(nn, k) for nn, k <= 32
                for (int i = threadIdx.x; i < 33 * 33; i += blockDim.x) {
                    const int nn = i / 33, k = i % 33;
                    uint64_t r = k <= nn ? 1u : 0u;
                    for (int q = 1; q <= k && q <= nn; ++q) r = r * (uint64_t)(nn - k + q) / (uint64_t)q;
                    c[i] = (uint32_t)r;
                }
                ctab = c;
            }
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
    pdl_wait();

    double dd1[V], dd2[V];
#pragma unroll
    for (int v = 0; v < V; ++v) dd1[v] = dd2[v] = 0.0;

    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t G = (uint32_t)a.G;
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < a.items; it += stride) {
        const uint32_t row = (G == 1u) ? it : it / G;
        const int c0 = (G == 1u) ? 0 : (int)(it - row * G) * V;
        const size_t off = (size_t)row * a.ld + c0;
        if constexpr (HASX) prefetch_l1(a.x + off);
        if constexpr (HASQ) prefetch_l1(a.q + off);
        if constexpr (HASP) prefetch_l1(a.p + off);
        T acc[V];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = T(0);
        T diag;
        if constexpr (DescTraits<Desc>::kind == OP_CHAIN && RK == 1)
            chain_row_local<T, V, HASQ, UB>(d, tab, ctab, row, a.ld, c0, a.q, acc, diag);
        else if constexpr (DescTraits<Desc>::kind == OP_CHAIN)
            chain_row<T, V, HASQ, UB>(d, tab, row, a.ld, c0, a.q, acc, diag);
        else if constexpr (DescTraits<Desc>::kind == OP_QSUN)
            qsun_row<T, V, HASQ, UB>(d, smem_t, row, a.ld, c0, a.q, acc, diag);
        else
            csr_row<T, V, HASQ, UB>(d, row, a.ld, c0, a.q, acc, diag);
        Pack<T, V> xo, qo, po, res;
#pragma unroll
        for (int v = 0; v < V; ++v) xo.v[v] = qo.v[v] = po.v[v] = T(0);
        if constexpr (HASX) xo = ldp_hint<T, V>(a.x + off, a.stream);
        if constexpr (HASQ) qo = ldp<T, V>(a.q + off);
        if constexpr (HASP) po = ldp_hint<T, V>(a.p + off, a.stream);
#pragma unroll
        for (int v = 0; v < V; ++v)
            res.v[v] = step_combine<T>(HASX, HASQ, HASP, a.cx, xo.v[v], a.alpha, acc[v], diag, qo.v[v], a.inva, a.boa,
                                       a.beta, po.v[v]);
        stp_hint<T, V>(a.out + off, res, a.stream);
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
    pdl_trigger();
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
    pdl_wait();
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
                    if (r[j] != 0xffffffffu) acc = fma_t(d.jhalf[b0 + j], g[j], acc);
            }
        }
        if (valid) {
            const T res = step_combine<T>(HASX, HASQ, HASP, a.cx, xo, a.alpha, acc, dgv, qo, a.inva, a.boa, a.beta, po);
            a.out[t] = res;
        }
    }
}


// ------------------------------------------------ asynchronous-gather QSun step
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Byte offset of the gather slots in k_step_qsun_async's shared memory.
template <typename T>
__host__ __device__ inline int qsun_async_slot_offset() {
    return (QSunSmem<T>::bytes(PF_MAX_GRAIN) + 15) / 16 * 16;
}

// Quantum Sun step whose row gathers are asynchronous global->shared copies
// (cp.async): all L_loc flipped rows and dg grain rows of an item are in
// flight at once while no register holds them, instead of a few per dependent
// round.  Each thread then waits for its own copies (no barrier: a thread
// reads only its own slots, laid out so consecutive threads read consecutive
// 16-byte words) and accumulates in qsun_row's order -- flips, then the grain
// row -- with the same rounded operations, so results equal every other
// variant's.
template <typename T, int V, int FLAGS>
__global__ void __launch_bounds__(kThreads) k_step_qsun_async(const QSunDesc<T> d, const StepArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_trigger();
    constexpr bool HASP = (FLAGS & StepFlags::P) != 0;
    constexpr bool HASX = (FLAGS & StepFlags::X) != 0;
    constexpr int CH = V * (int)sizeof(T) / 16;   // 16-byte copies per gathered segment
    static_assert(CH >= 1 && V * (int)sizeof(T) == 16 * CH, "segments must be whole 16-byte words");
    T *sm = reinterpret_cast<T *>(smem_raw);
    const int gs = d.dg + 1;
    for (int i = threadIdx.x; i < d.dg * d.dg; i += blockDim.x) sm[(i / d.dg) * gs + (i % d.dg)] = d.grain[i];
    T *dtab = sm + d.dg * gs;
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) {
        const int c = i >> 8, byte = i & 255;
        T acc = T(0);
        for (int t = 0; t < 8; ++t) {
            const int j = 8 * c + t;
            if (j < d.L_loc) acc += ((byte >> t) & 1) ? d.hhalf[j] : -d.hhalf[j];
        }
        dtab[i] = acc;
    }
    __syncthreads();
    pdl_wait();
    uint4 *slots = reinterpret_cast<uint4 *>(smem_raw + qsun_async_slot_offset<T>());
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t G = (uint32_t)a.G;
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < a.items; it += stride) {
        const uint32_t row = (G == 1u) ? it : it / G;
        const int c0 = (G == 1u) ? 0 : (int)(it - row * G) * V;
        const size_t off = (size_t)row * a.s + c0;
        const T *qc = a.q + c0;
        for (int k = 0; k < d.L_loc; ++k) {
            const T *src = qc + (size_t)(row ^ d.fmask[k]) * a.s;
#pragma unroll
            for (int c = 0; c < CH; ++c) cp_async16(&slots[(k * CH + c) * kThreads + threadIdx.x], src + c * (16 / sizeof(T)));
        }
        const uint32_t g = row & ((uint32_t)d.dg - 1u);
        const uint32_t base = row - g;
        for (int h = 0; h < d.dg; ++h) {
            const T *src = qc + (size_t)(base + h) * a.s;
#pragma unroll
            for (int c = 0; c < CH; ++c)
                cp_async16(&slots[((d.L_loc + h) * CH + c) * kThreads + threadIdx.x], src + c * (16 / sizeof(T)));
        }
        // the row's own operands travel while the copies are in flight
        Pack<T, V> xo, qo, po, res;
#pragma unroll
        for (int v = 0; v < V; ++v) xo.v[v] = po.v[v] = T(0);
        if constexpr (HASX) xo = ldp<T, V>(a.x + off);
        qo = ldp<T, V>(a.q + off);
        if constexpr (HASP) po = ldp<T, V>(a.p + off);
        const uint32_t outer = row >> d.L_grain;
        T diag = dtab[outer & 0xffu];
        if (d.L_loc > 8) diag += dtab[256 + ((outer >> 8) & 0xffu)];
        if (d.L_loc > 16) diag += dtab[512 + ((outer >> 16) & 0xffu)];
        if (d.L_loc > 24) diag += dtab[768 + ((outer >> 24) & 0xffu)];
        cp_async_wait_all();
        T acc[V];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = T(0);
        for (int k = 0; k < d.L_loc; ++k) {
            Pack<T, V> gv;
#pragma unroll
            for (int c = 0; c < CH; ++c)
                reinterpret_cast<uint4 *>(&gv)[c] = slots[(k * CH + c) * kThreads + threadIdx.x];
            const T cf = d.cflip[k];
#pragma unroll
            for (int v = 0; v < V; ++v) acc[v] = fma_t(cf, gv.v[v], acc[v]);
        }
        const T *grow = sm + g * gs;
        for (int h = 0; h < d.dg; ++h) {
            Pack<T, V> gv;
#pragma unroll
            for (int c = 0; c < CH; ++c)
                reinterpret_cast<uint4 *>(&gv)[c] = slots[((d.L_loc + h) * CH + c) * kThreads + threadIdx.x];
            const T w = grow[h];
#pragma unroll
            for (int v = 0; v < V; ++v) acc[v] = fma_t(w, gv.v[v], acc[v]);
        }
#pragma unroll
        for (int v = 0; v < V; ++v)
            res.v[v] = step_combine<T>(HASX, true, HASP, a.cx, xo.v[v], a.alpha, acc[v], diag, qo.v[v], a.inva, a.boa,
                                       a.beta, po.v[v]);
        stp<T, V>(a.out + off, res);
    }
}

// ------------------------------------------------------- tiled QSun step
// A flip of outer spin j changes state bits L_grain + j and nbr[j] < L_grain,
// so in an aligned tile of 2^t consecutive states the flips j < t - L_grain
// and the whole grain block (the low L_grain bits) stay inside the tile.  A
// CTA of kThreads threads owns one tile of R = IPT * kThreads / G rows (every
// column: one contiguous run of the row-interleaved block), stages it in
// shared memory from its threads' own-row loads, and serves the in-tile flips
// and the grain block from there; only the L_loc - (t - L_grain) out-of-tile
// flips gather from L2, the first batch of them in flight while the in-tile
// flips are summed.  The model tables come ready-made from the operator
// (k_qsun_tables), so a CTA's set-up is one coalesced copy and a grid of one
// CTA per tile balances itself.  Each row is summed in qsun_row's order (flips
// j = 0..L_loc-1, then the grain row) with the same rounded operations, so
// results equal every other variant's.
template <typename T>
__host__ __device__ inline int qsun_tile_offset() {
    return (QSunSmem<T>::bytes(PF_MAX_GRAIN) + 63) / 64 * 64;
}

template <typename T>
__global__ void k_qsun_tables(const QSunDesc<T> d, T *__restrict__ out) {
    const int gs = d.dg + 1;
    for (int i = threadIdx.x; i < d.dg * gs; i += blockDim.x) {
        const int g = i / gs, h = i - g * gs;
        out[i] = h < d.dg ? d.grain[g * d.dg + h] : T(0);
    }
    T *dtab = out + d.dg * gs;
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

template <typename T, int V, int FLAGS, int IPT>
__global__ void __launch_bounds__(kThreads, 2)
    k_step_qsun_tile(const QSunDesc<T> d, const StepArgs<T> a, const T *__restrict__ tabs, int tbits) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_trigger();
    constexpr bool HASP = (FLAGS & StepFlags::P) != 0;
    constexpr bool HASX = (FLAGS & StepFlags::X) != 0;
    constexpr int U = 4;
    T *sm = reinterpret_cast<T *>(smem_raw);
    const int gs = d.dg + 1;
    const int ntab = d.dg * gs + 4 * 256;
    for (int i = threadIdx.x; i < ntab; i += blockDim.x) sm[i] = __ldg(tabs + i);
    pdl_wait();
    const T *dtab = sm + d.dg * gs;
    Pack<T, V> *tile = reinterpret_cast<Pack<T, V> *>(smem_raw + qsun_tile_offset<T>());
    const uint32_t G = (uint32_t)a.G;   // a power of two dividing kThreads
    const uint32_t gi = threadIdx.x & (G - 1u);
    const int c0 = (int)gi * V;
    const uint32_t rl0 = threadIdx.x / G, rstep = kThreads / G;
    const int n_in = min(d.L_loc, max(0, tbits - d.L_grain));
    const uint32_t ntiles = a.D >> tbits;
    const T *qc = a.q + c0;
    for (uint32_t tl = blockIdx.x; tl < ntiles; tl += gridDim.x) {
        const uint32_t r0 = tl << tbits;
        __syncthreads();   // the tables are staged / the previous tile is consumed
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const uint32_t rl = rl0 + (uint32_t)k * rstep;
            tile[rl * G + gi] = ldp<T, V>(qc + (size_t)(r0 + rl) * a.s);
        }
        __syncthreads();
#pragma unroll 1
        for (int k = 0; k < IPT; ++k) {
            const uint32_t rl = rl0 + (uint32_t)k * rstep, row = r0 + rl;
            const size_t off = (size_t)row * a.s + c0;
            if constexpr (HASX) prefetch_l1(a.x + off);
            if constexpr (HASP) prefetch_l1(a.p + off);
            Pack<T, V> g[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (n_in + u < d.L_loc) g[u] = ldp<T, V>(qc + (size_t)(row ^ d.fmask[n_in + u]) * a.s);
            T acc[V];
#pragma unroll
            for (int v = 0; v < V; ++v) acc[v] = T(0);
            for (int j = 0; j < n_in; ++j) {
                const Pack<T, V> t = tile[(rl ^ d.fmask[j]) * G + gi];
                const T cf = d.cflip[j];
#pragma unroll
                for (int v = 0; v < V; ++v) acc[v] = fma_t(cf, t.v[v], acc[v]);
            }
            for (int j0 = n_in; j0 < d.L_loc; j0 += U) {
                if (j0 != n_in) {
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        if (j0 + u < d.L_loc) g[u] = ldp<T, V>(qc + (size_t)(row ^ d.fmask[j0 + u]) * a.s);
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (j0 + u < d.L_loc) {
                        const T cf = d.cflip[j0 + u];
#pragma unroll
                        for (int v = 0; v < V; ++v) acc[v] = fma_t(cf, g[u].v[v], acc[v]);
                    }
            }
            const uint32_t gr = rl & ((uint32_t)d.dg - 1u);
            const uint32_t gbase = rl - gr;
            const T *grow = sm + gr * gs;
            for (int h = 0; h < d.dg; ++h) {
                const Pack<T, V> xg = tile[(gbase + h) * G + gi];
                const T w = grow[h];
#pragma unroll
                for (int v = 0; v < V; ++v) acc[v] = fma_t(w, xg.v[v], acc[v]);
            }
            const uint32_t outer = row >> d.L_grain;
            T diag = dtab[outer & 0xffu];
            if (d.L_loc > 8) diag += dtab[256 + ((outer >> 8) & 0xffu)];
            if (d.L_loc > 16) diag += dtab[512 + ((outer >> 16) & 0xffu)];
            if (d.L_loc > 24) diag += dtab[768 + ((outer >> 24) & 0xffu)];
            Pack<T, V> xo, po, res;
            const Pack<T, V> qo = tile[rl * G + gi];
#pragma unroll
            for (int v = 0; v < V; ++v) xo.v[v] = po.v[v] = T(0);
            if constexpr (HASX) xo = ldp<T, V>(a.x + off);
            if constexpr (HASP) po = ldp<T, V>(a.p + off);
#pragma unroll
            for (int v = 0; v < V; ++v)
                res.v[v] = step_combine<T>(HASX, true, HASP, a.cx, xo.v[v], a.alpha, acc[v], diag, qo.v[v], a.inva,
                                           a.boa, a.beta, po.v[v]);
            stp<T, V>(a.out + off, res);
        }
    }
}

// Launches a step kernel on st, with programmatic dependent launch when the
// handle allows it (the kernels wait for their predecessor themselves).
template <typename... KArgs, typename... Args>
static void launch_step_kernel(pf_handle *h, void (*kern)(KArgs...), int grid, int smem, cudaStream_t st,
                               Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = h->overlap ? 1 : 0;
    PF_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
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

// Set by the autotuner: variants whose registers spill to local memory are
// refused (PF_ERR_UNSUPPORTED) instead of timed.
thread_local bool t_refuse_spilling = false;

static bool spills(const void *kern) {
    thread_local std::map<const void *, bool> cache;
    auto it = cache.find(kern);
    if (it != cache.end()) return it->second;
    cudaFuncAttributes attr;
    PF_CUDA(cudaFuncGetAttributes(&attr, kern));
    return cache[kern] = attr.localSizeBytes > 0;
}

template <typename T, int V, class Desc, int FLAGS, int UB = 0, int MB = 0, int RK = 0>
static void launch_one(pf_op *op, cudaStream_t st, const Desc &d, StepArgs<T> a, int smem) {
    auto kern = k_step<T, V, Desc, FLAGS, UB, MB, RK>;
    if (t_refuse_spilling && spills((const void *)kern))
        throw Error(PF_ERR_UNSUPPORTED, "step-kernel variant spills registers");
    if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    // one item per thread when the whole block fits on the device at once,
    // otherwise a persistent grid of every resident CTA
    const int grid = grid_for(op->h, a.items, kThreads, blocks_per_sm((const void *)kern, smem));
    if constexpr ((FLAGS & StepFlags::DOTS) != 0) {
        ensure_reduction(op->h, (size_t)grid * 2 * a.s);
        a.partials = op->h->red_partials;
        a.counter = op->h->red_counter;
    }
    launch_step_kernel(op->h, kern, grid, smem, st, d, a);
    PF_CUDA(cudaGetLastError());
    count_launches(1);
}

// The tuned (gather batch, register cap) profiles apply to the filter's
// steps (Q|P|X and Q|X); every other launch uses the defaults.
template <typename T, int V, class Desc, int UB, int MB, int RK = 0>
static bool dispatch_profile(pf_op *op, cudaStream_t st, const Desc &d, const StepArgs<T> &a, int flags, int smem) {
    using F = StepFlags;
    if (flags == (F::Q | F::P | F::X)) launch_one<T, V, Desc, F::Q | F::P | F::X, UB, MB, RK>(op, st, d, a, smem);
    else if (flags == (F::Q | F::X)) launch_one<T, V, Desc, F::Q | F::X, UB, MB, RK>(op, st, d, a, smem);
    else return false;
    return true;
}

template <typename T, int V, class Desc>
static void dispatch_flags(pf_op *op, cudaStream_t st, const Desc &d, const StepArgs<T> &a,
                           int flags, int smem, int profile) {
    using F = StepFlags;
    if (profile != 0) {
        // gather batch U = 4 or 8 at 2, 3 or 4 resident CTAs per SM
        bool done = false;
        switch (profile) {
            case 1: done = dispatch_profile<T, V, Desc, 8, 2>(op, st, d, a, flags, smem); break;
            case 2: done = dispatch_profile<T, V, Desc, 8, 3>(op, st, d, a, flags, smem); break;
            case 3: done = dispatch_profile<T, V, Desc, 4, 4>(op, st, d, a, flags, smem); break;
            case 4: done = dispatch_profile<T, V, Desc, 8, 4>(op, st, d, a, flags, smem); break;
            default: throw Error(PF_ERR_INVALID, "unknown step-kernel profile");
        }
        if (done) return;
    }
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

// Shared memory of the asynchronous-gather step: the model tables plus
// (L_loc + dg) segments of V columns per thread.
template <typename T>
static int qsun_async_smem(const QSunDesc<T> &d, int V) {
    return qsun_async_slot_offset<T>() + (d.L_loc + d.dg) * V * (int)sizeof(T) * kThreads;
}

bool qsun_async_eligible(const pf_op *op, int s, int V, int elem) {
    if (op->kind != OP_QSUN || s % V != 0) return false;
    const int seg = V * elem;
    if (seg != 16 && seg != 32) return false;
    const int smem = elem == 8 ? qsun_async_smem(op->qsun64, V) : qsun_async_smem(op->qsun32, V);
    return smem <= 227 * 1024;
}

template <typename T, int V, int FLAGS>
static void launch_qsun_async_one(pf_op *op, cudaStream_t st, const QSunDesc<T> &d, const StepArgs<T> &a) {
    auto kern = k_step_qsun_async<T, V, FLAGS>;
    const int smem = qsun_async_smem(d, V);
    PF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int grid = grid_for(op->h, a.items, kThreads, blocks_per_sm((const void *)kern, smem));
    launch_step_kernel(op->h, kern, grid, smem, st, d, a);
    PF_CUDA(cudaGetLastError());
    count_launches(1);
}

// The asynchronous-gather variant serves the filter's Q|P|X and Q|X steps of a
// Quantum Sun operator with 16- or 32-byte column segments; false: not offered
// (the caller launches the per-thread kernel instead).
template <typename T, int V>
static bool launch_qsun_async(pf_op *op, cudaStream_t st, const QSunDesc<T> &d, const StepArgs<T> &a, int flags) {
    using F = StepFlags;
    constexpr int seg = V * (int)sizeof(T);
    if constexpr (seg == 16 || seg == 32) {
        if (qsun_async_smem(d, V) > 227 * 1024) return false;
        if (flags == (F::Q | F::P | F::X)) launch_qsun_async_one<T, V, F::Q | F::P | F::X>(op, st, d, a);
        else if (flags == (F::Q | F::X)) launch_qsun_async_one<T, V, F::Q | F::X>(op, st, d, a);
        else return false;
        return true;
    } else {
        (void)op, (void)st, (void)d, (void)a, (void)flags;
        return false;
    }
}

// Rows per tile of the tiled QSun step: R = ipt * kThreads / G for G = s / V
// column groups (a power of two dividing kThreads).  Returns log2(R), or 0
// when the operator has no such tile: fewer states than R, a tile smaller
// than the grain block, or more than 64 KB of tile.
static int qsun_tile_bits(const pf_op *op, int s, int V, int elem, int ipt) {
    if (op->kind != OP_QSUN || ipt < 1 || V < 1 || s % V != 0 || V * elem > 64) return 0;
    const int G = s / V;
    if ((G & (G - 1)) != 0 || G > kThreads) return 0;
    const int64_t R = (int64_t)ipt * kThreads / G;
    int t = 0;
    while (((int64_t)1 << t) < R) ++t;
    if (t > op->L || t < op->L_grain || R * s * elem > 64 * 1024) return 0;
    return t;
}

int qsun_tile_ipt(int profile) {
    return profile == kProfileTile ? 1 : profile == kProfileTile2 ? 2 : profile == kProfileTile4 ? 4 : 0;
}

bool qsun_tile_eligible(const pf_op *op, int s, int V, int elem, int profile) {
    const int ipt = qsun_tile_ipt(profile);
    return ipt > 0 && op->d_qtab64 != nullptr && qsun_tile_bits(op, s, V, elem, ipt) > 0;
}

void build_qsun_tables(pf_op *op) {
    if (op->kind != OP_QSUN) return;
    const int n = op->qsun64.dg * (op->qsun64.dg + 1) + 4 * 256;
    PF_CUDA(cudaMalloc(&op->d_qtab64, n * sizeof(double)));
    PF_CUDA(cudaMalloc(&op->d_qtab32, n * sizeof(float)));
    cudaStream_t st = op->h->stream;
    k_qsun_tables<double><<<1, 256, 0, st>>>(op->qsun64, static_cast<double *>(op->d_qtab64));
    k_qsun_tables<float><<<1, 256, 0, st>>>(op->qsun32, static_cast<float *>(op->d_qtab32));
    PF_CUDA(cudaGetLastError());
    count_launches(2);
    PF_CUDA(cudaStreamSynchronize(st));
}

template <typename T>
static const T *qsun_tabs(const pf_op *op);
template <>
const double *qsun_tabs<double>(const pf_op *op) { return static_cast<const double *>(op->d_qtab64); }
template <>
const float *qsun_tabs<float>(const pf_op *op) { return static_cast<const float *>(op->d_qtab32); }

template <typename T, int V, int FLAGS, int IPT>
static void launch_qsun_tile_one(pf_op *op, cudaStream_t st, const QSunDesc<T> &d, const StepArgs<T> &a, int tbits) {
    auto kern = k_step_qsun_tile<T, V, FLAGS, IPT>;
    if (t_refuse_spilling && spills((const void *)kern))
        throw Error(PF_ERR_UNSUPPORTED, "step-kernel variant spills registers");
    const int smem = qsun_tile_offset<T>() + (int)(((int64_t)1 << tbits) * a.s * (int64_t)sizeof(T));
    if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    // one CTA per tile (the scheduler balances them) up to 8 waves, then a
    // persistent loop over the tiles
    const int64_t ntiles = (int64_t)a.D >> tbits;
    const int64_t cap = (int64_t)op->h->num_sms * blocks_per_sm((const void *)kern, smem) * 8;
    const int grid = (int)std::max<int64_t>(1, std::min(ntiles, cap));
    launch_step_kernel(op->h, kern, grid, smem, st, d, a, qsun_tabs<T>(op), tbits);
    PF_CUDA(cudaGetLastError());
    count_launches(1);
}

template <typename T, int V, int IPT>
static bool launch_qsun_tile_flags(pf_op *op, cudaStream_t st, const QSunDesc<T> &d, const StepArgs<T> &a, int flags,
                                   int tbits) {
    using F = StepFlags;
    if (flags == (F::Q | F::P | F::X)) launch_qsun_tile_one<T, V, F::Q | F::P | F::X, IPT>(op, st, d, a, tbits);
    else if (flags == (F::Q | F::X)) launch_qsun_tile_one<T, V, F::Q | F::X, IPT>(op, st, d, a, tbits);
    else return false;
    return true;
}

// The tiled variant serves the filter's Q|P|X and Q|X steps of a Quantum Sun
// operator on contiguous rows; false: not offered (the caller launches the
// per-thread kernel instead).
template <typename T, int V>
static bool launch_qsun_tile(pf_op *op, cudaStream_t st, const QSunDesc<T> &d, const StepArgs<T> &a, int flags,
                             int profile) {
    const int ipt = qsun_tile_ipt(profile);
    const int tbits = qsun_tile_bits(op, a.s, V, (int)sizeof(T), ipt);
    if (tbits == 0 || qsun_tabs<T>(op) == nullptr) return false;
    switch (ipt) {
        case 1: return launch_qsun_tile_flags<T, V, 1>(op, st, d, a, flags, tbits);
        case 2: return launch_qsun_tile_flags<T, V, 2>(op, st, d, a, flags, tbits);
        case 4: return launch_qsun_tile_flags<T, V, 4>(op, st, d, a, flags, tbits);
        default: return false;
    }
}

template <typename T, int V>
static void dispatch_op(pf_op *op, cudaStream_t st, const StepArgs<T> &a, int flags, int profile) {
    int smem = 0;
    const int lanes = a.G < 32 ? a.G : 32;
    const int dots_smem = (kThreads / 32) * lanes * 2 * V * 8 + 2 * a.s * 8;
    if (op->kind == OP_CHAIN) {
        const ChainDesc<T> &d = chain_of<T>(op);
        if ((flags & StepFlags::Q) && !d.full) smem = rank_table_entries(d.nchunks) * 4;
        if (flags & StepFlags::DOTS) smem = std::max(smem, dots_smem);
        if (profile == kProfileLocalRank && !d.full &&
            dispatch_profile<T, V, ChainDesc<T>, 0, 0, 1>(op, st, d, a, flags, smem + 33 * 33 * 4))
            return;
        dispatch_flags<T, V>(op, st, d, a, flags, smem, profile >= kProfileAsync ? 0 : profile);
    } else if (op->kind == OP_QSUN) {
        const QSunDesc<T> &d = qsun_of<T>(op);
        if (profile == kProfileAsync && a.ld == a.s && launch_qsun_async<T, V>(op, st, d, a, flags)) return;
        if (qsun_tile_ipt(profile) > 0 && a.ld == a.s && launch_qsun_tile<T, V>(op, st, d, a, flags, profile)) return;
        smem = QSunSmem<T>::bytes(d.dg);
        if (flags & StepFlags::DOTS) smem = std::max(smem, dots_smem);
        dispatch_flags<T, V>(op, st, d, a, flags, smem, profile >= kProfileAsync ? 0 : profile);
    } else {
        const CsrDesc<T> &d = csr_of<T>(op);
        if (flags & StepFlags::DOTS) smem = dots_smem;
        dispatch_flags<T, V>(op, st, d, a, flags, smem, profile >= kProfileAsync ? 0 : profile);
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
    launch_step_kernel(op->h, kern, grid, smem, st, d, a);
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
                       int code, int ld, int stream) {
    const int V = variant_width(code), profile = variant_profile(code);
    PF_CHECK(profile >= 0 && profile <= kStepProfiles, PF_ERR_INVALID, "unknown step-kernel profile");
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
    a.ld = ld > 0 ? ld : s;
    a.stream = stream ? 1 : 0;
    PF_CHECK(a.ld >= s, PF_ERR_INVALID, "row stride smaller than the column count");
    PF_CHECK(!coop || a.ld == s, PF_ERR_INVALID, "the warp-cooperative step needs contiguous rows");
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
        case 1: dispatch_op<T, 1>(op, st, a, flags, profile); break;
        case 2: dispatch_op<T, 2>(op, st, a, flags, profile); break;
        case 4: dispatch_op<T, 4>(op, st, a, flags, profile); break;
        case 8: dispatch_op<T, 8>(op, st, a, flags, profile); break;
        case 16:
            if constexpr (sizeof(T) == 4) { dispatch_op<T, 16>(op, st, a, flags, profile); break; }
            [[fallthrough]];
        default: throw Error(PF_ERR_INVALID, "bad vector width");
    }
}

template <typename T>
void launch_step(pf_op *op, cudaStream_t st, int64_t D, int s, const T *q, const T *p,
                 const T *x, T *out, double cx, double alpha, double beta, double inva,
                 double shift, int flags, double *dots, int ld, int stream) {
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
    const bool slab = ld > 0 && ld != s;
    if (V == kCoopWidth && (slab || !coop_eligible(op, s, flags))) V = default_width(s, (int)sizeof(T));
    if (variant_profile(V) != 0 && (flags & StepFlags::DOTS)) V = variant_width(V);
    launch_step_width<T>(op, st, D, s, q, p, x, out, cx, alpha, beta, inva, shift, flags, dots, V, ld, stream);
}

template void launch_step_width<double>(pf_op *, cudaStream_t, int64_t, int, const double *, const double *,
                                        const double *, double *, double, double, double, double, double, int,
                                        double *, int, int, int);
template void launch_step_width<float>(pf_op *, cudaStream_t, int64_t, int, const float *, const float *,
                                       const float *, float *, double, double, double, double, double, int,
                                       double *, int, int, int);
template void launch_step<double>(pf_op *, cudaStream_t, int64_t, int, const double *, const double *,
                                  const double *, double *, double, double, double, double, double,
                                  int, double *, int, int);
template void launch_step<float>(pf_op *, cudaStream_t, int64_t, int, const float *, const float *,
                                 const float *, float *, double, double, double, double, double,
                                 int, double *, int, int);

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
