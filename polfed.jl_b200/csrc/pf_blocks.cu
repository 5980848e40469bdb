// pf_blocks.cu -- the s-column block algebra of a Lanczos iteration in fused
// passes over the block (BlockLanczosFactorization.jl:102-131,
// orthogonalization.jl:31-33).
//
// A Lanczos iteration on an RI block (D rows of s contiguous values) needs a
// CholQR2 (two Gram products W^T W, two Cholesky factors, two right solves
// W <- W R^{-1}), the copy of the new block into the Krylov basis, the
// overlap alpha = V^T W and the three-term update r -= V alpha + V_prev
// beta^T.  As library calls that is about a dozen launches and copies of a
// few microseconds each, every one re-reading the block.  Here each pass over
// the block is one launch:
//
//   pass 1   Gram W^T W                       -> last CTA: R1 = chol, Rtot = R1
//   pass 2   W <- W R1^{-1}, Gram of the result -> last CTA: R2 = chol,
//            Rtot = R2 R1 (= beta), beta written into T
//   pass 3   W <- W R2^{-1}, also written into the basis at column k
//   overlap  Gram V^T W (upper triangle)      -> last CTA: alpha into T
//   update   r -= V alpha + V_prev beta^T
//
// Every CTA stages tiles of rows in shared memory (a tile is contiguous in
// the RI layout, so the loads are coalesced).  A CTA's Gram partial is the
// sum over its tiles, in order, of per-entry sums over a fixed split of the
// tile's rows; the last CTA of each group of 32 to finish (a counter per
// group) adds the group's partials in CTA order, and the last group to finish
// adds the group sums in group order and runs the epilogue.  The grid size
// depends only on D and s, and every product and sum is rounded on its own
// (fused multiply-adds where written), so a pass gives the same bits in every
// run and in both QR paths:
// the host-QR path runs the same Gram and solve passes and only moves the
// Cholesky to the host (host_cholesky's arithmetic, which the epilogue
// repeats operation for operation).
#include "pf_internal.h"
#include "pf_solver.h"

#include <algorithm>

namespace pf {

namespace {

constexpr int kBlkThreads = 256;
constexpr int kBlkPhases = 16;   // at most this many row phases per Gram entry in a tile
constexpr int kBlkRuns = 32;     // at most this many strided runs per entry over the CTA partials
constexpr int kBlkGroup = 32;    // CTAs whose partials the last of them adds into a group partial
constexpr int kBlkMaxGrid = 592;   // CTAs of a pass at most (4 per SM)
constexpr int kBlkMaxGroups = 63;

// row phases of a tile per Gram entry, and strided runs over the CTA
// partials per entry, for E = s (s + 1) / 2 entries
__host__ __device__ inline int blk_phases(int E) {
    const int p = E >= kBlkThreads ? 1 : kBlkThreads / E;
    return p < kBlkPhases ? p : kBlkPhases;
}
__host__ __device__ inline int blk_runs(int E) {
    const int q = E >= kBlkThreads ? 1 : kBlkThreads / E;
    return q < kBlkRuns ? q : kBlkRuns;
}

__host__ __device__ inline int blk_rows(int s) { return s <= 16 ? 128 : 64; }
__host__ __device__ inline int blk_pitch(int s) { return s | 1; }   // odd: no bank conflicts

// entry e of the upper triangle (i <= j), column by column
__device__ inline void upper_entry(int e, int s, int *i, int *j) {
    int jj = 0, base = 0;
    while (base + jj + 1 <= e) {
        base += jj + 1;
        ++jj;
    }
    (void)s;
    *j = jj;
    *i = e - base;
}

// out[e] = sum over rows b < n of src[b * E + e], in row order, by the calling
// CTA: Q strided runs per entry (eight loads in flight each, added in row
// order), then the runs added in run order.  runs: Q x E shared doubles.
__device__ void cta_sum_rows(const double *src, int n, int E, int Q, double *runs, double *out) {
    const int t = threadIdx.x;
    for (int w = t; w < Q * E; w += blockDim.x) {
        const int e = w % E, q = w / E;
        double v = 0.0;
        int b = q;
        for (; b + 7 * Q < n; b += 8 * Q) {
            double x[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) x[u] = __ldcg(src + (size_t)(b + u * Q) * E + e);
#pragma unroll
            for (int u = 0; u < 8; ++u) v = __dadd_rn(v, x[u]);
        }
        for (; b < n; b += Q) v = __dadd_rn(v, __ldcg(src + (size_t)b * E + e));
        runs[q * E + e] = v;
    }
    __syncthreads();
    for (int e = t; e < E; e += blockDim.x) {
        double v = 0.0;
        for (int q = 0; q < Q; ++q) v = __dadd_rn(v, runs[q * E + e]);
        out[e] = v;
    }
    __syncthreads();
}

}  // namespace

// host_cholesky's operations in its order, each rounded on its own, by the
// calling CTA: g (shared, s x s column-major, upper triangle read) = r^T r
// with r upper (shared).  A pivot host_cholesky rejects sets *bad (shared)
// and r = I.
__device__ void cta_cholesky(const double *g, double *r, int s, int *bad) {
    const int n = s * s;
    for (int i = threadIdx.x; i < n; i += blockDim.x) r[i] = 0.0;
    if (threadIdx.x == 0) *bad = 0;
    __syncthreads();
    for (int j = 0; j < s; ++j) {
        if (threadIdx.x == 0) {
            const double gjj = g[j + j * s];
            double d = gjj;
            for (int k = 0; k < j; ++k) d = __dsub_rn(d, __dmul_rn(r[k + j * s], r[k + j * s]));
            if (!(d > 1e-28 * fmax(1.0, fabs(gjj))) || !isfinite(d) || d <= 1e-13 * fabs(gjj)) *bad = 1;
            else r[j + j * s] = sqrt(d);
        }
        __syncthreads();
        if (*bad) break;
        const double rjj = r[j + j * s];
        for (int i = j + 1 + threadIdx.x; i < s; i += blockDim.x) {
            double v = g[j + i * s];
            for (int k = 0; k < j; ++k) v = __dsub_rn(v, __dmul_rn(r[k + j * s], r[k + i * s]));
            r[j + i * s] = __ddiv_rn(v, rjj);
        }
        __syncthreads();
    }
    if (*bad) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) r[i] = (i % (s + 1) == 0) ? 1.0 : 0.0;
        __syncthreads();
    }
}

// rtot_out = r * rtot_in (rtot_in null: the identity) with the host's
// product loop; both upper triangular.
__device__ void cta_compose(const double *r, int s, const double *rtot_in, double *rtot_out) {
    for (int idx = threadIdx.x; idx < s * s; idx += blockDim.x) {
        const int i = idx % s, j = idx / s;
        double v = 0.0;
        for (int k = i; k <= j; ++k) {
            const double t = rtot_in ? rtot_in[k + j * s] : (k == j ? 1.0 : 0.0);
            v = __dadd_rn(v, __dmul_rn(r[i + k * s], t));
        }
        rtot_out[idx] = v;
    }
}

// One CholQR pass on the device for blocks wider than the fused passes take:
// the Gram matrix from global memory, R and the running product out.
__global__ void k_small_chol(const double *__restrict__ G, int s, double *__restrict__ R,
                             const double *__restrict__ rtot_in, double *__restrict__ rtot_out, int *flag) {
    extern __shared__ double sh[];
    double *g = sh, *r = sh + s * s;
    __shared__ int bad;
    for (int i = threadIdx.x; i < s * s; i += blockDim.x) g[i] = G[i];
    __syncthreads();
    cta_cholesky(g, r, s, &bad);
    if (bad && threadIdx.x == 0) *flag = 1;
    for (int i = threadIdx.x; i < s * s; i += blockDim.x) R[i] = r[i];
    cta_compose(r, s, rtot_in, rtot_out);
}

// One fused pass (see the file comment).  Shared memory: the X tile, the Y
// tile (overlap only), R of the solve, the per-phase sums.
__global__ void __launch_bounds__(kBlkThreads) k_blk_pass(const BlkPass p) {
    extern __shared__ __align__(16) double smem[];
    const int s = p.s, rows = blk_rows(s), pitch = blk_pitch(s);
    const bool solve = (p.flags & BLK_SOLVE) != 0, gram = (p.flags & BLK_GRAM) != 0;
    const bool append = (p.flags & BLK_APPEND) != 0;
    const bool two = p.Y != nullptr;
    double *xt = smem;
    double *yt = xt + rows * pitch;
    double *rs = yt + (two ? rows * pitch : 0);
    double *red = rs + s * s;   // kBlkThreads
    const int E = s * (s + 1) / 2;
    const int P = blk_phases(E);   // row phases of a tile
    const int t = threadIdx.x;
    if (solve)
        for (int i = t; i < s * s; i += kBlkThreads) rs[i] = p.Rs[i];
    // this thread's Gram entries (up to 3 when E > kBlkThreads)
    double acc[3] = {0.0, 0.0, 0.0};
    int ei[3], ej[3], ne = 0, phase = 0;
    if (gram) {
        if (P > 1) {
            if (t < P * E) {
                upper_entry(t % E, s, &ei[0], &ej[0]);
                phase = t / E;
                ne = 1;
            }
        } else {
            for (int e = t; e < E && ne < 3; e += kBlkThreads) {
                upper_entry(e, s, &ei[ne], &ej[ne]);
                ++ne;
            }
        }
    }
    const int64_t ntiles = (p.D + rows - 1) / rows;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t r0 = tile * rows;
        const int n = p.D - r0 < rows ? (int)(p.D - r0) : rows;
        const int nv = n * s;
        const double *src = p.W + r0 * s;
        __syncthreads();   // the previous tile is consumed
        for (int idx = t; idx < nv; idx += kBlkThreads) {
            const int rr = idx / s, c = idx - rr * s;
            xt[rr * pitch + c] = __ldcg(src + idx);
        }
        if (two) {
            const double *ys = p.Y + r0 * s;
            for (int idx = t; idx < nv; idx += kBlkThreads) {
                const int rr = idx / s, c = idx - rr * s;
                yt[rr * pitch + c] = __ldcg(ys + idx);
            }
        }
        __syncthreads();
        if (solve) {
            // x R = w, R upper: x_j = (w_j - sum_{i<j} x_i R_ij) / R_jj
            for (int rr = t; rr < n; rr += kBlkThreads) {
                double *x = xt + rr * pitch;
                for (int j = 0; j < s; ++j) {
                    double v = x[j];
                    for (int i = 0; i < j; ++i) v = __dsub_rn(v, __dmul_rn(x[i], rs[i + j * s]));
                    x[j] = __ddiv_rn(v, rs[j + j * s]);
                }
            }
            __syncthreads();
            double *dst = p.W + r0 * s;
            for (int idx = t; idx < nv; idx += kBlkThreads) {
                const int rr = idx / s, c = idx - rr * s;
                dst[idx] = xt[rr * pitch + c];
            }
        }
        if (append) {
            for (int idx = t; idx < nv; idx += kBlkThreads) {
                const int rr = idx / s, c = idx - rr * s;
                p.basis[(r0 + rr) * p.ldb + p.col + c] = xt[rr * pitch + c];
            }
        }
        if (gram) {
            const double *yy = two ? yt : xt;
            for (int q = 0; q < ne; ++q) {
                const int i = ei[q], j = ej[q];
                double a = acc[q];
                for (int rr = (P > 1 ? phase : 0); rr < n; rr += P)
                    a = __fma_rn(xt[rr * pitch + i], yy[rr * pitch + j], a);
                acc[q] = a;
            }
        }
    }
    if (!gram) return;
    // the CTA's partial: the phases of each entry added in phase order
    __syncthreads();
    double *part = p.partial + (size_t)blockIdx.x * E;
    if (P > 1) {
        red[t] = ne ? acc[0] : 0.0;
        __syncthreads();
        for (int e = t; e < E; e += kBlkThreads) {
            double v = 0.0;
            for (int q = 0; q < P; ++q) v = __dadd_rn(v, red[q * E + e]);
            part[e] = v;
        }
    } else {
        for (int q = 0; q < ne; ++q) part[t + q * kBlkThreads] = acc[q];
    }
    // two levels: the last CTA of each group of kBlkGroup CTAs adds the
    // group's partials in CTA order; the last group to finish adds the group
    // sums in group order
    __shared__ bool last;
    __shared__ int bad;
    const int nb = gridDim.x;
    const int grp = blockIdx.x / kBlkGroup, g0 = grp * kBlkGroup;
    const int gn = nb - g0 < kBlkGroup ? nb - g0 : kBlkGroup;
    const int ngrp = (nb + kBlkGroup - 1) / kBlkGroup;
    double *gpart = p.partial + (size_t)nb * E;   // ngrp x E
    const int Q = blk_runs(E);
    double *g = smem;                 // s x s, reusing the tiles
    double *r = g + s * s;            // s x s
    double *rt = r + s * s;           // s x s
    double *runs = rt + s * s;        // Q x E
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(p.counter + 1 + grp, 1u) == (unsigned)gn - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    cta_sum_rows(p.partial + (size_t)g0 * E, gn, E, Q, runs, gpart + (size_t)grp * E);
    if (t == 0) p.counter[1 + grp] = 0u;
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(p.counter, 1u) == (unsigned)ngrp - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    double *tot = runs + Q * E;       // E
    cta_sum_rows(gpart, ngrp, E, Q, runs, tot);
    for (int e = t; e < E; e += kBlkThreads) {
        int i, j;
        upper_entry(e, s, &i, &j);
        g[i + j * s] = tot[e];
        g[j + i * s] = tot[e];
    }
    __syncthreads();
    for (int i = t; i < s * s; i += kBlkThreads) p.G[i] = g[i];
    if (p.epi == EPI_ALPHA) {
        // alpha, symmetric from its upper triangle, as T's diagonal block at (k, k)
        for (int idx = t; idx < s * s; idx += kBlkThreads) {
            const int i = idx % s, j = idx / s;
            p.T[(size_t)(p.k + i) + (size_t)(p.k + j) * p.ldT] = g[idx];
            p.keep[idx] = g[idx];
        }
    } else if (p.epi == EPI_CHOL || p.epi == EPI_CHOL_BETA) {
        cta_cholesky(g, r, s, &bad);
        if (bad && t == 0) *p.flag = 1;
        for (int i = t; i < s * s; i += kBlkThreads) p.R[i] = r[i];
        cta_compose(r, s, p.rtot_in, rt);
        __syncthreads();
        for (int idx = t; idx < s * s; idx += kBlkThreads) {
            p.rtot_out[idx] = rt[idx];
            if (p.epi == EPI_CHOL_BETA) {
                // beta = Rtot as T's blocks at rows k, columns k - s and the transpose
                const int i = idx % s, j = idx / s;
                p.T[(size_t)(p.k + i) + (size_t)(p.k - s + j) * p.ldT] = rt[idx];
                p.T[(size_t)(p.k - s + j) + (size_t)(p.k + i) * p.ldT] = rt[idx];
                p.keep[idx] = rt[idx];
            }
        }
    }
    if (t == 0) *p.counter = 0u;
}

// r -= V alpha + V_prev beta^T row by row (V_prev null: no beta term); alpha
// symmetric, beta as kept by the CholQR epilogue.
__global__ void __launch_bounds__(kBlkThreads)
    k_blk_update(int64_t D, int s, double *__restrict__ r, const double *__restrict__ V,
                 const double *__restrict__ Vp, const double *__restrict__ alpha, const double *__restrict__ beta) {
    extern __shared__ __align__(16) double ab[];
    for (int i = threadIdx.x; i < s * s; i += blockDim.x) {
        ab[i] = alpha[i];
        if (Vp) ab[s * s + i] = beta[i];
    }
    __syncthreads();
    const int64_t n = D * s;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = idx / s;
        const int c = (int)(idx - row * s);
        const double *v = V + row * s;
        double a = 0.0;
        for (int i = 0; i < s; ++i) a = __fma_rn(ab[i + c * s], __ldg(v + i), a);
        double val = __dsub_rn(r[idx], a);
        if (Vp) {
            const double *vp = Vp + row * s;
            double b = 0.0;
            for (int i = 0; i < s; ++i) b = __fma_rn(ab[s * s + c + i * s], __ldg(vp + i), b);
            val = __dsub_rn(val, b);
        }
        r[idx] = val;
    }
}

// The same update with one row per thread for s in {1, 2, 4, 8, 16} (the
// row's values in registers, read once), with the element form's operations
// in its order, so both give the same bits.
template <int S>
__global__ void __launch_bounds__(kBlkThreads)
    k_blk_update_rows(int64_t D, double *__restrict__ r, const double *__restrict__ V,
                      const double *__restrict__ Vp, const double *__restrict__ alpha,
                      const double *__restrict__ beta) {
    __shared__ double ab[2 * S * S];
    for (int i = threadIdx.x; i < S * S; i += blockDim.x) {
        ab[i] = alpha[i];
        if (Vp) ab[S * S + i] = beta[i];
    }
    __syncthreads();
    for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < D;
         row += (int64_t)gridDim.x * blockDim.x) {
        double v[S], w[S], x[S];
#pragma unroll
        for (int c = 0; c < S; ++c) v[c] = __ldg(V + row * S + c);
        if (Vp) {
#pragma unroll
            for (int c = 0; c < S; ++c) w[c] = __ldg(Vp + row * S + c);
        }
#pragma unroll
        for (int c = 0; c < S; ++c) x[c] = r[row * S + c];
#pragma unroll
        for (int c = 0; c < S; ++c) {
            double a = 0.0;
#pragma unroll
            for (int i = 0; i < S; ++i) a = __fma_rn(ab[i + c * S], v[i], a);
            double val = __dsub_rn(x[c], a);
            if (Vp) {
                double bb = 0.0;
#pragma unroll
                for (int i = 0; i < S; ++i) bb = __fma_rn(ab[S * S + c + i * S], w[i], bb);
                val = __dsub_rn(val, bb);
            }
            r[row * S + c] = val;
        }
    }
}

int blk_grid(int64_t D, int s) {
    const int64_t tiles = (D + blk_rows(s) - 1) / blk_rows(s);
    return (int)std::min<int64_t>(tiles, kBlkMaxGrid);
}

int blk_counters() { return 1 + kBlkMaxGroups; }

size_t blk_partial_doubles(int64_t D, int s) {
    const int nb = blk_grid(D, s);
    return (size_t)(nb + (nb + kBlkGroup - 1) / kBlkGroup) * (size_t)(s * (s + 1) / 2);
}

static size_t blk_smem(int s, bool two) {
    const int rows = blk_rows(s), pitch = blk_pitch(s), E = s * (s + 1) / 2;
    const int Q = blk_runs(E);
    const size_t pass = (size_t)rows * pitch * (two ? 2 : 1) + (size_t)s * s + kBlkThreads;
    const size_t epi = 3 * (size_t)s * s + (size_t)Q * E + E;
    return std::max(pass, epi) * sizeof(double);
}

void blk_pass(cudaStream_t st, const BlkPass &p) {
    PF_CHECK(p.s >= 1 && p.s <= kBlkMaxS, PF_ERR_INVALID, "fused block pass needs 1 <= s <= 32");
    static_assert((kBlkMaxGrid + kBlkGroup - 1) / kBlkGroup <= kBlkMaxGroups, "group counters");
    const size_t smem = blk_smem(p.s, p.Y != nullptr);
    if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(k_blk_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_blk_pass<<<blk_grid(p.D, p.s), kBlkThreads, smem, st>>>(p);
    PF_CUDA(cudaGetLastError());
    count_launches(1);
}

void blk_update(cudaStream_t st, int64_t D, int s, double *r, const double *V, const double *Vp, const double *alpha,
                const double *beta) {
    const int rgrid = (int)std::min<int64_t>((D + kBlkThreads - 1) / kBlkThreads, 148 * 8);
    switch (s) {
        case 1: k_blk_update_rows<1><<<rgrid, kBlkThreads, 0, st>>>(D, r, V, Vp, alpha, beta); break;
        case 2: k_blk_update_rows<2><<<rgrid, kBlkThreads, 0, st>>>(D, r, V, Vp, alpha, beta); break;
        case 4: k_blk_update_rows<4><<<rgrid, kBlkThreads, 0, st>>>(D, r, V, Vp, alpha, beta); break;
        case 8: k_blk_update_rows<8><<<rgrid, kBlkThreads, 0, st>>>(D, r, V, Vp, alpha, beta); break;
        case 16: k_blk_update_rows<16><<<rgrid, kBlkThreads, 0, st>>>(D, r, V, Vp, alpha, beta); break;
        default: {
            const int64_t n = D * s;
            const int grid = (int)std::min<int64_t>((n + kBlkThreads - 1) / kBlkThreads, 148 * 8);
            k_blk_update<<<grid, kBlkThreads, 2 * (size_t)s * s * sizeof(double), st>>>(D, s, r, V, Vp, alpha, beta);
        }
    }
    PF_CUDA(cudaGetLastError());
    count_launches(1);
}

void small_chol(cudaStream_t st, const double *G, int s, double *R, const double *rtot_in, double *rtot_out,
                int *flag) {
    const int smem = (int)(2 * (size_t)s * s * sizeof(double));
    if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(k_small_chol, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_small_chol<<<1, 64, smem, st>>>(G, s, R, rtot_in, rtot_out, flag);
    PF_CUDA(cudaGetLastError());
    count_launches(1);
}

}  // namespace pf
