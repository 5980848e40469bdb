// pf_tc.cu -- the split-BF16 Gram product of the reorthogonalisation on the
// 5th-generation tensor cores (tcgen05, sm_100a).
//
// G = B^T r for the Krylov basis B (row-major D x nB, FP64) and the Lanczos
// block r (row-major D x s, FP64), the Gram contraction of a reorthogonalisation
// pass (reorthogonalization.jl:77-84).  Each FP64 value v is split into two
// BF16 numbers, hi = bf16(v) and lo = bf16(v - hi), and
//   B^T r ~= Bhi^T rhi + Bhi^T rlo + Blo^T rhi
// (three tensor-core products accumulated in FP32; the dropped lo*lo term and
// the BF16 roundings leave a relative error of ~1e-5 of |B| |r|).  That is the
// first pass of CGS2: the FP64 second pass removes what the first leaves.
//
// One CTA of 128 threads owns 128 basis columns (the MMA's M) and a chunk of
// rows (the contraction K, split over CTAs: chunks of at least 256 rows, about
// a thousand of them at large D, so that several CTAs share each SM).  Per stage of 64 rows the threads
// read the FP64 values (coalesced along the basis columns), split them and
// write the BF16 tiles to shared memory in the MMA's K-major core-matrix
// layout (8 rows x 16 bytes per core matrix, no swizzle); one elected thread
// issues 4 k-steps x 3 products of tcgen05.mma.cta_group::1.kind::f16
// (M = 128, N = s rounded up to 8, K = 16) into an FP32 accumulator in tensor
// memory and commits them to an mbarrier, which every thread waits on (with an
// iteration limit) before the tiles are overwritten.  At the end each warp
// reads its 32 accumulator lanes with tcgen05.ld and writes the CTA's FP32
// partial; a second kernel sums the partials of the row chunks in FP64.
#include "pf_internal.h"
#include "pf_solver.h"

#include <cuda_bf16.h>

namespace pf {

constexpr int kTcThreads = 128;
constexpr int kTcM = 128;        // basis columns per CTA (MMA M)
constexpr int kTcStage = 64;     // rows of D per stage (4 MMA k-steps of 16)
constexpr long kTcWaitLimit = 1L << 22;

// Shared memory: A hi / lo tiles (128 x 64 BF16 each), B hi / lo tiles
// (NT x 64 BF16 each), then the mbarrier and the tensor-memory address.
struct TcSmem {
    static constexpr int a_bytes = kTcM * kTcStage * 2;
    static __host__ __device__ int b_bytes(int nt) { return nt * kTcStage * 2; }
    static __host__ __device__ int total(int nt) { return 2 * a_bytes + 2 * b_bytes(nt) + 16; }
};

// Byte offset of element (row mn, k) in a K-major core-matrix tile with 64
// columns of K: core matrices of 8 rows x 8 BF16 (16 bytes per row) are
// adjacent along K (128 bytes apart, the descriptor's leading byte offset)
// and 8-row groups are 8 x 128 bytes apart (its stride byte offset).
__device__ __forceinline__ int core_offset(int mn, int k) {
    return (mn >> 3) * 1024 + (k >> 3) * 128 + (mn & 7) * 16 + (k & 7) * 2;
}

// Shared-memory matrix descriptor: start address, leading byte offset 128,
// stride byte offset 1024 (all in 16-byte units), descriptor version 1, no
// swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long it = 0; it < kTcWaitLimit; ++it) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <int NT>
__device__ __forceinline__ void tmem_load_row(uint32_t addr, float (&v)[NT]) {
    uint32_t r[NT];
    if constexpr (NT == 8) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                     : "r"(addr));
    } else if constexpr (NT == 16) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(addr));
    } else {
#pragma unroll
        for (int h = 0; h < NT / 16; ++h) {
            float w[16];
            tmem_load_row<16>(addr + 16 * h, w);
#pragma unroll
            for (int i = 0; i < 16; ++i) r[16 * h + i] = __float_as_uint(w[i]);
        }
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < NT; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void split_bf16(double v, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __double2bfloat16(v);
    lo = __double2bfloat16(v - (double)__bfloat162float(hi));
}

// part[(blockIdx.y * Mpad + m) * NT + n] = sum over this CTA's rows of the
// split-BF16 products; *err is set when an mbarrier wait gives up.
template <int NT>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_gram_bf16x3(const double *__restrict__ B, int ldb, int nB, const double *__restrict__ r, int s, uint32_t D,
                  uint32_t chunk, float *__restrict__ part, int Mpad, int *err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *a_hi = smem, *a_lo = smem + TcSmem::a_bytes;
    unsigned char *b_hi = smem + 2 * TcSmem::a_bytes, *b_lo = b_hi + TcSmem::b_bytes(NT);
    uint64_t *bar = reinterpret_cast<uint64_t *>(b_lo + TcSmem::b_bytes(NT));
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t bar_addr = smem_u32(bar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_addr) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;\n" ::"r"(smem_u32(tmem_slot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    // kind::f16 with BF16 A and B, FP32 accumulator, both K-major, M = 128, N = NT
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
    const int m0 = blockIdx.x * kTcM;
    const uint32_t k_beg = blockIdx.y * chunk;
    const uint32_t k_end = min(D, k_beg + chunk);
    uint32_t phase = 0;
    bool ok = true, any = false;
    for (uint32_t k = k_beg; k < k_end && ok; k += kTcStage) {
#pragma unroll 8
        for (int idx = tid; idx < kTcM * kTcStage; idx += kTcThreads) {
            const int m = idx % kTcM, kk = idx / kTcM;
            const uint32_t row = k + kk;
            const double v = (row < k_end && m0 + m < nB) ? B[(size_t)row * ldb + m0 + m] : 0.0;
            __nv_bfloat16 hi, lo;
            split_bf16(v, hi, lo);
            const int off = core_offset(m, kk);
            *reinterpret_cast<__nv_bfloat16 *>(a_hi + off) = hi;
            *reinterpret_cast<__nv_bfloat16 *>(a_lo + off) = lo;
        }
#pragma unroll 4
        for (int idx = tid; idx < NT * kTcStage; idx += kTcThreads) {
            const int n = idx % NT, kk = idx / NT;
            const uint32_t row = k + kk;
            const double v = (row < k_end && n < s) ? r[(size_t)row * s + n] : 0.0;
            __nv_bfloat16 hi, lo;
            split_bf16(v, hi, lo);
            const int off = core_offset(n, kk);
            *reinterpret_cast<__nv_bfloat16 *>(b_hi + off) = hi;
            *reinterpret_cast<__nv_bfloat16 *>(b_lo + off) = lo;
        }
        // the generic-proxy tile writes become visible to the tensor cores
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo), bh = smem_u32(b_hi), bl = smem_u32(b_lo);
#pragma unroll
            for (int j = 0; j < kTcStage / 16; ++j) {
                const uint32_t o = 256u * j;   // two 128-byte core matrices of K per k-step
                tc_mma(tmem, smem_desc(ah + o), smem_desc(bh + o), idesc, (any || j > 0) ? 1u : 0u);
                tc_mma(tmem, smem_desc(ah + o), smem_desc(bl + o), idesc, 1u);
                tc_mma(tmem, smem_desc(al + o), smem_desc(bh + o), idesc, 1u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             bar_addr)
                         : "memory");
        }
        any = true;
        // the MMAs read the tiles: wait for them before the next stage rewrites
        // them (a CTA-wide verdict, so every thread leaves the loop together)
        ok = __syncthreads_and(mbar_wait(bar_addr, phase) ? 1 : 0) != 0;
        if (!ok) mbar_wait(bar_addr, phase);   // a last bounded wait for the MMAs in flight
        phase ^= 1u;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    float acc[NT];
    if (any && ok) {
        tmem_load_row<NT>(tmem + ((uint32_t)(32 * warp) << 16), acc);
    } else {
#pragma unroll
        for (int n = 0; n < NT; ++n) acc[n] = 0.f;
        if (!ok && lane == 0) atomicExch(err, 1);
    }
    const int m = m0 + 32 * warp + lane;
#pragma unroll
    for (int n = 0; n < NT; ++n) part[((size_t)blockIdx.y * Mpad + m) * NT + n] = acc[n];
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;\n" ::"r"(tmem) : "memory");
}

// G[i + c * nB] = sum over row chunks of part, one warp per entry: lane l
// sums chunks l, l + 32, ... in FP64, then a fixed butterfly of shuffles
// (the same association every run).
__global__ void k_gram_reduce(const float *__restrict__ part, int nchunks, int Mpad, int NT, int nB, int s,
                              double *__restrict__ G) {
    const int lane = threadIdx.x & 31;
    const int64_t w0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t n = (int64_t)nB * s;
    for (int64_t t = w0; t < n; t += nw) {
        const int i = (int)(t % nB), c = (int)(t / nB);
        double acc = 0.0;
        for (int q = lane; q < nchunks; q += 32) acc += (double)part[((size_t)q * Mpad + i) * NT + c];
        for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) G[t] = acc;
    }
}

// Rows of D per CTA: D / 1024 rounded up to whole 64-row stages, at least 256.
static int64_t gram_chunk_rows(int64_t D) {
    int64_t c = (D + 1023) / 1024;
    c = (c + kTcStage - 1) / kTcStage * kTcStage;
    return std::max<int64_t>(c, 256);
}

template <int NT>
static void launch_gram(pf_handle *h, cudaStream_t st, int64_t D, int nB, const double *B, int ldb, const double *r,
                        int s, double *G, float *part, int mtiles, int nchunks, int64_t chunk, int *err) {
    auto kern = k_gram_bf16x3<NT>;
    const int smem = TcSmem::total(NT);
    if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    kern<<<dim3(mtiles, nchunks), kTcThreads, smem, st>>>(B, ldb, nB, r, s, (uint32_t)D, (uint32_t)chunk, part,
                                                          mtiles * kTcM, err);
    PF_CUDA(cudaGetLastError());
    const int64_t warps = (int64_t)nB * s;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)h->num_sms * 8, (warps + 7) / 8));
    k_gram_reduce<<<grid, 256, 0, st>>>(part, nchunks, mtiles * kTcM, NT, nB, s, G);
    PF_CUDA(cudaGetLastError());
    count_launches(2);
}

size_t gram_bf16_workspace(int64_t D, int nB, int s) {
    const int NT = s <= 8 ? 8 : (s <= 16 ? 16 : 32);
    const int64_t chunk = gram_chunk_rows(D);
    const int64_t mtiles = (nB + kTcM - 1) / kTcM, nchunks = (D + chunk - 1) / chunk;
    return (size_t)nchunks * mtiles * kTcM * NT * sizeof(float) + 256;
}

// G (nB x s, column-major, FP64) = B^T r with B row-major D x nB (row stride
// ldb) and r row-major D x s, on the tensor cores in split BF16.  work holds
// gram_bf16_workspace(D, nB, s) bytes; err is a device int the kernel sets
// when a wait gives up (read by the caller at its next synchronisation).
void gram_bf16x3(pf_handle *h, cudaStream_t st, int64_t D, int nB, const double *B, int ldb, const double *r, int s,
                 double *G, void *work, int *err) {
    PF_CHECK(s >= 1 && s <= 32, PF_ERR_UNSUPPORTED, "the tensor-core Gram product needs 1 <= s <= 32");
    PF_CHECK(nB >= 1 && D >= 1 && ldb >= nB, PF_ERR_INVALID, "invalid Gram product shape");
    const int mtiles = (nB + kTcM - 1) / kTcM;
    const int64_t chunk = gram_chunk_rows(D);
    const int nchunks = (int)((D + chunk - 1) / chunk);
    PF_CHECK(nchunks <= 65535, PF_ERR_UNSUPPORTED, "block too tall for the tensor-core Gram product");
    float *part = static_cast<float *>(work);
    if (s <= 8) launch_gram<8>(h, st, D, nB, B, ldb, r, s, G, part, mtiles, nchunks, chunk, err);
    else if (s <= 16) launch_gram<16>(h, st, D, nB, B, ldb, r, s, G, part, mtiles, nchunks, chunk, err);
    else launch_gram<32>(h, st, D, nB, B, ldb, r, s, G, part, mtiles, nchunks, chunk, err);
}

}  // namespace pf
