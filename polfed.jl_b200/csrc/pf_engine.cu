// pf_engine.cu -- continuous batching of Chebyshev filter steps.
//
// A solve's filter application Y = sum_k c_k T_k(Htilde) X is K + 1
// dependent Clenshaw steps (ClenshawAlgorithm.jl:12-29).  On one solve a step
// at D ~ 10^4..10^5 is a few microseconds of latency-bound work that cannot
// fill 148 SMs.  The engine runs the steps of every filter in flight -- of
// all solves of a request pool, whatever their operators, dimensions, orders
// and progress -- as ONE kernel launch per step: k_step_multi walks
// (instance, row) work items over a table of instances passed as a kernel
// parameter.  A filter joins at the next launch after it is submitted and
// leaves after its own final sum, so solves with different orders K and
// different arrival times share launches (continuous batching), and each
// instance computes exactly what the per-solve kernel computes (same rows,
// same order of additions): a solve's result does not depend on its company.
//
// Host side: one engine thread per pool issues the launches on its own
// stream.  A worker submits a job (its RI blocks X, Y and two work blocks,
// the coefficients, an event marking X ready on the worker's stream) and
// blocks until the job's last step is enqueued; it then orders its stream
// after the job's completion event.  At most kMaxInFlight launches are queued
// ahead of the GPU, so new filters join within a few steps.
#include "pf_internal.h"
#include "pf_rows.cuh"
#include "pf_solver.h"

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <thread>
#include <tuple>

namespace pf {

constexpr int kMultiMax = 48;        // instances per launch
constexpr int kMultiThreads = 256;
constexpr int kMaxInFlight = 4;      // launches queued ahead of the GPU

template <typename T>
struct MultiEntry {
    const T *q;
    const T *p;
    const T *x;
    T *out;
    const void *desc;     // device copy of the instance's ChainDesc<T> / QSunDesc<T> / CsrDesc<T>
    uint32_t D;           // rows
    uint32_t tile0;       // first tile of the instance (a tile = kMultiThreads work items of one instance)
    int flags;            // StepFlags Q / P / X of this instance's step
    T cx, alpha, beta, inva, boa;
};

template <typename T>
struct MultiArgs {
    int n, s, G;
    uint32_t tiles;
    const uint32_t *rank_tab;  // chain: rank tables with nchunks chunks (the same for every L)
    int nchunks;
    int desc_words;            // sizeof(descriptor) / 16
    MultiEntry<T> e[kMultiMax];
};

template <int KIND, typename T>
struct KindDesc;
template <typename T>
struct KindDesc<OP_CHAIN, T> { using type = ChainDesc<T>; };
template <typename T>
struct KindDesc<OP_QSUN, T> { using type = QSunDesc<T>; };
template <typename T>
struct KindDesc<OP_CSR, T> { using type = CsrDesc<T>; };

// Shared memory of k_step_multi: the instance's descriptor, then the model's
// tables (chain: the rank tables, staged once; Quantum Sun: the padded grain
// block and the byte-wise diagonal tables of k_step, restaged per instance).
template <int KIND, typename T>
__host__ __device__ inline int multi_table_offset() {
    return ((int)sizeof(typename KindDesc<KIND, T>::type) + 15) / 16 * 16;
}

// out_i = cx_i X_i + alpha_i Htilde_i(q_i) + beta_i p_i for every instance i
// of the table.  Each CTA walks a contiguous range of tiles; a tile holds
// work items of one instance only, and when the instance changes the CTA
// stages its descriptor and tables in shared memory, so every row is
// evaluated by k_step's own row functions on the same shared-memory data
// (identical results).
template <typename T, int V, int KIND>
__global__ void __launch_bounds__(kMultiThreads, MinBlocks<T, V>::value)
    k_step_multi(const __grid_constant__ MultiArgs<T> a) {
    using Desc = typename KindDesc<KIND, T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Desc &d = *reinterpret_cast<const Desc *>(smem_raw);
    unsigned char *tabs = smem_raw + multi_table_offset<KIND, T>();
    const uint32_t *tab = reinterpret_cast<const uint32_t *>(tabs);
    const T *smem_t = reinterpret_cast<const T *>(tabs);
    if constexpr (KIND == OP_CHAIN) {
        const int n = rank_table_entries(a.nchunks);
        uint32_t *t = reinterpret_cast<uint32_t *>(tabs);
        for (int i = threadIdx.x; i < n; i += blockDim.x) t[i] = __ldg(a.rank_tab + i);
    }
    const uint32_t per = (a.tiles + gridDim.x - 1) / gridDim.x;
    const uint32_t t0 = blockIdx.x * per, t1 = min(a.tiles, t0 + per);
    int cur = -1;
    for (uint32_t tile = t0; tile < t1; ++tile) {
        int lo = 0, hi = a.n - 1;   // the instance owning this tile: last tile0 <= tile
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.e[mid].tile0 <= tile) lo = mid;
            else hi = mid - 1;
        }
        const MultiEntry<T> &e = a.e[lo];
        if (lo != cur) {
            __syncthreads();   // the previous instance's rows are done with the shared data
            const uint4 *src = static_cast<const uint4 *>(e.desc);
            uint4 *dst = reinterpret_cast<uint4 *>(smem_raw);
            for (int i = threadIdx.x; i < a.desc_words; i += blockDim.x) dst[i] = src[i];
            __syncthreads();
            if constexpr (KIND == OP_QSUN) {
                T *sm = reinterpret_cast<T *>(tabs);
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
            }
            __syncthreads();
            cur = lo;
        }
        const uint32_t local = (tile - e.tile0) * kMultiThreads + threadIdx.x;
        const uint32_t G = (uint32_t)a.G;
        if (local >= e.D * G) continue;
        const uint32_t row = (G == 1u) ? local : local / G;
        const int c0 = (G == 1u) ? 0 : (int)(local - row * G) * V;
        const size_t off = (size_t)row * a.s + c0;
        const bool hasq = (e.flags & StepFlags::Q) != 0;
        if (e.flags & StepFlags::X) prefetch_l1(e.x + off);
        if (hasq) prefetch_l1(e.q + off);
        if (e.flags & StepFlags::P) prefetch_l1(e.p + off);
        T acc[V];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = T(0);
        T diag = T(0);
        if (hasq) {
            if constexpr (KIND == OP_CHAIN)
                chain_row<T, V, true>(d, tab, row, a.s, c0, e.q, acc, diag);
            else if constexpr (KIND == OP_QSUN)
                qsun_row<T, V, true>(d, smem_t, row, a.s, c0, e.q, acc, diag);
            else
                csr_row<T, V, true>(d, row, a.s, c0, e.q, acc, diag);
        }
        const bool hasx = (e.flags & StepFlags::X) != 0, hasp = (e.flags & StepFlags::P) != 0;
        Pack<T, V> xo, qo, po, res;
#pragma unroll
        for (int v = 0; v < V; ++v) xo.v[v] = qo.v[v] = po.v[v] = T(0);
        if (hasx) xo = ldp<T, V>(e.x + off);
        if (hasq) qo = ldp<T, V>(e.q + off);
        if (hasp) po = ldp<T, V>(e.p + off);
#pragma unroll
        for (int v = 0; v < V; ++v)
            res.v[v] = step_combine<T>(hasx, hasq, hasp, e.cx, xo.v[v], e.alpha, acc[v], diag, qo.v[v], e.inva, e.boa,
                                       e.beta, po.v[v]);
        stp<T, V>(e.out + off, res);
    }
}

// Device copies of the descriptors (both precisions), read by the engine's
// multi-instance kernel; shared with every view of the operator.
void build_multi_tables(pf_op *op) {
    const int dev = op->h->device;
    void *d64 = nullptr, *d32 = nullptr;
    size_t b64 = 0, b32 = 0;
    const void *h64 = nullptr, *h32 = nullptr;
    if (op->kind == OP_CHAIN) {
        b64 = sizeof(ChainDesc<double>), b32 = sizeof(ChainDesc<float>);
        h64 = &op->chain64, h32 = &op->chain32;
    } else if (op->kind == OP_QSUN) {
        b64 = sizeof(QSunDesc<double>), b32 = sizeof(QSunDesc<float>);
        h64 = &op->qsun64, h32 = &op->qsun32;
    } else {
        b64 = sizeof(CsrDesc<double>), b32 = sizeof(CsrDesc<float>);
        h64 = &op->csr64, h32 = &op->csr32;
    }
    try {
        // rounded up to whole 16-byte words: the kernel stages descriptors as uint4
        PF_CUDA(cudaMalloc(&d64, (b64 + 15) / 16 * 16));
        PF_CUDA(cudaMalloc(&d32, (b32 + 15) / 16 * 16));
        PF_CUDA(cudaMemcpy(d64, h64, b64, cudaMemcpyHostToDevice));
        PF_CUDA(cudaMemcpy(d32, h32, b32, cudaMemcpyHostToDevice));
    } catch (...) {
        cudaFree(d64);
        cudaFree(d32);
        throw;
    }
    op->d_desc64 = d64;
    op->d_desc32 = d32;
    op->multi_owner = std::shared_ptr<void>(nullptr, [d64, d32, dev](void *) {
        cudaSetDevice(dev);
        cudaFree(d64);
        cudaFree(d32);
    });
}

bool multi_eligible(const pf_op *op, int dtype) {
    (void)dtype;
    return op->d_desc64 != nullptr && op->d_desc32 != nullptr;
}

// ------------------------------------------------------------- the engine
struct FilterJob {
    pf_op *op = nullptr;
    int elem = 8, s = 1, V = 1, K = 0;
    std::vector<double> c;
    double inva = 1.0, shift = 0.0;
    void *X = nullptr, *Y = nullptr, *A = nullptr, *B = nullptr;
    int t = 0;                       // next step: K, K-1, ..., 0
    cudaEvent_t ready = nullptr;     // X in place (submitting stream)
    cudaEvent_t done = nullptr;      // Y written (engine stream)
    bool joined = false, finished = false;
    int status = PF_OK;
    std::string error;
};

}  // namespace pf

struct pf_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::thread thread;
    std::mutex mu;
    std::condition_variable cv_in, cv_out;
    std::deque<pf::FilterJob *> incoming;
    bool stop = false;
    // accounting of the multi-instance launches (for the roofline)
    double launches = 0, kernel_seconds = 0, bytes = 0, instance_steps = 0;
    std::deque<std::pair<cudaEvent_t, cudaEvent_t>> timing;   // launches whose time is not read yet
    std::vector<cudaEvent_t> spare;
    std::deque<double> timing_bytes;
};

namespace pf {

// The RI block a job's step at index t reads as q / p and writes (the
// rotation of Filter::enqueue in pf_solver.cu).
template <typename T>
static MultiEntry<T> job_entry(const FilterJob &j) {
    MultiEntry<T> e{};
    const int K = j.K, t = j.t;
    T *X = (T *)j.X, *Y = (T *)j.Y, *A = (T *)j.A, *B = (T *)j.B;
    e.x = X;
    e.cx = (T)j.c[t];
    e.inva = (T)j.inva;
    e.boa = (T)(j.shift * j.inva);
    e.D = (uint32_t)j.op->dim;
    const pf_op *op = j.op;
    e.desc = sizeof(T) == 8 ? op->d_desc64 : op->d_desc32;
    using F = StepFlags;
    if (K == 0) {
        e.flags = F::X;
        e.out = Y;
    } else if (t == K) {
        e.flags = F::X;
        e.out = A;
    } else if (t == K - 1 && K >= 2) {
        e.flags = F::Q | F::X;
        e.q = A;
        e.alpha = 2;
        e.out = B;
    } else if (t >= 1) {
        T *q = ((K - t - 1) % 2 == 0) ? A : B;
        T *o = ((K - t) % 2 == 0) ? A : B;
        e.flags = F::Q | F::P | F::X;
        e.q = q;
        e.p = o;
        e.out = o;
        e.alpha = 2;
        e.beta = -1;
    } else {
        T *b1 = ((K - 1) % 2 == 0) ? A : B;
        e.q = b1;
        e.alpha = 1;
        e.out = Y;
        if (K == 1) {
            e.flags = F::Q | F::X;
        } else {
            e.flags = F::Q | F::P | F::X;
            e.p = ((K - 2) % 2 == 0) ? A : B;
            e.beta = -1;
        }
    }
    return e;
}

static int multi_blocks_per_sm(const void *kern, int smem) {
    thread_local std::map<std::pair<const void *, int>, int> cache;
    auto key = std::make_pair(kern, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int nb = 0;
    PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, kMultiThreads, smem));
    nb = std::max(nb, 1);
    cache[key] = nb;
    return nb;
}

template <typename T, int V, int KIND>
static void launch_multi_kind(pf_engine *eng, int num_sms, MultiArgs<T> &a) {
    auto kern = k_step_multi<T, V, KIND>;
    using Desc = typename KindDesc<KIND, T>::type;
    a.desc_words = ((int)sizeof(Desc) + 15) / 16;
    int smem = multi_table_offset<KIND, T>();
    if (KIND == OP_CHAIN) smem += rank_table_entries(a.nchunks) * 4;
    if (KIND == OP_QSUN) smem += QSunSmem<T>::bytes(PF_MAX_GRAIN);
    if (smem > 48 * 1024) PF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int64_t cap = (int64_t)num_sms * multi_blocks_per_sm((const void *)kern, smem);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(a.tiles, cap));
    kern<<<grid, kMultiThreads, smem, eng->stream>>>(a);
    PF_CUDA(cudaGetLastError());
}

template <typename T, int KIND>
static void launch_multi_v(pf_engine *eng, int num_sms, int V, MultiArgs<T> &a) {
    switch (V) {
        case 1: launch_multi_kind<T, 1, KIND>(eng, num_sms, a); break;
        case 2: launch_multi_kind<T, 2, KIND>(eng, num_sms, a); break;
        case 4: launch_multi_kind<T, 4, KIND>(eng, num_sms, a); break;
        case 8: launch_multi_kind<T, 8, KIND>(eng, num_sms, a); break;
        case 16:
            if constexpr (sizeof(T) == 4) { launch_multi_kind<T, 16, KIND>(eng, num_sms, a); break; }
            [[fallthrough]];
        default: throw Error(PF_ERR_INVALID, "bad vector width");
    }
}

// One launch over jobs[0..n) (same kind, precision, s and width).  Returns the
// algorithmic bytes it moves.
template <typename T>
static double launch_group(pf_engine *eng, int num_sms, FilterJob *const *jobs, int n) {
    MultiArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    const FilterJob &j0 = *jobs[0];
    a.n = n;
    a.s = j0.s;
    a.G = j0.s / j0.V;
    a.nchunks = 0;
    a.rank_tab = nullptr;
    uint64_t tiles = 0;
    double bytes = 0;
    for (int i = 0; i < n; ++i) {
        const FilterJob &j = *jobs[i];
        a.e[i] = job_entry<T>(j);
        a.e[i].tile0 = (uint32_t)tiles;
        tiles += ((uint64_t)j.op->dim * a.G + kMultiThreads - 1) / kMultiThreads;
        const int f = a.e[i].flags;
        const int streams = 1 + ((f & StepFlags::Q) ? 1 : 0) + ((f & StepFlags::P) ? 1 : 0) + ((f & StepFlags::X) ? 1 : 0);
        bytes += (double)streams * (double)j.op->dim * j.s * sizeof(T);
        if (j.op->kind == OP_CHAIN && !j.op->chain64.full && j.op->chain64.nchunks > a.nchunks) {
            a.nchunks = j.op->chain64.nchunks;
            a.rank_tab = j.op->d_rank_tab;
        }
    }
    PF_CHECK(tiles * kMultiThreads < 0xffffffffull, PF_ERR_UNSUPPORTED, "batched step too large for one launch");
    a.tiles = (uint32_t)tiles;
    switch (j0.op->kind) {
        case OP_CHAIN: launch_multi_v<T, OP_CHAIN>(eng, num_sms, j0.V, a); break;
        case OP_QSUN: launch_multi_v<T, OP_QSUN>(eng, num_sms, j0.V, a); break;
        default: launch_multi_v<T, OP_CSR>(eng, num_sms, j0.V, a); break;
    }
    return bytes;
}

static cudaEvent_t take_event(pf_engine *eng) {
    if (!eng->spare.empty()) {
        cudaEvent_t e = eng->spare.back();
        eng->spare.pop_back();
        return e;
    }
    cudaEvent_t e;
    PF_CUDA(cudaEventCreate(&e));
    return e;
}

// Read the times of finished launches into sec / bytes, blocking until at
// most `keep` launches remain queued ahead of the GPU.
static void drain_timing(pf_engine *eng, size_t keep, double &sec, double &bytes) {
    while (!eng->timing.empty()) {
        auto pr = eng->timing.front();
        if (eng->timing.size() > keep) {
            PF_CUDA(cudaEventSynchronize(pr.second));
        } else if (cudaEventQuery(pr.second) != cudaSuccess) {
            cudaGetLastError();   // cudaErrorNotReady is not an error here
            break;
        }
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) {
            sec += ms * 1e-3;
            bytes += eng->timing_bytes.front();
        }
        eng->timing.pop_front();
        eng->timing_bytes.pop_front();
        eng->spare.push_back(pr.first);
        eng->spare.push_back(pr.second);
    }
}

static void engine_loop(pf_engine *eng) {
    cudaSetDevice(eng->device);
    int num_sms = 148;
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, eng->device);
    std::vector<FilterJob *> active;
    while (true) {
        double pend_launches = 0, pend_steps = 0, pend_sec = 0, pend_bytes = 0;
        {
            std::unique_lock<std::mutex> lock(eng->mu);
            eng->cv_in.wait(lock, [&] { return eng->stop || !eng->incoming.empty() || !active.empty(); });
            if (eng->stop && eng->incoming.empty() && active.empty()) break;
            while (!eng->incoming.empty()) {
                active.push_back(eng->incoming.front());
                eng->incoming.pop_front();
            }
        }
        std::string err;
        int code = PF_OK;
        try {
            for (FilterJob *j : active)
                if (!j->joined) {
                    PF_CUDA(cudaStreamWaitEvent(eng->stream, j->ready, 0));
                    j->joined = true;
                }
            // one launch per (kind, precision, s, width) group, at most kMultiMax instances each
            std::vector<FilterJob *> order(active);
            std::stable_sort(order.begin(), order.end(), [](const FilterJob *x, const FilterJob *y) {
                return std::make_tuple(x->op->kind, x->elem, x->s, x->V) < std::make_tuple(y->op->kind, y->elem, y->s, y->V);
            });
            size_t i = 0;
            while (i < order.size()) {
                size_t k = i + 1;
                while (k < order.size() && k - i < (size_t)kMultiMax && order[k]->op->kind == order[i]->op->kind &&
                       order[k]->elem == order[i]->elem && order[k]->s == order[i]->s && order[k]->V == order[i]->V)
                    ++k;
                cudaEvent_t e0 = take_event(eng), e1 = take_event(eng);
                PF_CUDA(cudaEventRecord(e0, eng->stream));
                const double b = order[i]->elem == 8 ? launch_group<double>(eng, num_sms, order.data() + i, (int)(k - i))
                                                     : launch_group<float>(eng, num_sms, order.data() + i, (int)(k - i));
                PF_CUDA(cudaEventRecord(e1, eng->stream));
                eng->timing.push_back({e0, e1});
                eng->timing_bytes.push_back(b);
                pend_launches += 1;
                pend_steps += (double)(k - i);
                i = k;
            }
            for (FilterJob *j : active) --j->t;
            for (FilterJob *j : active)
                if (j->t < 0) PF_CUDA(cudaEventRecord(j->done, eng->stream));
            drain_timing(eng, kMaxInFlight, pend_sec, pend_bytes);
        } catch (const Error &e) {
            code = e.code;
            err = e.what();
        } catch (const std::exception &e) {
            code = PF_ERR_CUDA;
            err = e.what();
        }
        {
            std::lock_guard<std::mutex> lock(eng->mu);
            eng->launches += pend_launches;
            eng->instance_steps += pend_steps;
            eng->kernel_seconds += pend_sec;
            eng->bytes += pend_bytes;
            std::vector<FilterJob *> keep;
            for (FilterJob *j : active) {
                if (code != PF_OK) {
                    j->status = code;
                    j->error = err;
                    j->finished = true;
                } else if (j->t < 0) {
                    j->finished = true;
                } else {
                    keep.push_back(j);
                }
            }
            active.swap(keep);
        }
        eng->cv_out.notify_all();
    }
    try {
        double sec = 0, bytes = 0;
        drain_timing(eng, 0, sec, bytes);
        std::lock_guard<std::mutex> lock(eng->mu);
        eng->kernel_seconds += sec;
        eng->bytes += bytes;
    } catch (...) {
    }
}

pf_engine *engine_create(int device) {
    PF_CUDA(cudaSetDevice(device));
    pf_engine *eng = new pf_engine();
    eng->device = device;
    int least = 0, greatest = 0;
    try {
        PF_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        PF_CUDA(cudaStreamCreateWithPriority(&eng->stream, cudaStreamNonBlocking, greatest));
    } catch (...) {
        delete eng;
        throw;
    }
    eng->thread = std::thread(engine_loop, eng);
    return eng;
}

void engine_destroy(pf_engine *eng) {
    if (!eng) return;
    {
        std::lock_guard<std::mutex> lock(eng->mu);
        eng->stop = true;
    }
    eng->cv_in.notify_all();
    eng->thread.join();
    cudaSetDevice(eng->device);
    cudaStreamSynchronize(eng->stream);
    for (auto &pr : eng->timing) {
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    for (auto e : eng->spare) cudaEventDestroy(e);
    cudaStreamDestroy(eng->stream);
    delete eng;
}

void engine_stats(pf_engine *eng, double *launches, double *seconds, double *bytes, double *instance_steps) {
    std::lock_guard<std::mutex> lock(eng->mu);
    *launches = eng->launches;
    *seconds = eng->kernel_seconds;
    *bytes = eng->bytes;
    *instance_steps = eng->instance_steps;
}

// Run Y = sum_k c_k T_k(Htilde) X through the engine.  X, Y, A, B are RI
// D x s blocks of the job's precision; X must be written on `st` before the
// call.  Returns after the job's last step is enqueued, with `st` ordered
// after it.
void engine_filter(pf_engine *eng, pf_op *op, cudaStream_t st, int elem, int s, int V,
                   const std::vector<double> &coeffs, double a, double b, void *X, void *Y, void *A, void *B) {
    FilterJob job;
    job.op = op;
    job.elem = elem;
    job.s = s;
    job.V = V;
    job.K = (int)coeffs.size() - 1;
    job.c = coeffs;
    job.inva = 1.0 / a;
    job.shift = b;
    job.X = X, job.Y = Y, job.A = A, job.B = B;
    job.t = job.K;
    PF_CUDA(cudaEventCreateWithFlags(&job.ready, cudaEventDisableTiming));
    cudaError_t ce = cudaEventCreateWithFlags(&job.done, cudaEventDisableTiming);
    if (ce != cudaSuccess) {
        cudaEventDestroy(job.ready);
        throw Error(PF_ERR_CUDA, std::string("cudaEventCreate: ") + cudaGetErrorString(ce));
    }
    struct Events {
        FilterJob &j;
        ~Events() {
            cudaEventDestroy(j.ready);
            cudaEventDestroy(j.done);
        }
    } guard{job};
    PF_CUDA(cudaEventRecord(job.ready, st));
    {
        std::unique_lock<std::mutex> lock(eng->mu);
        PF_CHECK(!eng->stop, PF_ERR_INVALID, "filter engine is shutting down");
        eng->incoming.push_back(&job);
        eng->cv_in.notify_all();
        eng->cv_out.wait(lock, [&] { return job.finished; });
    }
    if (job.status != PF_OK) throw Error(job.status, job.error);
    PF_CUDA(cudaStreamWaitEvent(st, job.done, 0));
    count_launches(job.K + 1);
}

}  // namespace pf
