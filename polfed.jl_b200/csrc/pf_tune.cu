// pf_tune.cu -- the step-kernel autotuner.
//
// The Clenshaw / KPM / apply step can give each thread 1..16 columns of a
// row (more columns per thread amortise the per-row basis-state, diagonal
// and flip-rank work; fewer raise occupancy and parallelism), or, for chain
// operators, share each row among s lanes of a warp (width 0, the
// warp-cooperative step).  Each width comes in five profiles: the default
// gather batch and register cap, and the (gather batch U, resident CTAs per
// SM) pairs (8, 2), (8, 3), (4, 4), (8, 4) -- more independent gathers per
// thread against more resident warps.  Quantum Sun operators add the
// asynchronous-gather step and the shared-memory row-tile steps (tiles of
// 1, 2 or 4 rows per thread); sector chains add the local flip-rank step.  The best choice depends on the model,
// s, dtype and D, so it is measured: every variant runs the recurrence step
// (the filter's dominant launch) on scratch blocks, timed with CUDA events on
// the handle's stream, and the fastest is kept on the operator.  Every
// variant computes the same sums in the same order, so the choice changes
// speed only.
//
// Measurements persist across processes in a JSON cache (one object of
// "key": [variant code, microseconds] entries; the key names the device, the
// model and its sizes, s and the element size).  Its path is
// $POLFED_B200_TUNE_CACHE, else $HOME/.cache/polfed_b200/step_variants.json;
// an unreadable or unwritable cache is ignored.
#include "pf_internal.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

namespace pf {

// --------------------------------------------------------------- the cache
static std::mutex g_cache_mu;
static bool g_cache_loaded = false;
static std::map<std::string, std::pair<int, double>> g_cache;

static std::string cache_path() {
    const char *p = std::getenv("POLFED_B200_TUNE_CACHE");
    if (p && *p) return p;
    const char *home = std::getenv("HOME");
    if (!home || !*home) return "";
    return std::string(home) + "/.cache/polfed_b200/step_variants.json";
}

static void load_cache_locked() {
    if (g_cache_loaded) return;
    g_cache_loaded = true;
    const std::string path = cache_path();
    if (path.empty()) return;
    FILE *f = std::fopen(path.c_str(), "r");
    if (!f) return;
    char line[1024];
    while (std::fgets(line, sizeof line, f)) {
        // "key": [code, us]
        char *q0 = std::strchr(line, '"');
        if (!q0) continue;
        char *q1 = std::strchr(q0 + 1, '"');
        if (!q1) continue;
        int code = 0;
        double us = 0.0;
        if (std::sscanf(q1 + 1, " : [ %d , %lf ]", &code, &us) == 2)
            g_cache[std::string(q0 + 1, q1)] = {code, us};
    }
    std::fclose(f);
}

static void save_cache_locked() {
    const std::string path = cache_path();
    if (path.empty()) return;
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) {
        // create the directory chain (each level; errors surface at fopen)
        std::string dir = path.substr(0, slash);
        for (size_t i = 1; i <= dir.size(); ++i)
            if (i == dir.size() || dir[i] == '/') mkdir(dir.substr(0, i).c_str(), 0755);
    }
    const std::string tmp = path + ".tmp" + std::to_string((long)getpid());
    FILE *f = std::fopen(tmp.c_str(), "w");
    if (!f) return;
    std::fprintf(f, "{\n");
    size_t i = 0;
    for (const auto &kv : g_cache)
        std::fprintf(f, "  \"%s\": [%d, %.3f]%s\n", kv.first.c_str(), kv.second.first, kv.second.second,
                     ++i < g_cache.size() ? "," : "");
    std::fprintf(f, "}\n");
    std::fclose(f);
    std::rename(tmp.c_str(), path.c_str());   // atomic replace: readers see the old or the new file
}

static std::string cache_key(const pf_op *op, int s, int elem) {
    cudaDeviceProp prop;
    std::string dev = "cuda";
    if (cudaGetDeviceProperties(&prop, op->h->device) == cudaSuccess) dev = prop.name;
    for (char &c : dev)
        if (c == '"' || c == '\\') c = '_';
    std::string k = dev + "|";
    if (op->kind == OP_CHAIN)
        k += "chain|L=" + std::to_string(op->L) + "|Lup=" + std::to_string(op->Lup) + "|nb=" +
             std::to_string(op->bonds.size() / 2);
    else if (op->kind == OP_QSUN)
        k += "qsun|Lloc=" + std::to_string(op->L_loc) + "|Lgrain=" + std::to_string(op->L_grain);
    else
        k += "csr|nnz=" + std::to_string(op->nnz);
    k += "|D=" + std::to_string(op->dim) + "|s=" + std::to_string(s) + "|elem=" + std::to_string(elem);
    return k;
}

// ----------------------------------------------------------- the timing
template <typename T>
static int tune_typed(pf_op *op, int s, std::vector<std::pair<int, float>> *timings) {
    pf_handle *h = op->h;
    cudaStream_t st = h->stream;
    const int64_t D = op->dim;
    const size_t n = (size_t)D * s;
    T *buf = nullptr;
    PF_CUDA(cudaMalloc(&buf, 3 * n * sizeof(T)));
    T *q = buf, *p = buf + n, *x = buf + 2 * n;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int best = default_width(s, (int)sizeof(T));
    float best_ms = 1e30f;
    try {
        launch_probes<T>(st, D, s, PF_PROBE_GAUSSIAN, 1, 0, q);
        launch_probes<T>(st, D, s, PF_PROBE_GAUSSIAN, 2, 0, p);
        launch_probes<T>(st, D, s, PF_PROBE_GAUSSIAN, 3, 0, x);
        PF_CUDA(cudaEventCreate(&e0));
        PF_CUDA(cudaEventCreate(&e1));
        const int vmax = 64 / (int)sizeof(T);
        const int reps = 20;
        // The recurrence b_k = c X + 2 Ht b_{k+1} - b_{k+2} with a norm-preserving
        // scaling (alpha = 0.5, beta = -0.25) keeps the scratch data bounded.
        std::vector<int> codes;
        for (int V = 1; V <= vmax; V *= 2)
            if (s % V == 0)
                for (int prof = 0; prof <= kStepProfiles; ++prof)
                    if ((prof != kProfileAsync || qsun_async_eligible(op, s, V, (int)sizeof(T))) &&
                        (qsun_tile_ipt(prof) == 0 || qsun_tile_eligible(op, s, V, (int)sizeof(T), prof)) &&
                        (prof != kProfileLocalRank || (op->kind == OP_CHAIN && op->Lup >= 0)))
                        codes.push_back(variant_code(V, prof));
        if (coop_eligible(op, s, StepFlags::Q | StepFlags::P | StepFlags::X)) codes.push_back(kCoopWidth);
        struct Refuse {
            Refuse() { t_refuse_spilling = true; }
            ~Refuse() { t_refuse_spilling = false; }
        } refuse;
        for (int code : codes) {
            try {
                launch_step_width<T>(op, st, D, s, q, p, x, p, 0.1, 0.5, -0.25, 0.05, 0.0,
                                     StepFlags::Q | StepFlags::P | StepFlags::X, nullptr, code);
            } catch (const Error &e) {
                if (e.code == PF_ERR_UNSUPPORTED) continue;   // spills: not a candidate
                throw;
            }
            for (int r = 0; r < 2; ++r)
                launch_step_width<T>(op, st, D, s, q, p, x, p, 0.1, 0.5, -0.25, 0.05, 0.0,
                                     StepFlags::Q | StepFlags::P | StepFlags::X, nullptr, code);
            PF_CUDA(cudaEventRecord(e0, st));
            for (int r = 0; r < reps; ++r)
                launch_step_width<T>(op, st, D, s, q, p, x, p, 0.1, 0.5, -0.25, 0.05, 0.0,
                                     StepFlags::Q | StepFlags::P | StepFlags::X, nullptr, code);
            PF_CUDA(cudaEventRecord(e1, st));
            PF_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            PF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            ms /= reps;
            if (timings) timings->push_back({code, ms});
            if (ms < best_ms) {
                best_ms = ms;
                best = code;
            }
        }
    } catch (...) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaFree(buf);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PF_CUDA(cudaFree(buf));
    {
        std::lock_guard<std::mutex> lock(op->tune_mu);
        op->tuned_width[std::make_pair((int)sizeof(T), s)] = best;
    }
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        load_cache_locked();
        g_cache[cache_key(op, s, (int)sizeof(T))] = {best, best_ms * 1e3};
        save_cache_locked();
    }
    return best;
}

int autotune_step(pf_op *op, int s, int dtype, std::vector<std::pair<int, float>> *timings) {
    PF_CHECK(s >= 1, PF_ERR_INVALID, "s must be positive");
    PF_CUDA(cudaSetDevice(op->h->device));
    if (dtype == PF_F64) return tune_typed<double>(op, s, timings);
    if (dtype == PF_F32) return tune_typed<float>(op, s, timings);
    throw Error(PF_ERR_INVALID, "dtype must be PF_F64 or PF_F32");
}

void variant_params(int code, int elem, int *V, int *U, int *MB) {
    if (code == kCoopWidth) {
        *V = 0, *U = 0, *MB = 0;
        return;
    }
    *V = variant_width(code);
    const int prof = variant_profile(code);
    const int bytes = *V * elem;
    // defaults of the width (profiles 0 and 7 use them)
    *U = bytes >= 64 ? 2 : (bytes >= 16 ? 4 : 8);
    *MB = bytes >= 32 ? 2 : 3;
    static const int prof_u[5] = {0, 8, 8, 4, 8}, prof_mb[5] = {0, 2, 3, 4, 4};
    if (prof >= 1 && prof <= 4) *U = prof_u[prof], *MB = prof_mb[prof];
    if (prof == kProfileAsync) *U = 0, *MB = 0;   // every gather of a row at once
    if (qsun_tile_ipt(prof) > 0) *U = 4, *MB = 2;
}

bool cached_step_variant(pf_op *op, int s, int dtype) {
    const int elem = dtype == PF_F64 ? 8 : 4;
    std::lock_guard<std::mutex> lock(g_cache_mu);
    load_cache_locked();
    auto it = g_cache.find(cache_key(op, s, elem));
    if (it == g_cache.end()) return false;
    const int code = it->second.first;
    const int V = variant_width(code), prof = variant_profile(code);
    const bool ok = code == kCoopWidth ? coop_eligible(op, s, StepFlags::Q | StepFlags::P | StepFlags::X)
                                       : (V >= 1 && s % V == 0 && V * elem <= 64 && prof >= 0 && prof <= kStepProfiles);
    if (!ok) return false;
    std::lock_guard<std::mutex> lock2(op->tune_mu);
    op->tuned_width[std::make_pair(elem, s)] = code;
    return true;
}

// ------------------------------------------------- gather-throughput probe
// The roofline of a step whose blocks stay in L2: every thread owns half of a
// 64-byte row (32 bytes, the FP64 s = 8 step's segment) and reads that half
// of 16 other rows (row XOR a fixed mask per gather, the access pattern of
// spin flips) of an L2-resident block of D rows, summing them.  All indices
// stay below D (a power of two).
template <int NG>
__global__ void k_gather_probe(const double4 *__restrict__ q, double4 *__restrict__ out, uint32_t D) {
    const uint32_t items = 2 * D;
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < items; it += gridDim.x * blockDim.x) {
        const uint32_t row = it >> 1, half = it & 1u;
        double4 a = make_double4(0.0, 0.0, 0.0, 0.0);
#pragma unroll
        for (int k = 0; k < NG; ++k) {
            const uint32_t mask = (0x9e3779b9u * (uint32_t)(k + 1)) >> 7;
            const uint32_t nb = (row ^ mask) & (D - 1u);
            const double4 v = q[(size_t)nb * 2 + half];
            a.x += v.x;
            a.y += v.y;
            a.z += v.z;
            a.w += v.w;
        }
        out[it] = a;
    }
}

double gather_peak(pf_handle *h, int log2_rows) {
    PF_CHECK(log2_rows >= 10 && log2_rows <= 24, PF_ERR_INVALID, "log2_rows must be in [10, 24]");
    PF_CUDA(cudaSetDevice(h->device));
    const uint32_t D = 1u << log2_rows;
    double4 *q = nullptr, *out = nullptr;
    PF_CUDA(cudaMalloc(&q, (size_t)D * 64));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double best = 0.0;
    try {
        PF_CUDA(cudaMalloc(&out, (size_t)D * 64));
        PF_CUDA(cudaMemsetAsync(q, 0, (size_t)D * 64, h->stream));
        PF_CUDA(cudaEventCreate(&e0));
        PF_CUDA(cudaEventCreate(&e1));
        constexpr int NG = 16;
        for (int mult = 2; mult <= 8; mult *= 2) {
            const int grid = h->num_sms * mult;
            for (int r = 0; r < 3; ++r) k_gather_probe<NG><<<grid, 256, 0, h->stream>>>(q, out, D);
            PF_CUDA(cudaGetLastError());
            PF_CUDA(cudaEventRecord(e0, h->stream));
            const int reps = 50;
            for (int r = 0; r < reps; ++r) k_gather_probe<NG><<<grid, 256, 0, h->stream>>>(q, out, D);
            PF_CUDA(cudaEventRecord(e1, h->stream));
            PF_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            PF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            const double sec = ms * 1e-3 / reps;
            best = std::max(best, (double)D * 2 * NG * 32 / sec);   // bytes gathered per second
        }
    } catch (...) {
        cudaFree(q);
        cudaFree(out);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        throw;
    }
    cudaFree(q);
    cudaFree(out);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    count_launches(9 * 53);
    return best;
}

}  // namespace pf
