// pf_noalloc.cu -- pf_apply_noalloc: the operator apply without any device allocation.
//
// pf_apply stages column-major blocks (s > 1) through handle scratch that it
// grows with cudaMalloc on demand.  Some callers cannot let a library allocate
// device memory: a Julia CuArray or PyTorch caching-allocator pool that owns
// the whole HBM budget, or a latency-critical loop in which cudaMalloc /
// cudaFree's implicit device synchronisation is not acceptable.  This variant
// stages the blocks in one fixed array compiled into the library instead.
//
// The array: NOALLOC_BYTES (16 MiB) of file-scope device memory.  Every GPU
// that loads the library holds it until the process exits.  Host code cannot
// use the array's name as a device address (on the host it is only a
// stand-in), so the device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, and passed to the kernels.
// That look-up happens inside the first call on each device; make that first
// call before any stream capture.
//
// Every call on every stream shares the one array and it keeps the previous
// call's contents: calls that overlap on the GPU race and must be ordered by
// the caller.  Nothing in it needs to start at zero: each call overwrites
// exactly the part it then reads.
#include "pf_internal.h"
#include "pf_solver.h"

#include <cmath>
#include <mutex>

namespace pf {

constexpr size_t NOALLOC_BYTES = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
static void *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};
static std::mutex g_noalloc_mu;

// Device address of the scratch array on `device` (looked up once per device).
static void *noalloc_scratch(int device) {
    PF_CHECK(device >= 0 && device < NOALLOC_MAX_DEVICES, PF_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        PF_CUDA(cudaSetDevice(device));
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            throw Error(PF_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_ptr[device] = p;
    }
    return g_noalloc_ptr[device];
}

template <typename T>
static void apply_noalloc_typed(pf_op *op, double a, double b, int s, const T *X, int64_t ldx, T *Y, int64_t ldy) {
    pf_handle *h = op->h;
    const int64_t D = op->dim;
    void *scratch = noalloc_scratch(h->device);
    PF_CUDA(cudaSetDevice(h->device));
    if (s == 1) {  // a column-major vector is already row-interleaved: no staging
        launch_step<T>(op, h->stream, D, 1, X, nullptr, nullptr, Y, 0, 1.0, 0, 1.0 / a, b, StepFlags::Q, nullptr);
        return;
    }
    const size_t n = (size_t)D * s;
    const size_t half = (n * sizeof(T) + 255) / 256 * 256;
    T *xr = reinterpret_cast<T *>(scratch);
    T *yr = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(scratch) + half);
    launch_cm_to_ri<T, T>(h->stream, D, s, X, ldx, xr);
    launch_step<T>(op, h->stream, D, s, xr, nullptr, nullptr, yr, 0, 1.0, 0, 1.0 / a, b, StepFlags::Q, nullptr);
    launch_ri_to_cm<T, T>(h->stream, D, s, yr, Y, ldy);
}

void op_apply_noalloc(pf_op *op, int dtype, double a, double b, int s, const void *X, int64_t ldx, void *Y,
                      int64_t ldy) {
    PF_CHECK(X && Y && s >= 1, PF_ERR_INVALID, "invalid apply arguments");
    PF_CHECK(ldx >= op->dim && ldy >= op->dim, PF_ERR_INVALID, "leading dimension smaller than the operator dimension");
    PF_CHECK(a != 0.0 && std::isfinite(a) && std::isfinite(b), PF_ERR_INVALID, "rescaling a must be finite and nonzero");
    PF_CHECK(dtype == PF_F64 || dtype == PF_F32, PF_ERR_INVALID, "dtype must be PF_F64 or PF_F32");
    const size_t elem = dtype == PF_F64 ? 8 : 4;
    const size_t need = s == 1 ? 0 : 2 * ((((size_t)op->dim * s * elem) + 255) / 256 * 256);
    if (need > NOALLOC_BYTES)
        throw Error(PF_ERR_INVALID, "pf_apply_noalloc: the block needs " + std::to_string(need) +
                                        " bytes of staging but the fixed scratch holds " +
                                        std::to_string(NOALLOC_BYTES) +
                                        " (2*D*s*element_size must not exceed 16 MiB; use pf_apply)");
    if (dtype == PF_F64)
        apply_noalloc_typed<double>(op, a, b, s, (const double *)X, ldx, (double *)Y, ldy);
    else
        apply_noalloc_typed<float>(op, a, b, s, (const float *)X, ldx, (float *)Y, ldy);
}

}  // namespace pf
