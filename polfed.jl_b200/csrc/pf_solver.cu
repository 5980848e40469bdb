// pf_solver.cu -- POLFED driver on one B200: Clenshaw filter (graph-captured),
// KPM moments, block Lanczos with full reorthogonalisation, Ritz extraction
// and FP64 residuals.  Reference: Polfed.jl (see each function's citation).
#include "pf_internal.h"
#include "pf_solver.h"

#include <atomic>
#include <complex>
#include <exception>
#include <thread>
#include "pf_spectral.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <map>
#include <memory>
#include <numeric>

namespace pf {

// ------------------------------------------------------------- utilities
// Stream of the entry point running on this host thread.  DevArray allocates
// stream-ordered on it (cudaMallocAsync from the device pool, which keeps
// freed memory), so solves in flight on other handles are never stalled by a
// cudaMalloc / cudaFree device synchronisation.
static thread_local cudaStream_t t_alloc_stream = nullptr;
struct AllocStream {
    cudaStream_t prev;
    explicit AllocStream(cudaStream_t st) : prev(t_alloc_stream) { t_alloc_stream = st; }
    ~AllocStream() { t_alloc_stream = prev; }
};

template <typename T>
struct DevArray {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t st = nullptr;
    DevArray() = default;
    explicit DevArray(size_t count) { alloc(count); }
    void alloc(size_t count) {
        free();
        st = t_alloc_stream;
        if (count) {
            if (st) PF_CUDA(cudaMallocAsync((void **)&p, count * sizeof(T), st));
            else PF_CUDA(cudaMalloc(&p, count * sizeof(T)));
        }
        n = count;
    }
    void free() {
        if (p) {
            if (st) cudaFreeAsync(p, st);
            else cudaFree(p);
        }
        p = nullptr;
        n = 0;
    }
    ~DevArray() { free(); }
    DevArray(const DevArray &) = delete;
    DevArray &operator=(const DevArray &) = delete;
    DevArray(DevArray &&o) noexcept : p(o.p), n(o.n), st(o.st) {
        o.p = nullptr;
        o.n = 0;
    }
    DevArray &operator=(DevArray &&o) noexcept {
        if (this != &o) {
            free();
            p = o.p;
            n = o.n;
            st = o.st;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
};

// Accumulates stage times measured with CUDA events on the solve's stream.
// Events are never reused inside one solve, so a pending pair stays valid
// until flush() reads it after the stream has passed both events.
struct StageClock {
    pf_handle *h;
    cudaStream_t st;
    std::vector<cudaEvent_t> all;
    struct Pending { int stage; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    double *acc;
    StageClock(pf_handle *h_, cudaStream_t s, double *acc_) : h(h_), st(s), acc(acc_) {}
    // the events go back to the handle for the next solve (a later record
    // supersedes any still pending)
    ~StageClock() {
        for (auto e : all) h->timing_events.push_back(e);
    }
    // with no accumulator (an untimed run, e.g. the extremal probes) no
    // events are recorded at all
    cudaEvent_t mark() {
        if (!acc) return nullptr;
        cudaEvent_t e;
        if (!h->timing_events.empty()) {
            e = h->timing_events.back();
            h->timing_events.pop_back();
        } else {
            PF_CUDA(cudaEventCreate(&e));
        }
        all.push_back(e);
        PF_CUDA(cudaEventRecord(e, st));
        return e;
    }
    void add(int stage, cudaEvent_t a, cudaEvent_t b) {
        if (acc && a && b) pending.push_back({stage, a, b});
    }
    void flush() {
        for (auto &p : pending) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess && acc) acc[p.stage] += ms * 1e-3;
        }
        pending.clear();
    }
};

static void sync(pf_handle *h) { PF_CUDA(cudaStreamSynchronize(h->stream)); }

// ------------------------------------------------------------ the filter
// Y = sum_k c_k T_k(Htilde) X on RI blocks (ClenshawAlgorithm.jl:12-29).
// b_k is written in place over b_{k+2}, so two work blocks suffice.
template <typename T>
struct Filter {
    pf_op *op;
    int s, K;
    std::vector<double> c;
    double a, b;
    DevArray<T> X, Y, A, B;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    // io = false: only the two work blocks (the filter engine reads and
    // writes the caller's blocks directly)
    Filter(pf_op *op_, int s_, const std::vector<double> &coeffs, double a_, double b_, bool io = true)
        : op(op_), s(s_), K((int)coeffs.size() - 1), c(coeffs), a(a_), b(b_) {
        const size_t n = (size_t)op->dim * s;
        if (io) {
            X.alloc(n);
            Y.alloc(n);
        }
        if (K >= 1) A.alloc(n);
        if (K >= 2) B.alloc(n);
    }
    ~Filter() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
    // Columns per slab (pf_set_filter_slab): the filter can run in column
    // slabs whose gathered block (D x slab) stays in L2 while the once-touched
    // streams pass with evict-first hints; every column's arithmetic is
    // unchanged.  Off unless requested: at D = 2.7 M, s = 16 the step is
    // bound by the latency of its dependent gathers, not by DRAM traffic, and
    // slabs of 4 FP64 columns took 2.4 ms per step against 1.4 ms whole.
    int slab_cols() const {
        if (op->slab_cols > 0 && s % op->slab_cols == 0) return op->slab_cols;
        return s;
    }
    int launches_per_step() const { return s / slab_cols(); }
    // one step of the recurrence over every slab
    void step(cudaStream_t st, const T *q, const T *p, T *out, double ck, double alpha, double beta, int flags) {
        const int w = slab_cols();
        const int64_t D = op->dim;
        for (int c0 = 0; c0 < s; c0 += w)
            launch_step<T>(op, st, D, w, q ? q + c0 : nullptr, p ? p + c0 : nullptr, X.p + c0, out + c0, ck, alpha, beta,
                           1.0 / a, b, flags, nullptr, w == s ? 0 : s, w == s ? 0 : 1);
    }
    void enqueue(cudaStream_t st) {
        using F = StepFlags;
        if (K == 0) {
            step(st, nullptr, nullptr, Y.p, c[0], 0, 0, F::X);
            return;
        }
        step(st, nullptr, nullptr, A.p, c[K], 0, 0, F::X);
        if (K >= 2) step(st, A.p, nullptr, B.p, c[K - 1], 2.0, 0, F::Q | F::X);
        for (int k = K - 2; k >= 1; --k) {
            T *q = ((K - k - 1) % 2 == 0) ? A.p : B.p;  // b_{k+1}
            T *o = ((K - k) % 2 == 0) ? A.p : B.p;      // b_{k+2}, overwritten by b_k
            step(st, q, o, o, c[k], 2.0, -1.0, F::Q | F::P | F::X);
        }
        T *b1 = ((K - 1) % 2 == 0) ? A.p : B.p;
        if (K == 1) {
            step(st, b1, nullptr, Y.p, c[0], 1.0, 0, F::Q | F::X);
        } else {
            T *b2 = ((K - 2) % 2 == 0) ? A.p : B.p;
            step(st, b1, b2, Y.p, c[0], 1.0, -1.0, F::Q | F::P | F::X);
        }
    }
    // Capture the K+1 launches once; every later application is one graph launch.
    void run(cudaStream_t st) {
        if (!exec) {
            PF_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
            const int64_t before = thread_launches();  // captured launches do not execute
            try {
                enqueue(st);
                count_launches(before - thread_launches());
            } catch (...) {
                cudaGraph_t g;
                cudaStreamEndCapture(st, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            PF_CUDA(cudaStreamEndCapture(st, &graph));
            PF_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        }
        PF_CUDA(cudaGraphLaunch(exec, st));
        count_launches((int64_t)(K + 1) * launches_per_step());
    }
};

// ------------------------------------------------------------- the KPM
// mu_n = (D/R) sum_r <r|T_n(Htilde)|r>  (Moments.jl:42-140) evaluated with
// the doubling identities mu_{2n} = 2<v_n,v_n> - mu_0 and
// mu_{2n+1} = 2<v_{n+1},v_n> - mu_1 per probe (Weisse et al., Rev. Mod. Phys.
// 78, 275 (2006)), i.e. ceil((N-1)/2) block steps instead of N-1, with the
// dot products fused into the step kernel.  Probes are processed in
// power-of-two column blocks of at most 64.
template <typename T>
static std::vector<double> kpm_moments(pf_op *op, double a, double b, int N, int R, const T *probes_cm,
                                       int64_t ldp, int kind, uint64_t seed, int64_t *block_matvecs) {
    pf_handle *h = op->h;
    const int64_t D = op->dim;
    cudaStream_t st = h->stream;
    PF_CHECK(N >= 1 && R >= 1, PF_ERR_INVALID, "KPM needs N >= 1 and R >= 1");
    std::vector<double> mu(N, 0.0);
    const int M = (N - 1 + 1) / 2;  // steps: ceil((N-1)/2)
    const int RB = std::min(64, R);
    DevArray<T> v0((size_t)D * RB), v1((size_t)D * RB);
    DevArray<double> dots((size_t)std::max(M, 1) * 2 * RB), n0(RB), scl(RB);
    std::vector<double> hd((size_t)std::max(M, 1) * 2 * RB), h0(RB), hs(RB);
    int64_t mv = 0;
    int c0 = 0;
    while (c0 < R) {
        int nb = 64;
        while (nb > R - c0) nb /= 2;
        T *prev = v0.p, *cur = v1.p;
        if (probes_cm) {
            launch_cm_to_ri<T, T>(st, D, nb, probes_cm + (size_t)c0 * ldp, ldp, prev);
        } else {
            launch_probes<T>(st, D, nb, kind, seed, c0, prev);
            launch_coldots<T>(h, st, D, nb, prev, prev, n0.p);
            PF_CUDA(cudaMemcpyAsync(h0.data(), n0.p, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
            sync(h);
            for (int c = 0; c < nb; ++c) hs[c] = 1.0 / std::sqrt(h0[c]);
            PF_CUDA(cudaMemcpyAsync(scl.p, hs.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st));
            launch_scale_cols<T>(st, D, nb, prev, scl.p);
        }
        launch_coldots<T>(h, st, D, nb, prev, prev, n0.p);
        if (M >= 1) {
            launch_step<T>(op, st, D, nb, prev, nullptr, nullptr, cur, 0, 1.0, 0, 1.0 / a, b,
                           StepFlags::Q | StepFlags::DOTS, dots.p);
            for (int n = 1; n < M; ++n) {
                launch_step<T>(op, st, D, nb, cur, prev, nullptr, prev, 0, 2.0, -1.0, 1.0 / a, b,
                               StepFlags::Q | StepFlags::P | StepFlags::DOTS, dots.p + (size_t)n * 2 * nb);
                std::swap(prev, cur);
            }
        }
        PF_CUDA(cudaMemcpyAsync(h0.data(), n0.p, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (M >= 1)
            PF_CUDA(cudaMemcpyAsync(hd.data(), dots.p, (size_t)M * 2 * nb * sizeof(double), cudaMemcpyDeviceToHost, st));
        sync(h);
        for (int c = 0; c < nb; ++c) {
            const double m0 = h0[c];
            mu[0] += m0;
            if (M < 1) continue;
            const double m1 = hd[nb + c];  // <v1, v0>
            if (N > 1) mu[1] += m1;
            for (int n = 0; n < M; ++n) {
                const double dd = hd[(size_t)n * 2 * nb + c];
                const double dq = hd[(size_t)n * 2 * nb + nb + c];
                if (2 * n + 2 < N) mu[2 * n + 2] += 2.0 * dd - m0;
                if (n >= 1 && 2 * n + 1 < N) mu[2 * n + 1] += 2.0 * dq - m1;
            }
        }
        mv += (int64_t)nb * M;
        c0 += nb;
    }
    for (double &m : mu) m *= (double)D / (double)R;
    if (block_matvecs) *block_matvecs += mv;
    return mu;
}

// ----------------------------------------------------- small dense helpers
// Cholesky G = R^T R (upper R, column-major s x s).  Returns false on a
// non-positive or negligible pivot.
static bool host_cholesky(const std::vector<double> &G, int s, std::vector<double> &R) {
    R.assign((size_t)s * s, 0.0);
    for (int j = 0; j < s; ++j) {
        double d = G[j + j * s];
        for (int k = 0; k < j; ++k) d -= R[k + j * s] * R[k + j * s];
        if (!(d > 1e-28 * std::max(1.0, std::fabs(G[j + j * s]))) || !std::isfinite(d)) return false;
        if (d <= 1e-13 * std::fabs(G[j + j * s])) return false;
        const double rjj = std::sqrt(d);
        R[j + j * s] = rjj;
        for (int i = j + 1; i < s; ++i) {
            double v = G[j + i * s];
            for (int k = 0; k < j; ++k) v -= R[k + j * s] * R[k + i * s];
            R[j + i * s] = v / rjj;
        }
    }
    return true;
}

// Householder QR of an RI (row-major) D x s block on the host, with the LAPACK
// sign convention (R_jj = -sign(a_jj) ||x||).  Q overwrites A; R is s x s
// column-major.  Used only when CholQR breaks down (a rank-deficient block).
static void host_householder_qr(std::vector<double> &A, int64_t D, int s, std::vector<double> &R) {
    std::vector<std::vector<double>> V(s);
    std::vector<double> tau(s, 0.0);
    for (int j = 0; j < s; ++j) {
        double nrm2 = 0.0;
        for (int64_t i = j; i < D; ++i) nrm2 += A[i * s + j] * A[i * s + j];
        const double alpha = A[j * s + j];
        const double nrm = std::sqrt(nrm2);
        std::vector<double> v(D - j, 0.0);
        if (nrm == 0.0) {
            tau[j] = 0.0;
            V[j] = v;
            continue;
        }
        const double beta = -std::copysign(nrm, alpha);
        v[0] = 1.0;
        for (int64_t i = j + 1; i < D; ++i) v[i - j] = A[i * s + j] / (alpha - beta);
        tau[j] = (beta - alpha) / beta;
        for (int c = j; c < s; ++c) {
            double w = 0.0;
            for (int64_t i = j; i < D; ++i) w += v[i - j] * A[i * s + c];
            w *= tau[j];
            for (int64_t i = j; i < D; ++i) A[i * s + c] -= w * v[i - j];
        }
        V[j] = v;
    }
    R.assign((size_t)s * s, 0.0);
    for (int j = 0; j < s; ++j)
        for (int i = 0; i <= j; ++i) R[i + j * s] = A[(int64_t)i * s + j];
    std::vector<double> Q((size_t)D * s, 0.0);
    for (int j = 0; j < s; ++j) Q[(int64_t)j * s + j] = 1.0;
    for (int j = s - 1; j >= 0; --j) {
        if (tau[j] == 0.0) continue;
        for (int c = 0; c < s; ++c) {
            double w = 0.0;
            for (int64_t i = j; i < D; ++i) w += V[j][i - j] * Q[i * s + c];
            w *= tau[j];
            for (int64_t i = j; i < D; ++i) Q[i * s + c] -= w * V[j][i - j];
        }
    }
    A.swap(Q);
}

// ---------------------------------------------------------- block Lanczos
// Lanczos.jl:119-143, LanczosMethod.jl:55-83, LanczosAlgorithm.jl:11-54,
// Factorization/*, Convergence/* on RI blocks in FP64.  The basis is a
// row-major D x maxdim array; cuBLAS sees it as its column-major transpose.
struct LanczosOut {
    std::vector<double> vals;      // ascending, nconv entries
    DevArray<double> vecs;          // RI D x nconv, same order
    int nconv = 0;
    int numiter = 0, maxiter = 0, krylovdim = 0;
    int converged = 0, eigenconverged = 0;
    double residual = 1.0, eigenresidual = 1.0;
    int numofchecks = 0;
    std::vector<int> conv_hist, dim_hist;
    std::vector<double> res_hist;
    std::vector<double> resid;     // FP64 residual norms of the returned Ritz vectors (before the prefix)
    int refined = 0;               // pairs that met eigentol only after the FP64 refinement
    int qr_restarts = 0;           // restarts with the host QR after a device CholQR breakdown
    LanczosOut() = default;
    LanczosOut(LanczosOut &&) = default;
    LanczosOut &operator=(LanczosOut &&) = default;
};

using BlockMap = std::function<void(const double *X, double *Y)>;  // RI D x s, on h->stream

// The handle's page-locked staging area, at least n doubles.  Growing it
// waits for the handle's stream, so no copy in flight uses the old area.
static double *pinned_scratch(pf_handle *h, size_t n) {
    const size_t bytes = n * sizeof(double);
    if (h->pinned_bytes < bytes) {
        sync(h);
        if (h->pinned) cudaFreeHost(h->pinned);
        h->pinned = nullptr;
        h->pinned_bytes = 0;
        PF_CUDA(cudaMallocHost(&h->pinned, bytes));
        h->pinned_bytes = bytes;
    }
    return static_cast<double *>(h->pinned);
}

// keep_extra >= 0 (the mixed-precision solve): at the final check the
// Ritz vectors of the howmany + keep_extra leading Ritz values (in `which`
// order) are back-transformed, whatever converged, and returned in that order
// with their FP64 Rayleigh quotients and residuals -- no prefix, no sort -- as
// the starting subspace of the FP64 refinement.
// The first nconv of the pairs (vals, RI D x cw vecs), reordered ascending
// (LanczosMethod.jl:74-82); vals and vecs are replaced by the result.
static void ascending_prefix(pf_handle *h, int64_t D, int nconv, std::vector<double> &vals, DevArray<double> &vecs) {
    cudaStream_t st = h->stream;
    std::vector<int> ord(nconv);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return vals[x] < vals[y]; });
    std::vector<double> sv(nconv);
    for (int i = 0; i < nconv; ++i) sv[i] = vals[ord[i]];
    if (nconv > 0) {
        const int cw = (int)(vecs.n / (size_t)D);  // columns of the RI vecs block
        DevArray<double> perm((size_t)D * nconv);
        for (int i = 0; i < nconv; ++i)
            PF_CUDA(cudaMemcpy2DAsync(perm.p + i, nconv * sizeof(double), vecs.p + ord[i], cw * sizeof(double),
                                      sizeof(double), (size_t)D, cudaMemcpyDeviceToDevice, st));
        sync(h);
        std::swap(vecs.p, perm.p);
        std::swap(vecs.n, perm.n);
        std::swap(vecs.st, perm.st);
    }
    vals = sv;
}

// ------------------------------------------ device-side s x s block algebra
// The small dense work of a Lanczos iteration runs in single-CTA kernels on
// the solve's stream, so an iteration makes no host round trip: the host
// reads the device only at convergence checks.

// One CholQR pass for blocks wider than the fused passes take (s > 32):
// small_chol (pf_blocks.cu) factors the Gram matrix with host_cholesky's
// operations in its order, each rounded on its own, so R equals
// host_cholesky's bit for bit, and forms the running product R * rtot_in
// with the host's product loop.  A pivot host_cholesky rejects sets *flag
// and gives R = I (the triangular solve then leaves the block as it is).

// alpha (the overlap V^T W, s x s column-major) made symmetric from its upper
// triangle in place, and written as the diagonal block of T at (k0, k0).
__global__ void k_put_alpha(double *__restrict__ A, int s, double *__restrict__ T, int ldT, int k0) {
    for (int idx = threadIdx.x; idx < s * s; idx += blockDim.x) {
        const int i = idx % s, j = idx / s;
        const double v = i <= j ? A[i + j * s] : A[j + i * s];
        T[(size_t)(k0 + i) + (size_t)(k0 + j) * ldT] = v;
        if (i > j) A[idx] = v;   // only upper entries are read
    }
}

// beta = R (upper, s x s) written as the off-diagonal blocks of T at rows k,
// columns k - s and their transpose, and kept for the next iteration.
__global__ void k_put_beta(const double *__restrict__ R, int s, double *__restrict__ T, int ldT, int k,
                           double *__restrict__ beta) {
    for (int idx = threadIdx.x; idx < s * s; idx += blockDim.x) {
        const int i = idx % s, j = idx / s;
        const double v = R[idx];
        T[(size_t)(k + i) + (size_t)(k - s + j) * ldT] = v;
        T[(size_t)(k - s + j) + (size_t)(k + i) * ldT] = v;
        beta[idx] = v;
    }
}

// Eigenvalues of the symmetric tridiagonal matrix (diagonal d[0..n-1],
// subdiagonal e[0..n-2]) and the last component of each eigenvector, by the
// implicit QL iteration with shifts of tql2 (Bowdler, Martin, Reinsch and
// Wilkinson, Numer. Math. 11, 293 (1968)), carrying only the last row of the
// accumulated rotations.  d is replaced by the eigenvalues (unsorted), z
// receives the matching last components.  Returns false if an eigenvalue
// needs more than 60 iterations.
static bool tridiag_ql_last_row(std::vector<double> &d, std::vector<double> e, std::vector<double> &z) {
    const int n = (int)d.size();
    z.assign(n, 0.0);
    if (n == 0) return true;
    z[n - 1] = 1.0;
    e.resize(n, 0.0);
    e[n - 1] = 0.0;
    const double eps = std::numeric_limits<double>::epsilon();
    for (int l = 0; l < n; ++l) {
        int iter = 0, m;
        do {
            for (m = l; m < n - 1; ++m) {
                const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= eps * dd) break;
            }
            if (m != l) {
                if (iter++ == 60) return false;
                double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                double r = std::sqrt(g * g + 1.0);
                g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
                double sn = 1.0, c = 1.0, p = 0.0;
                int i;
                for (i = m - 1; i >= l; --i) {
                    double f = sn * e[i];
                    const double b = c * e[i];
                    r = std::sqrt(f * f + g * g);
                    e[i + 1] = r;
                    if (r == 0.0) {
                        d[i + 1] -= p;
                        e[m] = 0.0;
                        break;
                    }
                    sn = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * sn + 2.0 * c * b;
                    p = sn * r;
                    d[i + 1] = g + p;
                    g = c * r - b;
                    f = z[i + 1];
                    z[i + 1] = sn * z[i] + c * f;
                    z[i] = c * z[i] - sn * f;
                }
                if (r == 0.0 && i >= l) continue;
                d[l] -= p;
                e[l] = g;
                e[m] = 0.0;
            }
        } while (m != l);
    }
    return true;
}

static pf_handle *aux_handle(pf_handle *h);
static void lanczos_pass(pf_op *op, int s, int howmany, int maxdim_req, double tol, double eigentol, int which,
                         int reorth_passes, const double *x0_ri, const BlockMap &fmap, LanczosOut &out,
                         double *stage_acc, int keep_extra, bool host_qr, bool *breakdown);

// Block Lanczos with the s x s work on the device.  A CholQR pass whose
// Gram matrix is not numerically positive definite (a rank-deficient block)
// needs the host's Householder QR: the device pass flags it, and at its next
// convergence check the solve restarts with the host QR, whose every
// iteration reads the Gram matrix back (the same R bit for bit until the
// breakdown, then the Householder factors).
static void lanczos(pf_op *op, int s, int howmany, int maxdim_req, double tol, double eigentol, int which,
                    int reorth_passes, const double *x0_ri, const BlockMap &fmap, LanczosOut &out,
                    double *stage_acc, int keep_extra = -1, bool host_qr = false) {
    bool breakdown = false;
    // blocks wider than 64 columns (a Gram matrix beyond one CTA's shared
    // memory) always take the host QR
    lanczos_pass(op, s, howmany, maxdim_req, tol, eigentol, which, reorth_passes, x0_ri, fmap, out, stage_acc,
                 keep_extra, host_qr || s > 64, &breakdown);
    if (!breakdown) return;
    LanczosOut again;
    lanczos_pass(op, s, howmany, maxdim_req, tol, eigentol, which, reorth_passes, x0_ri, fmap, again, stage_acc,
                 keep_extra, true, nullptr);
    again.qr_restarts = 1;
    out = std::move(again);
}

static void lanczos_pass(pf_op *op, int s, int howmany, int maxdim_req, double tol, double eigentol, int which,
                         int reorth_passes, const double *x0_ri, const BlockMap &fmap, LanczosOut &out,
                         double *stage_acc, int keep_extra, bool host_qr, bool *breakdown) {
    pf_handle *h = op->h;
    const int64_t D = op->dim;
    cudaStream_t st = h->stream;
    cublasHandle_t blas = h->blas;
    PF_CUBLAS(cublasSetStream(blas, st));
    PF_CUSOLVER(cusolverDnSetStream(h->solver, st));

    const int maxiter = (maxdim_req + s - 1) / s;
    const int maxdim = maxiter * s;
    PF_CHECK(maxdim >= 1, PF_ERR_INVALID, "maxdim must be positive");
    out.maxiter = maxiter;
    int nextcheck = std::max(howmany / s + 1, 2);

    DevArray<double> basis((size_t)D * maxdim);
    DevArray<double> bufs((size_t)D * s * 3);
    double *vlast = bufs.p, *vprev = bufs.p + (size_t)D * s, *r = bufs.p + 2 * (size_t)D * s;
    const size_t ss = (size_t)s * s;
    // small device state: alpha, the pass's R, two running products, beta,
    // the Gram matrix, the breakdown flag
    DevArray<double> small(7 * ss), G((size_t)maxdim * s);
    double *dA = small.p, *dR = dA + ss, *dRt0 = dR + ss, *dRt1 = dRt0 + ss, *dBeta = dRt1 + ss, *dG = dBeta + ss;
    double *dR2 = dG + ss;
    // blocks of up to 32 columns take the fused block passes (pf_blocks.cu)
    const bool fused = s <= kBlkMaxS;
    DevArray<double> bpart(fused ? blk_partial_doubles(D, s) : 0);
    DevArray<unsigned> bcount(fused ? blk_counters() : 0);
    if (fused) PF_CUDA(cudaMemsetAsync(bcount.p, 0, blk_counters() * sizeof(unsigned), st));
    DevArray<int> dflag(1);
    PF_CUDA(cudaMemsetAsync(dflag.p, 0, sizeof(int), st));
    DevArray<double> Tfull((size_t)maxdim * maxdim);   // the projected matrix, column-major
    PF_CUDA(cudaMemsetAsync(Tfull.p, 0, (size_t)maxdim * maxdim * sizeof(double), st));
    PF_CUDA(cudaMemsetAsync(dBeta, 0, ss * sizeof(double), st));
    DevArray<unsigned char> tc_work(reorth_passes == 3 ? gram_bf16_workspace(D, maxdim, s) : 0);
    DevArray<int> tc_err(reorth_passes == 3 ? 1 : 0);
    if (reorth_passes == 3) PF_CUDA(cudaMemsetAsync(tc_err.p, 0, sizeof(int), st));
    std::vector<double> hR;
    const double one = 1.0, zero = 0.0, mone = -1.0;
    const int ldb = maxdim;  // row stride of the basis
    StageClock clk(h, st, stage_acc);
    // page-locked staging for the checks (rewritten only after the sync that
    // follows the copies which last used it)
    double *pin = pinned_scratch(h, 3 * ss + (size_t)maxdim * (s + 3) + 8);
    double *pinG = pin, *pinR = pinG + ss, *pinB = pinR + ss;
    double *pinLam = pinB + ss;                         // maxdim
    double *pinTail = pinLam + maxdim;                  // s x maxdim
    double *pinE = pinTail + (size_t)s * maxdim;        // maxdim
    double *pinRes = pinE + maxdim;                     // maxdim
    int *pinInfo = reinterpret_cast<int *>(pinRes + maxdim);   // [info, breakdown flag]

    auto append = [&](const double *src, int col) {
        PF_CUDA(cudaMemcpy2DAsync(basis.p + col, (size_t)ldb * sizeof(double), src, (size_t)s * sizeof(double),
                                  (size_t)s * sizeof(double), (size_t)D, cudaMemcpyDeviceToDevice, st));
    };
    auto pass_args = [&](double *W) {
        BlkPass p;
        p.D = D;
        p.s = s;
        p.W = W;
        p.partial = bpart.p;
        p.counter = bcount.p;
        p.G = dG;
        p.flag = dflag.p;
        p.T = Tfull.p;
        p.ldT = maxdim;
        return p;
    };
    // alpha = V^T W (s x s), upper triangle symmetrised, into T at (k0, k0)
    auto overlap = [&](const double *Vb, const double *Wb, int k0) {
        if (fused) {
            BlkPass p = pass_args(const_cast<double *>(Vb));
            p.Y = Wb;
            p.flags = BLK_GRAM;
            p.epi = EPI_ALPHA;
            p.k = k0;
            p.keep = dA;
            blk_pass(st, p);
            return;
        }
        PF_CUBLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_T, s, s, (int)D, &one, Vb, s, Wb, s, &zero, dA, s));
        k_put_alpha<<<1, 256, 0, st>>>(dA, s, Tfull.p, maxdim, k0);
        PF_CUDA(cudaGetLastError());
        count_launches(1);
    };
    // r -= vlast alpha + vprev beta^T (orthogonalization.jl:31-33; vprev null:
    // the first iteration, no beta term)
    auto update = [&](double *rb, const double *Vb, const double *Vp) {
        if (fused) {
            blk_update(st, D, s, rb, Vb, Vp, dA, dBeta);
            return;
        }
        PF_CUBLAS(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, s, (int)D, s, &mone, dA, s, Vb, s, &one, rb, s));
        if (Vp)
            PF_CUBLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, s, (int)D, s, &mone, dBeta, s, Vp, s, &one, rb, s));
    };
    // Q R = W in place (CholQR2) on the device; R ends in dRt1.  Fused: Q is
    // also written into the basis at column kcol and beta = R into T.
    auto qr_device = [&](double *W, int kcol) {
        if (fused) {
            BlkPass p = pass_args(W);
            p.flags = BLK_GRAM;
            p.epi = EPI_CHOL;
            p.R = dR;
            p.rtot_out = dRt0;
            blk_pass(st, p);
            p.flags = BLK_SOLVE | BLK_GRAM;
            p.epi = EPI_CHOL_BETA;
            p.Rs = dR;
            p.R = dR2;
            p.rtot_in = dRt0;
            p.rtot_out = dRt1;
            p.k = kcol;
            p.keep = dBeta;
            blk_pass(st, p);
            BlkPass q = pass_args(W);
            q.flags = BLK_SOLVE | BLK_APPEND;
            q.Rs = dR2;
            q.basis = basis.p;
            q.ldb = ldb;
            q.col = kcol;
            blk_pass(st, q);
            return;
        }
        for (int pass = 0; pass < 2; ++pass) {
            PF_CUBLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_T, s, s, (int)D, &one, W, s, W, s, &zero, dG, s));
            small_chol(st, dG, s, dR, pass == 0 ? nullptr : dRt0, pass == 0 ? dRt0 : dRt1, dflag.p);
            // W^T <- R^{-T} W^T  (i.e. W <- W R^{-1})
            PF_CUBLAS(cublasDtrsm(blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, s,
                                  (int)D, &one, dR, s, W, s));
        }
    };
    // Q R = W in place with the Gram matrices read back (CholQR2; Householder
    // on the host if it breaks down); R ends in dRt1.  Returns whether Q was
    // also written into the basis at column kcol (the fused passes).
    auto qr_host = [&](double *W, int kcol) -> bool {
        std::vector<double> Rtot((size_t)s * s, 0.0);
        for (int i = 0; i < s; ++i) Rtot[i + i * s] = 1.0;
        bool ok = true;
        for (int pass = 0; pass < 2 && ok; ++pass) {
            if (fused) {
                // the Gram matrix of W (pass 0) or of W R1^{-1} (pass 1, solved in place)
                BlkPass p = pass_args(W);
                p.flags = pass == 0 ? BLK_GRAM : (BLK_SOLVE | BLK_GRAM);
                p.Rs = dR;
                blk_pass(st, p);
            } else {
                PF_CUBLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_T, s, s, (int)D, &one, W, s, W, s, &zero, dG, s));
            }
            std::vector<double> hG((size_t)s * s), Rp;
            PF_CUDA(cudaMemcpyAsync(pinG, dG, ss * sizeof(double), cudaMemcpyDeviceToHost, st));
            sync(h);
            std::memcpy(hG.data(), pinG, ss * sizeof(double));
            for (int j = 0; j < s; ++j)
                for (int i = j + 1; i < s; ++i) hG[i + j * s] = hG[j + i * s];
            if (!host_cholesky(hG, s, Rp)) { ok = false; break; }
            std::memcpy(pinR, Rp.data(), ss * sizeof(double));
            PF_CUDA(cudaMemcpyAsync(dR, pinR, ss * sizeof(double), cudaMemcpyHostToDevice, st));
            if (!fused)
                PF_CUBLAS(cublasDtrsm(blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT,
                                      s, (int)D, &one, dR, s, W, s));
            // Rtot <- Rp * Rtot
            std::vector<double> Rn((size_t)s * s, 0.0);
            for (int j = 0; j < s; ++j)
                for (int i = 0; i <= j; ++i) {
                    double v = 0.0;
                    for (int k = i; k <= j; ++k) v += Rp[i + k * s] * Rtot[k + j * s];
                    Rn[i + j * s] = v;
                }
            Rtot.swap(Rn);
            sync(h);   // pinR is rewritten by the next pass
        }
        bool appended = false;
        if (ok && fused) {
            // W <- W R2^{-1}, also into the basis
            BlkPass q = pass_args(W);
            q.flags = BLK_SOLVE | BLK_APPEND;
            q.Rs = dR;
            q.basis = basis.p;
            q.ldb = ldb;
            q.col = kcol;
            blk_pass(st, q);
            appended = true;
        }
        if (!ok) {
            std::vector<double> hW((size_t)D * s);
            PF_CUDA(cudaMemcpyAsync(hW.data(), W, hW.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
            sync(h);
            host_householder_qr(hW, D, s, Rtot);
            PF_CUDA(cudaMemcpyAsync(W, hW.data(), hW.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        std::memcpy(pinR, Rtot.data(), ss * sizeof(double));
        PF_CUDA(cudaMemcpyAsync(dRt1, pinR, ss * sizeof(double), cudaMemcpyHostToDevice, st));
        sync(h);
        return appended;
    };

    // ---- lanczositer (Factorization.jl:50-67)
    PF_CUDA(cudaMemcpyAsync(vlast, x0_ri, (size_t)D * s * sizeof(double), cudaMemcpyDeviceToDevice, st));
    PF_CUDA(cudaMemsetAsync(vprev, 0, (size_t)D * s * sizeof(double), st));
    append(vlast, 0);
    int k = s;
    {
        cudaEvent_t e0 = clk.mark();
        fmap(vlast, r);
        clk.add(1, e0, clk.mark());
    }
    overlap(vlast, r, 0);
    // r^T -= alpha^T x0^T
    update(r, vlast, nullptr);
    int numiter = 1;

    // eigen workspace
    DevArray<double> dT((size_t)maxdim * maxdim), dW(maxdim);
    DevArray<int> dinfo(1);
    int lwork = 0;
    PF_CUSOLVER(cusolverDnDsyevd_bufferSize(h->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, maxdim, dT.p,
                                            maxdim, dW.p, &lwork));
    DevArray<double> dwork((size_t)std::max(lwork, 1));

    // A convergence check of the device form runs beside the next iteration:
    // the check reads only T's leading k x k block, beta and the breakdown
    // flag, all copied on the solve's stream before the next iteration is
    // enqueued, and that iteration writes T outside the block and the basis
    // beyond column k.  The next check is at least five iterations later, so
    // the extra iteration is the one that comes next anyway; if the check
    // says stop, it is discarded (the Ritz vectors use columns < k and the
    // check's eigenvectors).  Block solves run the check's dense eigensolver
    // on the auxiliary handle's stream; scalar solves run the host QL while
    // the GPU works.  Every decision is the synchronous form's.
    const bool speculate = !host_qr;
    pf_handle *ah = (speculate && s > 1) ? aux_handle(h) : nullptr;
    cudaEvent_t ev_data = nullptr, ev_eig = nullptr;
    PF_CUDA(cudaEventCreateWithFlags(&ev_data, cudaEventDisableTiming));
    PF_CUDA(cudaEventCreateWithFlags(&ev_eig, cudaEventDisableTiming));
    // destroyed before the work arrays: an exception while a check is in
    // flight on the auxiliary stream waits for it before they are freed
    struct CheckGuard {
        cudaEvent_t data, eig;
        bool aux_pending = false;
        ~CheckGuard() {
            if (aux_pending) cudaEventSynchronize(eig);
            cudaEventDestroy(data);
            cudaEventDestroy(eig);
        }
    } guard{ev_data, ev_eig};

    std::vector<double> lam, tail, beta_last;
    std::vector<int> idx;
    auto order_idx = [&](int kc) {
        idx.resize(kc);
        std::iota(idx.begin(), idx.end(), 0);
        if (which == PF_WHICH_LR)
            std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return lam[x] > lam[y]; });
        else
            std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return lam[x] < lam[y]; });
    };
    // the dense eigensolver on T's leading kc x kc block (upper triangle
    // read) on stream sst with solver handle sol: eigenvalues to pinLam, the
    // last s rows of the eigenvectors to pinTail, eigenvectors kept in dT
    auto enqueue_dense = [&](int kc, cudaStream_t sst, cusolverDnHandle_t sol) {
        PF_CUSOLVER(cusolverDnSetStream(sol, sst));
        PF_CUSOLVER(cusolverDnDsyevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, kc, dT.p, kc, dW.p,
                                     dwork.p, lwork, dinfo.p));
        PF_CUDA(cudaMemcpyAsync(pinLam, dW.p, kc * sizeof(double), cudaMemcpyDeviceToHost, sst));
        PF_CUDA(cudaMemcpy2DAsync(pinTail, s * sizeof(double), dT.p + (kc - s), (size_t)kc * sizeof(double),
                                  s * sizeof(double), kc, cudaMemcpyDeviceToHost, sst));
        PF_CUDA(cudaMemcpyAsync(pinInfo, dinfo.p, sizeof(int), cudaMemcpyDeviceToHost, sst));
    };
    auto copy_block = [&](int kc) {
        PF_CUDA(cudaMemcpy2DAsync(dT.p, (size_t)kc * sizeof(double), Tfull.p, (size_t)maxdim * sizeof(double),
                                  (size_t)kc * sizeof(double), kc, cudaMemcpyDeviceToDevice, st));
    };
    auto take_dense = [&](int kc) {
        PF_CHECK(*pinInfo == 0, PF_ERR_NUMERIC, "projected eigenproblem failed to converge");
        lam.assign(pinLam, pinLam + kc);
        tail.assign(pinTail, pinTail + (size_t)s * kc);
    };
    // the dense eigensolver now, on the solve's stream
    auto dense_sync = [&](int kc) {
        copy_block(kc);
        enqueue_dense(kc, st, h->solver);
        sync(h);
        take_dense(kc);
    };
    // A check of T's leading kc x kc block.  launch: enqueue its inputs (and,
    // for a dense check, the eigensolver: on the auxiliary stream when async).
    struct Check {
        int k = 0, numiter = 0;
        bool tridiag = false, async_dense = false;
    };
    auto launch_check = [&](int kc, int nc, bool async) -> Check {
        Check c;
        c.k = kc;
        c.numiter = nc;
        c.tridiag = s == 1 && kc <= 512;
        if (c.tridiag) {
            // scalar Lanczos: T is tridiagonal -- its diagonal and subdiagonal
            const size_t pitch = (size_t)(maxdim + 1) * sizeof(double);
            PF_CUDA(cudaMemcpy2DAsync(pinLam, sizeof(double), Tfull.p, pitch, sizeof(double), kc,
                                      cudaMemcpyDeviceToHost, st));
            if (kc > 1)
                PF_CUDA(cudaMemcpy2DAsync(pinTail, sizeof(double), Tfull.p + 1, pitch, sizeof(double), kc - 1,
                                          cudaMemcpyDeviceToHost, st));
        } else {
            copy_block(kc);
        }
        PF_CUDA(cudaMemcpyAsync(pinB, dBeta, ss * sizeof(double), cudaMemcpyDeviceToHost, st));
        PF_CUDA(cudaMemcpyAsync(pinInfo + 1, dflag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        PF_CUDA(cudaEventRecord(ev_data, st));
        if (!c.tridiag) {
            if (async && ah) {
                PF_CUDA(cudaStreamWaitEvent(ah->stream, ev_data, 0));
                enqueue_dense(kc, ah->stream, ah->solver);
                PF_CUDA(cudaEventRecord(ev_eig, ah->stream));
                c.async_dense = true;
                guard.aux_pending = true;
            } else {
                enqueue_dense(kc, st, h->solver);
                PF_CUDA(cudaEventRecord(ev_eig, st));
            }
        }
        return c;
    };
    // finish: wait for the check's data, decide (ConvergenceInfo.jl:63-130).
    // Returns 0 continue, 1 stop, 2 a device CholQR pass broke down.
    auto finish_check = [&](const Check &c) -> int {
        if (!c.tridiag) {
            PF_CUDA(cudaEventSynchronize(ev_eig));
            guard.aux_pending = false;
        }
        PF_CUDA(cudaEventSynchronize(ev_data));
        if (pinInfo[1] != 0) {
            PF_CHECK(breakdown != nullptr, PF_ERR_NUMERIC, "CholQR breakdown in the host-QR pass");
            return 2;
        }
        beta_last.assign(pinB, pinB + ss);
        bool have = false;
        if (c.tridiag) {
            lam.assign(pinLam, pinLam + c.k);
            std::vector<double> sub(pinTail, pinTail + std::max(c.k - 1, 0));
            have = tridiag_ql_last_row(lam, sub, tail);
            if (!have) dense_sync(c.k);
        } else {
            take_dense(c.k);
        }
        order_idx(c.k);
        int conv = 0;
        double maxres = 0.0;
        const int nwant = std::min(howmany, c.k);
        for (int i = 0; i < nwant; ++i) {
            const int pos = idx[i];
            double ss2 = 0.0;
            for (int a = 0; a < s; ++a) {
                double v = 0.0;
                for (int b2 = 0; b2 < s; ++b2) v += beta_last[a + b2 * s] * tail[b2 + (size_t)pos * s];
                ss2 += v * v;
            }
            const double res = std::sqrt(ss2);
            if (res > maxres || std::isnan(res)) maxres = std::isnan(res) ? res : std::max(maxres, res);
            if (maxres < tol) ++conv;
        }
        out.numofchecks += 1;
        out.converged = conv;
        out.residual = maxres;
        out.conv_hist.push_back(conv);
        out.dim_hist.push_back(c.k);
        out.res_hist.push_back(maxres);
        // next_checking! (NextChecking.jl:23-42)
        if (out.residual > 1e-2) nextcheck = c.numiter + 20;
        else if (out.residual > 1e-3) nextcheck = c.numiter + 10;
        else nextcheck = c.numiter + 5;
        if (!(conv == howmany || c.numiter >= maxiter)) return 0;
        if (c.tridiag && have) {
            // the Ritz vectors need the eigenvectors: the dense solver, re-ordered
            dense_sync(c.k);
            order_idx(c.k);
        }
        return 1;
    };
    // calculate_eigenvectors! (getvecs.jl:10-21): Psi = B Phi[:, idx[1:conv]]
    // for the stopping check of dimension kc
    auto extract = [&](int kc) {
        int conv = out.converged;
        if (keep_extra >= 0) conv = std::min(kc, howmany + keep_extra);
        out.vecs.alloc((size_t)D * std::max(conv, 1));
        if (conv > 0) {
            DevArray<double> phisel((size_t)kc * conv);
            for (int i = 0; i < conv; ++i)
                PF_CUDA(cudaMemcpyAsync(phisel.p + (size_t)i * kc, dT.p + (size_t)idx[i] * kc, kc * sizeof(double),
                                        cudaMemcpyDeviceToDevice, st));
            PF_CUBLAS(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, conv, (int)D, kc, &one, phisel.p, kc, basis.p, ldb,
                                  &zero, out.vecs.p, conv));
            // calculate_eigenvalues! / calculate_eigenresiduals! with the ORIGINAL H
            DevArray<double> HV((size_t)D * conv), E(conv), res2(conv);
            launch_step<double>(op, st, D, conv, out.vecs.p, nullptr, nullptr, HV.p, 0, 1.0, 0, 1.0, 0.0,
                                StepFlags::Q, nullptr);
            launch_coldots<double>(h, st, D, conv, out.vecs.p, HV.p, E.p);
            launch_colresid(h, st, D, conv, HV.p, out.vecs.p, E.p, res2.p);
            PF_CUDA(cudaMemcpyAsync(pinE, E.p, conv * sizeof(double), cudaMemcpyDeviceToHost, st));
            PF_CUDA(cudaMemcpyAsync(pinRes, res2.p, conv * sizeof(double), cudaMemcpyDeviceToHost, st));
            sync(h);
            std::vector<double> hE(pinE, pinE + conv), hr(pinRes, pinRes + conv);
            int ec = 0;
            bool counting = true;
            double maxe = 0.0;
            out.resid.assign(conv, 0.0);
            for (int i = 0; i < conv; ++i) {
                const double rr = std::sqrt(std::max(hr[i], 0.0));
                out.resid[i] = rr;
                if (counting && rr < eigentol) ++ec;
                else counting = false;
                maxe = std::max(maxe, rr);
            }
            out.vals = hE;
            out.eigenconverged = ec;
            out.eigenresidual = maxe;
        } else {
            out.vals.clear();
            out.eigenconverged = 0;
            out.eigenresidual = 0.0;
        }
    };

    out.converged = 0;
    out.eigenconverged = 0;
    Check pending;
    bool have_pending = false;
    while (true) {
        // 1 tridiagonalization: QR(r) -> beta (BlockLanczosFactorization.jl:115-131)
        cudaEvent_t e0 = clk.mark();
        bool appended = false;
        if (host_qr || !fused) {
            if (host_qr) appended = qr_host(r, k);
            else qr_device(r, k);
            k_put_beta<<<1, 256, 0, st>>>(dRt1, s, Tfull.p, maxdim, k, dBeta);
            PF_CUDA(cudaGetLastError());
            count_launches(1);
        } else {
            qr_device(r, k);   // beta into T and Q into the basis in its passes
            appended = true;
        }
        std::swap(vprev, vlast);
        std::swap(vlast, r);  // vlast <- Q ; r <- old vprev storage
        if (!appended) append(vlast, k);
        k += s;
        cudaEvent_t e1 = clk.mark();
        clk.add(0, e0, e1);
        // 2 mapping
        fmap(vlast, r);
        cudaEvent_t e2 = clk.mark();
        clk.add(1, e1, e2);
        // 3 overlap
        overlap(vlast, r, k - s);
        cudaEvent_t e3 = clk.mark();
        clk.add(2, e2, e3);
        // 4 orthogonalization: r -= vlast alpha + vprev beta^T  (orthogonalization.jl:31-33)
        update(r, vlast, vprev);
        cudaEvent_t e4 = clk.mark();
        clk.add(3, e3, e4);
        // 5 reorthogonalization: r -= B (B^T r), B = all but the last two blocks
        // (reorth_passes 3: CGS2 whose first Gram product runs on the tensor
        // cores in split BF16, the second in FP64)
        const int nB = k - 2 * s;
        if (nB > 0) {
            const int passes = reorth_passes == 3 ? 2 : reorth_passes;
            for (int pass = 0; pass < passes; ++pass) {
                if (reorth_passes == 3 && pass == 0)
                    gram_bf16x3(h, st, D, nB, basis.p, ldb, r, s, G.p, tc_work.p, tc_err.p);
                else
                    PF_CUBLAS(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_T, nB, s, (int)D, &one, basis.p, ldb, r, s,
                                          &zero, G.p, nB));
                PF_CUBLAS(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, s, (int)D, nB, &mone, G.p, nB, basis.p, ldb, &one,
                                      r, s));
            }
        }
        cudaEvent_t e5 = clk.mark();
        clk.add(4, e4, e5);

        numiter += 1;
        // the previous iteration's check, which ran beside this iteration
        if (have_pending) {
            have_pending = false;
            const int verdict = finish_check(pending);
            if (verdict == 2) {
                *breakdown = true;
                break;
            }
            if (verdict == 1) {
                k = pending.k;            // this iteration is discarded
                numiter = pending.numiter;
                extract(k);
                cudaEvent_t e6 = clk.mark();
                clk.add(5, e5, e6);
                break;
            }
        }
        // convergence (ConvergenceInfo.jl:63-130)
        if (nextcheck == numiter || numiter >= maxiter) {
            const bool async = speculate && numiter < maxiter;
            const Check c = launch_check(k, numiter, async);
            cudaEvent_t e6 = clk.mark();
            clk.add(5, e5, e6);
            if (async) {
                pending = c;
                have_pending = true;
                continue;
            }
            const int verdict = finish_check(c);
            if (verdict == 2) {
                *breakdown = true;
                break;
            }
            if (verdict == 1) {
                extract(k);
                cudaEvent_t e7 = clk.mark();
                clk.add(5, e6, e7);
                break;
            }
        }
    }
    if (breakdown && *breakdown) {
        sync(h);
        clk.flush();
        return;
    }
    sync(h);
    clk.flush();
    if (reorth_passes == 3) {
        int e = 0;
        PF_CUDA(cudaMemcpy(&e, tc_err.p, sizeof(int), cudaMemcpyDeviceToHost));
        PF_CHECK(e == 0, PF_ERR_CUDA, "the tensor-core Gram product gave up waiting for its MMAs");
    }
    out.numiter = numiter;
    out.krylovdim = k;
    if (keep_extra >= 0) {
        out.nconv = (int)(out.vecs.n / (size_t)D);
        if (out.vals.empty()) out.nconv = 0;
        return;   // the refinement takes the vectors as they are
    }
    // LanczosMethod.jl:74-82: keep the converged prefix, ascending order
    ascending_prefix(h, D, std::min(out.converged, out.eigenconverged), out.vals, out.vecs);
    out.nconv = (int)out.vals.size();
}

// ------------------------------------------------- FP64 refinement (mixed)
// Q R = W in place for an RI D x m block (CholQR2, Householder on the host
// if the Gram matrix is not numerically positive definite).
static void cholqr2_block(pf_handle *h, double *W, int64_t D, int m) {
    cudaStream_t st = h->stream;
    const double one = 1.0, zero = 0.0;
    DevArray<double> Gd((size_t)m * m), Rd((size_t)m * m);
    std::vector<double> G((size_t)m * m), R;
    for (int pass = 0; pass < 2; ++pass) {
        PF_CUBLAS(cublasDgemm(h->blas, CUBLAS_OP_N, CUBLAS_OP_T, m, m, (int)D, &one, W, m, W, m, &zero, Gd.p, m));
        double *pin = pinned_scratch(h, (size_t)m * m);
        PF_CUDA(cudaMemcpyAsync(pin, Gd.p, (size_t)m * m * sizeof(double), cudaMemcpyDeviceToHost, st));
        sync(h);
        std::memcpy(G.data(), pin, (size_t)m * m * sizeof(double));
        for (int j = 0; j < m; ++j)
            for (int i = j + 1; i < m; ++i) G[i + (size_t)j * m] = G[j + (size_t)i * m];
        if (!host_cholesky(G, m, R)) {
            std::vector<double> hW((size_t)D * m), Rh;
            PF_CUDA(cudaMemcpyAsync(hW.data(), W, hW.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
            sync(h);
            host_householder_qr(hW, D, m, Rh);
            PF_CUDA(cudaMemcpyAsync(W, hW.data(), hW.size() * sizeof(double), cudaMemcpyHostToDevice, st));
            sync(h);
            return;
        }
        std::memcpy(pin, R.data(), (size_t)m * m * sizeof(double));
        PF_CUDA(cudaMemcpyAsync(Rd.p, pin, (size_t)m * m * sizeof(double), cudaMemcpyHostToDevice, st));
        PF_CUBLAS(cublasDtrsm(h->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, m,
                              (int)D, &one, Rd.p, m, W, m));
        sync(h);   // the staging area is rewritten by the next pass
    }
}

// The mixed-precision solve's FP64 refinement.  An FP32 filter perturbs every
// Krylov block by ~1e-7 relative, so the Ritz vectors of the FP32 run stop
// near 1e-5 in FP64 residual: their error is spread over the whole spectrum,
// mostly far from the target window.  Each pass applies the FP64 filter to the
// current vectors (damping every component by its filter value), orthonormalises
// them, and runs a Rayleigh-Ritz step with the FP64 Hamiltonian on that
// subspace, which also undoes the mixing among the window's own eigenvectors.
// The subspace keeps m = nev + guard vectors; the nev of largest filter value
// are the targets (the order of the Lanczos selection, which = LR on the
// filter), the guards the next in |filter value|.  Each pass damps a target's
// error along an eigenvector outside the subspace by the ratio of their
// filter values.  Passes stop once the whole target prefix meets eigentol.
// Returns the number of passes run.
static int refine_fp64(pf_op *op, const std::vector<double> &coeffs, double a, double b, int nev, double eigentol,
                       int max_passes, DevArray<double> &Psi, int m, std::vector<double> &vals,
                       std::vector<double> &resid) {
    pf_handle *h = op->h;
    cudaStream_t st = h->stream;
    const int64_t D = op->dim;
    const int K = (int)coeffs.size() - 1;
    const double one = 1.0, zero = 0.0;
    auto filter_value = [&](double E) { return cheb_clenshaw(coeffs.data(), K, (E - b) / a); };
    DevArray<double> W((size_t)D * m), HW((size_t)D * m), Gd((size_t)m * m), Wd(m), HPsi((size_t)D * m), r2(m), ev(m);
    DevArray<int> dinfo(1);
    int lwork = 0;
    PF_CUSOLVER(cusolverDnDsyevd_bufferSize(h->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, m, Gd.p, m,
                                            Wd.p, &lwork));
    DevArray<double> dwork((size_t)std::max(lwork, 1));
    std::map<int, std::unique_ptr<Filter<double>>> filters;   // by column-chunk width
    const int wmax = 32;
    int passes = 0;
    for (int pass = 0; pass < max_passes; ++pass) {
        int ok = 0;
        while (ok < nev && ok < (int)resid.size() && resid[ok] < eigentol) ++ok;
        if (ok >= nev) break;
        ++passes;
        // W = P(Htilde) Psi, chunks of up to 32 columns through graph-captured filters
        for (int c0 = 0; c0 < m; c0 += wmax) {
            const int wc = std::min(wmax, m - c0);
            auto &f = filters[wc];
            if (!f) f.reset(new Filter<double>(op, wc, coeffs, a, b));
            PF_CUDA(cudaMemcpy2DAsync(f->X.p, (size_t)wc * sizeof(double), Psi.p + c0, (size_t)m * sizeof(double),
                                      (size_t)wc * sizeof(double), (size_t)D, cudaMemcpyDeviceToDevice, st));
            f->run(st);
            PF_CUDA(cudaMemcpy2DAsync(W.p + c0, (size_t)m * sizeof(double), f->Y.p, (size_t)wc * sizeof(double),
                                      (size_t)wc * sizeof(double), (size_t)D, cudaMemcpyDeviceToDevice, st));
        }
        cholqr2_block(h, W.p, D, m);
        // Rayleigh-Ritz with the FP64 Hamiltonian: G = W^T H W
        launch_step<double>(op, st, D, m, W.p, nullptr, nullptr, HW.p, 0, 1.0, 0, 1.0, 0.0, StepFlags::Q, nullptr);
        PF_CUBLAS(cublasDgemm(h->blas, CUBLAS_OP_N, CUBLAS_OP_T, m, m, (int)D, &one, W.p, m, HW.p, m, &zero, Gd.p, m));
        PF_CUSOLVER(cusolverDnDsyevd(h->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, m, Gd.p, m, Wd.p,
                                     dwork.p, lwork, dinfo.p));
        double *pin = pinned_scratch(h, (size_t)m + 1);
        PF_CUDA(cudaMemcpyAsync(pin, Wd.p, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, st));
        PF_CUDA(cudaMemcpyAsync(reinterpret_cast<int *>(pin + m), dinfo.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        sync(h);
        std::vector<double> theta(pin, pin + m);
        PF_CHECK(*reinterpret_cast<int *>(pin + m) == 0, PF_ERR_NUMERIC, "refinement eigenproblem failed to converge");
        // the nev targets: the Ritz pairs of largest filter value (the Lanczos
        // selection); the guards after them: the rest in decreasing |filter
        // value|, so the filter's negative side lobes, which damp as slowly as
        // the window's edge, are kept in the subspace and resolved by the
        // Rayleigh-Ritz step instead of polluting the targets
        std::vector<int> idx(m);
        std::iota(idx.begin(), idx.end(), 0);
        std::stable_sort(idx.begin(), idx.end(),
                         [&](int x, int y) { return filter_value(theta[x]) > filter_value(theta[y]); });
        std::stable_sort(idx.begin() + std::min(nev, m), idx.end(), [&](int x, int y) {
            return std::fabs(filter_value(theta[x])) > std::fabs(filter_value(theta[y]));
        });
        DevArray<double> Ysel((size_t)m * m);
        for (int i = 0; i < m; ++i)
            PF_CUDA(cudaMemcpyAsync(Ysel.p + (size_t)i * m, Gd.p + (size_t)idx[i] * m, m * sizeof(double),
                                    cudaMemcpyDeviceToDevice, st));
        // Psi = W Y, H Psi = (H W) Y (RI blocks: cuBLAS sees their column-major transposes)
        PF_CUBLAS(cublasDgemm(h->blas, CUBLAS_OP_T, CUBLAS_OP_N, m, (int)D, m, &one, Ysel.p, m, W.p, m, &zero, Psi.p, m));
        PF_CUBLAS(cublasDgemm(h->blas, CUBLAS_OP_T, CUBLAS_OP_N, m, (int)D, m, &one, Ysel.p, m, HW.p, m, &zero, HPsi.p,
                              m));
        vals.resize(m);
        for (int i = 0; i < m; ++i) vals[i] = theta[idx[i]];
        double *pe = pinned_scratch(h, 2 * (size_t)m);
        std::memcpy(pe, vals.data(), m * sizeof(double));
        PF_CUDA(cudaMemcpyAsync(ev.p, pe, m * sizeof(double), cudaMemcpyHostToDevice, st));
        launch_colresid(h, st, D, m, HPsi.p, Psi.p, ev.p, r2.p);
        PF_CUDA(cudaMemcpyAsync(pe + m, r2.p, m * sizeof(double), cudaMemcpyDeviceToHost, st));
        sync(h);
        resid.resize(m);
        for (int i = 0; i < m; ++i) resid[i] = std::sqrt(std::max(pe[m + i], 0.0));
    }
    return passes;
}

// ------------------------------------------------------------- extrema
// Emin / Emax by two scalar Lanczos probes on H (Plan.jl:136-168,
// Lanczos.jl:183-212): which = :SR then :LR, howmany 1, tol 1e-14,
// eigentol 1e-8 (the lanczos() defaults), mapvals = H.
static pf_handle *aux_handle(pf_handle *h) {
    std::lock_guard<std::mutex> lock(h->aux_mu);
    if (!h->aux) {
        pf_handle *a = nullptr;
        const int saved = t_new_handle_priority;
        t_new_handle_priority = h->priority;   // the probes run as urgently as their solve
        const int st = pf_handle_create(h->device, &a);
        t_new_handle_priority = saved;
        if (st != PF_OK) throw Error(PF_ERR_CUDA, pf_last_error());
        h->aux = a;
    }
    return h->aux;
}

static void extrema_from_device(pf_op *op, const double *v0_dev, int maxdim, double tol, double eigentol, double *Emin,
                                double *Emax, int *qr_restarts = nullptr, bool host_qr = false) {
    const int64_t D = op->dim;
    // The :SR probe runs here and the :LR probe at the same time on the
    // auxiliary handle (its own stream, cuBLAS and cuSOLVER): both only read
    // v0, so each gives exactly what it gives alone.
    pf_handle *ah = aux_handle(op->h);
    std::unique_ptr<pf_op, void (*)(pf_op *)> view(bind_op(op, ah), destroy_op);
    cudaEvent_t ready = nullptr;
    PF_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    PF_CUDA(cudaEventRecord(ready, op->h->stream));
    PF_CUDA(cudaStreamWaitEvent(ah->stream, ready, 0));
    auto probe = [&](pf_op *o, int which, double *out) -> int {
        BlockMap happly = [&](const double *X, double *Y) {
            launch_step<double>(o, o->h->stream, D, 1, X, nullptr, nullptr, Y, 0, 1.0, 0, 1.0, 0.0, StepFlags::Q,
                                nullptr);
        };
        LanczosOut lo;
        lanczos(o, 1, 1, maxdim, tol, eigentol, which, 1, v0_dev, happly, lo, nullptr, -1, host_qr);
        PF_CHECK(lo.nconv >= 1, PF_ERR_NUMERIC, "Failed to estimate extremal eigenvalue with Lanczos.");
        *out = which == PF_WHICH_SR ? lo.vals.front() : lo.vals.back();
        return lo.qr_restarts;
    };
    std::atomic<int> restarts{0};
    std::exception_ptr aux_err;
    int64_t aux_launches = 0;
    double hi = 0.0;
    std::thread t([&] {
        try {
            PF_CUDA(cudaSetDevice(ah->device));
            AllocStream guard(ah->stream);
            const int64_t before = thread_launches();
            restarts += probe(view.get(), PF_WHICH_LR, &hi);
            aux_launches = thread_launches() - before;
        } catch (...) {
            aux_err = std::current_exception();
        }
    });
    std::exception_ptr err;
    double lo = 0.0;
    try {
        restarts += probe(op, PF_WHICH_SR, &lo);
    } catch (...) {
        err = std::current_exception();
    }
    t.join();
    cudaEventDestroy(ready);
    count_launches(aux_launches);
    if (err) std::rethrow_exception(err);
    if (aux_err) std::rethrow_exception(aux_err);
    *Emin = lo;
    *Emax = hi;
    if (qr_restarts) *qr_restarts += restarts.load();
}

void lanczos_extrema(pf_op *op, const double *x0_host, int maxdim, double tol, double eigentol, double *Emin,
                     double *Emax) {
    PF_CHECK(x0_host && Emin && Emax, PF_ERR_INVALID, "null argument");
    const int64_t D = op->dim;
    std::vector<double> seed(x0_host, x0_host + D);
    double nrm = 0.0;
    for (double v : seed) nrm += v * v;
    nrm = std::sqrt(nrm);
    PF_CHECK(nrm > 0 && std::isfinite(nrm), PF_ERR_INVALID, "lanczos_extrema requires a nonzero starting vector.");
    for (double &v : seed) v /= nrm;
    PF_CUDA(cudaSetDevice(op->h->device));
    AllocStream alloc_guard(op->h->stream);
    DevArray<double> v0(D);
    PF_CUDA(cudaMemcpyAsync(v0.p, seed.data(), D * sizeof(double), cudaMemcpyHostToDevice, op->h->stream));
    extrema_from_device(op, v0.p, maxdim, tol, eigentol, Emin, Emax);
}

// ------------------------------------------- op-level tensor-core Gram product
void op_gram_bf16x3(pf_handle *h, int64_t D, int nB, const double *B, int64_t ldb, const double *r, int s, double *G) {
    PF_CHECK(h && B && r && G, PF_ERR_INVALID, "null argument");
    PF_CHECK(D >= 1 && nB >= 1 && ldb >= nB && ldb < (1ll << 31), PF_ERR_INVALID, "invalid Gram product shape");
    PF_CUDA(cudaSetDevice(h->device));
    AllocStream alloc_guard(h->stream);
    DevArray<unsigned char> work(gram_bf16_workspace(D, nB, s));
    DevArray<int> err(1);
    PF_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), h->stream));
    gram_bf16x3(h, h->stream, D, nB, B, (int)ldb, r, s, G, work.p, err.p);
    int e = 0;
    PF_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    sync(h);
    PF_CHECK(e == 0, PF_ERR_CUDA, "the tensor-core Gram product gave up waiting for its MMAs");
}

// ------------------------------------------------------- op-level filter
void op_filter(pf_op *op, int dtype, double a, double b, int K, const double *coeffs, int s, const void *X,
               int64_t ldx, void *Y, int64_t ldy) {
    PF_CHECK(coeffs && X && Y && K >= 0 && s >= 1, PF_ERR_INVALID, "invalid filter arguments");
    PF_CHECK(ldx >= op->dim && ldy >= op->dim, PF_ERR_INVALID, "leading dimension smaller than D");
    PF_CHECK(a != 0.0 && std::isfinite(a) && std::isfinite(b), PF_ERR_INVALID, "rescaling a must be finite and nonzero");
    PF_CUDA(cudaSetDevice(op->h->device));
    AllocStream alloc_guard(op->h->stream);
    std::vector<double> c(coeffs, coeffs + K + 1);
    cudaStream_t st = op->h->stream;
    const int64_t D = op->dim;
    if (dtype == PF_F64) {
        Filter<double> f(op, s, c, a, b);
        launch_cm_to_ri<double, double>(st, D, s, (const double *)X, ldx, f.X.p);
        f.enqueue(st);
        launch_ri_to_cm<double, double>(st, D, s, f.Y.p, (double *)Y, ldy);
        sync(op->h);
    } else if (dtype == PF_F32) {
        Filter<float> f(op, s, c, a, b);
        launch_cm_to_ri<float, float>(st, D, s, (const float *)X, ldx, f.X.p);
        f.enqueue(st);
        launch_ri_to_cm<float, float>(st, D, s, f.Y.p, (float *)Y, ldy);
        sync(op->h);
    } else throw Error(PF_ERR_INVALID, "dtype must be PF_F64 or PF_F32");
}

void op_kpm(pf_op *op, int dtype, double a, double b, int N, int R, const void *probes, int64_t ldp, int probe_kind,
            uint64_t seed, double *mu) {
    PF_CHECK(mu && N >= 1 && R >= 1, PF_ERR_INVALID, "invalid KPM arguments");
    PF_CHECK(!probes || ldp >= op->dim, PF_ERR_INVALID, "probe leading dimension smaller than D");
    PF_CHECK(a != 0.0 && std::isfinite(a) && std::isfinite(b), PF_ERR_INVALID, "rescaling a must be finite and nonzero");
    PF_CHECK(probe_kind == PF_PROBE_GAUSSIAN || probe_kind == PF_PROBE_RADEMACHER, PF_ERR_INVALID, "unknown probe kind");
    PF_CUDA(cudaSetDevice(op->h->device));
    AllocStream alloc_guard(op->h->stream);
    std::vector<double> m;
    if (dtype == PF_F64) m = kpm_moments<double>(op, a, b, N, R, (const double *)probes, ldp, probe_kind, seed, nullptr);
    else if (dtype == PF_F32) m = kpm_moments<float>(op, a, b, N, R, (const float *)probes, ldp, probe_kind, seed, nullptr);
    else throw Error(PF_ERR_INVALID, "dtype must be PF_F64 or PF_F32");
    std::copy(m.begin(), m.end(), mu);
}

// ------------------------------------------------------------- the solve
// Columns per thread of the engine's multi-instance step: the operator's tuned
// per-thread width (the warp-cooperative variant has no multi-instance form).
static int engine_width(pf_op *op, int s, int elem) {
    int V = default_width(s, elem);
    std::lock_guard<std::mutex> lock(op->tune_mu);
    auto it = op->tuned_width.find(std::make_pair(elem, s));
    if (it != op->tuned_width.end() && it->second != kCoopWidth) V = variant_width(it->second);
    return V;
}

static int64_t expected_krylov_dim(int howmany, int s, double eta) {
    return (int64_t)std::ceil((20.427 * s + 1.696 * howmany) * eta);  // PolfedDefaults.jl:61-62
}

// _prepare_polfed_initial_state (PolfedCore.jl:43-95) on a host D x s column-major copy.
static void prepare_initial_state(std::vector<double> &x, int64_t D, int s) {
    const double tol = std::max(1e-10, 10 * 2.220446049250313e-16);
    for (double v : x) PF_CHECK(std::isfinite(v), PF_ERR_INVALID, "POLFED initial state must contain finite values.");
    if (s == 1) {
        double nrm = 0.0;
        for (double v : x) nrm += v * v;
        nrm = std::sqrt(nrm);
        PF_CHECK(nrm != 0.0, PF_ERR_INVALID, "POLFED initial vector must be nonzero.");
        if (std::fabs(nrm - 1.0) <= std::max(tol, tol * std::max(nrm, 1.0))) return;
        for (double &v : x) v /= nrm;
        return;
    }
    PF_CHECK(s <= D, PF_ERR_INVALID,
             "POLFED initial matrix cannot have orthonormal columns when it has more columns than rows.");
    std::vector<double> G((size_t)s * s, 0.0);
    for (int i = 0; i < s; ++i)
        for (int j = 0; j < s; ++j) {
            double v = 0.0;
            for (int64_t r = 0; r < D; ++r) v += x[r + i * D] * x[r + j * D];
            G[i + j * s] = v;
        }
    double dn = 0.0, gn = 0.0;
    for (int i = 0; i < s; ++i)
        for (int j = 0; j < s; ++j) {
            const double e = G[i + j * s] - (i == j ? 1.0 : 0.0);
            dn += e * e;
            gn += G[i + j * s] * G[i + j * s];
        }
    if (std::sqrt(dn) <= std::max(tol, tol * std::max(std::sqrt(gn), std::sqrt((double)s)))) return;
    // orthonormalised copy: thin Q of a Householder QR (as Matrix(qr(x0).Q)[:, 1:s])
    std::vector<double> A((size_t)D * s);
    for (int64_t r = 0; r < D; ++r)
        for (int c = 0; c < s; ++c) A[r * s + c] = x[r + c * D];
    std::vector<double> R;
    host_householder_qr(A, D, s, R);
    for (int64_t r = 0; r < D; ++r)
        for (int c = 0; c < s; ++c) x[r + c * D] = A[r * s + c];
}

void solve(pf_op *op, const pf_params *P, int s, int nev, const double *x0, int x0_mem, double *vals, double *vecs,
           int vecs_mem, pf_report *rep, int *nconv) {
    PF_CHECK(op && P && x0 && vals && nconv, PF_ERR_INVALID, "null argument");
    PF_CHECK(s >= 1 && nev >= 1, PF_ERR_INVALID, "s and nev must be positive");
    PF_CHECK(P->precision == PF_PREC_FP64 || P->precision == PF_PREC_MIXED, PF_ERR_INVALID, "unknown precision");
    PF_CHECK(P->reorth_passes >= 1 && P->reorth_passes <= 3, PF_ERR_INVALID, "reorth_passes must be 1, 2 or 3");
    PF_CHECK(P->reorth_passes != 3 || s <= 32, PF_ERR_UNSUPPORTED,
             "the tensor-core reorthogonalisation (reorth_passes 3) needs s <= 32");
    pf_handle *h = op->h;
    PF_CUDA(cudaSetDevice(h->device));
    AllocStream alloc_guard(h->stream);
    cudaStream_t st = h->stream;
    const int64_t D = op->dim;
    PF_CHECK(s <= D, PF_ERR_INVALID,
             "POLFED initial matrix cannot have orthonormal columns when it has more columns than rows.");
    pf_report R;
    std::memset(&R, 0, sizeof(R));
    const int64_t launches0 = thread_launches();
    cudaEvent_t t_begin, t_end;
    PF_CUDA(cudaEventCreate(&t_begin));
    PF_CUDA(cudaEventCreate(&t_end));
    PF_CUDA(cudaEventRecord(t_begin, st));
    auto t_wall0 = std::chrono::steady_clock::now();

    // x0 -> host column-major, validate / orthonormalise, -> device RI
    std::vector<double> hx((size_t)D * s);
    if (x0_mem == PF_MEM_DEVICE)
    {
        PF_CUDA(cudaMemcpyAsync(hx.data(), x0, hx.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        sync(h);
    }
    else std::memcpy(hx.data(), x0, hx.size() * sizeof(double));
    prepare_initial_state(hx, D, s);
    DevArray<double> xcm((size_t)D * s), xri((size_t)D * s);
    PF_CUDA(cudaMemcpyAsync(xcm.p, hx.data(), hx.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    launch_cm_to_ri<double, double>(st, D, s, xcm.p, D, xri.p);

    // mapping plan (Plan.jl:128-191)
    double Emin = P->Emin, Emax = P->Emax;
    {
        auto w0 = std::chrono::steady_clock::now();
        if (!P->has_Emin || !P->has_Emax) {
            double lo = 0, hi = 0;
            // v0 = x0[:, 1] (column 0 of the column-major copy)
            extrema_from_device(op, xcm.p, P->extrema_maxdim > 0 ? P->extrema_maxdim : 1000, 1e-14, 1e-8, &lo, &hi,
                                &R.qr_restarts, P->host_qr != 0);
            if (!P->has_Emin) Emin = lo;
            if (!P->has_Emax) Emax = hi;
        }
        sync(h);
        R.stage_seconds[6] = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
    }
    const double a = (Emax - Emin) / 2, b = (Emax + Emin) / 2;
    PF_CHECK(a > 0 && std::isfinite(a) && std::isfinite(b), PF_ERR_NUMERIC, "degenerate spectral range Emax <= Emin");

    // transform plan (Plan.jl:203-236)
    TransformState t;
    t.target_kind = P->target_kind;
    t.target_value = P->target_value;
    t.a = a;
    t.b = b;
    t.howmany = nev;
    t.cutoff = P->cutoff;
    t.normalization = P->normalization;
    t.order_safety_factor = P->order_safety_factor;
    t.order = P->order;
    t.has_left = P->has_left != 0;
    t.has_right = P->has_right != 0;
    if (t.has_left) t.left = (P->left - b) / a;
    if (t.has_right) t.right = (P->right - b) / a;
    if (t.target_kind == PF_TARGET_UNRESCALED) { t.target = (t.target_value - b) / a; t.has_target = true; }
    else if (t.target_kind == PF_TARGET_RESCALED) { t.target = t.target_value; t.has_target = true; }
    else if (t.target_kind == PF_TARGET_MIDDLE) { t.target = 0.0; t.has_target = true; }
    else if (t.target_kind == PF_TARGET_OFFSET) {
        PF_CHECK(t.target_value >= -1 && t.target_value <= 1, PF_ERR_INVALID, "Offset target requires eta in [-1, 1]");
    } else if (t.target_kind != PF_TARGET_MAXDOS) throw Error(PF_ERR_INVALID, "Unsupported target specification");

    // DoS (DensitiesOfStates.jl:14-43)
    std::vector<double> mu;
    {
        auto w0 = std::chrono::steady_clock::now();
        DevArray<double> pr64;
        DevArray<float> pr32;
        if (P->probes) {
            pr64.alloc((size_t)D * P->dos_R);
            PF_CUDA(cudaMemcpyAsync(pr64.p, P->probes, pr64.n * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        if (P->precision == PF_PREC_FP64) {
            mu = kpm_moments<double>(op, a, b, P->dos_N, P->dos_R, pr64.p, D, P->probe_kind, P->seed, &R.kpm_block_matvecs);
        } else {
            if (P->probes) {
                pr32.alloc((size_t)D * P->dos_R);
                // FP64 host probes -> FP32 device copy (column-major kept)
                launch_ri_to_cm<double, float>(st, (int64_t)P->dos_R * D, 1, pr64.p, pr32.p, (int64_t)P->dos_R * D);
            }
            mu = kpm_moments<float>(op, a, b, P->dos_N, P->dos_R, pr32.p, D, P->probe_kind, P->seed, &R.kpm_block_matvecs);
        }
        R.stage_seconds[7] = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
    }
    Dos rho(mu, P->dos_N, P->dos_kernel);
    {
        auto w0 = std::chrono::steady_clock::now();
        get_bounds(t, &rho);
        get_order(t);
        R.stage_seconds[8] = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
    }
    const std::vector<double> coeffs = normalized_coefficients(t);

    // factorization (FactorizationConfig.jl:99-118, polfed_algorithm.jl:25-34)
    const int64_t maxdim = expected_krylov_dim(nev, s, P->overestimate_iters);
    PF_CHECK(maxdim >= s && maxdim < (1 << 20), PF_ERR_INVALID, "unreasonable Krylov dimension");
    LanczosOut out;
    double stage[6] = {0, 0, 0, 0, 0, 0};
    const int fdtype = P->precision == PF_PREC_FP64 ? PF_F64 : PF_F32;
    if (P->autotune) {
        bool have;
        {
            std::lock_guard<std::mutex> lock(op->tune_mu);
            have = op->tuned_width.count(std::make_pair(fdtype == PF_F64 ? 8 : 4, s)) > 0;
        }
        if (!have && !cached_step_variant(op, s, fdtype)) autotune_step(op, s, fdtype, nullptr);
    }
    // A handle working for a request pool hands its filters to the pool's
    // engine, which batches the Clenshaw steps of every solve in flight into
    // shared launches; otherwise the filter is this solve's own CUDA graph.
    pf_engine *eng = (h->engine && multi_eligible(op, fdtype)) ? h->engine : nullptr;
    const int ew = engine_width(op, s, fdtype == PF_F64 ? 8 : 4);
    if (P->precision == PF_PREC_FP64) {
        Filter<double> filt(op, s, coeffs, a, b, eng == nullptr);
        BlockMap fmap = [&](const double *X, double *Y) {
            if (eng) {
                engine_filter(eng, op, st, 8, s, ew, coeffs, a, b, (void *)X, Y, filt.A.p, filt.B.p);
                return;
            }
            PF_CUDA(cudaMemcpyAsync(filt.X.p, X, (size_t)D * s * sizeof(double), cudaMemcpyDeviceToDevice, st));
            filt.run(st);
            PF_CUDA(cudaMemcpyAsync(Y, filt.Y.p, (size_t)D * s * sizeof(double), cudaMemcpyDeviceToDevice, st));
        };
        lanczos(op, s, nev, (int)maxdim, P->tol, P->eigentol, P->which, P->reorth_passes, xri.p, fmap, out, stage, -1,
                P->host_qr != 0);
    } else {
        const bool refine = P->refine > 0;
        // as many guard vectors as targets: the subspace iteration's rate at the
        // last target is the filter ratio P(lambda_{2 nev}) / P(lambda_{nev})
        const int guard = std::max(s, nev);
        {
            Filter<float> filt(op, s, coeffs, a, b);
            BlockMap fmap = [&](const double *X, double *Y) {
                launch_ri_to_cm<double, float>(st, (int64_t)D * s, 1, X, filt.X.p, (int64_t)D * s);
                if (eng) engine_filter(eng, op, st, 4, s, ew, coeffs, a, b, filt.X.p, filt.Y.p, filt.A.p, filt.B.p);
                else filt.run(st);
                launch_ri_to_cm<float, double>(st, (int64_t)D * s, 1, filt.Y.p, Y, (int64_t)D * s);
            };
            lanczos(op, s, nev, (int)maxdim, P->tol, P->eigentol, P->which, P->reorth_passes, xri.p, fmap, out, stage,
                    refine ? guard : -1, P->host_qr != 0);
        }
        if (refine && out.nconv > 0) {
            // FP64 passes on the FP32 run's nev + guard leading Ritz vectors (filter order)
            auto r0 = std::chrono::steady_clock::now();
            const int m = out.nconv;
            int before = 0;
            while (before < nev && before < m && out.resid[before] < P->eigentol) ++before;
            std::vector<double> vals_f(out.vals), resid(out.resid);
            refine_fp64(op, coeffs, a, b, nev, P->eigentol, P->refine, out.vecs, m, vals_f, resid);
            int ec = 0;
            double maxe = 0.0;
            bool counting = true;
            for (int i = 0; i < std::min(nev, m); ++i) {
                if (counting && resid[i] < P->eigentol) ++ec;
                else counting = false;
                maxe = std::max(maxe, resid[i]);
            }
            out.eigenconverged = ec;
            out.eigenresidual = maxe;
            out.refined = std::max(0, ec - before);
            vals_f.resize(m);
            ascending_prefix(h, D, ec, vals_f, out.vecs);
            out.vals = vals_f;
            out.nconv = ec;
            stage[5] += std::chrono::duration<double>(std::chrono::steady_clock::now() - r0).count();
        } else if (refine) {
            out.nconv = 0;
            out.vals.clear();
        }
    }

    // outputs
    *nconv = out.nconv;
    for (int i = 0; i < out.nconv; ++i) vals[i] = out.vals[i];
    if (vecs && out.nconv > 0) {
        if (vecs_mem == PF_MEM_DEVICE) {
            launch_ri_to_cm<double, double>(st, D, out.nconv, out.vecs.p, vecs, D);
            sync(h);
        } else {
            DevArray<double> cm((size_t)D * out.nconv);
            launch_ri_to_cm<double, double>(st, D, out.nconv, out.vecs.p, cm.p, D);
            PF_CUDA(cudaMemcpyAsync(vecs, cm.p, cm.n * sizeof(double), cudaMemcpyDeviceToHost, st));
            sync(h);
        }
    }
    PF_CUDA(cudaEventRecord(t_end, st));
    sync(h);
    float tot_ms = 0.f;
    cudaEventElapsedTime(&tot_ms, t_begin, t_end);
    cudaEventDestroy(t_begin);
    cudaEventDestroy(t_end);
    (void)t_wall0;

    if (rep) {
        R.Emin = Emin; R.Emax = Emax; R.a = a; R.b = b;
        R.target = t.target; R.left = t.left; R.right = t.right;
        R.order = t.order;
        R.order_safety_factor = t.order_safety_factor;
        R.blocksize = s;
        R.howmany = nev;
        R.iters_needed = out.numiter;
        R.iters_reserved = out.maxiter;
        R.krylovdim = out.krylovdim;
        R.matvecs = (int64_t)t.order * s * out.numiter + nev;  // SpectralTransformReport.jl:54
        R.tol = P->tol;
        R.residual = out.residual;
        R.converged_tol = out.converged;
        R.eigentol = P->eigentol;
        R.eigenresidual = out.eigenresidual;
        R.converged_eigentol = out.eigenconverged;
        R.refined = out.refined;
        R.numofchecks = out.numofchecks;
        for (int i = 0; i < (int)out.conv_hist.size() && i < PF_REPORT_MAX_CHECKS; ++i) {
            R.converged_history[i] = out.conv_hist[i];
            R.krylovdim_history[i] = out.dim_hist[i];
            R.maxresidual_history[i] = out.res_hist[i];
        }
        for (int i = 0; i < 6; ++i) R.stage_seconds[i] = stage[i];
        R.stage_seconds[9] = tot_ms * 1e-3;
        R.basis_bytes_reserved = (double)D * out.maxiter * s * sizeof(double);
        R.basis_bytes_used = (double)D * out.krylovdim * sizeof(double);
        R.kernel_launches = thread_launches() - launches0;
        R.qr_restarts += out.qr_restarts;
        *rep = R;
    }
}

// ------------------------------------------------ complex Hermitian input
// polfed on H = A + iB (the reference's CPU path takes complex Hermitian
// matrices and runs Lanczos in complex arithmetic; its GPU path refuses them,
// PolfedCore.jl:160-162).  op is the real embedding M = [[A, -B], [B, A]],
// which commutes with J [x; y] = [-y; x] (multiplication by i).  The complex
// block Lanczos from x0 (s columns) spans, over the reals, the Krylov space of
// M from [v, Jv] (v = [Re x0; Im x0]): the real solve with 2s columns and
// 2 nev pairs is the complex one, each eigenvalue of H appearing twice.  Its
// Ritz vectors u = [x; y] become complex vectors x + iy; within each group of
// equal eigenvalues a pivoted complex Gram-Schmidt keeps one vector per complex
// direction (the two copies of an eigenvector are psi and i psi; a degenerate
// eigenvalue keeps its whole eigenspace).
void solve_hermitian(pf_op *op, const pf_params *P, int s, int nev, const double *x0, int x0_mem, double *vals,
                     double *vecs, int vecs_mem, pf_report *rep, int *nconv) {
    using cd = std::complex<double>;
    PF_CHECK(op && P && x0 && vals && nconv, PF_ERR_INVALID, "null argument");
    PF_CHECK(op->complex_dim > 0, PF_ERR_INVALID,
             "pf_solve_hermitian needs a Hermitian operator (pf_op_csr_create_hermitian)");
    PF_CHECK(s >= 1 && nev >= 1, PF_ERR_INVALID, "s and nev must be positive");
    const int64_t D = op->complex_dim;
    pf_handle *h = op->h;
    PF_CUDA(cudaSetDevice(h->device));
    AllocStream alloc_guard(h->stream);
    cudaStream_t st = h->stream;
    std::vector<double> xc((size_t)2 * D * s);
    if (x0_mem == PF_MEM_DEVICE) {
        PF_CUDA(cudaMemcpyAsync(xc.data(), x0, xc.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        sync(h);
    } else {
        std::memcpy(xc.data(), x0, xc.size() * sizeof(double));
    }
    // the real start block [v_1 .. v_s, J v_1 .. J v_s]
    const int64_t D2 = 2 * D;
    std::vector<double> xr((size_t)D2 * 2 * s);
    for (int c = 0; c < s; ++c)
        for (int64_t i = 0; i < D; ++i) {
            const double re = xc[2 * (i + (size_t)c * D)], im = xc[2 * (i + (size_t)c * D) + 1];
            xr[i + (size_t)c * D2] = re;
            xr[D + i + (size_t)c * D2] = im;
            xr[i + (size_t)(s + c) * D2] = -im;
            xr[D + i + (size_t)(s + c) * D2] = re;
        }
    const int m = 2 * nev;
    std::vector<double> rv(m);
    DevArray<double> rvec((size_t)D2 * m);
    int rn = 0;
    pf_report R;
    std::memset(&R, 0, sizeof(R));
    solve(op, P, 2 * s, m, xr.data(), PF_MEM_HOST, rv.data(), rvec.p, PF_MEM_DEVICE, &R, &rn);
    std::vector<double> hv((size_t)D2 * std::max(rn, 1));
    if (rn > 0) {
        PF_CUDA(cudaMemcpyAsync(hv.data(), rvec.p, (size_t)D2 * rn * sizeof(double), cudaMemcpyDeviceToHost, st));
        sync(h);
    }
    struct Pair {
        double val;
        std::vector<cd> psi;
    };
    std::vector<Pair> out;
    for (int i0 = 0; i0 < rn;) {
        int i1 = i0 + 1;
        while (i1 < rn && std::fabs(rv[i1] - rv[i0]) <= 1e-8 * std::max(1.0, std::fabs(rv[i0]))) ++i1;
        std::vector<std::vector<cd>> cand;
        std::vector<double> cval;
        for (int a = i0; a < i1; ++a) {
            std::vector<cd> psi((size_t)D);
            for (int64_t k = 0; k < D; ++k) psi[k] = cd(hv[k + (size_t)a * D2], hv[D + k + (size_t)a * D2]);
            cand.push_back(std::move(psi));
            cval.push_back(rv[a]);
        }
        std::vector<bool> used(cand.size(), false);
        std::vector<std::vector<cd>> kept;
        while (true) {
            // the candidate with the largest component outside the kept vectors
            int best = -1;
            double bestn = 0.3;
            std::vector<cd> bestv;
            for (size_t a = 0; a < cand.size(); ++a) {
                if (used[a]) continue;
                std::vector<cd> w = cand[a];
                for (const auto &b : kept) {
                    cd dot = 0.0;
                    for (int64_t k = 0; k < D; ++k) dot += std::conj(b[k]) * w[k];
                    for (int64_t k = 0; k < D; ++k) w[k] -= dot * b[k];
                }
                double n2 = 0.0;
                for (int64_t k = 0; k < D; ++k) n2 += std::norm(w[k]);
                if (std::sqrt(n2) > bestn) {
                    bestn = std::sqrt(n2);
                    best = (int)a;
                    bestv.swap(w);
                }
            }
            if (best < 0) break;
            used[best] = true;
            for (auto &z : bestv) z /= bestn;
            kept.push_back(bestv);
            out.push_back({cval[best], bestv});
        }
        i0 = i1;
    }
    std::stable_sort(out.begin(), out.end(), [](const Pair &x, const Pair &y) { return x.val < y.val; });
    if ((int)out.size() > nev) {
        // more complex directions than asked (an unpaired copy): the nev nearest the target
        const double tgt = R.a * R.target + R.b;
        std::vector<int> ord(out.size());
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(),
                         [&](int x, int y) { return std::fabs(out[x].val - tgt) < std::fabs(out[y].val - tgt); });
        ord.resize(nev);
        std::sort(ord.begin(), ord.end());
        std::vector<Pair> sel;
        for (int k : ord) sel.push_back(std::move(out[k]));
        out.swap(sel);
    }
    const int nc = (int)out.size();
    *nconv = nc;
    for (int k = 0; k < nc; ++k) vals[k] = out[k].val;
    if (vecs && nc > 0) {
        std::vector<double> packed((size_t)2 * D * nc);
        for (int k = 0; k < nc; ++k)
            for (int64_t i = 0; i < D; ++i) {
                packed[2 * (i + (size_t)k * D)] = out[k].psi[i].real();
                packed[2 * (i + (size_t)k * D) + 1] = out[k].psi[i].imag();
            }
        if (vecs_mem == PF_MEM_DEVICE) {
            PF_CUDA(cudaMemcpyAsync(vecs, packed.data(), packed.size() * sizeof(double), cudaMemcpyHostToDevice, st));
            sync(h);
        } else {
            std::memcpy(vecs, packed.data(), packed.size() * sizeof(double));
        }
    }
    if (rep) {
        // the real solve's report, in the complex problem's terms
        R.blocksize = s;
        R.howmany = nev;
        R.converged_eigentol = nc;
        *rep = R;
    }
}

}  // namespace pf
