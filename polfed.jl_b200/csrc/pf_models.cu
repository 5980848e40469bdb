// pf_models.cu -- the Quantum Sun family beyond the spin-1/2 full space:
// spin S > 1/2 (QuantumSun.jl:1-102) and the total-S_z sector of any spin
// (QuantumSun_U1_conserving.jl:1-212), assembled as a CSR matrix on the
// device and served by the CSR row of the step kernel.
//
// States.  A site holds a digit c in 0..d-1 (d = 2S+1, m = c - S).  The
// reference packs the digits into ceil(log2 d) bits per site and sorts the
// packed codes (HilbertSpace.jl:9-41), so a state's index in the full space is
// its base-d value sum_i c_i d^i (site 0 least significant).  In the sector
// sum_i m_i = S_z, i.e. sum_i c_i = T = S_z + L S, and the index is the rank of
// that value among the sector's states: walking from the most significant
// site down, every smaller digit c at site i adds cnt[i][R - c] states, where
// R is the digit sum still to place and cnt[i][t] the number of i-digit
// strings summing to t.
//
// Row entries, in the reference's assembly order (QuantumSun.jl:35-95):
//   * the localized fields, sum_j h_j m_{L_grain+j}, as one diagonal entry;
//   * for each localized spin j, S^x_loc S^x_grain(n_j): the states with the
//     localized digit raised / lowered and the grain digit raised / lowered,
//     value ((g0 c_j) a_loc) a_grain with a_up(m) = sqrt(S(S+1) - m(m+1))/2 and
//     a_down(m) = sqrt(S(S+1) - m(m-1))/2 (SpinOperators.jl:38-53).  In the
//     sector only the two exchanges that keep S_z survive, and S^y S^y adds an
//     equal element to each (SpinOperators.jl:55-69; the reference pushes
//     both and sums them), so each is one entry of twice the S^x S^x value;
//   * the grain block: for every grain configuration g' (of equal grain
//     magnetisation in the sector) the entry grain[g][g'] to the state with
//     the same localized digits.
// A row may list its own column twice (the fields and the grain's diagonal);
// the CSR step sums a row's entries in storage order.
#include "pf_internal.h"
#include "pf_solver.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace pf {

constexpr int kSpinMaxSites = 32;
constexpr int kSpinMaxDigits = 16;   // d = 2S + 1 <= 16
constexpr int kSpinMaxGrain = 4096;  // d^L_grain

struct SpinBuild {
    int d, L, L_grain, L_loc, u1, T, tmax;   // tmax = L (d - 1): columns of cnt
    int64_t D, dg;
    double g0;
    double coup[kSpinMaxSites], fields[kSpinMaxSites];
    int nbr[kSpinMaxSites];
    double aup[kSpinMaxDigits], adn[kSpinMaxDigits], m[kSpinMaxDigits];
    int64_t pw[kSpinMaxSites + 1];          // d^i
};

// cnt[i * (tmax + 1) + t]: i-digit strings with digit sum t (0 outside range)
__device__ __forceinline__ int64_t spin_cnt(const SpinBuild &b, const int64_t *cnt, int i, int t) {
    return (t < 0 || t > i * (b.d - 1)) ? 0 : cnt[(size_t)i * (b.tmax + 1) + t];
}

// Index of the digit string c (sites 0..L-1).
__device__ int64_t spin_index(const SpinBuild &b, const int64_t *cnt, const uint8_t *c) {
    if (!b.u1) {
        int64_t idx = 0;
        for (int i = b.L - 1; i >= 0; --i) idx = idx * b.d + c[i];
        return idx;
    }
    int64_t r = 0;
    int R = b.T;
    for (int i = b.L - 1; i >= 0; --i) {
        for (int v = 0; v < c[i]; ++v) r += spin_cnt(b, cnt, i, R - v);
        R -= c[i];
    }
    return r;
}

// Digit string of index r.
__device__ void spin_digits(const SpinBuild &b, const int64_t *cnt, int64_t r, uint8_t *c) {
    if (!b.u1) {
        for (int i = 0; i < b.L; ++i) {
            c[i] = (uint8_t)(r % b.d);
            r /= b.d;
        }
        return;
    }
    int R = b.T;
    for (int i = b.L - 1; i >= 0; --i) {
        int v = 0;
        for (; v < b.d - 1; ++v) {
            const int64_t n = spin_cnt(b, cnt, i, R - v);
            if (r < n) break;
            r -= n;
        }
        c[i] = (uint8_t)v;
        R -= v;
    }
}

// One row: COUNT = true counts its entries into *count; otherwise writes
// them at col/val (both precisions).
template <bool COUNT>
__device__ void spin_row(const SpinBuild &b, const int64_t *cnt, const double *grain, int64_t row, int *count,
                         int32_t *col, double *v64, float *v32) {
    uint8_t c[kSpinMaxSites];
    spin_digits(b, cnt, row, c);
    int n = 0;
    auto emit = [&](int64_t j, double v) {
        if (!COUNT) {
            col[n] = (int32_t)j;
            v64[n] = v;
            v32[n] = (float)v;
        }
        ++n;
    };
    // the localized fields (QuantumSun.jl:36-44): one diagonal entry
    double dsum = 0.0;
    for (int j = 0; j < b.L_loc; ++j) dsum += b.fields[j] * b.m[c[b.L_grain + j]];
    emit(row, dsum);
    // S^x S^x (and, in the sector, S^y S^y) of each localized spin with its grain neighbour
    for (int j = 0; j < b.L_loc; ++j) {
        const int sl = b.L_grain + j, sg = b.nbr[j];
        const int cl = c[sl], cg = c[sg];
        const double base = b.g0 * b.coup[j];
        for (int lu = 0; lu < 2; ++lu) {          // localized digit up, then down
            const bool lok = lu == 0 ? cl < b.d - 1 : cl > 0;
            if (!lok) continue;
            const double al = lu == 0 ? b.aup[cl] : b.adn[cl];
            for (int gu = 0; gu < 2; ++gu) {      // grain digit up, then down
                const bool gok = gu == 0 ? cg < b.d - 1 : cg > 0;
                if (!gok) continue;
                if (b.u1 && lu == gu) continue;   // changes S_z
                const double ag = gu == 0 ? b.aup[cg] : b.adn[cg];
                double v = base * al * ag;
                if (b.u1) v = v + v;              // S^x S^x + S^y S^y
                c[sl] = (uint8_t)(lu == 0 ? cl + 1 : cl - 1);
                c[sg] = (uint8_t)(gu == 0 ? cg + 1 : cg - 1);
                emit(spin_index(b, cnt, c), v);
                c[sl] = (uint8_t)cl;
                c[sg] = (uint8_t)cg;
            }
        }
    }
    // the grain block: kron(I_loc, H_grain) restricted to the basis
    int64_t g = 0;
    int gsum = 0;
    for (int i = b.L_grain - 1; i >= 0; --i) {
        g = g * b.d + c[i];
        gsum += c[i];
    }
    uint8_t keep[kSpinMaxSites];
    for (int i = 0; i < b.L_grain; ++i) keep[i] = c[i];
    for (int64_t g2 = 0; g2 < b.dg; ++g2) {
        int64_t t = g2;
        int s2 = 0;
        for (int i = 0; i < b.L_grain; ++i) {
            c[i] = (uint8_t)(t % b.d);
            s2 += c[i];
            t /= b.d;
        }
        if (b.u1 && s2 != gsum) continue;
        emit(spin_index(b, cnt, c), grain[g * b.dg + g2]);
    }
    for (int i = 0; i < b.L_grain; ++i) c[i] = keep[i];
    if (COUNT) *count = n;
}

__global__ void k_spin_count(const SpinBuild b, const int64_t *__restrict__ cnt, const double *__restrict__ grain,
                             int *__restrict__ counts) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < b.D; r += (int64_t)gridDim.x * blockDim.x)
        spin_row<true>(b, cnt, grain, r, counts + r, nullptr, nullptr, nullptr);
}

__global__ void k_spin_fill(const SpinBuild b, const int64_t *__restrict__ cnt, const double *__restrict__ grain,
                            const int64_t *__restrict__ indptr, int32_t *__restrict__ col, double *__restrict__ v64,
                            float *__restrict__ v32) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < b.D; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = indptr[r];
        spin_row<false>(b, cnt, grain, r, nullptr, col + p, v64 + p, v32 + p);
    }
}

pf_op *create_qsun_spin(pf_handle *h, int L_loc, int L_grain, int two_S, int u1, int two_Sz, double g0,
                        const double *coup, const int32_t *nbr, const double *fields, const double *grain) {
    PF_CHECK(h != nullptr, PF_ERR_INVALID, "null handle");
    PF_CHECK(coup && nbr && fields && grain, PF_ERR_INVALID, "null QSun parameter array");
    PF_CHECK(two_S >= 1 && two_S + 1 <= kSpinMaxDigits, PF_ERR_UNSUPPORTED, "spin S must be in 1/2 .. 15/2");
    PF_CHECK(L_loc >= 1 && L_grain >= 1 && L_loc + L_grain <= kSpinMaxSites, PF_ERR_INVALID,
             "need L_loc >= 1, L_grain >= 1 and L_loc + L_grain <= 32");
    PF_CHECK(std::isfinite(g0), PF_ERR_INVALID, "non-finite g0");
    SpinBuild b{};
    b.d = two_S + 1;
    b.L_loc = L_loc;
    b.L_grain = L_grain;
    b.L = L_loc + L_grain;
    b.u1 = u1 ? 1 : 0;
    b.g0 = g0;
    b.tmax = b.L * (b.d - 1);
    const double S = 0.5 * two_S;
    b.pw[0] = 1;
    for (int i = 1; i <= b.L; ++i) {
        PF_CHECK(b.pw[i - 1] <= ((int64_t)1 << 40) / b.d, PF_ERR_UNSUPPORTED, "Hilbert space too large");
        b.pw[i] = b.pw[i - 1] * b.d;
    }
    b.dg = b.pw[L_grain];
    PF_CHECK(b.dg <= kSpinMaxGrain, PF_ERR_UNSUPPORTED, "grain dimension (2S+1)^L_grain above 4096");
    for (int j = 0; j < L_loc; ++j) {
        PF_CHECK(nbr[j] >= 0 && nbr[j] < L_grain, PF_ERR_INVALID, "grain neighbour out of range");
        PF_CHECK(std::isfinite(coup[j]) && std::isfinite(fields[j]), PF_ERR_INVALID, "non-finite parameter");
        b.coup[j] = coup[j];
        b.fields[j] = fields[j];
        b.nbr[j] = nbr[j];
    }
    for (int64_t q = 0; q < b.dg * b.dg; ++q) PF_CHECK(std::isfinite(grain[q]), PF_ERR_INVALID, "non-finite grain block");
    // SpinOperators.jl:38-53, in the reference's operation order
    for (int cc = 0; cc < b.d; ++cc) {
        const double mm = cc - S;
        b.m[cc] = mm;
        b.aup[cc] = cc < b.d - 1 ? 0.5 * std::sqrt(S * (S + 1) - mm * (mm + 1)) : 0.0;
        b.adn[cc] = cc > 0 ? 0.5 * std::sqrt(S * (S + 1) - mm * (mm - 1)) : 0.0;
    }
    // digit-sum counts (sector ranks)
    std::vector<int64_t> cnt((size_t)(b.L + 1) * (b.tmax + 1), 0);
    cnt[0] = 1;
    for (int i = 1; i <= b.L; ++i)
        for (int t = 0; t <= i * (b.d - 1); ++t) {
            int64_t v = 0;
            for (int cc = 0; cc < b.d && cc <= t; ++cc) v += cnt[(size_t)(i - 1) * (b.tmax + 1) + t - cc];
            cnt[(size_t)i * (b.tmax + 1) + t] = v;
        }
    if (b.u1) {
        // QuantumSun_U1_conserving.jl:17-20
        const int twoT = two_Sz + b.L * two_S;   // 2 (S_z + L S)
        char msg[160];
        std::snprintf(msg, sizeof msg,
                      "Wrong total value of spin to given spin-S particles. You chose S = %g and S_z = %g.", S,
                      0.5 * two_Sz);
        PF_CHECK(std::abs(two_Sz) <= b.L * two_S && twoT % 2 == 0, PF_ERR_INVALID, msg);
        b.T = twoT / 2;
        b.D = cnt[(size_t)b.L * (b.tmax + 1) + b.T];
    } else {
        b.T = 0;
        b.D = b.pw[b.L];
    }
    PF_CHECK(b.D >= 1 && b.D < ((int64_t)1 << 31), PF_ERR_UNSUPPORTED, "matrix dimension must be in [1, 2^31)");

    PF_CUDA(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    int64_t *dcnt = nullptr, *dptr = nullptr;
    double *dgrain = nullptr, *dv64 = nullptr;
    int *dcount = nullptr;
    int32_t *didx = nullptr;
    float *dv32 = nullptr;
    auto release = [&]() {
        cudaFree(dcnt);
        cudaFree(dgrain);
        cudaFree(dcount);
    };
    try {
        PF_CUDA(cudaMalloc(&dcnt, cnt.size() * sizeof(int64_t)));
        PF_CUDA(cudaMalloc(&dgrain, (size_t)b.dg * b.dg * sizeof(double)));
        PF_CUDA(cudaMalloc(&dcount, (size_t)b.D * sizeof(int)));
        PF_CUDA(cudaMemcpyAsync(dcnt, cnt.data(), cnt.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        PF_CUDA(cudaMemcpyAsync(dgrain, grain, (size_t)b.dg * b.dg * sizeof(double), cudaMemcpyHostToDevice, st));
        const int grid = grid_for(h, b.D, 256, 8);
        k_spin_count<<<grid, 256, 0, st>>>(b, dcnt, dgrain, dcount);
        PF_CUDA(cudaGetLastError());
        std::vector<int> counts((size_t)b.D);
        PF_CUDA(cudaMemcpyAsync(counts.data(), dcount, (size_t)b.D * sizeof(int), cudaMemcpyDeviceToHost, st));
        PF_CUDA(cudaStreamSynchronize(st));
        std::vector<int64_t> indptr((size_t)b.D + 1, 0);
        for (int64_t r = 0; r < b.D; ++r) indptr[r + 1] = indptr[r] + counts[r];
        const int64_t nnz = indptr[b.D];
        PF_CUDA(cudaMalloc(&dptr, (b.D + 1) * sizeof(int64_t)));
        PF_CUDA(cudaMalloc(&didx, std::max<int64_t>(nnz, 1) * sizeof(int32_t)));
        PF_CUDA(cudaMalloc(&dv64, std::max<int64_t>(nnz, 1) * sizeof(double)));
        PF_CUDA(cudaMalloc(&dv32, std::max<int64_t>(nnz, 1) * sizeof(float)));
        PF_CUDA(cudaMemcpyAsync(dptr, indptr.data(), (b.D + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        k_spin_fill<<<grid, 256, 0, st>>>(b, dcnt, dgrain, dptr, didx, dv64, dv32);
        PF_CUDA(cudaGetLastError());
        count_launches(2);
        PF_CUDA(cudaStreamSynchronize(st));
        release();
        dcnt = nullptr;
        dgrain = nullptr;
        dcount = nullptr;
        int64_t *p = dptr;
        int32_t *ix = didx;
        double *a = dv64;
        float *f = dv32;
        dptr = nullptr, didx = nullptr, dv64 = nullptr, dv32 = nullptr;
        pf_op *op = adopt_csr(h, b.D, nnz, p, ix, a, f);
        op->L_loc = L_loc;
        op->L_grain = L_grain;
        op->g0 = g0;
        op->coup.assign(coup, coup + L_loc);
        op->nbr.assign(nbr, nbr + L_loc);
        op->fields.assign(fields, fields + L_loc);
        op->grain.assign(grain, grain + b.dg * b.dg);
        return op;
    } catch (...) {
        release();
        cudaFree(dptr);
        cudaFree(didx);
        cudaFree(dv64);
        cudaFree(dv32);
        throw;
    }
}

}  // namespace pf
