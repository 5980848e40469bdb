// pf_spectral.cpp -- host-side spectral planning of POLFED, restated in C++.
//
//   kernels        DensetiesOfStates/Kernels.jl:33-72
//   rho(x)         DensetiesOfStates/DensitiesOfStates.jl:27-34
//   clenshaw       Clenshaw/Algorithm/ClenshawAlgorithm.jl:35-54, FinalSum.jl:26-30
//   bisection      SpectralTransformation/Bisection.jl:18-40
//   quadgk         QuadGK.jl 2.x adaptive Gauss-Kronrod (7,15) (the published
//                  rule; QuadGK.jl itself is not part of the reference tree)
//   bounds / order GetBounds.jl:19-118, GetOrderOfExpansion.jl:8-70
//   target         Polfed/Plan/Plan.jl:203-281
//   coefficients   Polfed/Structs/PolfedDefaults.jl:104 (c_0 = 1, c_n = 2 cos(n acos t))
#include "pf_spectral.h"

#include <algorithm>
#include <cmath>
#include <queue>
#include <stdexcept>

#include "pf_internal.h"

namespace pf {

double kernel_weight(int kind, int n, int N) {
    const double pi = M_PI;
    switch (kind) {
        case PF_KERNEL_JACKSON:
            return ((N - n + 1) * std::cos(pi * n / (N + 1)) +
                    std::sin(pi * n / (N + 1)) / std::tan(pi / (N + 1))) / (N + 1);
        case PF_KERNEL_LORENTZ: return std::sinh(1.0 * (1.0 - (double)n / N)) / std::sinh(1.0);
        case PF_KERNEL_FEJER: return 1.0 - (double)n / N;
        case PF_KERNEL_LANCZOS:
            if (n == 0) return 1.0;
            return std::pow(std::sin(pi * n / N) / (pi * n / N), 3);
        case PF_KERNEL_WANGZUNGER: return std::exp(-std::pow(1.0 * n / N, 1.0));
        case PF_KERNEL_DIRICHLET: return 1.0;
        default: throw Error(PF_ERR_INVALID, "unknown DoS kernel");
    }
}

double cheb_clenshaw(const double *c, int K, double x) {
    double b2 = 0.0, b3 = 0.0;
    for (int k = K; k >= 1; --k) {
        const double b1 = c[k] + 2.0 * x * b2 + (-1.0) * b3;
        b3 = b2;
        b2 = b1;
    }
    return c[0] * 1.0 + 1.0 * x * b2 + (-1.0) * 1.0 * b3;
}

double filter_coefficient(double target, int n) {
    return (2.0 - (n == 0 ? 1.0 : 0.0)) * std::cos(n * std::acos(target));
}

std::vector<double> raw_coefficients(double target, int K) {
    std::vector<double> c(K + 1);
    for (int n = 0; n <= K; ++n) c[n] = filter_coefficient(target, n);
    return c;
}

Dos::Dos(const std::vector<double> &mu, int N, int kernel) : N_(N) {
    coeffs_.resize(N);
    for (int i = 0; i < N; ++i) coeffs_[i] = kernel_weight(kernel, i, N) * mu[i] * (2.0 - (i == 0 ? 1.0 : 0.0));
}

// Quadrature nodes that round onto x = +-1 (getbounds_from_dos integrates up
// to the spectrum's edges) are moved to the nearest double inside (-1, 1), so
// the 1/sqrt(1 - x^2) weight stays finite.
double Dos::operator()(double x) const {
    const double xm = std::nextafter(1.0, 0.0);
    x = std::min(std::max(x, -xm), xm);
    return cheb_clenshaw(coeffs_.data(), N_ - 1, x) / (M_PI * std::sqrt(1.0 - x * x));
}

// Bisection.jl:18-40.  Every caller is a planning step (the interval from
// the DoS, the order in the interval, the interval from the order): a bracket
// without a sign change means no filter meets the request's target and
// howmany, so the error is marked infeasible (a pool rejects the request).
double bisection(const std::function<int(double)> &f, double x1, double x2, double tol, int max_iter) {
    if ((double)f(x1) * (double)f(x2) > 0) {
        Error e(PF_ERR_NUMERIC, "The function must have opposite signs at a and b");
        e.infeasible = true;
        throw e;
    }
    int it = 0;
    while ((x2 - x1) / 2 >= tol && it < max_iter) {
        const double x = (x1 + x2) / 2;
        const int fc = f(x);
        if (fc == 0 || (x2 - x1) / 2 <= tol) return x;
        if (f(x1) * fc < 0) x2 = x;
        else x1 = x;
        ++it;
    }
    return (x1 + x2) / 2;
}

// Gauss-Kronrod 7/15 nodes and weights (QUADPACK qk15, published values).
static const double XGK[8] = {0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
                              0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
                              0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
                              0.207784955007898467600689403773245, 0.0};
static const double WGK[8] = {0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
                              0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
                              0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
                              0.204432940075298892414161999234649, 0.209482141084727828012999174891714};
static const double WG[4] = {0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
                             0.381830050505118944950369775488975, 0.417959183673469387755102040816327};

static void gk_rule(const std::function<double(double)> &f, double a, double b, double &I, double &E) {
    const double c = 0.5 * (a + b), h = 0.5 * (b - a);
    const double fc = f(c);
    double ik = WGK[7] * fc, ig = WG[3] * fc;
    for (int j = 0; j < 7; ++j) {
        const double fl = f(c - h * XGK[j]), fr = f(c + h * XGK[j]);
        ik += WGK[j] * (fl + fr);
        if (j % 2 == 1) ig += WG[j / 2] * (fl + fr);
    }
    I = ik * h;
    E = std::fabs((ik - ig) * h);
}

double quadgk(const std::function<double(double)> &f, double a, double b, double atol, double rtol,
              long maxevals) {
    if (a == b) return 0.0;
    struct Seg { double a, b, I, E; };
    auto cmp = [](const Seg &x, const Seg &y) { return x.E < y.E; };
    std::priority_queue<Seg, std::vector<Seg>, decltype(cmp)> heap(cmp);
    double I, E;
    gk_rule(f, a, b, I, E);
    heap.push({a, b, I, E});
    long nev = 15;
    while (E > std::max(atol, rtol * std::fabs(I)) && nev < maxevals) {
        Seg s = heap.top();
        const double mid = 0.5 * (s.a + s.b);
        if (!(s.a < mid && mid < s.b)) break;
        heap.pop();
        double I1, E1, I2, E2;
        gk_rule(f, s.a, mid, I1, E1);
        gk_rule(f, mid, s.b, I2, E2);
        nev += 30;
        I = (I - s.I) + I1 + I2;
        E = (E - s.E) + E1 + E2;
        heap.push({s.a, mid, I1, E1});
        heap.push({mid, s.b, I2, E2});
    }
    double sum = 0.0;
    while (!heap.empty()) { sum += heap.top().I; heap.pop(); }
    return sum;
}

double analytical_order(double lam, double delta) { return 2.65499 * std::sqrt(1 - lam * lam) / delta; }

static void bound_fns(int pos, double t, double d, double &lo, double &hi) {
    // :mean only is used by the driver; :left / :right kept for completeness
    if (pos == 0) { lo = t - d; hi = t + d; }
    else if (pos == 1) { lo = t; hi = t + 2 * d; }
    else { lo = t - 2 * d; hi = t; }
    lo = std::max(lo, -1.0);
    hi = std::min(hi, 1.0);
}

static double poly_at(const std::vector<double> &c, int K, double norm_, double normalization, double x) {
    return cheb_clenshaw(c.data(), K, x) / norm_ * normalization;
}

void bounds_from_dos(TransformState &t, const Dos &rho) {
    auto f = [&](double d) {
        double lo, hi;
        bound_fns(0, t.target, d, lo, hi);
        const double n = quadgk([&](double x) { return rho(x); }, lo, hi, 1e-12, 1e-12, 10000000L);
        return n >= t.howmany ? -1 : +1;
    };
    const double d = bisection(f, 0.0, 1.0, 1e-8, 500);   // infeasible: no interval holds howmany states
    bound_fns(0, t.target, d, t.left, t.right);
}

void bounds_from_K(TransformState &t) {
    const std::vector<double> c = raw_coefficients(t.target, t.order);
    const double norm_ = cheb_clenshaw(c.data(), t.order, t.target);
    auto f = [&](double d) {
        double lo, hi;
        bound_fns(0, t.target, d, lo, hi);
        const double m = std::max(poly_at(c, t.order, norm_, t.normalization, lo),
                                  poly_at(c, t.order, norm_, t.normalization, hi));
        return m >= t.cutoff ? -1 : +1;
    };
    const double d = bisection(f, 0.0, 1.0, 1e-8, 500);
    bound_fns(0, t.target, d, t.left, t.right);
}

void order_in_interval(TransformState &t) {
    const double target = (t.left + t.right) / 2;
    const double halfwidth = (t.right - t.left) / 2;
    auto f = [&](double order) {
        const int K = (int)std::floor(order);
        const std::vector<double> c = raw_coefficients(target, K);
        const double norm_ = cheb_clenshaw(c.data(), K, target);
        const double m = std::max(poly_at(c, K, norm_, t.normalization, t.left),
                                  poly_at(c, K, norm_, t.normalization, t.right));
        return m >= t.cutoff ? -1 : +1;
    };
    const double Kmax = std::ceil(analytical_order(target, halfwidth) * 2);
    const double K = bisection(f, 10.0, Kmax, 1.0, 500);
    t.order = (int)std::floor(K * t.order_safety_factor);
    if (t.order_safety_factor < 1.0) bounds_from_K(t);
}

double find_maximal_density(const Dos &rho) {
    double best = -INFINITY, xb = 0.0;
    for (int i = 0; i < 5000; ++i) {
        const double x = -0.99 + (1.98 * i) / 4999.0;
        const double v = rho(x);
        if (v > best) { best = v; xb = x; }
    }
    return xb;
}

void resolve_target(TransformState &t, const Dos *rho) {
    if (t.has_target) return;
    switch (t.target_kind) {
        case PF_TARGET_MAXDOS: t.target = find_maximal_density(*rho); break;
        case PF_TARGET_OFFSET: {
            const double peak = find_maximal_density(*rho);
            const double eta = t.target_value;
            t.target = eta >= 0 ? peak + eta * (1.0 - peak) : peak + eta * (1.0 + peak);
            break;
        }
        case PF_TARGET_MIDDLE: t.target = 0.0; break;
        case PF_TARGET_RESCALED: t.target = t.target_value; break;
        case PF_TARGET_UNRESCALED: t.target = (t.target_value - t.b) / t.a; break;
        default: throw Error(PF_ERR_INVALID, "Unsupported target specification");
    }
    t.has_target = true;
}

void get_bounds(TransformState &t, const Dos *rho) {
    const bool bounds_set = t.has_left && t.has_right;
    const bool order_set = t.order > 0;
    if (!t.has_target) resolve_target(t, rho);
    if (bounds_set && order_set)
        throw Error(PF_ERR_INVALID, "Both interval bounds and polynomial order are specified. "
                                    "Please set only one or neither.");
    else if (bounds_set) {
    } else if (order_set) bounds_from_K(t);
    else bounds_from_dos(t, *rho);
}

void get_order(TransformState &t) {
    if (t.order <= 0) order_in_interval(t);
}

std::vector<double> normalized_coefficients(const TransformState &t) {
    std::vector<double> c = raw_coefficients(t.target, t.order);
    const double norm_ = 1.0 / cheb_clenshaw(c.data(), t.order, t.target) * t.normalization;
    for (double &v : c) v *= norm_;
    return c;
}

}  // namespace pf
