// pf_spectral.h -- host-side spectral planning (DoS, interval, order, coefficients).
#pragma once
#include <functional>
#include <vector>

namespace pf {

double kernel_weight(int kind, int n, int N);
double cheb_clenshaw(const double *c, int K, double x);
double filter_coefficient(double target, int n);
std::vector<double> raw_coefficients(double target, int K);

// KPM density of states rho(x) = sum_n g_n mu_n (2 - delta_n0) T_n(x) / (pi sqrt(1 - x^2))
class Dos {
  public:
    Dos(const std::vector<double> &mu, int N, int kernel);
    double operator()(double x) const;

  private:
    int N_;
    std::vector<double> coeffs_;
};

double bisection(const std::function<int(double)> &f, double x1, double x2, double tol, int max_iter);
double quadgk(const std::function<double(double)> &f, double a, double b, double atol, double rtol,
              long maxevals);
double analytical_order(double lam, double delta);

// TransformPlan of Plan.jl:32-44 in rescaled units.
struct TransformState {
    int target_kind = 0;
    double target_value = 0.0;
    double a = 1.0, b = 0.0;
    bool has_target = false;
    double target = 0.0;
    bool has_left = false, has_right = false;
    double left = 0.0, right = 0.0;
    int order = 0;
    double cutoff = 0.17, normalization = 1.0, order_safety_factor = 0.97;
    int howmany = 1;
};

void bounds_from_dos(TransformState &t, const Dos &rho);
void bounds_from_K(TransformState &t);
void order_in_interval(TransformState &t);
double find_maximal_density(const Dos &rho);
void resolve_target(TransformState &t, const Dos *rho);
void get_bounds(TransformState &t, const Dos *rho);
void get_order(TransformState &t);
std::vector<double> normalized_coefficients(const TransformState &t);

}  // namespace pf
