// Host-side helpers shared by the C ABI translation units: error state,
// contract validation with the reference's rules, and the per-step invariants.
#pragma once

#include <cmath>
#include <cstdint>
#include <string>

#include "qk_internal.h"

namespace qk {

// Thread-local message behind qk_last_error().
void set_error(const std::string &msg);
qk_status fail(qk_status s, const std::string &msg);
extern thread_local std::string g_last_error;  // message of the last failing call on this thread

// UInputs::validate (include/core/config/Config.hpp:63-84, 119-137, 198-305, 347-373,
// 442-563) on the fields a contract carries, plus this engine's own limits.
qk_status validate_contract(const qk_contract &c, const qk_greeks *g);

// Per-step invariants exactly as the reference constructors compute them
// (MSchemes.hpp:102-123, 197-219, 303-353, 480-487, 535-550), in double, then
// rounded to R.  eps is the QE guard (1e-12 in FP64 builds, 1e-6 in FP32 builds).
template <class R>
inline StepConst<R> make_step_const(const qk_contract &c, double dt, double eps) {
    double q = c.q;
    if (c.model == QK_BATES) {
        // Bates martingale compensator folded into the dividend yield (MSchemes.hpp:535-550)
        const double kappa_j = std::exp(c.mu_j + 0.5 * c.sigma_j * c.sigma_j) - 1.0;
        q += c.lambda_j * kappa_j;
    }
    const double k = c.kappa, theta = c.theta, sigma = c.sigma;
    double rho = c.rho;
    const double sqrt_dt = std::sqrt(dt);
    StepConst<double> d{};
    d.r_minus_q_dt = (c.r - q) * dt;
    d.half_dt = 0.5 * dt;
    d.sqrt_dt = sqrt_dt;
    d.one_minus_k_dt = 1.0 - k * dt;
    d.k_theta_dt = k * theta * dt;
    d.sigma_sqrt_dt = sigma * sqrt_dt;
    d.quarter_sigma_sq_dt = 0.25 * sigma * sigma * dt;
    d.implicit_den = 1.0 / (1.0 + k * dt);
    // QE (Andersen 2008 as in Rouah, eqs 7.37-7.51)
    d.eps = eps;
    d.psi_c = c.psi_c > 0.0 ? c.psi_c : 1.5;
    d.inv_sqrt2 = 1.0 / std::sqrt(2.0);
    d.exp_mkdt = std::exp(-k * dt);
    if (k < eps) {
        d.theta_m = 0.0;
        d.s2f1 = sigma * sigma * dt;
        d.s2f2 = 0.0;
    } else {
        const double one_minus_exp = 1.0 - d.exp_mkdt;
        d.theta_m = theta * one_minus_exp;
        d.s2f1 = (sigma * sigma * d.exp_mkdt / k) * one_minus_exp;
        d.s2f2 = (theta * sigma * sigma / (2.0 * k)) * (one_minus_exp * one_minus_exp);
    }
    double rho_div_sigma;
    double rho_qe = rho;
    if (sigma < eps) {
        rho_div_sigma = 0.0;
        rho_qe = 0.0;
    } else {
        rho_div_sigma = rho / sigma;
    }
    const double one_m_rho2 = 1.0 - rho_qe * rho_qe;
    const double K12 = k * rho_div_sigma - 0.5;
    const double g1 = 0.5, g2 = 0.5;
    d.K1 = dt * g1 * K12 - rho_div_sigma;
    d.K2 = dt * g2 * K12 + rho_div_sigma;
    d.K3 = dt * g1 * one_m_rho2;
    d.K4 = dt * g2 * one_m_rho2;
    d.A = d.K2 + d.K4 * 0.5;
    d.K1_half_K3 = d.K1 + d.K3 * 0.5;
    d.rho = rho;
    d.rho_c = std::sqrt(1.0 - rho * rho);
    // Bates jumps
    const double lambda_dt = (c.model == QK_BATES) ? c.lambda_j * dt : 0.0;
    d.exp_m_lambda_dt = std::exp(-lambda_dt);
    d.mu_j = c.mu_j;
    d.sigma_j = c.sigma_j;
    if constexpr (sizeof(R) == sizeof(double)) {
        return d;
    } else {
        StepConst<R> f;
        const double *src = reinterpret_cast<const double *>(&d);
        R *dst = reinterpret_cast<R *>(&f);
        static_assert(sizeof(StepConst<double>) / sizeof(double) == sizeof(StepConst<R>) / sizeof(R), "layout");
        for (size_t i = 0; i < sizeof(StepConst<double>) / sizeof(double); ++i) dst[i] = static_cast<R>(src[i]);
        return f;
    }
}

}  // namespace qk
