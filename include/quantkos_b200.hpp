// quantkos_b200.hpp — C++17 wrappers over the C ABI with the reference's names.
//
// Besides the dispatcher and runners (the fused engine), the reference's building
// blocks are here too — SDEScheme::evolve_step, PayoffTracker, MSolver::execute_batch,
// OptionPricer, LSMEngine's statics and execute_mc_framework — each running the
// engine's own device code for its step, so a caller that composes them as the
// reference's ForwardMCRunner does gets the paths the fused kernels simulate.
//
// A reference user's code keeps its shape:
//   auto cfg = quantkos::Config::Parser::parse("QuantKosConfig.yaml");      // ConfigParser.cpp:36
//   quantkos::Engine::MCDispatcher disp(cfg);                               // Distpatcher.hpp:58
//   quantkos::Engine::MCResults res = disp.launch_montecarlo();             // Distpatcher.hpp:78
//   res.OptionPrice.option_price; res.Greeks.delta; ...                     // MCEngine.hpp:93-135
// Errors are rethrown as in the reference: std::invalid_argument for validation,
// std::runtime_error for everything else (app/main.cpp:95-102 catches both).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "quantkos_b200.h"

namespace quantkos {

namespace Implemented {
enum class OptType {
    European, Asian, BarrierUpAndOut, BarrierDownAndOut, BarrierUpAndIn, BarrierDownAndIn,
    LookbackFloatingStrike, LookbackFixedStrike, BinaryCashOrNothing, BinaryAssetOrNothing, American
};
enum class OptRight { Call, Put };
enum class MathModel { Heston, Bates };
enum class NumScheme { Euler, ImplicitMilstein, AndersonQE };
}  // namespace Implemented

namespace detail {
inline void check(qk_status s, const char *what) {
    if (s == QK_OK) return;
    const std::string msg = std::string(what) + ": " + qk_last_error();
    if (s == QK_ERR_INVALID_ARG || s == QK_ERR_PARSE) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}
}  // namespace detail

namespace Config {

// UInputs (include/core/config/Config.hpp:677-775) as the flat qk_config.
struct UInputs {
    qk_config c;
    UInputs() { qk_config_default(&c); }
    explicit UInputs(const qk_config &raw) : c(raw) {}
    void validate() { detail::check(qk_config_validate(&c), "UInputs::validate"); }
    bool must_compute_greeks() const { return c.greeks_mask != 0; }
    bool requires_paths_allocated() const { return c.paths_file[0] != '\0' || c.opt_type == QK_AMERICAN; }
};

struct Parser {
    static UInputs parse(const std::string &file) {
        qk_config raw;
        detail::check(qk_config_parse_file(file.c_str(), &raw), "Parser::parse");
        return UInputs(raw);
    }
};

}  // namespace Config

namespace Engine {

struct SDEState {
    double S, v;
};

struct MCOpPrices {
    double option_price = -999., standard_error = -999., prob_itm = -999.;
    double p0 = -999., p1 = -999., p5 = -999., p10 = -999., p20 = -999., p30 = -999., p40 = -999., median = -999.,
           p60 = -999., p70 = -999., p80 = -999., p90 = -999., p95 = -999., p99 = -999., p100 = -999.;
    bool is_computed = false;
};

struct MCGreeks {
    double delta = 0.0, gamma = 0.0, vega = 0.0, vomma = 0.0, vanna = 0.0, rho = 0.0, theta = 0.0;
};

struct MCTimer {
    double s_elapsed_total = 0.0, s_elapsed_for_pricing = 0.0, s_elapsed_for_greeks = 0.0;
    qk_timing device{};
};

struct MCResults {
    Config::UInputs MCConfig;
    MCOpPrices OptionPrice;
    MCGreeks Greeks;
    MCTimer Timing;
};

// One device context (Kokkos::initialize + the memory classes in the reference).
class Device {
public:
    explicit Device(int device = 0) {
        qk_handle *h = nullptr;
        detail::check(qk_create(device, &h), "qk_create");
        h_.reset(h);
    }
    qk_handle *get() const { return h_.get(); }
    static Device &shared() {
        static Device d(0);
        return d;
    }

private:
    struct Del {
        void operator()(qk_handle *h) const { qk_destroy(h); }
    };
    std::unique_ptr<qk_handle, Del> h_;
};

class MCDispatcher {
public:
    explicit MCDispatcher(const Config::UInputs &conf, Device &dev = Device::shared()) : config(conf), dev_(dev) {}
    MCDispatcher(const MCDispatcher &) = delete;
    MCDispatcher &operator=(const MCDispatcher &) = delete;

    MCResults launch_montecarlo() {
        qk_result r;
        double pct[15] = {0};
        detail::check(qk_run_config(dev_.get(), &config.c, &r, pct), "MCDispatcher::launch_montecarlo");
        MCResults out{config, {}, {}, {}};
        Config::UInputs validated = config;
        validated.validate();
        out.MCConfig = validated;
        const qk_payoff_result &p = r.p[0];
        out.OptionPrice.option_price = p.price;
        out.OptionPrice.standard_error = p.std_error;
        out.OptionPrice.prob_itm = p.prob_itm;
        if (config.c.analyze_distribution) {
            double *dst[15] = {&out.OptionPrice.p0, &out.OptionPrice.p1, &out.OptionPrice.p5, &out.OptionPrice.p10,
                               &out.OptionPrice.p20, &out.OptionPrice.p30, &out.OptionPrice.p40, &out.OptionPrice.median,
                               &out.OptionPrice.p60, &out.OptionPrice.p70, &out.OptionPrice.p80, &out.OptionPrice.p90,
                               &out.OptionPrice.p95, &out.OptionPrice.p99, &out.OptionPrice.p100};
            for (int i = 0; i < 15; ++i) *dst[i] = pct[i];
        }
        out.OptionPrice.is_computed = true;
        out.Greeks = MCGreeks{p.delta, p.gamma, p.vega, p.vomma, p.vanna, p.rho, p.theta};
        qk_last_timing(dev_.get(), &out.Timing.device);
        out.Timing.s_elapsed_total = out.Timing.device.device_ms * 1e-3;
        out.Timing.s_elapsed_for_pricing = out.Timing.s_elapsed_total;
        return out;
    }

private:
    Config::UInputs config;
    Device &dev_;
};

// ForwardMCRunner / ForwardBackwardMCRunner (ForwardMC.hpp:48-200, ForwardBackwardMC.hpp:68-256):
// the model/scheme/payoff are runtime values of the config here, so one runner covers both.
template <Implemented::MathModel M, Implemented::NumScheme S, Implemented::OptType T, Implemented::OptRight R>
class ForwardMCRunner {
public:
    explicit ForwardMCRunner(Config::UInputs conf) : config(std::move(conf)) {
        config.c.model = static_cast<int32_t>(M);
        config.c.scheme = static_cast<int32_t>(S);
        config.c.opt_type = static_cast<int32_t>(T);
        config.c.opt_right = static_cast<int32_t>(R);
    }
    MCResults run() const { return MCDispatcher(config).launch_montecarlo(); }

private:
    Config::UInputs config;
};

template <Implemented::MathModel M, Implemented::NumScheme S, Implemented::OptRight R>
class ForwardBackwardMCRunner {
public:
    explicit ForwardBackwardMCRunner(Config::UInputs conf) : config(std::move(conf)) {
        config.c.model = static_cast<int32_t>(M);
        config.c.scheme = static_cast<int32_t>(S);
        config.c.opt_type = static_cast<int32_t>(Implemented::OptType::American);
        config.c.opt_right = static_cast<int32_t>(R);
    }
    MCResults run() const { return MCDispatcher(config).launch_montecarlo(); }

private:
    Config::UInputs config;
};

// SDEScheme<M,S> (MSchemes.hpp:49-551): the device step functions driven with fed draws.
template <Implemented::MathModel M, Implemented::NumScheme S>
struct SDEScheme {
    explicit SDEScheme(const Config::UInputs &cfg, qk_precision prec = QK_FP64) : precision(prec) {
        qk_greeks g;
        detail::check(qk_config_to_contract(&cfg.c, &contract, &g), "SDEScheme");
        contract.model = static_cast<int32_t>(M);
        contract.scheme = static_cast<int32_t>(S);
        dt = cfg.c.dt > 0 ? cfg.c.dt : cfg.c.t_end / contract.n_steps;
    }
    // z: n x 3 {Z1, Z2, Zjump}; u: n x umax Poisson uniforms. Returns the n post-step states from (S0, v0).
    std::vector<SDEState> evolve_steps(double S0, double v0, const std::vector<double> &z, const std::vector<double> &u,
                                       int umax) const {
        const int n = static_cast<int>(z.size() / 3);
        qk_contract c = contract;
        c.S0 = S0;
        c.v0 = v0;
        c.T = dt * n;
        std::vector<double> Sv(n), vv(n);
        detail::check(qk_step_trace(precision, &c, z.data(), u.empty() ? nullptr : u.data(), umax, n, Sv.data(), vv.data()),
                      "SDEScheme::evolve_step");
        std::vector<SDEState> out(n);
        for (int i = 0; i < n; ++i) out[i] = SDEState{Sv[i], vv[i]};
        return out;
    }
    // evolve_step(S, v, RNG&) (MSchemes.hpp:49-66): one step from (S, v) with draws taken
    // from `rng`, which provides double normal() and double uniform().  Every step takes
    // exactly three normals (Z1, Z2, then the jump-size normal, used only when a jump
    // occurs) and, under Bates, `umax` uniforms for Knuth's Poisson loop (which reads them
    // in order until the product falls below exp(-lambda dt)).
    template <class RNG>
    SDEState evolve_step(double S_now, double v_now, RNG &rng, int umax = 16) const {
        double z[3] = {rng.normal(), rng.normal(), rng.normal()};
        const int nu = static_cast<int>(M) == QK_BATES ? umax : 0;
        std::vector<double> u(static_cast<size_t>(nu > 0 ? nu : 1), 0.5);
        for (int i = 0; i < nu; ++i) u[static_cast<size_t>(i)] = rng.uniform();
        qk_contract c = contract;
        c.S0 = S_now;
        c.v0 = v_now;
        c.T = dt;
        double So = 0.0, vo = 0.0;
        detail::check(qk_step_trace(precision, &c, z, u.data(), nu, 1, &So, &vo), "SDEScheme::evolve_step");
        return SDEState{So, vo};
    }
    qk_contract contract{};
    double dt = 0.0;
    qk_precision precision;
};

// PayoffTracker<OptType, OptRight> (Payoff.hpp:84-243): running sum / max / min of a path
// and the final payoff, evaluated by the engine's device tracking code on the tracked
// sequence.
template <Implemented::OptType T, Implemented::OptRight R>
struct PayoffTracker {
    explicit PayoffTracker(double S0, qk_precision prec = QK_FP64) : S0_(S0), precision(prec) {}
    void track_current_price(double S) { path_.push_back(S); }
    double evaluate_final_payoff(double S, double Strike, double BarrierPrice, int n_t_steps) const {
        std::vector<double> seq = path_;
        if (seq.empty() || seq.back() != S) seq.push_back(S);
        if (static_cast<int>(seq.size()) != n_t_steps)
            throw std::invalid_argument("PayoffTracker: n_t_steps differs from the tracked steps");
        qk_payoff leg{static_cast<int32_t>(T), static_cast<int32_t>(R), Strike, BarrierPrice};
        double out = 0.0;
        detail::check(qk_payoff_trace(&leg, seq.data(), n_t_steps, S0_, precision, &out),
                      "PayoffTracker::evaluate_final_payoff");
        return out;
    }

private:
    double S0_;
    qk_precision precision;
    std::vector<double> path_;
};

// RNGManager (RandNGenerator.hpp:40-130): the Philox key (MCConfig::rng_seed) and stream;
// the engine's draws are a function of (seed, stream, path, step), so there is no pool state.
struct RNGManager {
    explicit RNGManager(const Config::UInputs &cfg) : seed(cfg.c.seed), stream(cfg.c.stream) {}
    uint64_t seed, stream;
};

// PathsMCBatchMem (PathsMCBatchMem.hpp:330-420): host buffers of one batch of paths.
// first_path is the index of the batch's first path; the runner advances it.
class PathsMCBatchMem {
public:
    explicit PathsMCBatchMem(const Config::UInputs &cfg, Device &dev = Device::shared())
        : config(cfg), dev_(dev), batch_size(cfg.c.batch_size > 0 ? cfg.c.batch_size : cfg.c.n_paths) {
        d_payoffs.resize(static_cast<size_t>(batch_size));
    }
    PathsMCBatchMem(const PathsMCBatchMem &) = delete;
    PathsMCBatchMem &operator=(const PathsMCBatchMem &) = delete;
    Device &device() const { return dev_; }
    Config::UInputs config;
    std::vector<double> d_payoffs;  // per path payoff of the batch (normalised units)
    int64_t first_path = 0;

private:
    Device &dev_;

public:
    int batch_size;
};

// MSolver<M,S,T,R>::execute_batch (MSolver.hpp:173-232): the payoffs of the next
// n_active_sims_in_batch paths, simulated by the engine's path code.
template <Implemented::MathModel M, Implemented::NumScheme S, Implemented::OptType T, Implemented::OptRight R>
class MSolver {
public:
    explicit MSolver(const Config::UInputs &cfg) : config(cfg) {}
    MSolver(const MSolver &) = delete;
    MSolver &operator=(const MSolver &) = delete;
    void execute_batch(int n_active_sims_in_batch, PathsMCBatchMem &BatchMem, const RNGManager &RNGen) const {
        qk_contract c;
        qk_greeks g;
        detail::check(qk_config_to_contract(&config.c, &c, &g), "MSolver");
        c.model = static_cast<int32_t>(M);
        c.scheme = static_cast<int32_t>(S);
        c.payoffs[0].type = static_cast<int32_t>(T);
        c.payoffs[0].right = static_cast<int32_t>(R);
        c.seed = RNGen.seed;
        c.stream = RNGen.stream;
        if (BatchMem.d_payoffs.size() < static_cast<size_t>(n_active_sims_in_batch))
            BatchMem.d_payoffs.resize(static_cast<size_t>(n_active_sims_in_batch));
        detail::check(qk_payoffs_range(BatchMem.device().get(), &c, BatchMem.first_path, n_active_sims_in_batch,
                                       BatchMem.d_payoffs.data()),
                      "MSolver::execute_batch");
    }

private:
    Config::UInputs config;
};

// OptionPricer (OptionPricer.hpp:123-249): batch moments merged with Chan's update in
// FP64, then price = mean * discount * scale and SE = sqrt(M2 / (N - 1) / N) * the same.
class OptionPricer {
public:
    explicit OptionPricer(const Config::UInputs &cfg) : config(cfg) {}
    OptionPricer(const OptionPricer &) = delete;
    OptionPricer &operator=(const OptionPricer &) = delete;
    void accumulate_batch_payoffs(const std::vector<double> &d_payoffs, int curr_batch_size) {
        const double eps = config.c.precision == QK_FP32 ? 1e-6 : 1e-12;
        double sum = 0.0, itm = 0.0;
        for (int i = 0; i < curr_batch_size; ++i) {
            sum += d_payoffs[static_cast<size_t>(i)];
            if (d_payoffs[static_cast<size_t>(i)] > eps) itm += 1.0;
        }
        const double batch_mean = sum / curr_batch_size;
        double m2 = 0.0;
        for (int i = 0; i < curr_batch_size; ++i) {
            const double d = d_payoffs[static_cast<size_t>(i)] - batch_mean;
            m2 += d * d;
        }
        const double n_old = n_, n_new = n_ + curr_batch_size;
        const double delta = batch_mean - mean_;
        mean_ = (mean_ * n_old + batch_mean * curr_batch_size) / n_new;
        m2_ += m2 + delta * delta * (n_old * curr_batch_size / n_new);
        itm_ += itm;
        n_ = n_new;
    }
    void evaluate_option_price() {
        const double N = n_;
        if (N <= 0) throw std::runtime_error("Cannot compute metrics: Invalid number of paths.");
        const bool american = config.c.opt_type == QK_AMERICAN;
        const double disc = american ? 1.0 : std::exp(-config.c.r * config.c.t_end);
        const bool cash = config.c.opt_type == QK_BINARY_CASH;
        const double scale = (config.c.normalize && !cash) ? config.c.S0 : 1.0;
        const double var = N > 1.0 ? m2_ / (N - 1.0) : 0.0;
        metrics.option_price = mean_ * disc * scale;
        metrics.standard_error = std::sqrt(var / N) * disc * scale;
        metrics.prob_itm = itm_ / N;
        metrics.is_computed = true;
    }
    const MCOpPrices &get_option_price_data() const { return metrics; }

private:
    Config::UInputs config;
    double n_ = 0.0, mean_ = 0.0, m2_ = 0.0, itm_ = 0.0;
    MCOpPrices metrics;
};

// LSMEngine<OptRight, Basis> statics (LSMAmerican.hpp:217-614) on host slices of paths,
// each date's work run by the engine's device code (qk_lsm_date / qk_lsm_solve).
enum class LSRegressionBasis { LaguerreP03 = QK_LSM_LAGUERRE3, PolySV = QK_LSM_POLY_SV };
template <size_t NBasis>
struct Coeffs {
    double C[NBasis] = {};
};
template <size_t NBasis>
struct RegressionSums {
    double M[NBasis][NBasis] = {};
    double B[NBasis] = {};
    double count = 0.0;
};

template <Implemented::OptRight R, LSRegressionBasis Basis = LSRegressionBasis::LaguerreP03,
          qk_precision Precision = QK_FP64>
class LSMEngine {
public:
    static constexpr size_t NBasis = Basis == LSRegressionBasis::PolySV ? 6 : 4;
    static void initialize_cashflows(const std::vector<double> &S, std::vector<double> &cf, double strike) {
        cf.resize(S.size());
        run(0, S, nullptr, cf, strike, 1.0, 0.0, 0.0, nullptr);
    }
    // v, cx, cv: variance slice and centring of the {1,S,S^2,S^3,v,Sv} basis (PolySV only)
    static Coeffs<NBasis> perform_cross_paths_regression(const std::vector<double> &S, std::vector<double> &cf,
                                                         double discount_factor, double strike,
                                                         const std::vector<double> *v = nullptr, double cx = 0.0,
                                                         double cv = 0.0) {
        Coeffs<NBasis> out;
        run(1, S, v, cf, strike, discount_factor, cx, cv, out.C);
        return out;
    }
    static void update_cashflows(const std::vector<double> &S, std::vector<double> &cf, const Coeffs<NBasis> &c,
                                 double discount_factor, double strike, const std::vector<double> *v = nullptr,
                                 double cx = 0.0, double cv = 0.0) {
        Coeffs<NBasis> cc = c;
        run(2, S, v, cf, strike, discount_factor, cx, cv, cc.C);
    }
    // exercise today if intrinsic(S0) beats the mean discounted cash flow; the mean is the price
    static double apply_final_discount(std::vector<double> &cf, double discount_factor, double S0, double strike) {
        double total = 0.0;
        for (double &x : cf) {
            x *= discount_factor;
            total += x;
        }
        const double mean = total / static_cast<double>(cf.size());
        const double today = R == Implemented::OptRight::Call ? std::max(S0 - strike, 0.0) : std::max(strike - S0, 0.0);
        if (today > mean) {
            for (double &x : cf) x = today;
            return today;
        }
        return mean;
    }
    static Coeffs<NBasis> solve_system_on_host_cholesky(const RegressionSums<NBasis> &s) {
        std::vector<double> sums;
        for (size_t r = 0; r < NBasis; ++r)
            for (size_t q = r; q < NBasis; ++q) sums.push_back(s.M[r][q]);
        for (size_t r = 0; r < NBasis; ++r) sums.push_back(s.B[r]);
        sums.push_back(s.count);
        Coeffs<NBasis> out;
        int32_t method = 0;
        detail::check(qk_lsm_solve(static_cast<int32_t>(Basis), sums.data(), out.C, &method),
                      "LSMEngine::solve_system_on_host_cholesky");
        return out;
    }

private:
    static void run(int op, const std::vector<double> &S, const std::vector<double> *v, std::vector<double> &cf,
                    double K, double disc, double cx, double cv, double *coeffs) {
        int32_t method = 0;
        detail::check(qk_lsm_date(op, Precision, static_cast<int32_t>(Basis), static_cast<int32_t>(R),
                                  static_cast<int64_t>(S.size()), S.data(), v ? v->data() : nullptr, cf.data(), K, disc,
                                  cx, cv, coeffs, &method),
                      "LSMEngine");
    }
};

// execute_mc_framework<MemoryType>(config, pricing_function) (MCEngine.hpp:560-746): the
// base price, then every requested Greek by repricing bumped configs with the same
// callable and central differences (spot bump relative, in real units; volatility
// sqrt(v0) bumped absolutely; rho central; theta one-sided with the step count kept).
template <class MemoryType, class PricingCallable>
MCResults execute_mc_framework(const Config::UInputs &config, PricingCallable &&pricing_function) {
    MemoryType Mem(config);
    MCResults res{config, {}, {}, {}};
    res.OptionPrice = pricing_function(config, Mem);
    const qk_config &c = config.c;
    if (!config.must_compute_greeks()) return res;
    auto price = [&](const Config::UInputs &cfg) { return pricing_function(cfg, Mem).option_price; };
    const double p0 = res.OptionPrice.option_price;
    const double S0 = c.S0, h_S = S0 * c.bump_S_rel;
    const double vol0 = std::sqrt(c.v0), h_vol = c.bump_vol_abs;
    auto with = [&](double S, double v) {
        Config::UInputs u = config;
        u.c.S0 = S;
        u.c.v0 = v;
        return u;
    };
    if (c.greeks_mask & QK_GREEK_DELTA_GAMMA) {
        const double pu = price(with(S0 + h_S, c.v0)), pd = price(with(S0 - h_S, c.v0));
        res.Greeks.delta = (pu - pd) / (2.0 * h_S);
        res.Greeks.gamma = (pu - 2.0 * p0 + pd) / (h_S * h_S);
    }
    const double v_up = (vol0 + h_vol) * (vol0 + h_vol), v_dn = (vol0 - h_vol) * (vol0 - h_vol);
    if (c.greeks_mask & QK_GREEK_VEGA_VOMMA) {
        const double pu = price(with(S0, v_up)), pd = price(with(S0, v_dn));
        res.Greeks.vega = (pu - pd) / (2.0 * h_vol);
        res.Greeks.vomma = (pu - 2.0 * p0 + pd) / (h_vol * h_vol);
    }
    if (c.greeks_mask & QK_GREEK_RHO) {
        Config::UInputs up = config, dn = config;
        up.c.r += c.bump_r_abs;
        dn.c.r -= c.bump_r_abs;
        res.Greeks.rho = (price(up) - price(dn)) / (2.0 * c.bump_r_abs);
    }
    if (c.greeks_mask & QK_GREEK_THETA) {
        if (c.t_end > c.bump_T_abs) {
            Config::UInputs dn = config;
            dn.c.t_end = c.t_end - c.bump_T_abs;
            dn.c.dt = dn.c.t_end / c.n_steps;  // the step count is kept, the step shrinks
            dn.c.inp_dt = dn.c.dt;
            res.Greeks.theta = (price(dn) - p0) / c.bump_T_abs;
        }
    }
    if (c.greeks_mask & QK_GREEK_VANNA) {
        const double uu = price(with(S0 + h_S, v_up)), du = price(with(S0 - h_S, v_up));
        const double ud = price(with(S0 + h_S, v_dn)), dd = price(with(S0 - h_S, v_dn));
        res.Greeks.vanna = (uu - du - ud + dd) / (4.0 * h_S * h_vol);
    }
    return res;
}

}  // namespace Engine
}  // namespace quantkos
