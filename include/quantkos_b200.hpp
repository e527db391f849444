// quantkos_b200.hpp — C++17 wrappers over the C ABI with the reference's names.
//
// A reference user's code keeps its shape:
//   auto cfg = quantkos::Config::Parser::parse("QuantKosConfig.yaml");      // ConfigParser.cpp:36
//   quantkos::Engine::MCDispatcher disp(cfg);                               // Distpatcher.hpp:58
//   quantkos::Engine::MCResults res = disp.launch_montecarlo();             // Distpatcher.hpp:78
//   res.OptionPrice.option_price; res.Greeks.delta; ...                     // MCEngine.hpp:93-135
// Errors are rethrown as in the reference: std::invalid_argument for validation,
// std::runtime_error for everything else (app/main.cpp:95-102 catches both).
#pragma once

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
    qk_contract contract{};
    double dt = 0.0;
    qk_precision precision;
};

}  // namespace Engine
}  // namespace quantkos
