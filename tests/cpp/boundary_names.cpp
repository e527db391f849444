// The reference's C++ building blocks, composed the way its runners compose them,
// against the fused engine (quantkos_b200.hpp over the C ABI).  Built and run by
// tests/test_gpu_cpp_boundary.py on a GPU; prints one "ok|FAIL <what> <got> <want>"
// line per check and "payoff <type> <right> <value>" lines for the caller to check
// against the oracle; exits 1 if any check failed.
//
// 1. ForwardMCRunner's strategy (include/core/engine/ForwardMC.hpp:91-199) from
//    execute_mc_framework + MSolver::execute_batch + OptionPricer, with all Greeks,
//    equals MCDispatcher::launch_montecarlo (the same paths, merged in another order).
// 2. ForwardBackwardMCRunner::run_backward_phase (ForwardBackwardMC.hpp:204-255) from
//    LSMEngine's statics on the engine's paths equals the fused LSM price.
// 3. SDEScheme::evolve_step with a generator object equals the fed-vector trace.
// 4. PayoffTracker on a fixed sequence, every type and right (values printed).
#include <cmath>
#include <cstdio>
#include <vector>

#include "quantkos_b200.hpp"

namespace I = quantkos::Implemented;
namespace E = quantkos::Engine;
namespace KC = quantkos::Config;

static int g_fails = 0;

static void check_close(const char *what, double got, double want, double rel, double abs_tol) {
    const bool ok = std::fabs(got - want) <= abs_tol + rel * std::fabs(want);
    std::printf("%s %s %.17g %.17g\n", ok ? "ok" : "FAIL", what, got, want);
    if (!ok) ++g_fails;
}

// Deterministic draws for the generator-object test (a 64-bit LCG; Box-Muller).
struct LcgRng {
    uint64_t s = 0x9E3779B97F4A7C15ull;
    double uniform() {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        return (static_cast<double>(s >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    }
    double normal() {
        const double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

static void forward_strategy_equals_dispatcher(E::Device &dev) {
    KC::UInputs cfg;
    qk_config &c = cfg.c;
    c.S0 = 100.0;
    c.v0 = 0.04;
    c.r = 0.03;
    c.q = 0.0;
    c.model = QK_HESTON;
    c.heston_k = 2.0;
    c.heston_theta = 0.04;
    c.heston_sigma = 0.3;
    c.heston_rho = -0.7;
    c.scheme = QK_ANDERSEN_QE;
    c.opt_type = QK_ASIAN;
    c.opt_right = QK_CALL;
    c.K = 100.0;
    c.t_end = 1.0;
    c.inp_dt = 1.0 / 64.0;
    c.n_paths = 120000;
    c.seed = 7;
    c.normalize = 1;
    c.greeks_mask = QK_GREEK_ALL;
    c.bump_S_rel = 0.01;
    c.bump_vol_abs = 0.02;
    c.bump_r_abs = 1e-3;
    c.bump_T_abs = 2.0 / 365.0;
    c.paths_file[0] = '\0';
    cfg.validate();
    const int64_t n = c.n_paths;
    auto strategy = [&](const KC::UInputs &u, E::PathsMCBatchMem &mem) {
        E::MSolver<I::MathModel::Heston, I::NumScheme::AndersonQE, I::OptType::Asian, I::OptRight::Call> solver(u);
        const E::RNGManager rng(u);
        E::OptionPricer pricer(u);
        mem.first_path = 0;
        const int B = 50000;
        for (int64_t done = 0; done < n; done += B) {
            const int nb = static_cast<int>(std::min<int64_t>(B, n - done));
            solver.execute_batch(nb, mem, rng);
            pricer.accumulate_batch_payoffs(mem.d_payoffs, nb);
            mem.first_path += nb;
        }
        pricer.evaluate_option_price();
        return pricer.get_option_price_data();
    };
    const E::MCResults composed = E::execute_mc_framework<E::PathsMCBatchMem>(cfg, strategy);
    const E::MCResults fused = E::MCDispatcher(cfg, dev).launch_montecarlo();
    check_close("forward.price", composed.OptionPrice.option_price, fused.OptionPrice.option_price, 1e-11, 0.0);
    check_close("forward.std_error", composed.OptionPrice.standard_error, fused.OptionPrice.standard_error, 1e-8, 0.0);
    check_close("forward.prob_itm", composed.OptionPrice.prob_itm, fused.OptionPrice.prob_itm, 0.0, 1e-12);
    const double *g1 = &composed.Greeks.delta;
    const double *g2 = &fused.Greeks.delta;
    const char *names[7] = {"delta", "gamma", "vega", "vomma", "vanna", "rho", "theta"};
    for (int i = 0; i < 7; ++i) {
        char what[64];
        std::snprintf(what, sizeof(what), "forward.%s", names[i]);
        check_close(what, g1[i], g2[i], 1e-6, 1e-8);
    }
}

static void backward_statics_equal_fused_lsm(E::Device &dev) {
    KC::UInputs cfg;
    qk_config &c = cfg.c;
    c.S0 = 100.0;
    c.v0 = 0.04;
    c.r = 0.05;
    c.model = QK_HESTON;
    c.heston_k = 2.0;
    c.heston_theta = 0.04;
    c.heston_sigma = 0.3;
    c.heston_rho = -0.7;
    c.scheme = QK_ANDERSEN_QE;
    c.opt_type = QK_AMERICAN;
    c.opt_right = QK_PUT;
    c.K = 110.0;
    c.t_end = 1.0;
    c.inp_dt = 1.0 / 32.0;
    c.n_paths = 60000;
    c.seed = 11;
    c.normalize = 0;
    c.greeks_mask = 0;
    c.paths_file[0] = '\0';
    cfg.validate();
    qk_contract k;
    qk_greeks g;
    quantkos::detail::check(qk_config_to_contract(&c, &k, &g), "contract");
    const int n = static_cast<int>(k.n_paths), T = k.n_steps;
    std::vector<double> S(static_cast<size_t>(n) * T);
    quantkos::detail::check(qk_paths_dump(dev.get(), &k, 0, n, S.data(), nullptr), "qk_paths_dump");
    auto slice = [&](int t) {
        std::vector<double> s(static_cast<size_t>(n));
        for (int p = 0; p < n; ++p) s[static_cast<size_t>(p)] = S[static_cast<size_t>(p) * T + t];
        return s;
    };
    using Eng = E::LSMEngine<I::OptRight::Put>;
    const double disc = std::exp(-c.r * (c.t_end / T));
    std::vector<double> cf;
    Eng::initialize_cashflows(slice(T - 1), cf, c.K);
    for (int t = T - 2; t >= 0; --t) {
        const std::vector<double> st = slice(t);
        const auto co = Eng::perform_cross_paths_regression(st, cf, disc, c.K);
        Eng::update_cashflows(st, cf, co, disc, c.K);
    }
    const double price = Eng::apply_final_discount(cf, disc, c.S0, c.K);
    E::OptionPricer pricer(cfg);
    pricer.accumulate_batch_payoffs(cf, n);
    pricer.evaluate_option_price();
    const E::MCResults fused = E::MCDispatcher(cfg, dev).launch_montecarlo();
    check_close("american.price", price, fused.OptionPrice.option_price, 1e-9, 0.0);
    check_close("american.std_error", pricer.get_option_price_data().standard_error,
                fused.OptionPrice.standard_error, 1e-6, 0.0);
    // the regression pieces: a date's Gram sums solved by the static solver equal the solve
    // inside perform_cross_paths_regression (same sums, same FP64 solve)
    E::RegressionSums<4> sums;
    const std::vector<double> s0 = slice(T - 2);
    std::vector<double> cf0;
    Eng::initialize_cashflows(slice(T - 1), cf0, c.K);
    for (int p = 0; p < n; ++p) {
        const double x = s0[static_cast<size_t>(p)];
        if (c.K - x <= 0.0) continue;
        const double X = x / c.K;
        const double L[4] = {1.0, 1.0 - X, ((0.5 * X - 2.0) * X) + 1.0, (((-1.0 / 6.0 * X + 1.5) * X - 3.0) * X) + 1.0};
        const double y = cf0[static_cast<size_t>(p)] * disc;
        for (int r = 0; r < 4; ++r) {
            sums.B[r] += L[r] * y;
            for (int q = 0; q < 4; ++q) sums.M[r][q] += L[r] * L[q];
        }
        sums.count += 1.0;
    }
    const auto a = Eng::solve_system_on_host_cholesky(sums);
    const auto b = Eng::perform_cross_paths_regression(s0, cf0, disc, c.K);
    for (int i = 0; i < 4; ++i) {
        char what[64];
        std::snprintf(what, sizeof(what), "american.coeff%d", i);
        check_close(what, a.C[i], b.C[i], 1e-7, 1e-10);
    }
}

static void evolve_step_with_generator() {
    KC::UInputs cfg;
    qk_config &c = cfg.c;
    c.S0 = 100.0;
    c.v0 = 0.04;
    c.model = QK_BATES;
    c.bates_k = 2.0;
    c.bates_theta = 0.04;
    c.bates_sigma = 0.3;
    c.bates_rho = -0.7;
    c.bates_lambda = 2.0;
    c.bates_mu = -0.1;
    c.bates_sigma_j = 0.15;
    c.scheme = QK_ANDERSEN_QE;
    c.t_end = 1.0;
    c.inp_dt = 1.0 / 52.0;
    c.n_paths = 10;
    c.paths_file[0] = '\0';
    cfg.validate();
    E::SDEScheme<I::MathModel::Bates, I::NumScheme::AndersonQE> scheme(cfg);
    LcgRng a, b;
    double S = c.S0, v = c.v0;
    std::vector<double> z, u;
    const int umax = 16;
    for (int i = 0; i < 20; ++i) {
        const E::SDEState st = scheme.evolve_step(S, v, a, umax);
        S = st.S;
        v = st.v;
        for (int j = 0; j < 3; ++j) z.push_back(b.normal());
        for (int j = 0; j < umax; ++j) u.push_back(b.uniform());
    }
    const auto trace = scheme.evolve_steps(c.S0, c.v0, z, u, umax);
    check_close("evolve_step.S", S, trace.back().S, 1e-15, 0.0);
    check_close("evolve_step.v", v, trace.back().v, 1e-15, 1e-18);
}

template <I::OptType T, I::OptRight R>
static void payoff_case(const std::vector<double> &seq) {
    E::PayoffTracker<T, R> tr(1.0);
    for (double s : seq) tr.track_current_price(s);
    const double x = tr.evaluate_final_payoff(seq.back(), 1.02, T == I::OptType::BarrierDownAndOut ||
                                                                      T == I::OptType::BarrierDownAndIn
                                                                  ? 0.93
                                                                  : 1.08,
                                              static_cast<int>(seq.size()));
    std::printf("payoff %d %d %.17g\n", static_cast<int>(T), static_cast<int>(R), x);
}

template <I::OptType T>
static void payoff_both(const std::vector<double> &seq) {
    payoff_case<T, I::OptRight::Call>(seq);
    payoff_case<T, I::OptRight::Put>(seq);
}

static void payoff_trackers() {
    // a path that rises through 1.08, falls through 0.93 and ends near the strike
    std::vector<double> seq;
    for (int i = 0; i < 37; ++i) seq.push_back(1.0 + 0.12 * std::sin(0.31 * i) - 0.002 * i);
    std::printf("sequence");
    for (double s : seq) std::printf(" %.17g", s);
    std::printf("\n");
    payoff_both<I::OptType::European>(seq);
    payoff_both<I::OptType::Asian>(seq);
    payoff_both<I::OptType::BarrierUpAndOut>(seq);
    payoff_both<I::OptType::BarrierDownAndOut>(seq);
    payoff_both<I::OptType::BarrierUpAndIn>(seq);
    payoff_both<I::OptType::BarrierDownAndIn>(seq);
    payoff_both<I::OptType::LookbackFloatingStrike>(seq);
    payoff_both<I::OptType::LookbackFixedStrike>(seq);
    payoff_both<I::OptType::BinaryCashOrNothing>(seq);
    payoff_both<I::OptType::BinaryAssetOrNothing>(seq);
}

int main() {
    try {
        E::Device dev(0);
        forward_strategy_equals_dispatcher(dev);
        backward_statics_equal_fused_lsm(dev);
        evolve_step_with_generator();
        payoff_trackers();
    } catch (const std::exception &e) {
        std::printf("FAIL exception %s\n", e.what());
        return 1;
    }
    return g_fails == 0 ? 0 : 1;
}
