// C-ABI harness around the QuantKos reference headers (TEST INFRASTRUCTURE, oracle).
//
// Compiled by oracle/ref_harness/Makefile straight from the reference tree
// (include/core/**, include/IO/**) against the host shim in ./shim, once with
// Real = double and once with Real = float (-DQKOS_ENABLE_SINGLE_PRECISION).
// Outputs go to oracle/_ref/.  Used only by tests/, by __graft_entry__.smoke()
// as a checker, and by bench.py's CPU-baseline / reference arm.
//
// Entry points
//   qkref_step_trace   fed-draw trace of SDEScheme<M,S>::evolve_step
//                      (include/core/schemes/markovian/MSchemes.hpp:87-551);
//   qkref_price        the reference's whole pricing path for one UInputs:
//                      MCDispatcher::launch_montecarlo (include/core/engine/Distpatcher.hpp:78)
//                      -> ForwardMCRunner / ForwardBackwardMCRunner -> execute_mc_framework
//                      (include/core/engine/MCEngine.hpp:560-746), OpenMP through the shim;
//   qkref_exact_call   Black-Scholes / Heston / Bates closed forms
//                      (include/core/analytical/{BlackScholes,Heston,Bates}Exact.hpp);
//   qkref_lsm_solve / qkref_laguerre   LSMEngine pieces (include/core/options/LSMAmerican.hpp:157-613);
//   qkref_payoff       PayoffTracker on a fed spot sequence (include/core/options/Payoff.hpp:84-243);
//   qkref_set_threads  thread count of the shim's OpenMP loops (fixes the draw streams);
//   qkref_read_paths   BinReader::read_prices_at_target_time on a .paths file
//                      (include/IO/IOBinary.hpp:260-378).
#include <cstdint>
#include <cstdio>
#include <exception>
#include <iostream>
#include <sstream>
#include <string>

#include <omp.h>

#include "core/schemes/RandNGenerator.hpp"

// ----------------------------------------------------------------------------
// Fed random-number source.  One record per time step: z[3] = {Z1, Z2, Zjump},
// u[umax] = Poisson uniforms in consumption order.
// ----------------------------------------------------------------------------
struct FeedRNG {
    const double *z = nullptr;
    const double *u = nullptr;
    int umax = 0;
    int zi = 0;
    int ui = 0;
    int overflow = 0;
    double drand() {
        if (ui >= umax) { overflow = 1; return 0.0; }
        return u[ui++];
    }
    float frand() { return static_cast<float>(drand()); }
    double normal() { return z[zi < 3 ? zi++ : 2]; }
};

// The first pair drawn in a step is the scheme's (Z1, Z2); the next one is the
// Bates jump normal.  The Bates wrapper names its generator through decltype of
// a reference parameter (MSchemes.hpp:517), so both FeedRNG and FeedRNG& are fed.
namespace quantkos::Engine {
inline RVPair feed_pair(FeedRNG &g, bool skip_second) {
    RVPair p{KT::real_zero, KT::real_zero};
    if (g.zi == 0) {
        p.Z1 = static_cast<KT::Real>(g.z[0]);
        p.Z2 = skip_second ? KT::real_zero : static_cast<KT::Real>(g.z[1]);
        g.zi = 2;
    } else {
        p.Z1 = static_cast<KT::Real>(g.z[2]);
        g.zi = 3;
    }
    return p;
}
template <bool skip_second>
struct NormalPair<FeedRNG, skip_second> {
    RVPair operator()(FeedRNG &g) const { return feed_pair(g, skip_second); }
};
template <bool skip_second>
struct NormalPair<FeedRNG &, skip_second> {
    RVPair operator()(FeedRNG &g) const { return feed_pair(g, skip_second); }
};
}  // namespace quantkos::Engine

#include "core/analytical/BatesExact.hpp"
#include "core/analytical/BlackScholesExact.hpp"
#include "core/analytical/HestonExact.hpp"
#include "core/engine/Distpatcher.hpp"
#include "core/options/LSMAmerican.hpp"
#include "core/options/Payoff.hpp"
#include "core/schemes/markovian/MSchemes.hpp"
#include "IO/IOBinary.hpp"

namespace KC = quantkos::Config;
namespace KE = quantkos::Engine;
namespace KI = quantkos::Implemented;
namespace KT = quantkos::Types;

extern "C" {

// Flat mirror of quantkos::Config::UInputs (include/core/config/Config.hpp:677-775).
typedef struct {
    double S0, v0, r, q;
    int32_t opt_type, opt_right;
    double K, B;
    int32_t model, scheme;
    double kappa, theta, sigma, rho, lambda_j, mu_j, sigma_j;
    double T, dt_in;
    int32_t normalize, n_paths, batch_size, analyze_distribution;
    uint64_t seed;
    int64_t max_vram_mb, max_cpu_ram_mb;
    int32_t greeks_mask;  // bit0 delta+gamma, bit1 vega+vomma, bit2 vanna, bit3 rho, bit4 theta
    int32_t pad_;
    double bump_S_rel, bump_vol_abs, bump_r_abs, bump_T_abs;
} qkref_config;

typedef struct {
    double price, std_error, prob_itm;
    double pct[15];  // p0 p1 p5 p10 p20 p30 p40 p50 p60 p70 p80 p90 p95 p99 p100
    double delta, gamma, vega, vomma, vanna, rho, theta;
    int32_t n_steps;
    int32_t pad_;
    double dt;
    double seconds;
} qkref_result;

int qkref_real_bytes(void) { return static_cast<int>(sizeof(KT::Real)); }

// Threads of the shim's OpenMP loops.  The shim's generator pool has one state per
// thread and the loops use a static schedule, so a fixed thread count makes the
// reference's draws (and so its prices) the same on every machine.
void qkref_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
}
int qkref_get_threads(void) { return omp_get_max_threads(); }
}

namespace {

thread_local std::string g_last_error;

struct SilenceStdout {
    std::ostringstream sink;
    std::streambuf *old;
    SilenceStdout() : old(std::cout.rdbuf(sink.rdbuf())) {}
    ~SilenceStdout() { std::cout.rdbuf(old); }
};

KC::UInputs to_uinputs(const qkref_config &c) {
    KC::UInputs u;
    u.market.S0 = static_cast<KT::Real>(c.S0);
    u.market.v0 = static_cast<KT::Real>(c.v0);
    u.market.r = static_cast<KT::Real>(c.r);
    u.market.q = static_cast<KT::Real>(c.q);
    u.options.opt_type = static_cast<KI::OptType>(c.opt_type);
    u.options.opt_right = static_cast<KI::OptRight>(c.opt_right);
    u.options.StrikePrice = static_cast<KT::Real>(c.K);
    u.options.BarrierPrice = static_cast<KT::Real>(c.B);
    u.model.id_model = static_cast<KI::MathModel>(c.model);
    u.scheme.id_scheme = static_cast<KI::NumScheme>(c.scheme);
    u.model.heston.k = u.model.bates.k = static_cast<KT::Real>(c.kappa);
    u.model.heston.theta = u.model.bates.theta = static_cast<KT::Real>(c.theta);
    u.model.heston.sigma = u.model.bates.sigma = static_cast<KT::Real>(c.sigma);
    u.model.heston.rho = u.model.bates.rho = static_cast<KT::Real>(c.rho);
    u.model.bates.lambda_J = static_cast<KT::Real>(c.lambda_j);
    u.model.bates.mu_J = static_cast<KT::Real>(c.mu_j);
    u.model.bates.sigma_J = static_cast<KT::Real>(c.sigma_j);
    u.time.t_end = static_cast<KT::Real>(c.T);
    u.time.inp_dt = static_cast<KT::Real>(c.dt_in);
    u.mc.normalize_prices = c.normalize != 0;
    u.mc.N_Paths = c.n_paths;
    u.mc.batch_size = c.batch_size;
    u.mc.rng_seed = c.seed;
    u.mc.Max_VRAM_MB = c.max_vram_mb;
    u.mc.Max_CPU_RAM_MB = c.max_cpu_ram_mb;
    u.mc.analyze_risk_neutral_payoff_distribution = c.analyze_distribution != 0;
    u.mc.compute_delta_et_gamma = (c.greeks_mask & 1) != 0;
    u.mc.compute_vega_et_vomma = (c.greeks_mask & 2) != 0;
    u.mc.compute_vanna = (c.greeks_mask & 4) != 0;
    u.mc.compute_rho = (c.greeks_mask & 8) != 0;
    u.mc.compute_theta = (c.greeks_mask & 16) != 0;
    u.mc.spot_price_relative_bump_size = c.bump_S_rel;
    u.mc.volatility_absolute_bump_size = c.bump_vol_abs;
    u.mc.risk_free_rate_absolute_bump_size = c.bump_r_abs;
    u.mc.time_absolute_bump_size = c.bump_T_abs;
    u.output.out_dir = "";
    u.output.filename_paths_out = "";
    u.output.filename_log = "";
    return u;
}

template <KI::MathModel Mdl, KI::NumScheme Sch>
int trace_impl(const KC::UInputs &cfg, const double *z, const double *u, int umax, int n, double *S_out,
               double *v_out, int *n_uniforms) {
    const KE::SDEScheme<Mdl, Sch> scheme(cfg);
    KT::Real S = cfg.market.S0;
    KT::Real v = cfg.market.v0;
    for (int i = 0; i < n; ++i) {
        FeedRNG g;
        g.z = z + 3 * static_cast<size_t>(i);
        g.u = u + static_cast<size_t>(umax) * i;
        g.umax = umax;
        const auto st = scheme.evolve_step(S, v, g);
        if (g.overflow) return 3;
        S = st.S;
        v = st.v;
        S_out[i] = static_cast<double>(S);
        v_out[i] = static_cast<double>(v);
        if (n_uniforms) n_uniforms[i] = g.ui;
    }
    return 0;
}

}  // namespace

extern "C" {

const char *qkref_last_error(void) { return g_last_error.c_str(); }

// Steps (S0, v0) n times with fed draws; dt is taken as T / n (cfg.T, n steps).
int qkref_step_trace(const qkref_config *c, const double *z, const double *u, int umax, int n, double *S_out,
                     double *v_out, int *n_uniforms) {
    try {
        KC::UInputs cfg = to_uinputs(*c);
        cfg.time.N_time_steps = n;
        cfg.time.dt = static_cast<KT::Real>(c->dt_in);
        const int key = c->model * 3 + c->scheme;
        switch (key) {
            case 0: return trace_impl<KI::MathModel::Heston, KI::NumScheme::Euler>(cfg, z, u, umax, n, S_out, v_out, n_uniforms);
            case 1: return trace_impl<KI::MathModel::Heston, KI::NumScheme::ImplicitMilstein>(cfg, z, u, umax, n, S_out, v_out, n_uniforms);
            case 2: return trace_impl<KI::MathModel::Heston, KI::NumScheme::AndersonQE>(cfg, z, u, umax, n, S_out, v_out, n_uniforms);
            case 3: return trace_impl<KI::MathModel::Bates, KI::NumScheme::Euler>(cfg, z, u, umax, n, S_out, v_out, n_uniforms);
            case 4: return trace_impl<KI::MathModel::Bates, KI::NumScheme::ImplicitMilstein>(cfg, z, u, umax, n, S_out, v_out, n_uniforms);
            case 5: return trace_impl<KI::MathModel::Bates, KI::NumScheme::AndersonQE>(cfg, z, u, umax, n, S_out, v_out, n_uniforms);
            default: g_last_error = "unknown model/scheme"; return 1;
        }
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return 2;
    }
}

// Full reference pricing pass (validate + MCDispatcher), stdout silenced.
int qkref_price(const qkref_config *c, qkref_result *out) {
    try {
        SilenceStdout quiet;
        KC::UInputs cfg = to_uinputs(*c);
        cfg.validate();
        const auto t0 = std::chrono::steady_clock::now();
        KE::MCDispatcher disp(cfg);
        const KE::MCResults res = disp.launch_montecarlo();
        const auto t1 = std::chrono::steady_clock::now();
        const auto &p = res.OptionPrice;
        out->price = p.option_price;
        out->std_error = p.standard_error;
        out->prob_itm = p.prob_itm;
        const double pct[15] = {p.p0, p.p1, p.p5, p.p10, p.p20, p.p30, p.p40, p.median,
                                p.p60, p.p70, p.p80, p.p90, p.p95, p.p99, p.p100};
        for (int i = 0; i < 15; ++i) out->pct[i] = pct[i];
        out->delta = res.Greeks.delta;
        out->gamma = res.Greeks.gamma;
        out->vega = res.Greeks.vega;
        out->vomma = res.Greeks.vomma;
        out->vanna = res.Greeks.vanna;
        out->rho = res.Greeks.rho;
        out->theta = res.Greeks.theta;
        out->n_steps = cfg.time.N_time_steps;
        out->dt = cfg.time.dt;
        out->seconds = std::chrono::duration<double>(t1 - t0).count();
        return 0;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return 2;
    }
}

// kind: 0 Black-Scholes (vol = sqrt(v0)), 1 Heston (GL64 on [0, phi_max]), 2 Bates (50-wide GL64 chunks).
int qkref_exact_call(const qkref_config *c, int kind, double phi_max, double *price) {
    try {
        KC::UInputs cfg = to_uinputs(*c);
        cfg.options.opt_type = KI::OptType::European;
        cfg.options.opt_right = KI::OptRight::Call;
        if (kind == 0) {
            *price = static_cast<double>(quantkos::Engine::Analytical::BlackScholes::get_exact_eu_call_option_price(cfg));
        } else if (kind == 1) {
            *price = quantkos::Engine::Analytical::Heston::get_exact_eu_call_option_price(cfg, phi_max > 0 ? phi_max : 100.0);
        } else {
            *price = quantkos::Engine::Analytical::Bates::get_exact_eu_call_option_price(cfg, phi_max > 0 ? phi_max : 8000.0);
        }
        return 0;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return 2;
    }
}

// LSMEngine::solve_system_on_host_cholesky for NBasis in {3,4,5}; M row-major nb x nb.
int qkref_lsm_solve(const double *M, const double *B, double count, int nb, double *C) {
    auto run = [&](auto tag) {
        constexpr size_t NB = decltype(tag)::value;
        quantkos::Engine::LSM::RegressionSums<NB> s;
        s.count = count;
        for (size_t i = 0; i < NB; ++i) {
            s.B(i) = B[i];
            for (size_t j = 0; j < NB; ++j) s.M(i, j) = M[i * NB + j];
        }
        using Eng = quantkos::Engine::LSM::LSMEngine<
            KI::OptRight::Put, NB == 3 ? KI::LSRegressionBasis::LaguerreP02
                                       : (NB == 4 ? KI::LSRegressionBasis::LaguerreP03 : KI::LSRegressionBasis::LaguerreP04)>;
        const auto coef = Eng::solve_system_on_host_cholesky(s);
        for (size_t i = 0; i < NB; ++i) C[i] = coef[i];
        return 0;
    };
    if (nb == 3) return run(std::integral_constant<size_t, 3>{});
    if (nb == 4) return run(std::integral_constant<size_t, 4>{});
    if (nb == 5) return run(std::integral_constant<size_t, 5>{});
    return 1;
}

int qkref_laguerre(double X, int nb, double *L) {
    KT::Real l5[5] = {0, 0, 0, 0, 0};
    if (nb == 3) {
        KT::Real l[3];
        quantkos::Engine::LSM::LaguerreBasis<3>::evaluate(static_cast<KT::Real>(X), l);
        for (int i = 0; i < 3; ++i) l5[i] = l[i];
    } else if (nb == 4) {
        KT::Real l[4];
        quantkos::Engine::LSM::LaguerreBasis<4>::evaluate(static_cast<KT::Real>(X), l);
        for (int i = 0; i < 4; ++i) l5[i] = l[i];
    } else if (nb == 5) {
        quantkos::Engine::LSM::LaguerreBasis<5>::evaluate(static_cast<KT::Real>(X), l5);
    } else {
        return 1;
    }
    for (int i = 0; i < nb; ++i) L[i] = static_cast<double>(l5[i]);
    return 0;
}

}  // extern "C"

namespace {
template <KI::OptType T, KI::OptRight R>
double payoff_impl(const double *S, int n, double S0, double K, double B) {
    KE::PayoffTracker<T, R> tr(static_cast<KT::Real>(S0));
    for (int i = 0; i < n; ++i) tr.track_current_price(static_cast<KT::Real>(S[i]));
    return static_cast<double>(tr.evaluate_final_payoff(static_cast<KT::Real>(S[n - 1]), static_cast<KT::Real>(K),
                                                        static_cast<KT::Real>(B), n));
}
template <KI::OptType T>
double payoff_right(int right, const double *S, int n, double S0, double K, double B) {
    return right == 0 ? payoff_impl<T, KI::OptRight::Call>(S, n, S0, K, B)
                      : payoff_impl<T, KI::OptRight::Put>(S, n, S0, K, B);
}
}  // namespace

extern "C" int qkref_payoff(int type, int right, const double *S, int n, double S0, double K, double B, double *out) {
    if (n < 1) return 1;
    switch (static_cast<KI::OptType>(type)) {
        case KI::OptType::European: *out = payoff_right<KI::OptType::European>(right, S, n, S0, K, B); return 0;
        case KI::OptType::Asian: *out = payoff_right<KI::OptType::Asian>(right, S, n, S0, K, B); return 0;
        case KI::OptType::BarrierUpAndOut: *out = payoff_right<KI::OptType::BarrierUpAndOut>(right, S, n, S0, K, B); return 0;
        case KI::OptType::BarrierDownAndOut: *out = payoff_right<KI::OptType::BarrierDownAndOut>(right, S, n, S0, K, B); return 0;
        case KI::OptType::BarrierUpAndIn: *out = payoff_right<KI::OptType::BarrierUpAndIn>(right, S, n, S0, K, B); return 0;
        case KI::OptType::BarrierDownAndIn: *out = payoff_right<KI::OptType::BarrierDownAndIn>(right, S, n, S0, K, B); return 0;
        case KI::OptType::LookbackFloatingStrike: *out = payoff_right<KI::OptType::LookbackFloatingStrike>(right, S, n, S0, K, B); return 0;
        case KI::OptType::LookbackFixedStrike: *out = payoff_right<KI::OptType::LookbackFixedStrike>(right, S, n, S0, K, B); return 0;
        case KI::OptType::BinaryCashOrNothing: *out = payoff_right<KI::OptType::BinaryCashOrNothing>(right, S, n, S0, K, B); return 0;
        case KI::OptType::BinaryAssetOrNothing: *out = payoff_right<KI::OptType::BinaryAssetOrNothing>(right, S, n, S0, K, B); return 0;
        default: return 1;
    }
}

// BinReader (include/IO/IOBinary.hpp:260-378) on `dir`/`file`: the spot prices of every
// path at time t, in real units (the reader rescales the stored normalised values).
extern "C" int qkref_read_paths(const char *dir, const char *file, double t, double *out, int max_n, int *n_out) {
    try {
        KC::UInputs cfg;
        cfg.output.out_dir = dir;
        cfg.output.filename_paths_out = file;
        quantkos::IO::Binary::BinReader reader(cfg);
        const auto v = reader.read_prices_at_target_time(static_cast<KT::Real>(t));
        const int n = static_cast<int>(v.size());
        *n_out = n;
        for (int i = 0; i < n && i < max_n; ++i) out[i] = static_cast<double>(v[i]);
        return 0;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return 2;
    }
}
