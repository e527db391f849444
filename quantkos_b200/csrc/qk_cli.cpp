// quantkos — command-line driver with the reference's argv contract
// (app/main.cpp:51-110): `quantkos <config.yaml>`; prints the results; exits 1 on
// any error (message on stderr), 0 on success.
#include <cstdio>
#include <exception>
#include <iostream>
#include <string>

#include "quantkos_b200.hpp"

int main(int argc, char **argv) {
    if (argc != 2 || std::string(argv[1]) == "-h" || std::string(argv[1]) == "--help") {
        std::cout << "Usage: quantkos <config.yaml>\n"
                     "  Prices the option described by a QuantKos YAML configuration on the GPU.\n"
                     "  Extra MC keys: Precision (FP64|FP32), Engine (plain|batch), LSM_Basis (Laguerre3|PolySV),\n"
                     "  LSM_Dates (int), Vega_Mode (0|1), Stream (int).\n";
        return argc == 2 ? 0 : 1;
    }
    try {
        quantkos::Config::UInputs cfg = quantkos::Config::Parser::parse(argv[1]);
        quantkos::Engine::MCDispatcher disp(cfg);
        const quantkos::Engine::MCResults res = disp.launch_montecarlo();
        const auto &p = res.OptionPrice;
        std::printf("  ========================================================\n");
        std::printf("                     SIMULATION RESULTS\n");
        std::printf("  ========================================================\n");
        std::printf("   Estimated Option Price   :  %.6f\n", p.option_price);
        std::printf("   Statistical Std Error    :  %.6f\n", p.standard_error);
        std::printf("   Probability of ITM       :  %.6f %%\n", p.prob_itm * 100.0);
        if (cfg.c.analyze_distribution) {
            std::printf("   Min / Median / Max       :  %.6f / %.6f / %.6f\n", p.p0, p.median, p.p100);
            std::printf("   p1 p5 p10 p90 p95 p99    :  %.6f %.6f %.6f %.6f %.6f %.6f\n", p.p1, p.p5, p.p10, p.p90,
                        p.p95, p.p99);
        }
        if (cfg.must_compute_greeks()) {
            const auto &g = res.Greeks;
            std::printf("   Delta %.8g  Gamma %.8g  Vega %.8g  Vomma %.8g\n", g.delta, g.gamma, g.vega, g.vomma);
            std::printf("   Vanna %.8g  Rho %.8g  Theta %.8g\n", g.vanna, g.rho, g.theta);
        }
        std::printf("   Device time              :  %.3f ms (%lld kernel launches, %.4g path-steps)\n",
                    res.Timing.device.device_ms, static_cast<long long>(res.Timing.device.launches),
                    res.Timing.device.path_steps);
        return 0;
    } catch (const std::exception &e) {
        std::cerr << "[ Error ] " << e.what() << "\n";
        return 1;
    }
}
