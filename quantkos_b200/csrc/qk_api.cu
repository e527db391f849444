// C ABI of the B200 engine: handle lifecycle, contract validation, task and
// tile planning (base prices + finite-difference Greek bumps under common random
// numbers), launch sequencing on the handle's stream, and FP64 result assembly.
//
// Reference pieces replaced (paths relative to the reference project):
//   execute_mc_framework + Greeks    include/core/engine/MCEngine.hpp:560-746
//   ForwardMCRunner::run             include/core/engine/ForwardMC.hpp:91-199
//   OptionPricer::evaluate_option_price   include/core/options/OptionPricer.hpp:204-249
//   UInputs::apply_price_scaling     include/core/config/Config.hpp:710-723
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "qk_engine.h"
#include "qk_host.h"
#include "qk_kernels.h"

namespace qk {

thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }
qk_status fail(qk_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

#define QK_CUDA_TRY(call)                                                                          \
    do {                                                                                           \
        const cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                                     \
            return ::qk::fail(e_ == cudaErrorMemoryAllocation ? QK_ERR_OUT_OF_MEMORY : QK_ERR_CUDA, \
                              std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

// ---------------------------------------------------------------- validation
static std::string field(const char *block, const char *key, const char *msg) {
    return std::string("[") + block + "." + key + "] " + msg;
}

qk_status validate_contract(const qk_contract &c, const qk_greeks *g) {
    // MarketConfig::validate (Config.hpp:63-84)
    if (!(c.S0 > 0.0)) return fail(QK_ERR_INVALID_ARG, field("Market", "Price", "must be positive."));
    if (!(c.v0 >= 0.0)) return fail(QK_ERR_INVALID_ARG, field("Market", "Variance", "must be positive."));
    if (!(c.q >= 0.0)) return fail(QK_ERR_INVALID_ARG, field("Market", "q", "Dividend yield (q) cannot be negative."));
    if (!(std::fabs(c.r) <= 0.5))
        return fail(QK_ERR_INVALID_ARG,
                    field("Market", "r", "Risk-free rate (r) is unphysical (keep between -50% and +50%)."));
    if (c.q > 0.8) return fail(QK_ERR_INVALID_ARG, field("Market", "q", "Dividend yield (q) is unphysical (keep under 80%)."));
    // MathModelConfig::validate (Config.hpp:198-305)
    if (c.model != QK_HESTON && c.model != QK_BATES)
        return fail(QK_ERR_INVALID_ARG, field("Model", "Model", "Model selected is not a valid model !"));
    if (c.scheme < QK_EULER || c.scheme > QK_ANDERSEN_QE)
        return fail(QK_ERR_UNSUPPORTED, "SDESolver math kernel not yet implemented for this scheme combination!");
    if (!(c.kappa >= 0.0)) return fail(QK_ERR_INVALID_ARG, "[Model Config] kappa must be positive.");
    if (!(c.theta >= 0.0)) return fail(QK_ERR_INVALID_ARG, "[Model Config] theta must be positive.");
    if (!(c.sigma >= 0.0)) return fail(QK_ERR_INVALID_ARG, "[Model Config] sigma must be positive.");
    if (!(c.rho >= -1.0 && c.rho <= 1.0)) return fail(QK_ERR_INVALID_ARG, "[Model Config] rho must fall within [-1.0, 1.0].");
    if (c.model == QK_BATES) {
        if (!(c.lambda_j >= 0.0)) return fail(QK_ERR_INVALID_ARG, "[Model Config] Bates: Jump intensity (lambda) cannot be negative.");
        if (!(c.sigma_j >= 0.0)) return fail(QK_ERR_INVALID_ARG, "[Model Config] Bates: Jump volatility (sigmaJ) must be positive.");
    }
    // TimeConfig::validate (Config.hpp:347-373); n_steps is ceil(T/dt) computed by the caller
    if (!(c.T > 0.0)) return fail(QK_ERR_INVALID_ARG, field("Time", "T_End", "must be positive."));
    if (c.n_steps < 1 || c.n_steps > (1 << 28)) return fail(QK_ERR_INVALID_ARG, field("Time", "N_TSteps", "must be in [1, 2^28]."));
    if (c.model == QK_BATES && c.lambda_j * (c.T / c.n_steps) > kMaxLambdaDt)
        return fail(QK_ERR_INVALID_ARG, "[Model Config] Bates: lambda*dt above 512 is not supported by the bounded Poisson draw.");
    // MCConfig::validate (Config.hpp:442-472)
    if (c.n_paths < 1) return fail(QK_ERR_INVALID_ARG, field("MC", "N_Paths", "Must be a positive integer."));
    if (c.n_paths > 0xFFFFFFFFLL) return fail(QK_ERR_INVALID_ARG, field("MC", "N_Paths", "at most 2^32 - 1 paths per contract (32-bit Philox path counter)."));
    if (c.seed == 0) return fail(QK_ERR_INVALID_ARG, field("MC", "RNG_Seed", "The random number seed cannot be 0."));
    if (c.precision != QK_FP32 && c.precision != QK_FP64) return fail(QK_ERR_INVALID_ARG, "precision must be QK_FP32 or QK_FP64");
    if (c.n_payoffs < 1 || c.n_payoffs > QK_MAX_PAYOFFS) return fail(QK_ERR_INVALID_ARG, "n_payoffs must be in [1, 8]");
    bool american = false;
    for (int k = 0; k < c.n_payoffs; ++k) {
        const qk_payoff &p = c.payoffs[k];
        if (p.type < QK_EUROPEAN || p.type > QK_AMERICAN) return fail(QK_ERR_INVALID_ARG, field("Options", "OptionType", "invalid value"));
        if (p.right != QK_CALL && p.right != QK_PUT) return fail(QK_ERR_INVALID_ARG, field("Options", "OptionRight", "invalid value"));
        // OptionsConfig::validate (Config.hpp:119-137)
        if (!(p.strike > 0.0)) return fail(QK_ERR_INVALID_ARG, field("Options", "StrikePrice", "must be positive."));
        if (p.strike < c.S0 * 0.0001)
            return fail(QK_ERR_INVALID_ARG, "Config Error: Strike price (K) is too close to zero. Must be at least 1000 times smaller than the initial asset price (S0) to prevent numerical problems.");
        if (p.strike > c.S0 * 10000.0)
            return fail(QK_ERR_INVALID_ARG, "Config Error: Strike price (K) is absurdly high (exceeds 10000x of S0). This will likely result in zero-variance path generation and statistical breakdown.");
        if (p.type == QK_AMERICAN) american = true;
    }
    if (c.antithetic != 0 && c.antithetic != 1) return fail(QK_ERR_INVALID_ARG, "antithetic must be 0 or 1");
    if (c.antithetic && (c.n_paths % 2) != 0)
        return fail(QK_ERR_INVALID_ARG, field("MC", "N_Paths", "must be even for antithetic sampling."));
    if (c.antithetic && american)
        return fail(QK_ERR_UNSUPPORTED, "antithetic sampling covers forward payoff legs only (not American)");
    if (american) {
        if (c.n_payoffs != 1) return fail(QK_ERR_INVALID_ARG, "an American contract carries exactly one payoff leg");
        if (c.lsm_basis != QK_LSM_LAGUERRE3 && c.lsm_basis != QK_LSM_POLY_SV) return fail(QK_ERR_INVALID_ARG, "lsm_basis invalid");
        if (c.lsm_dates < 0 || c.lsm_dates > c.n_steps) return fail(QK_ERR_INVALID_ARG, "lsm_dates must be in [0, n_steps]");
        if (c.lsm_dates > 0 && c.n_steps % c.lsm_dates != 0) return fail(QK_ERR_INVALID_ARG, "lsm_dates must divide n_steps");
    }
    // MCConfig::validate_bump_sizes_for_greeks_computations (Config.hpp:493-563)
    if (g && g->mask) {
        if (g->mask & ~QK_GREEK_ALL) return fail(QK_ERR_INVALID_ARG, "unknown Greek bits");
        if (g->mask & (QK_GREEK_DELTA_GAMMA | QK_GREEK_VANNA)) {
            if (!(g->bump_S_rel > 0.0 && g->bump_S_rel <= 0.05))
                return fail(QK_ERR_INVALID_ARG, field("MC", "spot_price_relative_bump_size", "must be strictly positive and <= 5% (0.05)."));
        }
        if (g->mask & (QK_GREEK_VEGA_VOMMA | QK_GREEK_VANNA)) {
            if (g->vega_mode == 0) {
                const double vol0 = std::sqrt(c.v0);
                if (!(g->bump_vol > 0.0 && g->bump_vol <= vol0))
                    return fail(QK_ERR_INVALID_ARG, field("MC", "volatility_absolute_bump_size",
                                                         "must be strictly positive and and strictly smaller than sqrt(v0) when Vega/Vomma or Vanna is requested"));
            } else if (g->vega_mode == 1) {
                if (!(g->bump_vol > 0.0 && g->bump_vol < 1.0))
                    return fail(QK_ERR_INVALID_ARG, "relative v0 bump must be in (0, 1)");
            } else {
                return fail(QK_ERR_INVALID_ARG, "vega_mode must be 0 or 1");
            }
        }
        if (g->mask & QK_GREEK_RHO) {
            if (!(g->bump_r_abs > 0.0 && g->bump_r_abs <= 0.05))
                return fail(QK_ERR_INVALID_ARG, field("MC", "risk_free_rate_absolute_bump_size", "must be strictly positive and <= 0.05."));
        }
        if (g->mask & QK_GREEK_THETA) {
            if (!(g->bump_T_abs > 0.0 && g->bump_T_abs < c.T))
                return fail(QK_ERR_INVALID_ARG, field("MC", "time_absolute_bump_size",
                                                     "must be strictly positive and strictly smaller than T_End (t_end) when Theta is requested."));
        }
    }
    return QK_OK;
}

// ---------------------------------------------------------------- task building
// Bump roles of execute_mc_framework (MCEngine.hpp:586-730).
enum Role : int { kBase = 0, kSUp, kSDn, kVolUp, kVolDn, kRUp, kRDn, kTDn, kUU, kDU, kUD, kDD };
static_assert(kDD + 1 == kNumRoles, "role count");

// Normalised copy (UInputs::apply_price_scaling) and the factor results are scaled back by.
qk_contract normalised(const qk_contract &c, double *scale) {
    qk_contract n = c;
    *scale = 1.0;
    if (c.normalize) {
        *scale = c.S0;
        n.S0 = 1.0;
        for (int k = 0; k < c.n_payoffs; ++k) {
            n.payoffs[k].strike = c.payoffs[k].strike / c.S0;
            n.payoffs[k].barrier = c.payoffs[k].barrier / c.S0;
        }
    }
    return n;
}

// The bumped contract for `role`, with the spot bump h_S in (normalised) spot units.
qk_contract bumped(const qk_contract &n, const qk_greeks *g, int role) {
    qk_contract b = n;
    if (role == kBase || !g) return b;
    const double h_S = n.S0 * g->bump_S_rel;
    double v_up = n.v0, v_dn = n.v0;
    if (g->vega_mode == 0) {
        const double vol0 = std::sqrt(n.v0);
        v_up = (vol0 + g->bump_vol) * (vol0 + g->bump_vol);
        v_dn = (vol0 - g->bump_vol) * (vol0 - g->bump_vol);
    } else {
        v_up = n.v0 * (1.0 + g->bump_vol);
        v_dn = n.v0 * (1.0 - g->bump_vol);
    }
    switch (role) {
        case kSUp: b.S0 = n.S0 + h_S; break;
        case kSDn: b.S0 = n.S0 - h_S; break;
        case kVolUp: b.v0 = v_up; break;
        case kVolDn: b.v0 = v_dn; break;
        case kRUp: b.r = n.r + g->bump_r_abs; break;
        case kRDn: b.r = n.r - g->bump_r_abs; break;
        case kTDn: b.T = n.T - g->bump_T_abs; break;  // N_time_steps kept, dt shrinks (MCEngine.hpp:656-673)
        case kUU: b.S0 = n.S0 + h_S; b.v0 = v_up; break;
        case kDU: b.S0 = n.S0 - h_S; b.v0 = v_up; break;
        case kUD: b.S0 = n.S0 + h_S; b.v0 = v_dn; break;
        case kDD: b.S0 = n.S0 - h_S; b.v0 = v_dn; break;
        default: break;
    }
    return b;
}

std::vector<int> roles_for(const qk_greeks *g, double T) {
    std::vector<int> roles{kBase};
    if (!g) return roles;
    if (g->mask & QK_GREEK_DELTA_GAMMA) { roles.push_back(kSUp); roles.push_back(kSDn); }
    if (g->mask & QK_GREEK_VEGA_VOMMA) { roles.push_back(kVolUp); roles.push_back(kVolDn); }
    if (g->mask & QK_GREEK_RHO) { roles.push_back(kRUp); roles.push_back(kRDn); }
    if ((g->mask & QK_GREEK_THETA) && T > g->bump_T_abs) roles.push_back(kTDn);
    if (g->mask & QK_GREEK_VANNA) { roles.push_back(kUU); roles.push_back(kDU); roles.push_back(kUD); roles.push_back(kDD); }
    return roles;
}

// Asian, barrier and lookback legs read the running sum, max or min of the path;
// European, binary and American legs only its final spot.
static bool needs_path_state(const qk_contract &c) {
    for (int k = 0; k < c.n_payoffs; ++k)
        if (c.payoffs[k].type >= QK_ASIAN && c.payoffs[k].type <= QK_LOOKBACK_FIXED) return true;
    return false;
}

TaskDev make_task(const qk_contract &b, int ppt, int lane_mode) {
    TaskDev t;
    std::memset(&t, 0, sizeof(t));
    const double dt = b.T / b.n_steps;
    t.cf = make_step_const<float>(b, dt, 1e-6);
    t.cd = make_step_const<double>(b, dt, 1e-12);
    t.S0 = b.S0;
    t.v0 = b.v0;
    t.model = b.model;
    t.scheme = b.scheme;
    t.n_steps = b.n_steps;
    t.n_payoffs = b.n_payoffs;
    t.precision = b.precision;
    t.key0 = static_cast<uint32_t>(b.seed & 0xFFFFFFFFull);
    t.key1 = static_cast<uint32_t>(b.seed >> 32);
    t.stream = static_cast<uint32_t>(b.stream);
    t.n_paths = b.n_paths;
    t.ppt = ppt;
    // FP32 jump test on the raw word: u01(w) = ((w >> 9) + 1/2) 2^-23 >= L  <=>  (w >> 9) >= kmin
    const float Lf = t.cf.exp_m_lambda_dt;
    const double kd = std::ceil(static_cast<double>(Lf) * 8388608.0 - 0.5);
    t.jump_kmin = static_cast<uint32_t>(std::min(std::max(kd, 0.0), 8388608.0));
    t.lane_mode = b.antithetic ? kLanePair : lane_mode;
    t.track = needs_path_state(b) ? 1 : 0;
    const int64_t units = lane_units(b.n_paths, t.lane_mode);
    const int64_t tile_units = static_cast<int64_t>(kWarpTilePaths) * ppt;
    t.n_tiles = static_cast<int32_t>((units + tile_units - 1) / tile_units);
    t.n_big = t.n_tiles;  // uniform tiles unless split_tail is applied
    t.ppt_tail = ppt;
    for (int k = 0; k < b.n_payoffs; ++k) {
        t.pay[k].type = b.payoffs[k].type;
        t.pay[k].right = b.payoffs[k].right;
        t.pay[k].K = b.payoffs[k].strike;
        t.pay[k].B = b.payoffs[k].barrier;
    }
    return t;
}

// Guided tail for a task that fills the GPU many times over on its own: big tiles
// of 2 x ppt rounds first, then the last rounds (about half a big tile per warp
// slot) in tiles of a quarter of ppt.  Warps that finish their last big tile early
// take short tail tiles, so all warps end within a short tile of each other; the
// record count stays below that of uniform ppt-round tiles.
static void split_tail(TaskDev &t, int64_t warp_slots) {
    const int64_t units = lane_units(t.n_paths, t.lane_mode);
    const int64_t rounds = (units + kWarpTilePaths - 1) / kWarpTilePaths;
    if (t.ppt < 4 || rounds < 4 * warp_slots * static_cast<int64_t>(t.ppt)) return;
    const int big = 2 * t.ppt;
    const int tail = std::max(1, t.ppt / 4);
    const int64_t tail_target = warp_slots * big / 2;
    const int64_t n_big = (rounds - tail_target) / big;
    const int64_t tail_rounds = rounds - n_big * big;
    t.ppt = big;
    t.ppt_tail = tail;
    t.n_big = static_cast<int32_t>(n_big);
    t.n_tiles = static_cast<int32_t>(n_big + (tail_rounds + tail - 1) / tail);
}

// Relative device cost of one path-step (QE and jumps cost more SFU work).
static double step_cost(const TaskDev &t) {
    double c = 1.0;
    if (t.scheme == QK_ANDERSEN_QE) c *= 1.6;
    if (t.model == QK_BATES) c *= 1.25;
    if (t.precision == QK_FP64) c *= 6.0;
    if (t.lane_mode == kLanePair) c *= 1.7;  // two paths per lane, one set of draws
    if (t.lane_mode == kLaneTwo) c *= 2.0;
    return c;
}

// The plain method's launch shape (one task per launch; not tuned).
constexpr int kPlainTilesPerWarp = 24;

// Rounds per warp tile: enough tiles to keep every warp slot of the GPU busy
// several times over, few enough that per-tile records stay negligible.
int choose_ppt(int64_t n_paths, int64_t total_paths_all, int sm_count, int tiles_per_warp) {
    const int64_t target_tiles = static_cast<int64_t>(sm_count) * 32 * tiles_per_warp;
    int64_t ppt = total_paths_all / (target_tiles * kWarpTilePaths);
    ppt = std::max<int64_t>(1, std::min<int64_t>(ppt, 64));
    const int64_t need = (n_paths + kWarpTilePaths - 1) / kWarpTilePaths;
    ppt = std::min<int64_t>(ppt, std::max<int64_t>(1, need));
    return static_cast<int>(ppt);
}

// ---------------------------------------------------------------- the device pool
namespace {
std::mutex g_pool_mu;
size_t g_pool_keep[64] = {};  // bytes the live servers hold in each device's pool
}  // namespace

qk_status pool_reserve(int device, cudaStream_t s, size_t bytes) {
    if (bytes == 0) return QK_OK;
    if (device < 0 || device >= 64) return fail(QK_ERR_INVALID_ARG, "device index out of range");
    void *p = nullptr;
    if (cudaMallocAsync(&p, bytes, s) != cudaSuccess) {
        cudaGetLastError();
        return fail(QK_ERR_CAPACITY, "cannot reserve " + std::to_string(bytes >> 20) + " MiB in the device pool");
    }
    QK_CUDA_TRY(cudaFreeAsync(p, s));
    QK_CUDA_TRY(cudaStreamSynchronize(s));
    std::lock_guard<std::mutex> lk(g_pool_mu);
    g_pool_keep[device] += bytes;
    return QK_OK;
}

void pool_release(int device, size_t bytes) {
    if (device < 0 || device >= 64) return;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        g_pool_keep[device] -= std::min(bytes, g_pool_keep[device]);
    }
    pool_trim(device);
}

void pool_trim(int device) {
    if (device < 0 || device >= 64) return;
    cudaMemPool_t pool;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, g_pool_keep[device]);
}

// ---------------------------------------------------------------- device arenas
qk_status DevArena::ensure(size_t bytes) {
    if (bytes <= cap) return QK_OK;
    const size_t want = std::max<size_t>({bytes, cap + cap / 2, 4096});
    if (stream) {
        if (ptr) cudaFreeAsync(ptr, stream);
        ptr = nullptr;
        cap = 0;
        QK_CUDA_TRY(cudaMallocAsync(&ptr, want, stream));
    } else {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
        QK_CUDA_TRY(cudaMalloc(&ptr, want));
    }
    cap = want;
    return QK_OK;
}
void DevArena::release() {
    if (ptr) {
        if (stream) cudaFreeAsync(ptr, stream);
        else cudaFree(ptr);
    }
    ptr = nullptr;
    cap = 0;
}
qk_status HostArena::ensure(size_t bytes) {
    if (bytes <= cap) return QK_OK;
    const size_t want = std::max<size_t>({bytes, cap + cap / 2, size_t(1) << 20});
    if (ptr) retired.push_back(ptr);  // freed by release(): no device-wide synchronization here
    ptr = nullptr;
    cap = 0;
    QK_CUDA_TRY(cudaMallocHost(&ptr, want));
    cap = want;
    return QK_OK;
}
void HostArena::release() {
    if (ptr) cudaFreeHost(ptr);
    for (void *r : retired) cudaFreeHost(r);
    retired.clear();
    ptr = nullptr;
    cap = 0;
}

// ---------------------------------------------------------------- forward plan
// Build the task list of a set of contracts; tasks are grouped by precision and
// ordered by decreasing tile cost (longest-processing-time-first), tile ranges
// and per-tile record offsets assigned in that order.
qk_status build_plan(qk_handle *h, const qk_contract *cs, int32_t n, const qk_greeks *gs, bool plain, Plan &plan) {
    plan = Plan{};
    plan.greeks.resize(n);
    for (int i = 0; i < n; ++i) {
        if (gs && gs[i].mask) plan.greeks[i] = gs[i];
        else std::memset(&plan.greeks[i], 0, sizeof(qk_greeks));
    }
    plan.n_contracts = n;
    plan.scale.resize(n);
    plan.norm.resize(n);
    plan.status.assign(n, QK_OK);
    plan.task_of.assign(static_cast<size_t>(n) * kNumRoles, -1);
    // paths per kernel kind (precision, model, scheme): each kind is one launch
    int64_t kind_paths[2][2][3][3][2] = {};  // [precision][model][scheme][lane mode][track]: lane units per launch
    auto lane_mode_of = [&](const qk_contract &c, int pr) {
        if (c.antithetic) return static_cast<int>(kLanePair);
        if (plain) return static_cast<int>(kLaneOne);
        return h->tune_lanes[pr][c.model][c.scheme] == 2 ? static_cast<int>(kLaneTwo) : static_cast<int>(kLaneOne);
    };
    for (int i = 0; i < n; ++i) {
        const qk_greeks *g = plan.g_of(i);
        const qk_status s = validate_contract(cs[i], g);
        if (s != QK_OK) return fail(s, "contract " + std::to_string(i) + ": " + g_last_error);
        plan.norm[i] = normalised(cs[i], &plan.scale[i]);
        if (plain) plan.norm[i].precision = QK_FP64;
        if (cs[i].payoffs[0].type == QK_AMERICAN) {
            plan.american.push_back(i);
            continue;
        }
        const int pr = plain ? QK_FP64 : cs[i].precision;
        const int lm = lane_mode_of(cs[i], pr);
        kind_paths[pr][cs[i].model][cs[i].scheme][lm][needs_path_state(cs[i])] +=
            lane_units(cs[i].n_paths, lm) * static_cast<int64_t>(roles_for(g, cs[i].T).size());
    }
    struct Item {
        TaskDev t;
        int contract, role;
        double cost;
    };
    std::vector<Item> items;
    for (int i = 0; i < n; ++i) {
        if (cs[i].payoffs[0].type == QK_AMERICAN) continue;
        const int pr = plain ? QK_FP64 : cs[i].precision;
        const int lm = lane_mode_of(cs[i], pr);
        const int64_t units = lane_units(cs[i].n_paths, lm);
        const bool trk = needs_path_state(cs[i]);
        const int64_t launch_units = plain ? units : kind_paths[pr][cs[i].model][cs[i].scheme][lm][trk];
        const int ppt = choose_ppt(units, launch_units, h->sm_count,
                                   plain ? kPlainTilesPerWarp : h->tune_tpw[pr][cs[i].model][cs[i].scheme]);
        const bool tail = !plain && h->tune_tail[pr][cs[i].model][cs[i].scheme];
        const int blk = plain ? kPathBlock : h->tune_block[pr][cs[i].model][cs[i].scheme];
        const int64_t warp_slots = static_cast<int64_t>(h->sm_count) *
                                   price_tiles_max_blocks_per_sm(pr, cs[i].model, cs[i].scheme, lm, trk, blk) *
                                   (blk / 32);
        const qk_greeks *g = plan.g_of(i);
        for (int role : roles_for(g, cs[i].T)) {
            const qk_contract b = bumped(plan.norm[i], g, role);
            Item it{make_task(b, ppt, lm), i, role, 0.0};
            if (tail) split_tail(it.t, warp_slots);
            it.cost = step_cost(it.t) * b.n_steps * b.n_payoffs * 0.02 + step_cost(it.t) * b.n_steps;
            items.push_back(it);
        }
    }
    if (!plain) {
        // group by kernel (precision, lane mode, path state, model, scheme); longest tiles
        // first inside a group
        std::stable_sort(items.begin(), items.end(), [](const Item &a, const Item &b) {
            if (a.t.precision != b.t.precision) return a.t.precision < b.t.precision;
            if (a.t.lane_mode != b.t.lane_mode) return a.t.lane_mode < b.t.lane_mode;
            if (a.t.track != b.t.track) return a.t.track > b.t.track;
            if (a.t.model != b.t.model) return a.t.model < b.t.model;
            if (a.t.scheme != b.t.scheme) return a.t.scheme < b.t.scheme;
            return a.cost > b.cost;
        });
    }
    int64_t slot = 0, rec = 0, chunk = 0;
    for (size_t k = 0; k < items.size(); ++k) {
        TaskDev &t = items[k].t;
        t.tile_begin = slot;
        t.partial_base = rec;
        t.chunk_base = chunk;
        t.n_chunks = (t.n_tiles + kMergeChunkTiles - 1) / kMergeChunkTiles;
        slot += t.n_tiles;
        rec += static_cast<int64_t>(t.n_tiles) * t.n_payoffs;
        chunk += t.n_chunks;
        plan.tasks.push_back(t);
        plan.task_contract.push_back(items[k].contract);
        plan.task_role.push_back(items[k].role);
        plan.task_of[static_cast<size_t>(items[k].contract) * kNumRoles + items[k].role] = static_cast<int>(k);
        plan.path_steps += static_cast<double>(t.n_paths) * t.n_steps;
    }
    plan.total_slots = slot;
    plan.total_records = rec;
    plan.total_chunks = chunk;
    plan.plain = plain;
    return QK_OK;
}

// Device arenas for the plan and the copy of its task descriptors and tile
// prefix to the device.
static qk_status upload_plan(qk_handle *h, const Plan &plan) {
    const size_t nt = plan.tasks.size();
    qk_status s;
    if ((s = h->d_tasks.ensure(nt * sizeof(TaskDev))) != QK_OK) return s;
    if ((s = h->d_prefix.ensure(nt * sizeof(int64_t))) != QK_OK) return s;
    if ((s = h->d_partials.ensure(static_cast<size_t>(plan.total_records) * sizeof(Moments))) != QK_OK) return s;
    if ((s = h->d_moments.ensure(nt * QK_MAX_PAYOFFS * sizeof(Moments))) != QK_OK) return s;
    if ((s = h->d_chunks.ensure(static_cast<size_t>(plan.total_chunks) * QK_MAX_PAYOFFS * sizeof(Moments))) != QK_OK)
        return s;
    if ((s = h->d_cursor.ensure(nt * sizeof(unsigned long long))) != QK_OK) return s;
    if ((s = h->h_tasks.ensure(nt * sizeof(TaskDev) + nt * sizeof(int64_t))) != QK_OK) return s;
    if ((s = h->h_moments.ensure(nt * QK_MAX_PAYOFFS * sizeof(Moments))) != QK_OK) return s;
    TaskDev *ht = static_cast<TaskDev *>(h->h_tasks.ptr);
    int64_t *hp = reinterpret_cast<int64_t *>(ht + nt);
    std::memcpy(ht, plan.tasks.data(), nt * sizeof(TaskDev));
    for (size_t i = 0; i < nt; ++i) hp[i] = plan.tasks[i].tile_begin;
    QK_CUDA_TRY(cudaMemcpyAsync(h->d_tasks.ptr, ht, nt * sizeof(TaskDev), cudaMemcpyHostToDevice, h->stream));
    QK_CUDA_TRY(cudaMemcpyAsync(h->d_prefix.ptr, hp, nt * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream));
    return QK_OK;
}

// The steady part of a run: clear the queue cursors, launch the path kernels
// (one persistent launch per kernel kind for the batched engine, one launch per
// task for the plain method), merge the tile moments and copy them to the host.
// `capture`: the stream is being captured into a graph, so the timing events
// are recorded as external event nodes of that graph.
static qk_status enqueue_plan(qk_handle *h, const Plan &plan, bool capture) {
    const size_t nt = plan.tasks.size();
    const unsigned ev_flags = capture ? cudaEventRecordExternal : cudaEventRecordDefault;
    QK_CUDA_TRY(cudaMemsetAsync(h->d_cursor.ptr, 0, nt * sizeof(unsigned long long), h->stream));
    QK_CUDA_TRY(cudaEventRecordWithFlags(h->ev_paths0, h->stream, ev_flags));
    const TaskDev *dt = static_cast<const TaskDev *>(h->d_tasks.ptr);
    const int64_t *dp = static_cast<const int64_t *>(h->d_prefix.ptr);
    unsigned long long *dc = static_cast<unsigned long long *>(h->d_cursor.ptr);
    Moments *dpart = static_cast<Moments *>(h->d_partials.ptr);
    if (plan.plain) {
        for (size_t i = 0; i < nt; ++i) {
            const TaskDev &t = plan.tasks[i];
            const int per_sm = price_tiles_max_blocks_per_sm(t.precision, t.model, t.scheme, t.lane_mode, t.track);
            const int grid = static_cast<int>(std::min<int64_t>(t.n_tiles, static_cast<int64_t>(h->sm_count) * per_sm));
            // one task: its own queue cursor, its own tile range (prefix of one task = itself)
            const uint64_t seed = static_cast<uint64_t>(t.key0) | (static_cast<uint64_t>(t.key1) << 32);
            QK_CUDA_TRY(launch_price_tiles(t.precision, t.model, t.scheme, grid, h->stream, dt + i, dp + i, 1,
                                           t.tile_begin, t.tile_begin + t.n_tiles, dc + i, dpart, true, seed,
                                           t.lane_mode, t.track));
            h->launches++;
        }
    } else {
        // kinds on forked streams: every launch waits for the cursor reset and the start
        // event; the handle's stream waits for all of them before the merge
        int n_kinds = 0;
        for (size_t i = 0; i < nt; ++i)
            if (i == 0 || plan.tasks[i].precision != plan.tasks[i - 1].precision ||
                plan.tasks[i].model != plan.tasks[i - 1].model || plan.tasks[i].scheme != plan.tasks[i - 1].scheme ||
                plan.tasks[i].lane_mode != plan.tasks[i - 1].lane_mode || plan.tasks[i].track != plan.tasks[i - 1].track)
                ++n_kinds;
        const int n_streams = std::min(n_kinds, kKindStreams);
        if (n_streams > 1) {
            QK_CUDA_TRY(cudaEventRecordWithFlags(h->kind_fork, h->stream, 0));
            for (int k = 0; k < n_streams; ++k) QK_CUDA_TRY(cudaStreamWaitEvent(h->kind_stream[k], h->kind_fork, 0));
        }
        int kind = 0;
        size_t b = 0;
        while (b < nt) {
            size_t e = b;
            const TaskDev &tb = plan.tasks[b];
            while (e < nt && plan.tasks[e].precision == tb.precision && plan.tasks[e].model == tb.model &&
                   plan.tasks[e].scheme == tb.scheme && plan.tasks[e].lane_mode == tb.lane_mode &&
                   plan.tasks[e].track == tb.track)
                ++e;
            const int64_t slots_end = plan.tasks[e - 1].tile_begin + plan.tasks[e - 1].n_tiles;
            const int64_t slots = slots_end - tb.tile_begin;
            const int blk = h->tune_block[tb.precision][tb.model][tb.scheme];
            const int per_sm =
                price_tiles_max_blocks_per_sm(tb.precision, tb.model, tb.scheme, tb.lane_mode, tb.track, blk);
            const int grid = static_cast<int>(std::min<int64_t>(slots, static_cast<int64_t>(h->sm_count) * per_sm));
            bool uniform_key = true;
            for (size_t i = b; i < e; ++i)
                uniform_key &= plan.tasks[i].key0 == tb.key0 && plan.tasks[i].key1 == tb.key1;
            const uint64_t seed = static_cast<uint64_t>(tb.key0) | (static_cast<uint64_t>(tb.key1) << 32);
            cudaStream_t ks = n_streams > 1 ? h->kind_stream[kind % n_streams] : h->stream;
            QK_CUDA_TRY(launch_price_tiles(tb.precision, tb.model, tb.scheme, grid, ks, dt + b, dp + b,
                                           static_cast<int32_t>(e - b), tb.tile_begin, slots_end, dc + b, dpart,
                                           uniform_key, seed, tb.lane_mode, tb.track, blk));
            h->launches++;
            ++kind;
            b = e;
        }
        if (n_streams > 1) {
            for (int k = 0; k < n_streams; ++k) {
                QK_CUDA_TRY(cudaEventRecordWithFlags(h->kind_join[k], h->kind_stream[k], 0));
                QK_CUDA_TRY(cudaStreamWaitEvent(h->stream, h->kind_join[k], 0));
            }
        }
    }
    QK_CUDA_TRY(cudaEventRecordWithFlags(h->ev_paths1, h->stream, ev_flags));
    QK_CUDA_TRY(launch_merge_two_level(static_cast<int>(nt), plan.total_chunks, h->stream, dt, dpart,
                                       static_cast<Moments *>(h->d_chunks.ptr),
                                       static_cast<Moments *>(h->d_moments.ptr)));
    h->launches += 2;
    QK_CUDA_TRY(cudaMemcpyAsync(h->h_moments.ptr, h->d_moments.ptr, nt * QK_MAX_PAYOFFS * sizeof(Moments),
                                cudaMemcpyDeviceToHost, h->stream));
    return QK_OK;
}

// Upload the plan and queue its kernels.
qk_status run_plan(qk_handle *h, Plan &plan) {
    const size_t nt = plan.tasks.size();
    h->launches = 0;
    h->h2d_bytes = static_cast<int64_t>(nt * (sizeof(TaskDev) + sizeof(int64_t)));
    h->d2h_bytes = static_cast<int64_t>(nt * QK_MAX_PAYOFFS * sizeof(Moments));
    QK_CUDA_TRY(cudaEventRecord(h->ev_start, h->stream));
    if (nt > 0) {
        qk_status s = upload_plan(h, plan);
        if (s != QK_OK) return s;
        return enqueue_plan(h, plan, false);
    }
    QK_CUDA_TRY(cudaEventRecord(h->ev_paths0, h->stream));
    QK_CUDA_TRY(cudaEventRecord(h->ev_paths1, h->stream));
    return QK_OK;
}

void release_prepared(qk_handle *h) {
    if (h->graph) cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
    h->graph_launches = 0;
    h->prepared = false;
}

// Capture the prepared plan's steady sequence (enqueue_plan) into a graph; the
// descriptors are uploaded once, before the capture, and stay on the device.
static qk_status capture_prepared(qk_handle *h) {
    Plan &plan = h->plan;
    qk_status s = upload_plan(h, plan);
    if (s != QK_OK) return s;
    QK_CUDA_TRY(cudaStreamSynchronize(h->stream));
    QK_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    h->launches = 0;
    s = enqueue_plan(h, plan, true);
    const std::string err = s != QK_OK ? g_last_error : std::string();
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
    if (s != QK_OK || ec != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return fail(s != QK_OK ? s : QK_ERR_CUDA,
                    "qk_batch_prepare: graph capture failed: " + (s != QK_OK ? err : std::string(cudaGetErrorString(ec))));
    }
    const cudaError_t ei = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        h->graph = nullptr;
        return fail(QK_ERR_CUDA, std::string("qk_batch_prepare: cudaGraphInstantiate: ") + cudaGetErrorString(ei));
    }
    h->graph_launches = h->launches;
    return QK_OK;
}

// ---------------------------------------------------------------- result assembly
// OptionPricer::evaluate_option_price (OptionPricer.hpp:204-249) for one task leg.
static void leg_price(const Moments &m, const qk_contract &b, const qk_payoff &pay, double scale, double *price,
                      double *se, double *itm) {
    const double N = m.n;
    const double disc = (pay.type == QK_AMERICAN) ? 1.0 : std::exp(-b.r * b.T);
    const double eff = disc * ((pay.type == QK_BINARY_CASH) ? 1.0 : scale);
    const double var = (N > 1.0) ? m.m2 / (N - 1.0) : 0.0;
    *price = m.mean * eff;
    *se = (N > 0.0) ? std::sqrt(var / N) * eff : 0.0;
    *itm = (N > 0.0) ? m.itm / N : 0.0;
}

qk_status assemble_results(qk_handle *h, const Plan &plan, const Moments *task_moments, qk_result *out) {
    (void)h;
    for (int i = 0; i < plan.n_contracts; ++i) {
        const qk_greeks *g = plan.g_of(i);
        if (plan.norm[i].payoffs[0].type == QK_AMERICAN) continue;
        qk_result &r = out[i];
        std::memset(&r, 0, sizeof(r));
        const qk_contract &n = plan.norm[i];
        r.status = plan.status[i];
        r.n_payoffs = n.n_payoffs;
        r.n_paths = n.n_paths;
        auto price_of = [&](int role, int k) -> double {
            const int ti = plan.task_of[static_cast<size_t>(i) * kNumRoles + role];
            if (ti < 0) return 0.0;
            const qk_contract b = bumped(n, g, role);
            double p, se, itm;
            leg_price(task_moments[static_cast<size_t>(ti) * QK_MAX_PAYOFFS + k], b, b.payoffs[k], plan.scale[i], &p, &se, &itm);
            return p;
        };
        for (int role = 0; role < kNumRoles; ++role) {
            const int ti = plan.task_of[static_cast<size_t>(i) * kNumRoles + role];
            if (ti >= 0) r.path_steps += static_cast<double>(plan.tasks[ti].n_paths) * plan.tasks[ti].n_steps;
        }
        for (int k = 0; k < n.n_payoffs; ++k) {
            qk_payoff_result &pr = r.p[k];
            const int t0 = plan.task_of[static_cast<size_t>(i) * kNumRoles + kBase];
            if (t0 < 0) continue;
            leg_price(task_moments[static_cast<size_t>(t0) * QK_MAX_PAYOFFS + k], n, n.payoffs[k], plan.scale[i], &pr.price,
                      &pr.std_error, &pr.prob_itm);
            if (!g) continue;
            const double p0 = pr.price;
            // spot bump in real units (MCEngine.hpp:589-595)
            const double h_S_real = (n.normalize ? plan.scale[i] : n.S0) * g->bump_S_rel;
            double h_vol = g->bump_vol;
            if (g->vega_mode == 1) h_vol = n.v0 * g->bump_vol;
            if (g->mask & QK_GREEK_DELTA_GAMMA) {
                const double pu = price_of(kSUp, k), pd = price_of(kSDn, k);
                pr.delta = (pu - pd) / (2.0 * h_S_real);
                pr.gamma = (pu - 2.0 * p0 + pd) / (h_S_real * h_S_real);
            }
            if (g->mask & QK_GREEK_VEGA_VOMMA) {
                const double pu = price_of(kVolUp, k), pd = price_of(kVolDn, k);
                pr.vega = (pu - pd) / (2.0 * h_vol);
                pr.vomma = (pu - 2.0 * p0 + pd) / (h_vol * h_vol);
            }
            if (g->mask & QK_GREEK_RHO) {
                const double pu = price_of(kRUp, k), pd = price_of(kRDn, k);
                pr.rho = (pu - pd) / (2.0 * g->bump_r_abs);
            }
            if (g->mask & QK_GREEK_THETA) {
                if (n.T > g->bump_T_abs) pr.theta = (price_of(kTDn, k) - p0) / g->bump_T_abs;
                else pr.theta = 0.0;
            }
            if (g->mask & QK_GREEK_VANNA) {
                const double uu = price_of(kUU, k), du = price_of(kDU, k), ud = price_of(kUD, k), dd = price_of(kDD, k);
                pr.vanna = (uu - du - ud + dd) / (4.0 * h_S_real * h_vol);
            }
        }
    }
    return QK_OK;
}

// Leg-0 payoffs (undiscounted, normalised units) of paths first .. first + count - 1.
qk_status payoffs_range(qk_handle *h, const qk_contract &c, int64_t first, int64_t count, double *out) {
    qk_status s = validate_contract(c, nullptr);
    if (s != QK_OK) return s;
    if (c.antithetic) return fail(QK_ERR_UNSUPPORTED, "per-path payoffs of antithetic pairs are not dumped");
    if (first < 0 || count < 1 || first + count > c.n_paths) return fail(QK_ERR_INVALID_ARG, "path range beyond n_paths");
    QK_CUDA_TRY(cudaSetDevice(h->device));
    double scale = 1.0;
    const qk_contract n = normalised(c, &scale);
    const TaskDev t = make_task(n, 1);
    const size_t head = ((sizeof(TaskDev) + 255) / 256) * 256;
    if ((s = h->d_trace.ensure(head + static_cast<size_t>(count) * sizeof(double))) != QK_OK) return s;
    TaskDev *dt = static_cast<TaskDev *>(h->d_trace.ptr);
    double *dp = reinterpret_cast<double *>(static_cast<char *>(h->d_trace.ptr) + head);
    QK_CUDA_TRY(cudaMemcpyAsync(dt, &t, sizeof(TaskDev), cudaMemcpyHostToDevice, h->stream));
    QK_CUDA_TRY(launch_payoff_paths(c.precision == QK_FP32 ? QK_FP32 : QK_FP64, h->stream, dt, first, count, dp));
    QK_CUDA_TRY(cudaMemcpyAsync(out, dp, static_cast<size_t>(count) * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    QK_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return QK_OK;
}

qk_status payoffs_dump(qk_handle *h, const qk_contract &c, std::vector<double> &out) {
    out.resize(static_cast<size_t>(c.n_paths));
    return payoffs_range(h, c, 0, c.n_paths, out.data());
}

qk_status finish_timing(qk_handle *h, double path_steps) {
    float ms_all = 0.f, ms_paths = 0.f, ms_rest = 0.f;
    QK_CUDA_TRY(cudaEventElapsedTime(&ms_all, h->ev_start, h->ev_end));
    QK_CUDA_TRY(cudaEventElapsedTime(&ms_paths, h->ev_paths0, h->ev_paths1));
    QK_CUDA_TRY(cudaEventElapsedTime(&ms_rest, h->ev_paths1, h->ev_end));
    double lsm_paths = 0.0, lsm_sweep = 0.0;
    if (h->lsm_jobs > 0) lsm_timing(h, &lsm_paths, &lsm_sweep);
    // LSM jobs of one call may overlap on several streams: their summed forward time
    // is capped at the part of the call outside the forward path kernels
    lsm_paths = std::min(lsm_paths, std::max(0.0, static_cast<double>(ms_all) - ms_paths));
    h->timing.device_ms = ms_all;
    h->timing.paths_ms = ms_paths + lsm_paths;
    h->timing.reduce_ms = ms_all - ms_paths - lsm_paths;
    h->timing.launches = h->launches + h->lsm_launches;
    h->timing.path_steps = path_steps;
    h->timing.h2d_bytes = h->h2d_bytes;
    h->timing.d2h_bytes = h->d2h_bytes;
    return QK_OK;
}

qk_status price_contracts(qk_handle *h, const qk_contract *c, int32_t n, const qk_greeks *gs, qk_result *out,
                              bool plain) {
    if (!h || !c || !out || n < 0) return fail(QK_ERR_INVALID_ARG, "NULL argument or negative count");
    QK_CUDA_TRY(cudaSetDevice(h->device));
    release_prepared(h);  // the plan and arenas are about to change
    qk_status s = build_plan(h, c, n, gs, plain, h->plan);
    if (s != QK_OK) return s;
    h->lsm_ms = h->lsm_paths_ms = 0.0;
    h->lsm_launches = 0;
    h->lsm_jobs = 0;
    if ((s = run_plan(h, h->plan)) != QK_OK) return s;
    std::vector<Moments> lsm_moments;
    if (!h->plan.american.empty()) {
        if ((s = run_lsm_contracts(h, h->plan, plain, lsm_moments)) != QK_OK) return s;
    }
    QK_CUDA_TRY(cudaEventRecord(h->ev_end, h->stream));
    QK_CUDA_TRY(cudaStreamSynchronize(h->stream));
    if ((s = assemble_results(h, h->plan, static_cast<const Moments *>(h->h_moments.ptr), out)) != QK_OK) return s;
    if (!h->plan.american.empty()) assemble_lsm_results(h, h->plan, lsm_moments, out);
    double ps = h->plan.path_steps + h->plan.lsm_path_steps;
    return finish_timing(h, ps);
}

}  // namespace qk

using namespace qk;

// ============================================================================
// extern "C"
// ============================================================================
extern "C" {

const char *qk_version(void) { return "quantkos_b200 1.0 (sm_100a)"; }
const char *qk_last_error(void) { return qk::g_last_error.c_str(); }

qk_status qk_create(int32_t device, qk_handle **out) {
    if (!out) return fail(QK_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(QK_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (device < 0 || device >= count) return fail(QK_ERR_INVALID_ARG, "device index out of range");
    QK_CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    QK_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(QK_ERR_UNSUPPORTED, std::string("built for sm_100a; device is ") + prop.name);
    {
        // every kernel's device code is loaded once per device, before any pricing call
        static std::mutex mu;
        static bool loaded[64] = {};
        std::lock_guard<std::mutex> lk(mu);
        if (device < 64 && !loaded[device]) {
            cudaError_t e = preload_path_kernels();
            if (e == cudaSuccess) e = preload_lsm_kernels();
            if (e != cudaSuccess) return fail(QK_ERR_CUDA, std::string("loading the kernels: ") + cudaGetErrorString(e));
            loaded[device] = true;
        }
    }
    qk_handle *h = new qk_handle();
    h->device = device;
    h->sm_count = prop.multiProcessorCount;
    bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreate(&h->ev_start) == cudaSuccess && cudaEventCreate(&h->ev_paths0) == cudaSuccess &&
              cudaEventCreate(&h->ev_paths1) == cudaSuccess && cudaEventCreate(&h->ev_end) == cudaSuccess &&
              cudaEventCreateWithFlags(&h->kind_fork, cudaEventDisableTiming) == cudaSuccess;
    for (int k = 0; ok && k < kKindStreams; ++k)
        ok = cudaStreamCreateWithFlags(&h->kind_stream[k], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&h->kind_join[k], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        delete h;
        return fail(QK_ERR_CUDA, "stream/event creation failed");
    }
    // device arenas grow stream-ordered on the handle's stream (the LSM working sets are
    // used by the LSM streams only after they fork from it); the device's memory pool
    // keeps freed blocks for reuse instead of returning them at every synchronization
    for (qk::DevArena *a : {&h->d_tasks, &h->d_prefix, &h->d_partials, &h->d_moments, &h->d_cursor, &h->d_trace,
                            &h->d_chunks, &h->d_lsm_moments, &h->lsm_task, &h->lsm_centre})
        a->stream = h->stream;
    for (int l = 0; l < kLsmLanes; ++l)
        for (qk::DevArena *a : {&h->lsm[l].slab_S, &h->lsm[l].slab_v, &h->lsm[l].cashflow, &h->lsm[l].block_sums,
                                &h->lsm[l].coeffs, &h->lsm[l].status})
            a->stream = h->stream;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    *out = h;
    return QK_OK;
}

qk_status qk_destroy(qk_handle *h) {
    if (!h) return QK_OK;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    release_prepared(h);
    lsm_release(h);
    h->d_tasks.release();
    h->d_prefix.release();
    h->d_partials.release();
    h->d_moments.release();
    h->d_chunks.release();
    h->d_cursor.release();
    h->d_trace.release();
    h->h_tasks.release();
    h->h_moments.release();
    cudaStreamSynchronize(h->stream);  // the stream-ordered frees above have completed
    pool_trim(h->device);  // unused blocks back, down to what live servers hold
    cudaEventDestroy(h->ev_start);
    cudaEventDestroy(h->ev_paths0);
    cudaEventDestroy(h->ev_paths1);
    for (int k = 0; k < kKindStreams; ++k) {
        cudaStreamDestroy(h->kind_stream[k]);
        cudaEventDestroy(h->kind_join[k]);
    }
    cudaEventDestroy(h->kind_fork);
    cudaEventDestroy(h->ev_end);
    cudaStreamDestroy(h->stream);
    delete h;
    return QK_OK;
}

qk_status qk_get_stream(qk_handle *h, void **stream) {
    if (!h || !stream) return fail(QK_ERR_INVALID_ARG, "NULL argument");
    *stream = static_cast<void *>(h->stream);
    return QK_OK;
}

qk_status qk_last_timing(const qk_handle *h, qk_timing *out) {
    if (!h || !out) return fail(QK_ERR_INVALID_ARG, "NULL argument");
    *out = h->timing;
    return QK_OK;
}

qk_status qk_measure_sfu(qk_handle *h, double *mufu_ops_per_s) {
    if (!h || !mufu_ops_per_s) return fail(QK_ERR_INVALID_ARG, "NULL argument");
    QK_CUDA_TRY(cudaSetDevice(h->device));
    qk_status s = h->d_trace.ensure(1 << 20);
    if (s != QK_OK) return s;
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        float ms = 0.f;
        double ops = 0.0;
        QK_CUDA_TRY(launch_sfu_probe(h->stream, h->sm_count, static_cast<float *>(h->d_trace.ptr), h->ev_start,
                                     h->ev_end, &ms, &ops));
        if (ms > 0.f) best = std::max(best, ops / (ms * 1e-3));
    }
    *mufu_ops_per_s = best;
    return QK_OK;
}

qk_status qk_validate(const qk_contract *c, const qk_greeks *g) {
    if (!c) return fail(QK_ERR_INVALID_ARG, "contract is NULL");
    return validate_contract(*c, g);
}

static std::vector<qk_greeks> repeat_greeks(const qk_greeks *g, int32_t n) {
    std::vector<qk_greeks> v(n > 0 ? n : 0);
    for (auto &x : v) {
        if (g) x = *g;
        else std::memset(&x, 0, sizeof(x));
    }
    return v;
}

qk_status qk_price_plain(qk_handle *h, const qk_contract *c, const qk_greeks *g, qk_result *out) {
    const auto gs = repeat_greeks(g, 1);
    return price_contracts(h, c, 1, gs.data(), out, true);
}

qk_status qk_price_batch(qk_handle *h, const qk_contract *c, int32_t n, const qk_greeks *g, qk_result *out) {
    const auto gs = repeat_greeks(g, n);
    return price_contracts(h, c, n, gs.data(), out, false);
}

qk_status qk_batch_prepare(qk_handle *h, const qk_contract *c, int32_t n, const qk_greeks *g) {
    if (!h || !c || n < 0) return fail(QK_ERR_INVALID_ARG, "NULL argument or negative count");
    QK_CUDA_TRY(cudaSetDevice(h->device));
    release_prepared(h);
    const auto gs = repeat_greeks(g, n);
    qk_status s = build_plan(h, c, n, gs.data(), false, h->plan);
    if (s != QK_OK) return s;
    if (!h->plan.american.empty()) return fail(QK_ERR_UNSUPPORTED, "qk_batch_prepare: American contracts go through qk_price_batch");
    if (!h->plan.tasks.empty() && (s = capture_prepared(h)) != QK_OK) return s;
    h->prepared = true;
    return QK_OK;
}

qk_status qk_batch_run(qk_handle *h) {
    if (!h || !h->prepared) return fail(QK_ERR_STATE, "qk_batch_run before qk_batch_prepare");
    QK_CUDA_TRY(cudaSetDevice(h->device));
    h->lsm_ms = h->lsm_paths_ms = 0.0;
    h->lsm_launches = 0;
    h->lsm_jobs = 0;
    const size_t nt = h->plan.tasks.size();
    h->h2d_bytes = 0;  // descriptors stay on the device between runs
    h->d2h_bytes = static_cast<int64_t>(nt * QK_MAX_PAYOFFS * sizeof(Moments));
    QK_CUDA_TRY(cudaEventRecord(h->ev_start, h->stream));
    if (h->graph) {
        QK_CUDA_TRY(cudaGraphLaunch(h->graph, h->stream));
        h->launches = h->graph_launches;
    } else {
        QK_CUDA_TRY(cudaEventRecord(h->ev_paths0, h->stream));
        QK_CUDA_TRY(cudaEventRecord(h->ev_paths1, h->stream));
        h->launches = 0;
    }
    QK_CUDA_TRY(cudaEventRecord(h->ev_end, h->stream));
    return QK_OK;
}

qk_status qk_batch_fetch(qk_handle *h, qk_result *out, int32_t n) {
    if (!h || !h->prepared || !out) return fail(QK_ERR_STATE, "qk_batch_fetch before qk_batch_prepare");
    if (n != h->plan.n_contracts) return fail(QK_ERR_INVALID_ARG, "result count differs from the prepared set");
    QK_CUDA_TRY(cudaStreamSynchronize(h->stream));
    qk_status s = assemble_results(h, h->plan, static_cast<const Moments *>(h->h_moments.ptr), out);
    if (s != QK_OK) return s;
    return finish_timing(h, h->plan.path_steps);
}

qk_status qk_payoffs_range(qk_handle *h, const qk_contract *c, int64_t first, int64_t count, double *payoffs) {
    if (!h || !c || !payoffs) return fail(QK_ERR_INVALID_ARG, "NULL argument");
    return payoffs_range(h, *c, first, count, payoffs);
}

qk_status qk_payoff_trace(const qk_payoff *leg, const double *S, int32_t n, double S0, int32_t precision,
                          double *payoff) {
    if (!leg || !S || !payoff || n < 1) return fail(QK_ERR_INVALID_ARG, "invalid payoff trace arguments");
    if (leg->type < QK_EUROPEAN || leg->type > QK_BINARY_ASSET || (leg->right != QK_CALL && leg->right != QK_PUT))
        return fail(QK_ERR_INVALID_ARG, "payoff type or right invalid (American legs have no path payoff)");
    PayoffSpec ps{leg->type, leg->right, leg->strike, leg->barrier};
    void *d = nullptr;
    QK_CUDA_TRY(cudaMalloc(&d, (static_cast<size_t>(n) + 1) * sizeof(double)));
    double *dS = static_cast<double *>(d);
    double *dout = dS + n;
    cudaError_t e = cudaMemcpy(dS, S, static_cast<size_t>(n) * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_payoff_trace(precision == QK_FP32 ? QK_FP32 : QK_FP64, 0, ps, dS, n, S0, dout);
    if (e == cudaSuccess) e = cudaMemcpy(payoff, dout, sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(QK_ERR_CUDA, std::string("qk_payoff_trace: ") + cudaGetErrorString(e));
    return QK_OK;
}

qk_status qk_step_trace(int32_t precision, const qk_contract *c, const double *z, const double *u, int32_t umax,
                        int32_t n_steps, double *S_out, double *v_out) {
    if (!c || !z || !S_out || !v_out || n_steps < 1 || umax < 0 || (umax > 0 && !u))
        return fail(QK_ERR_INVALID_ARG, "invalid trace arguments");
    if (c->model != QK_HESTON && c->model != QK_BATES) return fail(QK_ERR_INVALID_ARG, "model");
    if (c->scheme < 0 || c->scheme > 2) return fail(QK_ERR_UNSUPPORTED, "scheme");
    int dev = 0;
    QK_CUDA_TRY(cudaGetDevice(&dev));
    qk_contract b = *c;
    b.n_steps = n_steps;
    b.n_payoffs = 1;
    TaskDev t = make_task(b, 1);
    const size_t nz = static_cast<size_t>(n_steps) * 3, nu = static_cast<size_t>(n_steps) * std::max(umax, 1);
    const size_t bytes = sizeof(TaskDev) + (nz + nu + 2 * static_cast<size_t>(n_steps)) * sizeof(double) + 16;
    void *d = nullptr;
    QK_CUDA_TRY(cudaMalloc(&d, bytes));
    char *base = static_cast<char *>(d);
    TaskDev *dt = reinterpret_cast<TaskDev *>(base);
    double *dz = reinterpret_cast<double *>(base + sizeof(TaskDev));
    double *du = dz + nz;
    double *dS = du + nu;
    double *dv = dS + n_steps;
    int *dstat = reinterpret_cast<int *>(dv + n_steps);
    qk_status st = QK_OK;
    int hstat = 0;
    cudaError_t e = cudaMemcpy(dt, &t, sizeof(TaskDev), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dz, z, nz * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && umax > 0) e = cudaMemcpy(du, u, static_cast<size_t>(n_steps) * umax * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_step_trace(precision == QK_FP32 ? QK_FP32 : QK_FP64, 0, dt, dz, du, umax, n_steps, dS, dv, dstat);
    if (e == cudaSuccess) e = cudaMemcpy(&hstat, dstat, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(S_out, dS, n_steps * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(v_out, dv, n_steps * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = fail(QK_ERR_CUDA, std::string("qk_step_trace: ") + cudaGetErrorString(e));
    else if (hstat != 0) st = fail(QK_ERR_INVALID_ARG, "qk_step_trace: a step needed more Poisson uniforms than umax");
    cudaFree(d);
    return st;
}

qk_status qk_paths_dump(qk_handle *h, const qk_contract *c, int64_t first, int64_t count, double *S_out,
                        double *v_out) {
    if (!h || !c || !S_out || count < 1 || first < 0) return fail(QK_ERR_INVALID_ARG, "invalid dump arguments");
    qk_status s = validate_contract(*c, nullptr);
    if (s != QK_OK) return s;
    if (c->antithetic) return fail(QK_ERR_UNSUPPORTED, "qk_paths_dump: antithetic pairs are not dumped");
    if (first + count > c->n_paths) return fail(QK_ERR_INVALID_ARG, "path range beyond n_paths");
    QK_CUDA_TRY(cudaSetDevice(h->device));
    double scale = 1.0;
    const qk_contract n = normalised(*c, &scale);
    const TaskDev t = make_task(n, 1);
    const int prec = c->precision == QK_FP32 ? QK_FP32 : QK_FP64;
    const size_t esz = prec == QK_FP32 ? 4 : 8;
    const size_t cells = static_cast<size_t>(count) * c->n_steps;
    if ((s = h->d_trace.ensure(sizeof(TaskDev) + 2 * cells * esz + 256)) != QK_OK) return s;
    char *base = static_cast<char *>(h->d_trace.ptr);
    TaskDev *dt = reinterpret_cast<TaskDev *>(base);
    char *dS = base + ((sizeof(TaskDev) + 255) / 256) * 256;
    char *dv = dS + cells * esz;
    QK_CUDA_TRY(cudaMemcpyAsync(dt, &t, sizeof(TaskDev), cudaMemcpyHostToDevice, h->stream));
    QK_CUDA_TRY(launch_slab_paths(prec, n.model, n.scheme, n.seed, h->stream, dt, first, count, 1, dS, dv, count));
    std::vector<char> hS(cells * esz), hv(cells * esz);
    QK_CUDA_TRY(cudaMemcpyAsync(hS.data(), dS, cells * esz, cudaMemcpyDeviceToHost, h->stream));
    QK_CUDA_TRY(cudaMemcpyAsync(hv.data(), dv, cells * esz, cudaMemcpyDeviceToHost, h->stream));
    QK_CUDA_TRY(cudaStreamSynchronize(h->stream));
    // slab rows are dates (steps), columns paths; output is row-major path x step in real units
    for (int64_t p = 0; p < count; ++p)
        for (int j = 0; j < c->n_steps; ++j) {
            const size_t src = static_cast<size_t>(j) * count + p;
            const double sv = prec == QK_FP32 ? reinterpret_cast<const float *>(hS.data())[src]
                                              : reinterpret_cast<const double *>(hS.data())[src];
            const double vv = prec == QK_FP32 ? reinterpret_cast<const float *>(hv.data())[src]
                                              : reinterpret_cast<const double *>(hv.data())[src];
            S_out[static_cast<size_t>(p) * c->n_steps + j] = sv * scale;
            if (v_out) v_out[static_cast<size_t>(p) * c->n_steps + j] = vv;
        }
    return QK_OK;
}

}  // extern "C"
