/*
 * quantkos_b200.h — C ABI of the B200-native QuantKos Monte Carlo hot path.
 *
 * The reference (QuantKos) has no FFI: its boundary is a C++ template API whose
 * pieces are named beside each entry point below (paths relative to the
 * reference project).  This header is the drop-in boundary that replaces them:
 * plain C types, caller-owned host arrays, handle-owned device memory, integer
 * status codes (never abort, never trap).  The C++ wrappers with the
 * reference's own names live in quantkos_b200.hpp.
 *
 * Threading: a handle is used by one host thread at a time, except
 * qk_serve_submit / qk_serve_poll / qk_serve_cancel, which are thread-safe.
 */
#ifndef QUANTKOS_B200_H
#define QUANTKOS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QK_ABI_VERSION 2
#define QK_MAX_PAYOFFS 8

/* ---------------------------------------------------------------- status */
typedef enum qk_status {
    QK_OK = 0,
    QK_ERR_INVALID_ARG = 1,   /* std::invalid_argument in the reference (Config.hpp validate()) */
    QK_ERR_CUDA = 2,          /* a CUDA runtime call failed */
    QK_ERR_OUT_OF_MEMORY = 3, /* std::runtime_error "[Memory Capacity Error]" (PathsMCBatchMem.hpp:396-415) */
    QK_ERR_UNSUPPORTED = 4,   /* runtime_error "not yet implemented for this scheme combination" (MSchemes.hpp:51-54) */
    QK_ERR_TIMEOUT = 5,       /* a bounded device/host wait gave up */
    QK_ERR_CAPACITY = 6,      /* request larger than the admission budget */
    QK_ERR_NO_DEVICE = 7,
    QK_ERR_PARSE = 8,         /* runtime_error "Config Error: ..." (src/IO/ConfigParser.cpp:36-294) */
    QK_ERR_STATE = 9,         /* call out of order (e.g. poll of an unknown ticket) */
    QK_ERR_CANCELLED = 10     /* the request was cancelled before it was admitted (qk_serve_cancel) */
} qk_status;

/* ---------------------------------------------------------------- enums
 * Same order as quantkos::Implemented (include/core/config/ConfigFileEnums.hpp:24-124). */
typedef enum qk_model { QK_HESTON = 0, QK_BATES = 1 } qk_model;
typedef enum qk_scheme { QK_EULER = 0, QK_IMPLICIT_MILSTEIN = 1, QK_ANDERSEN_QE = 2 } qk_scheme;
typedef enum qk_opt_type {
    QK_EUROPEAN = 0,
    QK_ASIAN = 1,
    QK_BARRIER_UP_OUT = 2,
    QK_BARRIER_DOWN_OUT = 3,
    QK_BARRIER_UP_IN = 4,
    QK_BARRIER_DOWN_IN = 5,
    QK_LOOKBACK_FLOATING = 6,
    QK_LOOKBACK_FIXED = 7,
    QK_BINARY_CASH = 8,
    QK_BINARY_ASSET = 9,
    QK_AMERICAN = 10
} qk_opt_type;
typedef enum qk_right { QK_CALL = 0, QK_PUT = 1 } qk_right;
typedef enum qk_precision { QK_FP64 = 0, QK_FP32 = 1 } qk_precision;
/* Longstaff-Schwartz regression basis.
 *  QK_LSM_LAGUERRE3: the reference's LaguerreP03 on X = S/K, 4 terms, every step an
 *                    exercise date, Tikhonov 1e-8 + Cholesky + mean fallback
 *                    (include/core/options/LSMAmerican.hpp:157-613);
 *  QK_LSM_POLY_SV:   {1, S, S^2, S^3, v, S*v} on S/K-scaled values, ITM paths, FP64
 *                    Cholesky of the centred and scaled Gram, pivoted QR when the
 *                    condition estimate exceeds 1e8 (no reference counterpart). */
typedef enum qk_lsm_basis { QK_LSM_LAGUERRE3 = 0, QK_LSM_POLY_SV = 1 } qk_lsm_basis;

/* ---------------------------------------------------------------- contract
 * One pricing request.  Mirrors quantkos::Config::UInputs (include/core/config/Config.hpp:677-775)
 * restricted to what the hot path reads.  Monetary inputs are in real units; the
 * engine applies UInputs::apply_price_scaling (Config.hpp:710-723) itself when
 * `normalize` is set and scales results back (OptionPricer.hpp:323-332). */
typedef struct qk_payoff {
    int32_t type;   /* qk_opt_type */
    int32_t right;  /* qk_right */
    double strike;  /* K */
    double barrier; /* B (barrier types only) */
} qk_payoff;

typedef struct qk_contract {
    double S0, v0, r, q;                          /* MarketConfig */
    int32_t model, scheme;                        /* qk_model, qk_scheme */
    double kappa, theta, sigma, rho;              /* MathModelConfig::Heston */
    double lambda_j, mu_j, sigma_j;               /* MathModelConfig::Bates (ignored for Heston) */
    double psi_c;                                 /* QE switching level; 0 means 1.5 (MSchemes.hpp:290) */
    double T;                                     /* TimeConfig::t_end */
    int32_t n_steps;                              /* TimeConfig::N_time_steps (= ceil(T/dt)) */
    int32_t normalize;                            /* MCConfig::normalize_prices */
    int64_t n_paths;                              /* MCConfig::N_Paths */
    uint64_t seed;                                /* MCConfig::rng_seed (Philox key) */
    uint64_t stream;                              /* common-random-number stream id (Philox counter word) */
    int32_t precision;                            /* qk_precision for the path stepping */
    int32_t n_payoffs;                            /* 1..QK_MAX_PAYOFFS, all priced in one pass */
    qk_payoff payoffs[QK_MAX_PAYOFFS];
    int32_t lsm_basis;                            /* qk_lsm_basis (American only) */
    int32_t lsm_dates;                            /* exercise dates; 0 = every time step (American only) */
    int32_t antithetic;                           /* 1: antithetic pairs (not in the reference): paths 2k and
                                                     2k+1 share pair k's draws, the second with every normal
                                                     negated (spot, variance, jump size; Poisson uniforms
                                                     shared); estimates over pair averages, n_paths even,
                                                     forward legs only */
    int32_t reserved_;                            /* zero */
} qk_contract;

/* Finite-difference Greeks by re-pricing under common random numbers
 * (execute_mc_framework, include/core/engine/MCEngine.hpp:576-735). */
#define QK_GREEK_DELTA_GAMMA 1
#define QK_GREEK_VEGA_VOMMA 2
#define QK_GREEK_VANNA 4
#define QK_GREEK_RHO 8
#define QK_GREEK_THETA 16
#define QK_GREEK_ALL 31
typedef struct qk_greeks {
    int32_t mask;       /* QK_GREEK_* bits (MCConfig compute_* flags, Config.hpp:409-417) */
    int32_t vega_mode;  /* 0: absolute bump of sqrt(v0) (reference, MCEngine.hpp:611-632);
                           1: relative bump of v0, vega/vomma/vanna reported per unit of v0 */
    double bump_S_rel;  /* spot_price_relative_bump_size, default 0.001 */
    double bump_vol;    /* vega_mode 0: volatility_absolute_bump_size (0.01); mode 1: relative v0 bump */
    double bump_r_abs;  /* risk_free_rate_absolute_bump_size, default 1e-4 */
    double bump_T_abs;  /* time_absolute_bump_size, default 1/365 */
} qk_greeks;

typedef struct qk_payoff_result {
    double price;     /* MCOpPrices::option_price (OptionPricer.hpp:50-70) */
    double std_error; /* MCOpPrices::standard_error */
    double prob_itm;  /* MCOpPrices::prob_itm */
    double delta, gamma, vega, vomma, vanna, rho, theta; /* MCGreeks (MCEngine.hpp:93-120) */
} qk_payoff_result;

typedef struct qk_result {
    int32_t status;     /* qk_status of this contract */
    int32_t n_payoffs;
    int64_t n_paths;
    double path_steps;  /* path-steps simulated for this contract, bumps included */
    qk_payoff_result p[QK_MAX_PAYOFFS];
} qk_result;

/* Device timings of the most recent pricing call on a handle (CUDA events on the handle's stream). */
typedef struct qk_timing {
    double device_ms;     /* first kernel start to last kernel end */
    double paths_ms;      /* path-generation kernels (LSM forward kernels of concurrent jobs summed, capped at the call) */
    double reduce_ms;     /* merge / LSM regression kernels */
    int64_t launches;     /* kernels launched by the call */
    double path_steps;    /* path-steps simulated */
    int64_t h2d_bytes;    /* host-to-device bytes the call copied (descriptors) */
    int64_t d2h_bytes;    /* device-to-host bytes the call copied (results) */
} qk_timing;

typedef struct qk_handle qk_handle;

/* ---------------------------------------------------------------- lifecycle */
const char *qk_version(void);
/* Thread-local message of the last failing call on this thread. */
const char *qk_last_error(void);
/* Replaces Kokkos::initialize + the per-run Memory classes (app/main.cpp:78;
 * PathsMCBatchMem.hpp:330-372): binds `device`, creates a stream and the
 * handle-owned device arenas. */
qk_status qk_create(int32_t device, qk_handle **out);
qk_status qk_destroy(qk_handle *h);
/* The CUDA stream (cudaStream_t) all work of the handle is queued on. */
qk_status qk_get_stream(qk_handle *h, void **stream);
qk_status qk_last_timing(const qk_handle *h, qk_timing *out);
/* Measured SFU (MUFU) throughput of the device, in operations per second: a
 * kernel of independent ex2.approx chains on every SM, timed with CUDA events.
 * The roofline denominator of the fused path kernels, which are SFU/issue-bound. */
qk_status qk_measure_sfu(qk_handle *h, double *mufu_ops_per_s);
/* Host-side validation with the reference's rules (UInputs::validate, Config.hpp:694-704). */
qk_status qk_validate(const qk_contract *c, const qk_greeks *g);

/* ---------------------------------------------------------------- pricing
 * qk_price_plain — the plain method, the drop-in: one contract, one all-FP64
 * path kernel launch (plus its reduction), like one
 * MCDispatcher(UInputs).launch_montecarlo() (include/core/engine/Distpatcher.hpp:78)
 * with every Greek bump a further launch (MCEngine.hpp:586-730).  `c->precision`
 * is ignored (FP64).  `g` may be NULL. */
qk_status qk_price_plain(qk_handle *h, const qk_contract *c, const qk_greeks *g, qk_result *out);

/* qk_price_batch — the batched mixed-precision engine: all contracts and all
 * their Greek bumps go into one persistent kernel through a device queue of
 * (task, path-block) tiles; FP32 stepping unless a contract asks for FP64;
 * FP64 accumulation.  American contracts run the device-resident LSM.  Replaces a
 * host loop of MCDispatcher runs; `out` has `n` entries. */
qk_status qk_price_batch(qk_handle *h, const qk_contract *c, int32_t n, const qk_greeks *g, qk_result *out);

/* Device-resident form of qk_price_batch for callers that reprice the same set:
 * prepare uploads the task/tile descriptors once and captures the steady launch
 * sequence (queue reset, path kernels, merge, copy of the moments to the host)
 * in a CUDA graph; run replays the graph (asynchronously, on the handle's
 * stream), fetch waits and fills `out`.  Any other pricing call on the handle
 * drops the prepared set (run then returns QK_ERR_STATE). */
qk_status qk_batch_prepare(qk_handle *h, const qk_contract *c, int32_t n, const qk_greeks *g);
qk_status qk_batch_run(qk_handle *h);
qk_status qk_batch_fetch(qk_handle *h, qk_result *out, int32_t n);

/* ---------------------------------------------------------------- autotuner
 * Launch shape of the batched engine, per kernel kind (precision x model x
 * scheme): the target number of warp tiles per resident warp slot (sets the
 * paths per tile), whether a task that fills the GPU many times over ends in
 * short "tail" tiles, and whether a lane simulates one path or two independent
 * paths (2u, 2u+1) interleaved.  The reference sizes its path batches from a memory budget
 * (include/core/memory/PathsMCBatchMem.hpp:330-420); there it has no tuner.
 * Defaults: FP32 48 tiles per warp slot, two paths per lane, the guided tail except
 * for Heston QE; FP64 24 tiles, one path per lane, no guided tail. */
#define QK_TUNE_KINDS 12
typedef struct qk_tune_report {
    int32_t n_kinds;                         /* kinds present in the sample */
    int32_t precision[QK_TUNE_KINDS];
    int32_t model[QK_TUNE_KINDS];
    int32_t scheme[QK_TUNE_KINDS];
    int32_t tiles_per_warp[QK_TUNE_KINDS];   /* chosen */
    int32_t guided_tail[QK_TUNE_KINDS];      /* chosen: 1 = on */
    int32_t paths_per_lane[QK_TUNE_KINDS];   /* chosen: 1 or 2 */
    double best_ms[QK_TUNE_KINDS];           /* device time of pricing the sample's tasks of this kind, chosen shape */
    double default_ms[QK_TUNE_KINDS];        /* the same with the defaults */
    int32_t candidates;                      /* shapes timed per kind */
    int32_t block_size[QK_TUNE_KINDS];       /* chosen: threads per block of the pricing kernel */
} qk_tune_report;

/* Times the sample `c` (forward contracts; American ones are skipped) kind by
 * kind under every candidate shape (tiles per warp slot 4, 8, 12, 24, 48; tail
 * off, on; 1 or 2 paths per lane), then the threads per block (128, 256, 512; FP64
 * 128, 256) at the best of those, `reps` timed runs each after one warm-up, keeps the fastest shape per kind
 * in the handle for later qk_price_batch / qk_batch_prepare calls and reports it.
 * Prices do not depend on the shape beyond the last bits of the moment merge. */
qk_status qk_autotune(qk_handle *h, const qk_contract *c, int32_t n, const qk_greeks *g, int32_t reps,
                      qk_tune_report *out);
/* Restores the default shape of every kind (256 threads per block). */
qk_status qk_tune_reset(qk_handle *h);
/* Threads per block of one kind's pricing kernel: 128, 256 or 512 (FP64: 128 or 256). */
qk_status qk_tune_set_block(qk_handle *h, int32_t precision, int32_t model, int32_t scheme, int32_t threads_per_block);
/* Sets one kind's shape by hand (for example a stored autotuner result). */
qk_status qk_tune_set(qk_handle *h, int32_t precision, int32_t model, int32_t scheme, int32_t tiles_per_warp,
                      int32_t guided_tail, int32_t paths_per_lane);

/* qk_price_noalloc — no counterpart in the reference.  The base price (no Greeks)
 * of one forward contract for callers that cannot allocate device memory on the
 * pricing path (a host application owning all GPU memory through its own pool,
 * or a latency-critical caller that cannot take cudaMalloc/cudaFree and their
 * device synchronisation between requests).  Same kernels as qk_price_batch; all
 * scratch lives in one fixed device array of about 4.1 MiB per device; no handle
 * is needed.  Limit: ceil(n_paths / 2048) * n_payoffs <= 131072 (QK_ERR_CAPACITY
 * beyond).  The first call on each device is its set-up and does take device
 * memory: with that device current it looks up the array's address, and the CUDA
 * runtime, which loads device code lazily, then reserves the array and loads the
 * kernels' code on that device.  Make that first call during set-up, before a
 * memory pool takes the device's free memory, and before any stream capture.
 * Later calls allocate nothing, except that the first launch of a kernel kind
 * (precision x model x scheme, with or without path-dependent legs) can make the
 * driver grow its local-memory reservation: price one small contract of each
 * kind you will use during set-up.  Calls share the array: calls whose GPU work
 * overlaps race, so serialize them.  `stream` is a cudaStream_t (NULL = default
 * stream); the call returns after its work has finished. */
qk_status qk_price_noalloc(const qk_contract *c, void *stream, qk_result *out);

/* ---------------------------------------------------------------- parity harness
 * qk_step_trace — SDEScheme<M,S>::evolve_step with fed draws
 * (include/core/schemes/markovian/MSchemes.hpp:133-156, 229-253, 363-442, 493-526),
 * run on the device by the same step code the pricing kernels use.
 * Per step i: z[3i..3i+2] = {Z1, Z2, Zjump}; u[umax*i ..] = Poisson uniforms in the
 * order Knuth's loop consumes them.  Starts from (c->S0, c->v0) as given, dt = c->T / n_steps.
 * precision: qk_precision.  Returns QK_ERR_INVALID_ARG if a step needs more than umax uniforms. */
qk_status qk_step_trace(int32_t precision, const qk_contract *c, const double *z, const double *u, int32_t umax,
                        int32_t n_steps, double *S_out, double *v_out);

/* qk_paths_dump — the spot paths of paths [first, first+count) of contract `c` as the
 * pricing kernels generate them (same Philox counters), row-major count x n_steps
 * (the .paths payload layout, include/IO/IOBinary.hpp:96-249), FP64 output. */
qk_status qk_paths_dump(qk_handle *h, const qk_contract *c, int64_t first, int64_t count, double *S_out,
                        double *v_out);

/* ---------------------------------------------------------------- engine pieces
 * The building blocks the reference's C++ engine exposes, run by the same device code
 * the fused kernels use (the C++ wrappers in quantkos_b200.hpp carry the reference's
 * names).  They serve tests, parity checks and callers that drive the steps themselves;
 * the pricing entry points above do not go through them.
 *
 * qk_payoff_trace — PayoffTracker<T,R> (include/core/options/Payoff.hpp:84-243):
 * track_current_price over S[0..n-1] starting from S0, then evaluate_final_payoff at
 * S[n-1] with leg->strike and leg->barrier, in `precision` (qk_precision). */
qk_status qk_payoff_trace(const qk_payoff *leg, const double *S, int32_t n, double S0, int32_t precision,
                          double *payoff);
/* qk_payoffs_range — the per-path payoffs of one batch of paths as
 * MSolver<M,S,T,R>::execute_batch writes them (include/core/schemes/markovian/MSolver.hpp:195-232):
 * leg 0 of paths [first, first + count) of contract c, undiscounted, in normalised
 * units when c->normalize (the OptionPricer rescales), the same paths the pricing
 * kernels simulate. */
qk_status qk_payoffs_range(qk_handle *h, const qk_contract *c, int64_t first, int64_t count, double *payoffs);
/* qk_lsm_date — one exercise date of LSMEngine<R,Basis> on n caller paths
 * (include/core/options/LSMAmerican.hpp:252-335): op 0 initialize_cashflows (cf =
 * intrinsic(S)); op 1 perform_cross_paths_regression (sums over in-the-money paths with
 * Y = cf * disc, then the FP64 solve into coeffs[4 or 6], *method 0 Cholesky, 1 pivoted
 * QR, 2 mean fallback); op 2 update_cashflows (exercise iff intrinsic beats the
 * continuation of coeffs, else cf * disc).  S and K in the units of the contract (S/K is
 * what the basis sees); v (variance) only for QK_LSM_POLY_SV, whose basis is centred at
 * (cx, cv).  precision: arithmetic of the path values, as the sweep kernel. */
qk_status qk_lsm_date(int32_t op, int32_t precision, int32_t basis, int32_t right, int64_t n, const double *S,
                      const double *v, double *cf, double K, double disc, double cx, double cv, double *coeffs,
                      int32_t *method);
/* qk_lsm_solve — LSMEngine::solve_system_on_host_cholesky (LSMAmerican.hpp:516-613) for
 * QK_LSM_LAGUERRE3, the scaled Cholesky / pivoted QR for QK_LSM_POLY_SV: sums = upper
 * Gram row-major, right-hand side, count (15 or 28 values). */
qk_status qk_lsm_solve(int32_t basis, const double *sums, double *coeffs, int32_t *method);
/* qk_paths_write — BinWriter (include/IO/IOBinary.hpp:72-249) on host arrays, no device
 * involved: the header and n_paths x n_steps spot values given in real units, row-major,
 * stored normalised (divided by `scale`) in `precision`, as qk_run_config writes them. */
qk_status qk_paths_write(const char *path, int32_t precision, int64_t n_paths, int32_t n_steps, double dt,
                         double scale, const double *S);

/* ---------------------------------------------------------------- configuration
 * qk_config mirrors quantkos::Config::UInputs (include/core/config/Config.hpp:677-775)
 * field by field; qk_config_parse_file is Parser::parse (src/IO/ConfigParser.cpp:36-294)
 * for the same YAML files (blocks Market, Options, Model{Heston|Bates}, Numerics,
 * Time, MC, Output; unknown keys ignored, as there).  Keys this engine adds, all
 * optional: MC.Precision (FP64 | FP32), MC.Engine (plain | batch),
 * MC.LSM_Basis (Laguerre3 | PolySV), MC.LSM_Dates (int), MC.Vega_Mode (0 | 1),
 * MC.Stream (int). */
typedef struct qk_config {
    double S0, v0, r, q;                                        /* MarketConfig */
    int32_t opt_type, opt_right;                                /* OptionsConfig */
    double K, B;
    int32_t model;                                              /* MathModelConfig::id_model */
    double heston_k, heston_theta, heston_sigma, heston_rho;    /* MathModelConfig::Heston */
    double bates_k, bates_theta, bates_sigma, bates_rho;        /* MathModelConfig::Bates */
    double bates_lambda, bates_mu, bates_sigma_j;
    int32_t scheme;                                             /* NumSchemeConfig */
    double t_end, inp_dt, dt;                                   /* TimeConfig */
    int32_t n_steps;
    int32_t normalize, n_paths, batch_size;                     /* MCConfig */
    uint64_t seed;
    int64_t max_vram_mb, max_cpu_ram_mb;
    int32_t analyze_distribution;
    int32_t greeks_mask;
    double bump_S_rel, bump_vol_abs, bump_r_abs, bump_T_abs;
    int32_t verbosity, format;                                  /* OutputConfig */
    char out_dir[256], paths_file[256], log_file[256];
    int32_t precision, engine, lsm_basis, lsm_dates, vega_mode; /* engine extensions */
    uint64_t stream;
    int32_t antithetic;                                         /* MC.Antithetic (extension) */
    int32_t reserved_;
} qk_config;

/* Defaults of UInputs (Config.hpp:50-623) plus engine extensions (FP64, plain). */
qk_status qk_config_default(qk_config *out);
/* Parse + validate (Parser::parse ends with UInputs::validate). */
qk_status qk_config_parse_file(const char *path, qk_config *out);
qk_status qk_config_parse_string(const char *yaml, qk_config *out);
/* UInputs::validate: checks and fills n_steps = ceil(t_end / inp_dt), dt = t_end / n_steps. */
qk_status qk_config_validate(qk_config *c);
/* The contract and Greeks request a validated config prices (MCDispatcher's dispatch). */
qk_status qk_config_to_contract(const qk_config *c, qk_contract *out, qk_greeks *g);
/* MCDispatcher(UInputs).launch_montecarlo() (include/core/engine/Distpatcher.hpp:78):
 * prices the config with the plain (FP64) or batched engine per c->engine, writes
 * the .paths file when c->paths_file is set, fills the payoff percentiles when
 * analyze_distribution is set (pct[15]: p0 p1 p5 p10 p20 p30 p40 p50 p60 p70 p80
 * p90 p95 p99 p100, discounted and scaled as OptionPricer.hpp:340-360). */
qk_status qk_run_config(qk_handle *h, const qk_config *c, qk_result *out, double *pct);

/* ---------------------------------------------------------------- serving
 * A continuous-batching request loop.  Requests are admitted by the HBM their
 * LSM slabs and partials need (budget in MiB; 0 = 80% of free HBM) into waves of a
 * few milliseconds of estimated GPU time, batched with whatever else has arrived;
 * several lanes' waves run on the GPU at once; results are polled by ticket.  The
 * lanes use h's device and the launch shapes h holds when the server starts
 * (defaults, or those set by qk_autotune / qk_tune_set). */
typedef struct qk_server qk_server;
typedef struct qk_serve_stats {
    int64_t submitted, completed, rejected;
    double p50_ms, p99_ms, p999_ms, max_ms; /* over the most recent 1,048,576 requests */
    double contracts_per_s, path_steps_per_s;
    int64_t batches;
    double busy_s;
    int64_t reserved_mib; /* HBM the server holds in the device's memory pool */
} qk_serve_stats;
qk_status qk_serve_start(qk_handle *h, int64_t hbm_budget_mib, int32_t max_batch, qk_server **out);
/* The same with all options: lanes = host threads, each with its own handle and stream,
 * whose waves run on the GPU at the same time (0 = 4); wave_ms = estimated GPU time at
 * which a lane closes the wave it is admitting, raised to the lane's share of the
 * waiting requests' estimated time when that is larger (0 = 2.5 ms; a wave always takes
 * at least one request); reserve_mib = HBM mapped into the device's memory pool at the
 * start and held until qk_serve_stop, from which the lanes' buffers grow (0 = the
 * budget; -1 = none; mapping new memory while lanes run blocks every lane's driver
 * calls for up to hundreds of milliseconds).  A default reservation that does not fit
 * is skipped; an explicit one that does not fit fails with QK_ERR_CAPACITY.
 * hbm_budget_mib and max_batch as above.  plain_fp64 = 1 serves every request alone
 * with the plain FP64 method (qk_price_plain: one contract, all FP64, one launch per
 * pricing task) behind the same lanes and admission, for comparing the two methods on
 * one request stream; 0 = the batched engine.  qk_serve_start uses the defaults for
 * lanes, wave_ms, reserve_mib and plain_fp64. */
typedef struct qk_serve_options {
    int64_t hbm_budget_mib;
    int32_t max_batch;
    int32_t lanes;
    double wave_ms;
    int64_t reserve_mib;
    int32_t plain_fp64;
    int32_t pad_;
} qk_serve_options;
qk_status qk_serve_start_ex(qk_handle *h, const qk_serve_options *opt, qk_server **out);
qk_status qk_serve_submit(qk_server *s, const qk_contract *c, const qk_greeks *g, int64_t *ticket);
/* done = 1 and *out filled once the ticket finished; wait_ms bounds the wait (0 = poll). */
qk_status qk_serve_poll(qk_server *s, int64_t ticket, int32_t wait_ms, int32_t *done, qk_result *out);
/* Withdraws a request that is still waiting for admission: *cancelled = 1 and its
 * poll then reports QK_ERR_CANCELLED.  A request already admitted to a batch runs to
 * completion (*cancelled = 0).  Thread-safe. */
qk_status qk_serve_cancel(qk_server *s, int64_t ticket, int32_t *cancelled);
qk_status qk_serve_stats_get(qk_server *s, qk_serve_stats *out);
/* Per-request accounting of the most recent completed requests (at most 1,048,576, the
 * window the latency percentiles of qk_serve_stats_get also cover), oldest first: copies
 * up to `capacity` records and sets *count to the number held. */
typedef struct qk_serve_record {
    int64_t ticket;
    int64_t wave;          /* the wave it was priced in, numbered in order of admission */
    int32_t lane;          /* the lane that priced that wave */
    int32_t wave_requests; /* requests in that wave */
    double submit_s;       /* submit time, seconds after the server's first submit */
    double admit_ms;       /* from submit to the start of its wave */
    double latency_ms;     /* from submit to completion */
    double wave_ms;        /* wall time of its wave (plan, upload, kernels, results) */
    double wave_est_ms;    /* estimated GPU time of its wave */
    double est_ms;         /* estimated GPU time of the request */
} qk_serve_record;
qk_status qk_serve_records(qk_server *s, qk_serve_record *out, int64_t capacity, int64_t *count);
qk_status qk_serve_stop(qk_server *s);

#ifdef __cplusplus
}
#endif
#endif /* QUANTKOS_B200_H */
