// Plain-old-data layouts shared by the host engine and the device kernels.
#pragma once

#include <cstdint>

#include "../../include/quantkos_b200.h"

#if defined(__CUDACC__)
#define QK_HD __host__ __device__
#else
#define QK_HD
#endif

namespace qk {

// Philox4x32 round multipliers and Weyl key increments (Salmon et al., SC'11).
constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

enum : int { kHeston = 0, kBates = 1 };
enum : int { kEuler = 0, kMilstein = 1, kQE = 2 };
enum : int {
    kEuropean = 0,
    kAsian = 1,
    kBarrierUpOut = 2,
    kBarrierDownOut = 3,
    kBarrierUpIn = 4,
    kBarrierDownIn = 5,
    kLookbackFloating = 6,
    kLookbackFixed = 7,
    kBinaryCash = 8,
    kBinaryAsset = 9,
    kAmerican = 10
};
enum : int { kCall = 0, kPut = 1 };

// Bound on Knuth's Poisson loop per step (the reference loops without bound);
// validation rejects lambda*dt > kMaxLambdaDt so the bound is never reached in practice.
constexpr int kMaxJumpsPerStep = 4096;
constexpr double kMaxLambdaDt = 512.0;

// Per-step invariants of SDEScheme<M,S>, precomputed on the host exactly as the
// reference constructors do (MSchemes.hpp:102-123, 197-219, 303-353, 480-487).
template <class R>
struct StepConst {
    R r_minus_q_dt, half_dt, sqrt_dt, rho, rho_c;
    R one_minus_k_dt, k_theta_dt, sigma_sqrt_dt;   // Euler
    R quarter_sigma_sq_dt, implicit_den;           // Milstein
    R eps, psi_c, inv_sqrt2, exp_mkdt, theta_m, s2f1, s2f2, K1, K2, K3, K4, A, K1_half_K3;  // QE
    R exp_m_lambda_dt, mu_j, sigma_j;              // Bates
};

struct PayoffSpec {
    int32_t type, right;
    double K, B;  // normalised like the spot
};

// One pricing task on the device: a contract, or one of its Greek bumps.
// What one lane of the path kernel simulates: one path; an antithetic pair
// (paths 2u and 2u+1 from pair u's draws, the second negated); or two independent
// consecutive paths 2u and 2u+1 (instruction-level parallelism).
enum : int { kLaneOne = 0, kLanePair = 1, kLaneTwo = 2 };

__host__ __device__ inline int64_t lane_units(int64_t n_paths, int lane_mode) {
    return lane_mode == kLaneOne ? n_paths : (lane_mode == kLanePair ? n_paths / 2 : (n_paths + 1) / 2);
}

struct TaskDev {
    StepConst<float> cf;
    StepConst<double> cd;
    double S0, v0;         // starting state (normalised spot)
    int32_t model, scheme, n_steps, n_payoffs;
    int32_t precision;     // qk_precision
    uint32_t key0, key1;   // Philox key = seed
    uint32_t stream;       // Philox counter word 2 (common random numbers across bumps)
    uint32_t jump_kmin;    // FP32 jump test: a step jumps iff (first Poisson word >> 9) >= jump_kmin
    int64_t n_paths;
    int64_t tile_begin;    // first queue slot of the task (tiles of a task are consecutive)
    int64_t partial_base;  // first per-tile moments record of the task
    int32_t n_tiles;
    int32_t ppt;           // rounds of a big tile: a round is one lane unit (lane_mode) per lane of a warp
    int32_t n_big;         // tiles 0 .. n_big-1 have ppt rounds; the rest (the tail) ppt_tail rounds
    int32_t ppt_tail;
    int64_t chunk_base;    // first merge chunk of the task (two-level merge of the tile records)
    int32_t n_chunks;      // merge chunks of the task: ceil(n_tiles / kMergeChunkTiles)
    int32_t lane_mode;     // kLaneOne / kLanePair / kLaneTwo: what a lane simulates; tiles count lane units
    int32_t track;         // 1 if a leg reads the path state (Asian sum, running max / min)
    PayoffSpec pay[QK_MAX_PAYOFFS];
};

// FP64 moments of a set of payoffs: count, mean, sum of squared deviations, #ITM.
struct Moments {
    double n, mean, m2, itm;
};
using TaskMoments = Moments;

}  // namespace qk
