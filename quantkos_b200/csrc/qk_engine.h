// Host engine state: the opaque qk_handle, device/pinned arenas, and the plan
// (task list) of one pricing call.
#pragma once

#include <array>
#include <cuda_runtime.h>

#include <vector>

#include "qk_internal.h"

namespace qk {

// Grow-only device allocation owned by a handle (replaces the per-run Kokkos
// Views of PathsMCBatchMem / BackwardLSMMemory: allocated once, reused).  With a
// stream set, growth is stream-ordered (cudaFreeAsync / cudaMallocAsync on that
// stream, from the device's memory pool), so growing one handle's arena does not
// synchronize the device and stall other handles' work; it grows by at least half
// its size, so growth events are few.
struct DevArena {
    void *ptr = nullptr;
    size_t cap = 0;
    cudaStream_t stream = nullptr;  // the owning handle's stream (nullptr: cudaMalloc / cudaFree)
    qk_status ensure(size_t bytes);
    void release();
};

// Grow-only pinned host staging buffer (at least 1 MiB, grows by at least half its size:
// pinning host memory is slow and can stall other work, so it happens rarely).
struct HostArena {
    void *ptr = nullptr;
    size_t cap = 0;
    // Buffers outgrown while the handle lives: cudaFreeHost synchronizes the whole
    // device, so a growth keeps the old buffer here and release() (at handle
    // destruction, after its stream has drained) frees them all.  Geometric growth
    // keeps their total below the current buffer's size.
    std::vector<void *> retired;
    qk_status ensure(size_t bytes);
    void release();
};

struct LsmTaskInfo {
    int contract, role, grid;  // grid: blocks whose moments the job wrote
    int64_t moments_base;      // first of them in the per-block moments
    int64_t n_paths;
    double intrinsic0, eps;
};

struct Plan {
    int n_contracts = 0;
    bool plain = false;
    std::vector<qk_greeks> greeks;     // per contract; mask 0 = no Greeks
    const qk_greeks *g_of(int i) const { return greeks[i].mask ? &greeks[i] : nullptr; }
    std::vector<qk_contract> norm;     // normalised contracts
    std::vector<double> scale;         // price scale factor per contract
    std::vector<int32_t> status;       // per-contract status
    std::vector<TaskDev> tasks;        // forward tasks in schedule order
    std::vector<int> task_contract, task_role;
    std::vector<int> task_of;          // [contract * kNumRoles + role] -> task index or -1
    std::vector<int> american;         // contracts priced by LSM
    int64_t total_slots = 0;
    int64_t total_records = 0;
    int64_t total_chunks = 0;  // level-1 merge chunks over all tasks
    double path_steps = 0.0;
    double lsm_path_steps = 0.0;
    std::vector<LsmTaskInfo> lsm_tasks;
};

// LSM working set of one task on the device.
struct LsmArena {
    DevArena slab_S, slab_v, cashflow, block_sums, coeffs, status;
};

// American jobs of one call run on up to kLsmLanes streams at once, each stream with
// its own working set, so that the fixed per-date cost of small jobs overlaps.
constexpr int kLsmLanes = 4;
// The persistent launches of the kernel kinds of one call run on up to kKindStreams
// streams forked from the handle's stream, so that one kind's tail overlaps the next.
constexpr int kKindStreams = 8;

}  // namespace qk

// Launch shape of each kernel kind, [precision (FP64, FP32)][model][scheme], that a
// handle starts with: in FP32 48 tiles per warp slot, two paths per lane and blocks of
// 512 threads, with the guided tail except for Heston QE (the shapes measured fastest
// on large contracts; qk_autotune picks per workload); in FP64 24 tiles, one path per
// lane and blocks of 256 threads.
using ShapeTable = std::array<std::array<std::array<int, 3>, 2>, 2>;
constexpr ShapeTable kDefaultTilesPerWarp = {{{{{{24, 24, 24}}, {{24, 24, 24}}}}, {{{{48, 48, 48}}, {{48, 48, 48}}}}}};
constexpr ShapeTable kDefaultGuidedTail = {{{{{{0, 0, 0}}, {{0, 0, 0}}}}, {{{{1, 1, 0}}, {{1, 1, 1}}}}}};
constexpr ShapeTable kDefaultPathsPerLane = {{{{{{1, 1, 1}}, {{1, 1, 1}}}}, {{{{2, 2, 2}}, {{2, 2, 2}}}}}};
constexpr ShapeTable kDefaultBlock = {{{{{{256, 256, 256}}, {{256, 256, 256}}}}, {{{{512, 512, 512}}, {{512, 512, 512}}}}}};

struct qk_handle {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_paths0 = nullptr, ev_paths1 = nullptr, ev_end = nullptr;
    qk::DevArena d_tasks, d_prefix, d_partials, d_moments, d_cursor, d_trace, d_chunks;
    qk::HostArena h_tasks, h_moments, h_lsm;
    qk::DevArena d_lsm_moments;
    qk::LsmArena lsm[qk::kLsmLanes];
    qk::DevArena lsm_task, lsm_centre;    // descriptors and centring shifts of all jobs of a call
    cudaStream_t lsm_stream[qk::kLsmLanes] = {};
    cudaStream_t kind_stream[qk::kKindStreams] = {};
    cudaEvent_t kind_fork = nullptr, kind_join[qk::kKindStreams] = {};
    cudaEvent_t lsm_fork = nullptr, lsm_join[qk::kLsmLanes] = {};
    qk::Plan plan;
    bool prepared = false;
    cudaGraphExec_t graph = nullptr;  // the prepared batch's launch sequence (qk_batch_prepare)
    int64_t graph_launches = 0;
    // launch shape per kernel kind [precision][model][scheme] (autotuner); starts at, and
    // qk_tune_reset restores, the kDefault* tables
    ShapeTable tune_tpw = kDefaultTilesPerWarp;
    ShapeTable tune_tail = kDefaultGuidedTail;
    ShapeTable tune_lanes = kDefaultPathsPerLane;  // paths per lane: 1 or 2
    ShapeTable tune_block = kDefaultBlock;         // threads per block of the pricing kernel
    qk_timing timing{};
    int64_t launches = 0;
    int64_t h2d_bytes = 0, d2h_bytes = 0;
    double lsm_ms = 0.0, lsm_paths_ms = 0.0;
    int64_t lsm_launches = 0;
    std::vector<cudaEvent_t> lsm_events;  // per LSM job: forward start, forward end, sweep end
    size_t lsm_jobs = 0;
};

namespace qk {

enum : int { kNumRoles = 12 };

TaskDev make_task(const qk_contract &b, int ppt, int lane_mode = kLaneOne);
qk_contract normalised(const qk_contract &c, double *scale);
qk_contract bumped(const qk_contract &n, const qk_greeks *g, int role);
std::vector<int> roles_for(const qk_greeks *g, double T);

// Plan, run and assemble a set of contracts; `gs` holds one Greeks request per
// contract (or NULL).  Used by qk_price_* and by the serving lanes.
qk_status price_contracts(qk_handle *h, const qk_contract *c, int32_t n, const qk_greeks *gs, qk_result *out, bool plain);

// Memory held in a device's default pool (whose release threshold the handles raise so
// that it keeps what it has mapped): pool_reserve maps `bytes` into it once (allocate and
// free on `s`) and adds them to what handle destruction trims the pool down to; a
// server reserves its budget this way, so that its lanes' arena growth is served from
// memory the pool holds instead of mapping new memory, which blocks every other lane's
// driver calls while it runs.  pool_release gives them back and trims the pool.
qk_status pool_reserve(int device, cudaStream_t s, size_t bytes);
void pool_release(int device, size_t bytes);
void pool_trim(int device);

// Every path's leg-0 payoff (undiscounted, normalised) of a contract, on the host.
qk_status payoffs_dump(qk_handle *h, const qk_contract &c, std::vector<double> &out);
qk_status payoffs_range(qk_handle *h, const qk_contract &c, int64_t first, int64_t count, double *out);

// Longstaff-Schwartz for the American contracts of a plan (qk_lsm.cu).
qk_status run_lsm_contracts(qk_handle *h, Plan &plan, bool plain, std::vector<Moments> &moments);
void assemble_lsm_results(qk_handle *h, const Plan &plan, const std::vector<Moments> &moments, qk_result *out);
void lsm_release(qk_handle *h);
qk_status lsm_events_ensure(qk_handle *h, size_t n);
// Device time of the last call's LSM jobs: forward slab kernels and backward sweeps.
void lsm_timing(qk_handle *h, double *paths_ms, double *sweep_ms);
// Drop the prepared batch (its graph holds pointers into the handle's arenas).
void release_prepared(qk_handle *h);

}  // namespace qk
