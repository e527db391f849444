// Host-visible launchers of the device kernels.
#pragma once

#include <cuda_runtime.h>

#include "qk_internal.h"

namespace qk {

constexpr int kPathBlock = 256;     // threads per block of the path kernels (default of the pricing kernel)
// Largest block of the pricing kernel, per precision: FP32 blocks of 128, 256 or 512
// threads under the same 64-register budget; FP64 blocks of up to 256 threads.
template <class R>
constexpr int path_block_max() {
    return sizeof(R) == 4 ? 512 : 256;
}
constexpr int kWarpTilePaths = 32;  // paths per round of a warp tile (one per lane)
#ifndef QK_PATH_MIN_BLOCKS_FP32
#define QK_PATH_MIN_BLOCKS_FP32 4
#endif
constexpr int kPathMinBlocksFp32 = QK_PATH_MIN_BLOCKS_FP32;  // resident blocks per SM the FP32 path kernel is register-budgeted for

// uniform_key: every task of the launch has Philox key `seed` (round keys go in the
// kernel parameters); otherwise each task's key is read from its descriptor.
// lane_mode: what a lane simulates for every task of the launch (TaskDev::lane_mode).
// track: some task of the launch has a leg that reads the path state (TaskDev::track);
// false selects the kernel that keeps none.
cudaError_t launch_price_tiles(int precision, int model, int scheme, int grid, cudaStream_t s, const TaskDev *tasks,
                               const int64_t *prefix, int32_t n_tasks, int64_t slot_begin, int64_t slot_end,
                               unsigned long long *cursor, Moments *partials, bool uniform_key, uint64_t seed,
                               int lane_mode = kLaneOne, bool track = true, int block = kPathBlock);
// max_tiles: the largest n_tiles among the tasks (sets the block width).
cudaError_t launch_merge_tasks(int n_tasks, cudaStream_t s, const TaskDev *tasks, const Moments *partials,
                               TaskMoments *out, int64_t max_tiles = 0);
// Tile records per level-1 merge chunk.
constexpr int kMergeChunkTiles = 512;
// Two-level merge: level 1 reduces chunks of kMergeChunkTiles tile records
// (n_chunks = sum of the tasks' n_chunks) into chunks[n_chunks][QK_MAX_PAYOFFS],
// level 2 reduces each task's chunk records into out[task][QK_MAX_PAYOFFS].
cudaError_t launch_merge_two_level(int n_tasks, int64_t n_chunks, cudaStream_t s, const TaskDev *tasks,
                                   const Moments *partials, Moments *chunks, TaskMoments *out);
// paths_per_thread 2: each thread simulates two consecutive paths (same values).
cudaError_t launch_slab_paths(int precision, int model, int scheme, uint64_t seed, cudaStream_t s, const TaskDev *task,
                              int64_t first_path, int64_t count, int stride, void *slab_S, void *slab_v, int64_t ld,
                              int paths_per_thread = 1);
cudaError_t launch_step_trace(int precision, cudaStream_t s, const TaskDev *task, const double *z, const double *u,
                              int umax, int n, double *S_out, double *v_out, int *status);
// Leg-0 payoffs of paths first .. first + count - 1 of the task (undiscounted, normalised).
cudaError_t launch_payoff_paths(int precision, cudaStream_t s, const TaskDev *task, int64_t first, int64_t count,
                                double *out);
// One leg's payoff on the fed spot sequence S[0..n-1] starting from S0 (one thread).
cudaError_t launch_payoff_trace(int precision, cudaStream_t s, const PayoffSpec &ps, const double *S, int n, double S0,
                                double *out);
int price_tiles_max_blocks_per_sm(int precision, int model, int scheme, int lane_mode = kLaneOne,
                                  bool track = true, int block = kPathBlock);
// Whether `block` threads per block is a valid launch of the pricing kernel in `precision`.
bool price_tiles_block_ok(int precision, int block);
// Loads the device code of every one-path-per-lane pricing kernel (both precisions,
// every model and scheme, with and without path state) and of the one-block-per-task
// merge, without launching anything.
cudaError_t preload_noalloc_kernels();
// Load the device code of every kernel of the engine on the current device (path and
// merge kernels; the LSM kernels).  With lazy module loading, a kernel's first launch
// loads its code and can synchronize the context while other streams' kernels run;
// handles preload everything once per device so that no pricing call pays that.
cudaError_t preload_path_kernels();
cudaError_t preload_lsm_kernels();
// Times a kernel of independent ex2.approx chains; returns its duration and MUFU op count.
cudaError_t launch_sfu_probe(cudaStream_t s, int sm_count, float *sink, cudaEvent_t e0, cudaEvent_t e1, float *ms,
                             double *ops);

}  // namespace qk
