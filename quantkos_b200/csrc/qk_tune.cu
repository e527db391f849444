// Autotuner of the batched engine's launch shape.
//
// The persistent path kernel balances its work through a device queue of warp
// tiles; how many rounds a tile holds trades the queue's end-of-launch tail (big
// tiles leave warps idle while the last ones finish) against per-tile overhead
// (one FP64 record per tile and leg, merged afterwards), and a lane may carry two
// independent paths (more instruction-level parallelism, twice the registers).  The best point depends
// on the kernel kind and on the mix of contracts, so it is measured: the sample is
// split by kind (precision, model, scheme), every kind is priced under each
// candidate shape and the shortest device time of the call (CUDA events on the
// handle's stream around descriptor upload, path kernels and merge) wins; then the
// threads per block of the pricing kernel are timed at that shape.  Tiles of a contract cover the same paths
// whatever the shape, so the shape changes no price beyond the rounding of the
// moment merge.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <iterator>
#include <limits>
#include <string>
#include <vector>

#include "qk_engine.h"
#include "qk_host.h"
#include "qk_kernels.h"

namespace {

constexpr int kTilesPerWarp[] = {4, 8, 12, 24, 48};
constexpr int kTails[] = {0, 1};
constexpr int kLanes[] = {1, 2};
// second stage: threads per block at the best (tiles, tail, lanes) of the first
constexpr int kBlocks[] = {128, 256, 512};
// The handle's default shape of a kind (the tables in qk_engine.h).
void default_shape(int precision, int model, int scheme, int &tpw, int &tail, int &lanes) {
    tpw = kDefaultTilesPerWarp[precision][model][scheme];
    tail = kDefaultGuidedTail[precision][model][scheme];
    lanes = kDefaultPathsPerLane[precision][model][scheme];
}
int default_block(int precision, int model, int scheme) { return kDefaultBlock[precision][model][scheme]; }

}  // namespace

extern "C" qk_status qk_tune_reset(qk_handle *h) {
    if (!h) return qk::fail(QK_ERR_INVALID_ARG, "qk_tune_reset: NULL handle");
    for (int pr = 0; pr < 2; ++pr)
        for (int md = 0; md < 2; ++md)
            for (int sc = 0; sc < 3; ++sc)
                default_shape(pr, md, sc, h->tune_tpw[pr][md][sc], h->tune_tail[pr][md][sc], h->tune_lanes[pr][md][sc]);
    h->tune_block = kDefaultBlock;
    return QK_OK;
}

extern "C" qk_status qk_tune_set_block(qk_handle *h, int32_t precision, int32_t model, int32_t scheme,
                                       int32_t threads_per_block) {
    if (!h) return qk::fail(QK_ERR_INVALID_ARG, "qk_tune_set_block: NULL handle");
    if (precision < 0 || precision > 1 || model < 0 || model > 1 || scheme < 0 || scheme > 2)
        return qk::fail(QK_ERR_INVALID_ARG, "qk_tune_set_block: precision, model or scheme out of range");
    if (!qk::price_tiles_block_ok(precision, threads_per_block) ||
        (threads_per_block != 128 && threads_per_block != 256 && threads_per_block != 512))
        return qk::fail(QK_ERR_INVALID_ARG, "qk_tune_set_block: 128, 256 or 512 threads (FP64: 128 or 256)");
    h->tune_block[precision][model][scheme] = threads_per_block;
    return QK_OK;
}

extern "C" qk_status qk_tune_set(qk_handle *h, int32_t precision, int32_t model, int32_t scheme,
                                 int32_t tiles_per_warp, int32_t guided_tail, int32_t paths_per_lane) {
    if (!h) return qk::fail(QK_ERR_INVALID_ARG, "qk_tune_set: NULL handle");
    if (precision < 0 || precision > 1 || model < 0 || model > 1 || scheme < 0 || scheme > 2)
        return qk::fail(QK_ERR_INVALID_ARG, "qk_tune_set: precision, model or scheme out of range");
    if (tiles_per_warp < 1 || tiles_per_warp > 1024)
        return qk::fail(QK_ERR_INVALID_ARG, "qk_tune_set: tiles_per_warp must be in [1, 1024]");
    if (paths_per_lane != 1 && paths_per_lane != 2)
        return qk::fail(QK_ERR_INVALID_ARG, "qk_tune_set: paths_per_lane must be 1 or 2");
    h->tune_tpw[precision][model][scheme] = tiles_per_warp;
    h->tune_tail[precision][model][scheme] = guided_tail ? 1 : 0;
    h->tune_lanes[precision][model][scheme] = paths_per_lane;
    return QK_OK;
}

extern "C" qk_status qk_autotune(qk_handle *h, const qk_contract *c, int32_t n, const qk_greeks *g, int32_t reps,
                                 qk_tune_report *out) {
    if (!h || !c || !out || n < 1) return qk::fail(QK_ERR_INVALID_ARG, "qk_autotune: NULL argument or empty sample");
    if (reps < 1 || reps > 100) return qk::fail(QK_ERR_INVALID_ARG, "qk_autotune: reps must be in [1, 100]");
    std::memset(out, 0, sizeof(*out));
    out->candidates = static_cast<int32_t>(std::size(kTilesPerWarp) * std::size(kTails) * std::size(kLanes) +
                                           std::size(kBlocks) - 1);
    // sample indices per kind, forward contracts only
    std::vector<int> by_kind[QK_TUNE_KINDS];
    for (int i = 0; i < n; ++i) {
        const qk_status s = qk::validate_contract(c[i], g);
        if (s != QK_OK) return qk::fail(s, "qk_autotune: contract " + std::to_string(i) + ": " + qk::g_last_error);
        if (c[i].payoffs[0].type == QK_AMERICAN) continue;
        by_kind[(c[i].precision * 2 + c[i].model) * 3 + c[i].scheme].push_back(i);
    }
    for (int kind = 0; kind < QK_TUNE_KINDS; ++kind) {
        if (by_kind[kind].empty()) continue;
        const int pr = kind / 6, md = (kind / 3) % 2, sc = kind % 3;
        std::vector<qk_contract> sub;
        std::vector<qk_greeks> gsub;
        for (int i : by_kind[kind]) {
            sub.push_back(c[i]);
            qk_greeks x;
            if (g) x = *g;
            else std::memset(&x, 0, sizeof(x));
            gsub.push_back(x);
        }
        std::vector<qk_result> res(sub.size());
        double best = std::numeric_limits<double>::infinity(), dflt = 0.0;
        int dflt_tpw, dflt_tail, dflt_lanes;
        default_shape(pr, md, sc, dflt_tpw, dflt_tail, dflt_lanes);
        int best_tpw = dflt_tpw, best_tail = dflt_tail, best_lanes = dflt_lanes;
        const int dflt_block = default_block(pr, md, sc);
        h->tune_block[pr][md][sc] = dflt_block;
        auto time_shape = [&](double &ms) -> qk_status {
            ms = std::numeric_limits<double>::infinity();
            for (int r = 0; r <= reps; ++r) {  // run 0 warms up
                const qk_status s = qk::price_contracts(h, sub.data(), static_cast<int32_t>(sub.size()), gsub.data(),
                                                        res.data(), false);
                if (s != QK_OK) {
                    default_shape(pr, md, sc, h->tune_tpw[pr][md][sc], h->tune_tail[pr][md][sc],
                                  h->tune_lanes[pr][md][sc]);
                    h->tune_block[pr][md][sc] = dflt_block;
                    return s;
                }
                if (r > 0) ms = std::min(ms, h->timing.device_ms);
            }
            return QK_OK;
        };
        for (int lanes : kLanes)
            for (int tpw : kTilesPerWarp)
                for (int tail : kTails) {
                    h->tune_tpw[pr][md][sc] = tpw;
                    h->tune_tail[pr][md][sc] = tail;
                    h->tune_lanes[pr][md][sc] = lanes;
                    double ms;
                    const qk_status s = time_shape(ms);
                    if (s != QK_OK) return s;
                    if (tpw == dflt_tpw && tail == dflt_tail && lanes == dflt_lanes) dflt = ms;
                    if (ms < best) {
                        best = ms;
                        best_tpw = tpw;
                        best_tail = tail;
                        best_lanes = lanes;
                    }
                }
        h->tune_tpw[pr][md][sc] = best_tpw;
        h->tune_tail[pr][md][sc] = best_tail;
        h->tune_lanes[pr][md][sc] = best_lanes;
        // threads per block at that shape (the tiles and their paths do not depend on it)
        int best_block = dflt_block;
        for (int blk : kBlocks) {
            if (blk == dflt_block || !qk::price_tiles_block_ok(pr, blk)) continue;
            h->tune_block[pr][md][sc] = blk;
            double ms;
            const qk_status s = time_shape(ms);
            if (s != QK_OK) return s;
            if (ms < best) {
                best = ms;
                best_block = blk;
            }
        }
        h->tune_block[pr][md][sc] = best_block;
        const int k = out->n_kinds++;
        out->precision[k] = pr;
        out->model[k] = md;
        out->scheme[k] = sc;
        out->tiles_per_warp[k] = best_tpw;
        out->guided_tail[k] = best_tail;
        out->paths_per_lane[k] = best_lanes;
        out->block_size[k] = best_block;
        out->best_ms[k] = best;
        out->default_ms[k] = dflt;
    }
    return QK_OK;
}
