// Allocation-free pricing entry point.
//
// Some callers cannot allocate device memory on the pricing path: a host
// application that owns all GPU memory through its own pool and forbids any
// allocation outside it, or a latency-critical caller for which cudaMalloc /
// cudaFree (which can synchronize the device and take milliseconds) is not
// acceptable between requests.  qk_price_noalloc serves them: it runs the same
// fused path kernel and tile merge as qk_price_batch, but every byte of scratch
// it needs (task descriptor, queue cursor, per-tile moment records, merged
// moments) lives in one file-scope device array of fixed size.  No handle is
// involved, and after the first call on a device nothing is allocated.
//
// Limits and rules of use:
//   * scratch is kNoAllocScratchBytes (about 4.1 MiB) per device, held until the
//     process exits;
//   * the first call on each device is its set-up, and that call does take device
//     memory: the CUDA runtime loads device code lazily, so the array is reserved
//     and the pricing kernels' code is loaded on that device then (the set-up
//     loads every kernel kind the entry point can launch).  Make the first call
//     during the caller's own set-up, before its memory pool takes the device's
//     free memory.  The first launch of a kernel kind can also make the driver
//     grow its per-thread local-memory reservation, so a caller that must see no
//     allocation at all afterwards prices one small contract of each kind
//     (precision x model x scheme, with or without path-dependent legs) it will
//     use during set-up;
//   * one forward contract (no American leg), no Greeks, at most
//     kNoAllocMaxRecords tile records: ceil(n_paths / 2048) * n_payoffs <= 131072
//     (for example 33,554,432 paths with 8 legs, 53,687,091 with 5);
//   * the set-up looks up the array's device address (cudaGetSymbolAddress) with
//     that device current; make the first call before any stream capture;
//   * every call shares the one array and it keeps the previous call's contents;
//     the queue cursor is cleared at the start of each call, every other field is
//     overwritten before it is read.  Calls whose GPU work overlaps (different
//     streams, threads or processes sharing the library on one device) race on
//     the array: serialize them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "qk_engine.h"
#include "qk_host.h"
#include "qk_kernels.h"

namespace {

constexpr size_t kNoAllocMaxRecords = 131072;
constexpr size_t kNoAllocTaskBytes = (sizeof(qk::TaskDev) + 255) / 256 * 256;
constexpr size_t kNoAllocSmallBytes = 256;  // prefix (int64) + cursor (uint64)
constexpr size_t kNoAllocMomentBytes = (QK_MAX_PAYOFFS * sizeof(qk::Moments) + 255) / 256 * 256;
constexpr size_t kNoAllocScratchBytes =
    kNoAllocTaskBytes + kNoAllocSmallBytes + kNoAllocMomentBytes + kNoAllocMaxRecords * sizeof(qk::Moments);
constexpr int kMaxDevices = 64;
constexpr int kNoAllocPathsPerTile = qk::kWarpTilePaths * 64;  // warp tiles of 64 rounds

// The scratch array.  In host code `g_noalloc_scratch` is only a handle for the
// symbol, never a device address: the address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
void *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device).
qk_status scratch_for_current_device(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return qk::fail(QK_ERR_NO_DEVICE, std::string("qk_price_noalloc: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return qk::fail(QK_ERR_UNSUPPORTED, "qk_price_noalloc: device index above 63");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return qk::fail(QK_ERR_CUDA, std::string("qk_price_noalloc: cudaGetSymbolAddress failed: ") +
                                             cudaGetErrorString(e));
        // load the device code of every kernel this entry point launches now, so that
        // later calls do not load it (with lazy module loading, a kernel's code is
        // loaded into device memory on its first use)
        e = qk::preload_noalloc_kernels();
        if (e != cudaSuccess)
            return qk::fail(QK_ERR_CUDA, std::string("qk_price_noalloc: loading the kernels failed: ") +
                                             cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return QK_OK;
}

}  // namespace

extern "C" qk_status qk_price_noalloc(const qk_contract *c, void *stream, qk_result *out) {
    if (!c || !out) return qk::fail(QK_ERR_INVALID_ARG, "qk_price_noalloc: NULL argument");
    qk_status s = qk::validate_contract(*c, nullptr);
    if (s != QK_OK) return s;
    for (int k = 0; k < c->n_payoffs; ++k)
        if (c->payoffs[k].type == QK_AMERICAN)
            return qk::fail(QK_ERR_UNSUPPORTED, "qk_price_noalloc: American contracts need LSM slabs; use qk_price_batch");
    if (c->antithetic) return qk::fail(QK_ERR_UNSUPPORTED, "qk_price_noalloc: antithetic pairs go through qk_price_batch");
    const int64_t tiles = (c->n_paths + kNoAllocPathsPerTile - 1) / kNoAllocPathsPerTile;
    if (static_cast<size_t>(tiles) * c->n_payoffs > kNoAllocMaxRecords)
        return qk::fail(QK_ERR_CAPACITY, "qk_price_noalloc: ceil(n_paths / 2048) * n_payoffs = " +
                                             std::to_string(tiles * c->n_payoffs) +
                                             " exceeds the fixed scratch of 131072 tile records");
    void *base = nullptr;
    if ((s = scratch_for_current_device(&base)) != QK_OK) return s;
    char *b = static_cast<char *>(base);
    qk::TaskDev *d_task = reinterpret_cast<qk::TaskDev *>(b);
    int64_t *d_prefix = reinterpret_cast<int64_t *>(b + kNoAllocTaskBytes);
    unsigned long long *d_cursor = reinterpret_cast<unsigned long long *>(b + kNoAllocTaskBytes + 128);
    qk::Moments *d_moments = reinterpret_cast<qk::Moments *>(b + kNoAllocTaskBytes + kNoAllocSmallBytes);
    qk::Moments *d_partials =
        reinterpret_cast<qk::Moments *>(b + kNoAllocTaskBytes + kNoAllocSmallBytes + kNoAllocMomentBytes);

    double scale = 1.0;
    const qk_contract n = qk::normalised(*c, &scale);
    qk::TaskDev t = qk::make_task(n, 64);
    t.tile_begin = 0;
    t.partial_base = 0;
    const int64_t prefix0 = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int dev = 0;
    cudaGetDevice(&dev);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int per_sm = qk::price_tiles_max_blocks_per_sm(t.precision, t.model, t.scheme, t.lane_mode, t.track != 0);
    const int grid = static_cast<int>(std::min<int64_t>((t.n_tiles + 7) / 8, static_cast<int64_t>(sms) * per_sm));
    qk::Moments m[QK_MAX_PAYOFFS];
    cudaError_t e = cudaMemcpyAsync(d_task, &t, sizeof(t), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_prefix, &prefix0, sizeof(prefix0), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_cursor, 0, sizeof(unsigned long long), st);  // queue starts empty
    if (e == cudaSuccess)
        e = qk::launch_price_tiles(t.precision, t.model, t.scheme, std::max(grid, 1), st, d_task, d_prefix, 1, 0,
                                   t.n_tiles, d_cursor, d_partials, true, c->seed, t.lane_mode, t.track != 0);
    if (e == cudaSuccess) e = qk::launch_merge_tasks(1, st, d_task, d_partials, d_moments);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m, d_moments, sizeof(m), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return qk::fail(QK_ERR_CUDA, std::string("qk_price_noalloc: ") + cudaGetErrorString(e));

    // OptionPricer::evaluate_option_price (OptionPricer.hpp:204-249) per leg
    std::memset(out, 0, sizeof(*out));
    out->status = QK_OK;
    out->n_payoffs = n.n_payoffs;
    out->n_paths = n.n_paths;
    out->path_steps = static_cast<double>(n.n_paths) * n.n_steps;
    for (int k = 0; k < n.n_payoffs; ++k) {
        const double N = m[k].n;
        const double eff = std::exp(-n.r * n.T) * (n.payoffs[k].type == QK_BINARY_CASH ? 1.0 : scale);
        out->p[k].price = m[k].mean * eff;
        out->p[k].std_error = N > 1.0 ? std::sqrt(m[k].m2 / (N - 1.0) / N) * eff : 0.0;
        out->p[k].prob_itm = N > 0.0 ? m[k].itm / N : 0.0;
    }
    return QK_OK;
}
