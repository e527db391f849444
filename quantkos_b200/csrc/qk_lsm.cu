// Longstaff-Schwartz American pricing, fully device-resident (sm_100a).
//
// Reference path (paths relative to the reference project): the forward pass
// stores every path to a host master matrix (include/core/memory/LSMMemory.hpp:145-183),
// then a host loop streams one time slice per step over PCIe, reduces the
// regression sums on the device, solves a Cholesky on the host and updates the
// cash flows (include/core/engine/ForwardBackwardMC.hpp:204-255,
// include/core/options/LSMAmerican.hpp:252-613).
//
// Here: the forward kernel writes spot (and variance) only at the exercise
// dates, as SoA slabs slab[date][path] in HBM; the backward sweep is one kernel
// per date that applies the exercise decision of date d and accumulates the
// regression sums of date d-1 in the same pass, streaming the slabs through
// shared memory with cp.async; the last block to finish reduces the block sums
// and solves the normal equations in FP64 on the device.  No host round trip
// happens inside the sweep.
//
// Two regression modes:
//   QK_LSM_LAGUERRE3 — the reference's: X = S/K, Laguerre L0..L3 (LSMAmerican.hpp:157-199),
//     ITM paths, Tikhonov 1e-8 on the diagonal, Cholesky with a 1e-14 pivot floor and
//     the mean fallback (LSMAmerican.hpp:516-613);
//   QK_LSM_POLY_SV — basis {1, S, S^2, S^3, v, S v} on S/K-scaled values, evaluated in the
//     shifted coordinates x = S/K - c_x(d), w = v - c_v(d) (same span), FP64 Cholesky of
//     the Jacobi-scaled Gram, Householder QR with column pivoting when the Cholesky
//     condition estimate exceeds 1e8, mean fallback below 6 ITM paths.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "qk_device.cuh"
#include "qk_engine.h"
#include "qk_host.h"
#include "qk_kernels.h"

namespace qk {

constexpr int kLsmBlock = 256;
#ifndef QK_LSM_MIN_BLOCKS
#define QK_LSM_MIN_BLOCKS 2  // resident sweep blocks per SM the register budget is set for
#endif
constexpr int kMaxCoef = 8;

template <int BASIS>
struct BasisTraits;
template <>
struct BasisTraits<QK_LSM_LAGUERRE3> {
    static constexpr int NB = 4;
};
template <>
struct BasisTraits<QK_LSM_POLY_SV> {
    static constexpr int NB = 6;
};
template <int NB>
struct Sums {
    static constexpr int NSUM = NB * (NB + 1) / 2 + NB + 1;  // upper Gram, rhs, count
};

struct LsmArgs {
    int64_t N, ld;
    int right;
    int n_dates;
    double K;     // normalised strike
    double disc;  // exp(-r * date spacing)
};

template <class R>
__device__ __forceinline__ R lsm_intrinsic(int right, R S, R K) {
    return right == kCall ? (S > K ? S - K : R(0)) : (K > S ? K - S : R(0));
}

// Basis values of one path at one date.  LAGUERRE3 in the working precision
// (LaguerreBasis<4>::evaluate, Horner form, LSMAmerican.hpp:183-192); POLY_SV in
// double on the centred coordinates x = S/K - c_x, w = v - c_v.
template <class R>
__device__ __forceinline__ void laguerre_basis(R S, R K, R *b) {
    const R X = S / K;
    b[0] = R(1);
    b[1] = R(1) - X;
    b[2] = ((R(0.5) * X - R(2)) * X) + R(1);
    b[3] = (((static_cast<R>(-1.0 / 6.0) * X + R(1.5)) * X - R(3)) * X) + R(1);
}

struct PolyPoint {
    double x, w;
};
template <class R>
__device__ __forceinline__ PolyPoint poly_point(R S, R v, double inv_K, double cx, double cv) {
    return PolyPoint{static_cast<double>(S) * inv_K - cx, static_cast<double>(v) - cv};
}

// Expected value of holding: sum of coefficients times basis, in double (LSMAmerican.hpp:484-502).
template <class R, int BASIS>
__device__ __forceinline__ double continuation(const double *c, R S, R v, R K, double inv_K, double cx, double cv) {
    if constexpr (BASIS == QK_LSM_LAGUERRE3) {
        R b[4];
        laguerre_basis<R>(S, K, b);
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) s += c[i] * static_cast<double>(b[i]);
        return s;
    } else {
        const PolyPoint q = poly_point<R>(S, v, inv_K, cx, cv);
        const double x = q.x, w = q.w;
        return c[0] + x * (c[1] + x * (c[2] + x * c[3])) + w * (c[4] + x * c[5]);
    }
}

// Regression sums kept per thread.  LAGUERRE3: the reference's products of basis
// values — upper Gram (10), right-hand side (4), count — 15 sums.  POLY_SV: every
// Gram entry of {1, x, x^2, x^3, w, x w} is a monomial x^a w^c, so the thread keeps
// the 15 distinct monomial sums (x^0..x^6, w x^0..x^4, w^2 x^0..x^2) and the 6
// right-hand sides, 21 sums, expanded to the Gram before the solve.
template <int BASIS>
struct AccTraits;
template <>
struct AccTraits<QK_LSM_LAGUERRE3> {
    static constexpr int N = 15;
};
template <>
struct AccTraits<QK_LSM_POLY_SV> {
    static constexpr int N = 21;
};

template <class R, int BASIS>
__device__ __forceinline__ void accumulate(double *acc, R S, R v, R K, double inv_K, double cx, double cv, R Y) {
    const double y = static_cast<double>(Y);
    if constexpr (BASIS == QK_LSM_LAGUERRE3) {
        R b[4];
        laguerre_basis<R>(S, K, b);
        int j = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const double br = static_cast<double>(b[r]);
#pragma unroll
            for (int q = r; q < 4; ++q) acc[j++] += br * static_cast<double>(b[q]);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[j++] += static_cast<double>(b[r]) * y;
        acc[j] += 1.0;
    } else {
        const PolyPoint q = poly_point<R>(S, v, inv_K, cx, cv);
        const double x = q.x, w = q.w;
        const double x2 = x * x, x3 = x2 * x, ww = w * w;
        acc[0] += 1.0;
        acc[1] += x;
        acc[2] += x2;
        acc[3] += x3;
        acc[4] += x2 * x2;
        acc[5] += x2 * x3;
        acc[6] += x3 * x3;
        acc[7] += w;
        acc[8] += w * x;
        acc[9] += w * x2;
        acc[10] += w * x3;
        acc[11] += w * x2 * x2;
        acc[12] += ww;
        acc[13] += ww * x;
        acc[14] += ww * x2;
        acc[15] += y;
        acc[16] += y * x;
        acc[17] += y * x2;
        acc[18] += y * x3;
        acc[19] += y * w;
        acc[20] += y * x * w;
    }
}

// FP32 slab with the 6-term basis: the per-path work (centred point, monomials,
// continuation) in FP32 on path pairs (sm_100 paired FP32 instructions), without
// branches — a path out of the money contributes the point (0, 0) with weight 0 —
// and the 21 sums kept in FP32 for kF32Flush chunk rounds (64 paths per thread)
// before the thread adds them to its FP64 sums.  An FP32 partial over 64 paths
// carries a relative rounding error of order 1e-6 at most, and partials round
// independently, so the FP64 totals over N paths stay accurate to far below the
// Monte Carlo error; the block and grid reductions and the solve remain FP64.
constexpr int kF32Flush = 16;

// Continuation value of two paths from the 6-term coefficients c (FP32, each
// duplicated into a pair).
__device__ __forceinline__ float2 continuation_f32x2(const float2 *c, float2 x, float2 w) {
    const float2 px = __ffma2_rn(x, __ffma2_rn(x, __ffma2_rn(x, c[3], c[2]), c[1]), c[0]);
    return __ffma2_rn(w, __ffma2_rn(x, c[5], c[4]), px);
}

// Same 21 sums as accumulate<R, QK_LSM_POLY_SV>, in FP32 on two paths; one = path
// weight (1 in the money, 0 otherwise, with x = w = y = 0).
__device__ __forceinline__ void accumulate_f32x2(float2 *acc, float2 x, float2 w, float2 y, float2 one) {
    const float2 x2 = __fmul2_rn(x, x), x3 = __fmul2_rn(x2, x), ww = __fmul2_rn(w, w);
    const float2 wx = __fmul2_rn(w, x), wx2 = __fmul2_rn(w, x2);
    acc[0] = __fadd2_rn(acc[0], one);
    acc[1] = __fadd2_rn(acc[1], x);
    acc[2] = __fadd2_rn(acc[2], x2);
    acc[3] = __fadd2_rn(acc[3], x3);
    acc[4] = __ffma2_rn(x2, x2, acc[4]);
    acc[5] = __ffma2_rn(x2, x3, acc[5]);
    acc[6] = __ffma2_rn(x3, x3, acc[6]);
    acc[7] = __fadd2_rn(acc[7], w);
    acc[8] = __fadd2_rn(acc[8], wx);
    acc[9] = __fadd2_rn(acc[9], wx2);
    acc[10] = __ffma2_rn(wx2, x, acc[10]);
    acc[11] = __ffma2_rn(wx2, x2, acc[11]);
    acc[12] = __fadd2_rn(acc[12], ww);
    acc[13] = __ffma2_rn(ww, x, acc[13]);
    acc[14] = __ffma2_rn(ww, x2, acc[14]);
    acc[15] = __fadd2_rn(acc[15], y);
    acc[16] = __ffma2_rn(y, x, acc[16]);
    acc[17] = __ffma2_rn(y, x2, acc[17]);
    acc[18] = __ffma2_rn(y, x3, acc[18]);
    acc[19] = __ffma2_rn(y, w, acc[19]);
    acc[20] = __ffma2_rn(y, wx, acc[20]);
}

// The solver's input: upper Gram (row-major), right-hand side, count.
template <int BASIS>
__device__ __forceinline__ void expand_sums(const double *acc, double *sums) {
    if constexpr (BASIS == QK_LSM_LAGUERRE3) {
        for (int j = 0; j < AccTraits<BASIS>::N; ++j) sums[j] = acc[j];
    } else {
        // basis i = x^pa[i] w^pc[i]
        const int pa[6] = {0, 1, 2, 3, 0, 1};
        const int pc[6] = {0, 0, 0, 0, 1, 1};
        int j = 0;
        for (int r = 0; r < 6; ++r)
            for (int q = r; q < 6; ++q) {
                const int a = pa[r] + pa[q], c = pc[r] + pc[q];
                sums[j++] = c == 0 ? acc[a] : (c == 1 ? acc[7 + a] : acc[12 + a]);
            }
        for (int r = 0; r < 6; ++r) sums[j++] = pc[r] == 0 ? acc[15 + pa[r]] : acc[19 + pa[r]];
        sums[j] = acc[0];
    }
}

// ---------------------------------------------------------------- FP64 solves
// Reference solve: Tikhonov 1e-8, Cholesky, 1e-14 pivot floor, mean fallback
// (LSMAmerican.hpp:516-613).  Returns 0 on success, 2 on fallback.
template <int NB>
__device__ int solve_reference(const double *sums, double *c) {
    double M[NB][NB], B[NB], L[NB][NB];
    int j = 0;
    for (int r = 0; r < NB; ++r)
        for (int q = r; q < NB; ++q) {
            M[r][q] = sums[j];
            M[q][r] = sums[j];
            ++j;
        }
    for (int r = 0; r < NB; ++r) B[r] = sums[j++];
    const double count = sums[j];
    for (int i = 0; i < NB; ++i) c[i] = 0.0;
    auto fallback = [&]() {
        if (count > 0.0) c[0] = B[0] / count;
        return 2;
    };
    if (count < static_cast<double>(NB)) return fallback();
    for (int i = 0; i < NB; ++i) M[i][i] += 1e-8;
    for (int i = 0; i < NB; ++i)
        for (int k = 0; k < NB; ++k) L[i][k] = 0.0;
    for (int i = 0; i < NB; ++i) {
        for (int jj = 0; jj <= i; ++jj) {
            double s = 0.0;
            for (int k = 0; k < jj; ++k) s += L[i][k] * L[jj][k];
            if (i == jj) {
                const double val = M[i][i] - s;
                if (val < 1e-14) return fallback();
                L[i][i] = sqrt(val);
            } else {
                L[i][jj] = (M[i][jj] - s) / L[jj][jj];
            }
        }
    }
    double y[NB];
    for (int i = 0; i < NB; ++i) {
        double s = 0.0;
        for (int k = 0; k < i; ++k) s += L[i][k] * y[k];
        y[i] = (B[i] - s) / L[i][i];
    }
    for (int i = NB - 1; i >= 0; --i) {
        double s = 0.0;
        for (int k = i + 1; k < NB; ++k) s += L[k][i] * c[k];
        c[i] = (y[i] - s) / L[i][i];
    }
    return 0;
}

// Centred/scaled Gram: Jacobi scaling, Cholesky with a condition estimate
// (max/min pivot)^2, Householder QR with column pivoting when that exceeds 1e8
// or the Cholesky breaks down.  Returns 0 Cholesky, 1 QR, 2 mean fallback.
template <int NB>
__device__ int solve_scaled(const double *sums, double *c) {
    double G[NB][NB], b[NB], D[NB];
    int j = 0;
    for (int r = 0; r < NB; ++r)
        for (int q = r; q < NB; ++q) {
            G[r][q] = sums[j];
            G[q][r] = sums[j];
            ++j;
        }
    for (int r = 0; r < NB; ++r) b[r] = sums[j++];
    const double count = sums[j];
    for (int i = 0; i < NB; ++i) c[i] = 0.0;
    if (count < static_cast<double>(NB)) {
        if (count > 0.0) c[0] = b[0] / count;
        return 2;
    }
    // one division per scale and per pivot (reciprocals), multiplications elsewhere:
    // this runs on one thread between two dates, in the sweep's critical path
    double invD[NB];
    for (int i = 0; i < NB; ++i) {
        D[i] = G[i][i] > 0.0 ? sqrt(G[i][i]) : 1.0;
        invD[i] = 1.0 / D[i];
    }
    for (int r = 0; r < NB; ++r) {
        b[r] *= invD[r];
        for (int q = 0; q < NB; ++q) G[r][q] *= invD[r] * invD[q];
    }
    // Cholesky
    double L[NB][NB], invL[NB];
    bool ok = true;
    double lmin = 1e300, lmax = 0.0;
    for (int i = 0; i < NB && ok; ++i) {
        for (int jj = 0; jj <= i; ++jj) {
            double s = G[i][jj];
            for (int k = 0; k < jj; ++k) s -= L[i][k] * L[jj][k];
            if (i == jj) {
                if (!(s > 0.0)) {
                    ok = false;
                    break;
                }
                L[i][i] = sqrt(s);
                invL[i] = 1.0 / L[i][i];
                lmin = fmin(lmin, L[i][i]);
                lmax = fmax(lmax, L[i][i]);
            } else {
                L[i][jj] = s * invL[jj];
            }
        }
    }
    if (ok && (lmax / lmin) * (lmax / lmin) <= 1e8) {
        double y[NB];
        for (int i = 0; i < NB; ++i) {
            double s = b[i];
            for (int k = 0; k < i; ++k) s -= L[i][k] * y[k];
            y[i] = s * invL[i];
        }
        for (int i = NB - 1; i >= 0; --i) {
            double s = y[i];
            for (int k = i + 1; k < NB; ++k) s -= L[k][i] * c[k];
            c[i] = s * invL[i];
        }
        for (int i = 0; i < NB; ++i) c[i] *= invD[i];
        return 0;
    }
    // Householder QR with column pivoting on the scaled Gram (rank-revealing), then
    // the basic solution of the truncated triangular system.
    double A[NB][NB], rhs[NB], norms[NB];
    int perm[NB];
    for (int r = 0; r < NB; ++r) {
        rhs[r] = b[r];
        for (int q = 0; q < NB; ++q) A[r][q] = G[r][q];
    }
    for (int q = 0; q < NB; ++q) {
        perm[q] = q;
        double s = 0.0;
        for (int r = 0; r < NB; ++r) s += A[r][q] * A[r][q];
        norms[q] = s;
    }
    int rank = 0;
    double r00 = 0.0;
    for (int k = 0; k < NB; ++k) {
        int best = k;
        for (int q = k + 1; q < NB; ++q)
            if (norms[q] > norms[best]) best = q;
        if (best != k) {
            for (int r = 0; r < NB; ++r) {
                const double t = A[r][k];
                A[r][k] = A[r][best];
                A[r][best] = t;
            }
            const double tn = norms[k];
            norms[k] = norms[best];
            norms[best] = tn;
            const int tp = perm[k];
            perm[k] = perm[best];
            perm[best] = tp;
        }
        double alpha = 0.0;
        for (int r = k; r < NB; ++r) alpha += A[r][k] * A[r][k];
        alpha = sqrt(alpha);
        if (k == 0) r00 = alpha;
        if (alpha <= 1e-10 * r00 || alpha == 0.0) break;
        if (A[k][k] > 0.0) alpha = -alpha;
        double vk[NB];
        for (int r = 0; r < NB; ++r) vk[r] = (r >= k) ? A[r][k] : 0.0;
        vk[k] -= alpha;
        double vnorm2 = 0.0;
        for (int r = k; r < NB; ++r) vnorm2 += vk[r] * vk[r];
        if (vnorm2 > 0.0) {
            for (int q = k; q < NB; ++q) {
                double s = 0.0;
                for (int r = k; r < NB; ++r) s += vk[r] * A[r][q];
                const double f = 2.0 * s / vnorm2;
                for (int r = k; r < NB; ++r) A[r][q] -= f * vk[r];
            }
            double s = 0.0;
            for (int r = k; r < NB; ++r) s += vk[r] * rhs[r];
            const double f = 2.0 * s / vnorm2;
            for (int r = k; r < NB; ++r) rhs[r] -= f * vk[r];
        }
        for (int q = k + 1; q < NB; ++q) norms[q] -= A[k][q] * A[k][q];
        ++rank;
    }
    double z[NB];
    for (int i = 0; i < NB; ++i) z[i] = 0.0;
    for (int i = rank - 1; i >= 0; --i) {
        double s = rhs[i];
        for (int k = i + 1; k < rank; ++k) s -= A[i][k] * z[k];
        z[i] = s / A[i][i];
    }
    for (int i = 0; i < NB; ++i) c[perm[i]] = z[i];
    for (int i = 0; i < NB; ++i) c[i] /= D[i];
    return 1;
}

// ---------------------------------------------------------------- streaming
// cp.async (16 bytes, L2 only) into shared memory with an L2 eviction-priority
// hint; completion is tracked per thread with commit/wait groups (no spin).
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, uint64_t policy) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "l"(policy)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// Programmatic dependent launch: the next date's kernel may start while this one
// finishes; griddepcontrol.wait returns once the preceding grid has completed and
// its writes are visible (immediately when there is no programmatic dependency).
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_wait_preceding() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_pending() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

constexpr int kLsmChunk = 4 * kLsmBlock;  // paths per staged chunk: four per thread

// Four consecutive entries at a 16-byte aligned address (shared or global).
__device__ __forceinline__ void load4(const float *p, float v[4]) {
    const float4 q = *reinterpret_cast<const float4 *>(p);
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
    v[3] = q.w;
}
__device__ __forceinline__ void load4(const double *p, double v[4]) {
    const double2 a = *reinterpret_cast<const double2 *>(p);
    const double2 b = *reinterpret_cast<const double2 *>(p + 2);
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
}
__device__ __forceinline__ void store4(float *p, const float v[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void store4(double *p, const double v[4]) {
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
    *reinterpret_cast<double2 *>(p + 2) = make_double2(v[2], v[3]);
}

// Shared-memory slots of one stage: spot at the update date, cash flows, spot at
// the Gram date, then (POLY_SV) variance at both dates.
template <int BASIS>
struct StageLayout {
    static constexpr int kArrays = BASIS == QK_LSM_POLY_SV ? 5 : 3;
    static constexpr int kSu = 0, kCf = 1, kSg = 2, kVu = 3, kVg = 4;
};

// Chunks in flight per block: with two resident blocks per SM, four FP32 stages keep
// about 48 KB of slab rows per SM outstanding (enough to cover HBM latency at full
// bandwidth); FP64 rows are twice the size, so two stages hold a comparable amount.
template <class R, int BASIS>
constexpr bool lsm_f32_poly() {
    return sizeof(R) == 4 && BASIS == QK_LSM_POLY_SV;
}
template <class R>
constexpr int lsm_stages() {
    return sizeof(R) == 4 ? 4 : 2;
}

template <class R, int BASIS>
constexpr size_t lsm_sweep_smem() {
    return lsm_stages<R>() * StageLayout<BASIS>::kArrays * kLsmChunk * sizeof(R);
}

// Backward sweep over one date pair.  init: cash flows start as the payoff at
// date d_upd (maturity); otherwise the exercise decision of date d_upd is
// applied with its solved coefficients.  Then, if d_gram >= 0, the ITM
// regression sums of date d_gram are accumulated with Y = cf * disc, reduced per
// block, and the last block to finish (counted on `done`) reduces all block sums
// in a fixed order and solves date d_gram's coefficients — no separate launch and
// no wait: every other block simply exits.
//
// Each block streams chunks of kLsmChunk paths (its chunks are blockIdx.x +
// k * gridDim.x) through two shared-memory stages: while chunk k is processed the
// copies of chunk k+1 are in flight.  The spot/variance rows of the update date are
// read for the last time here (L2 evict-first); those of the Gram date are read
// again by the next date's launch (L2 evict-last), so they are served from L2.
template <class R, int BASIS>
__global__ void __launch_bounds__(kLsmBlock, QK_LSM_MIN_BLOCKS) lsm_sweep_kernel(LsmArgs a, const R *__restrict__ slab_S,
                                                             const R *__restrict__ slab_v, R *__restrict__ cf,
                                                             int d_upd, int init, int d_gram,
                                                             double *__restrict__ coeffs,
                                                             const double *__restrict__ centre,
                                                             double *__restrict__ block_sums,
                                                             unsigned int *__restrict__ done, int *__restrict__ flags) {
    constexpr int NB = BasisTraits<BASIS>::NB;
    constexpr int NSUM = Sums<NB>::NSUM;
    constexpr int NACC = AccTraits<BASIS>::N;
    constexpr bool use_v = BASIS == QK_LSM_POLY_SV;
    constexpr bool kF32 = lsm_f32_poly<R, BASIS>();  // FP32 paired per-path work
    using L = StageLayout<BASIS>;
    extern __shared__ __align__(16) unsigned char lsm_smem[];
    R *stage = reinterpret_cast<R *>(lsm_smem);

    pdl_launch_dependents();  // the next date's blocks may take SM slots as this grid drains
    const R K = static_cast<R>(a.K);
    const double inv_K = 1.0 / a.K;
    const R disc = static_cast<R>(a.disc);
    const bool gram = d_gram >= 0;
    double acc[NACC];
#pragma unroll
    for (int j = 0; j < NACC; ++j) acc[j] = 0.0;
    float2 acc2[kF32 ? NACC : 1];
#pragma unroll
    for (int j = 0; j < (kF32 ? NACC : 1); ++j) acc2[j] = make_float2(0.0f, 0.0f);
    // adds this thread's FP32 partials to its FP64 sums
    auto flush = [&]() {
        if constexpr (kF32) {
#pragma unroll
            for (int j = 0; j < NACC; ++j) {
                acc[j] += static_cast<double>(acc2[j].x + acc2[j].y);
                acc2[j] = make_float2(0.0f, 0.0f);
            }
        }
    };
    double cxu = 0.0, cvu = 0.0, cxg = 0.0, cvg = 0.0;
    if (!init) {
        cxu = centre[2 * d_upd];
        cvu = centre[2 * d_upd + 1];
    }
    if (gram) {
        cxg = centre[2 * d_gram];
        cvg = centre[2 * d_gram + 1];
    }
    const float inv_Kf = static_cast<float>(inv_K);
    const float cxuf = static_cast<float>(cxu), cvuf = static_cast<float>(cvu);
    const float cxgf = static_cast<float>(cxg), cvgf = static_cast<float>(cvg);
    const R *Su = slab_S + static_cast<int64_t>(d_upd) * a.ld;
    const R *Vu = use_v ? slab_v + static_cast<int64_t>(d_upd) * a.ld : nullptr;
    const R *Sg = slab_S + static_cast<int64_t>(gram ? d_gram : 0) * a.ld;
    const R *Vg = use_v ? slab_v + static_cast<int64_t>(gram ? d_gram : 0) * a.ld : nullptr;
    const uint64_t pol_first = l2_policy_evict_first();
    const uint64_t pol_last = l2_policy_evict_last();
    const int64_t n_chunks = (a.ld + kLsmChunk - 1) / kLsmChunk;
    constexpr int kPer16 = 16 / static_cast<int>(sizeof(R));  // elements per 16-byte copy

    // Queue the copies of one chunk into stage st: the slab rows (written by the
    // forward kernel) and, unless `rows_only`, the cash flows (written by the
    // previous date's launch).  Rows hold ld elements, ld a multiple of 4, so no
    // 16-byte group straddles the end of a row.
    auto issue = [&](int64_t chunk, int st, bool rows, bool flows) {
        R *base = stage + static_cast<size_t>(st) * L::kArrays * kLsmChunk;
        const int64_t p0 = chunk * kLsmChunk;
        for (int e = threadIdx.x * kPer16; e < kLsmChunk; e += kLsmBlock * kPer16) {
            const int64_t i = p0 + e;
            if (i >= a.ld) break;
            if (rows) {
                cp_async16(base + L::kSu * kLsmChunk + e, Su + i, pol_first);
                if (gram) cp_async16(base + L::kSg * kLsmChunk + e, Sg + i, pol_last);
                if constexpr (use_v) {
                    cp_async16(base + L::kVu * kLsmChunk + e, Vu + i, pol_first);
                    if (gram) cp_async16(base + L::kVg * kLsmChunk + e, Vg + i, pol_last);
                }
            }
            if (flows && !init) cp_async16(base + L::kCf * kLsmChunk + e, cf + i, pol_last);
        }
    };

    // The first chunks' slab rows do not depend on the previous date: fetch them
    // before waiting for it; the cash flows and this date's coefficients after.
    // Chunk k of this block (blockIdx.x + k * gridDim.x) goes to stage k mod ST.
    // Commit groups: the first holds the rows of chunks 0 .. ST-2 and the cash flows
    // of chunk 0, group g (1 <= g <= ST-2) the cash flows of chunk g, and loop
    // iteration k commits chunk k + ST - 1 (possibly an empty group), so chunk k has
    // landed once at most ST - 2 groups are pending.
    constexpr int ST = lsm_stages<R>();
    int64_t chunk = blockIdx.x;
    for (int s = 0; s < ST - 1; ++s) {
        const int64_t c = chunk + static_cast<int64_t>(s) * gridDim.x;
        if (c < n_chunks) issue(c, s, true, false);
    }
    pdl_wait_preceding();
    // this date's coefficients, read by every thread from shared memory (broadcast);
    // the loop's first barrier orders these stores before any read
    __shared__ double cu[kMaxCoef];
    __shared__ float cuf[kMaxCoef];
    if (threadIdx.x < NB) {
        const double c = init ? 0.0 : coeffs[d_upd * kMaxCoef + threadIdx.x];
        cu[threadIdx.x] = c;
        cuf[threadIdx.x] = static_cast<float>(c);
    }
    for (int s = 0; s < ST - 1; ++s) {
        const int64_t c = chunk + static_cast<int64_t>(s) * gridDim.x;
        if (c < n_chunks) issue(c, s, false, true);
        cp_async_commit();
    }
    // With 4-byte rows every thread copies (issue) and later reads back exactly the
    // same four paths of each array (elements 4t .. 4t+3 of a chunk), so its own
    // cp.async.wait_group is all the ordering a chunk needs and a stage it refills
    // holds only data it has itself consumed: no block barrier per chunk.  With
    // 8-byte rows a thread reads slots that other threads copied.
    constexpr bool kOwnSlots = kPer16 == 4;
    static_assert(!kOwnSlots || kLsmChunk == 4 * kLsmBlock, "one 16-byte copy per thread and array");
    if constexpr (kOwnSlots) __syncthreads();  // this date's coefficient stores visible
    // FP32 6-term kernel: the coefficients in registers, as pairs for the paired FMAs
    float2 cc[kF32 ? 6 : 1];
    if constexpr (kF32) {
#pragma unroll
        for (int i = 0; i < 6; ++i) cc[i] = make_float2(cuf[i], cuf[i]);
    }
    for (int k = 0; chunk < n_chunks; ++k, chunk += gridDim.x) {
        cp_async_wait_pending<ST - 2>();  // this thread's copies of `chunk` have landed
        if constexpr (!kOwnSlots) __syncthreads();  // ... and every other thread's; all are done with chunk k - 1
        // refill the stage chunk k - 1 used, overlapping this chunk's arithmetic
        const int64_t ahead = chunk + static_cast<int64_t>(ST - 1) * gridDim.x;
        if (ahead < n_chunks) issue(ahead, (k + ST - 1) % ST, true, true);
        cp_async_commit();
        const R *base = stage + static_cast<size_t>(k % ST) * L::kArrays * kLsmChunk;
        // four consecutive paths per thread: 16-byte shared loads, no bank conflicts
        const int j0 = 4 * threadIdx.x;
        const int64_t i0 = chunk * kLsmChunk + j0;
        if constexpr (kF32) {
            if (i0 < a.N) {
                float S4[4], c4[4], v4[4];
                load4(base + L::kSu * kLsmChunk + j0, S4);
                if (!init) load4(base + L::kCf * kLsmChunk + j0, c4);
                load4(base + L::kVu * kLsmChunk + j0, v4);
                if (init) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) c4[q] = lsm_intrinsic<float>(a.right, S4[q], K);
                } else {
#pragma unroll
                    for (int h = 0; h < 4; h += 2) {
                        const float2 x = __ffma2_rn(make_float2(S4[h], S4[h + 1]), make_float2(inv_Kf, inv_Kf),
                                                    make_float2(-cxuf, -cxuf));
                        const float2 w = __fadd2_rn(make_float2(v4[h], v4[h + 1]), make_float2(-cvuf, -cvuf));
                        const float2 hold = continuation_f32x2(cc, x, w);
                        const float iv0 = lsm_intrinsic<float>(a.right, S4[h], K);
                        const float iv1 = lsm_intrinsic<float>(a.right, S4[h + 1], K);
                        c4[h] = (iv0 > 0.0f && iv0 > hold.x) ? iv0 : c4[h] * disc;
                        c4[h + 1] = (iv1 > 0.0f && iv1 > hold.y) ? iv1 : c4[h + 1] * disc;
                    }
                }
                store4(cf + i0, c4);  // i0 + 3 < ld: rows are padded to a multiple of 4
                if (gram) {
                    float Sg4[4], vg4[4], x[4], w[4], y[4], one[4];
                    load4(base + L::kSg * kLsmChunk + j0, Sg4);
                    load4(base + L::kVg * kLsmChunk + j0, vg4);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const bool itm = i0 + q < a.N && lsm_intrinsic<float>(a.right, Sg4[q], K) > 0.0f;
                        x[q] = itm ? fmaf(Sg4[q], inv_Kf, -cxgf) : 0.0f;
                        w[q] = itm ? vg4[q] - cvgf : 0.0f;
                        y[q] = itm ? c4[q] * disc : 0.0f;
                        one[q] = itm ? 1.0f : 0.0f;
                    }
                    accumulate_f32x2(acc2, make_float2(x[0], x[1]), make_float2(w[0], w[1]),
                                     make_float2(y[0], y[1]), make_float2(one[0], one[1]));
                    accumulate_f32x2(acc2, make_float2(x[2], x[3]), make_float2(w[2], w[3]),
                                     make_float2(y[2], y[3]), make_float2(one[2], one[3]));
                }
            }
            if ((k & (kF32Flush - 1)) == kF32Flush - 1) flush();
            continue;
        }
        if (i0 < a.N) {
            R S4[4], c4[4], v4[4] = {R(0), R(0), R(0), R(0)};
            load4(base + L::kSu * kLsmChunk + j0, S4);
            if (!init) load4(base + L::kCf * kLsmChunk + j0, c4);
            if (use_v) load4(base + L::kVu * kLsmChunk + j0, v4);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const R iv = lsm_intrinsic<R>(a.right, S4[q], K);
                if (init) {
                    c4[q] = iv;
                } else {
                    const R disc_c = c4[q] * disc;
                    R c = disc_c;
                    if (iv > R(0)) {
                        const double hold = continuation<R, BASIS>(cu, S4[q], v4[q], K, inv_K, cxu, cvu);
                        if (static_cast<double>(iv) > hold) c = iv;
                    }
                    c4[q] = c;
                }
            }
            store4(cf + i0, c4);  // i0 + 3 < ld: rows are padded to a multiple of 4
            if (gram) {
                R Sg4[4], vg4[4] = {R(0), R(0), R(0), R(0)};
                load4(base + L::kSg * kLsmChunk + j0, Sg4);
                if (use_v) load4(base + L::kVg * kLsmChunk + j0, vg4);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (i0 + q < a.N && lsm_intrinsic<R>(a.right, Sg4[q], K) > R(0))
                        accumulate<R, BASIS>(acc, Sg4[q], vg4[q], K, inv_K, cxg, cvg, c4[q] * disc);
                }
            }
        }
    }
    if (!gram) return;
    flush();
    // block reduction of the NACC sums
    __shared__ double s_red[kLsmBlock / 32][NACC];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NACC; ++j) {
        const double v = warp_sum(acc[j]);
        if (lane == 0) s_red[warp][j] = v;
    }
    __syncthreads();
    if (threadIdx.x < NACC) {
        double t = 0.0;
        for (int w = 0; w < kLsmBlock / 32; ++w) t += s_red[w][threadIdx.x];
        block_sums[static_cast<int64_t>(blockIdx.x) * NACC + threadIdx.x] = t;
        __threadfence();  // this block's sums are visible device-wide before it is counted
    }
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    // last block: fixed-order reduction of all block sums, then the FP64 solve
    __threadfence();
    __shared__ double s_part[kLsmBlock / 32][NACC];
    if (lane < NACC) {
        // warp w sums blocks w, w + 8, ...: eight independent loads in flight per
        // iteration (eight partial sums, folded in a fixed order)
        constexpr int kW = kLsmBlock / 32;
        const int G = static_cast<int>(gridDim.x);
        double part[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        int b = warp;
        for (; b + 7 * kW < G; b += 8 * kW) {
#pragma unroll
            for (int u = 0; u < 8; ++u) part[u] += __ldcg(block_sums + static_cast<int64_t>(b + u * kW) * NACC + lane);
        }
        for (; b < G; b += kW) part[0] += __ldcg(block_sums + static_cast<int64_t>(b) * NACC + lane);
        s_part[warp][lane] = ((part[0] + part[1]) + (part[2] + part[3])) + ((part[4] + part[5]) + (part[6] + part[7]));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot[NACC];
        for (int j = 0; j < NACC; ++j) {
            double t = 0.0;
            for (int w = 0; w < kLsmBlock / 32; ++w) t += s_part[w][j];
            tot[j] = t;
        }
        double sums[NSUM];
        expand_sums<BASIS>(tot, sums);
        double c[NB];
        const int f = (BASIS == QK_LSM_LAGUERRE3) ? solve_reference<NB>(sums, c) : solve_scaled<NB>(sums, c);
        for (int i = 0; i < kMaxCoef; ++i) coeffs[d_gram * kMaxCoef + i] = i < NB ? c[i] : 0.0;
        flags[d_gram] = f;
        *done = 0u;  // ready for the next date
    }
}

// Exercise decision at date 0 (or the maturity payoff when there is a single
// date), discount to t = 0, and per-block FP64 moments of the discounted cash
// flows (ForwardBackwardMC.hpp:245-248 then OptionPricer::accumulate_batch_payoffs).
template <class R, int BASIS>
__global__ void __launch_bounds__(kLsmBlock) lsm_final_kernel(LsmArgs a, const R *__restrict__ slab_S,
                                                             const R *__restrict__ slab_v, R *__restrict__ cf,
                                                             int init, const double *__restrict__ coeffs,
                                                             const double *__restrict__ centre,
                                                             Moments *__restrict__ block_moments) {
    constexpr int NB = BasisTraits<BASIS>::NB;
    const R K = static_cast<R>(a.K);
    const R disc = static_cast<R>(a.disc);
    const R eps_payoff = sizeof(R) == 4 ? R(1e-6) : R(1e-12);
    double cu[NB];
    for (int i = 0; i < NB; ++i) cu[i] = init ? 0.0 : coeffs[i];
    const double cx = centre[0], cv = centre[1];
    const double inv_K = 1.0 / a.K;
    const bool use_v = BASIS == QK_LSM_POLY_SV;
    __shared__ Moments s_warp[kLsmBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Moments acc{0.0, 0.0, 0.0, 0.0};
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    const int64_t n_iter = (a.N + stride - 1) / stride;
    for (int64_t it = 0; it < n_iter; ++it) {
        const int64_t i = it * stride + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
        const bool active = i < a.N;
        R val = R(0);
        if (active) {
            const R S = slab_S[i];
            const R iv = lsm_intrinsic<R>(a.right, S, K);
            R c;
            if (init) {
                c = iv;
            } else {
                c = cf[i];
                const R disc_c = c * disc;
                if (iv > R(0)) {
                    const R v = use_v ? slab_v[i] : R(0);
                    const double hold = continuation<R, BASIS>(cu, S, v, K, inv_K, cx, cv);
                    c = (static_cast<double>(iv) > hold) ? iv : disc_c;
                } else {
                    c = disc_c;
                }
            }
            val = c * disc;  // t_1 -> 0 (LSMAmerican.hpp:401-405)
            cf[i] = val;
        }
        const Moments wm = warp_moments(static_cast<double>(val), active, val > eps_payoff);
        acc = chan_merge(acc, wm);
    }
    if (lane == 0) s_warp[warp] = acc;
    __syncthreads();
    if (warp == 0) {
        Moments m = lane < kLsmBlock / 32 ? s_warp[lane] : Moments{0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) m = chan_merge(m, shfl_down_moments(m, off));
        if (lane == 0) block_moments[blockIdx.x] = m;
    }
}

// ---------------------------------------------------------------- one date on caller arrays
// The pieces of one backward step as separate operations on n paths given by the
// caller (LSMEngine's statics, LSMAmerican.hpp:252-419): the cash flows start as the
// payoff; the in-the-money regression sums of a date with Y = cf * disc, reduced per
// block and then in block order, and the FP64 solve; the exercise decision.  Same
// basis, accumulation, continuation and solve code as the sweep.
template <class R, int BASIS>
__global__ void __launch_bounds__(kLsmBlock) lsm_date_sums_kernel(int right, int64_t n, const double *__restrict__ S,
                                                                 const double *__restrict__ v,
                                                                 const double *__restrict__ cf, double K, double disc,
                                                                 double cx, double cv, double *__restrict__ block_sums) {
    constexpr int NACC = AccTraits<BASIS>::N;
    __shared__ double s_red[kLsmBlock / 32][NACC];
    double acc[NACC];
#pragma unroll
    for (int j = 0; j < NACC; ++j) acc[j] = 0.0;
    const R Kr = static_cast<R>(K), dr = static_cast<R>(disc);
    const double inv_K = 1.0 / K;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const R s = static_cast<R>(S[i]);
        if (lsm_intrinsic<R>(right, s, Kr) > R(0))
            accumulate<R, BASIS>(acc, s, v ? static_cast<R>(v[i]) : R(0), Kr, inv_K, cx, cv, static_cast<R>(cf[i]) * dr);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NACC; ++j) {
        const double s = warp_sum(acc[j]);
        if (lane == 0) s_red[warp][j] = s;
    }
    __syncthreads();
    if (threadIdx.x < NACC) {
        double s = 0.0;
        for (int w = 0; w < kLsmBlock / 32; ++w) s += s_red[w][threadIdx.x];
        block_sums[static_cast<int64_t>(blockIdx.x) * NACC + threadIdx.x] = s;
    }
}

// One thread: block sums in block order (or, with nblocks = 0, `sums` given directly in
// the solver's layout), then the FP64 solve.  method: 0 Cholesky, 1 pivoted QR, 2 mean.
template <int BASIS>
__global__ void lsm_date_solve_kernel(int nblocks, const double *__restrict__ in, double *__restrict__ coeffs,
                                      int *__restrict__ method) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    constexpr int NB = BasisTraits<BASIS>::NB;
    constexpr int NSUM = Sums<NB>::NSUM;
    constexpr int NACC = AccTraits<BASIS>::N;
    double sums[NSUM];
    if (nblocks > 0) {
        double tot[NACC];
        for (int j = 0; j < NACC; ++j) {
            double s = 0.0;
            for (int b = 0; b < nblocks; ++b) s += in[static_cast<int64_t>(b) * NACC + j];
            tot[j] = s;
        }
        expand_sums<BASIS>(tot, sums);
    } else {
        for (int j = 0; j < NSUM; ++j) sums[j] = in[j];
    }
    double c[NB];
    *method = BASIS == QK_LSM_LAGUERRE3 ? solve_reference<NB>(sums, c) : solve_scaled<NB>(sums, c);
    for (int i = 0; i < NB; ++i) coeffs[i] = c[i];
}

// init: cf = intrinsic(S); otherwise the exercise decision with `coeffs`.
template <class R, int BASIS>
__global__ void __launch_bounds__(kLsmBlock) lsm_date_update_kernel(int right, int64_t n, const double *__restrict__ S,
                                                                   const double *__restrict__ v, double *__restrict__ cf,
                                                                   double K, double disc, double cx, double cv,
                                                                   const double *__restrict__ coeffs, int init) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const R Kr = static_cast<R>(K);
    const R s = static_cast<R>(S[i]);
    const R iv = lsm_intrinsic<R>(right, s, Kr);
    if (init) {
        cf[i] = static_cast<double>(iv);
        return;
    }
    double c[kMaxCoef];
    for (int k = 0; k < BasisTraits<BASIS>::NB; ++k) c[k] = coeffs[k];
    R out = static_cast<R>(cf[i]) * static_cast<R>(disc);
    if (iv > R(0) &&
        static_cast<double>(iv) > continuation<R, BASIS>(c, s, v ? static_cast<R>(v[i]) : R(0), Kr, 1.0 / K, cx, cv))
        out = iv;
    cf[i] = static_cast<double>(out);
}

template <class R, int BASIS>
static cudaError_t preload_lsm_kernels_of() {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, lsm_sweep_kernel<R, BASIS>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, lsm_final_kernel<R, BASIS>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, lsm_date_sums_kernel<R, BASIS>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, lsm_date_update_kernel<R, BASIS>);
    return e;
}

cudaError_t preload_lsm_kernels() {
    cudaFuncAttributes fa;
    cudaError_t e = preload_lsm_kernels_of<float, QK_LSM_LAGUERRE3>();
    if (e == cudaSuccess) e = preload_lsm_kernels_of<float, QK_LSM_POLY_SV>();
    if (e == cudaSuccess) e = preload_lsm_kernels_of<double, QK_LSM_LAGUERRE3>();
    if (e == cudaSuccess) e = preload_lsm_kernels_of<double, QK_LSM_POLY_SV>();
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, lsm_date_solve_kernel<QK_LSM_LAGUERRE3>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, lsm_date_solve_kernel<QK_LSM_POLY_SV>);
    return e;
}

// ---------------------------------------------------------------- host side
namespace {

#define QK_CUDA_LSM(call)                                                                            \
    do {                                                                                             \
        const cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                       \
            return fail(e_ == cudaErrorMemoryAllocation ? QK_ERR_OUT_OF_MEMORY : QK_ERR_CUDA,        \
                        std::string("LSM: ") + #call + ": " + cudaGetErrorString(e_));               \
    } while (0)

template <class R, int BASIS>
cudaError_t enqueue_backward(cudaStream_t s, int grid, int sm_count, const LsmArgs &a, const R *S, const R *V, R *cf,
                             double *coeffs, int *flags, const double *centre, double *block_sums,
                             unsigned int *done, Moments *block_moments, int64_t *launches) {
    const int D = a.n_dates;
    if (D == 1) {
        lsm_final_kernel<R, BASIS><<<grid, kLsmBlock, 0, s>>>(a, S, V, cf, 1, coeffs, centre, block_moments);
        ++*launches;
        return cudaGetLastError();
    }
    // sweep grid: every resident block slot of the GPU (at most 4 per SM; the
    // block-sum arena holds 4 * sm_count * 32 doubles)
    const size_t smem = lsm_sweep_smem<R, BASIS>();
    // the shared-memory attribute (context-wide) and the occupancy, once per device (a
    // serving lane enqueues many small jobs; each query is a driver call)
    static std::atomic<int> per_sm_cache[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int per_sm = dev >= 0 && dev < 64 ? per_sm_cache[dev].load(std::memory_order_relaxed) : 0;
    if (per_sm == 0) {
        e = cudaFuncSetAttribute(lsm_sweep_kernel<R, BASIS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lsm_sweep_kernel<R, BASIS>, kLsmBlock, smem);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64 && per_sm > 0) per_sm_cache[dev].store(per_sm, std::memory_order_relaxed);
    }
    // and no more blocks than chunks: a small job's empty blocks would still launch,
    // check in on the counter and have their (zero) sums folded by the last block
    const int64_t n_chunks = (a.ld + kLsmChunk - 1) / kLsmChunk;
    const int sgrid = static_cast<int>(
        std::min<int64_t>(static_cast<int64_t>(sm_count) * std::min(std::max(per_sm, 1), 4), std::max<int64_t>(n_chunks, 1)));
    e = cudaMemsetAsync(done, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    lsm_sweep_kernel<R, BASIS><<<sgrid, kLsmBlock, smem, s>>>(a, S, V, cf, D - 1, 1, D - 2, coeffs, centre,
                                                              block_sums, done, flags);
    ++*launches;
    // later dates: programmatic dependent launches (each may start while the
    // previous date's last block solves; it waits in-kernel before reading)
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(sgrid));
    cfg.blockDim = dim3(kLsmBlock);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    for (int d = D - 2; d >= 1; --d) {
        e = cudaLaunchKernelEx(&cfg, lsm_sweep_kernel<R, BASIS>, a, S, V, cf, d, 0, d - 1, coeffs, centre, block_sums,
                               done, flags);
        if (e != cudaSuccess) return e;
        ++*launches;
    }
    lsm_final_kernel<R, BASIS><<<grid, kLsmBlock, 0, s>>>(a, S, V, cf, 0, coeffs, centre, block_moments);
    ++*launches;
    return cudaGetLastError();
}

}  // namespace

qk_status lsm_events_ensure(qk_handle *h, size_t n) {
    // grown geometrically: creating events takes the driver's lock, which other lanes' calls wait on
    const size_t want = h->lsm_events.size() >= n ? n : std::max<size_t>({n, 2 * h->lsm_events.size(), 48});
    while (h->lsm_events.size() < want) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return fail(QK_ERR_CUDA, "LSM: cudaEventCreate failed");
        h->lsm_events.push_back(e);
    }
    h->lsm_jobs = n / 3;
    return QK_OK;
}

void lsm_timing(qk_handle *h, double *paths_ms, double *sweep_ms) {
    *paths_ms = *sweep_ms = 0.0;
    for (size_t k = 0; k < h->lsm_jobs; ++k) {
        float a = 0.f, b = 0.f;
        if (cudaEventElapsedTime(&a, h->lsm_events[3 * k], h->lsm_events[3 * k + 1]) == cudaSuccess) *paths_ms += a;
        if (cudaEventElapsedTime(&b, h->lsm_events[3 * k + 1], h->lsm_events[3 * k + 2]) == cudaSuccess) *sweep_ms += b;
    }
}

void lsm_release(qk_handle *h) {
    for (cudaEvent_t e : h->lsm_events) cudaEventDestroy(e);
    h->lsm_events.clear();
    h->lsm_jobs = 0;
    for (int l = 0; l < kLsmLanes; ++l) {
        LsmArena &L = h->lsm[l];
        L.slab_S.release();
        L.slab_v.release();
        L.cashflow.release();
        L.block_sums.release();
        L.coeffs.release();
        L.status.release();
        if (h->lsm_stream[l]) cudaStreamDestroy(h->lsm_stream[l]);
        if (h->lsm_join[l]) cudaEventDestroy(h->lsm_join[l]);
        h->lsm_stream[l] = nullptr;
        h->lsm_join[l] = nullptr;
    }
    if (h->lsm_fork) cudaEventDestroy(h->lsm_fork);
    h->lsm_fork = nullptr;
    h->lsm_task.release();
    h->lsm_centre.release();
    h->h_lsm.release();
    h->d_lsm_moments.release();
}

namespace {

// Streams and fork/join events of the LSM lanes (created on first use).
qk_status lsm_lanes_ensure(qk_handle *h, int lanes) {
    if (!h->lsm_fork && cudaEventCreateWithFlags(&h->lsm_fork, cudaEventDisableTiming) != cudaSuccess)
        return fail(QK_ERR_CUDA, "LSM: cudaEventCreate failed");
    for (int l = 0; l < lanes; ++l) {
        if (!h->lsm_stream[l] && cudaStreamCreateWithFlags(&h->lsm_stream[l], cudaStreamNonBlocking) != cudaSuccess)
            return fail(QK_ERR_CUDA, "LSM: cudaStreamCreate failed");
        if (!h->lsm_join[l] && cudaEventCreateWithFlags(&h->lsm_join[l], cudaEventDisableTiming) != cudaSuccess)
            return fail(QK_ERR_CUDA, "LSM: cudaEventCreate failed");
    }
    return QK_OK;
}

}  // namespace

qk_status run_lsm_contracts(qk_handle *h, Plan &plan, bool plain, std::vector<Moments> &moments) {
    (void)moments;
    plan.lsm_tasks.clear();
    // task list
    struct Job {
        qk_contract b;
        int contract, role;
    };
    std::vector<Job> jobs;
    for (int i : plan.american)
        for (int role : roles_for(plan.g_of(i), plan.norm[i].T)) {
            qk_contract b = bumped(plan.norm[i], plan.g_of(i), role);
            if (plain) b.precision = QK_FP64;
            jobs.push_back({b, i, role});
        }
    const int grid = h->sm_count * 2;
    const size_t nj = jobs.size();
    qk_status st;
    // per-job working-set sizes
    auto dates_of = [](const qk_contract &b) { return b.lsm_dates > 0 ? b.lsm_dates : b.n_steps; };
    auto ld_of = [](const qk_contract &b) { return (b.n_paths + 3) / 4 * 4; };
    auto esz_of = [](const qk_contract &b) { return static_cast<size_t>(b.precision == QK_FP32 ? 4 : 8); };
    auto slab_of = [&](const Job &j) { return static_cast<size_t>(dates_of(j.b)) * ld_of(j.b) * esz_of(j.b); };
    // Jobs go to the lanes longest first, each to the least loaded lane (by path-steps);
    // a lane runs its jobs in order on its own stream and working set, sized for the
    // largest of them, so the lanes together hold at most the sum over the jobs.
    const int lanes = static_cast<int>(std::min<size_t>(kLsmLanes, std::max<size_t>(nj, 1)));
    std::vector<size_t> order(nj);
    for (size_t k = 0; k < nj; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
        return static_cast<double>(jobs[x].b.n_paths) * jobs[x].b.n_steps >
               static_cast<double>(jobs[y].b.n_paths) * jobs[y].b.n_steps;
    });
    std::vector<int> lane_of(nj, 0);
    std::vector<double> load(lanes, 0.0);
    std::vector<size_t> lane_slab(lanes, 0), lane_cf(lanes, 0);
    std::vector<int> lane_dates(lanes, 1);
    std::vector<bool> lane_v(lanes, false);
    for (size_t k : order) {
        const int l = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
        lane_of[k] = l;
        load[l] += static_cast<double>(jobs[k].b.n_paths) * jobs[k].b.n_steps;
        lane_slab[l] = std::max(lane_slab[l], slab_of(jobs[k]));
        lane_cf[l] = std::max(lane_cf[l], static_cast<size_t>(ld_of(jobs[k].b)) * esz_of(jobs[k].b));
        lane_dates[l] = std::max(lane_dates[l], dates_of(jobs[k].b));
        lane_v[l] = lane_v[l] || jobs[k].b.lsm_basis == QK_LSM_POLY_SV;
    }
    if ((st = lsm_lanes_ensure(h, lanes)) != QK_OK) return st;
    for (int l = 0; l < lanes; ++l) {
        LsmArena &L = h->lsm[l];
        if ((st = L.slab_S.ensure(lane_slab[l])) != QK_OK) return st;
        if (lane_v[l] && (st = L.slab_v.ensure(lane_slab[l])) != QK_OK) return st;
        if ((st = L.cashflow.ensure(lane_cf[l])) != QK_OK) return st;
        if ((st = L.block_sums.ensure(static_cast<size_t>(h->sm_count) * 4 * 32 * sizeof(double))) != QK_OK) return st;
        if ((st = L.coeffs.ensure(static_cast<size_t>(lane_dates[l]) * kMaxCoef * sizeof(double) + 64)) != QK_OK)
            return st;
        if ((st = L.status.ensure(static_cast<size_t>(lane_dates[l]) * sizeof(int) + 256)) != QK_OK) return st;
    }
    if ((st = lsm_events_ensure(h, 3 * nj)) != QK_OK) return st;
    if ((st = h->lsm_task.ensure(nj * sizeof(TaskDev))) != QK_OK) return st;
    if ((st = h->d_lsm_moments.ensure(nj * grid * sizeof(Moments))) != QK_OK) return st;
    if ((st = h->h_lsm.ensure(nj * grid * sizeof(Moments))) != QK_OK) return st;
    // descriptors and per-date centring constants of all jobs (one upload, blocking)
    std::vector<TaskDev> tasks(nj);
    std::vector<double> centres;
    std::vector<size_t> centre_off(nj);
    for (size_t k = 0; k < nj; ++k) {
        const qk_contract &b = jobs[k].b;
        tasks[k] = make_task(b, 1);
        const int D = dates_of(b);
        const int stride = b.n_steps / D;
        const double dt = b.T / b.n_steps;
        const double K = b.payoffs[0].strike;
        centre_off[k] = centres.size();
        for (int d = 0; d < D; ++d) {
            const double t = (d + 1) * stride * dt;
            // forward level of S/K and the mean of v_t: shifts that centre the regression basis
            centres.push_back(b.S0 / K * std::exp((b.r - b.q) * t));
            centres.push_back(b.theta + (b.v0 - b.theta) * std::exp(-b.kappa * t));
        }
    }
    if ((st = h->lsm_centre.ensure(std::max<size_t>(centres.size(), 1) * sizeof(double))) != QK_OK) return st;
    const double *d_centre = static_cast<const double *>(h->lsm_centre.ptr);
    QK_CUDA_LSM(cudaMemcpy(h->lsm_task.ptr, tasks.data(), nj * sizeof(TaskDev), cudaMemcpyHostToDevice));
    QK_CUDA_LSM(cudaMemcpy(h->lsm_centre.ptr, centres.data(), centres.size() * sizeof(double),
                           cudaMemcpyHostToDevice));
    // fork: the lanes start after the work already queued on the handle's stream
    QK_CUDA_LSM(cudaEventRecord(h->lsm_fork, h->stream));
    for (int l = 0; l < lanes; ++l) QK_CUDA_LSM(cudaStreamWaitEvent(h->lsm_stream[l], h->lsm_fork, 0));
    for (size_t k = 0; k < nj; ++k) {
        const qk_contract &b = jobs[k].b;
        const int l = lane_of[k];
        LsmArena &L = h->lsm[l];
        cudaStream_t s = h->lsm_stream[l];
        const int D = dates_of(b);
        const int stride = b.n_steps / D;
        const int64_t ld = ld_of(b);
        const int prec = b.precision;
        const bool use_v = b.lsm_basis == QK_LSM_POLY_SV;
        // forward: exercise-date slabs
        QK_CUDA_LSM(cudaEventRecord(h->lsm_events[3 * k], s));
        // FP32: two paths per thread, stepped as pairs
        QK_CUDA_LSM(launch_slab_paths(prec, b.model, b.scheme, b.seed, s,
                                      static_cast<const TaskDev *>(h->lsm_task.ptr) + k, 0, b.n_paths, stride,
                                      L.slab_S.ptr, use_v ? L.slab_v.ptr : nullptr, ld, prec == QK_FP32 ? 2 : 1));
        h->lsm_launches++;
        QK_CUDA_LSM(cudaEventRecord(h->lsm_events[3 * k + 1], s));
        LsmArgs a;
        a.N = b.n_paths;
        a.ld = ld;
        a.right = b.payoffs[0].right;
        a.n_dates = D;
        a.K = b.payoffs[0].strike;
        a.disc = std::exp(-b.r * stride * (b.T / b.n_steps));
        Moments *bm = static_cast<Moments *>(h->d_lsm_moments.ptr) + k * grid;
        const double *cen = d_centre + centre_off[k];
        double *d_coeffs = static_cast<double *>(L.coeffs.ptr);
        double *bs = static_cast<double *>(L.block_sums.ptr);
        int *fl = static_cast<int *>(L.status.ptr);
        unsigned int *done = reinterpret_cast<unsigned int *>(
            static_cast<char *>(L.status.ptr) + ((static_cast<size_t>(lane_dates[l]) * sizeof(int) + 127) / 128) * 128);
        cudaError_t e;
        if (prec == QK_FP32) {
            if (use_v)
                e = enqueue_backward<float, QK_LSM_POLY_SV>(s, grid, h->sm_count, a,
                                                           static_cast<const float *>(L.slab_S.ptr),
                                                           static_cast<const float *>(L.slab_v.ptr),
                                                           static_cast<float *>(L.cashflow.ptr), d_coeffs, fl, cen, bs,
                                                           done, bm, &h->lsm_launches);
            else
                e = enqueue_backward<float, QK_LSM_LAGUERRE3>(s, grid, h->sm_count, a,
                                                             static_cast<const float *>(L.slab_S.ptr), nullptr,
                                                             static_cast<float *>(L.cashflow.ptr), d_coeffs, fl, cen,
                                                             bs, done, bm, &h->lsm_launches);
        } else {
            if (use_v)
                e = enqueue_backward<double, QK_LSM_POLY_SV>(s, grid, h->sm_count, a,
                                                            static_cast<const double *>(L.slab_S.ptr),
                                                            static_cast<const double *>(L.slab_v.ptr),
                                                            static_cast<double *>(L.cashflow.ptr), d_coeffs, fl, cen,
                                                            bs, done, bm, &h->lsm_launches);
            else
                e = enqueue_backward<double, QK_LSM_LAGUERRE3>(s, grid, h->sm_count, a,
                                                              static_cast<const double *>(L.slab_S.ptr), nullptr,
                                                              static_cast<double *>(L.cashflow.ptr), d_coeffs, fl, cen,
                                                              bs, done, bm, &h->lsm_launches);
        }
        if (e != cudaSuccess) return fail(QK_ERR_CUDA, std::string("LSM launch: ") + cudaGetErrorString(e));
        QK_CUDA_LSM(cudaEventRecord(h->lsm_events[3 * k + 2], s));
        LsmTaskInfo info;
        info.contract = jobs[k].contract;
        info.role = jobs[k].role;
        info.grid = grid;
        info.moments_base = static_cast<int64_t>(k) * grid;
        info.n_paths = b.n_paths;
        // immediate exercise value today at S0 (LSMAmerican.hpp:410-418)
        const double K = b.payoffs[0].strike;
        info.intrinsic0 = b.payoffs[0].right == QK_CALL ? std::max(b.S0 - K, 0.0) : std::max(K - b.S0, 0.0);
        info.eps = prec == QK_FP32 ? 1e-6 : 1e-12;
        plan.lsm_tasks.push_back(info);
        plan.lsm_path_steps += static_cast<double>(b.n_paths) * b.n_steps;
    }
    // join: the handle's stream continues once every lane is done
    for (int l = 0; l < lanes; ++l) {
        QK_CUDA_LSM(cudaEventRecord(h->lsm_join[l], h->lsm_stream[l]));
        QK_CUDA_LSM(cudaStreamWaitEvent(h->stream, h->lsm_join[l], 0));
    }
    QK_CUDA_LSM(cudaMemcpyAsync(h->h_lsm.ptr, h->d_lsm_moments.ptr, nj * grid * sizeof(Moments),
                                cudaMemcpyDeviceToHost, h->stream));
    return QK_OK;
}

void assemble_lsm_results(qk_handle *h, const Plan &plan, const std::vector<Moments> &, qk_result *out) {
    const Moments *hm = static_cast<const Moments *>(h->h_lsm.ptr);
    // per task merged moments after the day-zero decision
    std::vector<double> price(plan.lsm_tasks.size()), se(plan.lsm_tasks.size()), itm(plan.lsm_tasks.size());
    for (size_t k = 0; k < plan.lsm_tasks.size(); ++k) {
        const LsmTaskInfo &info = plan.lsm_tasks[k];
        Moments m{0.0, 0.0, 0.0, 0.0};
        for (int b = 0; b < info.grid; ++b) {
            const Moments &o = hm[info.moments_base + b];
            const double n = m.n + o.n;
            if (o.n <= 0.0) continue;
            if (m.n <= 0.0) {
                m = o;
                continue;
            }
            const double d = o.mean - m.mean;
            m.mean += d * (o.n / n);
            m.m2 += o.m2 + d * d * (m.n * o.n / n);
            m.itm += o.itm;
            m.n = n;
        }
        // LSMEngine::apply_final_discount: exercise today if intrinsic(S0) beats the mean
        if (info.intrinsic0 > m.mean) {
            m.mean = info.intrinsic0;
            m.m2 = 0.0;
            m.itm = info.intrinsic0 > info.eps ? m.n : 0.0;
        }
        const double scale = plan.scale[info.contract];
        const double N = m.n;
        price[k] = m.mean * scale;
        se[k] = N > 1.0 ? std::sqrt(m.m2 / (N - 1.0) / N) * scale : 0.0;
        itm[k] = N > 0.0 ? m.itm / N : 0.0;
    }
    for (int i : plan.american) {
        const qk_greeks *g = plan.g_of(i);
        qk_result &r = out[i];
        std::memset(&r, 0, sizeof(r));
        const qk_contract &n = plan.norm[i];
        r.status = QK_OK;
        r.n_payoffs = 1;
        r.n_paths = n.n_paths;
        auto find = [&](int role) -> int {
            for (size_t k = 0; k < plan.lsm_tasks.size(); ++k)
                if (plan.lsm_tasks[k].contract == i && plan.lsm_tasks[k].role == role) return static_cast<int>(k);
            return -1;
        };
        auto p_of = [&](int role) {
            const int k = find(role);
            return k >= 0 ? price[k] : 0.0;
        };
        for (size_t k = 0; k < plan.lsm_tasks.size(); ++k)
            if (plan.lsm_tasks[k].contract == i)
                r.path_steps += static_cast<double>(plan.lsm_tasks[k].n_paths) * n.n_steps;
        const int k0 = find(0);
        qk_payoff_result &pr = r.p[0];
        pr.price = price[k0];
        pr.std_error = se[k0];
        pr.prob_itm = itm[k0];
        if (!g) continue;
        const double p0 = pr.price;
        const double h_S_real = (n.normalize ? plan.scale[i] : n.S0) * g->bump_S_rel;
        const double h_vol = g->vega_mode == 1 ? n.v0 * g->bump_vol : g->bump_vol;
        if (g->mask & QK_GREEK_DELTA_GAMMA) {
            const double pu = p_of(1), pd = p_of(2);
            pr.delta = (pu - pd) / (2.0 * h_S_real);
            pr.gamma = (pu - 2.0 * p0 + pd) / (h_S_real * h_S_real);
        }
        if (g->mask & QK_GREEK_VEGA_VOMMA) {
            const double pu = p_of(3), pd = p_of(4);
            pr.vega = (pu - pd) / (2.0 * h_vol);
            pr.vomma = (pu - 2.0 * p0 + pd) / (h_vol * h_vol);
        }
        if (g->mask & QK_GREEK_RHO) pr.rho = (p_of(5) - p_of(6)) / (2.0 * g->bump_r_abs);
        if (g->mask & QK_GREEK_THETA) pr.theta = n.T > g->bump_T_abs ? (p_of(7) - p0) / g->bump_T_abs : 0.0;
        if (g->mask & QK_GREEK_VANNA)
            pr.vanna = (p_of(8) - p_of(9) - p_of(10) + p_of(11)) / (4.0 * h_S_real * h_vol);
    }
}

}  // namespace qk

// ============================================================================
// extern "C": one exercise date on caller arrays (LSMEngine's statics)
// ============================================================================
namespace {

template <class R, int BASIS>
cudaError_t lsm_date_run(int op, int right, int64_t n, const double *S, const double *v, double *cf, double K,
                         double disc, double cx, double cv, double *coeffs, int *method) {
    using namespace qk;
    constexpr int NACC = AccTraits<BASIS>::N;
    constexpr int NB = BasisTraits<BASIS>::NB;
    const int threads = kLsmBlock;
    const int blocks_all = static_cast<int>((n + threads - 1) / threads);
    const int sum_blocks = std::min(blocks_all, 512);
    const size_t bytes = (2 * static_cast<size_t>(n) + (v ? n : 0)) * sizeof(double) +
                         (static_cast<size_t>(sum_blocks) * NACC + kMaxCoef + 2) * sizeof(double);
    void *d = nullptr;
    cudaError_t e = cudaMalloc(&d, bytes);
    if (e != cudaSuccess) return e;
    double *dS = static_cast<double *>(d);
    double *dcf = dS + n;
    double *dv = v ? dcf + n : nullptr;
    double *dsums = (v ? dv : dcf) + n;
    double *dco = dsums + static_cast<size_t>(sum_blocks) * NACC;
    int *dm = reinterpret_cast<int *>(dco + kMaxCoef);
    e = cudaMemcpy(dS, S, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && op != 0) e = cudaMemcpy(dcf, cf, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && v) e = cudaMemcpy(dv, v, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && op == 1) {
        lsm_date_sums_kernel<R, BASIS><<<sum_blocks, threads>>>(right, n, dS, dv, dcf, K, disc, cx, cv, dsums);
        lsm_date_solve_kernel<BASIS><<<1, 1>>>(sum_blocks, dsums, dco, dm);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(coeffs, dco, NB * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && method) e = cudaMemcpy(method, dm, sizeof(int), cudaMemcpyDeviceToHost);
    } else if (e == cudaSuccess) {
        if (op == 2) e = cudaMemcpy(dco, coeffs, NB * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            lsm_date_update_kernel<R, BASIS><<<blocks_all, threads>>>(right, n, dS, dv, dcf, K, disc, cx, cv, dco,
                                                                    op == 0 ? 1 : 0);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpy(cf, dcf, n * sizeof(double), cudaMemcpyDeviceToHost);
    }
    cudaFree(d);
    return e;
}

}  // namespace

extern "C" qk_status qk_lsm_date(int32_t op, int32_t precision, int32_t basis, int32_t right, int64_t n,
                                 const double *S, const double *v, double *cf, double K, double disc, double cx,
                                 double cv, double *coeffs, int32_t *method) {
    using namespace qk;
    if (op < 0 || op > 2 || n < 1 || !S || !cf || (op != 0 && !coeffs) || !(K > 0.0))
        return fail(QK_ERR_INVALID_ARG, "qk_lsm_date: invalid arguments");
    if (basis != QK_LSM_LAGUERRE3 && basis != QK_LSM_POLY_SV) return fail(QK_ERR_INVALID_ARG, "qk_lsm_date: basis");
    if (right != QK_CALL && right != QK_PUT) return fail(QK_ERR_INVALID_ARG, "qk_lsm_date: right");
    if (basis == QK_LSM_POLY_SV && !v) return fail(QK_ERR_INVALID_ARG, "qk_lsm_date: the {1,S,S^2,S^3,v,Sv} basis needs v");
    if (basis == QK_LSM_LAGUERRE3) v = nullptr;
    int m = 0;
    cudaError_t e;
    if (precision == QK_FP32)
        e = basis == QK_LSM_POLY_SV ? lsm_date_run<float, QK_LSM_POLY_SV>(op, right, n, S, v, cf, K, disc, cx, cv, coeffs, &m)
                                    : lsm_date_run<float, QK_LSM_LAGUERRE3>(op, right, n, S, v, cf, K, disc, cx, cv, coeffs, &m);
    else
        e = basis == QK_LSM_POLY_SV ? lsm_date_run<double, QK_LSM_POLY_SV>(op, right, n, S, v, cf, K, disc, cx, cv, coeffs, &m)
                                    : lsm_date_run<double, QK_LSM_LAGUERRE3>(op, right, n, S, v, cf, K, disc, cx, cv, coeffs, &m);
    if (e != cudaSuccess) return fail(QK_ERR_CUDA, std::string("qk_lsm_date: ") + cudaGetErrorString(e));
    if (method) *method = m;
    return QK_OK;
}

extern "C" qk_status qk_lsm_solve(int32_t basis, const double *sums, double *coeffs, int32_t *method) {
    using namespace qk;
    if (!sums || !coeffs) return fail(QK_ERR_INVALID_ARG, "qk_lsm_solve: NULL argument");
    if (basis != QK_LSM_LAGUERRE3 && basis != QK_LSM_POLY_SV) return fail(QK_ERR_INVALID_ARG, "qk_lsm_solve: basis");
    const int nsum = basis == QK_LSM_POLY_SV ? Sums<6>::NSUM : Sums<4>::NSUM;
    const int nb = basis == QK_LSM_POLY_SV ? 6 : 4;
    void *d = nullptr;
    cudaError_t e = cudaMalloc(&d, (nsum + kMaxCoef + 2) * sizeof(double));
    if (e != cudaSuccess) return fail(QK_ERR_CUDA, std::string("qk_lsm_solve: ") + cudaGetErrorString(e));
    double *ds = static_cast<double *>(d);
    double *dc = ds + nsum;
    int *dm = reinterpret_cast<int *>(dc + kMaxCoef);
    int m = 0;
    e = cudaMemcpy(ds, sums, nsum * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        if (basis == QK_LSM_POLY_SV) lsm_date_solve_kernel<QK_LSM_POLY_SV><<<1, 1>>>(0, ds, dc, dm);
        else lsm_date_solve_kernel<QK_LSM_LAGUERRE3><<<1, 1>>>(0, ds, dc, dm);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(coeffs, dc, nb * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&m, dm, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(QK_ERR_CUDA, std::string("qk_lsm_solve: ") + cudaGetErrorString(e));
    if (method) *method = m;
    return QK_OK;
}
