// Path-generation kernels (sm_100a): the fused path + payoff pricing kernel
// (persistent, fed by a device queue of (task, path-block) tiles), the per-task
// FP64 merge, the exercise-date slab writer used by Longstaff-Schwartz and by
// the path dump, and the fed-draw parity trace.
#include <cuda_runtime.h>

#include "qk_device.cuh"
#include "qk_kernels.h"

namespace qk {

// ----------------------------------------------------------------------------
// One path of one task.  Mirrors MarkovianIntegrationKernel::operator()
// (include/core/schemes/markovian/MSolver.hpp:98-130): start at (S0, v0), step
// n_steps times, track the running average / max / min after every step.
// SINK is called after each step with (step index, S, v).
// ----------------------------------------------------------------------------
template <class R>
struct PathState {
    R S, v;
    double ssum;  // running sum of S for the Asian average, in double (Payoff.hpp:87, 110)
    R smax, smin;
};

struct NoSink {
    template <class R>
    __device__ __forceinline__ void operator()(int, R, R) const {}
};

template <class R>
struct SlabSink {
    R *slab_S;
    R *slab_v;
    int64_t ld;     // leading dimension (paths per slab row)
    int64_t pos;    // slab index of this path's next stored date: row * ld + column
    int stride;     // steps between stored dates
    int left;       // steps until the next stored date
    // Called once per step, in order: every stride-th step is stored.
    __device__ __forceinline__ void operator()(int, R S, R v) {
        if (--left == 0) {
            left = stride;
            slab_S[pos] = S;
            if (slab_v) slab_v[pos] = v;
            pos += ld;
        }
    }
};

// Two paths per thread: stores S (and v) of paths a and b (b only if it exists).
struct NoSink2 {
    template <class R>
    __device__ __forceinline__ void operator()(int, R, R, R, R) const {}
};

template <class R>
struct SlabSink2 {
    R *slab_S;
    R *slab_v;
    int64_t ld;
    int64_t pos;   // slab index of path a's next stored date; path b is the next column
    int stride;
    int left;
    bool has_b;
    __device__ __forceinline__ void operator()(int, R Sa, R va, R Sb, R vb) {
        if (--left == 0) {
            left = stride;
            slab_S[pos] = Sa;
            if (has_b) slab_S[pos + 1] = Sb;
            if (slab_v) {
                slab_v[pos] = va;
                if (has_b) slab_v[pos + 1] = vb;
            }
            pos += ld;
        }
    }
};

// Steps are taken in chunks of kSumChunk; the Asian running sum is accumulated in
// the working precision inside a chunk and folded into the FP64 sum after it.
constexpr int kSumChunk = 16;

template <class R>
__device__ __forceinline__ void track(PathState<R> &st, R &blk) {
    blk += st.S;
    st.smax = rmax(st.smax, st.S);
    st.smin = rmin(st.smin, st.S);
}

// Philox with round keys read from the kernel's parameter bank (all tasks of the
// launch share the seed) or computed per round from the task's key.
struct ParamKeys {
    const PhiloxRoundKeys &rk;
    __device__ __forceinline__ U4 operator()(U4 c) const { return philox4x32_10(c, rk); }
};
struct RegKeys {
    uint32_t k0, k1;
    __device__ __forceinline__ U4 operator()(U4 c) const { return philox4x32_10(c, k0, k1); }
};

// The step's first Poisson uniform decides whether a jump happened (Knuth's loop
// continues only if it is >= exp(-lambda dt)).
//
// FP32: the uniform's 23 bits are k = hi:lo.  hi (18 bits) are the low 9 bits of the
// step's two normal words — FP32 Box-Muller reads only their top 23 bits, so hi is
// independent of the normals — and lo (5 bits) the top bits of word n mod 4 of block
// (n/4, path, stream, domain 2).  The test k >= kmin (equivalent to
// u01 >= exp(-lambda dt) in float, kmin precomputed exactly) cannot pass while
// hi < kmin >> 5, so the common step compares hi alone and lo is drawn only past that
// threshold (about lambda dt of the steps).
__device__ __forceinline__ uint32_t poisson_hi_f32(uint32_t wa, uint32_t wb) {
    return ((wa & 0x1FFu) << 9) | (wb & 0x1FFu);
}

// pois: FP32 the 18 high bits (poisson_hi_f32), FP64 the full word.  On a jump,
// `word` holds the full first-uniform word (top 23 bits k in FP32).
template <class R>
__device__ __forceinline__ bool jump_first(uint32_t pois, const StepConst<R> &p, uint32_t kmin, uint32_t k0,
                                           uint32_t k1, uint32_t path, uint32_t stream, int n, uint32_t &word) {
    if constexpr (sizeof(R) == 4) {
        if (pois < (kmin >> 5)) return false;
        const U4 q = philox4x32_10(U4{static_cast<uint32_t>(n >> 2), path, stream, 2u}, k0, k1);
        const int j = n & 3;
        const uint32_t w = j == 0 ? q.x : (j == 1 ? q.y : (j == 2 ? q.z : q.w));
        word = ((pois << 5) | (w >> 27)) << 9;
        return (word >> 9) >= kmin;
    } else {
        word = pois;
        return Math<R>::u01(pois) >= p.exp_m_lambda_dt;
    }
}

// First-Poisson-uniform inputs of steps n and n+1 (n even): FP32 the high bits from
// the normal block w of those steps; FP64 word n mod 4 of the domain-2 block wp
// (fetched by the caller every fourth step).
template <class R>
__device__ __forceinline__ void poisson_words(const U4 &w, const U4 &wp, int n, uint32_t &p0, uint32_t &p1) {
    if constexpr (sizeof(R) == 4) {
        p0 = poisson_hi_f32(w.x, w.y);
        p1 = poisson_hi_f32(w.z, w.w);
    } else {
        const bool lo = (n & 3) == 0;
        p0 = lo ? wp.x : wp.z;
        p1 = lo ? wp.y : wp.w;
    }
}

template <class R, int MODEL, int SCHEME>
__device__ __forceinline__ void one_step_z(const StepConst<R> &p, PathState<R> &st, R z1, R z2, uint32_t wpois,
                                           uint32_t kmin, uint32_t k0, uint32_t k1, uint32_t path, uint32_t stream,
                                           int n) {
    heston_step<R, SCHEME>(p, st.S, st.v, z1, z2);
    if constexpr (MODEL == kBates) {
        uint32_t word;
        if (jump_first<R>(wpois, p, kmin, k0, k1, path, stream, n, word)) {
            PhiloxJumpDraws<R> d{k0, k1, path, stream, static_cast<uint32_t>(n), Math<R>::u01(word), 1, 0, U4{0, 0, 0, 0}};
            st.S *= jump_factor<R>(p, d.first, d);
        }
    }
}

template <class R, int MODEL, int SCHEME>
__device__ __forceinline__ void one_step(const StepConst<R> &p, PathState<R> &st, uint32_t wa, uint32_t wb,
                                         uint32_t wpois, uint32_t kmin, uint32_t k0, uint32_t k1, uint32_t path,
                                         uint32_t stream, int n) {
    R z1, z2;
    Math<R>::box_muller(wa, wb, z1, z2);
    one_step_z<R, MODEL, SCHEME>(p, st, z1, z2, wpois, kmin, k0, k1, path, stream, n);
}

// TRK: keep the path state that Asian, barrier and lookback legs read (running sum,
// max, min); false for launches whose legs read only the final spot.
template <class R, int MODEL, int SCHEME, bool TRK = true, class Gen, class Sink>
__device__ __forceinline__ void simulate_path(const StepConst<R> &p, R S0, R v0, int n_steps, const Gen &gen,
                                              uint32_t k0, uint32_t k1, uint32_t path, uint32_t stream, uint32_t kmin,
                                              PathState<R> &st, Sink &&sink) {
    st.S = S0;
    st.v = v0;
    st.ssum = 0.0;
    st.smax = S0;
    st.smin = S0;
    for (int n0 = 0; n0 < n_steps; n0 += kSumChunk) {
        const int n1 = min(n0 + kSumChunk, n_steps);
        R blk = R(0);
        U4 wp{0u, 0u, 0u, 0u};  // Poisson words of steps 4m .. 4m+3 (n0 is a multiple of 4)
        int n = n0;
        for (; n + 1 < n1; n += 2) {
            const U4 w = gen(U4{static_cast<uint32_t>(n >> 1), path, stream, 0u});
            uint32_t pw0 = 0u, pw1 = 0u;
            if constexpr (MODEL == kBates) {
                if constexpr (sizeof(R) == 8) {
                    if ((n & 3) == 0) wp = gen(U4{static_cast<uint32_t>(n >> 2), path, stream, 2u});
                }
                poisson_words<R>(w, wp, n, pw0, pw1);
            }
            if constexpr (sizeof(R) == 4) {
                // the normals of both steps (independent of the path state) in one paired
                // Box-Muller; the same bits as two one-pair calls
                float2 Z1, Z2;
                Math<float>::box_muller_two(w.x, w.y, w.z, w.w, Z1, Z2);
                one_step_z<R, MODEL, SCHEME>(p, st, Z1.x, Z2.x, pw0, kmin, k0, k1, path, stream, n);
                if constexpr (TRK) track(st, blk);
                sink(n, st.S, st.v);
                one_step_z<R, MODEL, SCHEME>(p, st, Z1.y, Z2.y, pw1, kmin, k0, k1, path, stream, n + 1);
            } else {
                one_step<R, MODEL, SCHEME>(p, st, w.x, w.y, pw0, kmin, k0, k1, path, stream, n);
                if constexpr (TRK) track(st, blk);
                sink(n, st.S, st.v);
                one_step<R, MODEL, SCHEME>(p, st, w.z, w.w, pw1, kmin, k0, k1, path, stream, n + 1);
            }
            if constexpr (TRK) track(st, blk);
            sink(n + 1, st.S, st.v);
        }
        if (n < n1) {
            const U4 w = gen(U4{static_cast<uint32_t>(n >> 1), path, stream, 0u});
            uint32_t pw0 = 0u, pw1 = 0u;
            if constexpr (MODEL == kBates) {
                if constexpr (sizeof(R) == 8) {
                    if ((n & 3) == 0) wp = gen(U4{static_cast<uint32_t>(n >> 2), path, stream, 2u});
                }
                poisson_words<R>(w, wp, n, pw0, pw1);
            }
            one_step<R, MODEL, SCHEME>(p, st, w.x, w.y, pw0, kmin, k0, k1, path, stream, n);
            if constexpr (TRK) track(st, blk);
            sink(n, st.S, st.v);
        }
        if constexpr (TRK) st.ssum += static_cast<double>(blk);
    }
}

// Two paths per lane.  NEG: an antithetic pair — one set of draws (those of path
// a), path b with every normal negated and the same Poisson uniforms.  Otherwise
// two independent paths, each with its own draws, interleaved for instruction-level
// parallelism.
// FP32 normals of one step of a lane's two paths: paired Box-Muller, or path b the
// mirror of path a (antithetic pair).
template <bool NEG>
__device__ __forceinline__ void normals_two_f32(uint32_t wa1, uint32_t wa2, uint32_t wb1, uint32_t wb2, float2 &Z1,
                                                float2 &Z2) {
    if constexpr (NEG) {
        float za1, za2;
        Math<float>::box_muller(wa1, wa2, za1, za2);
        Z1 = make_float2(za1, -za1);
        Z2 = make_float2(za2, -za2);
    } else {
        Math<float>::box_muller_two(wa1, wa2, wb1, wb2, Z1, Z2);
    }
}

// Bates jumps of both paths of a lane after their Heston step.
template <class R, int MODEL, bool NEG>
__device__ __forceinline__ void jumps_two(const StepConst<R> &p, PathState<R> &a, PathState<R> &b, uint32_t pois_a,
                                          uint32_t pois_b, uint32_t kmin, uint32_t k0, uint32_t k1, uint32_t path_a,
                                          uint32_t path_b, uint32_t stream, int n) {
    if constexpr (MODEL == kBates) {
        uint32_t word;
        if constexpr (NEG) {
            if (jump_first<R>(pois_a, p, kmin, k0, k1, path_a, stream, n, word)) {
                PhiloxJumpDraws<R> d{k0, k1, path_a, stream, static_cast<uint32_t>(n), Math<R>::u01(word), 1, 0,
                                     U4{0, 0, 0, 0}};
                R fa, fb;
                jump_factor_pair<R>(p, d.first, d, fa, fb);
                a.S *= fa;
                b.S *= fb;
            }
        } else if constexpr (sizeof(R) == 4) {
            // the one-compare tests of both paths inline; one copy of the rest of the
            // jump code for both (rare; keeps the loop body small)
            const uint32_t kmin_hi = kmin >> 5;
            if (pois_a >= kmin_hi || pois_b >= kmin_hi) {
#pragma unroll 1
                for (int i = 0; i < 2; ++i) {
                    const uint32_t pois = i ? pois_b : pois_a, path = i ? path_b : path_a;
                    if (jump_first<R>(pois, p, kmin, k0, k1, path, stream, n, word)) {
                        PhiloxJumpDraws<R> d{k0, k1, path, stream, static_cast<uint32_t>(n), Math<R>::u01(word), 1, 0,
                                             U4{0, 0, 0, 0}};
                        const R f = jump_factor<R>(p, d.first, d);
                        if (i) b.S *= f;
                        else a.S *= f;
                    }
                }
            }
        } else {
            if (jump_first<R>(pois_a, p, kmin, k0, k1, path_a, stream, n, word)) {
                PhiloxJumpDraws<R> d{k0, k1, path_a, stream, static_cast<uint32_t>(n), Math<R>::u01(word), 1, 0,
                                     U4{0, 0, 0, 0}};
                a.S *= jump_factor<R>(p, d.first, d);
            }
            if (jump_first<R>(pois_b, p, kmin, k0, k1, path_b, stream, n, word)) {
                PhiloxJumpDraws<R> d{k0, k1, path_b, stream, static_cast<uint32_t>(n), Math<R>::u01(word), 1, 0,
                                     U4{0, 0, 0, 0}};
                b.S *= jump_factor<R>(p, d.first, d);
            }
        }
    }
}

// One FP32 step of a lane's two paths from their normals (the paired scheme step, then
// the jumps).
template <int MODEL, int SCHEME, bool NEG>
__device__ __forceinline__ void step_two_z_f32(const StepConst<float> &p, PathState<float> &a, PathState<float> &b,
                                               float2 Z1, float2 Z2, uint32_t pois_a, uint32_t pois_b, uint32_t kmin,
                                               uint32_t k0, uint32_t k1, uint32_t path_a, uint32_t path_b,
                                               uint32_t stream, int n) {
    float2 S2 = make_float2(a.S, b.S), v2 = make_float2(a.v, b.v);
    if constexpr (SCHEME == kQE) step_qe_two_f32(p, S2, v2, Z1, Z2);
    else if constexpr (SCHEME == kMilstein) step_milstein_two_f32(p, S2, v2, Z1, Z2);
    else step_euler_two_f32(p, S2, v2, Z1, Z2);
    a.S = S2.x;
    b.S = S2.y;
    a.v = v2.x;
    b.v = v2.y;
    jumps_two<float, MODEL, NEG>(p, a, b, pois_a, pois_b, kmin, k0, k1, path_a, path_b, stream, n);
}

template <class R, int MODEL, int SCHEME, bool NEG>
__device__ __forceinline__ void one_step_two(const StepConst<R> &p, PathState<R> &a, PathState<R> &b, uint32_t wa1,
                                             uint32_t wa2, uint32_t wb1, uint32_t wb2, uint32_t pois_a,
                                             uint32_t pois_b, uint32_t kmin, uint32_t k0, uint32_t k1, uint32_t path_a,
                                             uint32_t path_b, uint32_t stream, int n) {
    if constexpr (sizeof(R) == 4) {
        float2 Z1, Z2;
        normals_two_f32<NEG>(wa1, wa2, wb1, wb2, Z1, Z2);
        step_two_z_f32<MODEL, SCHEME, NEG>(p, a, b, Z1, Z2, pois_a, pois_b, kmin, k0, k1, path_a, path_b, stream, n);
    } else {
        R za1, za2, zb1, zb2;
        Math<R>::box_muller(wa1, wa2, za1, za2);
        if constexpr (NEG) {
            zb1 = -za1;
            zb2 = -za2;
        } else {
            Math<R>::box_muller(wb1, wb2, zb1, zb2);
        }
        heston_step<R, SCHEME>(p, a.S, a.v, za1, za2);
        heston_step<R, SCHEME>(p, b.S, b.v, zb1, zb2);
        jumps_two<R, MODEL, NEG>(p, a, b, pois_a, pois_b, kmin, k0, k1, path_a, path_b, stream, n);
    }
}

// ssum_slot: where the two paths' Asian running sums (x: path a, y: path b) are kept
// between the 16-step blocks that add to them: this thread's shared-memory slot (two
// FP64 sums read and written once per block, four registers fewer in the step loop),
// or nullptr for a.ssum and b.ssum.
template <class R, int MODEL, int SCHEME, bool NEG, bool TRK = true, class Gen, class Sink2>
__device__ __forceinline__ void simulate_two(const StepConst<R> &p, R S0, R v0, int n_steps, const Gen &gen,
                                             uint32_t k0, uint32_t k1, uint32_t path_a, uint32_t path_b,
                                             uint32_t stream, uint32_t kmin, PathState<R> &a, PathState<R> &b,
                                             Sink2 &&sink, double2 *ssum_slot = nullptr) {
    a.S = b.S = S0;
    a.v = b.v = v0;
    a.ssum = b.ssum = 0.0;
    if (TRK && ssum_slot) *ssum_slot = make_double2(0.0, 0.0);
    a.smax = b.smax = S0;
    a.smin = b.smin = S0;
    for (int n0 = 0; n0 < n_steps; n0 += kSumChunk) {
        const int n1 = min(n0 + kSumChunk, n_steps);
        R blk_a = R(0), blk_b = R(0);
        U4 pa{0u, 0u, 0u, 0u}, pb{0u, 0u, 0u, 0u};
        int n = n0;
        for (; n + 1 < n1; n += 2) {
            const U4 wa = gen(U4{static_cast<uint32_t>(n >> 1), path_a, stream, 0u});
            U4 wb{0u, 0u, 0u, 0u};
            if constexpr (!NEG) wb = gen(U4{static_cast<uint32_t>(n >> 1), path_b, stream, 0u});
            uint32_t qa0 = 0u, qa1 = 0u, qb0 = 0u, qb1 = 0u;
            if constexpr (MODEL == kBates) {
                if constexpr (sizeof(R) == 8) {
                    if ((n & 3) == 0) {
                        pa = gen(U4{static_cast<uint32_t>(n >> 2), path_a, stream, 2u});
                        if constexpr (!NEG) pb = gen(U4{static_cast<uint32_t>(n >> 2), path_b, stream, 2u});
                    }
                }
                poisson_words<R>(wa, pa, n, qa0, qa1);
                if constexpr (!NEG) poisson_words<R>(wb, pb, n, qb0, qb1);
            }
            if constexpr (sizeof(R) == 4 && SCHEME != kQE) {
                // Euler and Milstein: both steps' normals first, so that the second step's
                // Box-Muller (independent of the first step) overlaps the first step's work
                // (QE, whose step holds more live values, measures faster without it)
                float2 Z1a, Z2a, Z1b, Z2b;
                normals_two_f32<NEG>(wa.x, wa.y, wb.x, wb.y, Z1a, Z2a);
                normals_two_f32<NEG>(wa.z, wa.w, wb.z, wb.w, Z1b, Z2b);
                step_two_z_f32<MODEL, SCHEME, NEG>(p, a, b, Z1a, Z2a, qa0, qb0, kmin, k0, k1, path_a, path_b, stream, n);
                if constexpr (TRK) track(a, blk_a);
                if constexpr (TRK) track(b, blk_b);
                sink(n, a.S, a.v, b.S, b.v);
                step_two_z_f32<MODEL, SCHEME, NEG>(p, a, b, Z1b, Z2b, qa1, qb1, kmin, k0, k1, path_a, path_b, stream,
                                                   n + 1);
            } else {
            one_step_two<R, MODEL, SCHEME, NEG>(p, a, b, wa.x, wa.y, wb.x, wb.y, qa0, qb0, kmin, k0, k1, path_a,
                                                path_b, stream, n);
            if constexpr (TRK) track(a, blk_a);
            if constexpr (TRK) track(b, blk_b);
            sink(n, a.S, a.v, b.S, b.v);
            one_step_two<R, MODEL, SCHEME, NEG>(p, a, b, wa.z, wa.w, wb.z, wb.w, qa1, qb1, kmin, k0, k1, path_a,
                                                path_b, stream, n + 1);
            }
            if constexpr (TRK) track(a, blk_a);
            if constexpr (TRK) track(b, blk_b);
            sink(n + 1, a.S, a.v, b.S, b.v);
        }
        if (n < n1) {
            const U4 wa = gen(U4{static_cast<uint32_t>(n >> 1), path_a, stream, 0u});
            U4 wb{0u, 0u, 0u, 0u};
            if constexpr (!NEG) wb = gen(U4{static_cast<uint32_t>(n >> 1), path_b, stream, 0u});
            uint32_t qa0 = 0u, qa1 = 0u, qb0 = 0u, qb1 = 0u;
            if constexpr (MODEL == kBates) {
                if constexpr (sizeof(R) == 8) {
                    if ((n & 3) == 0) {
                        pa = gen(U4{static_cast<uint32_t>(n >> 2), path_a, stream, 2u});
                        if constexpr (!NEG) pb = gen(U4{static_cast<uint32_t>(n >> 2), path_b, stream, 2u});
                    }
                }
                poisson_words<R>(wa, pa, n, qa0, qa1);
                if constexpr (!NEG) poisson_words<R>(wb, pb, n, qb0, qb1);
            }
            one_step_two<R, MODEL, SCHEME, NEG>(p, a, b, wa.x, wa.y, wb.x, wb.y, qa0, qb0, kmin, k0, k1, path_a,
                                                path_b, stream, n);
            if constexpr (TRK) track(a, blk_a);
            if constexpr (TRK) track(b, blk_b);
            sink(n, a.S, a.v, b.S, b.v);
        }
        if constexpr (TRK) {
            if (ssum_slot) {
                double2 s = *ssum_slot;
                s.x += static_cast<double>(blk_a);
                s.y += static_cast<double>(blk_b);
                *ssum_slot = s;
            } else {
                a.ssum += static_cast<double>(blk_a);
                b.ssum += static_cast<double>(blk_b);
            }
        }
    }
    if (TRK && ssum_slot) {
        a.ssum = ssum_slot->x;
        b.ssum = ssum_slot->y;
    }
}

template <class R>
__device__ __forceinline__ const StepConst<R> &task_const(const TaskDev &t);
template <>
__device__ __forceinline__ const StepConst<float> &task_const<float>(const TaskDev &t) { return t.cf; }
template <>
__device__ __forceinline__ const StepConst<double> &task_const<double>(const TaskDev &t) { return t.cd; }

template <class R, class Sink>
__device__ __forceinline__ void simulate_dispatch(const TaskDev &t, const StepConst<R> &p, uint32_t path,
                                                  PathState<R> &st, Sink &&sink) {
    const R S0 = static_cast<R>(t.S0);
    const R v0 = static_cast<R>(t.v0);
    const uint32_t km = t.jump_kmin;
    const RegKeys g{t.key0, t.key1};
    switch (t.model * 3 + t.scheme) {
        case 0: simulate_path<R, kHeston, kEuler>(p, S0, v0, t.n_steps, g, t.key0, t.key1, path, t.stream, km, st, sink); break;
        case 1: simulate_path<R, kHeston, kMilstein>(p, S0, v0, t.n_steps, g, t.key0, t.key1, path, t.stream, km, st, sink); break;
        case 2: simulate_path<R, kHeston, kQE>(p, S0, v0, t.n_steps, g, t.key0, t.key1, path, t.stream, km, st, sink); break;
        case 3: simulate_path<R, kBates, kEuler>(p, S0, v0, t.n_steps, g, t.key0, t.key1, path, t.stream, km, st, sink); break;
        case 4: simulate_path<R, kBates, kMilstein>(p, S0, v0, t.n_steps, g, t.key0, t.key1, path, t.stream, km, st, sink); break;
        default: simulate_path<R, kBates, kQE>(p, S0, v0, t.n_steps, g, t.key0, t.key1, path, t.stream, km, st, sink); break;
    }
}

// ----------------------------------------------------------------------------
// Fused pricing kernel.  Persistent: each warp pops queue slots from a device
// cursor; slot q belongs to the task whose tile range [tile_begin, tile_begin +
// n_tiles) holds it (binary search over the task prefix, tasks ordered by the
// host's schedule).  A tile is a number of rounds in which every lane simulates
// one lane unit (a path, an antithetic pair or two paths); every requested payoff leg is evaluated in registers and folded into per-warp FP64
// moments (n, mean, M2, #ITM), then into one record per tile and leg.  The
// reference writes payoffs to memory and reduces them in two more passes
// (OptionPricer.hpp:123-193); here nothing per path leaves registers.
// ----------------------------------------------------------------------------
__device__ __forceinline__ int find_task(const int64_t *__restrict__ prefix, int n_tasks, int64_t q) {
    int lo = 0, hi = n_tasks - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= q) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// LANE: kLaneOne (a lane simulates one path), kLanePair (an antithetic pair),
// kLaneTwo (two independent paths 2u and 2u+1).
// Blocks of 128, 256 or 512 threads (FP32; up to 256 in FP64): the register budget is
// set for kPathMinBlocksFp32 resident 256-thread blocks per SM (64 registers a thread).
template <class R, int MODEL, int SCHEME, bool UK, int LANE, bool TRK>
__global__ void __launch_bounds__(path_block_max<R>(),
                                  sizeof(R) == 4 ? kPathMinBlocksFp32 * kPathBlock / path_block_max<R>() : 1)
    price_tiles_kernel(const TaskDev *__restrict__ tasks, const int64_t *__restrict__ prefix, int32_t n_tasks,
                       int64_t slot_begin, int64_t slot_end, unsigned long long *__restrict__ cursor,
                       Moments *__restrict__ partials, const PhiloxRoundKeys rk) {
    // Every warp is an independent worker: it pops a tile (kWarpTilePaths * ppt paths of one
    // task), keeps the tile's running moments per leg in its own shared-memory slots and
    // writes one record per leg.  No block-wide barrier anywhere.
    __shared__ Moments s_acc[path_block_max<R>() / 32][QK_MAX_PAYOFFS];
    // the Asian running sums of a lane's two independent paths (simulate_two); one slot per
    // thread (antithetic pairs keep theirs in registers, which measures faster there)
    constexpr bool kSumSlot = LANE == kLaneTwo && TRK;
    __shared__ double2 s_ssum[kSumSlot ? path_block_max<R>() : 1];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const R eps_payoff = sizeof(R) == 4 ? R(1e-6) : R(1e-12);  // OptionPricer.hpp:316
    Moments *acc = s_acc[warp];

    for (;;) {
        long long q = 0;
        if (lane == 0) q = slot_begin + static_cast<long long>(atomicAdd(cursor, 1ull));
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= slot_end) return;

        const int ti = find_task(prefix, n_tasks, q);
        const TaskDev &t = tasks[ti];
        const int64_t tile = q - t.tile_begin;
        const StepConst<R> p = task_const<R>(t);
        const int np = t.n_payoffs;
        const int n_steps = t.n_steps;
        const int64_t n_paths = t.n_paths;
        const uint32_t k0 = t.key0, k1 = t.key1, stream = t.stream, kmin = t.jump_kmin;
        const R S0 = static_cast<R>(t.S0), v0 = static_cast<R>(t.v0);
        // big tiles of ppt rounds, then the tail in tiles of ppt_tail rounds
        const bool big = tile < t.n_big;
        const int tile_rounds = big ? t.ppt : t.ppt_tail;
        const int64_t first_round = big ? tile * t.ppt
                                        : static_cast<int64_t>(t.n_big) * t.ppt + (tile - t.n_big) * t.ppt_tail;
        const int64_t tile_first = first_round * kWarpTilePaths;
        if (lane < np) acc[lane] = Moments{0.0, 0.0, 0.0, 0.0};
        __syncwarp();

        // a lane's unit: one path, one antithetic pair, or two consecutive paths
        const int64_t n_units = lane_units(n_paths, LANE);
        const int64_t left = n_units - tile_first;
        const int rounds =
            static_cast<int>(min(static_cast<int64_t>(tile_rounds), (left + kWarpTilePaths - 1) / kWarpTilePaths));
        for (int j = 0; j < rounds; ++j) {
            const int64_t unit = tile_first + static_cast<int64_t>(j) * kWarpTilePaths + lane;
            const bool active = unit < n_units;
            if constexpr (LANE != kLaneOne) {
                constexpr bool NEG = LANE == kLanePair;
                const uint32_t pa = NEG ? static_cast<uint32_t>(unit) : static_cast<uint32_t>(2 * unit);
                const uint32_t pb = NEG ? pa : pa + 1u;
                const bool active_b = NEG ? active : (active && static_cast<int64_t>(pb) < n_paths);
                PathState<R> sa, sb;
                if (active) {
                    if constexpr (UK) {
                        simulate_two<R, MODEL, SCHEME, NEG, TRK>(p, S0, v0, n_steps, ParamKeys{rk}, k0, k1, pa, pb, stream,
                                                            kmin, sa, sb, NoSink2{}, kSumSlot ? &s_ssum[threadIdx.x] : nullptr);
                    } else {
                        simulate_two<R, MODEL, SCHEME, NEG, TRK>(p, S0, v0, n_steps, RegKeys{k0, k1}, k0, k1, pa, pb,
                                                            stream, kmin, sa, sb, NoSink2{}, kSumSlot ? &s_ssum[threadIdx.x] : nullptr);
                    }
                } else {
                    sa.S = sa.smax = sa.smin = sb.S = sb.smax = sb.smin = R(0);
                    sa.ssum = sb.ssum = 0.0;
                }
                for (int k = 0; k < np; ++k) {
                    const PayoffSpec ps = t.pay[k];
                    const R xa = active ? final_payoff<R>(ps, sa.S, sa.ssum, sa.smax, sa.smin, n_steps) : R(0);
                    const R xb = active_b ? final_payoff<R>(ps, sb.S, sb.ssum, sb.smax, sb.smin, n_steps) : R(0);
                    Moments wm;
                    if constexpr (NEG) {
                        const double y = 0.5 * (static_cast<double>(xa) + static_cast<double>(xb));
                        wm = warp_moments_pair(y, active, xa > eps_payoff, xb > eps_payoff);
                    } else {
                        wm = chan_merge(warp_moments(static_cast<double>(xa), active, xa > eps_payoff),
                                        warp_moments(static_cast<double>(xb), active_b, xb > eps_payoff));
                    }
                    if (lane == 0) acc[k] = chan_merge(acc[k], wm);
                }
            } else {
                PathState<R> st;
                if (active) {
                    if constexpr (UK) {
                        simulate_path<R, MODEL, SCHEME, TRK>(p, S0, v0, n_steps, ParamKeys{rk}, k0, k1,
                                                        static_cast<uint32_t>(unit), stream, kmin, st, NoSink{});
                    } else {
                        simulate_path<R, MODEL, SCHEME, TRK>(p, S0, v0, n_steps, RegKeys{k0, k1}, k0, k1,
                                                        static_cast<uint32_t>(unit), stream, kmin, st, NoSink{});
                    }
                } else {
                    st.S = st.smax = st.smin = R(0);
                    st.ssum = 0.0;
                }
                for (int k = 0; k < np; ++k) {
                    const PayoffSpec ps = t.pay[k];
                    const R x = active ? final_payoff<R>(ps, st.S, st.ssum, st.smax, st.smin, n_steps) : R(0);
                    const Moments wm = warp_moments(static_cast<double>(x), active, x > eps_payoff);
                    if (lane == 0) acc[k] = chan_merge(acc[k], wm);
                }
            }
        }
        __syncwarp();
        if (lane < np) partials[t.partial_base + tile * np + lane] = acc[lane];
        __syncwarp();
    }
}

template <class R>
using PriceKernel = void (*)(const TaskDev *, const int64_t *, int32_t, int64_t, int64_t, unsigned long long *,
                             Moments *, const PhiloxRoundKeys);

template <class R, bool UK, int LANE, bool TRK>
__host__ PriceKernel<R> price_kernel_for_keys(int model, int scheme) {
    switch (model * 3 + scheme) {
        case 0: return price_tiles_kernel<R, kHeston, kEuler, UK, LANE, TRK>;
        case 1: return price_tiles_kernel<R, kHeston, kMilstein, UK, LANE, TRK>;
        case 2: return price_tiles_kernel<R, kHeston, kQE, UK, LANE, TRK>;
        case 3: return price_tiles_kernel<R, kBates, kEuler, UK, LANE, TRK>;
        case 4: return price_tiles_kernel<R, kBates, kMilstein, UK, LANE, TRK>;
        default: return price_tiles_kernel<R, kBates, kQE, UK, LANE, TRK>;
    }
}

template <class R, int LANE>
__host__ PriceKernel<R> price_kernel_for_lane(int model, int scheme, bool uniform_key, bool track) {
    if (track)
        return uniform_key ? price_kernel_for_keys<R, true, LANE, true>(model, scheme)
                           : price_kernel_for_keys<R, false, LANE, true>(model, scheme);
    return uniform_key ? price_kernel_for_keys<R, true, LANE, false>(model, scheme)
                       : price_kernel_for_keys<R, false, LANE, false>(model, scheme);
}

template <class R>
__host__ PriceKernel<R> price_kernel_for(int model, int scheme, bool uniform_key = true, int lane_mode = kLaneOne,
                                         bool track = true) {
    switch (lane_mode) {
        case kLanePair: return price_kernel_for_lane<R, kLanePair>(model, scheme, uniform_key, track);
        case kLaneTwo: return price_kernel_for_lane<R, kLaneTwo>(model, scheme, uniform_key, track);
        default: return price_kernel_for_lane<R, kLaneOne>(model, scheme, uniform_key, track);
    }
}

// Merging moment records.  A set of records (n_i, mean_i, M2_i, itm_i) is merged
// in one pass about a shift c (the first record's mean).  With d_i = mean_i - c:
// N = sum n_i,  D = sum n_i d_i,  Q = sum (M2_i + n_i d_i^2), then
// mean = c + D / N and M2 = Q - D^2 / N (the pairwise update of Chan et al.
// applied to all records at once; c lies within a few standard errors of the
// mean, so D^2 / N is a small correction to Q).  No division per record;
// per-thread sums fold through a fixed-shape tree, so the result is deterministic
// for a given tile plan.
__device__ __forceinline__ void block_sum4(double &a, double &b, double &c, double &d, double (*red)[32]) {
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    d = warp_sum(d);
    const int warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][warp] = a;
        red[1][warp] = b;
        red[2][warp] = c;
        red[3][warp] = d;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = b = c = d = 0.0;
        for (int w = 0; w < nw; ++w) {
            a += red[0][w];
            b += red[1][w];
            c += red[2][w];
            d += red[3][w];
        }
    }
    __syncthreads();
}

// Neumaier's compensated addition (Neumaier, ZAMM 54, 1974): s + c carries the sum
// of the added values with the rounding error of every addition kept in c.
__device__ __forceinline__ void neumaier_add(double &s, double &c, double x) {
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
}

// Block-wide merge of rec[i * stride], i < count; the result is valid in thread 0.
// Each thread sums its records' D and Q with compensation; the per-thread sums and
// their compensations are reduced separately and added at the end.
__device__ __forceinline__ Moments merge_range(const Moments *__restrict__ rec, int64_t count, int64_t stride,
                                               double (*red)[32]) {
    const double c = count > 0 ? rec[0].mean : 0.0;
    double n = 0.0, D = 0.0, Q = 0.0, itm = 0.0, cD = 0.0, cQ = 0.0;
    for (int64_t i = threadIdx.x; i < count; i += blockDim.x) {
        const Moments m = rec[i * stride];
        const double d = m.mean - c;
        const double nd = m.n * d;
        n += m.n;
        neumaier_add(D, cD, nd);
        neumaier_add(Q, cQ, fma(nd, d, m.m2));
        itm += m.itm;
    }
    block_sum4(n, D, Q, itm, red);
    double z0 = 0.0, z1 = 0.0;
    block_sum4(cD, cQ, z0, z1, red);
    Moments r{0.0, 0.0, 0.0, 0.0};
    if (n > 0.0) {
        D += cD;
        Q += cQ;
        r.n = n;
        r.mean = c + D / n;
        r.m2 = fmax(Q - D * (D / n), 0.0);
        r.itm = itm;
    }
    return r;
}

// One block per task: merge all its tile records (tasks with few tiles; the
// allocation-free entry point).
__global__ void __launch_bounds__(1024) merge_tasks_kernel(const TaskDev *__restrict__ tasks,
                                                           const Moments *__restrict__ partials,
                                                           TaskMoments *__restrict__ out) {
    __shared__ double red[4][32];
    const TaskDev &t = tasks[blockIdx.x];
    const int np = t.n_payoffs;
    for (int k = 0; k < np; ++k) {
        const Moments r = merge_range(partials + t.partial_base + k, t.n_tiles, np, red);
        if (threadIdx.x == 0) out[static_cast<int64_t>(blockIdx.x) * QK_MAX_PAYOFFS + k] = r;
    }
}

// Two-level merge, level 1: one block per chunk of kMergeChunkTiles consecutive
// tile records of one task, writing one record per chunk and leg
// (chunks[chunk][QK_MAX_PAYOFFS]).  The chunk's task is found by binary search
// over the tasks' chunk_base (ascending, every task has at least one chunk).
__global__ void __launch_bounds__(256) merge_chunks_kernel(const TaskDev *__restrict__ tasks, int32_t n_tasks,
                                                           const Moments *__restrict__ partials,
                                                           Moments *__restrict__ chunks) {
    __shared__ double red[4][32];
    const int64_t b = blockIdx.x;
    int lo = 0, hi = n_tasks - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tasks[mid].chunk_base <= b) lo = mid;
        else hi = mid - 1;
    }
    const TaskDev &t = tasks[lo];
    const int np = t.n_payoffs;
    const int64_t first = (b - t.chunk_base) * kMergeChunkTiles;
    const int64_t count = min(static_cast<int64_t>(kMergeChunkTiles), static_cast<int64_t>(t.n_tiles) - first);
    for (int k = 0; k < np; ++k) {
        const Moments r = merge_range(partials + t.partial_base + first * np + k, count, np, red);
        if (threadIdx.x == 0) chunks[b * QK_MAX_PAYOFFS + k] = r;
    }
}

// Level 2: one block per task merges its chunk records.
__global__ void __launch_bounds__(128) merge_task_chunks_kernel(const TaskDev *__restrict__ tasks,
                                                                const Moments *__restrict__ chunks,
                                                                TaskMoments *__restrict__ out) {
    __shared__ double red[4][32];
    const TaskDev &t = tasks[blockIdx.x];
    for (int k = 0; k < t.n_payoffs; ++k) {
        const Moments r = merge_range(chunks + t.chunk_base * QK_MAX_PAYOFFS + k, t.n_chunks, QK_MAX_PAYOFFS, red);
        if (threadIdx.x == 0) out[static_cast<int64_t>(blockIdx.x) * QK_MAX_PAYOFFS + k] = r;
    }
}

// Exercise-date slabs (LSM) / full path dump: one path per thread (a two-path
// variant follows), S (and v)
// after every `stride`-th step stored as SoA rows slab[date][path] (coalesced:
// consecutive threads write consecutive columns).  Specialised per kind, with the
// Philox round keys in the kernel parameters.
template <class R, int MODEL, int SCHEME>
__global__ void __launch_bounds__(kPathBlock) slab_paths_kernel(const TaskDev *__restrict__ task, int64_t first_path,
                                                               int64_t count, int stride, R *__restrict__ slab_S,
                                                               R *__restrict__ slab_v, int64_t ld,
                                                               const PhiloxRoundKeys rk) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const TaskDev &t = *task;
    const StepConst<R> p = task_const<R>(t);
    SlabSink<R> sink{slab_S, slab_v, ld, i, stride, stride};
    PathState<R> st;
    simulate_path<R, MODEL, SCHEME>(p, static_cast<R>(t.S0), static_cast<R>(t.v0), t.n_steps, ParamKeys{rk}, t.key0,
                                    t.key1, static_cast<uint32_t>(first_path + i), t.stream, t.jump_kmin, st, sink);
}

// Two paths per thread (first + 2i and first + 2i + 1), interleaved and, in FP32,
// stepped as pairs; same values as the one-path kernel.
template <class R, int MODEL, int SCHEME>
__global__ void __launch_bounds__(kPathBlock) slab_paths_two_kernel(const TaskDev *__restrict__ task,
                                                                   int64_t first_path, int64_t count, int stride,
                                                                   R *__restrict__ slab_S, R *__restrict__ slab_v,
                                                                   int64_t ld, const PhiloxRoundKeys rk) {
    const int64_t i = 2 * (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x);
    if (i >= count) return;
    const TaskDev &t = *task;
    const StepConst<R> p = task_const<R>(t);
    SlabSink2<R> sink{slab_S, slab_v, ld, i, stride, stride, i + 1 < count};
    PathState<R> sa, sb;
    const uint32_t pa = static_cast<uint32_t>(first_path + i);
    simulate_two<R, MODEL, SCHEME, false>(p, static_cast<R>(t.S0), static_cast<R>(t.v0), t.n_steps, ParamKeys{rk},
                                          t.key0, t.key1, pa, pa + 1u, t.stream, t.jump_kmin, sa, sb, sink);
}

template <class R>
using SlabKernel = void (*)(const TaskDev *, int64_t, int64_t, int, R *, R *, int64_t, const PhiloxRoundKeys);

template <class R>
SlabKernel<R> slab_two_kernel_for(int model, int scheme) {
    switch (model * 3 + scheme) {
        case 0: return slab_paths_two_kernel<R, kHeston, kEuler>;
        case 1: return slab_paths_two_kernel<R, kHeston, kMilstein>;
        case 2: return slab_paths_two_kernel<R, kHeston, kQE>;
        case 3: return slab_paths_two_kernel<R, kBates, kEuler>;
        case 4: return slab_paths_two_kernel<R, kBates, kMilstein>;
        default: return slab_paths_two_kernel<R, kBates, kQE>;
    }
}

template <class R>
SlabKernel<R> slab_kernel_for(int model, int scheme) {
    switch (model * 3 + scheme) {
        case 0: return slab_paths_kernel<R, kHeston, kEuler>;
        case 1: return slab_paths_kernel<R, kHeston, kMilstein>;
        case 2: return slab_paths_kernel<R, kHeston, kQE>;
        case 3: return slab_paths_kernel<R, kBates, kEuler>;
        case 4: return slab_paths_kernel<R, kBates, kMilstein>;
        default: return slab_paths_kernel<R, kBates, kQE>;
    }
}

// Per-path payoff of leg 0 (undiscounted, normalised units), for the payoff
// distribution analysis (OptionPricer.hpp:340-360 sorts every path's payoff).
template <class R>
__global__ void __launch_bounds__(kPathBlock) payoff_paths_kernel(const TaskDev *__restrict__ task, int64_t first,
                                                                 int64_t count, double *__restrict__ out) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const TaskDev &t = *task;
    const StepConst<R> p = task_const<R>(t);
    PathState<R> st;
    simulate_dispatch<R>(t, p, static_cast<uint32_t>(first + i), st, NoSink{});
    out[i] = static_cast<double>(final_payoff<R>(t.pay[0], st.S, st.ssum, st.smax, st.smin, t.n_steps));
}

// Payoff of one leg on a fed spot sequence S_1..S_n (one thread): the path kernel's
// tracking (running max / min, the Asian sum in blocks of kSumChunk steps in the working
// precision folded into FP64) and final_payoff, on the given values instead of simulated
// ones (PayoffTracker::track_current_price + evaluate_final_payoff, Payoff.hpp:84-243).
template <class R>
__global__ void payoff_trace_kernel(const PayoffSpec ps, const double *__restrict__ S, int n, double S0,
                                    double *__restrict__ out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    PathState<R> st;
    st.S = static_cast<R>(S0);
    st.v = R(0);
    st.ssum = 0.0;
    st.smax = st.S;
    st.smin = st.S;
    for (int n0 = 0; n0 < n; n0 += kSumChunk) {
        R blk = R(0);
        const int n1 = min(n0 + kSumChunk, n);
        for (int i = n0; i < n1; ++i) {
            st.S = static_cast<R>(S[i]);
            track(st, blk);
        }
        st.ssum += static_cast<double>(blk);
    }
    *out = static_cast<double>(final_payoff<R>(ps, st.S, st.ssum, st.smax, st.smin, n));
}

// Fed-draw trace of the step functions (one thread).
template <class R>
__global__ void step_trace_kernel(const TaskDev *__restrict__ task, const double *__restrict__ z,
                                  const double *__restrict__ u, int umax, int n, double *__restrict__ S_out,
                                  double *__restrict__ v_out, int *__restrict__ status) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const TaskDev &t = *task;
    const StepConst<R> p = task_const<R>(t);
    R S = static_cast<R>(t.S0);
    R v = static_cast<R>(t.v0);
    for (int i = 0; i < n; ++i) {
        FedStep<R> d{z + 3 * static_cast<int64_t>(i), u + static_cast<int64_t>(umax) * i, umax, 0, 0};
        switch (t.model * 3 + t.scheme) {
            case 0: evolve_step<R, kHeston, kEuler>(p, S, v, d); break;
            case 1: evolve_step<R, kHeston, kMilstein>(p, S, v, d); break;
            case 2: evolve_step<R, kHeston, kQE>(p, S, v, d); break;
            case 3: evolve_step<R, kBates, kEuler>(p, S, v, d); break;
            case 4: evolve_step<R, kBates, kMilstein>(p, S, v, d); break;
            default: evolve_step<R, kBates, kQE>(p, S, v, d); break;
        }
        if (d.overflow) {
            *status = 1;
            return;
        }
        S_out[i] = static_cast<double>(S);
        v_out[i] = static_cast<double>(v);
    }
    *status = 0;
}

// ----------------------------------------------------------------------------
// Launchers
// ----------------------------------------------------------------------------
cudaError_t launch_price_tiles(int precision, int model, int scheme, int grid, cudaStream_t s, const TaskDev *tasks,
                               const int64_t *prefix, int32_t n_tasks, int64_t slot_begin, int64_t slot_end,
                               unsigned long long *cursor, Moments *partials, bool uniform_key, uint64_t seed,
                               int lane_mode, bool track, int block) {
    if (!price_tiles_block_ok(precision, block)) return cudaErrorInvalidConfiguration;
    const PhiloxRoundKeys rk = philox_round_keys(static_cast<uint32_t>(seed & 0xFFFFFFFFull),
                                                 static_cast<uint32_t>(seed >> 32));
    if (precision == QK_FP32)
        price_kernel_for<float>(model, scheme, uniform_key, lane_mode, track)<<<grid, block, 0, s>>>(
            tasks, prefix, n_tasks, slot_begin, slot_end, cursor, partials, rk);
    else
        price_kernel_for<double>(model, scheme, uniform_key, lane_mode, track)<<<grid, block, 0, s>>>(
            tasks, prefix, n_tasks, slot_begin, slot_end, cursor, partials, rk);
    return cudaGetLastError();
}

bool price_tiles_block_ok(int precision, int block) {
    const int mx = precision == QK_FP32 ? path_block_max<float>() : path_block_max<double>();
    return block >= 64 && block <= mx && block % 32 == 0;
}

cudaError_t launch_merge_tasks(int n_tasks, cudaStream_t s, const TaskDev *tasks, const Moments *partials,
                               TaskMoments *out, int64_t max_tiles) {
    // one block per task; wide blocks only when some task has many tiles to read
    const int threads = max_tiles >= 4096 ? 1024 : 256;
    merge_tasks_kernel<<<n_tasks, threads, 0, s>>>(tasks, partials, out);
    return cudaGetLastError();
}

cudaError_t launch_merge_two_level(int n_tasks, int64_t n_chunks, cudaStream_t s, const TaskDev *tasks,
                                   const Moments *partials, Moments *chunks, TaskMoments *out) {
    merge_chunks_kernel<<<static_cast<unsigned>(n_chunks), 256, 0, s>>>(tasks, n_tasks, partials, chunks);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    merge_task_chunks_kernel<<<n_tasks, 128, 0, s>>>(tasks, chunks, out);
    return cudaGetLastError();
}

cudaError_t launch_slab_paths(int precision, int model, int scheme, uint64_t seed, cudaStream_t s, const TaskDev *task,
                              int64_t first_path, int64_t count, int stride, void *slab_S, void *slab_v, int64_t ld,
                              int paths_per_thread) {
    const PhiloxRoundKeys rk = philox_round_keys(static_cast<uint32_t>(seed & 0xFFFFFFFFull),
                                                 static_cast<uint32_t>(seed >> 32));
    if (paths_per_thread == 2) {
        const int64_t threads = (count + 1) / 2;
        const unsigned blocks2 = static_cast<unsigned>((threads + kPathBlock - 1) / kPathBlock);
        if (precision == QK_FP32)
            slab_two_kernel_for<float>(model, scheme)<<<blocks2, kPathBlock, 0, s>>>(
                task, first_path, count, stride, static_cast<float *>(slab_S), static_cast<float *>(slab_v), ld, rk);
        else
            slab_two_kernel_for<double>(model, scheme)<<<blocks2, kPathBlock, 0, s>>>(
                task, first_path, count, stride, static_cast<double *>(slab_S), static_cast<double *>(slab_v), ld, rk);
        return cudaGetLastError();
    }
    const int64_t blocks = (count + kPathBlock - 1) / kPathBlock;
    if (precision == QK_FP32)
        slab_kernel_for<float>(model, scheme)<<<static_cast<unsigned>(blocks), kPathBlock, 0, s>>>(
            task, first_path, count, stride, static_cast<float *>(slab_S), static_cast<float *>(slab_v), ld, rk);
    else
        slab_kernel_for<double>(model, scheme)<<<static_cast<unsigned>(blocks), kPathBlock, 0, s>>>(
            task, first_path, count, stride, static_cast<double *>(slab_S), static_cast<double *>(slab_v), ld, rk);
    return cudaGetLastError();
}

cudaError_t launch_step_trace(int precision, cudaStream_t s, const TaskDev *task, const double *z, const double *u,
                              int umax, int n, double *S_out, double *v_out, int *status) {
    if (precision == QK_FP32)
        step_trace_kernel<float><<<1, 1, 0, s>>>(task, z, u, umax, n, S_out, v_out, status);
    else
        step_trace_kernel<double><<<1, 1, 0, s>>>(task, z, u, umax, n, S_out, v_out, status);
    return cudaGetLastError();
}

cudaError_t launch_payoff_paths(int precision, cudaStream_t s, const TaskDev *task, int64_t first, int64_t count,
                                double *out) {
    const int64_t blocks = (count + kPathBlock - 1) / kPathBlock;
    if (precision == QK_FP32)
        payoff_paths_kernel<float><<<static_cast<unsigned>(blocks), kPathBlock, 0, s>>>(task, first, count, out);
    else
        payoff_paths_kernel<double><<<static_cast<unsigned>(blocks), kPathBlock, 0, s>>>(task, first, count, out);
    return cudaGetLastError();
}

cudaError_t launch_payoff_trace(int precision, cudaStream_t s, const PayoffSpec &ps, const double *S, int n, double S0,
                                double *out) {
    if (precision == QK_FP32)
        payoff_trace_kernel<float><<<1, 1, 0, s>>>(ps, S, n, S0, out);
    else
        payoff_trace_kernel<double><<<1, 1, 0, s>>>(ps, S, n, S0, out);
    return cudaGetLastError();
}

// SFU throughput probe: 8 independent chains x = 2^(-x) per thread (ex2.approx.ftz in
// hand-written PTX), so every iteration issues 8 MUFU.EX2 with no other dependency.
__global__ void __launch_bounds__(256) sfu_probe_kernel(float *sink, int iters) {
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = 0.001f * (threadIdx.x + 1) + 0.1f * k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(x[k]) : "f"(-x[k]));
    }
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += x[k];
    if (acc == 12345.0f) sink[threadIdx.x] = acc;  // keeps the chains live
}

cudaError_t launch_sfu_probe(cudaStream_t s, int sm_count, float *sink, cudaEvent_t e0, cudaEvent_t e1, float *ms,
                             double *ops) {
    const int blocks = sm_count * 8, threads = 256, iters = 4096;
    sfu_probe_kernel<<<blocks, threads, 0, s>>>(sink, 64);  // warm-up
    cudaEventRecord(e0, s);
    sfu_probe_kernel<<<blocks, threads, 0, s>>>(sink, iters);
    cudaEventRecord(e1, s);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) return e;
    e = cudaEventElapsedTime(ms, e0, e1);
    *ops = static_cast<double>(blocks) * threads * iters * 8.0;
    return e == cudaSuccess ? cudaGetLastError() : e;
}

// Loads the device code of every kernel in this file on the current device.
template <class R>
static cudaError_t preload_path_kernels_of() {
    cudaFuncAttributes fa;
    cudaError_t e = cudaSuccess;
    for (int model = 0; model < 2 && e == cudaSuccess; ++model)
        for (int scheme = 0; scheme < 3 && e == cudaSuccess; ++scheme) {
            for (int uk = 0; uk < 2 && e == cudaSuccess; ++uk)
                for (int lane = 0; lane < 3 && e == cudaSuccess; ++lane)
                    for (int trk = 0; trk < 2 && e == cudaSuccess; ++trk)
                        e = cudaFuncGetAttributes(&fa, price_kernel_for<R>(model, scheme, uk != 0, lane, trk != 0));
            if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, slab_kernel_for<R>(model, scheme));
            if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, slab_two_kernel_for<R>(model, scheme));
        }
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, payoff_paths_kernel<R>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, payoff_trace_kernel<R>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, step_trace_kernel<R>);
    return e;
}

cudaError_t preload_path_kernels() {
    cudaFuncAttributes fa;
    cudaError_t e = preload_path_kernels_of<float>();
    if (e == cudaSuccess) e = preload_path_kernels_of<double>();
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, merge_tasks_kernel);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, merge_chunks_kernel);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, merge_task_chunks_kernel);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, sfu_probe_kernel);
    return e;
}

cudaError_t preload_noalloc_kernels() {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, merge_tasks_kernel);
    for (int model = 0; model < 2 && e == cudaSuccess; ++model)
        for (int scheme = 0; scheme < 3 && e == cudaSuccess; ++scheme)
            for (int trk = 0; trk < 2 && e == cudaSuccess; ++trk) {
                e = cudaFuncGetAttributes(&fa, price_kernel_for<float>(model, scheme, true, kLaneOne, trk != 0));
                if (e == cudaSuccess)
                    e = cudaFuncGetAttributes(&fa, price_kernel_for<double>(model, scheme, true, kLaneOne, trk != 0));
            }
    return e;
}

int price_tiles_max_blocks_per_sm(int precision, int model, int scheme, int lane_mode, bool track, int block) {
    // answered once per device, kernel variant and block size on each host thread
    // (planning asks for every contract of every call)
    constexpr int kDevs = 16, kVariants = 2 * 2 * 3 * 3 * 2 * 3;
    static thread_local int cache[kDevs][kVariants] = {};
    int dev = 0;
    const int bidx = block == 128 ? 0 : (block == 256 ? 1 : (block == 512 ? 2 : -1));
    int *slot = nullptr;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < kDevs && bidx >= 0 && precision >= 0 &&
        precision < 2 && model >= 0 && model < 2 && scheme >= 0 && scheme < 3 && lane_mode >= 0 && lane_mode < 3) {
        slot = &cache[dev][((((precision * 2 + model) * 3 + scheme) * 3 + lane_mode) * 2 + (track ? 1 : 0)) * 3 + bidx];
        if (*slot > 0) return *slot;
    }
    int nb = 0;
    if (precision == QK_FP32)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &nb, price_kernel_for<float>(model, scheme, true, lane_mode, track), block, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &nb, price_kernel_for<double>(model, scheme, true, lane_mode, track), block, 0);
    if (nb > 0 && slot) *slot = nb;
    return nb > 0 ? nb : 1;
}

}  // namespace qk
