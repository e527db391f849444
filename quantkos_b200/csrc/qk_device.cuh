// Device building blocks of the Monte Carlo hot path (sm_100a).
//
//   * Philox4x32-10 counter-based generator and the fixed draw layout that makes
//     every path reproducible whatever the launch shape;
//   * the Heston / Bates step functions under Euler, implicit Milstein and
//     Andersen QE, written once, templated on the arithmetic type and on the
//     draw source (Philox in the pricing kernels, fed draws in the parity trace);
//   * payoff trackers and final payoffs for the ten forward option types;
//   * FP64 statistics helpers (Welford / Chan merge).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "qk_internal.h"

namespace qk {

// ============================================================================
// Philox4x32-10 (J. Salmon, M. Moraes, R. Dror, D. Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies
// with a Weyl-sequence key schedule.  Counter = (block, path, stream, domain),
// key = (lo32(seed), hi32(seed)).
// ============================================================================
struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        // one 32x32 -> 64-bit multiply per product (IMAD.WIDE.U32)
        const uint64_t p0 = static_cast<uint64_t>(kPhiloxM0) * c.x;
        const uint64_t p1 = static_cast<uint64_t>(kPhiloxM1) * c.z;
        const uint32_t lo0 = static_cast<uint32_t>(p0), hi0 = static_cast<uint32_t>(p0 >> 32);
        const uint32_t lo1 = static_cast<uint32_t>(p1), hi1 = static_cast<uint32_t>(p1 >> 32);
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
    }
    return c;
}

// Round keys k_r = (k0 + r W0, k1 + r W1), r = 0..9, precomputed on the host and
// passed by value as a kernel parameter: the XORs then read them straight from
// the parameter bank, with no key arithmetic per round.
struct PhiloxRoundKeys {
    uint32_t k[20];
};

inline PhiloxRoundKeys philox_round_keys(uint32_t k0, uint32_t k1) {
    PhiloxRoundKeys rk;
    for (int r = 0; r < 10; ++r) {
        rk.k[2 * r] = k0 + static_cast<uint32_t>(r) * kPhiloxW0;
        rk.k[2 * r + 1] = k1 + static_cast<uint32_t>(r) * kPhiloxW1;
    }
    return rk;
}

__device__ __forceinline__ U4 philox4x32_10(U4 c, const PhiloxRoundKeys &rk) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(kPhiloxM0) * c.x;
        const uint64_t p1 = static_cast<uint64_t>(kPhiloxM1) * c.z;
        const uint32_t lo0 = static_cast<uint32_t>(p0), hi0 = static_cast<uint32_t>(p0 >> 32);
        const uint32_t lo1 = static_cast<uint32_t>(p1), hi1 = static_cast<uint32_t>(p1 >> 32);
        c = U4{hi1 ^ c.y ^ rk.k[2 * r], lo1, hi0 ^ c.w ^ rk.k[2 * r + 1], lo0};
    }
    return c;
}

// ============================================================================
// Arithmetic policy.  FP32 uses the SFU (MUFU) approximations explicitly;
// FP64 uses the correctly-rounded / IEEE CUDA library functions.
// ============================================================================
template <class R>
struct Math;

// Single SFU instructions (hand-written PTX): approximate base-2 exponential and
// logarithm, reciprocal and square root, flushing subnormals to zero.
__device__ __forceinline__ float ptx_ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ptx_lg2(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ptx_rcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ptx_sqrt(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

template <>
struct Math<float> {
    static constexpr float kLog2e = 1.44269504088896341f;
    static constexpr float kLn2 = 0.693147180559945309f;
    static __device__ __forceinline__ float exp(float x) { return ptx_ex2(x * kLog2e); }
    static __device__ __forceinline__ float log(float x) { return ptx_lg2(x) * kLn2; }
    // arguments are >= 0 here (variances, moment ratios); sqrt.approx(0) = 0
    static __device__ __forceinline__ float sqrt(float x) { return ptx_sqrt(x); }
    static __device__ __forceinline__ float rcp(float x) { return ptx_rcp(x); }
    static __device__ __forceinline__ float div(float a, float b) { return a * ptx_rcp(b); }
    static __device__ __forceinline__ float erf(float x) { return erff(x); }
    // uniform in (0,1): (k + 1/2) / 2^23, k = top 23 bits of the word.  The float
    // 1 + k 2^-23 is built from its bits (k as the mantissa) and 1 - 2^-24 subtracted;
    // both are exact and so is the difference (2k + 1) 2^-24, so this equals
    // k * 2^-23 + 2^-24 bit for bit without an integer-to-float conversion.
    static __device__ __forceinline__ float u01(uint32_t w) {
        return __fsub_rn(__uint_as_float(0x3F800000u | (w >> 9)), 0.99999994039535522f);
    }
    static constexpr float kU01Offset = 0.99999994039535522f;  // 1 - 2^-24
    static constexpr float kTwoPi = 6.28318530717958648f;
    // Box-Muller pair: R = sqrt(-2 ln u1), angle = 2*pi*(u2 - 1/2); IEEE-rounded
    // operations in a fixed order (box_muller_two repeats them on pairs)
    static __device__ __forceinline__ void box_muller(uint32_t w1, uint32_t w2, float &z1, float &z2) {
        const float u1 = u01(w1);
        const float u2 = u01(w2);
        const float rad = ptx_sqrt(__fmul_rn(-2.0f * kLn2, ptx_lg2(u1)));
        float s, c;
        __sincosf(__fmul_rn(kTwoPi, __fadd_rn(u2, -0.5f)), &s, &c);
        z1 = __fmul_rn(rad, c);
        z2 = __fmul_rn(rad, s);
    }
    // Two independent Box-Muller pairs, (a1, a2) and (b1, b2): the same operations as
    // box_muller with the FP32 multiplies and adds on the paired pipe, so each pair
    // gets the same bits as from box_muller.  z1 = (z1 of a, z1 of b), z2 likewise.
    static __device__ __forceinline__ void box_muller_two(uint32_t a1, uint32_t a2, uint32_t b1, uint32_t b2,
                                                          float2 &z1, float2 &z2) {
        const float2 off = make_float2(-kU01Offset, -kU01Offset);
        const float2 u1 = __fadd2_rn(make_float2(__uint_as_float(0x3F800000u | (a1 >> 9)),
                                                 __uint_as_float(0x3F800000u | (b1 >> 9))), off);
        const float2 u2 = __fadd2_rn(make_float2(__uint_as_float(0x3F800000u | (a2 >> 9)),
                                                 __uint_as_float(0x3F800000u | (b2 >> 9))), off);
        const float2 t = __fmul2_rn(make_float2(-2.0f * kLn2, -2.0f * kLn2),
                                    make_float2(ptx_lg2(u1.x), ptx_lg2(u1.y)));
        const float2 rad = make_float2(ptx_sqrt(t.x), ptx_sqrt(t.y));
        const float2 ang = __fmul2_rn(make_float2(kTwoPi, kTwoPi), __fadd2_rn(u2, make_float2(-0.5f, -0.5f)));
        float sa, ca, sb, cb;
        __sincosf(ang.x, &sa, &ca);
        __sincosf(ang.y, &sb, &cb);
        z1 = __fmul2_rn(rad, make_float2(ca, cb));
        z2 = __fmul2_rn(rad, make_float2(sa, sb));
    }
};

template <>
struct Math<double> {
    static __device__ __forceinline__ double exp(double x) { return ::exp(x); }
    static __device__ __forceinline__ double log(double x) { return ::log(x); }
    static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
    static __device__ __forceinline__ double div(double a, double b) { return a / b; }
    static __device__ __forceinline__ double erf(double x) { return ::erf(x); }
    static __device__ __forceinline__ double u01(uint32_t w) {
        return (static_cast<double>(w) + 0.5) * (1.0 / 4294967296.0);
    }
    static __device__ __forceinline__ void box_muller(uint32_t w1, uint32_t w2, double &z1, double &z2) {
        const double u1 = u01(w1);
        const double u2 = u01(w2);
        const double rad = ::sqrt(-2.0 * ::log(u1));
        double s, c;
        ::sincospi(2.0 * u2 - 1.0, &s, &c);
        z1 = rad * c;
        z2 = rad * s;
    }
};

template <class R>
__device__ __forceinline__ R rmax(R a, R b) { return fmax(a, b); }
template <class R>
__device__ __forceinline__ R rmin(R a, R b) { return fmin(a, b); }

// ============================================================================
// Draw sources.  A step asks for: one normal pair (Z1, Z2); Bates steps then ask
// for Poisson uniforms one at a time and, when a jump occurred, one jump normal.
//
// Philox layout per path p of stream s (counter = (block, p, s, domain)):
//   normal pair of step n:        domain 0, block floor(n/2), words (x,y) if n even, (z,w) if odd;
//   1st Poisson uniform of step n: FP64 domain 2, block floor(n/4), word n mod 4;
//                                  FP32 23 bits: the low 9 bits of each of the step's two
//                                  normal words (18 bits), then the top 5 bits of that
//                                  domain-2 word, drawn only when the first 18 cannot
//                                  decide the jump test;
//   jump normal of step n:         domain 1, block n, Box-Muller of words (x,y), first output;
//   Poisson uniforms 2, 3:         domain 1, block n, words z, w;
//   Poisson uniform k >= 4:        domain 3 + (k-4)/4, block n, word (k-4) mod 4.
// A step costs half a Philox block for the normals and, under Bates in FP64, a
// quarter block for the jump test (in FP32 nearly nothing); the rest is drawn only
// on the rare steps with a jump.
// ============================================================================
template <class R>
struct PhiloxJumpDraws {
    uint32_t k0, k1, path, stream, step;
    R first;    // the step's first Poisson uniform
    int used;   // Poisson uniforms consumed so far in this step
    int domain; // block currently held in wx (0 = none)
    U4 wx;

    __device__ __forceinline__ U4 block(uint32_t d) {
        return philox4x32_10(U4{step, path, stream, d}, k0, k1);
    }
    __device__ __forceinline__ R uniform() {
        const int k = used++;
        if (k == 0) return first;
        const int d = (k < 3) ? 1 : 3 + (k - 3) / 4;
        if (domain != d) {
            wx = block(static_cast<uint32_t>(d));
            domain = d;
        }
        const int slot = (k < 3) ? k + 1 : ((k - 3) & 3);
        const uint32_t word = slot == 0 ? wx.x : (slot == 1 ? wx.y : (slot == 2 ? wx.z : wx.w));
        return Math<R>::u01(word);
    }
    __device__ __forceinline__ R jump_normal() {
        const U4 j = block(1u);
        R z1, z2;
        Math<R>::box_muller(j.x, j.y, z1, z2);
        return z1;
    }
};

// Fed draws for the parity trace: z[3] = {Z1, Z2, Zjump}; u[umax] Poisson uniforms.
template <class R>
struct FedStep {
    const double *z;
    const double *u;
    int umax;
    int used;
    int overflow;
    __device__ __forceinline__ void normal_pair(R &z1, R &z2) {
        z1 = static_cast<R>(z[0]);
        z2 = static_cast<R>(z[1]);
    }
    __device__ __forceinline__ R uniform() {
        if (used >= umax) {
            overflow = 1;
            return R(0);
        }
        return static_cast<R>(u[used++]);
    }
    __device__ __forceinline__ R jump_normal() { return static_cast<R>(z[2]); }
};

// ============================================================================
// Scheme steps.  Each follows the reference's evolve_step line for line; the
// only rewrite is QE's quadratic-branch martingale term, where
// log(exp(X)/sqrt(t)) is evaluated as X - log(t)/2 (the same quantity without
// an exp/rsqrt/log round trip).
// ============================================================================

// Heston + Euler: include/core/schemes/markovian/MSchemes.hpp:133-156
template <class R>
__device__ __forceinline__ void step_euler(const StepConst<R> &p, R &S, R &v, R Z1, R Z2) {
    const R Zv = Z1;
    const R ZS = p.rho * Z1 + p.rho_c * Z2;
    const R sqv = Math<R>::sqrt(v);
    const R ex = p.r_minus_q_dt - v * p.half_dt + (sqv * p.sqrt_dt) * ZS;
    const R Sn = S * Math<R>::exp(ex);
    const R vn = v * p.one_minus_k_dt + p.k_theta_dt + (p.sigma_sqrt_dt * sqv) * Zv;
    S = Sn;
    v = rmax(vn, R(0));
}

// Heston + implicit Milstein: MSchemes.hpp:229-253
template <class R>
__device__ __forceinline__ void step_milstein(const StepConst<R> &p, R &S, R &v, R Z1, R Z2) {
    const R Zv = Z1;
    const R ZS = p.rho * Z1 + p.rho_c * Z2;
    const R sqv = Math<R>::sqrt(v);
    const R ex = p.r_minus_q_dt - v * p.half_dt + (sqv * p.sqrt_dt) * ZS;
    const R Sn = S * Math<R>::exp(ex);
    const R corr = p.quarter_sigma_sq_dt * (Zv * Zv - R(1));
    const R vn = p.implicit_den * (v + p.k_theta_dt + (p.sigma_sqrt_dt * sqv) * Zv + corr);
    S = Sn;
    v = rmax(vn, R(0));
}

// Heston + Andersen QE with martingale correction: MSchemes.hpp:363-442
template <class R>
__device__ __forceinline__ void step_qe(const StepConst<R> &p, R &S, R &v, R Zv, R Zind) {
    const R m = v * p.exp_mkdt + p.theta_m;
    const R s2 = v * p.s2f1 + p.s2f2;
    R vn;
    R logM;  // log of the martingale factor M
    if (m <= p.eps) {
        vn = R(0);
        logM = R(0);
    } else {
        // psi = s2 / m^2 is compared as s2 against eps m^2 and psi_c m^2 (m > 0)
        const R m2 = m * m;
        if (s2 <= p.eps * m2) {
            vn = m;
            logM = R(0);
        } else if (s2 <= p.psi_c * m2) {
            const R two_ip = R(2) * m2 * Math<R>::rcp(s2);  // 2 / psi
            const R b2 = two_ip - R(1) + Math<R>::sqrt(two_ip * (two_ip - R(1)));
            const R a = m * Math<R>::rcp(R(1) + b2);
            const R bz = Math<R>::sqrt(b2) + Zv;
            vn = a * bz * bz;
            // min(A, 0.5/a - eps) enters only through its product with a > 0:
            // safe_A a = min(A a, 0.5 - eps a)
            const R Aa = rmin(p.A * a, R(0.5) - p.eps * a);
            const R term = R(1) - R(2) * Aa;
            // M = exp(A b2 a / term) / sqrt(term)  =>  log M = A b2 a / term - log(term) / 2
            logM = Aa * b2 * Math<R>::rcp(term) - R(0.5) * Math<R>::log(term);
        } else {
            const R inv_m = Math<R>::rcp(m);
            const R psi = s2 * inv_m * inv_m;
            const R pz = Math<R>::div(psi - R(1), psi + R(1));
            const R beta = (R(1) - pz) * inv_m;
            const R U = R(0.5) * (R(1) + Math<R>::erf(Zv * p.inv_sqrt2));
            if (U <= pz) {
                vn = R(0);
            } else {
                const R safe_U = rmin(U, R(1) - p.eps);
                vn = Math<R>::div(Math<R>::log(Math<R>::div(R(1) - pz, R(1) - safe_U)), beta);
            }
            const R safe_A = rmin(p.A, beta - p.eps);
            const R M = pz + Math<R>::div(beta * (R(1) - pz), beta - safe_A);
            logM = Math<R>::log(M);
        }
    }
    const R K0 = -logM - p.K1_half_K3 * v;
    const R isig = p.K3 * v + p.K4 * vn;
    const R ex = p.r_minus_q_dt + K0 + (p.K1 * v + p.K2 * vn) + Math<R>::sqrt(isig) * Zind;
    S = S * Math<R>::exp(ex);
    v = vn;
}

// ----------------------------------------------------------------------------
// FP32 QE and Euler with an explicit rounding order.  Every FP32 operation below
// is an IEEE-rounded intrinsic (no compiler contraction), and the paired two-path
// forms further down perform the same operations on float2 pairs with the sm_100
// paired FP32 instructions, so one path gives the same bits whichever form
// simulates it.  Same algebra as the generic steps above.
__device__ __forceinline__ void qe_quadratic_f32(const StepConst<float> &p, float m, float m2, float s2, float Zv,
                                                 float &vn, float &logM) {
    const float two_ip = __fmul_rn(__fmul_rn(2.0f, m2), ptx_rcp(s2));
    const float t1 = __fadd_rn(two_ip, -1.0f);
    const float b2 = __fadd_rn(t1, ptx_sqrt(__fmul_rn(two_ip, t1)));
    const float a = __fmul_rn(m, ptx_rcp(__fadd_rn(1.0f, b2)));
    const float bz = __fadd_rn(ptx_sqrt(b2), Zv);
    vn = __fmul_rn(__fmul_rn(a, bz), bz);
    const float Aa = fminf(__fmul_rn(p.A, a), __fmaf_rn(-p.eps, a, 0.5f));
    const float term = __fmaf_rn(-2.0f, Aa, 1.0f);
    logM = __fmaf_rn(__fmul_rn(Aa, b2), ptx_rcp(term), __fmul_rn(-0.5f * Math<float>::kLn2, ptx_lg2(term)));
}

__device__ __forceinline__ void qe_spot_f32(const StepConst<float> &p, float &S, float v, float vn, float logM,
                                            float Zind) {
    const float K0n = __fmaf_rn(p.K1_half_K3, v, logM);  // -K0
    const float isig = __fmaf_rn(p.K3, v, __fmul_rn(p.K4, vn));
    const float e12 = __fadd_rn(__fadd_rn(p.r_minus_q_dt, -K0n), __fmaf_rn(p.K1, v, __fmul_rn(p.K2, vn)));
    const float ex = __fmaf_rn(ptx_sqrt(isig), Zind, e12);
    S = __fmul_rn(S, ptx_ex2(__fmul_rn(ex, Math<float>::kLog2e)));
}

template <>
__device__ __forceinline__ void step_qe<float>(const StepConst<float> &p, float &S, float &v, float Zv, float Zind) {
    const float m = __fmaf_rn(v, p.exp_mkdt, p.theta_m);
    const float s2 = __fmaf_rn(v, p.s2f1, p.s2f2);
    const float m2 = __fmul_rn(m, m);
    // the quadratic regime unconditionally (the common case, no branch before its
    // SFU chain); the other regimes overwrite its result
    float vn, logM;
    qe_quadratic_f32(p, m, m2, s2, Zv, vn, logM);
    if (m <= p.eps) {
        vn = 0.0f;
        logM = 0.0f;
    } else if (s2 <= __fmul_rn(p.eps, m2)) {
        vn = m;
        logM = 0.0f;
    } else if (!(s2 <= __fmul_rn(p.psi_c, m2))) {
        // exponential branch (rare at the usual parameters): as the generic step
        const float inv_m = ptx_rcp(m);
        const float psi = s2 * inv_m * inv_m;
        const float pz = Math<float>::div(psi - 1.0f, psi + 1.0f);
        const float beta = (1.0f - pz) * inv_m;
        const float U = 0.5f * (1.0f + erff(Zv * p.inv_sqrt2));
        if (U <= pz) {
            vn = 0.0f;
        } else {
            const float safe_U = fminf(U, 1.0f - p.eps);
            vn = Math<float>::div(Math<float>::log(Math<float>::div(1.0f - pz, 1.0f - safe_U)), beta);
        }
        const float safe_A = fminf(p.A, beta - p.eps);
        const float M = pz + Math<float>::div(beta * (1.0f - pz), beta - safe_A);
        logM = Math<float>::log(M);
    }
    qe_spot_f32(p, S, v, vn, logM, Zind);
    v = vn;
}

template <>
__device__ __forceinline__ void step_euler<float>(const StepConst<float> &p, float &S, float &v, float Z1, float Z2) {
    const float ZS = __fmaf_rn(p.rho, Z1, __fmul_rn(p.rho_c, Z2));
    const float sqv = ptx_sqrt(v);
    const float ex = __fmaf_rn(__fmul_rn(sqv, p.sqrt_dt), ZS, __fmaf_rn(v, -p.half_dt, p.r_minus_q_dt));
    S = __fmul_rn(S, ptx_ex2(__fmul_rn(ex, Math<float>::kLog2e)));
    v = fmaxf(__fmaf_rn(__fmul_rn(p.sigma_sqrt_dt, sqv), Z1, __fmaf_rn(v, p.one_minus_k_dt, p.k_theta_dt)), 0.0f);
}

// Implicit Milstein variance update with an explicit rounding order.
__device__ __forceinline__ float milstein_variance_f32(const StepConst<float> &p, float v, float sqv, float Z1) {
    const float corr = __fmul_rn(p.quarter_sigma_sq_dt, __fmaf_rn(Z1, Z1, -1.0f));
    const float t = __fadd_rn(__fmaf_rn(__fmul_rn(p.sigma_sqrt_dt, sqv), Z1, __fadd_rn(v, p.k_theta_dt)), corr);
    return fmaxf(__fmul_rn(p.implicit_den, t), 0.0f);
}

template <>
__device__ __forceinline__ void step_milstein<float>(const StepConst<float> &p, float &S, float &v, float Z1,
                                                     float Z2) {
    const float ZS = __fmaf_rn(p.rho, Z1, __fmul_rn(p.rho_c, Z2));
    const float sqv = ptx_sqrt(v);
    const float ex = __fmaf_rn(__fmul_rn(sqv, p.sqrt_dt), ZS, __fmaf_rn(v, -p.half_dt, p.r_minus_q_dt));
    S = __fmul_rn(S, ptx_ex2(__fmul_rn(ex, Math<float>::kLog2e)));
    v = milstein_variance_f32(p, v, sqv, Z1);
}

// Paired FP32: component-wise IEEE operations on two paths at once.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 rcp2(float2 x) { return make_float2(ptx_rcp(x.x), ptx_rcp(x.y)); }
__device__ __forceinline__ float2 sqrt2(float2 x) { return make_float2(ptx_sqrt(x.x), ptx_sqrt(x.y)); }
__device__ __forceinline__ float2 lg2_2(float2 x) { return make_float2(ptx_lg2(x.x), ptx_lg2(x.y)); }
__device__ __forceinline__ float2 ex2_2(float2 x) { return make_float2(ptx_ex2(x.x), ptx_ex2(x.y)); }
__device__ __forceinline__ float2 min2(float2 a, float2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
__device__ __forceinline__ float2 max0_2(float2 a) { return make_float2(fmaxf(a.x, 0.0f), fmaxf(a.y, 0.0f)); }

// QE step of two paths (spot S, variance v as pairs): paired when both take the
// quadratic branch (the common case), otherwise each path through step_qe<float>.
__device__ __forceinline__ void step_qe_two_f32(const StepConst<float> &p, float2 &S, float2 &v, float2 Zv,
                                                float2 Zind) {
    const float2 m = __ffma2_rn(v, f2(p.exp_mkdt), f2(p.theta_m));
    const float2 s2 = __ffma2_rn(v, f2(p.s2f1), f2(p.s2f2));
    const float2 m2 = __fmul2_rn(m, m);
    const float2 em2 = __fmul2_rn(f2(p.eps), m2);
    const float2 pm2 = __fmul2_rn(f2(p.psi_c), m2);
    const bool quad = m.x > p.eps && m.y > p.eps && s2.x > em2.x && s2.y > em2.y && s2.x <= pm2.x && s2.y <= pm2.y;
    // the quadratic form for both paths first (no branch before the long SFU chain);
    // a pair not both in the quadratic regime is redone per path below
    const float2 S_old = S, v_old = v;
    // qe_quadratic_f32, paired
    const float2 two_ip = __fmul2_rn(__fmul2_rn(f2(2.0f), m2), rcp2(s2));
    const float2 t1 = __fadd2_rn(two_ip, f2(-1.0f));
    const float2 b2 = __fadd2_rn(t1, sqrt2(__fmul2_rn(two_ip, t1)));
    const float2 a = __fmul2_rn(m, rcp2(__fadd2_rn(f2(1.0f), b2)));
    const float2 bz = __fadd2_rn(sqrt2(b2), Zv);
    const float2 vn = __fmul2_rn(__fmul2_rn(a, bz), bz);
    const float2 Aa = min2(__fmul2_rn(f2(p.A), a), __ffma2_rn(f2(-p.eps), a, f2(0.5f)));
    const float2 term = __ffma2_rn(f2(-2.0f), Aa, f2(1.0f));
    const float2 logM = __ffma2_rn(__fmul2_rn(Aa, b2), rcp2(term),
                                   __fmul2_rn(f2(-0.5f * Math<float>::kLn2), lg2_2(term)));
    // qe_spot_f32, paired
    const float2 K0n = __ffma2_rn(f2(p.K1_half_K3), v, logM);
    const float2 isig = __ffma2_rn(f2(p.K3), v, __fmul2_rn(f2(p.K4), vn));
    const float2 e12 = __fadd2_rn(__fadd2_rn(f2(p.r_minus_q_dt), __fmul2_rn(K0n, f2(-1.0f))),
                                  __ffma2_rn(f2(p.K1), v, __fmul2_rn(f2(p.K2), vn)));
    const float2 ex = __ffma2_rn(sqrt2(isig), Zind, e12);
    S = __fmul2_rn(S, ex2_2(__fmul2_rn(ex, f2(Math<float>::kLog2e))));
    v = vn;
    if (!quad) {
        // one copy of the one-path step for both paths (rare; keeps the loop body small)
        S = S_old;
        v = v_old;
#pragma unroll 1
        for (int i = 0; i < 2; ++i) {
            float Si = i ? S.y : S.x, vi = i ? v.y : v.x;
            step_qe<float>(p, Si, vi, i ? Zv.y : Zv.x, i ? Zind.y : Zind.x);
            if (i) {
                S.y = Si;
                v.y = vi;
            } else {
                S.x = Si;
                v.x = vi;
            }
        }
    }
}

// Milstein for two paths: the spot update (the same as Euler's) paired, the
// variance update per path.
__device__ __forceinline__ void step_milstein_two_f32(const StepConst<float> &p, float2 &S, float2 &v, float2 Z1,
                                                      float2 Z2) {
    const float2 ZS = __ffma2_rn(f2(p.rho), Z1, __fmul2_rn(f2(p.rho_c), Z2));
    const float2 sqv = sqrt2(v);
    const float2 ex = __ffma2_rn(__fmul2_rn(sqv, f2(p.sqrt_dt)), ZS, __ffma2_rn(v, f2(-p.half_dt), f2(p.r_minus_q_dt)));
    S = __fmul2_rn(S, ex2_2(__fmul2_rn(ex, f2(Math<float>::kLog2e))));
    v = make_float2(milstein_variance_f32(p, v.x, sqv.x, Z1.x), milstein_variance_f32(p, v.y, sqv.y, Z1.y));
}

__device__ __forceinline__ void step_euler_two_f32(const StepConst<float> &p, float2 &S, float2 &v, float2 Z1,
                                                   float2 Z2) {
    const float2 ZS = __ffma2_rn(f2(p.rho), Z1, __fmul2_rn(f2(p.rho_c), Z2));
    const float2 sqv = sqrt2(v);
    const float2 ex = __ffma2_rn(__fmul2_rn(sqv, f2(p.sqrt_dt)), ZS, __ffma2_rn(v, f2(-p.half_dt), f2(p.r_minus_q_dt)));
    S = __fmul2_rn(S, ex2_2(__fmul2_rn(ex, f2(Math<float>::kLog2e))));
    v = max0_2(__ffma2_rn(__fmul2_rn(f2(p.sigma_sqrt_dt), sqv), Z1,
                          __ffma2_rn(v, f2(p.one_minus_k_dt), f2(p.k_theta_dt))));
}

template <class R, int SCHEME>
__device__ __forceinline__ void heston_step(const StepConst<R> &p, R &S, R &v, R Z1, R Z2) {
    if constexpr (SCHEME == kEuler) {
        step_euler<R>(p, S, v, Z1, Z2);
    } else if constexpr (SCHEME == kMilstein) {
        step_milstein<R>(p, S, v, Z1, Z2);
    } else {
        step_qe<R>(p, S, v, Z1, Z2);
    }
}

// Bates jump part after the (drift-compensated) Heston step: MSchemes.hpp:493-526.
// Knuth's Poisson draw: multiply uniforms until the product drops below exp(-lambda dt).
// `prod` holds the first uniform, already known to be >= exp(-lambda dt) (a jump).
template <class R, class Draws>
__device__ __noinline__ R jump_factor(const StepConst<R> &p, R prod, Draws &d) {
    int N = 0;
    do {
        ++N;
        prod *= d.uniform();
    } while (prod >= p.exp_m_lambda_dt && N < kMaxJumpsPerStep);
    const R Z = d.jump_normal();
    const R rN = static_cast<R>(N);
    return Math<R>::exp(rN * p.mu_j + Math<R>::sqrt(rN) * p.sigma_j * Z);
}

// Both members of an antithetic pair: the same jump count, jump sizes with the
// normal of opposite sign.
template <class R, class Draws>
__device__ __noinline__ void jump_factor_pair(const StepConst<R> &p, R prod, Draws &d, R &fa, R &fb) {
    int N = 0;
    do {
        ++N;
        prod *= d.uniform();
    } while (prod >= p.exp_m_lambda_dt && N < kMaxJumpsPerStep);
    const R Z = d.jump_normal();
    const R rN = static_cast<R>(N);
    const R m = rN * p.mu_j;
    const R s = Math<R>::sqrt(rN) * p.sigma_j * Z;
    fa = Math<R>::exp(m + s);
    fb = Math<R>::exp(m - s);
}

template <class R, class Draws>
__device__ __forceinline__ void bates_jump(const StepConst<R> &p, R &S, Draws &d) {
    const R first = d.uniform();
    if (first >= p.exp_m_lambda_dt) S *= jump_factor<R>(p, first, d);
}

template <class R, int MODEL, int SCHEME, class Draws>
__device__ __forceinline__ void evolve_step(const StepConst<R> &p, R &S, R &v, Draws &d) {
    R Z1, Z2;
    d.normal_pair(Z1, Z2);
    heston_step<R, SCHEME>(p, S, v, Z1, Z2);
    if constexpr (MODEL == kBates) bates_jump<R>(p, S, d);
}

// ============================================================================
// Payoffs: include/core/options/Payoff.hpp:35-243.  Trackers (running sum in
// double, running max / min started at S0) are kept for every path; the final
// payoff per requested contract leg reads the ones it needs.
// ============================================================================
template <class R>
__device__ __forceinline__ R intrinsic(int right, R S, R K) {
    return right == kCall ? (S > K ? S - K : R(0)) : (K > S ? K - S : R(0));
}

template <class R>
__device__ __forceinline__ R final_payoff(const PayoffSpec &ps, R S, double ssum, R smax, R smin, int n_steps) {
    const R K = static_cast<R>(ps.K);
    const R B = static_cast<R>(ps.B);
    switch (ps.type) {
        case kEuropean: return intrinsic<R>(ps.right, S, K);
        case kAsian: return intrinsic<R>(ps.right, static_cast<R>(ssum / static_cast<double>(n_steps)), K);
        case kBarrierUpOut: return smax < B ? intrinsic<R>(ps.right, S, K) : R(0);
        case kBarrierDownOut: return smin > B ? intrinsic<R>(ps.right, S, K) : R(0);
        case kBarrierUpIn: return smax >= B ? intrinsic<R>(ps.right, S, K) : R(0);
        case kBarrierDownIn: return smin <= B ? intrinsic<R>(ps.right, S, K) : R(0);
        case kLookbackFloating:
            return ps.right == kCall ? intrinsic<R>(kCall, S, smin) : intrinsic<R>(kPut, S, smax);
        case kLookbackFixed:
            return ps.right == kCall ? intrinsic<R>(kCall, smax, K) : intrinsic<R>(kPut, smin, K);
        case kBinaryCash:
            return ps.right == kCall ? (S > K ? R(1) : R(0)) : (S < K ? R(1) : R(0));
        case kBinaryAsset:
            return ps.right == kCall ? (S > K ? S : R(0)) : (S < K ? S : R(0));
        default: return intrinsic<R>(ps.right, S, K);  // American legs priced at maturity only here
    }
}

// ============================================================================
// FP64 statistics: (n, mean, M2) merged with Chan et al.'s parallel update.
// ============================================================================
__device__ __forceinline__ Moments chan_merge(const Moments &a, const Moments &b) {
    const double n = a.n + b.n;
    if (n <= 0.0) return Moments{0.0, 0.0, 0.0, 0.0};
    if (a.n <= 0.0) return b;
    if (b.n <= 0.0) return a;
    const double d = b.mean - a.mean;
    Moments r;
    r.n = n;
    r.mean = a.mean + d * (b.n / n);
    r.m2 = a.m2 + b.m2 + d * d * (a.n * b.n / n);
    r.itm = a.itm + b.itm;
    return r;
}

__device__ __forceinline__ Moments shfl_down_moments(const Moments &m, int off) {
    Moments r;
    r.n = __shfl_down_sync(0xffffffffu, m.n, off);
    r.mean = __shfl_down_sync(0xffffffffu, m.mean, off);
    r.m2 = __shfl_down_sync(0xffffffffu, m.m2, off);
    r.itm = __shfl_down_sync(0xffffffffu, m.itm, off);
    return r;
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    return x;
}

// Exact two-pass moments of the 32 values of a warp (inactive lanes excluded):
// the values are in registers, so the second pass costs one more shuffle tree.
__device__ __forceinline__ Moments warp_moments(double x, bool active, bool itm) {
    const unsigned act = __ballot_sync(0xffffffffu, active);
    const unsigned im = __ballot_sync(0xffffffffu, active && itm);
    const double n = static_cast<double>(__popc(act));
    const double s = warp_sum(active ? x : 0.0);
    const double mean = n > 0.0 ? s / n : 0.0;
    const double dv = active ? x - mean : 0.0;
    const double m2 = warp_sum(dv * dv);
    return Moments{n, mean, m2, static_cast<double>(__popc(im))};
}

// Moments of the 32 pair averages of a warp (antithetic sampling): each lane's
// value is (x_a + x_b) / 2 and its in-the-money weight (1{a} + 1{b}) / 2.
__device__ __forceinline__ Moments warp_moments_pair(double y, bool active, bool itm_a, bool itm_b) {
    const unsigned act = __ballot_sync(0xffffffffu, active);
    const unsigned ia = __ballot_sync(0xffffffffu, active && itm_a);
    const unsigned ib = __ballot_sync(0xffffffffu, active && itm_b);
    const double n = static_cast<double>(__popc(act));
    const double s = warp_sum(active ? y : 0.0);
    const double mean = n > 0.0 ? s / n : 0.0;
    const double dv = active ? y - mean : 0.0;
    const double m2 = warp_sum(dv * dv);
    return Moments{n, mean, m2, 0.5 * static_cast<double>(__popc(ia) + __popc(ib))};
}

}  // namespace qk
