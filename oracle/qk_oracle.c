/*
 * qk_oracle.c — TEST INFRASTRUCTURE: CPU restatement of the QuantKos reference
 * algorithm for the Monte Carlo hot path, used only as the parity checker by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.  The engine
 * never loads it.
 *
 * It restates, in plain C (paths relative to the reference project):
 *   - the scheme invariants and steps of SDEScheme<M,S>
 *     (include/core/schemes/markovian/MSchemes.hpp:87-551), in double and in float;
 *   - the payoff trackers and final payoffs (include/core/options/Payoff.hpp:35-243);
 *   - the pricer statistics: mean, M2 about the mean, ITM count, discount and scale
 *     (include/core/options/OptionPricer.hpp:123-249, 323-332);
 *   - the finite-difference Greeks by full re-pricing
 *     (include/core/engine/MCEngine.hpp:576-735);
 *   - Longstaff-Schwartz backward induction (include/core/engine/ForwardBackwardMC.hpp:204-255,
 *     include/core/options/LSMAmerican.hpp:252-613) in the reference's Laguerre mode, plus
 *     the {1,S,S^2,S^3,v,Sv} regression mode solved in long double;
 *   - the Black-Scholes, Heston and Bates closed forms (include/core/analytical/*),
 *     with Gauss-Legendre nodes computed here by Newton iteration on P_64.
 * Random numbers: the reference draws from a Kokkos XorShift64 pool whose stream
 * cannot be reproduced (not vendored, schedule-dependent).  The oracle therefore
 * consumes the same Philox4x32-10 counters as the engine (Salmon et al., SC'11), so
 * GPU and CPU follow the same paths; the reference's own code is checked against this
 * file step by step with fed draws (oracle/ref_harness, tests/test_oracle_pins.py).
 *
 * Build: gcc -std=c11 -O2 -fPIC -shared -fopenmp -o oracle/libqkoracle.so oracle/qk_oracle.c -lm
 */
#define _DEFAULT_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/quantkos_b200.h"

/* ================================================================ Philox4x32-10 */
void qko_philox(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static void philox_block(uint32_t block, uint32_t path, uint32_t stream, uint32_t domain, uint32_t k0, uint32_t k1,
                         uint32_t w[4]) {
    const uint32_t c[4] = {block, path, stream, domain};
    const uint32_t k[2] = {k0, k1};
    qko_philox(c, k, w);
}

/* uniforms in (0,1): float (k + 1/2)/2^23 on the top 23 bits; double (w + 1/2)/2^32 */
static float u01f(uint32_t w) { return (float)(w >> 9) * (1.0f / 8388608.0f) + (1.0f / 16777216.0f); }
static double u01d(uint32_t w) { return ((double)w + 0.5) * (1.0 / 4294967296.0); }

/* Box-Muller: R = sqrt(-2 ln u1), angle 2 pi (u2 - 1/2) */
static void bm_d(uint32_t w1, uint32_t w2, double *z1, double *z2) {
    const double r = sqrt(-2.0 * log(u01d(w1)));
    const double a = 6.283185307179586476925 * (u01d(w2) - 0.5);
    *z1 = r * cos(a);
    *z2 = r * sin(a);
}
static void bm_f(uint32_t w1, uint32_t w2, float *z1, float *z2) {
    const float r = sqrtf(-2.0f * logf(u01f(w1)));
    const float a = 6.28318530717958648f * (u01f(w2) - 0.5f);
    *z1 = r * cosf(a);
    *z2 = r * sinf(a);
}

/* ================================================================ scheme invariants
 * Constructors of SDEScheme (MSchemes.hpp:102-123 Euler, 197-219 Milstein, 303-353 QE,
 * 480-487 Bates, 535-550 Bates drift compensator), computed in double. */
typedef struct {
    double r_minus_q_dt, half_dt, sqrt_dt, rho, rho_c;
    double one_minus_k_dt, k_theta_dt, sigma_sqrt_dt;
    double quarter_sigma_sq_dt, implicit_den;
    double eps, psi_c, inv_sqrt2, exp_mkdt, theta_m, s2f1, s2f2, K1, K2, K3, K4, A;
    double exp_m_lambda_dt, mu_j, sigma_j;
} Inv;

static Inv make_inv(const qk_contract *c, double dt, double eps) {
    Inv p;
    memset(&p, 0, sizeof(p));
    double q = c->q;
    if (c->model == QK_BATES) q += c->lambda_j * (exp(c->mu_j + 0.5 * c->sigma_j * c->sigma_j) - 1.0);
    const double k = c->kappa, th = c->theta, sg = c->sigma;
    double rho = c->rho;
    p.sqrt_dt = sqrt(dt);
    p.rho = rho;
    p.rho_c = sqrt(1.0 - rho * rho);
    p.one_minus_k_dt = 1.0 - k * dt;
    p.k_theta_dt = k * th * dt;
    p.sigma_sqrt_dt = sg * p.sqrt_dt;
    p.r_minus_q_dt = (c->r - q) * dt;
    p.half_dt = 0.5 * dt;
    p.quarter_sigma_sq_dt = 0.25 * sg * sg * dt;
    p.implicit_den = 1.0 / (1.0 + k * dt);
    p.eps = eps;
    p.psi_c = c->psi_c > 0.0 ? c->psi_c : 1.5;
    p.inv_sqrt2 = 1.0 / sqrt(2.0);
    p.exp_mkdt = exp(-k * dt);
    if (k < eps) {
        p.theta_m = 0.0;
        p.s2f1 = sg * sg * dt;
        p.s2f2 = 0.0;
    } else {
        const double ome = 1.0 - p.exp_mkdt;
        p.theta_m = th * ome;
        p.s2f1 = (sg * sg * p.exp_mkdt / k) * ome;
        p.s2f2 = (th * sg * sg / (2.0 * k)) * (ome * ome);
    }
    double rds;
    double rq = rho;
    if (sg < eps) { rds = 0.0; rq = 0.0; } else { rds = rho / sg; }
    const double om = 1.0 - rq * rq;
    const double K12 = k * rds - 0.5;
    p.K1 = dt * 0.5 * K12 - rds;
    p.K2 = dt * 0.5 * K12 + rds;
    p.K3 = dt * 0.5 * om;
    p.K4 = dt * 0.5 * om;
    p.A = p.K2 + p.K4 * 0.5;
    p.exp_m_lambda_dt = exp(-((c->model == QK_BATES) ? c->lambda_j * dt : 0.0));
    p.mu_j = c->mu_j;
    p.sigma_j = c->sigma_j;
    return p;
}

/* ================================================================ draw sources */
typedef struct {
    int fed;
    /* fed */
    const double *z, *u;
    int umax, used, overflow;
    /* philox */
    uint32_t k0, k1, path, stream, step;
    uint32_t w_first; /* word of the step's first Poisson uniform */
    uint32_t wx[4];
    int domain;
    int neg; /* antithetic member: the jump normal is negated */
} Draws;

static double draw_uniform_d(Draws *d, int as_float) {
    if (d->fed) {
        if (d->used >= d->umax) { d->overflow = 1; return 0.0; }
        return d->u[d->used++];
    }
    /* Philox layout of the Poisson uniforms of step n (engine's draw layout):
       1st: w_first (FP64 domain 2, block n/4, word n%4; FP32 see run_path_sign);
       2nd, 3rd: domain 1, block n, words z, w;
       k-th (k >= 4, 1-based): domain 3 + (k-4)/4, block n, word (k-4)%4. */
    const int k = d->used++;
    uint32_t word;
    if (k == 0) word = d->w_first;
    else {
        const int dom = (k < 3) ? 1 : 3 + (k - 3) / 4;
        if (d->domain != dom) { philox_block(d->step, d->path, d->stream, (uint32_t)dom, d->k0, d->k1, d->wx); d->domain = dom; }
        const int slot = (k < 3) ? k + 1 : ((k - 3) & 3);
        word = d->wx[slot];
    }
    return as_float ? (double)u01f(word) : u01d(word);
}

/* ================================================================ steps, double
 * MSchemes.hpp:133-156 (Euler), 229-253 (Milstein), 363-442 (QE), 493-526 (Bates). */
static void step_d(const Inv *p, int model, int scheme, double *S_io, double *v_io, double Z1, double Z2, Draws *d) {
    const double S = *S_io, v = *v_io;
    double Sn, vn;
    if (scheme == QK_EULER || scheme == QK_IMPLICIT_MILSTEIN) {
        const double ZS = p->rho * Z1 + p->rho_c * Z2;
        const double sv = sqrt(v);
        Sn = S * exp(p->r_minus_q_dt - (v * p->half_dt) + (sv * p->sqrt_dt) * ZS);
        if (scheme == QK_EULER) {
            vn = v * p->one_minus_k_dt + p->k_theta_dt + (p->sigma_sqrt_dt * sv) * Z1;
        } else {
            const double corr = p->quarter_sigma_sq_dt * (Z1 * Z1 - 1.0);
            vn = p->implicit_den * (v + p->k_theta_dt + (p->sigma_sqrt_dt * sv) * Z1 + corr);
        }
        vn = fmax(vn, 0.0);
    } else {
        const double m = v * p->exp_mkdt + p->theta_m;
        const double s2 = v * p->s2f1 + p->s2f2;
        double M;
        if (m <= p->eps) { vn = 0.0; M = 1.0; }
        else {
            const double psi = s2 / (m * m);
            if (psi <= p->eps) { vn = m; M = 1.0; }
            else if (psi <= p->psi_c) {
                const double ip = 1.0 / psi;
                const double b2 = 2.0 * ip - 1.0 + sqrt(2.0 * ip * (2.0 * ip - 1.0));
                const double a = m / (1.0 + b2);
                const double bz = sqrt(b2) + Z1;
                vn = a * bz * bz;
                const double sA = fmin(p->A, (0.5 / a) - p->eps);
                const double t = 1.0 - 2.0 * sA * a;
                M = exp((sA * b2 * a) / t) / sqrt(t);
            } else {
                const double pz = (psi - 1.0) / (psi + 1.0);
                const double beta = (1.0 - pz) / m;
                const double U = 0.5 * (1.0 + erf(Z1 * p->inv_sqrt2));
                if (U <= pz) vn = 0.0;
                else {
                    const double sU = fmin(U, 1.0 - p->eps);
                    vn = log((1.0 - pz) / (1.0 - sU)) / beta;
                }
                const double sA = fmin(p->A, beta - p->eps);
                M = pz + (beta * (1.0 - pz)) / (beta - sA);
            }
        }
        const double K0 = -log(M) - (p->K1 + p->K3 * 0.5) * v;
        const double isig = p->K3 * v + p->K4 * vn;
        Sn = S * exp(p->r_minus_q_dt + K0 + (p->K1 * v + p->K2 * vn) + sqrt(isig) * Z2);
    }
    if (model == QK_BATES) {
        int N = -1;
        double prod = 1.0;
        do { ++N; prod *= draw_uniform_d(d, 0); } while (prod >= p->exp_m_lambda_dt && N < 4096);
        if (N > 0) {
            double Z;
            if (d->fed) Z = d->z[2];
            else { uint32_t w[4]; double z2; philox_block(d->step, d->path, d->stream, 1u, d->k0, d->k1, w); bm_d(w[0], w[1], &Z, &z2); if (d->neg) Z = -Z; }
            Sn *= exp((double)N * p->mu_j + sqrt((double)N) * p->sigma_j * Z);
        }
    }
    *S_io = Sn;
    *v_io = vn;
}

/* ================================================================ steps, float (the reference's FP32 build) */
typedef struct {
    float r_minus_q_dt, half_dt, sqrt_dt, rho, rho_c, one_minus_k_dt, k_theta_dt, sigma_sqrt_dt;
    float quarter_sigma_sq_dt, implicit_den, eps, psi_c, inv_sqrt2, exp_mkdt, theta_m, s2f1, s2f2, K1, K2, K3, K4, A;
    float exp_m_lambda_dt, mu_j, sigma_j;
} InvF;

static InvF to_f(const Inv *p) {
    InvF f;
    f.r_minus_q_dt = (float)p->r_minus_q_dt; f.half_dt = (float)p->half_dt; f.sqrt_dt = (float)p->sqrt_dt;
    f.rho = (float)p->rho; f.rho_c = (float)p->rho_c; f.one_minus_k_dt = (float)p->one_minus_k_dt;
    f.k_theta_dt = (float)p->k_theta_dt; f.sigma_sqrt_dt = (float)p->sigma_sqrt_dt;
    f.quarter_sigma_sq_dt = (float)p->quarter_sigma_sq_dt; f.implicit_den = (float)p->implicit_den;
    f.eps = (float)p->eps; f.psi_c = (float)p->psi_c; f.inv_sqrt2 = (float)p->inv_sqrt2; f.exp_mkdt = (float)p->exp_mkdt;
    f.theta_m = (float)p->theta_m; f.s2f1 = (float)p->s2f1; f.s2f2 = (float)p->s2f2; f.K1 = (float)p->K1;
    f.K2 = (float)p->K2; f.K3 = (float)p->K3; f.K4 = (float)p->K4; f.A = (float)p->A;
    f.exp_m_lambda_dt = (float)p->exp_m_lambda_dt; f.mu_j = (float)p->mu_j; f.sigma_j = (float)p->sigma_j;
    return f;
}

static void step_f(const InvF *p, int model, int scheme, float *S_io, float *v_io, float Z1, float Z2, Draws *d) {
    const float S = *S_io, v = *v_io;
    float Sn, vn;
    if (scheme == QK_EULER || scheme == QK_IMPLICIT_MILSTEIN) {
        const float ZS = p->rho * Z1 + p->rho_c * Z2;
        const float sv = sqrtf(v);
        Sn = S * expf(p->r_minus_q_dt - (v * p->half_dt) + (sv * p->sqrt_dt) * ZS);
        if (scheme == QK_EULER) vn = v * p->one_minus_k_dt + p->k_theta_dt + (p->sigma_sqrt_dt * sv) * Z1;
        else vn = p->implicit_den * (v + p->k_theta_dt + (p->sigma_sqrt_dt * sv) * Z1 + p->quarter_sigma_sq_dt * (Z1 * Z1 - 1.0f));
        vn = fmaxf(vn, 0.0f);
    } else {
        const float m = v * p->exp_mkdt + p->theta_m;
        const float s2 = v * p->s2f1 + p->s2f2;
        float M;
        if (m <= p->eps) { vn = 0.0f; M = 1.0f; }
        else {
            const float psi = s2 / (m * m);
            if (psi <= p->eps) { vn = m; M = 1.0f; }
            else if (psi <= p->psi_c) {
                const float ip = 1.0f / psi;
                const float b2 = 2.0f * ip - 1.0f + sqrtf(2.0f * ip * (2.0f * ip - 1.0f));
                const float a = m / (1.0f + b2);
                const float bz = sqrtf(b2) + Z1;
                vn = a * bz * bz;
                const float sA = fminf(p->A, (0.5f / a) - p->eps);
                const float t = 1.0f - 2.0f * sA * a;
                M = expf((sA * b2 * a) / t) / sqrtf(t);
            } else {
                const float pz = (psi - 1.0f) / (psi + 1.0f);
                const float beta = (1.0f - pz) / m;
                const float U = 0.5f * (1.0f + erff(Z1 * p->inv_sqrt2));
                if (U <= pz) vn = 0.0f;
                else vn = logf((1.0f - pz) / (1.0f - fminf(U, 1.0f - p->eps))) / beta;
                const float sA = fminf(p->A, beta - p->eps);
                M = pz + (beta * (1.0f - pz)) / (beta - sA);
            }
        }
        const float K0 = -logf(M) - (p->K1 + p->K3 * 0.5f) * v;
        const float isig = p->K3 * v + p->K4 * vn;
        Sn = S * expf(p->r_minus_q_dt + K0 + (p->K1 * v + p->K2 * vn) + sqrtf(isig) * Z2);
    }
    if (model == QK_BATES) {
        int N = -1;
        float prod = 1.0f;
        do { ++N; prod *= (float)draw_uniform_d(d, 1); } while (prod >= p->exp_m_lambda_dt && N < 4096);
        if (N > 0) {
            float Z;
            if (d->fed) Z = (float)d->z[2];
            else { uint32_t w[4]; float z2; philox_block(d->step, d->path, d->stream, 1u, d->k0, d->k1, w); bm_f(w[0], w[1], &Z, &z2); if (d->neg) Z = -Z; }
            Sn *= expf((float)N * p->mu_j + sqrtf((float)N) * p->sigma_j * Z);
        }
    }
    *S_io = Sn;
    *v_io = vn;
}

/* ================================================================ fed-draw trace */
int qko_step_trace(int precision, const qk_contract *c, const double *z, const double *u, int umax, int n,
                   double *S_out, double *v_out) {
    const double dt = c->T / n;
    const Inv p = make_inv(c, dt, precision == QK_FP32 ? 1e-6 : 1e-12);
    const InvF pf = to_f(&p);
    double S = c->S0, v = c->v0;
    float Sf = (float)c->S0, vf = (float)c->v0;
    for (int i = 0; i < n; ++i) {
        Draws d;
        memset(&d, 0, sizeof(d));
        d.fed = 1;
        d.z = z + 3 * (size_t)i;
        d.u = u + (size_t)umax * i;
        d.umax = umax;
        if (precision == QK_FP32) {
            step_f(&pf, c->model, c->scheme, &Sf, &vf, (float)d.z[0], (float)d.z[1], &d);
            S_out[i] = Sf;
            v_out[i] = vf;
        } else {
            step_d(&p, c->model, c->scheme, &S, &v, d.z[0], d.z[1], &d);
            S_out[i] = S;
            v_out[i] = v;
        }
        if (d.overflow) return 3;
    }
    return 0;
}

/* ================================================================ one path with Philox draws
 * Mirrors MarkovianIntegrationKernel::operator() (MSolver.hpp:98-130). */
typedef struct {
    double S, v, ssum, smax, smin;
} PathOut;

static void normalise(const qk_contract *c, qk_contract *n, double *scale) {
    *n = *c;
    *scale = 1.0;
    if (c->normalize) {  /* UInputs::apply_price_scaling (Config.hpp:710-723) */
        *scale = c->S0;
        n->S0 = 1.0;
        for (int k = 0; k < c->n_payoffs; ++k) {
            n->payoffs[k].strike = c->payoffs[k].strike / c->S0;
            n->payoffs[k].barrier = c->payoffs[k].barrier / c->S0;
        }
    }
}

/* store: optional callback rows (every `stride` steps) into S_rows/v_rows[row*ld + col] */
/* neg: the antithetic member of pair `path` (every normal negated, uniforms shared) */
static void run_path_sign(const qk_contract *c, const Inv *p, const InvF *pf, uint32_t path, int neg, PathOut *o,
                          int stride, double *S_rows, double *v_rows, int64_t ld, int64_t col) {
    const uint32_t k0 = (uint32_t)(c->seed & 0xFFFFFFFFu), k1 = (uint32_t)(c->seed >> 32);
    const uint32_t stream = (uint32_t)c->stream;
    const int fp32 = c->precision == QK_FP32;
    double S = c->S0, v = c->v0;
    float Sf = (float)c->S0, vf = (float)c->v0;
    double ssum = 0.0, smax = fp32 ? (double)Sf : S, smin = smax;
    float smaxf = Sf, sminf = Sf;
    uint32_t w[4] = {0, 0, 0, 0}, wp[4] = {0, 0, 0, 0};
    for (int n = 0; n < c->n_steps; ++n) {
        Draws d;
        memset(&d, 0, sizeof(d));
        d.k0 = k0; d.k1 = k1; d.path = path; d.stream = stream; d.step = (uint32_t)n;
        d.neg = neg;
        /* normal pair of step n: domain 0, block n/2, words (x,y) for even n, (z,w) for odd n */
        if ((n & 1) == 0) philox_block((uint32_t)(n >> 1), path, stream, 0u, k0, k1, w);
        const uint32_t wa = (n & 1) ? w[2] : w[0];
        const uint32_t wb = (n & 1) ? w[3] : w[1];
        if (c->model == QK_BATES) {
            if ((n & 3) == 0) philox_block((uint32_t)(n >> 2), path, stream, 2u, k0, k1, wp);
            if (fp32) {
                /* FP32: 23-bit uniform from the low 9 bits of the two normal words and the
                   top 5 bits of the domain-2 word (the engine fetches that word only when
                   the first 18 bits cannot decide the jump test) */
                const uint32_t hi = ((wa & 0x1FFu) << 9) | (wb & 0x1FFu);
                d.w_first = ((hi << 5) | (wp[n & 3] >> 27)) << 9;
            } else {
                d.w_first = wp[n & 3];
            }
        }
        if (fp32) {
            float z1, z2;
            bm_f(wa, wb, &z1, &z2);
            if (neg) { z1 = -z1; z2 = -z2; }
            step_f(pf, c->model, c->scheme, &Sf, &vf, z1, z2, &d);
            ssum += (double)Sf;
            smaxf = fmaxf(smaxf, Sf);
            sminf = fminf(sminf, Sf);
            S = Sf; v = vf;
        } else {
            double z1, z2;
            bm_d(wa, wb, &z1, &z2);
            if (neg) { z1 = -z1; z2 = -z2; }
            step_d(p, c->model, c->scheme, &S, &v, z1, z2, &d);
            ssum += S;
            smax = fmax(smax, S);
            smin = fmin(smin, S);
        }
        if (stride > 0 && ((n + 1) % stride) == 0) {
            const int64_t row = (n + 1) / stride - 1;
            S_rows[row * ld + col] = S;
            if (v_rows) v_rows[row * ld + col] = v;
        }
    }
    o->S = S;
    o->v = v;
    o->ssum = ssum;
    o->smax = fp32 ? (double)smaxf : smax;
    o->smin = fp32 ? (double)sminf : smin;
}

static void run_path(const qk_contract *c, const Inv *p, const InvF *pf, uint32_t path, PathOut *o, int stride,
                     double *S_rows, double *v_rows, int64_t ld, int64_t col) {
    run_path_sign(c, p, pf, path, 0, o, stride, S_rows, v_rows, ld, col);
}

/* Payoff.hpp:51-72, 157-242, in double (float legs rounded through float like the FP32 build). */
static double intrinsic(int right, double S, double K) { return right == QK_CALL ? (S > K ? S - K : 0.0) : (K > S ? K - S : 0.0); }

static double payoff_of(const qk_payoff *ps, const PathOut *o, int n_steps, int fp32) {
    double S = o->S, K = ps->strike, B = ps->barrier, avg = o->ssum / (double)n_steps;
    double smax = o->smax, smin = o->smin;
    if (fp32) { K = (float)K; B = (float)B; avg = (float)avg; }
    double x;
    switch (ps->type) {
        case QK_EUROPEAN: x = intrinsic(ps->right, S, K); break;
        case QK_ASIAN: x = intrinsic(ps->right, avg, K); break;
        case QK_BARRIER_UP_OUT: x = smax < B ? intrinsic(ps->right, S, K) : 0.0; break;
        case QK_BARRIER_DOWN_OUT: x = smin > B ? intrinsic(ps->right, S, K) : 0.0; break;
        case QK_BARRIER_UP_IN: x = smax >= B ? intrinsic(ps->right, S, K) : 0.0; break;
        case QK_BARRIER_DOWN_IN: x = smin <= B ? intrinsic(ps->right, S, K) : 0.0; break;
        case QK_LOOKBACK_FLOATING: x = ps->right == QK_CALL ? intrinsic(QK_CALL, S, smin) : intrinsic(QK_PUT, S, smax); break;
        case QK_LOOKBACK_FIXED: x = ps->right == QK_CALL ? intrinsic(QK_CALL, smax, K) : intrinsic(QK_PUT, smin, K); break;
        case QK_BINARY_CASH: x = ps->right == QK_CALL ? (S > K ? 1.0 : 0.0) : (S < K ? 1.0 : 0.0); break;
        case QK_BINARY_ASSET: x = ps->right == QK_CALL ? (S > K ? S : 0.0) : (S < K ? S : 0.0); break;
        default: x = intrinsic(ps->right, S, K); break;
    }
    if (fp32) x = (float)x;
    return x;
}

/* PayoffTracker on a fed spot sequence S_1..S_n (Payoff.hpp:84-160: the trackers start
 * at S0, track_current_price after every step, evaluate_final_payoff at S_n): the same
 * running sum / max / min updates as the path loop above, then payoff_of.  fp32: the
 * sequence and the trackers in float, as the FP32 path loop keeps them. */
int qko_payoff_path(const qk_payoff *ps, const double *S, int n, double S0, int fp32, double *out) {
    if (n < 1 || !ps || !S || !out) return 1;
    PathOut o;
    double ssum = 0.0, smax = fp32 ? (double)(float)S0 : S0, smin = smax;
    float smaxf = (float)S0, sminf = (float)S0;
    for (int i = 0; i < n; ++i) {
        if (fp32) {
            const float s = (float)S[i];
            ssum += (double)s;
            smaxf = fmaxf(smaxf, s);
            sminf = fminf(sminf, s);
        } else {
            ssum += S[i];
            smax = fmax(smax, S[i]);
            smin = fmin(smin, S[i]);
        }
    }
    o.S = fp32 ? (double)(float)S[n - 1] : S[n - 1];
    o.v = 0.0;
    o.ssum = ssum;
    o.smax = fp32 ? (double)smaxf : smax;
    o.smin = fp32 ? (double)sminf : smin;
    *out = payoff_of(ps, &o, n, fp32);
    return 0;
}

/* Spot and variance paths (row-major count x n_steps, real units). */
int qko_paths(const qk_contract *c, int64_t first, int64_t count, double *S_out, double *v_out) {
    qk_contract n;
    double scale;
    normalise(c, &n, &scale);
    const double dt = n.T / n.n_steps;
    const Inv p = make_inv(&n, dt, n.precision == QK_FP32 ? 1e-6 : 1e-12);
    const InvF pf = to_f(&p);
    double *tmpS = (double *)malloc(sizeof(double) * (size_t)n.n_steps * (size_t)count);
    double *tmpv = (double *)malloc(sizeof(double) * (size_t)n.n_steps * (size_t)count);
    if (!tmpS || !tmpv) { free(tmpS); free(tmpv); return 1; }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < count; ++i) {
        PathOut o;
        run_path(&n, &p, &pf, (uint32_t)(first + i), &o, 1, tmpS, tmpv, count, i);
    }
    for (int64_t i = 0; i < count; ++i)
        for (int j = 0; j < n.n_steps; ++j) {
            S_out[i * n.n_steps + j] = tmpS[(size_t)j * count + i] * scale;
            if (v_out) v_out[i * n.n_steps + j] = tmpv[(size_t)j * count + i];
        }
    free(tmpS);
    free(tmpv);
    return 0;
}

/* Every path's leg-`leg` payoff, undiscounted, normalised units. */
int qko_payoffs(const qk_contract *c, int leg, double *out) {
    qk_contract n;
    double scale;
    normalise(c, &n, &scale);
    const Inv p = make_inv(&n, n.T / n.n_steps, n.precision == QK_FP32 ? 1e-6 : 1e-12);
    const InvF pf = to_f(&p);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n.n_paths; ++i) {
        PathOut o;
        run_path(&n, &p, &pf, (uint32_t)i, &o, 0, NULL, NULL, 0, 0);
        out[i] = payoff_of(&n.payoffs[leg], &o, n.n_steps, n.precision == QK_FP32);
    }
    return 0;
}

/* ================================================================ statistics */
typedef struct {
    double n, mean, m2, itm;
} Mom;

static Mom mom_merge(Mom a, Mom b) {
    const double n = a.n + b.n;
    if (b.n <= 0.0) return a;
    if (a.n <= 0.0) return b;
    const double d = b.mean - a.mean;
    Mom r = {n, a.mean + d * (b.n / n), a.m2 + b.m2 + d * d * (a.n * b.n / n), a.itm + b.itm};
    return r;
}

/* Forward pricing of one (normalised) task: moments per leg. */
static void forward_moments(const qk_contract *n, Mom *legs) {
    const double dt = n->T / n->n_steps;
    const int fp32 = n->precision == QK_FP32;
    const Inv p = make_inv(n, dt, fp32 ? 1e-6 : 1e-12);
    const InvF pf = to_f(&p);
    const double eps = fp32 ? 1e-6 : 1e-12; /* OptionPricer.hpp:316 */
    const int nl = n->n_payoffs;
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    Mom *part = (Mom *)calloc((size_t)nt * QK_MAX_PAYOFFS, sizeof(Mom));
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        Mom loc[QK_MAX_PAYOFFS];
        memset(loc, 0, sizeof(loc));
        if (n->antithetic) {
            /* one sample per antithetic pair: the average of its two payoffs */
#pragma omp for schedule(static)
            for (int64_t i = 0; i < n->n_paths / 2; ++i) {
                PathOut oa, ob;
                run_path_sign(n, &p, &pf, (uint32_t)i, 0, &oa, 0, NULL, NULL, 0, 0);
                run_path_sign(n, &p, &pf, (uint32_t)i, 1, &ob, 0, NULL, NULL, 0, 0);
                for (int k = 0; k < nl; ++k) {
                    const double xa = payoff_of(&n->payoffs[k], &oa, n->n_steps, fp32);
                    const double xb = payoff_of(&n->payoffs[k], &ob, n->n_steps, fp32);
                    Mom one = {1.0, 0.5 * (xa + xb), 0.0, 0.5 * ((xa > eps ? 1.0 : 0.0) + (xb > eps ? 1.0 : 0.0))};
                    loc[k] = mom_merge(loc[k], one);
                }
            }
        } else {
#pragma omp for schedule(static)
            for (int64_t i = 0; i < n->n_paths; ++i) {
                PathOut o;
                run_path(n, &p, &pf, (uint32_t)i, &o, 0, NULL, NULL, 0, 0);
                for (int k = 0; k < nl; ++k) {
                    const double x = payoff_of(&n->payoffs[k], &o, n->n_steps, fp32);
                    Mom one = {1.0, x, 0.0, x > eps ? 1.0 : 0.0};
                    loc[k] = mom_merge(loc[k], one);
                }
            }
        }
        for (int k = 0; k < nl; ++k) part[(size_t)tid * QK_MAX_PAYOFFS + k] = loc[k];
    }
    for (int k = 0; k < nl; ++k) {
        Mom m = {0, 0, 0, 0};
        for (int t = 0; t < nt; ++t) m = mom_merge(m, part[(size_t)t * QK_MAX_PAYOFFS + k]);
        legs[k] = m;
    }
    free(part);
}

/* ================================================================ Longstaff-Schwartz */
static void laguerre4(double X, double *L, int fp32) {
    /* LaguerreBasis<4>::evaluate, Horner form (LSMAmerican.hpp:183-192) */
    if (fp32) {
        const float x = (float)X;
        L[0] = 1.0f; L[1] = 1.0f - x; L[2] = ((0.5f * x - 2.0f) * x) + 1.0f;
        L[3] = (((-1.0f / 6.0f) * x + 1.5f) * x - 3.0f) * x + 1.0f;
        L[3] = (float)L[3];
    } else {
        L[0] = 1.0; L[1] = 1.0 - X; L[2] = ((0.5 * X - 2.0) * X) + 1.0;
        L[3] = (((-1.0 / 6.0) * X + 1.5) * X - 3.0) * X + 1.0;
    }
}

/* LSMEngine::solve_system_on_host_cholesky (LSMAmerican.hpp:516-581) + fallback (:605-613) */
int qko_lsm_solve_reference(const double *M_in, const double *B, double count, int nb, double *C) {
    double M[8][8], L[8][8], y[8];
    for (int i = 0; i < nb; ++i) C[i] = 0.0;
    if (count < (double)nb) { if (count > 0.0) C[0] = B[0] / count; return 2; }
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) { M[i][j] = M_in[i * nb + j] + (i == j ? 1e-8 : 0.0); L[i][j] = 0.0; }
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = 0.0;
            for (int k = 0; k < j; ++k) s += L[i][k] * L[j][k];
            if (i == j) {
                const double val = M[i][i] - s;
                if (val < 1e-14) { for (int q = 0; q < nb; ++q) C[q] = 0.0; if (count > 0.0) C[0] = B[0] / count; return 2; }
                L[i][i] = sqrt(val);
            } else L[i][j] = (M[i][j] - s) / L[j][j];
        }
    for (int i = 0; i < nb; ++i) { double s = 0.0; for (int k = 0; k < i; ++k) s += L[i][k] * y[k]; y[i] = (B[i] - s) / L[i][i]; }
    for (int i = nb - 1; i >= 0; --i) { double s = 0.0; for (int k = i + 1; k < nb; ++k) s += L[k][i] * C[k]; C[i] = (y[i] - s) / L[i][i]; }
    return 0;
}

/* Least squares on the {1,S,S^2,S^3,v,Sv} basis: normal equations of the raw
 * monomials of S/K and v, solved by Gaussian elimination with partial pivoting in
 * long double (independent of the engine's centred/scaled FP64 route). */
static int solve_ld(long double G[6][6], long double b[6], double count, double *c) {
    for (int i = 0; i < 6; ++i) c[i] = 0.0;
    if (count < 6.0) { if (count > 0.0) c[0] = (double)(b[0] / count); return 2; }
    long double A[6][7];
    for (int i = 0; i < 6; ++i) { for (int j = 0; j < 6; ++j) A[i][j] = G[i][j]; A[i][6] = b[i]; }
    for (int k = 0; k < 6; ++k) {
        int piv = k;
        for (int i = k + 1; i < 6; ++i) if (fabsl(A[i][k]) > fabsl(A[piv][k])) piv = i;
        if (fabsl(A[piv][k]) == 0.0L) { if (count > 0.0) c[0] = (double)(b[0] / count); return 2; }
        if (piv != k) for (int j = 0; j < 7; ++j) { long double t = A[k][j]; A[k][j] = A[piv][j]; A[piv][j] = t; }
        for (int i = k + 1; i < 6; ++i) {
            const long double f = A[i][k] / A[k][k];
            for (int j = k; j < 7; ++j) A[i][j] -= f * A[k][j];
        }
    }
    long double x[6];
    for (int i = 5; i >= 0; --i) { long double s = A[i][6]; for (int j = i + 1; j < 6; ++j) s -= A[i][j] * x[j]; x[i] = s / A[i][i]; }
    for (int i = 0; i < 6; ++i) c[i] = (double)x[i];
    return 0;
}

static void poly6(double x, double v, double *b) { b[0] = 1.0; b[1] = x; b[2] = x * x; b[3] = x * x * x; b[4] = v; b[5] = x * v; }

/* Backward induction over a normalised task: returns moments of the discounted cash flows. */
static Mom lsm_moments(const qk_contract *n) {
    const int D = n->lsm_dates > 0 ? n->lsm_dates : n->n_steps;
    const int stride = n->n_steps / D;
    const int64_t N = n->n_paths;
    const double dt = n->T / n->n_steps;
    const int fp32 = n->precision == QK_FP32;
    const Inv p = make_inv(n, dt, fp32 ? 1e-6 : 1e-12);
    const InvF pf = to_f(&p);
    const int poly = n->lsm_basis == QK_LSM_POLY_SV;
    double *Sr = (double *)malloc(sizeof(double) * (size_t)D * N);
    double *vr = poly ? (double *)malloc(sizeof(double) * (size_t)D * N) : NULL;
    double *cf = (double *)malloc(sizeof(double) * N);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        PathOut o;
        run_path(n, &p, &pf, (uint32_t)i, &o, stride, Sr, vr, N, i);
    }
    const double K = fp32 ? (float)n->payoffs[0].strike : n->payoffs[0].strike;
    const int right = n->payoffs[0].right;
    double disc = exp(-n->r * stride * dt); /* ForwardBackwardMC.hpp:209 */
    if (fp32) disc = (float)disc;
    /* initialise at maturity (LSMAmerican.hpp:252-264) */
    for (int64_t i = 0; i < N; ++i) cf[i] = intrinsic(right, Sr[(size_t)(D - 1) * N + i], K);
    for (int d = D - 2; d >= 0; --d) {
        const double *S = Sr + (size_t)d * N;
        const double *V = poly ? vr + (size_t)d * N : NULL;
        double coef[8] = {0};
        if (!poly) {
            double M[16] = {0}, B[4] = {0}, cnt = 0.0;
            for (int64_t i = 0; i < N; ++i) {
                const double iv = fp32 ? (float)intrinsic(right, S[i], K) : intrinsic(right, S[i], K);
                if (iv > 0.0) {
                    const double Y = fp32 ? (double)(float)((float)cf[i] * (float)disc) : cf[i] * disc;
                    double L[4];
                    laguerre4(fp32 ? (double)((float)S[i] / (float)K) : S[i] / K, L, fp32);
                    for (int r = 0; r < 4; ++r) { B[r] += L[r] * Y; for (int q = 0; q < 4; ++q) M[r * 4 + q] += L[r] * L[q]; }
                    cnt += 1.0;
                }
            }
            qko_lsm_solve_reference(M, B, cnt, 4, coef);
        } else {
            long double G[6][6], b[6];
            double cnt = 0.0;
            memset(G, 0, sizeof(G)); memset(b, 0, sizeof(b));
            for (int64_t i = 0; i < N; ++i) {
                const double iv = intrinsic(right, S[i], K);
                if (iv > 0.0) {
                    const double Y = cf[i] * disc;
                    double bb[6];
                    poly6(S[i] / K, V[i], bb);
                    for (int r = 0; r < 6; ++r) { b[r] += (long double)bb[r] * Y; for (int q = 0; q < 6; ++q) G[r][q] += (long double)bb[r] * bb[q]; }
                    cnt += 1.0;
                }
            }
            solve_ld(G, b, cnt, coef);
        }
        /* update_cashflows (LSMAmerican.hpp:310-341) */
        for (int64_t i = 0; i < N; ++i) {
            const double iv = fp32 ? (float)intrinsic(right, S[i], K) : intrinsic(right, S[i], K);
            const double dcf = fp32 ? (double)((float)cf[i] * (float)disc) : cf[i] * disc;
            if (iv > 0.0) {
                double hold = 0.0;
                if (!poly) { double L[4]; laguerre4(fp32 ? (double)((float)S[i] / (float)K) : S[i] / K, L, fp32); for (int r = 0; r < 4; ++r) hold += coef[r] * L[r]; }
                else { double bb[6]; poly6(S[i] / K, V[i], bb); for (int r = 0; r < 6; ++r) hold += coef[r] * bb[r]; }
                cf[i] = iv > hold ? iv : dcf;
            } else cf[i] = dcf;
        }
    }
    /* apply_final_discount (LSMAmerican.hpp:393-419) and the pricer moments */
    const double eps = fp32 ? 1e-6 : 1e-12;
    Mom m = {0, 0, 0, 0};
    for (int64_t i = 0; i < N; ++i) {
        const double x = fp32 ? (double)((float)cf[i] * (float)disc) : cf[i] * disc;
        Mom one = {1.0, x, 0.0, x > eps ? 1.0 : 0.0};
        m = mom_merge(m, one);
    }
    const double today = intrinsic(right, n->S0, K);
    if (today > m.mean) { m.mean = today; m.m2 = 0.0; m.itm = today > eps ? m.n : 0.0; }
    free(Sr); free(vr); free(cf);
    return m;
}

/* ================================================================ pricing with Greeks
 * execute_mc_framework (MCEngine.hpp:560-746): base price, then every requested
 * Greek by re-pricing a bumped copy with the same random numbers. */
enum { R_BASE = 0, R_SU, R_SD, R_VU, R_VD, R_RU, R_RD, R_TD, R_UU, R_DU, R_UD, R_DD, R_N };

static void price_task(const qk_contract *b, double scale, double *price, double *se, double *itm) {
    Mom legs[QK_MAX_PAYOFFS];
    const int american = b->payoffs[0].type == QK_AMERICAN;
    if (american) legs[0] = lsm_moments(b);
    else forward_moments(b, legs);
    for (int k = 0; k < b->n_payoffs; ++k) {
        const Mom m = legs[k];
        const double disc = american ? 1.0 : exp(-b->r * b->T);
        const double eff = disc * (b->payoffs[k].type == QK_BINARY_CASH ? 1.0 : scale);
        const double var = m.n > 1.0 ? m.m2 / (m.n - 1.0) : 0.0;
        price[k] = m.mean * eff;
        se[k] = m.n > 0.0 ? sqrt(var / m.n) * eff : 0.0;
        itm[k] = m.n > 0.0 ? m.itm / m.n : 0.0;
    }
}

int qko_price(const qk_contract *c, const qk_greeks *g, qk_result *out) {
    memset(out, 0, sizeof(*out));
    qk_contract n;
    double scale;
    normalise(c, &n, &scale);
    out->n_payoffs = n.n_payoffs;
    out->n_paths = n.n_paths;
    double P[R_N][QK_MAX_PAYOFFS], SE[QK_MAX_PAYOFFS], IT[QK_MAX_PAYOFFS], tmp_se[QK_MAX_PAYOFFS], tmp_it[QK_MAX_PAYOFFS];
    price_task(&n, scale, P[R_BASE], SE, IT);
    out->path_steps = (double)n.n_paths * n.n_steps;
    for (int k = 0; k < n.n_payoffs; ++k) { out->p[k].price = P[R_BASE][k]; out->p[k].std_error = SE[k]; out->p[k].prob_itm = IT[k]; }
    if (!g || !g->mask) return 0;
    const double hS = n.S0 * g->bump_S_rel;
    const double hS_real = (n.normalize ? scale : n.S0) * g->bump_S_rel;
    double vup, vdn, hv;
    if (g->vega_mode == 0) { const double vol0 = sqrt(n.v0); vup = (vol0 + g->bump_vol) * (vol0 + g->bump_vol); vdn = (vol0 - g->bump_vol) * (vol0 - g->bump_vol); hv = g->bump_vol; }
    else { vup = n.v0 * (1.0 + g->bump_vol); vdn = n.v0 * (1.0 - g->bump_vol); hv = n.v0 * g->bump_vol; }
#define BUMP(role, field_stmt)                                   \
    do {                                                         \
        qk_contract b = n;                                       \
        field_stmt;                                              \
        price_task(&b, scale, P[role], tmp_se, tmp_it);          \
        out->path_steps += (double)b.n_paths * b.n_steps;        \
    } while (0)
    if (g->mask & QK_GREEK_DELTA_GAMMA) { BUMP(R_SU, b.S0 = n.S0 + hS); BUMP(R_SD, b.S0 = n.S0 - hS); }
    if (g->mask & QK_GREEK_VEGA_VOMMA) { BUMP(R_VU, b.v0 = vup); BUMP(R_VD, b.v0 = vdn); }
    if (g->mask & QK_GREEK_RHO) { BUMP(R_RU, b.r = n.r + g->bump_r_abs); BUMP(R_RD, b.r = n.r - g->bump_r_abs); }
    if ((g->mask & QK_GREEK_THETA) && n.T > g->bump_T_abs) { BUMP(R_TD, b.T = n.T - g->bump_T_abs); }
    if (g->mask & QK_GREEK_VANNA) {
        BUMP(R_UU, (b.S0 = n.S0 + hS, b.v0 = vup)); BUMP(R_DU, (b.S0 = n.S0 - hS, b.v0 = vup));
        BUMP(R_UD, (b.S0 = n.S0 + hS, b.v0 = vdn)); BUMP(R_DD, (b.S0 = n.S0 - hS, b.v0 = vdn));
    }
#undef BUMP
    for (int k = 0; k < n.n_payoffs; ++k) {
        qk_payoff_result *r = &out->p[k];
        const double p0 = P[R_BASE][k];
        if (g->mask & QK_GREEK_DELTA_GAMMA) {
            r->delta = (P[R_SU][k] - P[R_SD][k]) / (2.0 * hS_real);
            r->gamma = (P[R_SU][k] - 2.0 * p0 + P[R_SD][k]) / (hS_real * hS_real);
        }
        if (g->mask & QK_GREEK_VEGA_VOMMA) {
            r->vega = (P[R_VU][k] - P[R_VD][k]) / (2.0 * hv);
            r->vomma = (P[R_VU][k] - 2.0 * p0 + P[R_VD][k]) / (hv * hv);
        }
        if (g->mask & QK_GREEK_RHO) r->rho = (P[R_RU][k] - P[R_RD][k]) / (2.0 * g->bump_r_abs);
        if (g->mask & QK_GREEK_THETA) r->theta = n.T > g->bump_T_abs ? (P[R_TD][k] - p0) / g->bump_T_abs : 0.0;
        if (g->mask & QK_GREEK_VANNA) r->vanna = (P[R_UU][k] - P[R_DU][k] - P[R_UD][k] + P[R_DD][k]) / (4.0 * hS_real * hv);
    }
    return 0;
}

/* ================================================================ closed forms
 * BlackScholesExact.hpp:46-65; HestonExact.hpp:56-195 (Albrecher form, P_j by 64-point
 * Gauss-Legendre on [0, phi_max]); BatesExact.hpp:49-145 (Merton jump exponent added,
 * 50-wide chunks).  Complex arithmetic written out on (re, im) pairs. */
typedef struct { double re, im; } cx;
static cx cmk(double a, double b) { cx z = {a, b}; return z; }
static cx cadd(cx a, cx b) { return cmk(a.re + b.re, a.im + b.im); }
static cx csub(cx a, cx b) { return cmk(a.re - b.re, a.im - b.im); }
static cx cmul(cx a, cx b) { return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static cx cdiv(cx a, cx b) { const double d = b.re * b.re + b.im * b.im; return cmk((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d); }
static cx cexp_(cx a) { const double e = exp(a.re); return cmk(e * cos(a.im), e * sin(a.im)); }
static cx clog_(cx a) { return cmk(log(hypot(a.re, a.im)), atan2(a.im, a.re)); }
static cx csqrt_(cx a) {
    const double r = hypot(a.re, a.im);
    double re = sqrt(0.5 * (r + a.re)), im = sqrt(0.5 * (r - a.re));
    if (a.im < 0.0) im = -im;
    return cmk(re, im);
}
static cx cscale(cx a, double s) { return cmk(a.re * s, a.im * s); }

static double gl_x[64], gl_w[64];
static int gl_ready = 0;
static void gl_init(void) {
    /* nodes of P_64 by Newton iteration from Chebyshev-like starting points */
    const int n = 64;
    for (int i = 0; i < n; ++i) {
        double x = cos(M_PI * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; ++k) { const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k; p0 = p1; p1 = p2; }
            const double dp = n * (x * p1 - p0) / (x * x - 1.0);
            const double dx = p1 / dp;
            x -= dx;
            if (fabs(dx) < 1e-16) break;
        }
        double p0 = 1.0, p1 = x;
        for (int k = 2; k <= n; ++k) { const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k; p0 = p1; p1 = p2; }
        const double dp = n * (x * p1 - p0) / (x * x - 1.0);
        gl_x[i] = x;
        gl_w[i] = 2.0 / ((1.0 - x * x) * dp * dp);
    }
    gl_ready = 1;
}

/* exponent C + D v0 + i phi ln S0 of f_j (HestonExact.hpp:56-101) */
static cx heston_exponent(double phi, const qk_contract *c, int j) {
    const double rho = c->rho, sg = c->sigma, k = c->kappa, th = c->theta, T = c->T;
    const double u = (j == 1) ? 0.5 : -0.5;
    const double b = (j == 1) ? k - rho * sg : k;
    const cx i_phi = cmk(0.0, phi);
    const cx rsip_b = csub(cscale(i_phi, rho * sg), cmk(b, 0.0));
    const cx t1 = cmul(rsip_b, rsip_b);
    const cx t2 = cscale(cadd(cscale(i_phi, 2.0 * u), cmk(-phi * phi, 0.0)), sg * sg);
    const cx d = csqrt_(csub(t1, t2));
    const cx bmr = csub(cmk(b, 0.0), cscale(i_phi, rho * sg));
    const cx g = cdiv(csub(bmr, d), cadd(bmr, d));
    const cx edt = cexp_(cscale(d, -T));
    const cx C1 = cscale(i_phi, (c->r - c->q) * T);
    const cx lg = clog_(cdiv(csub(cmk(1.0, 0.0), cmul(g, edt)), csub(cmk(1.0, 0.0), g)));
    const cx C2 = cscale(csub(cscale(csub(bmr, d), T), cscale(lg, 2.0)), (k * th) / (sg * sg));
    const cx D = cmul(cscale(csub(bmr, d), 1.0 / (sg * sg)), cdiv(csub(cmk(1.0, 0.0), edt), csub(cmk(1.0, 0.0), cmul(g, edt))));
    return cadd(cadd(cadd(C1, C2), cscale(D, c->v0)), cscale(i_phi, log(c->S0)));
}

static double integrand(double phi, const qk_contract *c, int j, double K, int bates) {
    cx ex = heston_exponent(phi, c, j);
    if (bates) { /* BatesExact.hpp:49-80 */
        const double kbar = exp(c->mu_j + 0.5 * c->sigma_j * c->sigma_j) - 1.0;
        const double uj = (j == 1) ? 1.0 : 0.0;
        const double muj = (j == 1) ? c->mu_j + c->sigma_j * c->sigma_j : c->mu_j;
        const cx inner = csub(cexp_(cmk(-0.5 * c->sigma_j * c->sigma_j * phi * phi, phi * muj)), cmk(1.0, 0.0));
        const cx E = cscale(cadd(cmk(0.0, -phi * kbar), cscale(inner, pow(1.0 + kbar, uj))), c->lambda_j * c->T);
        ex = cadd(ex, E);
    }
    const cx f = cexp_(ex);
    const cx num = cmul(cexp_(cmk(0.0, -phi * log(K))), f);
    return cdiv(num, cmk(0.0, phi)).re;
}

static double gl_integrate(const qk_contract *c, int j, double K, int bates, double a, double b) {
    if (!gl_ready) gl_init();
    const double sc = 0.5 * (b - a), sh = 0.5 * (a + b);
    double s = 0.0;
    for (int i = 0; i < 64; ++i) s += gl_w[i] * integrand(sc * gl_x[i] + sh, c, j, K, bates);
    return s * sc;
}

/* kind 0 Black-Scholes, 1 Heston, 2 Bates; European call on c->payoffs[0].strike. */
int qko_exact_call(int kind, const qk_contract *c, double phi_max, double *price) {
    const double S = c->S0, K = c->payoffs[0].strike, T = c->T, r = c->r, q = c->q;
    if (kind == 0) {
        const double vol = sqrt(c->v0);
        const double d1 = (log(S / K) + (r - q + 0.5 * vol * vol) * T) / (vol * sqrt(T));
        const double d2 = d1 - vol * sqrt(T);
        *price = S * exp(-q * T) * 0.5 * (1.0 + erf(d1 / sqrt(2.0))) - K * exp(-r * T) * 0.5 * (1.0 + erf(d2 / sqrt(2.0)));
        return 0;
    }
    double P[3];
    for (int j = 1; j <= 2; ++j) {
        double integral = 0.0;
        if (kind == 1) integral = gl_integrate(c, j, K, 0, 0.0, phi_max > 0 ? phi_max : 100.0);
        else {
            const double pm = phi_max > 0 ? phi_max : 8000.0;
            const int chunks = (int)(pm / 50.0);
            for (int i = 0; i < chunks; ++i) integral += gl_integrate(c, j, K, 1, i * 50.0, (i + 1) * 50.0);
        }
        P[j] = 0.5 + integral / M_PI;
    }
    *price = S * exp(-q * T) * P[1] - K * exp(-r * T) * P[2];
    return 0;
}

int qko_gl_nodes(double *x, double *w) {
    if (!gl_ready) gl_init();
    memcpy(x, gl_x, sizeof(gl_x));
    memcpy(w, gl_w, sizeof(gl_w));
    return 0;
}
