// oracle.cpp -- CPU restatement of UncertainTea's batched density + sampler
// hot path.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and
// the CPU-baseline leg of bench.py load it as the test oracle.  The product
// library (uncertaintea_b200/csrc) never links, loads or calls it.
//
// Parity pinning: Philox4x32-10 is pinned by the Random123 known-answer
// vectors the reference's own test holds (test/uncertaintea/core/device_rng.jl:77-93);
// the ChEES scalar helpers by the reference's unit pins
// (test/uncertaintea/core/batched_chees_adaptation.jl:29-72); the NUTS U-turn
// helpers by its U-turn unit vectors (nuts_uturn_turning.jl:204-380); the MEADS
// eigenvalue estimator and slice drift by its MEADS pins (batched_meads.jl:32-57).
// The samplers (NUTS, HMC, MEADS, the ADVI step) are checked on the CPU against
// exact posteriors (the reference's conjugate gate model, a grid posterior, an
// analytic hierarchical marginal).  The reference is
// Julia, which is not installed here, so its density/gradient/sampler code
// cannot be run: those functions are restated from the cited source lines and
// checked against closed forms and central finite differences instead, on
// the reference's own parity-case inputs where it has them
// (test/uncertaintea/core/device_lowering_parity.jl:131-176); parity for them
// is unpinned by reference outputs.
//
// Everything is templated on the arithmetic type T (float / double), like the
// reference's precision-generic kernels (Float32 on Metal, Float64 on CPU()).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/ut_b200.h"
#include "oracle_mlp.h"
#include "oracle_program.h"

namespace {

// ---------------------------------------------------------------------------
// Philox4x32-10 (src/device/rng.jl:54-119)
// ---------------------------------------------------------------------------
const uint32_t kPhiloxM0 = 0xD2511F53u;  // rng.jl:54
const uint32_t kPhiloxM1 = 0xCD9E8D57u;  // rng.jl:55
const uint32_t kPhiloxW0 = 0x9E3779B9u;  // rng.jl:56
const uint32_t kPhiloxW1 = 0xBB67AE85u;  // rng.jl:57

struct Block { uint32_t w[4]; };

inline Block philox_round(const Block& c, uint32_t k0, uint32_t k1) {  // rng.jl:71-75
    uint64_t p0 = (uint64_t)kPhiloxM0 * c.w[0];
    uint64_t p1 = (uint64_t)kPhiloxM1 * c.w[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    Block r;
    r.w[0] = hi1 ^ c.w[1] ^ k0;
    r.w[1] = lo1;
    r.w[2] = hi0 ^ c.w[3] ^ k1;
    r.w[3] = lo0;
    return r;
}

inline Block philox(uint32_t k0, uint32_t k1, Block c) {  // rng.jl:95-119
    c = philox_round(c, k0, k1);
    for (int r = 1; r < 10; ++r) {
        k0 += kPhiloxW0;  // rng.jl:78-79 (bump before each later round)
        k1 += kPhiloxW1;
        c = philox_round(c, k0, k1);
    }
    return c;
}

inline Block coord_block(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw) {
    Block c = {{stream, draw, 0u, 0u}};  // rng.jl:172
    return philox(chain, iter, c);
}

inline float u01_f32(uint32_t w) { return (float)(w >> 8) * 0x1p-24f; }  // rng.jl:131
inline double u01_f64(uint32_t w0, uint32_t w1) {                       // rng.jl:135-138
    uint64_t bits = ((uint64_t)w0 << 32) | (uint64_t)w1;
    return (double)(bits >> 11) * 0x1p-53;
}

template <class T> T rand_uniform(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw);
template <> float rand_uniform<float>(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw) {
    return u01_f32(coord_block(chain, iter, stream, draw).w[0]);  // rng.jl:143-144
}
template <> double rand_uniform<double>(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw) {
    Block b = coord_block(chain, iter, stream, draw);
    return u01_f64(b.w[0], b.w[1]);  // rng.jl:145-146
}

template <class T> T rand_normal(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw);
template <> float rand_normal<float>(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw) {
    Block b = coord_block(chain, iter, stream, draw);  // rng.jl:208-213
    float u1 = u01_f32(b.w[0]);
    float u2 = u01_f32(b.w[1]);
    float radius = std::sqrt(-2.0f * std::log(1.0f - u1));
    return radius * std::cos(6.2831855f * u2);
}
template <> double rand_normal<double>(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw) {
    Block b = coord_block(chain, iter, stream, draw);  // rng.jl:214-219
    double u1 = u01_f64(b.w[0], b.w[1]);
    double u2 = u01_f64(b.w[2], b.w[3]);
    double radius = std::sqrt(-2.0 * std::log(1.0 - u1));
    return radius * std::cos(6.283185307179586 * u2);
}

// ---------------------------------------------------------------------------
// Device math (src/device/math.jl)
// ---------------------------------------------------------------------------
template <class T> inline T normal_logpdf(T mu, T sigma, T x) {  // math.jl:88-91
    T z = (x - mu) / sigma;
    return -std::log(sigma) - T(0.9189385332046727) - z * z / T(2);
}
template <class T> inline T halfcauchy_logpdf(T scale, T x) {  // math.jl:126-130
    T z = x / scale;
    T base = T(0.6931471805599453) - T(1.1447298858494002) - std::log(scale) - std::log1p(z * z);
    return x >= T(0) ? base : -std::numeric_limits<T>::infinity();
}
template <class T> inline T log1p_exp(T eta) {  // math.jl:202-203
    return eta > T(0) ? eta + std::log1p(std::exp(-eta)) : std::log1p(std::exp(eta));
}
template <class T> inline T bernoullilogit_logpdf(T eta, T x) {  // math.jl:212-217
    T base = x * eta - log1p_exp(eta);
    bool in_support = (x == T(0)) || (x == T(1));
    return in_support ? base : -std::numeric_limits<T>::infinity();
}
template <class T> inline T logistic(T eta) { return std::exp(-log1p_exp(-eta)); }  // math.jl:224
// math.jl:103-107 (support: a positive normal float, math.jl:66); the
// normaliser uses the C library's lgamma in double, where the reference's
// device code uses its own Lanczos loggamma (math.jl:30-50).
template <class T> inline T gamma_logpdf(T shape, T rate, T x) {
    T base = shape * std::log(rate) - (T)std::lgamma((double)shape) + (shape - T(1)) * std::log(x) - rate * x;
    return x >= std::numeric_limits<T>::min() ? base : -std::numeric_limits<T>::infinity();
}

// ---------------------------------------------------------------------------
// Models: unconstrained logjoint + analytic gradient of one chain.
// ---------------------------------------------------------------------------
struct ModelData {
    ut_plan_desc plan;
    oracle_program::Program prog;  // UT_FAMILY_PROGRAM: the step program (y holds its staged rows)
    std::vector<double> X;   // N x D row-major (observation-major), GLM
    std::vector<double> y;   // N
    std::vector<double> sig; // J, HIER
    std::vector<int32_t> start, count;  // J, HIER
};

ModelData make_model(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                     const int32_t* loop_starts) {
    ModelData m;
    m.plan = *plan;
    const int N = plan->num_obs;
    if (plan->family == UT_FAMILY_GLM_BERNOULLI_LOGIT) {
        const int D = plan->num_coefs;
        m.X.resize((size_t)N * D);
        m.y.resize(N);
        for (int i = 0; i < N; ++i) {  // staged rows: D covariates then y (staging.jl:332)
            for (int d = 0; d < D; ++d) m.X[(size_t)i * D + d] = observed[(size_t)i * (D + 1) + d];
            m.y[i] = observed[(size_t)i * (D + 1) + D];
        }
    } else if (plan->family == UT_FAMILY_PROGRAM) {
        m.prog = oracle_program::current();
        m.y.assign(observed, observed + N);
    } else if (plan->family == UT_FAMILY_NORMAL_LOCATION_SCALE || plan->family == UT_FAMILY_BERNOULLI_BETA ||
               plan->family == UT_FAMILY_LOGNORMAL_GAMMA_NORMAL || plan->family == UT_FAMILY_STUDENTT_HEAVY_TAIL ||
               plan->family == UT_FAMILY_NORMAL_KNOWN_SCALE) {
        m.y.assign(observed, observed + N);
    } else {
        const int J = plan->num_groups;
        m.y.assign(observed, observed + N);
        m.sig.assign(observed + N, observed + N + J);
        m.start.assign(loop_starts, loop_starts + J);
        m.count.assign(trip_counts, trip_counts + J);
    }
    return m;
}

// GLM: logjoint value = intercept prior + coefficient prior + likelihood, in the
// plan's step order (logjoint_kernel.jl:378-399, 514-533); gradient is the
// analytic form d/d_eta = y - logistic(eta) fanned to the coefficient rows
// (gradient_kernel.jl:579-627; CPU analog observed_loop.jl:238-275).
// Sums are accumulated in the wide type W (double for the f64 oracle).
template <class T, class W>
W glm_logjoint_grad(const ModelData& m, const T* q, T* g) {
    const ut_plan_desc& p = m.plan;
    const int N = p.num_obs, D = p.num_coefs;
    const int off = p.has_intercept ? 1 : 0;
    const int P = off + D;
    std::vector<W> gw(P, W(0));
    W total = 0;
    T a = off ? q[0] : T(0);
    if (off) {
        total += (W)normal_logpdf<T>(T(p.intercept_mu), T(p.intercept_sigma), a);
        gw[0] += -(W)(a - T(p.intercept_mu)) / ((W)p.intercept_sigma * (W)p.intercept_sigma);
    }
    for (int d = 0; d < D; ++d) {
        T b = q[off + d];
        total += (W)normal_logpdf<T>(T(p.coef_mu), T(p.coef_sigma), b);
        gw[off + d] += -(W)(b - T(p.coef_mu)) / ((W)p.coef_sigma * (W)p.coef_sigma);
    }
    for (int i = 0; i < N; ++i) {
        const double* x = &m.X[(size_t)i * D];
        W eta = off ? (W)a : W(0);
        for (int d = 0; d < D; ++d) eta += (W)q[off + d] * (W)x[d];
        T et = (T)eta, yt = (T)m.y[i];
        total += (W)bernoullilogit_logpdf<T>(et, yt);
        if (g) {
            W r = (W)yt - (W)logistic<T>(et);
            if (off) gw[0] += r;
            for (int d = 0; d < D; ++d) gw[off + d] += r * (W)x[d];
        }
    }
    if (g) for (int k = 0; k < P; ++k) g[k] = (T)gw[k];
    return total;
}

// Hierarchical non-centred normal (steps: Normal, HalfCauchy with log transform
// logjoint_kernel.jl:105-111,177-182 + math.jl:1144-1146 (lad = u), Noncentered
// logjoint_kernel.jl:113-129, then the observation loop).
template <class T, class W>
W hier_logjoint_grad(const ModelData& m, const T* q, T* g) {
    const ut_plan_desc& p = m.plan;
    const int J = p.num_groups;
    T mu = q[0], u = q[1];
    T tau = std::exp(u);
    W total = (W)normal_logpdf<T>(T(p.mu_loc), T(p.mu_scale), mu);
    total += (W)halfcauchy_logpdf<T>(T(p.tau_scale), tau) + (W)u;
    W gmu = -(W)(mu - T(p.mu_loc)) / ((W)p.mu_scale * (W)p.mu_scale);
    W s2 = (W)p.tau_scale * (W)p.tau_scale;
    W gu = W(1) - W(2) * (W)tau * (W)tau / (s2 + (W)tau * (W)tau);
    for (int j = 0; j < J; ++j) {
        T z = q[2 + j];
        total += (W)normal_logpdf<T>(T(0), T(1), z);
        T theta = mu + tau * z;
        T sj = (T)m.sig[j];
        W dtheta = 0;
        for (int k = 0; k < m.count[j]; ++k) {
            T yv = (T)m.y[m.start[j] + k];
            total += (W)normal_logpdf<T>(theta, sj, yv);
            dtheta += (W)(yv - theta) / ((W)sj * (W)sj);
        }
        gmu += dtheta;
        gu += (W)tau * (W)z * dtheta;
        if (g) g[2 + j] = (T)(-(W)z + (W)tau * dtheta);
    }
    if (g) { g[0] = (T)gmu; g[1] = (T)gu; }
    return total;
}

// Normal location/scale (steps: Normal on mu, Gamma on s with log transform,
// lad = u (math.jl:1144-1146), then the loop of normal observations;
// logjoint_kernel.jl:105-111, 146-151).  Every observation term is scored
// separately, in order.
template <class T, class W>
W gauss_logjoint_grad(const ModelData& m, const T* q, T* g) {
    const ut_plan_desc& p = m.plan;
    const int N = p.num_obs;
    T mu = q[0], u = q[1];
    T s = std::exp(u);
    W total = (W)normal_logpdf<T>(T(p.mu_loc), T(p.mu_scale), mu);
    total += (W)gamma_logpdf<T>(T(p.scale_shape), T(p.scale_rate), s) + (W)u;
    W gmu = -(W)(mu - T(p.mu_loc)) / ((W)p.mu_scale * (W)p.mu_scale);
    W gu = (W)p.scale_shape - (W)p.scale_rate * (W)s;  // gamma prior + lad, d/du
    for (int i = 0; i < N; ++i) {
        T yv = (T)m.y[i];
        total += (W)normal_logpdf<T>(mu, s, yv);
        W r = (W)yv - (W)mu;
        gmu += r / ((W)s * (W)s);
        gu += r * r / ((W)s * (W)s) - W(1);
    }
    if (g) { g[0] = (T)gmu; g[1] = (T)gu; }
    return total;
}

// Normal location with a known observation scale (steps: Normal on mu, then
// the loop of normal observations with a constant scale argument;
// logjoint_kernel.jl:105-111, the reference's conjugate gate model
// test/uncertaintea/core/device_persistent_nuts.jl:33-38).
template <class T, class W>
W nks_logjoint_grad(const ModelData& m, const T* q, T* g) {
    const ut_plan_desc& p = m.plan;
    const T mu = q[0], sigma = T(p.obs_scale);
    W total = (W)normal_logpdf<T>(T(p.mu_loc), T(p.mu_scale), mu);
    W gmu = -(W)(mu - T(p.mu_loc)) / ((W)p.mu_scale * (W)p.mu_scale);
    for (int i = 0; i < p.num_obs; ++i) {
        const T yv = (T)m.y[i];
        total += (W)normal_logpdf<T>(mu, sigma, yv);
        gmu += ((W)yv - (W)mu) / ((W)sigma * (W)sigma);
    }
    if (g) g[0] = (T)gmu;
    return total;
}

// Bernoulli observations of a beta probability (steps: Beta with the logit
// transform, math.jl:161-165, 1150-1155, then the loop of Bernoulli
// observations, math.jl:191-195), every observation scored separately.
template <class T, class W>
W bern_logjoint_grad(const ModelData& m, const T* q, T* g) {
    const ut_plan_desc& pl = m.plan;
    const T u = q[0];
    const T p = T(1) / (T(1) + std::exp(-u));
    const T a = T(pl.prob_alpha), b = T(pl.prob_beta);
    const T lbeta = (T)(std::lgamma(pl.prob_alpha) + std::lgamma(pl.prob_beta) -
                        std::lgamma(pl.prob_alpha + pl.prob_beta));
    const T au = std::fabs(u);
    W total = (p > T(0) && p < T(1)) ? (W)((a - T(1)) * std::log(p) + (b - T(1)) * std::log1p(-p) - lbeta)
                                     : -std::numeric_limits<W>::infinity();
    total += (W)(-au - T(2) * std::log1p(std::exp(-au)));
    W gu = (W)(a - T(1)) * (W(1) - (W)p) - (W)(b - T(1)) * (W)p + W(1) - W(2) * (W)p;
    for (size_t i = 0; i < m.y.size(); ++i) {
        const T z = (T)m.y[i];
        const bool in_support = z == T(0) || z == T(1);
        total += in_support ? (W)(z > T(0.5) ? std::log(p) : std::log1p(-p)) : -std::numeric_limits<W>::infinity();
        gu += z > T(0.5) ? W(1) - (W)p : -(W)p;
    }
    if (g) g[0] = (T)gu;
    return total;
}

// Lognormal log-scale and gamma location (steps: LogNormal on a and Gamma on b,
// both with the log transform, lad = u; math.jl:93-97, 103-107; then the loop
// of Normal(b, exp(a)) observations), every observation scored separately.
template <class T, class W>
W lgn_logjoint_grad(const ModelData& m, const T* q, T* g) {
    const ut_plan_desc& p = m.plan;
    const T ua = q[0], ub = q[1];
    const T a = std::exp(ua), b = std::exp(ub), s = std::exp(a);
    const T lx = std::log(a);
    const T z = (lx - T(p.mu_loc)) / T(p.mu_scale);
    W total = a >= std::numeric_limits<T>::min()
                  ? (W)(-std::log(T(p.mu_scale)) - T(0.9189385332046727) - z * z / T(2) - lx)
                  : -std::numeric_limits<W>::infinity();
    total += (W)ua;
    total += (W)gamma_logpdf<T>(T(p.scale_shape), T(p.scale_rate), b) + (W)ub;
    W ga = -(W)(ua - T(p.mu_loc)) / ((W)p.mu_scale * (W)p.mu_scale);
    W gb = (W)p.scale_shape - (W)p.scale_rate * (W)b;
    const W inv_s2 = W(1) / ((W)s * (W)s);
    for (size_t i = 0; i < m.y.size(); ++i) {
        const T yv = (T)m.y[i];
        total += (W)normal_logpdf<T>(b, s, yv);
        const W r = (W)yv - (W)b;
        ga += (W)a * (-W(1) + r * r * inv_s2);
        gb += (W)b * r * inv_s2;
    }
    if (g) { g[0] = (T)ga; g[1] = (T)gb; }
    return total;
}

// Heavy-tailed location with two scales (steps: StudentT identity, InverseGamma
// and Weibull with the log transform, then the loop of StudentT observations with
// scale s + w; densities as math.jl:167-186, loggamma ratio by the C library in
// double), every observation scored separately.
template <class T>
inline T studentt_logpdf(T nu, T mu, T sigma, T x) {
    const T z = (x - mu) / sigma;
    const T c = (T)(std::lgamma(((double)nu + 1.0) / 2.0) - std::lgamma((double)nu / 2.0));
    return c - (std::log(nu) + T(1.1447298858494002)) / T(2) - std::log(sigma) - (nu + T(1)) * std::log1p(z * z / nu) / T(2);
}

template <class T, class W>
W ht_logjoint_grad(const ModelData& m, const T* q, T* g) {
    const ut_plan_desc& p = m.plan;
    const T loc = q[0], us = q[1], uw = q[2];
    const T s = std::exp(us), w = std::exp(uw), sig = s + w;
    const T nu0 = T(p.nu_prior), mu0 = T(p.mu_loc), s0 = T(p.mu_scale), nu1 = T(p.nu_obs);
    const T a = T(p.scale_shape), b = T(p.scale_rate), k = T(p.weibull_shape), lam = T(p.weibull_scale);
    W total = (W)studentt_logpdf<T>(nu0, mu0, s0, loc);
    const T ig = a * std::log(b) - (T)std::lgamma((double)a) - (a + T(1)) * std::log(s) - b / s;  // math.jl:175-179
    total += (s >= std::numeric_limits<T>::min() ? (W)ig : -std::numeric_limits<W>::infinity()) + (W)us;
    const T wb = std::log(k) + (k - T(1)) * std::log(w) - k * std::log(lam) - std::exp(k * (std::log(w) - std::log(lam)));
    total += (w >= std::numeric_limits<T>::min() ? (W)wb : -std::numeric_limits<W>::infinity()) + (W)uw;
    const W d0 = (W)loc - (W)mu0;
    W gl = -((W)nu0 + 1) * d0 / ((W)nu0 * (W)s0 * (W)s0 + d0 * d0);
    W dsig = 0;
    const W ns2 = (W)nu1 * (W)sig * (W)sig;
    for (size_t i = 0; i < m.y.size(); ++i) {
        const T yv = (T)m.y[i];
        total += (W)studentt_logpdf<T>(nu1, loc, sig, yv);
        const W r = (W)yv - (W)loc, t = r * r;
        gl += ((W)nu1 + 1) * r / (ns2 + t);
        dsig += -W(1) / (W)sig + ((W)nu1 + 1) * t / ((W)sig * (ns2 + t));
    }
    if (g) {
        g[0] = (T)gl;
        g[1] = (T)(-(W)a + (W)b / (W)s + (W)s * dsig);
        g[2] = (T)((W)k - (W)k * std::pow((W)w / (W)lam, (W)k) + (W)w * dsig);
    }
    return total;
}

template <class T, class W>
W logjoint_grad(const ModelData& m, const T* q, T* g) {
    if (m.plan.family == UT_FAMILY_PROGRAM) {  // float64 plan walk, cast to T
        const int P = m.plan.num_params;
        std::vector<double> qd(q, q + P), gd(g ? P : 0);
        const double v = oracle_program::logjoint_grad(m.prog, m.y, qd.data(), g ? gd.data() : nullptr);
        if (g) for (int k = 0; k < P; ++k) g[k] = (T)gd[k];
        return (W)v;
    }
    if (m.plan.family == UT_FAMILY_STUDENTT_HEAVY_TAIL) return ht_logjoint_grad<T, W>(m, q, g);
    if (m.plan.family == UT_FAMILY_LOGNORMAL_GAMMA_NORMAL) return lgn_logjoint_grad<T, W>(m, q, g);
    if (m.plan.family == UT_FAMILY_BERNOULLI_BETA) return bern_logjoint_grad<T, W>(m, q, g);
    if (m.plan.family == UT_FAMILY_GLM_BERNOULLI_LOGIT) return glm_logjoint_grad<T, W>(m, q, g);
    if (m.plan.family == UT_FAMILY_NORMAL_LOCATION_SCALE) return gauss_logjoint_grad<T, W>(m, q, g);
    if (m.plan.family == UT_FAMILY_NORMAL_KNOWN_SCALE) return nks_logjoint_grad<T, W>(m, q, g);
    return hier_logjoint_grad<T, W>(m, q, g);
}

// ---------------------------------------------------------------------------
// Gradient magnitudes (float64): for every gradient element, the sum of the
// absolute values of the terms the gradient adds up, each term's magnitude
// taken over the inputs of its own subtractions (so a term whose FP32 inputs
// cancel keeps the size of those inputs).  An FP32 evaluation of a sum errs by
// a multiple of the unit roundoff times this magnitude, not times the sum
// itself, so it is the scale of the absolute part of the elementwise gradient
// tolerance.  The GLM also carries the error a residual inherits from its
// FP32 linear predictor: sigma'(eta) * sum_f |theta_f x_if| per observation.
// Same terms as the *_logjoint_grad functions above.
// ---------------------------------------------------------------------------
void grad_magnitude(const ModelData& m, const double* q, double* a) {
    const ut_plan_desc& p = m.plan;
    const int P = p.num_params;
    for (int k = 0; k < P; ++k) a[k] = 0.0;
    switch (p.family) {
    case UT_FAMILY_PROGRAM:  // per row: the magnitudes of every contribution to the derivative
        oracle_program::logjoint_grad(m.prog, m.y, q, nullptr, a);
        break;
    case UT_FAMILY_GLM_BERNOULLI_LOGIT: {
        const int N = p.num_obs, D = p.num_coefs, off = p.has_intercept ? 1 : 0;
        const double al = off ? q[0] : 0.0;
        if (off) a[0] += (std::fabs(al) + std::fabs(p.intercept_mu)) / (p.intercept_sigma * p.intercept_sigma);
        for (int d = 0; d < D; ++d)
            a[off + d] += (std::fabs(q[off + d]) + std::fabs(p.coef_mu)) / (p.coef_sigma * p.coef_sigma);
        for (int i = 0; i < N; ++i) {
            const double* x = &m.X[(size_t)i * D];
            double eta = al, A = std::fabs(al);
            for (int d = 0; d < D; ++d) {
                eta += q[off + d] * x[d];
                A += std::fabs(q[off + d] * x[d]);
            }
            const double s = 1.0 / (1.0 + std::exp(-eta));
            const double w = std::fabs(m.y[i] - s) + s * (1.0 - s) * A;
            if (off) a[0] += w;
            for (int d = 0; d < D; ++d) a[off + d] += w * std::fabs(x[d]);
        }
        break;
    }
    case UT_FAMILY_HIER_NORMAL_NONCENTERED: {
        const double mu = q[0], tau = std::exp(q[1]), s2 = p.tau_scale * p.tau_scale;
        a[0] = (std::fabs(mu) + std::fabs(p.mu_loc)) / (p.mu_scale * p.mu_scale);
        a[1] = 1.0 + 2.0 * tau * tau / (s2 + tau * tau);
        for (int j = 0; j < p.num_groups; ++j) {
            const double z = q[2 + j], thm = std::fabs(mu) + std::fabs(tau * z), sj2 = m.sig[j] * m.sig[j];
            double S = 0.0;
            for (int k = 0; k < m.count[j]; ++k) S += (std::fabs(m.y[m.start[j] + k]) + thm) / sj2;
            a[0] += S;
            a[1] += std::fabs(tau * z) * S;
            a[2 + j] = std::fabs(z) + tau * S;
        }
        break;
    }
    case UT_FAMILY_NORMAL_LOCATION_SCALE: {
        const double mu = q[0], s = std::exp(q[1]);
        a[0] = (std::fabs(mu) + std::fabs(p.mu_loc)) / (p.mu_scale * p.mu_scale);
        a[1] = p.scale_shape + p.scale_rate * s;
        for (size_t i = 0; i < m.y.size(); ++i) {
            const double d = std::fabs(m.y[i]) + std::fabs(mu);
            a[0] += d / (s * s);
            a[1] += d * d / (s * s) + 1.0;
        }
        break;
    }
    case UT_FAMILY_NORMAL_KNOWN_SCALE: {
        const double mu = q[0], s2 = p.obs_scale * p.obs_scale;
        a[0] = (std::fabs(mu) + std::fabs(p.mu_loc)) / (p.mu_scale * p.mu_scale);
        for (size_t i = 0; i < m.y.size(); ++i) a[0] += (std::fabs(m.y[i]) + std::fabs(mu)) / s2;
        break;
    }
    case UT_FAMILY_BERNOULLI_BETA: {
        const double pr = 1.0 / (1.0 + std::exp(-q[0]));
        a[0] = std::fabs(p.prob_alpha - 1.0) * (1.0 + pr) + std::fabs(p.prob_beta - 1.0) * pr + 1.0 + 2.0 * pr;
        for (size_t i = 0; i < m.y.size(); ++i) a[0] += m.y[i] > 0.5 ? 1.0 + pr : pr;
        break;
    }
    case UT_FAMILY_LOGNORMAL_GAMMA_NORMAL: {
        const double ea = std::exp(q[0]), b = std::exp(q[1]), s = std::exp(ea);
        a[0] = (std::fabs(q[0]) + std::fabs(p.mu_loc)) / (p.mu_scale * p.mu_scale);
        a[1] = p.scale_shape + p.scale_rate * b;
        for (size_t i = 0; i < m.y.size(); ++i) {
            const double d = std::fabs(m.y[i]) + b;
            a[0] += ea * (1.0 + d * d / (s * s));
            a[1] += b * d / (s * s);
        }
        break;
    }
    case UT_FAMILY_STUDENTT_HEAVY_TAIL: {
        const double loc = q[0], s = std::exp(q[1]), w = std::exp(q[2]), sig = s + w;
        const double nu0 = p.nu_prior, s0 = p.mu_scale, nu1 = p.nu_obs, d0 = loc - p.mu_loc;
        a[0] = (nu0 + 1.0) * (std::fabs(loc) + std::fabs(p.mu_loc)) / (nu0 * s0 * s0 + d0 * d0);
        const double ns2 = nu1 * sig * sig;
        double md = 0.0;
        for (size_t i = 0; i < m.y.size(); ++i) {
            const double r = m.y[i] - loc, t = r * r, ra = std::fabs(m.y[i]) + std::fabs(loc);
            a[0] += (nu1 + 1.0) * ra / (ns2 + t);
            md += 1.0 / sig + (nu1 + 1.0) * ra * ra / (sig * (ns2 + t));
        }
        a[1] = p.scale_shape + p.scale_rate / s + s * md;
        a[2] = p.weibull_shape + p.weibull_shape * std::pow(w / p.weibull_scale, p.weibull_shape) + w * md;
        break;
    }
    default:
        break;
    }
}

// ---------------------------------------------------------------------------
// HMC iteration with Philox randomness (f32).  Momentum p = z / sqrt(M^-1)
// (hmc_support.jl:350-367, persistent_nuts.jl:244-249); leapfrog as
// _device_leapfrog_integrate_perchain! (hmc_kernels.jl:255-287) / host
// batched_leapfrog_trajectory! (integrator.jl:146-220); accept as
// hmc_kernels.jl:553-577 with the uniform from Philox stream 4.
// ---------------------------------------------------------------------------
const uint32_t kStreamMomentum = 0, kStreamDirection = 1, kStreamLeaf = 2, kStreamMerge = 3,
               kStreamAccept = 4;

inline bool all_finite(const float* v, int n) {
    for (int i = 0; i < n; ++i) if (!std::isfinite(v[i])) return false;
    return true;
}

inline float logjoint_grad_f32(const ModelData& m, const float* q, float* g) {
    return (float)logjoint_grad<float, double>(m, q, g);
}

struct ChainTrajectory {
    bool valid;
    float lj1;
};

// Integrates one chain in place: q, p, g hold the start state and receive the
// end state (momentum negated at the end).  Returns validity + end logjoint.
ChainTrajectory leapfrog_chain(const ModelData& m, int P, float* q, float* p, float* g,
                               const float* im, float h, int L) {
    ChainTrajectory r{true, 0.0f};
    float half = 0.5f * h;
    if (!all_finite(g, P)) r.valid = false;                     // validity_init
    if (r.valid) for (int k = 0; k < P; ++k) p[k] += half * g[k];  // half kick
    for (int l = 1; l <= L; ++l) {
        if (r.valid) for (int k = 0; k < P; ++k) q[k] += h * im[k] * p[k];  // drift
        if (!r.valid) break;
        float lj = logjoint_grad_f32(m, q, g);
        if (l < L) {
            if (!all_finite(g, P)) { r.valid = false; break; }
            for (int k = 0; k < P; ++k) p[k] += h * g[k];
        } else {
            if (!all_finite(g, P) || !std::isfinite(lj)) { r.valid = false; break; }
            r.lj1 = lj;
        }
    }
    if (r.valid) for (int k = 0; k < P; ++k) p[k] = -(p[k] + half * g[k]);  // final half kick + flip
    return r;
}

inline float kinetic(const float* p, const float* im, int P) {
    float acc = 0.0f;
    for (int k = 0; k < P; ++k) acc += p[k] * p[k] * im[k];
    return acc / 2.0f;
}

// ---------------------------------------------------------------------------
// Persistent NUTS, one chain (persistent_nuts.jl:226-491), f32.
// ---------------------------------------------------------------------------
inline float logaddexp(float x, float y) {  // persistent_nuts.jl:83-92
    const float ninf = -std::numeric_limits<float>::infinity();
    if (x == ninf) return y;
    if (y == ninf) return x;
    float hi = std::max(x, y);
    return hi + std::log1p(std::exp(std::min(x, y) - hi));
}

// ---------------------------------------------------------------------------
// U-turn criterion and dyadic checkpoints (src/inference/nuts/state_init.jl:296-350,
// src/inference/nuts/tree_expand.jl:57-102; device form persistent_nuts.jl:109-155).
// Velocities are metric-aware: M^-1 p with the diagonal inverse mass `im`.
// ---------------------------------------------------------------------------
template <class T>
bool is_turning(int P, const T* qL, const T* qR, const T* pL, const T* pR, const T* im) {
    T ld = T(0), rd = T(0);
    for (int k = 0; k < P; ++k) {
        const T delta = qR[k] - qL[k];
        ld += delta * im[k] * pL[k];
        rd += delta * im[k] * pR[k];
    }
    return ld <= T(0) || rd <= T(0);
}

// Even leaf: (position, momentum) into checkpoint slot popcount(leaf_index)
// (0-based; the reference's count_ones(leaf_index) + 1).  ckpt holds
// [slot][0 = position, 1 = momentum][P].
template <class T>
void store_tree_checkpoint(int P, T* ckpt, int leaf_index, const T* q, const T* p) {
    const int slot = __builtin_popcount((unsigned)leaf_index);
    for (int k = 0; k < P; ++k) {
        ckpt[((size_t)slot * 2 + 0) * P + k] = q[k];
        ckpt[((size_t)slot * 2 + 1) * P + k] = p[k];
    }
}

// Odd leaf: every dyadic block ending at leaf_index (one per trailing one)
// tested from its start checkpoint to the current endpoint, oriented by the
// direction of the subtree.
template <class T>
bool dyadic_turning(int P, const T* ckpt, int leaf_index, const T* q, const T* p, bool forward, const T* im) {
    const int nt = __builtin_ctz(~(unsigned)leaf_index);  // trailing ones
    for (int kk = 1; kk <= nt; ++kk) {
        const int block_start = leaf_index - (1 << kk) + 1;
        const int slot = __builtin_popcount((unsigned)block_start);
        const T* cq = ckpt + ((size_t)slot * 2 + 0) * P;
        const T* cp = ckpt + ((size_t)slot * 2 + 1) * P;
        const bool turned = forward ? is_turning(P, cq, q, cp, p, im) : is_turning(P, q, cq, p, cp, im);
        if (turned) return true;
    }
    return false;
}

// MEADS persistent-slice drift (api_batched_meads.jl:140): ((u + 1 + delta) mod 2) - 1
// with the floored modulo, so the result stays in [-1, 1).
template <class T>
T meads_slice_drift(T u, T delta) {
    const T x = u + T(1) + delta;
    return (x - T(2) * std::floor(x * T(0.5))) - T(1);
}

struct NutsOut {
    float accept, energy, error;
    int32_t depth, steps;
    uint8_t divergent, moved;
};

NutsOut nuts_chain(const ModelData& m, int P, uint32_t chain, uint32_t iter, float* q, float* g, float& lj,
                   const float* im, float h, int max_depth, float thr) {
    std::vector<float> p(P), q0(P), L(3 * P), R(3 * P), sub(2 * P), prop_pos(P), prop_grad(P),
        ckpt((size_t)(max_depth + 1) * 2 * P);
    float lj3[3];
    float lj0 = lj;
    float kin0 = 0.0f;
    for (int k = 0; k < P; ++k) {  // :243-250
        float z = rand_normal<float>(chain, iter, kStreamMomentum, (uint32_t)k);
        float pk = z / std::sqrt(im[k]);
        p[k] = pk;
        kin0 += pk * pk * im[k];
    }
    float H0 = kin0 / 2.0f - lj0;
    for (int k = 0; k < P; ++k) {  // :255-268
        q0[k] = q[k];
        L[k] = q[k]; L[P + k] = p[k]; L[2 * P + k] = g[k];
        R[k] = q[k]; R[P + k] = p[k]; R[2 * P + k] = g[k];
        prop_pos[k] = q[k]; prop_grad[k] = g[k];
    }
    lj3[0] = lj0; lj3[1] = lj0;
    float prop_lj = lj0;
    auto is_turning_lr = [&]() {  // :109-119
        return is_turning<float>(P, L.data(), R.data(), L.data() + P, R.data() + P, im);
    };
    float cont_w = -H0, accept_sum = 0.0f;
    int accept_count = 0, depth = 1, isteps = 0;
    bool divergent = false, turning = false;
    float prop_energy = H0, prop_error = 0.0f;
    int leaf_counter = 0;

    // first single-leaf trajectory (:284-338)
    float u = rand_uniform<float>(chain, iter, kStreamDirection, 0u);
    float dir = u < 0.5f ? -1.0f : 1.0f;
    bool forward = dir > 0.0f;
    float hs = dir * h, half = hs / 2.0f;
    for (int k = 0; k < P; ++k) {
        p[k] += half * g[k];
        q[k] += hs * (im[k] * p[k]);
    }
    float lj1 = logjoint_grad_f32(m, q, g);
    bool ok1 = std::isfinite(lj1) && all_finite(g, P);
    if (!ok1) {
        divergent = true;
    } else {
        for (int k = 0; k < P; ++k) p[k] += half * g[k];
        float* F = forward ? R.data() : L.data();
        for (int k = 0; k < P; ++k) { F[k] = q[k]; F[P + k] = p[k]; F[2 * P + k] = g[k]; }
        lj3[forward ? 1 : 0] = lj1;
        float pe = kinetic(p.data(), im, P) - lj1;
        float delta = pe - H0;
        isteps = 1;
        if (!std::isfinite(delta) || delta > thr) {
            divergent = true;
        } else {
            float ap = std::min(1.0f, std::exp(std::min(0.0f, -delta)));
            accept_sum += ap; accept_count += 1;
            float cand = -pe;
            float comb = logaddexp(cont_w, cand);
            float ul = rand_uniform<float>(chain, iter, kStreamLeaf, (uint32_t)leaf_counter);
            if (!std::isfinite(cont_w) || std::log(ul) < cand - comb) {
                for (int k = 0; k < P; ++k) { prop_pos[k] = q[k]; prop_grad[k] = g[k]; }
                prop_lj = lj1; prop_energy = pe; prop_error = delta;
            }
            cont_w = comb;
            turning = is_turning_lr();
        }
        leaf_counter += 1;
    }

    // doubling loop (:341-475)
    while (depth < max_depth && !divergent && !turning) {
        int round = depth;
        float ud = rand_uniform<float>(chain, iter, kStreamDirection, (uint32_t)round);
        dir = ud < 0.5f ? -1.0f : 1.0f;
        forward = dir > 0.0f;
        hs = dir * h; half = hs / 2.0f;
        float* F = forward ? R.data() : L.data();
        for (int k = 0; k < P; ++k) { q[k] = F[k]; p[k] = F[P + k]; g[k] = F[2 * P + k]; }
        float cur_lj = lj3[forward ? 1 : 0];
        float sub_w = -std::numeric_limits<float>::infinity();
        int sub_int = 0, sub_acc_n = 0;
        float sub_acc = 0.0f, sub_energy = 0.0f, sub_error = 0.0f;
        bool sub_div = false, sub_turn = false;
        int nleaves = 1 << depth;
        for (int leaf = 0; leaf < nleaves; ++leaf) {
            for (int k = 0; k < P; ++k) {
                p[k] += half * g[k];
                q[k] += hs * (im[k] * p[k]);
            }
            float ljc = logjoint_grad_f32(m, q, g);
            if (!(std::isfinite(ljc) && all_finite(g, P))) { sub_div = true; break; }
            for (int k = 0; k < P; ++k) p[k] += half * g[k];
            cur_lj = ljc;
            sub_int += 1;
            float pe = kinetic(p.data(), im, P) - ljc;
            float delta = pe - H0;
            if (!std::isfinite(delta) || delta > thr) { sub_div = true; break; }
            float ap = std::min(1.0f, std::exp(std::min(0.0f, -delta)));
            sub_acc += ap; sub_acc_n += 1;
            float cand = -pe;
            float comb = logaddexp(sub_w, cand);
            float ul = rand_uniform<float>(chain, iter, kStreamLeaf, (uint32_t)leaf_counter);
            if (!std::isfinite(sub_w) || std::log(ul) < cand - comb) {
                for (int k = 0; k < P; ++k) { sub[k] = q[k]; sub[P + k] = g[k]; }
                lj3[2] = ljc; sub_energy = pe; sub_error = delta;
            }
            sub_w = comb;
            leaf_counter += 1;
            int leaf_index = sub_int - 1;
            if ((leaf_index & 1) == 0) {  // even leaf: checkpoint (:412-417)
                store_tree_checkpoint<float>(P, ckpt.data(), leaf_index, q, p.data());
            } else if (dyadic_turning<float>(P, ckpt.data(), leaf_index, q, p.data(), forward, im)) {
                sub_turn = true;  // odd leaf: dyadic U-turn (:126-155)
                break;
            }
        }
        depth += 1;
        if (sub_int == 0) { divergent = sub_div; break; }
        if (sub_turn || sub_div) {
            isteps += sub_int; accept_sum += sub_acc; accept_count += sub_acc_n;
            turning = sub_turn; divergent = sub_div;
            break;
        }
        for (int k = 0; k < P; ++k) { F[k] = q[k]; F[P + k] = p[k]; F[2 * P + k] = g[k]; }
        lj3[forward ? 1 : 0] = cur_lj;
        float comb_cw = cont_w;
        if (std::isfinite(sub_w)) {
            comb_cw = logaddexp(cont_w, sub_w);
            float um = rand_uniform<float>(chain, iter, kStreamMerge, (uint32_t)round);
            if (std::log(um) < sub_w - cont_w) {
                for (int k = 0; k < P; ++k) { prop_pos[k] = sub[k]; prop_grad[k] = sub[P + k]; }
                prop_lj = lj3[2]; prop_energy = sub_energy; prop_error = sub_error;
            }
        }
        isteps += sub_int; accept_sum += sub_acc; accept_count += sub_acc_n;
        if (std::isfinite(sub_w)) cont_w = comb_cw;
        turning = sub_turn || is_turning_lr();
    }

    NutsOut o;
    o.moved = 0;
    for (int k = 0; k < P; ++k) if (prop_pos[k] != q0[k]) o.moved = 1;
    o.accept = accept_count == 0 ? 0.0f : accept_sum / (float)accept_count;
    o.energy = prop_energy;
    o.error = prop_error;
    o.divergent = divergent ? 1 : 0;
    o.depth = depth;
    o.steps = isteps;
    // host applies the proposal when moved (api_batched_nuts.jl:879-885)
    if (o.moved) {
        for (int k = 0; k < P; ++k) { q[k] = prop_pos[k]; g[k] = prop_grad[k]; }
        lj = prop_lj;
    } else {
        for (int k = 0; k < P; ++k) q[k] = q0[k];
        // gradient at q0: the input gradient, restored from the frontier seed
    }
    return o;
}

int set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
    return omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

}  // namespace

// ===========================================================================
// C entry points (test side)
// ===========================================================================
extern "C" {

void orc_philox4x32(uint32_t k0, uint32_t k1, const uint32_t* ctr, uint32_t* out) {
    Block c = {{ctr[0], ctr[1], ctr[2], ctr[3]}};
    Block r = philox(k0, k1, c);
    for (int i = 0; i < 4; ++i) out[i] = r.w[i];
}

void orc_rand_uniform_f32(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw_start, int64_t n,
                          float* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = rand_uniform<float>(chain, iter, stream, draw_start + (uint32_t)i);
}
void orc_rand_normal_f32(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw_start, int64_t n,
                         float* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = rand_normal<float>(chain, iter, stream, draw_start + (uint32_t)i);
}
void orc_rand_uniform_f64(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw_start, int64_t n,
                          double* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = rand_uniform<double>(chain, iter, stream, draw_start + (uint32_t)i);
}
void orc_rand_normal_f64(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw_start, int64_t n,
                         double* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = rand_normal<double>(chain, iter, stream, draw_start + (uint32_t)i);
}

// Batched logjoint (+ gradient when grads != NULL) in float64.
// params: C x P (chain-major), totals: C, grads: C x P.
int orc_logjoint_gradient_f64(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                              const int32_t* loop_starts, const double* params, int32_t C, double* totals,
                              double* grads, int32_t threads) {
    ModelData m = make_model(plan, observed, trip_counts, loop_starts);
    const int P = plan->num_params;
    set_threads(threads);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < C; ++c) {
        totals[c] = logjoint_grad<double, double>(m, params + (size_t)c * P, grads ? grads + (size_t)c * P : nullptr);
    }
    return 0;
}

// Batched logjoint/gradient in float32 arithmetic with sequential float32
// accumulation over observations (the reference CPU()-backend scan at
// Float32).  This is the timed CPU baseline: chain-parallel over OpenMP
// threads like the reference's threaded batched runtime (batched/workspace.jl:131).
int orc_logjoint_gradient_f32(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                              const int32_t* loop_starts, const float* params, int32_t C, float* totals,
                              float* grads, int32_t threads) {
    ModelData m = make_model(plan, observed, trip_counts, loop_starts);
    const int P = plan->num_params;
    set_threads(threads);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < C; ++c) {
        totals[c] = logjoint_grad<float, float>(m, params + (size_t)c * P, grads ? grads + (size_t)c * P : nullptr);
    }
    return 0;
}

// Gradient magnitudes (see grad_magnitude) in float64; params C x P, out C x P.
int orc_gradient_magnitude_f64(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                               const int32_t* loop_starts, const double* params, int32_t C, double* out,
                               int32_t threads) {
    ModelData m = make_model(plan, observed, trip_counts, loop_starts);
    const int P = plan->num_params;
    set_threads(threads);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < C; ++c) grad_magnitude(m, params + (size_t)c * P, out + (size_t)c * P);
    return 0;
}

// The step program that models of family UT_FAMILY_PROGRAM use from here on
// (their plan carries num_params and the staged row count as num_obs).
void orc_program_set(const ut_program_step* steps, int32_t num_steps, const ut_expr_node* nodes, int32_t num_nodes,
                     int32_t num_slots, int32_t num_params) {
    oracle_program::Program& p = oracle_program::current();
    p.steps.assign(steps, steps + num_steps);
    p.nodes.assign(nodes, nodes + num_nodes);
    p.nslots = num_slots;
    p.P = num_params;
}

int orc_max_threads(void) { return set_threads(0); }

// ---------------------------------------------------------------------------
// MEADS (api_batched_meads.jl): fold parameters in double, the literal
// off-diagonal Gram sum of _meads_max_eig (:48-78); chain updates in float
// with the device's Philox draws (refresh noise: stream 0 at (chain, coord, p)).
// ---------------------------------------------------------------------------
static double meads_max_eig(const std::vector<double>& cols, int P, int N) {  // cols: N x P
    if (N < 2) return 0.0;
    double tr = 0.0;
    for (int n = 0; n < N; ++n)
        for (int d = 0; d < P; ++d) tr += cols[(size_t)n * P + d] * cols[(size_t)n * P + d];
    const double lam = tr / N;
    if (!(lam > 0.0)) return 0.0;
    double off = 0.0;
    for (int a = 0; a < N; ++a)
        for (int b = 0; b < N; ++b) {
            if (a == b) continue;
            double gram = 0.0;
            for (int d = 0; d < P; ++d) gram += cols[(size_t)a * P + d] * cols[(size_t)b * P + d];
            off += gram * gram;
        }
    return (off / ((double)N * (N - 1))) / lam;
}

// cols: N members x P (member-major)
double orc_meads_max_eig(const double* cols, int32_t P, int32_t N) {
    return meads_max_eig(std::vector<double>(cols, cols + (size_t)P * N), P, N);
}

int orc_meads_iteration_f32(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                            const int32_t* loop_starts, int32_t C, int32_t K, int32_t iteration, uint32_t coord,
                            float thr, float* position, float* gradient, float* logjoint, float* momentum,
                            float* slice, float* accept_prob, float* energy, float* energy_error,
                            uint8_t* accepted, uint8_t* divergent, int32_t* steps, float* fold_params) {
    ModelData m = make_model(plan, observed, trip_counts, loop_starts);
    const int P = plan->num_params;
    std::vector<int> start(K), size(K);
    const int base = C / K, rem = C % K;
    for (int f = 0, s0 = 0; f < K; ++f) {  // contiguous folds (:263-276)
        size[f] = base + (f < rem ? 1 : 0);
        start[f] = s0;
        s0 += size[f];
    }
    std::vector<float> sdf((size_t)K * P), eps(K), alpha(K), delta(K);
    for (int f = 0; f < K; ++f) {  // _meads_fold_parameters! (:89-153) from the neighbour's pre-update states
        const int nb = f == 0 ? K - 1 : f - 1, s0 = start[nb], N = size[nb];
        std::vector<double> wp((size_t)N * P), wg((size_t)N * P);
        for (int d = 0; d < P; ++d) {
            double mean = 0.0;
            for (int i = 0; i < N; ++i) mean += position[(size_t)(s0 + i) * P + d];
            mean /= N;
            double var = 0.0;
            for (int i = 0; i < N; ++i) {
                const double x = position[(size_t)(s0 + i) * P + d] - mean;
                var += x * x;
            }
            var /= N;
            double sd = std::sqrt(var);
            sd = sd > 1e-10 ? sd : 1e-10;
            sdf[(size_t)f * P + d] = (float)sd;
            for (int i = 0; i < N; ++i) {
                wp[(size_t)i * P + d] = (position[(size_t)(s0 + i) * P + d] - mean) / sd;
                wg[(size_t)i * P + d] = gradient[(size_t)(s0 + i) * P + d] * sd;
            }
        }
        const double eg = meads_max_eig(wg, P, N), ep = meads_max_eig(wp, P, N);
        const double e = std::min(1.0, 0.5 / std::sqrt(std::max(eg, 1e-12)));
        const double gamma = std::max(1.0 / (iteration * e), 1.0 / std::sqrt(std::max(ep, 1e-12)));
        double a = 1.0 - std::exp(-2.0 * e * gamma);
        a = std::min(std::max(a, 0.0), 1.0);
        eps[f] = (float)e;
        alpha[f] = (float)a;
        delta[f] = (float)(a / 2.0);
        if (fold_params) {
            fold_params[f * 4] = eps[f]; fold_params[f * 4 + 1] = alpha[f];
            fold_params[f * 4 + 2] = delta[f]; fold_params[f * 4 + 3] = 0.0f;
        }
    }
    const int skip = (iteration - 1) % K;
    std::vector<float> q(P), g(P), p(P), mt(P);
    for (int c = 0; c < C; ++c) {
        int f = 0;
        while (!(c >= start[f] && c < start[f] + size[f])) ++f;
        float* mc = momentum + (size_t)c * P;
        if (f == skip) {
            double kin = 0.0;
            for (int d = 0; d < P; ++d) kin += (double)mc[d] * mc[d];
            accept_prob[c] = 1.0f; accepted[c] = 1; divergent[c] = 0; energy_error[c] = 0.0f; steps[c] = 0;
            energy[c] = (float)(0.5 * kin - logjoint[c]);
            continue;
        }
        const float* sd = &sdf[(size_t)f * P];
        const float keep = std::sqrt(std::max(0.0f, 1.0f - alpha[f])), refresh = std::sqrt(std::max(0.0f, alpha[f]));
        double kin0 = 0.0;
        for (int d = 0; d < P; ++d) {
            const float xi = rand_normal<float>((uint32_t)c, coord, kStreamMomentum, (uint32_t)d);
            mt[d] = std::fma(keep, mc[d], refresh * xi);
            p[d] = mt[d] / sd[d];
            kin0 += (double)mt[d] * mt[d];
            q[d] = position[(size_t)c * P + d];
            g[d] = gradient[(size_t)c * P + d];
        }
        const float H0 = (float)(0.5 * kin0) - logjoint[c];
        bool valid = all_finite(g.data(), P);
        const float e = eps[f];
        for (int d = 0; d < P; ++d) {
            p[d] = std::fma(0.5f * e, g[d], p[d]);
            q[d] = std::fma(e * sd[d] * sd[d], p[d], q[d]);
        }
        const float lj1 = logjoint_grad_f32(m, q.data(), g.data());
        valid = valid && all_finite(g.data(), P) && all_finite(q.data(), P) && std::isfinite(lj1);
        double kin1 = 0.0;
        for (int d = 0; d < P; ++d) {
            p[d] = -std::fma(0.5f * e, g[d], p[d]);
            kin1 += (double)p[d] * p[d] * sd[d] * sd[d];
        }
        float lar = -std::numeric_limits<float>::infinity(), ee = std::numeric_limits<float>::infinity();
        bool div = true;
        if (valid) {
            const float H1 = (float)(0.5 * kin1) - lj1;
            lar = H0 - H1;
            ee = H1 - H0;
            div = !std::isfinite(ee) || ee > thr;
        }
        const float ap = std::isnan(lar) ? 0.0f : std::min(1.0f, std::exp(lar));
        const float u = meads_slice_drift<float>(slice[c], delta[f]);  // (:163) floored modulo
        const bool acc = valid && std::log(std::fabs(u)) <= lar;
        double km = 0.0;
        for (int d = 0; d < P; ++d) {
            mc[d] = acc ? -p[d] * sd[d] : -mt[d];
            km += (double)mc[d] * mc[d];
            if (acc) {
                position[(size_t)c * P + d] = q[d];
                gradient[(size_t)c * P + d] = g[d];
            }
        }
        if (acc) logjoint[c] = lj1;
        slice[c] = acc ? u * std::exp(ee) : u;
        accept_prob[c] = ap; accepted[c] = acc ? 1 : 0; divergent[c] = div ? 1 : 0; energy_error[c] = ee;
        steps[c] = 1;
        energy[c] = (float)(0.5 * km) - logjoint[c];
    }
    return 0;
}

// One mean-field ADVI step (f32 arithmetic, the device step's Philox noise at
// (particle j, coord, stream 5, parameter p)): particles, their logjoints, and
// the per-parameter means of grad and grad * scale * eps over particles,
// accumulated in double in particle order (advi_kernels.jl:15-38).
int orc_advi_step_f32(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                      const int32_t* loop_starts, int32_t M, const float* location, const float* scale,
                      uint32_t coord, float* particles, float* values, float* loc_grad, float* scale_grad) {
    ModelData m = make_model(plan, observed, trip_counts, loop_starts);
    const int P = plan->num_params;
    std::vector<float> eps((size_t)M * P), g((size_t)M * P);
    for (int j = 0; j < M; ++j)
        for (int p = 0; p < P; ++p) {
            const float e = rand_normal<float>((uint32_t)j, coord, 5u, (uint32_t)p);
            eps[(size_t)j * P + p] = e;
            particles[(size_t)j * P + p] = std::fma(scale[p], e, location[p]);
        }
    for (int j = 0; j < M; ++j)
        values[j] = logjoint_grad<float, double>(m, particles + (size_t)j * P, g.data() + (size_t)j * P);
    for (int p = 0; p < P; ++p) {
        double a = 0.0, b = 0.0;
        for (int j = 0; j < M; ++j) {
            a += g[(size_t)j * P + p];
            b += (double)g[(size_t)j * P + p] * scale[p] * eps[(size_t)j * P + p];
        }
        loc_grad[p] = (float)(a / M);
        scale_grad[p] = (float)(b / M);
    }
    return 0;
}

// One HMC iteration (f32, Philox randomness).  position/gradient: C x P,
// logjoint/step/outputs: C.  proposal/endpoint_momentum: optional C x P.
int orc_hmc_iteration_f32(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                          const int32_t* loop_starts, int32_t C, float* position, float* gradient,
                          float* logjoint, const float* inverse_mass, const float* step, int32_t L,
                          uint32_t coord, float thr, float* accept_prob, float* energy, float* energy_error,
                          uint8_t* accepted, uint8_t* divergent, float* proposal, float* endpoint_momentum,
                          int32_t threads) {
    ModelData m = make_model(plan, observed, trip_counts, loop_starts);
    const int P = plan->num_params;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int c = 0; c < C; ++c) {
        std::vector<float> q(position + (size_t)c * P, position + (size_t)(c + 1) * P);
        std::vector<float> g(gradient + (size_t)c * P, gradient + (size_t)(c + 1) * P);
        std::vector<float> p(P);
        for (int k = 0; k < P; ++k)
            p[k] = rand_normal<float>((uint32_t)c, coord, kStreamMomentum, (uint32_t)k) / std::sqrt(inverse_mass[k]);
        float H0 = kinetic(p.data(), inverse_mass, P) - logjoint[c];
        ChainTrajectory t = leapfrog_chain(m, P, q.data(), p.data(), g.data(), inverse_mass, step[c], L);
        float H1 = t.valid ? kinetic(p.data(), inverse_mass, P) - t.lj1 : std::numeric_limits<float>::infinity();
        bool acc = false, div = true;
        float ap = 0.0f, ee = std::numeric_limits<float>::infinity();
        if (t.valid) {
            float lar = H0 - H1;
            ee = H1 - H0;
            div = !std::isfinite(ee) || ee > thr;
            ap = !std::isfinite(lar) ? 0.0f : (lar >= 0.0f ? 1.0f : std::exp(lar));  // adaptation.jl:262-269
            float uacc = rand_uniform<float>((uint32_t)c, coord, kStreamAccept, 0u);
            acc = std::log(uacc) < std::min(0.0f, lar);
        }
        accept_prob[c] = ap;
        energy_error[c] = ee;
        accepted[c] = acc ? 1 : 0;
        divergent[c] = div ? 1 : 0;
        energy[c] = acc ? H1 : H0;  // hmc_kernels.jl:674-675
        if (proposal) for (int k = 0; k < P; ++k) proposal[(size_t)c * P + k] = q[k];
        if (endpoint_momentum) for (int k = 0; k < P; ++k) endpoint_momentum[(size_t)c * P + k] = p[k];
        if (acc) {
            for (int k = 0; k < P; ++k) { position[(size_t)c * P + k] = q[k]; gradient[(size_t)c * P + k] = g[k]; }
            logjoint[c] = t.lj1;
        }
    }
    return 0;
}

// One surrogate-driven HMC iteration (f32): the same Philox momentum, leapfrog
// and accept as orc_hmc_iteration_f32, except that every kick (start,
// intermediate, end) uses the MLP surrogate gradient (oracle_mlp, BF16
// rounding points when bf16 != 0) and only the end point's exact logjoint is
// evaluated, for the accept.  No reference counterpart: the project's
// surrogate HMC.  The gradient array is not used.
int orc_surrogate_hmc_iteration_f32(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                                    const int32_t* loop_starts, int32_t C, const float* mlp_weights,
                                    const float* mlp_norm, int32_t bf16, float* position, float* logjoint,
                                    const float* inverse_mass, const float* step, int32_t L, uint32_t coord,
                                    float thr, float* accept_prob, float* energy, float* energy_error,
                                    uint8_t* accepted, uint8_t* divergent, float* proposal,
                                    float* endpoint_momentum, int32_t threads) {
    ModelData m = make_model(plan, observed, trip_counts, loop_starts);
    const int P = plan->num_params;
    const oracle_mlp::Evaluator net(mlp_weights, mlp_norm, P, bf16);
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int c = 0; c < C; ++c) {
        std::vector<float> q(position + (size_t)c * P, position + (size_t)(c + 1) * P);
        std::vector<float> g(P), p(P);
        for (int k = 0; k < P; ++k)
            p[k] = rand_normal<float>((uint32_t)c, coord, kStreamMomentum, (uint32_t)k) / std::sqrt(inverse_mass[k]);
        const float H0 = kinetic(p.data(), inverse_mass, P) - logjoint[c];
        const float h = step[c], half = 0.5f * h;
        bool valid = true;
        float lj1 = 0.0f;
        net(q.data(), g.data());
        if (!all_finite(g.data(), P)) valid = false;
        if (valid) for (int k = 0; k < P; ++k) p[k] += half * g[k];
        for (int l = 1; l <= L && valid; ++l) {
            for (int k = 0; k < P; ++k) q[k] += h * inverse_mass[k] * p[k];
            net(q.data(), g.data());
            if (l < L) {
                if (!all_finite(g.data(), P)) { valid = false; break; }
                for (int k = 0; k < P; ++k) p[k] += h * g[k];
            } else {
                const float lj = (float)logjoint_grad<float, double>(m, q.data(), nullptr);
                if (!all_finite(g.data(), P) || !std::isfinite(lj)) { valid = false; break; }
                lj1 = lj;
            }
        }
        if (valid) for (int k = 0; k < P; ++k) p[k] = -(p[k] + half * g[k]);
        const float H1 = valid ? kinetic(p.data(), inverse_mass, P) - lj1 : std::numeric_limits<float>::infinity();
        bool acc = false, div = true;
        float ap = 0.0f, ee = std::numeric_limits<float>::infinity();
        if (valid) {
            const float lar = H0 - H1;
            ee = H1 - H0;
            div = !std::isfinite(ee) || ee > thr;
            ap = !std::isfinite(lar) ? 0.0f : (lar >= 0.0f ? 1.0f : std::exp(lar));
            const float uacc = rand_uniform<float>((uint32_t)c, coord, kStreamAccept, 0u);
            acc = std::log(uacc) < std::min(0.0f, lar);
        }
        accept_prob[c] = ap;
        energy_error[c] = ee;
        accepted[c] = acc ? 1 : 0;
        divergent[c] = div ? 1 : 0;
        energy[c] = acc ? H1 : H0;
        if (proposal) for (int k = 0; k < P; ++k) proposal[(size_t)c * P + k] = q[k];
        if (endpoint_momentum) for (int k = 0; k < P; ++k) endpoint_momentum[(size_t)c * P + k] = p[k];
        if (acc) {
            for (int k = 0; k < P; ++k) position[(size_t)c * P + k] = q[k];
            logjoint[c] = lj1;
        }
    }
    return 0;
}

// One-step leapfrog probe (adaptation.jl:389-425) with Philox momentum at coord.
int orc_leapfrog_probe_f32(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                           const int32_t* loop_starts, int32_t C, const float* position, const float* gradient,
                           const float* logjoint, const float* inverse_mass, const float* trial_step,
                           uint32_t coord, float* log_accept_ratio, int32_t threads) {
    ModelData m = make_model(plan, observed, trip_counts, loop_starts);
    const int P = plan->num_params;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int c = 0; c < C; ++c) {
        std::vector<float> q(position + (size_t)c * P, position + (size_t)(c + 1) * P);
        std::vector<float> g(gradient + (size_t)c * P, gradient + (size_t)(c + 1) * P);
        std::vector<float> p(P);
        for (int k = 0; k < P; ++k)
            p[k] = rand_normal<float>((uint32_t)c, coord, kStreamMomentum, (uint32_t)k) / std::sqrt(inverse_mass[k]);
        float H0 = kinetic(p.data(), inverse_mass, P) - logjoint[c];
        ChainTrajectory t = leapfrog_chain(m, P, q.data(), p.data(), g.data(), inverse_mass, trial_step[c], 1);
        log_accept_ratio[c] = t.valid ? H0 - (kinetic(p.data(), inverse_mass, P) - t.lj1)
                                      : -std::numeric_limits<float>::infinity();
    }
    return 0;
}

// One persistent-NUTS iteration for C chains (f32).  State arrays C x P / C,
// updated in place with the proposal when moved.
int orc_nuts_iteration_keyed_f32(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                                 const int32_t* loop_starts, int32_t C, uint32_t chain_key_offset, float* position,
                                 float* gradient, float* logjoint, const float* inverse_mass, const float* step,
                                 int32_t max_depth, float thr, uint32_t coord, float* accept_prob, float* energy,
                                 float* energy_error, int32_t* tree_depth, int32_t* integration_steps,
                                 uint8_t* divergent, uint8_t* moved, int32_t threads);

double orc_meads_slice_drift_f64(double u, double delta) { return meads_slice_drift<double>(u, delta); }

// The U-turn helpers in double, for their unit pins.  ckpt: [slots][2][P].
int orc_is_turning_f64(int32_t P, const double* qL, const double* qR, const double* pL, const double* pR,
                       const double* im) {
    return is_turning<double>(P, qL, qR, pL, pR, im) ? 1 : 0;
}

void orc_store_tree_checkpoint_f64(int32_t P, double* ckpt, int32_t leaf_index, const double* q, const double* p) {
    store_tree_checkpoint<double>(P, ckpt, leaf_index, q, p);
}

int orc_dyadic_turning_f64(int32_t P, const double* ckpt, int32_t leaf_index, const double* q, const double* p,
                           int32_t direction, const double* im) {
    return dyadic_turning<double>(P, ckpt, leaf_index, q, p, direction > 0, im) ? 1 : 0;
}

int orc_nuts_iteration_f32(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                           const int32_t* loop_starts, int32_t C, float* position, float* gradient,
                           float* logjoint, const float* inverse_mass, const float* step, int32_t max_depth,
                           float thr, uint32_t coord, float* accept_prob, float* energy, float* energy_error,
                           int32_t* tree_depth, int32_t* integration_steps, uint8_t* divergent, uint8_t* moved,
                           int32_t threads) {
    return orc_nuts_iteration_keyed_f32(plan, observed, trip_counts, loop_starts, C, 0u, position, gradient,
                                        logjoint, inverse_mass, step, max_depth, thr, coord, accept_prob, energy,
                                        energy_error, tree_depth, integration_steps, divergent, moved, threads);
}

// The same with chain c's Philox streams keyed by chain_key_offset + c (a
// model whose chains sit at an offset of a larger batch).
int orc_nuts_iteration_keyed_f32(const ut_plan_desc* plan, const float* observed, const int32_t* trip_counts,
                                 const int32_t* loop_starts, int32_t C, uint32_t chain_key_offset, float* position,
                                 float* gradient, float* logjoint, const float* inverse_mass, const float* step,
                                 int32_t max_depth, float thr, uint32_t coord, float* accept_prob, float* energy,
                                 float* energy_error, int32_t* tree_depth, int32_t* integration_steps,
                                 uint8_t* divergent, uint8_t* moved, int32_t threads) {
    ModelData m = make_model(plan, observed, trip_counts, loop_starts);
    const int P = plan->num_params;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < C; ++c) {
        std::vector<float> g0(gradient + (size_t)c * P, gradient + (size_t)(c + 1) * P);
        float lj = logjoint[c];
        NutsOut o = nuts_chain(m, P, chain_key_offset + (uint32_t)c, coord, position + (size_t)c * P,
                               gradient + (size_t)c * P, lj,
                               inverse_mass, step[c], max_depth, thr);
        if (!o.moved) for (int k = 0; k < P; ++k) gradient[(size_t)c * P + k] = g0[k];
        logjoint[c] = lj;
        accept_prob[c] = o.accept; energy[c] = o.energy; energy_error[c] = o.error;
        tree_depth[c] = o.depth; integration_steps[c] = o.steps;
        divergent[c] = o.divergent; moved[c] = o.moved;
    }
    return 0;
}

// ChEES cross-chain numerator / denominator (api_batched_chees.jl:158-228),
// float64 arithmetic over float32 inputs (C x P arrays).
void orc_chees_reduce(int32_t P, int32_t C, const float* initials, const float* proposals, const float* momenta,
                      const float* accept_prob, const uint8_t* divergent, const float* inverse_mass, double* out) {
    std::vector<double> pm(P, 0.0), im0(P, 0.0);
    double wsum = 0.0;
    int icount = 0;
    auto col_finite = [&](const float* a, int c) {
        for (int k = 0; k < P; ++k) if (!std::isfinite(a[(size_t)c * P + k])) return false;
        return true;
    };
    for (int c = 0; c < C; ++c) {
        if (col_finite(initials, c)) {
            for (int k = 0; k < P; ++k) im0[k] += initials[(size_t)c * P + k];
            icount++;
        }
        if (!divergent[c] && col_finite(proposals, c)) {
            double w = accept_prob[c];
            wsum += w;
            for (int k = 0; k < P; ++k) pm[k] += w * proposals[(size_t)c * P + k];
        }
    }
    if (icount > 0) for (int k = 0; k < P; ++k) im0[k] /= icount;
    double inv = 1.0 / (wsum + 1e-20);
    for (int k = 0; k < P; ++k) pm[k] *= inv;
    double num = 0.0, den = 0.0;
    for (int c = 0; c < C; ++c) {
        if (divergent[c]) continue;
        if (!(col_finite(proposals, c) && col_finite(momenta, c))) continue;
        double pa = accept_prob[c];
        den += pa + 1e-20;
        double se = 0.0, ss = 0.0, ev = 0.0;
        for (int k = 0; k < P; ++k) {
            double sigma = inverse_mass[k];
            double is = 1.0 / std::sqrt(sigma);
            double we = ((double)proposals[(size_t)c * P + k] - pm[k]) * is;
            double ws = ((double)initials[(size_t)c * P + k] - im0[k]) * is;
            double wv = (double)momenta[(size_t)c * P + k] * sigma * is;
            se += we * we; ss += ws * ws; ev += we * wv;
        }
        num += pa * (se - ss) * ev;
    }
    out[0] = num;
    out[1] = den;
}

}  // extern "C"
