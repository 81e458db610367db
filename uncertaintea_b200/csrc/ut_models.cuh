// ut_models.cuh -- warp-cooperative logjoint + analytic gradient of ONE chain
// for each supported kernel-description family.
//
// A chain's P unconstrained parameters are spread over the 32 lanes of a warp:
// parameter p lives in slot k = p / 32 of lane p % 32.  Every function below is
// called by all 32 lanes with the same chain and returns the same logjoint in
// every lane (warp_sum is an xor butterfly, so all lanes see bit-identical
// sums and control flow that depends on them stays warp-uniform).
#pragma once

#include <cfloat>

#include "ut_common.cuh"

namespace ut {

// Bernoulli-logit GLM (reference steps DeviceBernoulliLogitGLMChoiceStepDyn +
// DeviceDiagNormalChoiceStepDyn; value at logjoint_kernel.jl:378-399, 514-533;
// analytic gradient at gradient_kernel.jl:579-627 and 658-681).
// Observation data is read covariate-major (XT[d * N + i]), so the 32 lanes of
// a warp, which own consecutive observations, read consecutive addresses.
struct GlmModel {
    int N, D, off;  // off = 1 when an intercept row leads the parameters
    float icpt_mu, icpt_sigma, coef_mu, coef_sigma;
    const float* XT;  // D x N (covariate-major), shared memory or global
    const float* y;   // N
};

// Hierarchical non-centred normal (reference semantics of the iid noncentered
// latent, docs/noncentered-reparam.md:22-36; value terms of the Normal /
// HalfCauchy(log) / Noncentered steps, logjoint_kernel.jl:105-129,177-182).
struct HierModel {
    int N, J;
    float mu_loc, mu_scale, tau_scale;
    const float* y;        // N, group after group
    const float* sig;      // J
    const int32_t* start;  // J
    const int32_t* count;  // J
};

// Normal location/scale with a gamma scale (reference gaussian device model:
// Normal + Gamma(log transform) choice steps and a loop of normal observations,
// logjoint_kernel.jl:105-111, 146-151; gamma density math.jl:103-107).
// lgc = shape * log(rate) - loggamma(shape), a constant the host computes.
// known = 1: the observation scale is the constant sigma and mu is the only
// parameter (the reference's conjugate gate model, normal observations with a
// constant scale argument); log_sigma = log(sigma), computed by the host.
struct GaussModel {
    int N;
    float mu_loc, mu_scale, shape, rate, lgc;
    int known;
    float sigma, log_sigma;
    const float* y;  // N
};

// Bernoulli observations of a beta probability (reference device steps: Beta
// with the logit transform, math.jl:161-165, 1150-1155; a loop of Bernoulli
// observations, math.jl:191-195).  lbeta = loggamma(a) + loggamma(b) -
// loggamma(a + b), a constant the host computes.
struct BernModel {
    int N;
    float a, b, lbeta;
    const float* z;  // N
};

// Normal observations with a lognormal log-scale and a gamma location (the
// reference's lognormal/gamma device model: LogNormal and Gamma choice steps
// with the log transform, math.jl:93-97, 103-107, and a loop of Normal
// observations whose scale is exp(a)).  lgc = shape log(rate) - loggamma(shape).
struct LgnModel {
    int N;
    float mu, sigma, shape, rate, lgc;
    const float* y;  // N
};

// Heavy-tailed location with two scales (the reference's heavy-tail device
// model: StudentT (identity), InverseGamma and Weibull (log transform) choice
// steps and a loop of StudentT observations with scale s + w; math.jl:167-186).
// Host constants: c_prior = loggamma((nu0+1)/2) - loggamma(nu0/2)
// - log(nu0 pi)/2 - log(sigma0), c_obs likewise for nu1 without the scale,
// c_ig = a log b - loggamma(a), c_wb = log k - k log lambda.
struct HtModel {
    int N;
    float nu0, mu0, sigma0, nu1, ig_a, ig_b, wb_k, wb_l;
    float c_prior, c_obs, c_ig, c_wb;
    const float* y;  // N
};

// Parameters in per-warp shared memory so every lane can read any coefficient
// with a broadcast load.  `qs` has room for P floats.
template <int K, int DMAX>
__device__ __forceinline__ float glm_lj_grad(const GlmModel& m, int P, const float (&q)[K], float (&g)[K],
                                             float* qs, bool want_grad) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        int p = lane + 32 * k;
        if (p < P) qs[p] = q[k];
    }
    __syncwarp();
    const int D = m.D, off = m.off, N = m.N;
    const float a = off ? qs[0] : 0.0f;
    float gacc[DMAX];
    float gicpt = 0.0f;
#pragma unroll
    for (int d = 0; d < DMAX; ++d) gacc[d] = 0.0f;
    float ll = 0.0f;
    for (int i = lane; i < N; i += 32) {
        float eta = a;
#pragma unroll
        for (int d = 0; d < DMAX; ++d)
            if (d < D) eta = fmaf(qs[off + d], m.XT[(size_t)d * N + i], eta);
        float yv = m.y[i];
        ll += bernoullilogit_logpdf(eta, yv);
        if (want_grad) {
            float r = yv - logistic(eta);
            gicpt += r;
#pragma unroll
            for (int d = 0; d < DMAX; ++d)
                if (d < D) gacc[d] = fmaf(r, m.XT[(size_t)d * N + i], gacc[d]);
        }
    }
    // prior terms by the owner lane of each parameter
    float prior = 0.0f;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        int p = lane + 32 * k;
        if (p < P) {
            if (off && p == 0) prior += normal_logpdf(m.icpt_mu, m.icpt_sigma, q[k]);
            else prior += normal_logpdf(m.coef_mu, m.coef_sigma, q[k]);
        }
    }
    float total = warp_sum(ll + prior);
    if (want_grad) {
        gicpt = warp_sum(gicpt);
#pragma unroll
        for (int d = 0; d < DMAX; ++d)
            if (d < D) gacc[d] = warp_sum(gacc[d]);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            int p = lane + 32 * k;
            float gv = 0.0f;
            if (p < P) {
                if (off && p == 0) {
                    gv = gicpt - (q[k] - m.icpt_mu) / (m.icpt_sigma * m.icpt_sigma);
                } else {
                    int d = p - off;
#pragma unroll
                    for (int dd = 0; dd < DMAX; ++dd)
                        if (dd == d) gv = gacc[dd];
                    gv -= (q[k] - m.coef_mu) / (m.coef_sigma * m.coef_sigma);
                }
            }
            g[k] = gv;
        }
    }
    __syncwarp();
    return total;
}

template <int K>
__device__ __forceinline__ float hier_lj_grad(const HierModel& m, int P, const float (&q)[K], float (&g)[K],
                                              bool want_grad) {
    const int lane = threadIdx.x & 31;
    const float mu = __shfl_sync(UT_FULL_MASK, q[0], 0);
    const float u = __shfl_sync(UT_FULL_MASK, q[0], 1);
    const float tau = expf(u);
    float ll = 0.0f, gmu = 0.0f, gtz = 0.0f;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        int p = lane + 32 * k;
        float gv = 0.0f;
        if (p >= 2 && p < P) {
            int j = p - 2;
            float z = q[k];
            ll += normal_logpdf(0.0f, 1.0f, z);
            float theta = mu + tau * z;
            float sj = m.sig[j];
            float inv_s2 = 1.0f / (sj * sj);
            float ls = -logf(sj) - kHalfLog2Pi;
            float inv_s = 1.0f / sj;
            float dtheta = 0.0f, sq = 0.0f;
            const int s0 = m.start[j], n = m.count[j];
            for (int t = 0; t < n; ++t) {
                float r = m.y[s0 + t] - theta;
                sq = fmaf(r, r, sq);
                dtheta += r;
            }
            // sum_t normal_logpdf(theta, sj, y_t) = n*ls - sq/(2 sj^2)
            ll += (float)n * ls - 0.5f * sq * inv_s * inv_s;
            dtheta *= inv_s2;
            gmu += dtheta;
            gtz += z * dtheta;
            gv = -z + tau * dtheta;
        }
        g[k] = gv;
    }
    float prior = 0.0f;
    if (lane == 0) prior += normal_logpdf(m.mu_loc, m.mu_scale, mu);
    if (lane == 1) {
        float z = tau / m.tau_scale;
        prior += kLog2 - kLogPi - logf(m.tau_scale) - log1pf(z * z) + u;  // halfcauchy + log|J| = u
    }
    float total = warp_sum(ll + prior);
    if (want_grad) {
        gmu = warp_sum(gmu);
        gtz = warp_sum(gtz);
        if (lane == 0) g[0] = gmu - (mu - m.mu_loc) / (m.mu_scale * m.mu_scale);
        if (lane == 1) {
            float s2 = m.tau_scale * m.tau_scale;
            g[0] = 1.0f - 2.0f * tau * tau / (s2 + tau * tau) + tau * gtz;
        }
    }
    return total;
}

// Two parameters: lane 0 holds mu, lane 1 holds u = log s.  The observation
// loop accumulates sum (y - mu) and sum (y - mu)^2 over the warp's lanes:
//   sum_i normal_logpdf(mu, s, y_i) = N (-log s - log(2 pi) / 2) - sq / (2 s^2),
//   d/dmu = sum (y - mu) / s^2,   d/du = -N + sq / s^2 (chain rule ds/du = s);
// the gamma prior on s with log|J| = u adds (shape - 1) u - rate s + u + lgc,
// d/du = shape - rate s; -Inf when s is not a positive normal float (math.jl:66).
template <int K>
__device__ __forceinline__ float gauss_lj_grad(const GaussModel& m, const float (&q)[K], float (&g)[K],
                                               bool want_grad) {
    const int lane = threadIdx.x & 31;
    const float mu = __shfl_sync(UT_FULL_MASK, q[0], 0);
    const float u = m.known ? m.log_sigma : __shfl_sync(UT_FULL_MASK, q[0], 1);
    const float s = m.known ? m.sigma : expf(u);
    float sr = 0.0f, sq = 0.0f;
    for (int i = lane; i < m.N; i += 32) {
        const float r = m.y[i] - mu;
        sr += r;
        sq = fmaf(r, r, sq);
    }
    sr = warp_sum(sr);
    sq = warp_sum(sq);
    const float inv_s = 1.0f / s;
    const float nf = (float)m.N;
    float lj = nf * (-u - kHalfLog2Pi) - 0.5f * sq * inv_s * inv_s;
    lj += normal_logpdf(m.mu_loc, m.mu_scale, mu);
    if (!m.known) lj += s >= FLT_MIN ? m.lgc + (m.shape - 1.0f) * u - m.rate * s + u : -INFINITY;
    if (want_grad) {
#pragma unroll
        for (int k = 0; k < K; ++k) g[k] = 0.0f;
        if (lane == 0) g[0] = sr * inv_s * inv_s - (mu - m.mu_loc) / (m.mu_scale * m.mu_scale);
        if (lane == 1 && !m.known) g[0] = -nf + sq * inv_s * inv_s + m.shape - m.rate * s;
    }
    return lj;
}

// One parameter u = logit p in lane 0.  The observation loop counts ones,
// zeros and values outside {0, 1} (which score -Inf):
//   sum_i bernoulli(p, z_i) = S log p + (n - S) log1p(-p),
//   d/du = S - n p;  beta prior (a-1) log p + (b-1) log1p(-p) - lbeta,
//   d/du = (a-1)(1-p) - (b-1) p;  log|J| = -|u| - 2 log1p(exp(-|u|)),
//   d/du = 1 - 2p.  -Inf when p is not strictly inside (0, 1).
template <int K>
__device__ __forceinline__ float bern_lj_grad(const BernModel& m, const float (&q)[K], float (&g)[K],
                                              bool want_grad) {
    const int lane = threadIdx.x & 31;
    const float u = __shfl_sync(UT_FULL_MASK, q[0], 0);
    float ones = 0.0f, zeros = 0.0f, bad = 0.0f;
    for (int i = lane; i < m.N; i += 32) {
        const float zv = m.z[i];
        ones += zv == 1.0f ? 1.0f : 0.0f;
        zeros += zv == 0.0f ? 1.0f : 0.0f;
        bad += (zv == 0.0f || zv == 1.0f) ? 0.0f : 1.0f;
    }
    ones = warp_sum(ones);
    zeros = warp_sum(zeros);
    bad = warp_sum(bad);
    const float p = 1.0f / (1.0f + expf(-u));
    const float lp = logf(p), l1p = log1pf(-p);
    const float au = fabsf(u);
    // A count of zero contributes nothing, even where its log is -inf: at the
    // float32 logit cliff (|u| >= ~17, p rounds to 0 or 1) 0 * -inf would be
    // NaN; the value there is the prior's -inf, as the reference scores it.
    float lj = (ones > 0.0f ? ones * lp : 0.0f) + (zeros > 0.0f ? zeros * l1p : 0.0f);
    lj += (p > 0.0f && p < 1.0f) ? (m.a - 1.0f) * lp + (m.b - 1.0f) * l1p - m.lbeta : -INFINITY;
    lj += -au - 2.0f * log1pf(expf(-au));
    if (bad > 0.0f) lj = -INFINITY;
    if (want_grad) {
#pragma unroll
        for (int k = 0; k < K; ++k) g[k] = 0.0f;
        if (lane == 0) g[0] = ones + m.a - (ones + zeros + m.a + m.b) * p;
    }
    return lj;
}

// Lane 0 holds ua = log a, lane 1 ub = log b; s = exp(a), log s = a:
//   sum_i normal_logpdf(b, s, y_i) = N (-a - log(2 pi) / 2) - sq / (2 s^2),
//   d/dua = a (-N + sq / s^2) - (ua - mu) / sigma^2   (lognormal + log|J| = ua),
//   d/dub = b sr / s^2 + shape - rate b               (gamma + log|J| = ub).
template <int K>
__device__ __forceinline__ float lgn_lj_grad(const LgnModel& m, const float (&q)[K], float (&g)[K],
                                             bool want_grad) {
    const int lane = threadIdx.x & 31;
    const float ua = __shfl_sync(UT_FULL_MASK, q[0], 0);
    const float ub = __shfl_sync(UT_FULL_MASK, q[0], 1);
    const float a = expf(ua), b = expf(ub);
    const float s = expf(a);
    float sr = 0.0f, sq = 0.0f;
    for (int i = lane; i < m.N; i += 32) {
        const float r = m.y[i] - b;
        sr += r;
        sq = fmaf(r, r, sq);
    }
    sr = warp_sum(sr);
    sq = warp_sum(sq);
    const float inv_s2 = 1.0f / (s * s);
    const float nf = (float)m.N;
    float lj = nf * (-a - kHalfLog2Pi) - 0.5f * sq * inv_s2;
    const float z = (ua - m.mu) / m.sigma;
    lj += a >= FLT_MIN ? -logf(m.sigma) - kHalfLog2Pi - 0.5f * z * z : -INFINITY;  // lognormal - log a + log|J|
    lj += b >= FLT_MIN ? m.lgc + (m.shape - 1.0f) * ub - m.rate * b + ub : -INFINITY;
    if (want_grad) {
#pragma unroll
        for (int k = 0; k < K; ++k) g[k] = 0.0f;
        if (lane == 0) g[0] = a * (-nf + sq * inv_s2) - z / m.sigma;
        if (lane == 1) g[0] = b * sr * inv_s2 + m.shape - m.rate * b;
    }
    return lj;
}

// Lanes 0, 1, 2 hold loc, us = log s, uw = log w; sigma = s + w.  Per
// observation r = y - loc, t = r^2:
//   sum_i studentt = N (c_obs - log sigma) - (nu1+1)/2 sum log1p(t / (nu1 sigma^2)),
//   d/dloc = (nu1+1) sum r / (nu1 sigma^2 + t),
//   d/dsigma = -N / sigma + (nu1+1) / sigma sum t / (nu1 sigma^2 + t);
// priors with log|J|: d/dloc of studentt = -(nu0+1)(loc-mu0)/(nu0 sigma0^2 + (loc-mu0)^2),
// inverse gamma + us: d/dus = -a + b / s, weibull + uw: d/duw = k - k (w/lambda)^k.
template <int K>
__device__ __forceinline__ float ht_lj_grad(const HtModel& m, const float (&q)[K], float (&g)[K],
                                            bool want_grad) {
    const int lane = threadIdx.x & 31;
    const float loc = __shfl_sync(UT_FULL_MASK, q[0], 0);
    const float us = __shfl_sync(UT_FULL_MASK, q[0], 1);
    const float uw = __shfl_sync(UT_FULL_MASK, q[0], 2);
    const float s = expf(us), w = expf(uw);
    const float sig = s + w;
    const float ns2 = m.nu1 * sig * sig;
    float a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
    for (int i = lane; i < m.N; i += 32) {
        const float r = m.y[i] - loc;
        const float t = r * r;
        const float den = 1.0f / (ns2 + t);
        a1 += log1pf(t / ns2);
        a2 += r * den;
        a3 += t * den;
    }
    a1 = warp_sum(a1);
    a2 = warp_sum(a2);
    a3 = warp_sum(a3);
    const float nf = (float)m.N;
    float lj = nf * (m.c_obs - logf(sig)) - 0.5f * (m.nu1 + 1.0f) * a1;
    const float d0 = loc - m.mu0, z = d0 / m.sigma0;
    lj += m.c_prior - 0.5f * (m.nu0 + 1.0f) * log1pf(z * z / m.nu0);
    lj += s >= FLT_MIN ? m.c_ig - (m.ig_a + 1.0f) * us - m.ig_b / s + us : -INFINITY;
    const float wl = expf(m.wb_k * (uw - logf(m.wb_l)));  // (w / lambda)^k
    lj += w >= FLT_MIN ? m.c_wb + (m.wb_k - 1.0f) * uw - wl + uw : -INFINITY;
    if (want_grad) {
        const float dsig = -nf / sig + (m.nu1 + 1.0f) * a3 / sig;
#pragma unroll
        for (int k = 0; k < K; ++k) g[k] = 0.0f;
        if (lane == 0) g[0] = (m.nu1 + 1.0f) * a2 - (m.nu0 + 1.0f) * d0 / (m.nu0 * m.sigma0 * m.sigma0 + d0 * d0);
        if (lane == 1) g[0] = -m.ig_a + m.ig_b / s + s * dsig;
        if (lane == 2) g[0] = m.wb_k - m.wb_k * wl + w * dsig;
    }
    return lj;
}

}  // namespace ut
