// ut_glm_tiled.cuh -- batched Bernoulli-logit GLM logjoint + gradient for
// large N, CUDA-core (FP32 FMA) version.
//
// Work decomposition: CTA (chain tile of 64 chains) x (observation split).
// Each CTA keeps its 64 parameter columns in shared memory, streams its
// observation range in chunks of 64 rows, and accumulates
//   eta   = X_chunk . Theta^T            (64 obs x 64 chains)
//   r     = y - logistic(eta),  ll += y*eta - log1p_exp(eta)
//   G    += r^T . X_chunk                 (64 chains x P features)
// in registers.  The intercept is a covariate column of ones (feature 0), so
// one code path covers both GLM forms.  Split partials are folded by a second
// kernel in a fixed order (deterministic, no float atomics), which also adds
// the prior terms -- the reference's tiled prelude/partials/reduce structure
// (src/device/tiled_gradient.jl:180-283) collapsed into one fused pass.
#pragma once

#include "ut_common.cuh"

namespace ut {

constexpr int kGlmCT = 64;   // chains per CTA
constexpr int kGlmOT = 64;   // observations per chunk
constexpr int kGlmXS = kGlmOT + 4;  // padded row stride of the transposed chunk
constexpr int kGlmRS = kGlmCT + 4;  // padded row stride of the residual tile
constexpr int kGlmMaxF = 256;       // max features (P) of the tiled path

struct GlmTiledArgs {
    const float* Xa;      // N x F row-major, F = P (ones column first when intercept)
    const float* y;       // N
    const float* params;  // C x F
    float* part_ll;       // S x C
    float* part_g;        // S x C x F   (only when GRAD)
    int N, F, C;
    int obs_per_split;    // multiple of kGlmOT
};

template <bool GRAD, int FPT>
__global__ void __launch_bounds__(256) glm_tiled_kernel(GlmTiledArgs a) {
    extern __shared__ float sm[];
    float* Th = sm;                         // F x CT   (feature-major)
    float* Xs = Th + a.F * kGlmCT;          // F x XS   (feature-major chunk)
    float* Rs = Xs + a.F * kGlmXS;          // OT x RS
    float* ys = Rs + kGlmOT * kGlmRS;       // OT
    float* red = ys + kGlmOT;               // 16 x CT  (ll reduction)

    const int F = a.F, N = a.N;
    const int c0 = blockIdx.x * kGlmCT;
    const int s = blockIdx.y;
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;  // phase A/B: chains tx*4.., obs ty*4..

    for (int i = tid; i < F * kGlmCT; i += 256) {
        int f = i / kGlmCT, cl = i % kGlmCT;
        int c = c0 + cl;
        Th[f * kGlmCT + cl] = c < a.C ? a.params[(size_t)c * F + f] : 0.0f;
    }

    float llacc[4] = {0.f, 0.f, 0.f, 0.f};
    float gacc[4][FPT];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < FPT; ++j) gacc[i][j] = 0.0f;

    const int obs_begin = s * a.obs_per_split;
    const int obs_end = min(N, obs_begin + a.obs_per_split);
    for (int o0 = obs_begin; o0 < obs_end; o0 += kGlmOT) {
        __syncthreads();
        for (int i = tid; i < kGlmOT * F; i += 256) {
            int o = i / F, f = i % F;
            int n = o0 + o;
            Xs[f * kGlmXS + o] = n < obs_end ? a.Xa[(size_t)n * F + f] : 0.0f;
        }
        for (int o = tid; o < kGlmOT; o += 256) ys[o] = (o0 + o < obs_end) ? a.y[o0 + o] : 0.0f;
        __syncthreads();

        // phase A: eta (4 obs x 4 chains per thread)
        float eta[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) eta[i][j] = 0.0f;
        for (int f = 0; f < F; ++f) {
            float4 xv = *reinterpret_cast<const float4*>(&Xs[f * kGlmXS + ty * 4]);
            float4 tv = *reinterpret_cast<const float4*>(&Th[f * kGlmCT + tx * 4]);
            float xa[4] = {xv.x, xv.y, xv.z, xv.w}, ta[4] = {tv.x, tv.y, tv.z, tv.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) eta[i][j] = fmaf(xa[i], ta[j], eta[i][j]);
        }
        // phase B: residuals + log-likelihood
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int o = ty * 4 + i;
            bool live = (o0 + o) < obs_end;
            float yv = ys[o];
            float r4[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float e = eta[i][j];
                float lp = bernoullilogit_logpdf(e, yv);
                llacc[j] += live ? lp : 0.0f;
                r4[j] = live ? (yv - logistic(e)) : 0.0f;
            }
            if (GRAD) *reinterpret_cast<float4*>(&Rs[o * kGlmRS + tx * 4]) = make_float4(r4[0], r4[1], r4[2], r4[3]);
        }
        if (GRAD) {
            __syncthreads();
            // phase C: G[chain, f] += sum_o r[o, chain] * X[o, f]; chains tx*4.., features ty + 16*j
#pragma unroll 4
            for (int o = 0; o < kGlmOT; ++o) {
                float4 rv = *reinterpret_cast<const float4*>(&Rs[o * kGlmRS + tx * 4]);
                float ra[4] = {rv.x, rv.y, rv.z, rv.w};
#pragma unroll
                for (int j = 0; j < FPT; ++j) {
                    int f = ty + 16 * j;
                    float xv = f < F ? Xs[f * kGlmXS + o] : 0.0f;
#pragma unroll
                    for (int i = 0; i < 4; ++i) gacc[i][j] = fmaf(ra[i], xv, gacc[i][j]);
                }
            }
        }
    }

    // ll: reduce the 16 obs-rows of threads (fixed order)
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) red[ty * kGlmCT + tx * 4 + j] = llacc[j];
    __syncthreads();
    if (tid < kGlmCT) {
        float t = 0.0f;
        for (int r = 0; r < 16; ++r) t += red[r * kGlmCT + tid];
        int c = c0 + tid;
        if (c < a.C) a.part_ll[(size_t)s * a.C + c] = t;
    }
    if (GRAD) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int c = c0 + tx * 4 + i;
            if (c >= a.C) continue;
#pragma unroll
            for (int j = 0; j < FPT; ++j) {
                int f = ty + 16 * j;
                if (f < F) a.part_g[((size_t)s * a.C + c) * F + f] = gacc[i][j];
            }
        }
    }
}

// Fold the S split partials (fixed order) and add the prior terms.
struct GlmReduceArgs {
    const float* params;   // C x F
    const float* part_ll;  // S x C
    const float* part_g;   // S x C x F (or null)
    float* totals;         // C
    float* grads;          // C x F (or null)
    int S, C, F, off;
    float icpt_mu, icpt_sigma, coef_mu, coef_sigma;
};

__global__ void __launch_bounds__(256) glm_reduce_kernel(GlmReduceArgs a) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * 8 + warp;
    if (c >= a.C) return;
    float prior = 0.0f;
    for (int f = lane; f < a.F; f += 32) {
        float th = a.params[(size_t)c * a.F + f];
        bool icpt = a.off && f == 0;
        float mu = icpt ? a.icpt_mu : a.coef_mu, sg = icpt ? a.icpt_sigma : a.coef_sigma;
        prior += normal_logpdf(mu, sg, th);
        if (a.grads) {
            float gsum = 0.0f;
            for (int s = 0; s < a.S; ++s) gsum += a.part_g[((size_t)s * a.C + c) * a.F + f];
            a.grads[(size_t)c * a.F + f] = gsum - (th - mu) / (sg * sg);
        }
    }
    prior = warp_sum(prior);
    if (lane == 0) {
        float t = 0.0f;
        for (int s = 0; s < a.S; ++s) t += a.part_ll[(size_t)s * a.C + c];
        a.totals[c] = t + prior;
    }
}

}  // namespace ut
