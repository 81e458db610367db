// ut_common.cuh -- shared device helpers: Philox4x32-10, the device math of
// the supported families, warp reductions.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define UT_FULL_MASK 0xffffffffu

namespace ut {

// ---------------------------------------------------------------------------
// Philox4x32-10.  Same bijection as the reference (src/device/rng.jl:54-119):
// two 32x32->64 multiply lanes per round, Weyl key bump between rounds.
// __umulhi gives the high word of the product directly on the GPU.
// ---------------------------------------------------------------------------
struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox4x32(uint32_t k0, uint32_t k1, U4 c) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k0 += W0; k1 += W1; }
        uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        U4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
    }
    return c;
}

// key = (chain, iteration), counter = (stream, draw, 0, 0)  (rng.jl:172)
__device__ __forceinline__ U4 coord_block(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw) {
    U4 c = {stream, draw, 0u, 0u};
    return philox4x32(chain, iter, c);
}

// Top 24 bits * 2^-24: exact, in [0, 1 - 2^-24]  (rng.jl:131)
__device__ __forceinline__ float u01(uint32_t w) { return (float)(w >> 8) * 0x1p-24f; }

__device__ __forceinline__ float rand_uniform(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw) {
    return u01(coord_block(chain, iter, stream, draw).x);
}

// Box-Muller from words 1 and 2 of one block (rng.jl:208-213).  logf/cosf are
// CUDA's accurate (non-fast-math) single-precision functions.
__device__ __forceinline__ float rand_normal(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw) {
    U4 b = coord_block(chain, iter, stream, draw);
    float u1 = u01(b.x), u2 = u01(b.y);
    float radius = sqrtf(-2.0f * logf(1.0f - u1));
    return radius * cosf(6.2831855f * u2);
}

// Philox stream ids (persistent_nuts.jl:70-73, plus the HMC accept stream).
constexpr uint32_t kStreamMomentum = 0;
constexpr uint32_t kStreamDirection = 1;
constexpr uint32_t kStreamLeaf = 2;
constexpr uint32_t kStreamMerge = 3;
constexpr uint32_t kStreamAccept = 4;

// ---------------------------------------------------------------------------
// Device math (src/device/math.jl)
// ---------------------------------------------------------------------------
constexpr float kHalfLog2Pi = 0.9189385332046727f;  // log(2 pi) / 2
constexpr float kLog2 = 0.6931471805599453f;
constexpr float kLogPi = 1.1447298858494002f;

__device__ __forceinline__ float normal_logpdf(float mu, float sigma, float x) {  // math.jl:88-91
    float z = (x - mu) / sigma;
    return -logf(sigma) - kHalfLog2Pi - z * z * 0.5f;
}

// log(1 + exp(eta)) without overflow (math.jl:202-203)
__device__ __forceinline__ float log1p_exp(float eta) {
    return eta > 0.0f ? eta + log1pf(expf(-eta)) : log1pf(expf(eta));
}

// x*eta - log1p_exp(eta) on support {0, 1}, else -Inf (math.jl:212-217)
__device__ __forceinline__ float bernoullilogit_logpdf(float eta, float x) {
    float base = x * eta - log1p_exp(eta);
    bool in_support = (x == 0.0f) | (x == 1.0f);
    return in_support ? base : -INFINITY;
}

// logistic(eta) = exp(-log1p_exp(-eta))  (math.jl:224)
__device__ __forceinline__ float logistic(float eta) { return expf(-log1p_exp(-eta)); }

// ---------------------------------------------------------------------------
// Warp reductions (xor butterfly: every lane ends with the full sum, and the
// summation tree is fixed, so results are deterministic).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(UT_FULL_MASK, v, o);
    return v;
}

__device__ __forceinline__ bool warp_all(bool b) { return __all_sync(UT_FULL_MASK, b); }

}  // namespace ut
