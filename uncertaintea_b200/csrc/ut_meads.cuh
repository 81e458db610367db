// ut_meads.cuh -- MEADS (generalized HMC with ensemble-adapted step size,
// damping and diagonal preconditioner; the reference's batched_meads,
// src/inference/api_batched_meads.jl:170-547, CPU-only there) with every
// reduction and update on the device.
//
// Chains are split into K contiguous folds; fold f's parameters come from the
// pre-update states of its neighbour fold (f - 1) mod K (api_batched_meads.jl:
// 89-153), fold (t - 1) mod K is left unchanged at iteration t.  Per
// iteration:
//   meads_stats_kernel     per (fold, parameter): mean and population std over
//                          the neighbour's members (two passes, double)
//   meads_moment_kernel    per (fold, which in {whitened states, whitened
//                          gradients}, 16x16 tile of (d, d')): the squared
//                          entries of A = sum_n x_n x_n^T, summed per tile
//   meads_norm_kernel      per (fold, which): sum_n |x_n|^2 and sum_n |x_n|^4
//   meads_params_kernel    per fold: the trace-ratio eigenvalue estimate
//                          lambda2 / lambda with lambda = sum |x_n|^2 / N and
//                          lambda2 = (|A|_F^2 - sum |x_n|^4) / (N (N - 1))
//                          (= the reference's off-diagonal Gram sum, :48-78),
//                          then eps, alpha, delta (:140-152)
//   meads_begin_kernel     warp per chain: partial refresh of the whitened
//                          momentum, half kick, drift (inverse mass = std^2)
//   (batched logjoint + gradient at the drifted positions)
//   meads_end_kernel       half kick, negate, Hamiltonians, persistent-slice
//                          accept (:389-456), state update and the draw's outputs
// Every sum has a fixed order (deterministic).  Draws: the refresh noise from
// Philox stream 0 at (chain, coord, p); the initial momentum and slice from
// streams 0 and 4 at the initial coordinate.
#pragma once

#include "ut_warp_kernels.cuh"

namespace ut {

constexpr double kMeadsStepMargin = 0.5;   // api_batched_meads.jl:32-34
constexpr double kMeadsEigFloor = 1e-12;
constexpr double kMeadsStdFloor = 1e-10;
constexpr int kMeadsTile = 16;

struct MeadsFolds {
    int C, P, K;
    __device__ __forceinline__ int start(int f) const {
        const int base = C / K, rem = C % K;
        return f * base + min(f, rem);
    }
    __device__ __forceinline__ int size(int f) const { return C / K + (f < C % K ? 1 : 0); }
    __device__ __forceinline__ int fold_of(int c) const {
        const int base = C / K, rem = C % K;
        const int big = rem * (base + 1);
        return c < big ? c / (base + 1) : rem + (c - big) / base;
    }
    __device__ __forceinline__ int neighbour(int f) const { return f == 0 ? K - 1 : f - 1; }
};

struct MeadsScratch {
    double* mean;      // K x P  (fold f: statistics of its neighbour's members)
    double* sd;        // K x P
    double* tiles;     // K x 2 x ntiles  per-tile sums of squared A entries
    double* norms;     // K x 2 x 2      sum |x|^2, sum |x|^4
    float* sdf;        // K x P  float copy of sd (sqrt inverse mass)
    float* fold;       // K x 4  eps, alpha, delta, (unused)
    float* refreshed;  // C x P  refreshed whitened momentum
    int ntiles;
};

__device__ __forceinline__ double block_sum_256(double v, double* sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w) sh[t] += sh[t + w];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// grid (P, K), 256 threads
__global__ void __launch_bounds__(256) meads_stats_kernel(MeadsFolds fo, const float* __restrict__ pos,
                                                          MeadsScratch s) {
    __shared__ double sh[256];
    const int d = blockIdx.x, f = blockIdx.y, P = fo.P;
    const int nb = fo.neighbour(f), s0 = fo.start(nb), n = fo.size(nb);
    double a = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) a += (double)pos[(size_t)(s0 + i) * P + d];
    const double mean = block_sum_256(a, sh) / n;
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) {
        const double x = (double)pos[(size_t)(s0 + i) * P + d] - mean;
        v += x * x;
    }
    const double var = block_sum_256(v, sh) / n;
    if (threadIdx.x == 0) {
        double sd = sqrt(var);
        sd = sd > kMeadsStdFloor ? sd : kMeadsStdFloor;
        s.mean[(size_t)f * P + d] = mean;
        s.sd[(size_t)f * P + d] = sd;
        s.sdf[(size_t)f * P + d] = (float)sd;
    }
}

// whitened value of member i (of fold f's neighbour) at parameter d
__device__ __forceinline__ double meads_x(const MeadsFolds& fo, const MeadsScratch& s, const float* pos,
                                          const float* grad, int f, int which, int row, int d) {
    const size_t k = (size_t)f * fo.P + d;
    return which == 0 ? ((double)pos[(size_t)row * fo.P + d] - s.mean[k]) / s.sd[k]
                      : (double)grad[(size_t)row * fo.P + d] * s.sd[k];
}

// grid (tiles_x, tiles_y, 2K), 16 x 16 threads: A[d][d'] for d <= d' in the tile
__global__ void __launch_bounds__(256) meads_moment_kernel(MeadsFolds fo, const float* __restrict__ pos,
                                                           const float* __restrict__ grad, MeadsScratch s) {
    __shared__ double sh[256];
    const int f = blockIdx.z >> 1, which = blockIdx.z & 1, P = fo.P;
    const int d = blockIdx.x * kMeadsTile + threadIdx.x, e = blockIdx.y * kMeadsTile + threadIdx.y;
    const int nb = fo.neighbour(f), s0 = fo.start(nb), n = fo.size(nb);
    double contrib = 0.0;
    if (blockIdx.x <= blockIdx.y && d < P && e < P && d <= e) {
        double a = 0.0;
        for (int i = 0; i < n; ++i)
            a += meads_x(fo, s, pos, grad, f, which, s0 + i, d) * meads_x(fo, s, pos, grad, f, which, s0 + i, e);
        contrib = (d == e ? 1.0 : 2.0) * a * a;
    }
    const int t = threadIdx.y * kMeadsTile + threadIdx.x;
    sh[t] = contrib;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w) sh[t] += sh[t + w];
        __syncthreads();
    }
    if (t == 0) s.tiles[((size_t)f * 2 + which) * s.ntiles + blockIdx.y * gridDim.x + blockIdx.x] = sh[0];
}

// grid (2K), 256 threads
__global__ void __launch_bounds__(256) meads_norm_kernel(MeadsFolds fo, const float* __restrict__ pos,
                                                         const float* __restrict__ grad, MeadsScratch s) {
    __shared__ double sh[256];
    const int f = blockIdx.x >> 1, which = blockIdx.x & 1;
    const int nb = fo.neighbour(f), s0 = fo.start(nb), n = fo.size(nb);
    double a2 = 0.0, a4 = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) {
        double q = 0.0;
        for (int d = 0; d < fo.P; ++d) {
            const double x = meads_x(fo, s, pos, grad, f, which, s0 + i, d);
            q += x * x;
        }
        a2 += q;
        a4 += q * q;
    }
    a2 = block_sum_256(a2, sh);
    a4 = block_sum_256(a4, sh);
    if (threadIdx.x == 0) {
        s.norms[((size_t)f * 2 + which) * 2] = a2;
        s.norms[((size_t)f * 2 + which) * 2 + 1] = a4;
    }
}

// one thread per fold
__global__ void meads_params_kernel(MeadsFolds fo, MeadsScratch s, int iteration) {
    const int f = threadIdx.x;
    if (f >= fo.K) return;
    const int n = fo.size(fo.neighbour(f));
    double eig[2];
    for (int which = 0; which < 2; ++which) {
        const double* nr = s.norms + ((size_t)f * 2 + which) * 2;
        double fro = 0.0;
        for (int t = 0; t < s.ntiles; ++t) fro += s.tiles[((size_t)f * 2 + which) * s.ntiles + t];
        const double lambda = nr[0] / n;
        eig[which] = (n < 2 || !(lambda > 0.0)) ? 0.0 : ((fro - nr[1]) / ((double)n * (n - 1))) / lambda;
    }
    const double eps = fmin(1.0, kMeadsStepMargin / sqrt(fmax(eig[1], kMeadsEigFloor)));
    const double gamma = fmax(1.0 / (iteration * eps), 1.0 / sqrt(fmax(eig[0], kMeadsEigFloor)));
    double alpha = 1.0 - exp(-2.0 * eps * gamma);
    alpha = fmin(fmax(alpha, 0.0), 1.0);
    s.fold[f * 4 + 0] = (float)eps;
    s.fold[f * 4 + 1] = (float)alpha;
    s.fold[f * 4 + 2] = (float)(alpha / 2.0);
    s.fold[f * 4 + 3] = 0.0f;
}

struct MeadsArgs {
    float* position;       // C x P
    float* gradient;       // C x P
    float* logjoint;       // C
    float* momentum;       // C x P  persistent whitened momentum m
    float* slice;          // C      persistent slice variable u in [-1, 1)
    float* accept_prob;    // C
    float* energy;         // C
    float* energy_error;   // C
    uint8_t* accepted;     // C
    uint8_t* divergent;    // C
    int32_t* steps;        // C      1, or 0 for the skipped fold
    int C, P, skip;
    uint32_t coord;
    float thr;
};

template <int K>
__global__ void __launch_bounds__(256) meads_init_kernel(MeadsArgs a) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= a.C) return;
    float m[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int p = lane + 32 * k;
        m[k] = p < a.P ? rand_normal((uint32_t)c, a.coord, kStreamMomentum, (uint32_t)p) : 0.0f;
    }
    store_vec(a.momentum + (size_t)c * a.P, m, a.P);
    if (lane == 0) a.slice[c] = 2.0f * rand_uniform((uint32_t)c, a.coord, kStreamAccept, 0u) - 1.0f;
}

template <int K>
__global__ void __launch_bounds__(256) meads_begin_kernel(MeadsArgs a, MeadsFolds fo, MeadsScratch s,
                                                          LfScratch w) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= a.C) return;
    const int P = a.P, f = fo.fold_of(c);
    const float eps = s.fold[f * 4], alpha = s.fold[f * 4 + 1];
    const float keep = sqrtf(fmaxf(0.0f, 1.0f - alpha)), refresh = sqrtf(fmaxf(0.0f, alpha));
    float q[K], g[K], m[K], sd[K], p[K];
    load_vec(q, a.position + (size_t)c * P, P);
    load_vec(g, a.gradient + (size_t)c * P, P);
    load_vec(m, a.momentum + (size_t)c * P, P);
    load_vec(sd, s.sdf + (size_t)f * P, P);
    float kin = 0.0f;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int pi = lane + 32 * k;
        const float xi = pi < P ? rand_normal((uint32_t)c, a.coord, kStreamMomentum, (uint32_t)pi) : 0.0f;
        m[k] = pi < P ? fmaf(keep, m[k], refresh * xi) : 0.0f;        // refreshed whitened momentum
        p[k] = pi < P ? m[k] / sd[k] : 0.0f;                           // original-coordinate momentum
        kin = fmaf(m[k], m[k], kin);
    }
    store_vec(s.refreshed + (size_t)c * P, m, P);
    const float H0 = 0.5f * warp_sum(kin) - a.logjoint[c];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        p[k] = fmaf(0.5f * eps, g[k], p[k]);
        q[k] = fmaf(eps * sd[k] * sd[k], p[k], q[k]);
    }
    store_vec(w.wq + (size_t)c * P, q, P);
    store_vec(w.wp + (size_t)c * P, p, P);
    if (lane == 0) {
        w.H0[c] = H0;
        w.valid[c] = own_finite(g, P) ? 1 : 0;
    }
}

template <int K>
__global__ void __launch_bounds__(256) meads_end_kernel(MeadsArgs a, MeadsFolds fo, MeadsScratch s, LfScratch w) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= a.C) return;
    const int P = a.P, f = fo.fold_of(c);
    float m[K];
    if (f == a.skip) {  // identity transition (api_batched_meads.jl:431-434, 484-491)
        load_vec(m, a.momentum + (size_t)c * P, P);
        float kin = 0.0f;
#pragma unroll
        for (int k = 0; k < K; ++k) kin = fmaf(m[k], m[k], kin);
        kin = warp_sum(kin);
        if (lane == 0) {
            a.accept_prob[c] = 1.0f;
            a.accepted[c] = 1;
            a.divergent[c] = 0;
            a.energy_error[c] = 0.0f;
            a.steps[c] = 0;
            a.energy[c] = 0.5f * kin - a.logjoint[c];
        }
        return;
    }
    const float eps = s.fold[f * 4], delta = s.fold[f * 4 + 2];
    float q[K], g[K], p[K], sd[K];
    load_vec(q, w.wq + (size_t)c * P, P);
    load_vec(p, w.wp + (size_t)c * P, P);
    load_vec(g, w.wg + (size_t)c * P, P);
    load_vec(sd, s.sdf + (size_t)f * P, P);
    const float lj1 = w.wlj[c];
    bool valid = w.valid[c] != 0 && own_finite(g, P) && own_finite(q, P) && isfinite(lj1);
    float kin = 0.0f;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        p[k] = -fmaf(0.5f * eps, g[k], p[k]);   // final half kick, negated (reversible leapfrog)
        kin = fmaf(p[k] * p[k], sd[k] * sd[k], kin);
    }
    kin = warp_sum(kin);
    const float H0 = w.H0[c];
    float lar = -INFINITY, ee = INFINITY;
    bool div = true;
    if (valid) {
        const float H1 = 0.5f * kin - lj1;
        lar = H0 - H1;
        ee = H1 - H0;
        div = !isfinite(ee) || ee > a.thr;
    }
    const float ap = isnan(lar) ? 0.0f : fminf(1.0f, expf(lar));
    // persistent-slice drift u~ = ((u + 1 + delta) mod 2) - 1 (floored modulo)
    const float x = a.slice[c] + 1.0f + delta;
    const float u = (x - 2.0f * floorf(x * 0.5f)) - 1.0f;
    const bool acc = valid && logf(fabsf(u)) <= lar;
    if (acc) {
#pragma unroll
        for (int k = 0; k < K; ++k) m[k] = -p[k] * sd[k];
        store_vec(a.position + (size_t)c * P, q, P);
        store_vec(a.gradient + (size_t)c * P, g, P);
    } else {
        load_vec(m, s.refreshed + (size_t)c * P, P);
#pragma unroll
        for (int k = 0; k < K; ++k) m[k] = -m[k];
    }
    store_vec(a.momentum + (size_t)c * P, m, P);
    float km = 0.0f;
#pragma unroll
    for (int k = 0; k < K; ++k) km = fmaf(m[k], m[k], km);
    km = warp_sum(km);
    if (lane == 0) {
        if (acc) a.logjoint[c] = lj1;
        a.slice[c] = acc ? u * expf(ee) : u;
        a.accept_prob[c] = ap;
        a.accepted[c] = acc ? 1 : 0;
        a.divergent[c] = div ? 1 : 0;
        a.energy_error[c] = ee;
        a.steps[c] = 1;
        a.energy[c] = 0.5f * km - (acc ? lj1 : a.logjoint[c]);
    }
}

}  // namespace ut
