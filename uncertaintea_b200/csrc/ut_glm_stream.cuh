// ut_glm_stream.cuh -- batched Bernoulli-logit GLM logjoint + gradient for a
// few chains (C <= 16): an HBM-streaming kernel.
//
// With few chains every element of X is used 2C times (C for eta, C for the
// gradient), so the evaluation is bound by reading X once from HBM.  Every
// warp streams its own 32-row chunks of the row-major X (N x F, F % 4 == 0,
// F <= 128) through a private two-stage cp.async pipeline (16-byte pieces:
// the next chunk is in flight while the current one is used) -- no block-wide
// barrier inside the loop, so the warps of an SM overlap each other's load
// latency and arithmetic.  Per chunk:
//   lane = row      eta_c = x_row . theta_c (theta broadcast from shared
//                   memory), r_c = y - logistic(eta_c), log-likelihood terms;
//   lane = feature  G_c[f4] += sum_rows r_c(row) x_row[f4] (r by warp shuffle,
//   group (of 4)    X rows read as float4, conflict-free).
// At the end the warps' partials are added in warp order into one per-CTA
// partial; glm_stream_fold_kernel folds the CTAs' partials in a fixed order and
// adds the priors (deterministic).
#pragma once

#include "ut_common.cuh"

namespace ut {

constexpr int kStreamRows = 32;      // observations per chunk (one per lane)
constexpr int kStreamMaxC = 16;      // chains
constexpr int kStreamMaxF = 128;     // features (a multiple of 4): one float4 group per lane
constexpr int kStreamStages = 2;  // chunks in flight per warp

struct GlmStreamArgs {
    const float* Xa;      // N x F row-major (ones column first when intercept), F % 4 == 0
    const float* y;       // N
    const float* params;  // C x F
    float* part_ll;       // S x C
    float* part_g;        // S x C x F (only when GRAD)
    int N, F, C;
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Shared memory: theta (CB x F), then per warp kStreamStages x (32 x F X rows
// + 32 y) floats.  After the loop the warp areas hold the warps' partials
// (CB + CB * F floats <= the area since CB <= 16 < 2 * 32).
__host__ __device__ inline size_t glm_stream_warp_floats(int F) {
    return (size_t)kStreamStages * kStreamRows * (F + 1);
}
__host__ __device__ inline size_t glm_stream_smem(int CB, int F, int warps) {
    return sizeof(float) * ((size_t)CB * F + (size_t)warps * glm_stream_warp_floats(F));
}
// Warps per CTA: as many as fit in 220 KB of shared memory (at most 8).
__host__ __device__ inline int glm_stream_warps(int CB, int F) {
    int w = 8;
    while (w > 1 && glm_stream_smem(CB, F, w) > 220 * 1024) --w;
    return w;
}

template <int CB, bool GRAD>
__global__ void __launch_bounds__(256) glm_stream_kernel(GlmStreamArgs a) {
    extern __shared__ __align__(16) float sm[];
    const int F = a.F, F4 = F / 4, N = a.N, C = a.C;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
    float* Th = sm;  // [CB][F]
    for (int i = threadIdx.x; i < CB * F; i += blockDim.x) {
        const int c = i / F, f = i % F;
        Th[i] = c < C ? a.params[(size_t)c * F + f] : 0.0f;
    }
    __syncthreads();
    const size_t wf = glm_stream_warp_floats(F);
    float* Wb = sm + CB * F + warp * wf;  // this warp's stages
    const int nchunks = (N + kStreamRows - 1) / kStreamRows;
    const int gw = blockIdx.x * W + warp, GW = gridDim.x * W;

    auto stage_x = [&](int st) { return Wb + st * kStreamRows * (F + 1); };  // 32 x F rows
    auto stage_y = [&](int st) { return Wb + st * kStreamRows * (F + 1) + kStreamRows * F; };
    auto issue = [&](int chunk, int st) {
        if (chunk < nchunks) {
            const int r0 = chunk * kStreamRows;
            const int nrows = min(kStreamRows, N - r0);
            const float* src = a.Xa + (size_t)r0 * F;
            float* dst = stage_x(st);
            for (int i = lane; i < nrows * F4; i += 32) cp_async16(dst + 4 * i, src + 4 * i);
            if (lane < nrows) cp_async4(stage_y(st) + lane, a.y + r0 + lane);
        }
        cp_async_commit();  // one group per call (empty past the end) keeps the counts exact
    };

    float ll[CB];
    float4 g[CB];
#pragma unroll
    for (int c = 0; c < CB; ++c) {
        ll[c] = 0.0f;
        g[c] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    const float4* Th4 = reinterpret_cast<const float4*>(Th);

    int it = 0;
#pragma unroll
    for (int p = 0; p < kStreamStages - 1; ++p) issue(gw + p * GW, p);  // the pipeline's first chunks
    for (int chunk = gw; chunk < nchunks; chunk += GW, ++it) {
        const int st = it % kStreamStages;
        issue(chunk + (kStreamStages - 1) * GW, (it + kStreamStages - 1) % kStreamStages);
        cp_async_wait<kStreamStages - 1>();
        __syncwarp();
        const int nrows = min(kStreamRows, N - chunk * kStreamRows);
        const float4* X4 = reinterpret_cast<const float4*>(stage_x(st));
        // lane = row: eta (four independent component sums per chain), residual,
        // log-likelihood
        float r[CB];
        {
            float4 e4[CB];
#pragma unroll
            for (int c = 0; c < CB; ++c) e4[c] = make_float4(0.f, 0.f, 0.f, 0.f);
            const bool live = lane < nrows;
            if (live) {
                for (int f4 = 0; f4 < F4; ++f4) {
                    const float4 x = X4[lane * F4 + f4];
#pragma unroll
                    for (int c = 0; c < CB; ++c) {
                        const float4 t = Th4[c * F4 + f4];
                        e4[c].x = fmaf(x.x, t.x, e4[c].x);
                        e4[c].y = fmaf(x.y, t.y, e4[c].y);
                        e4[c].z = fmaf(x.z, t.z, e4[c].z);
                        e4[c].w = fmaf(x.w, t.w, e4[c].w);
                    }
                }
            }
            float e[CB];
#pragma unroll
            for (int c = 0; c < CB; ++c) e[c] = (e4[c].x + e4[c].y) + (e4[c].z + e4[c].w);
            const float yo = live ? stage_y(st)[lane] : 0.0f;
#pragma unroll
            for (int c = 0; c < CB; ++c) {
                const bool use = live && c < C;
                ll[c] += use ? bernoullilogit_logpdf(e[c], yo) : 0.0f;
                r[c] = use ? (yo - logistic(e[c])) : 0.0f;
            }
        }
        // lane = feature group: gradient
        if (GRAD) {
            for (int rr = 0; rr < nrows; ++rr) {
                const float4 x = lane < F4 ? X4[rr * F4 + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int c = 0; c < CB; ++c) {
                    const float rv = __shfl_sync(UT_FULL_MASK, r[c], rr);
                    g[c].x = fmaf(rv, x.x, g[c].x);
                    g[c].y = fmaf(rv, x.y, g[c].y);
                    g[c].z = fmaf(rv, x.z, g[c].z);
                    g[c].w = fmaf(rv, x.w, g[c].w);
                }
            }
        }
        __syncwarp();  // the stage is refilled by the next iteration's issue
    }
    cp_async_wait<0>();  // (only empty groups can remain)

    // per-warp partials into the warp's area, then added in warp order
#pragma unroll
    for (int c = 0; c < CB; ++c) ll[c] = warp_sum(ll[c]);
    float* mine = Wb;  // [CB] ll, then [CB][F] gradient
    if (lane == 0) {
#pragma unroll
        for (int c = 0; c < CB; ++c) mine[c] = ll[c];
    }
    if (GRAD && lane < F4) {
#pragma unroll
        for (int c = 0; c < CB; ++c) {
            float* dst = mine + CB + c * F + 4 * lane;
            dst[0] = g[c].x; dst[1] = g[c].y; dst[2] = g[c].z; dst[3] = g[c].w;
        }
    }
    __syncthreads();
    const int s = blockIdx.x;
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        float t = 0.0f;
        for (int w = 0; w < W; ++w) t += (sm + CB * F + w * wf)[c];
        a.part_ll[(size_t)s * C + c] = t;
    }
    if (GRAD) {
        for (int i = threadIdx.x; i < C * F; i += blockDim.x) {
            float t = 0.0f;
            for (int w = 0; w < W; ++w) t += (sm + CB * F + w * wf)[CB + i];
            a.part_g[(size_t)s * C * F + i] = t;
        }
    }
}

// Fold of the streaming kernel's S per-CTA partials, one 1024-thread CTA per
// chain: thread (s-group g, feature f) adds partials s = g, g + G, ... (G =
// 1024 / Fw groups, Fw = F rounded up to 32) in 4 interleaved accumulators;
// the G group sums are then added in group order, the log-likelihood partials
// likewise by 1024 threads and a fixed tree; the prior terms are added last
// (glm_reduce_kernel's formulas).  Deterministic: every sum's order is fixed.
struct GlmStreamFoldArgs {
    const float* params;
    const float* part_ll;  // S x C
    const float* part_g;   // S x C x F (or null)
    float* totals;
    float* grads;          // C x F (or null)
    int S, C, F, off;
    float icpt_mu, icpt_sigma, coef_mu, coef_sigma;
};

__global__ void __launch_bounds__(1024) glm_stream_fold_kernel(GlmStreamFoldArgs a) {
    __shared__ float part[1024];
    const int c = blockIdx.x, tid = threadIdx.x, F = a.F, S = a.S, C = a.C;
    const int Fw = (F + 31) / 32 * 32;
    const int G = 1024 / Fw;
    float l = 0.0f;
    for (int s = tid; s < S; s += 1024) l += a.part_ll[(size_t)s * C + c];
    part[tid] = l;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if (tid < w) part[tid] += part[tid + w];
        __syncthreads();
    }
    const float ll = part[0];
    __syncthreads();
    const int g = tid / Fw, f = tid % Fw;
    float gs = 0.0f;
    if (a.grads && g < G && f < F) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        int s = g;
        for (; s + 3 * G < S; s += 4 * G) {
#pragma unroll
            for (int u = 0; u < 4; ++u) acc[u] += a.part_g[((size_t)(s + u * G) * C + c) * F + f];
        }
        for (int u = 0; s < S; s += G, ++u) acc[u] += a.part_g[((size_t)s * C + c) * F + f];
        gs = (acc[0] + acc[1]) + (acc[2] + acc[3]);
    }
    if (g < G) part[g * Fw + f] = gs;
    __syncthreads();
    float prior = 0.0f;
    if (tid < F) {
        const float th = a.params[(size_t)c * F + tid];
        const bool icpt = a.off && tid == 0;
        const float mu = icpt ? a.icpt_mu : a.coef_mu, sg = icpt ? a.icpt_sigma : a.coef_sigma;
        prior = normal_logpdf(mu, sg, th);
        if (a.grads) {
            float gsum = 0.0f;
            for (int h = 0; h < G; ++h) gsum += part[h * Fw + tid];
            a.grads[(size_t)c * F + tid] = gsum - (th - mu) / (sg * sg);
        }
    }
    __syncthreads();
    part[tid] = prior;  // priors: a fixed tree over the feature threads
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if (tid < w) part[tid] += part[tid + w];
        __syncthreads();
    }
    if (tid == 0) a.totals[c] = ll + part[0];
}

}  // namespace ut
