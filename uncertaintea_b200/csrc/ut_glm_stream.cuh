// ut_glm_stream.cuh -- batched Bernoulli-logit GLM logjoint + gradient for a
// few chains (C <= 16): an HBM-streaming kernel.
//
// With few chains every element of X is used 2C times (C for eta, C for the
// gradient), so the evaluation is bound by reading X once from HBM.  One CTA
// per SM owns a contiguous range of 32-row chunks of the row-major X
// (N x F, F % 4 == 0, F <= 128) and streams it through a deep ring of
// shared-memory stages filled with plain bulk copies (cp.async.bulk, one per
// chunk for X and one for y, completing on the stage's mbarrier): at launch the
// ring requests most of the CTA's range at once, so the whole GPU has tens of
// MB in flight, and the warps that finish a chunk refill its stage with the
// chunk NS further on (with a warp pair, the first warp after a bounded wait
// for its partner's release).  Every stage belongs to one chunk slot (NS is a
// multiple of the slot count), so a warp only ever waits for the next use of a
// stage after it has consumed the previous one: the mbarrier phase parity it
// waits on is never ambiguous.  Sixteen consumer warps share the chunks: with two or more
// chains a pair of warps takes each chunk, each warp half of the chains (more
// warps per scheduler hide the shared-memory latency, and half the chains keep
// a warp within 120 registers); chunk i goes to warp pair i mod 8 (with one
// chain: warp i mod 16), a fixed assignment, so every sum has a fixed order:
//   lane = row      eta_c = x_row . theta_c (theta broadcast from shared
//                   memory), r_c = y - logistic(eta_c), log-likelihood terms;
//   lane = feature  G_c[f4] += sum_rows r_c(row) x_row[f4] (r broadcast from
//   group (of 4)    shared memory, X rows read as float4, conflict-free);
// then release the stage to the producer.
// The fold is fused: each CTA adds its warps' partials in warp order into a
// per-CTA partial; the last CTA of each group of kStreamGroup CTAs (an atomic
// ticket) folds its group's partials in CTA order; the last group to finish
// folds the group partials in group order and adds the priors.  Deterministic:
// which CTA folds depends on timing, the order of every sum does not.
#pragma once

#include <algorithm>

#include "ut_common.cuh"
#include "ut_tc_glm.cuh"

namespace ut {

constexpr int kStreamRows = 32;       // observations per chunk (one per lane)
constexpr int kStreamMaxC = 16;       // chains
constexpr int kStreamMaxF = 128;      // features (a multiple of 4): one float4 group per lane
constexpr int kStreamWarps = 16;      // consumer warps; they also refill the stages they free
constexpr int kStreamThreads = 32 * kStreamWarps;
constexpr int kStreamGroup = 12;      // CTAs per first-level fold group
constexpr int kStreamMaxStages = 48;
constexpr int kStreamHeader = 1024;   // mbarriers (2 x kStreamMaxStages x 8 B), rounded up

struct GlmStreamArgs {
    const float* Xa;      // N x F row-major (ones column first when intercept), F % 4 == 0, 16-byte aligned
    const float* ypad;    // N rounded up to whole chunks, zero padded
    const float* params;  // C x F
    float* part;          // S x C x Wd  per-CTA partials (Wd = F + 1 with the gradient, else 1): [ll, g_0..g_F-1]
    float* gpart;         // groups x C x Wd
    unsigned* tickets;    // groups + 1 counters, zero between launches
    int* err;             // sticky error word (a bounded wait gave up)
    float* totals;        // C
    float* grads;         // C x F (GRAD)
    int N, F, C, stages, slots, off;  // stages = slots * (stages per slot)
    float icpt_mu, icpt_sigma, coef_mu, coef_sigma;
};

// Chains per consumer warp: a chunk's CB chains are split over CG warps.
__host__ __device__ constexpr int glm_stream_cg(int CB) { return CB >= 2 ? 2 : 1; }
__host__ __device__ constexpr int glm_stream_ch(int CB) { return CB / glm_stream_cg(CB); }

__host__ __device__ inline size_t glm_stream_stage_floats(int F) { return (size_t)kStreamRows * F + kStreamRows; }
// header | theta (CB x F) | residuals (warps x 32 x CH) | stages
__host__ __device__ inline size_t glm_stream_fixed_bytes(int CB, int F) {
    return kStreamHeader +
           sizeof(float) * ((size_t)CB * F + (size_t)kStreamWarps * kStreamRows * glm_stream_ch(CB));
}
__host__ __device__ inline size_t glm_stream_smem(int CB, int F, int stages) {
    return glm_stream_fixed_bytes(CB, F) + sizeof(float) * (size_t)stages * glm_stream_stage_floats(F);
}
inline int glm_stream_groups(int S) { return (S + kStreamGroup - 1) / kStreamGroup; }
// Chunk slots and stages: slots = kStreamWarps / CG when that many stages fit in
// smem_limit bytes (else one per stage that fits), stages = the largest multiple
// of slots that fits, at most kStreamMaxStages.  The ring also holds the warps'
// partials afterwards: 16 x CH x (F + 1) floats <= 4 stages of 32 x (F + 1).
// Returns false when fewer than 4 stages fit.
inline bool glm_stream_plan(int CB, int F, size_t smem_limit, int* stages, int* slots) {
    const size_t fixed = glm_stream_fixed_bytes(CB, F), per = sizeof(float) * glm_stream_stage_floats(F);
    int fit = smem_limit > fixed ? (int)((smem_limit - fixed) / per) : 0;
    fit = std::min(fit, kStreamMaxStages);
    if (fit < 4) return false;
    *slots = std::min(kStreamWarps / glm_stream_cg(CB), fit);
    *stages = fit - fit % *slots;
    return true;
}

template <int CB, bool GRAD>
__global__ void __launch_bounds__(kStreamThreads, 1) glm_stream_kernel(GlmStreamArgs a) {
    constexpr int CG = glm_stream_cg(CB), CH = glm_stream_ch(CB), SLOTS = kStreamWarps / CG;
    extern __shared__ __align__(1024) uint8_t stream_smem[];
    __shared__ int s_last;
    const int F = a.F, F4 = F / 4, N = a.N, C = a.C, NS = a.stages, SL = a.slots;
    const int Wd = GRAD ? F + 1 : 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint64_t* full = reinterpret_cast<uint64_t*>(stream_smem);
    uint64_t* empty = full + kStreamMaxStages;
    float* Th = reinterpret_cast<float*>(stream_smem + kStreamHeader);    // [CB][F]
    float* R = Th + CB * F;                                                // [warps][32][CH]
    float* ring = R + kStreamWarps * kStreamRows * CH;                     // [NS][32 x F X rows, 32 y]
    const size_t stage_floats = glm_stream_stage_floats(F);

    const int NC = (N + kStreamRows - 1) / kStreamRows;
    const int c0 = (int)((long long)blockIdx.x * NC / gridDim.x);
    const int c1 = (int)((long long)(blockIdx.x + 1) * NC / gridDim.x);
    const int n = c1 - c0;

    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, CG);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < CB * F; i += blockDim.x) {
        const int c = i / F, f = i % F;
        Th[i] = c < C ? a.params[(size_t)c * F + f] : 0.0f;
    }
    __syncthreads();

    float ll[CH];
    float4 g[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        ll[c] = 0.0f;
        g[c] = make_float4(0.f, 0.f, 0.f, 0.f);
    }

    // chunk i of this CTA -> slot i % SL, stage slot + SL * ((i / SL) % P), use (i / SL) / P
    const int P = NS / SL;
    auto stage_of = [&](int i) { return i % SL + SL * ((i / SL) % P); };
    auto issue = [&](int i) {
        const int s = stage_of(i);
        const int r0 = (c0 + i) * kStreamRows;
        const int nrows = min(kStreamRows, N - r0);
        float* st = ring + s * stage_floats;
        const uint32_t xbytes = (uint32_t)(nrows * F * 4);
        mbar_expect_tx(full + s, xbytes + kStreamRows * 4);
        bulk_load(st, a.Xa + (size_t)r0 * F, xbytes, full + s);
        bulk_load(st + kStreamRows * F, a.ypad + r0, kStreamRows * 4, full + s);
    };
    if (tid == 0)
        for (int i = 0; i < min(n, NS); ++i) issue(i);
    {
        // ---------------- consumers ----------------
        const int slot = warp % SLOTS, cb0 = (warp / SLOTS) * CH;  // this warp's chunks and chains
        const float4* Th4 = reinterpret_cast<const float4*>(Th + cb0 * F);
        float* Rw = R + warp * kStreamRows * CH;
        for (int i = slot < SL ? slot : n; i < n; i += SL) {  // warps of unused slots stay idle
            const int s = stage_of(i);
            const uint32_t use = (uint32_t)((i / SL) / P);
            if (!mbar_wait(full + s, use & 1, a.err)) break;
            const int nrows = min(kStreamRows, N - (c0 + i) * kStreamRows);
            const float* st = ring + s * stage_floats;
            const float4* X4 = reinterpret_cast<const float4*>(st);
            // lane = row: eta (four independent component sums per chain), residual, log-likelihood
            {
                float4 e4[CH];
#pragma unroll
                for (int c = 0; c < CH; ++c) e4[c] = make_float4(0.f, 0.f, 0.f, 0.f);
                const bool live = lane < nrows;
                if (live) {
                    for (int f4 = 0; f4 < F4; ++f4) {
                        const float4 x = X4[lane * F4 + f4];
#pragma unroll
                        for (int c = 0; c < CH; ++c) {
                            const float4 t = Th4[c * F4 + f4];
                            e4[c].x = fmaf(x.x, t.x, e4[c].x);
                            e4[c].y = fmaf(x.y, t.y, e4[c].y);
                            e4[c].z = fmaf(x.z, t.z, e4[c].z);
                            e4[c].w = fmaf(x.w, t.w, e4[c].w);
                        }
                    }
                }
                const float yo = live ? st[kStreamRows * F + lane] : 0.0f;
                float r[CH];
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    const float e = (e4[c].x + e4[c].y) + (e4[c].z + e4[c].w);
                    const bool use = live && cb0 + c < C;
                    ll[c] += use ? bernoullilogit_logpdf(e, yo) : 0.0f;
                    r[c] = use ? (yo - logistic(e)) : 0.0f;
                }
                if constexpr (CH % 4 == 0) {
#pragma unroll
                    for (int c4 = 0; c4 < CH / 4; ++c4)
                        reinterpret_cast<float4*>(Rw + lane * CH)[c4] =
                            make_float4(r[4 * c4], r[4 * c4 + 1], r[4 * c4 + 2], r[4 * c4 + 3]);
                } else {
#pragma unroll
                    for (int c = 0; c < CH; ++c) Rw[lane * CH + c] = r[c];
                }
            }
            __syncwarp();
            // lane = feature group: gradient
            if (GRAD && lane < F4) {
                for (int rr = 0; rr < nrows; ++rr) {
                    const float4 x = X4[rr * F4 + lane];
                    const float* Rr = Rw + rr * CH;
                    if constexpr (CH % 4 == 0) {
#pragma unroll
                        for (int c4 = 0; c4 < CH / 4; ++c4) {
                            const float4 r = reinterpret_cast<const float4*>(Rr)[c4];
                            const float rv[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                float4& gc = g[4 * c4 + u];
                                gc.x = fmaf(rv[u], x.x, gc.x);
                                gc.y = fmaf(rv[u], x.y, gc.y);
                                gc.z = fmaf(rv[u], x.z, gc.z);
                                gc.w = fmaf(rv[u], x.w, gc.w);
                            }
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < CH; ++c) {
                            const float rv = Rr[c];
                            g[c].x = fmaf(rv, x.x, g[c].x);
                            g[c].y = fmaf(rv, x.y, g[c].y);
                            g[c].z = fmaf(rv, x.z, g[c].z);
                            g[c].w = fmaf(rv, x.w, g[c].w);
                        }
                    }
                }
            }
            __syncwarp();  // the stage and the residual rows are free again
            if (i + NS < n) {
                if constexpr (CG == 1) {
                    if (lane == 0) issue(i + NS);
                } else {
                    if (lane == 0) mbar_arrive(empty + s);
                    if (cb0 == 0) {
                        bool ok = true;
                        if (lane == 0) {
                            ok = mbar_wait(empty + s, use & 1, a.err);
                            if (ok) issue(i + NS);
                        }
                        if (!__shfl_sync(UT_FULL_MASK, ok ? 1 : 0, 0)) break;
                    }
                }
            }
        }
    }
    __syncthreads();  // every chunk consumed: the ring is free

    // warp partials into the ring ([warp][CH][Wd]), then added in chunk-slot order
    if (warp < kStreamWarps) {
        float* mine = ring + (size_t)warp * CH * Wd;
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const float l = warp_sum(ll[c]);
            if (lane == 0) mine[c * Wd] = l;
            if (GRAD && lane < F4) {
                float* dst = mine + c * Wd + 1 + 4 * lane;
                dst[0] = g[c].x; dst[1] = g[c].y; dst[2] = g[c].z; dst[3] = g[c].w;
            }
        }
    }
    __syncthreads();
    const int S = gridDim.x, b = blockIdx.x, CW = C * Wd;
    for (int i = tid; i < CW; i += blockDim.x) {
        const int c = i / Wd, k = i % Wd, w0 = (c / CH) * SLOTS, cl = c % CH;
        float t = 0.0f;
        for (int w = 0; w < SLOTS; ++w) t += ring[(size_t)(w0 + w) * CH * Wd + cl * Wd + k];
        a.part[(size_t)b * CW + i] = t;
    }

    // first-level fold: the last CTA of this group adds the group's partials in CTA
    // order.  The ticket is taken by one thread after the CTA barrier (its fence
    // orders the whole CTA's partial stores before the ticket); every level issues
    // all of its loads before the first add, so a level costs one L2 round trip.
    __syncthreads();
    const int grp = b / kStreamGroup, g0 = grp * kStreamGroup, g1 = min(S, g0 + kStreamGroup);
    if (tid == 0) {
        __threadfence();
        s_last = atomicAdd(a.tickets + grp, 1u) == (unsigned)(g1 - g0 - 1);
        __threadfence();
    }
    __syncthreads();
    if (!s_last) return;
    for (int i = tid; i < CW; i += blockDim.x) {
        float v[kStreamGroup];
#pragma unroll
        for (int q = 0; q < kStreamGroup; ++q) v[q] = g0 + q < g1 ? __ldcg(a.part + (size_t)(g0 + q) * CW + i) : 0.0f;
        float t = v[0];
#pragma unroll
        for (int q = 1; q < kStreamGroup; ++q) t += v[q];
        a.gpart[(size_t)grp * CW + i] = t;
    }
    __syncthreads();
    const int NG = (S + kStreamGroup - 1) / kStreamGroup;
    if (tid == 0) {
        __threadfence();
        s_last = atomicAdd(a.tickets + NG, 1u) == (unsigned)(NG - 1);
        __threadfence();
    }
    __syncthreads();
    if (!s_last) return;

    // second level (one CTA): group partials in group order, then the priors
    float* V = ring;  // [C][Wd]
    for (int i = tid; i < CW; i += blockDim.x) {
        float t = 0.0f;
        for (int q0 = 0; q0 < NG; q0 += 16) {
            float v[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = q0 + q < NG ? __ldcg(a.gpart + (size_t)(q0 + q) * CW + i) : 0.0f;
#pragma unroll
            for (int q = 0; q < 16; ++q) t += v[q];
        }
        V[i] = t;
    }
    __syncthreads();
    for (int c = warp; c < C; c += blockDim.x >> 5) {
        float prior = 0.0f;
        for (int f = lane; f < F; f += 32) {
            const float th = Th[c * F + f];
            const bool icpt = a.off && f == 0;
            const float mu = icpt ? a.icpt_mu : a.coef_mu, sg = icpt ? a.icpt_sigma : a.coef_sigma;
            prior += normal_logpdf(mu, sg, th);
            if (GRAD) a.grads[(size_t)c * F + f] = V[c * Wd + 1 + f] - (th - mu) / (sg * sg);
        }
        prior = warp_sum(prior);
        if (lane == 0) a.totals[c] = V[c * Wd] + prior;
    }
    // every CTA has taken its tickets: reset them for the next launch
    for (int i = tid; i <= NG; i += blockDim.x) a.tickets[i] = 0u;
}

}  // namespace ut
