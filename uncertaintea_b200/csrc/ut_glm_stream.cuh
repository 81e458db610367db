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

// One CTA's share of one evaluation: load theta (a.params) into shared
// memory, stream this CTA's chunks through the ring, and write the CTA's
// partial sums ([ll, g_0..g_F-1] per chain, summed over its warps in
// chunk-slot order) to a.part[blockIdx.x].  The ring's mbarriers are
// initialised by the first call of a launch (call = 0); a later call (once
// every thread of the CTA has left the previous one) keeps them and offsets
// its wait parities by the phases each stage completed in the earlier calls:
// stage s takes U_s = ceil((n - s) / NS) chunks per call and is released for
// a refill U_s - 1 times.
template <int CB, bool GRAD>
__device__ __forceinline__ void stream_cta_partial(const GlmStreamArgs& a, uint8_t* stream_smem, int call = 0) {
    constexpr int CG = glm_stream_cg(CB), CH = glm_stream_ch(CB), SLOTS = kStreamWarps / CG;
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

    if (tid == 0 && call == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, CG);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < CB * F; i += blockDim.x) {
        const int c = i / F, f = i % F;
        Th[i] = c < C ? __ldcg(a.params + (size_t)c * F + f) : 0.0f;   // L2: another SM may have written it
    }
    // the ring's previous contents were written through the generic proxy (partial
    // sums, a fold's scratch): order them before the bulk copies that refill it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
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
    // phases stage s completed in the earlier calls of this launch (full, empty)
    auto full_base = [&](int s) { return (uint32_t)call * (uint32_t)(s < n ? (n - s + NS - 1) / NS : 0); };
    auto empty_base = [&](int s) { return (uint32_t)call * (uint32_t)(s < n ? (n - s + NS - 1) / NS - 1 : 0); };
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
            if (!mbar_wait(full + s, (full_base(s) + use) & 1, a.err)) break;
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
                            ok = mbar_wait(empty + s, (empty_base(s) + use) & 1, a.err);
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
}

template <int CB, bool GRAD>
__global__ void __launch_bounds__(kStreamThreads, 1) glm_stream_kernel(GlmStreamArgs a) {
    extern __shared__ __align__(1024) uint8_t stream_smem[];
    __shared__ int s_last;
    stream_cta_partial<CB, GRAD>(a, stream_smem);
    const int F = a.F, C = a.C;
    const int Wd = GRAD ? F + 1 : 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float* Th = reinterpret_cast<const float*>(stream_smem + kStreamHeader);    // [CB][F]
    float* ring = reinterpret_cast<float*>(stream_smem + kStreamHeader) + CB * F + kStreamWarps * kStreamRows * glm_stream_ch(CB);
    const int S = gridDim.x, b = blockIdx.x, CW = C * Wd;

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

// ---------------------------------------------------------------------------
// A whole leapfrog trajectory in one launch (few chains).
//
// The batched leapfrog path runs L x [batched gradient -> lf_step_kernel]: at
// a design of 40 MB each evaluation is one launch whose ramp and fold tail
// cost as much as its streaming.  glm_stream_traj_kernel runs the L
// evaluations, and the L - 1 intermediate kicks and drifts between them, in
// one cooperative launch (one CTA per SM, all resident): per step every CTA
// streams its rows (stream_cta_partial), a grid barrier, then CTA c folds
// chain c's per-CTA partials -- in exactly the order of glm_stream_kernel's
// two-level fold, so every value is bit-identical to the step-by-step path --
// adds the prior term, and applies lf_step_kernel's kick and drift; a second
// grid barrier publishes the new positions.  After step L it leaves the
// gradient and logjoint at the final position for lf_step_kernel (l = L),
// which closes the trajectory.  Barrier waits are bounded: one that gives up
// raises the error word and the CTA returns.
// ---------------------------------------------------------------------------
struct GlmTrajArgs {
    GlmStreamArgs s;            // s.params = wq, s.part = per-CTA partials (S x C x (F + 1))
    float* wq;                  // C x F working position
    float* wp;                  // C x F working momentum
    float* wg;                  // C x F gradient at wq
    float* wlj;                 // C     logjoint at wq (written after the last step)
    uint8_t* valid;             // C
    const float* inverse_mass;  // F
    const float* step;          // C
    unsigned* bar;              // [arrivals, generation]: arrivals are 0 between barriers
    int L;
};

// Grid-wide barrier of a cooperative launch.  gen: the generation thread 0
// last saw.  Returns false (error word raised) when the wait gave up.
__device__ __forceinline__ bool stream_grid_sync(unsigned* bar, unsigned& gen, int* err, int* s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned target = gen + 1u;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicExch(bar + 1, target);
        } else {
            const long long t0 = clock64();
            for (unsigned it = 1;; ++it) {
                if (*reinterpret_cast<volatile unsigned*>(bar + 1) == target) break;
                if ((it & 255u) == 0u &&
                    (clock64() - t0 > kTcWaitClocks || *reinterpret_cast<volatile int*>(err))) {
                    atomicCAS(err, 0, 2);   // 2: a grid barrier gave up (1: a ring wait)
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        gen = target;
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

template <int CB>
__global__ void __launch_bounds__(kStreamThreads, 1) glm_stream_traj_kernel(GlmTrajArgs t) {
    extern __shared__ __align__(1024) uint8_t stream_smem[];
    __shared__ int s_ok;
    const GlmStreamArgs& a = t.s;
    const int F = a.F, C = a.C, Wd = F + 1, S = gridDim.x, CW = C * Wd;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int NG = (S + kStreamGroup - 1) / kStreamGroup;
    float* G = reinterpret_cast<float*>(stream_smem + kStreamHeader);  // [NG][Wd] group sums (reuses theta/ring)
    float* V = G + (size_t)NG * Wd;                                     // [Wd] chain totals
    unsigned gen = 0;
    if (tid == 0) gen = *reinterpret_cast<volatile unsigned*>(t.bar + 1);
    const int c = blockIdx.x;  // the chain this CTA folds and steps (c < C)
    bool valid = c < C && __ldcg(t.valid + c) != 0;
    for (int l = 1; l <= t.L; ++l) {
        stream_cta_partial<CB, true>(a, stream_smem, l - 1);
        if (!stream_grid_sync(t.bar, gen, a.err, &s_ok)) return;
        if (c < C) {
            // first level: groups of kStreamGroup CTAs, in CTA order
            for (int idx = tid; idx < NG * Wd; idx += blockDim.x) {
                const int grp = idx / Wd, k = idx % Wd, g0 = grp * kStreamGroup, g1 = min(S, g0 + kStreamGroup);
                float v[kStreamGroup];
#pragma unroll
                for (int q = 0; q < kStreamGroup; ++q)
                    v[q] = g0 + q < g1 ? __ldcg(a.part + (size_t)(g0 + q) * CW + (size_t)c * Wd + k) : 0.0f;
                float sum = v[0];
#pragma unroll
                for (int q = 1; q < kStreamGroup; ++q) sum += v[q];
                G[grp * Wd + k] = sum;
            }
            __syncthreads();
            // second level: the groups in group order
            for (int k = tid; k < Wd; k += blockDim.x) {
                float sum = 0.0f;
                for (int q0 = 0; q0 < NG; q0 += 16) {
                    float v[16];
#pragma unroll
                    for (int q = 0; q < 16; ++q) v[q] = q0 + q < NG ? G[(q0 + q) * Wd + k] : 0.0f;
#pragma unroll
                    for (int q = 0; q < 16; ++q) sum += v[q];
                }
                V[k] = sum;
            }
            __syncthreads();
            // the gradient as glm_stream_kernel writes it (likelihood + prior term)
            const float h = t.step[c];
            bool fin = true;
            for (int f = tid; f < F; f += blockDim.x) {
                const float th = __ldcg(t.wq + (size_t)c * F + f);
                const bool icpt = a.off && f == 0;
                const float mu = icpt ? a.icpt_mu : a.coef_mu, sg = icpt ? a.icpt_sigma : a.coef_sigma;
                const float gv = V[1 + f] - (th - mu) / (sg * sg);
                t.wg[(size_t)c * F + f] = gv;
                fin &= (bool)isfinite(gv);
                if (l < t.L && valid) V[1 + f] = gv;  // kept for the step below
            }
            fin = __syncthreads_and(fin) != 0;
            if (l < t.L) {
                // lf_step_kernel's intermediate step: kick and drift, or the chain turns invalid
                if (valid) {
                    if (!fin) {
                        valid = false;
                    } else {
                        for (int f = tid; f < F; f += blockDim.x) {
                            const float im = t.inverse_mass[f];
                            float p = __ldcg(t.wp + (size_t)c * F + f), q = __ldcg(t.wq + (size_t)c * F + f);
                            p = fmaf(h, V[1 + f], p);
                            q = fmaf(h * im, p, q);
                            t.wp[(size_t)c * F + f] = p;
                            t.wq[(size_t)c * F + f] = q;
                        }
                    }
                }
                if (tid == 0) t.valid[c] = valid ? 1 : 0;
            } else if (warp == 0) {
                // the logjoint at the final position: likelihood + priors, as glm_stream_kernel sums them
                float prior = 0.0f;
                for (int f = lane; f < F; f += 32) {
                    const float th = __ldcg(t.wq + (size_t)c * F + f);
                    const bool icpt = a.off && f == 0;
                    const float mu = icpt ? a.icpt_mu : a.coef_mu, sg = icpt ? a.icpt_sigma : a.coef_sigma;
                    prior += normal_logpdf(mu, sg, th);
                }
                prior = warp_sum(prior);
                if (lane == 0) t.wlj[c] = V[0] + prior;
            }
        }
        if (l < t.L && !stream_grid_sync(t.bar, gen, a.err, &s_ok)) return;
    }
}

}  // namespace ut
