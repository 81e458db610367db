// ut_warp_kernels.cuh -- warp-per-chain kernels: batched density, fused HMC
// iteration, leapfrog probe and the persistent NUTS tree.  One warp owns one
// chain; the chain's vectors live in registers (K slots per lane), the model's
// observation data is staged once per CTA into shared memory and shared by all
// of the CTA's chains.
#pragma once

#include "ut_models.cuh"
#include "ut_program.cuh"

namespace ut {

enum Family : int { kFamGlm = 1, kFamHier = 2, kFamGauss = 3, kFamBern = 4, kFamLgn = 5, kFamHt = 6, kFamProg = 7 };

struct DevModel {
    int family;
    int P;
    int Ppad;           // per-warp scratch stride (floats), multiple of 32
    int stage;          // 1 = copy observation data into shared memory
    int staged_floats;  // floats of staged data at the head of dynamic smem
    GlmModel glm;
    HierModel hier;
    GaussModel gauss;
    BernModel bern;
    LgnModel lgn;
    HtModel ht;
    ProgModel prog;   // the step program (ut_program.cuh)
};

// Copies the model's observation data into shared memory (when dm.stage) and
// points the model at it.  Called by every thread of the CTA.
template <int FAM>
__device__ __forceinline__ void stage_model(DevModel& dm, float* smem) {
    if (!dm.stage) return;
    if constexpr (FAM == kFamGlm) {
        const int n = dm.glm.N * dm.glm.D;
        const float4* src = reinterpret_cast<const float4*>(dm.glm.XT);
        float4* dst = reinterpret_cast<float4*>(smem);
        const int n4 = n / 4;  // host pads the device copy to a multiple of 4
        for (int i = threadIdx.x; i < n4; i += blockDim.x) dst[i] = src[i];
        for (int i = 4 * n4 + threadIdx.x; i < n; i += blockDim.x) smem[i] = dm.glm.XT[i];
        float* ys = smem + n;
        for (int i = threadIdx.x; i < dm.glm.N; i += blockDim.x) ys[i] = dm.glm.y[i];
        __syncthreads();
        dm.glm.XT = smem;
        dm.glm.y = ys;
    } else if constexpr (FAM == kFamGauss) {
        for (int i = threadIdx.x; i < dm.gauss.N; i += blockDim.x) smem[i] = dm.gauss.y[i];
        __syncthreads();
        dm.gauss.y = smem;
    } else if constexpr (FAM == kFamHt) {
        for (int i = threadIdx.x; i < dm.ht.N; i += blockDim.x) smem[i] = dm.ht.y[i];
        __syncthreads();
        dm.ht.y = smem;
    } else if constexpr (FAM == kFamLgn) {
        for (int i = threadIdx.x; i < dm.lgn.N; i += blockDim.x) smem[i] = dm.lgn.y[i];
        __syncthreads();
        dm.lgn.y = smem;
    } else if constexpr (FAM == kFamBern) {
        for (int i = threadIdx.x; i < dm.bern.N; i += blockDim.x) smem[i] = dm.bern.z[i];
        __syncthreads();
        dm.bern.z = smem;
    } else if constexpr (FAM == kFamProg) {
        // observations, then the compiled nodes and steps (all 4-byte words)
        ProgModel& m = dm.prog;
        float* o = smem;
        PNode* nd = reinterpret_cast<PNode*>(smem + ((m.nobs + 3) / 4) * 4);
        PStep* st = reinterpret_cast<PStep*>(nd + m.nnodes);
        for (int i = threadIdx.x; i < m.nobs; i += blockDim.x) o[i] = m.obs[i];
        const int nw = m.nnodes * (int)(sizeof(PNode) / 4), sw = m.nsteps * (int)(sizeof(PStep) / 4);
        for (int i = threadIdx.x; i < nw; i += blockDim.x)
            reinterpret_cast<int*>(nd)[i] = reinterpret_cast<const int*>(m.nodes)[i];
        for (int i = threadIdx.x; i < sw; i += blockDim.x)
            reinterpret_cast<int*>(st)[i] = reinterpret_cast<const int*>(m.steps)[i];
        __syncthreads();
        m.obs = o;
        m.nodes = nd;
        m.steps = st;
    } else {
        const int N = dm.hier.N, J = dm.hier.J;
        float* ys = smem;
        float* ss = smem + N;
        int32_t* st = reinterpret_cast<int32_t*>(smem + N + J);
        int32_t* ct = st + J;
        for (int i = threadIdx.x; i < N; i += blockDim.x) ys[i] = dm.hier.y[i];
        for (int i = threadIdx.x; i < J; i += blockDim.x) {
            ss[i] = dm.hier.sig[i];
            st[i] = dm.hier.start[i];
            ct[i] = dm.hier.count[i];
        }
        __syncthreads();
        dm.hier.y = ys;
        dm.hier.sig = ss;
        dm.hier.start = st;
        dm.hier.count = ct;
    }
}

template <int FAM, int K, int DMAX>
__device__ __forceinline__ float eval_lj(const DevModel& dm, const float (&q)[K], float (&g)[K], float* qs,
                                         bool want_grad) {
    if constexpr (FAM == kFamGlm) return glm_lj_grad<K, DMAX>(dm.glm, dm.P, q, g, qs, want_grad);
    else if constexpr (FAM == kFamGauss) return gauss_lj_grad<K>(dm.gauss, q, g, want_grad);
    else if constexpr (FAM == kFamBern) return bern_lj_grad<K>(dm.bern, q, g, want_grad);
    else if constexpr (FAM == kFamLgn) return lgn_lj_grad<K>(dm.lgn, q, g, want_grad);
    else if constexpr (FAM == kFamHt) return ht_lj_grad<K>(dm.ht, q, g, want_grad);
    else if constexpr (FAM == kFamProg) return prog_lj_grad<K>(dm.prog, q, g, qs, want_grad);
    else return hier_lj_grad<K>(dm.hier, dm.P, q, g, want_grad);
}

template <int K>
__device__ __forceinline__ bool own_finite(const float (&v)[K], int P) {
    const int lane = threadIdx.x & 31;
    bool ok = true;
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (lane + 32 * k < P) ok &= isfinite(v[k]);
    return warp_all(ok);
}

template <int K>
__device__ __forceinline__ void load_vec(float (&v)[K], const float* src, int P) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        int p = lane + 32 * k;
        v[k] = p < P ? src[p] : 0.0f;
    }
}

template <int K>
__device__ __forceinline__ void store_vec(float* dst, const float (&v)[K], int P) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        int p = lane + 32 * k;
        if (p < P) dst[p] = v[k];
    }
}

template <int K>
__device__ __forceinline__ float kinetic(const float (&p)[K], const float (&im)[K]) {
    float acc = 0.0f;
#pragma unroll
    for (int k = 0; k < K; ++k) acc = fmaf(p[k] * p[k], im[k], acc);
    return warp_sum(acc) * 0.5f;
}

// ---------------------------------------------------------------------------
// Batched density, one warp per chain.
// ---------------------------------------------------------------------------
template <int FAM, int K, int DMAX>
__global__ void __launch_bounds__(256) density_warp_kernel(DevModel dm, const float* __restrict__ params,
                                                           float* __restrict__ totals, float* __restrict__ grads,
                                                           int C) {
    extern __shared__ float smem[];
    stage_model<FAM>(dm, smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= C) return;
    float* qs = smem + dm.staged_floats + warp * dm.Ppad;
    const int P = dm.P;
    float q[K], g[K];
    load_vec(q, params + (size_t)c * P, P);
    float lj = eval_lj<FAM, K, DMAX>(dm, q, g, qs, grads != nullptr);
    if (lane == 0) totals[c] = lj;
    if (grads) store_vec(grads + (size_t)c * P, g, P);
}

// ---------------------------------------------------------------------------
// Fused HMC iteration (momentum, H0, leapfrog trajectory, H1, accept), one
// launch for all chains.  Mirrors _device_leapfrog_integrate_perchain!
// (hmc_kernels.jl:255-287) and the accept loop of hmc_kernels.jl:553-590.
// ---------------------------------------------------------------------------
struct HmcArgs {
    float* position;
    float* gradient;
    float* logjoint;
    const float* inverse_mass;
    const float* step;
    float* accept_prob;
    float* energy;
    float* energy_error;
    uint8_t* accepted;
    uint8_t* divergent;
    float* proposal;
    float* endpoint_momentum;
    int C;
    int L;
    uint32_t coord;
    float thr;
};

template <int FAM, int K, int DMAX>
__global__ void __launch_bounds__(256) hmc_warp_kernel(DevModel dm, HmcArgs a) {
    extern __shared__ float smem[];
    stage_model<FAM>(dm, smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= a.C) return;
    float* qs = smem + dm.staged_floats + warp * dm.Ppad;
    const int P = dm.P;
    const uint32_t chain = (uint32_t)c;
    float q[K], g[K], p[K], im[K];
    load_vec(q, a.position + (size_t)c * P, P);
    load_vec(g, a.gradient + (size_t)c * P, P);
    load_vec(im, a.inverse_mass, P);
    const float lj0 = a.logjoint[c];
    const float h = a.step[c];
    const float half = 0.5f * h;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        int pp = lane + 32 * k;
        p[k] = pp < P ? rand_normal(chain, a.coord, kStreamMomentum, (uint32_t)pp) / sqrtf(im[k]) : 0.0f;
    }
    const float H0 = kinetic(p, im) - lj0;
    bool valid = own_finite(g, P);
    float lj1 = 0.0f;
    if (valid) {
#pragma unroll
        for (int k = 0; k < K; ++k) p[k] = fmaf(half, g[k], p[k]);
        for (int l = 1; l <= a.L; ++l) {
#pragma unroll
            for (int k = 0; k < K; ++k) q[k] = fmaf(h * im[k], p[k], q[k]);
            float lj = eval_lj<FAM, K, DMAX>(dm, q, g, qs, true);
            bool gfin = own_finite(g, P);
            if (l < a.L) {
                if (!gfin) { valid = false; break; }
#pragma unroll
                for (int k = 0; k < K; ++k) p[k] = fmaf(h, g[k], p[k]);
            } else {
                if (!gfin || !isfinite(lj)) { valid = false; break; }
                lj1 = lj;
            }
        }
        if (valid) {
#pragma unroll
            for (int k = 0; k < K; ++k) p[k] = -fmaf(half, g[k], p[k]);
        }
    }
    float ap = 0.0f, ee = INFINITY, H1 = INFINITY;
    bool acc = false, div = true;
    if (valid) {
        H1 = kinetic(p, im) - lj1;
        float lar = H0 - H1;
        ee = H1 - H0;
        div = !isfinite(ee) || ee > a.thr;
        ap = !isfinite(lar) ? 0.0f : (lar >= 0.0f ? 1.0f : expf(lar));
        float u = rand_uniform(chain, a.coord, kStreamAccept, 0u);
        acc = logf(u) < fminf(0.0f, lar);
    }
    if (lane == 0) {
        a.accept_prob[c] = ap;
        a.energy_error[c] = ee;
        a.accepted[c] = acc ? 1 : 0;
        a.divergent[c] = div ? 1 : 0;
        a.energy[c] = acc ? H1 : H0;
        if (acc) a.logjoint[c] = lj1;
    }
    if (a.proposal) store_vec(a.proposal + (size_t)c * P, q, P);
    if (a.endpoint_momentum) store_vec(a.endpoint_momentum + (size_t)c * P, p, P);
    if (acc) {
        store_vec(a.position + (size_t)c * P, q, P);
        store_vec(a.gradient + (size_t)c * P, g, P);
    }
}

// One-step probe for the reasonable-step-size search (adaptation.jl:389-425).
struct ProbeArgs {
    const float* position;
    const float* gradient;
    const float* logjoint;
    const float* inverse_mass;
    const float* trial_step;
    float* log_accept_ratio;
    int C;
    uint32_t coord;
};

template <int FAM, int K, int DMAX>
__global__ void __launch_bounds__(256) probe_warp_kernel(DevModel dm, ProbeArgs a) {
    extern __shared__ float smem[];
    stage_model<FAM>(dm, smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= a.C) return;
    float* qs = smem + dm.staged_floats + warp * dm.Ppad;
    const int P = dm.P;
    float q[K], g[K], p[K], im[K];
    load_vec(q, a.position + (size_t)c * P, P);
    load_vec(g, a.gradient + (size_t)c * P, P);
    load_vec(im, a.inverse_mass, P);
    const float h = a.trial_step[c], half = 0.5f * h;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        int pp = lane + 32 * k;
        p[k] = pp < P ? rand_normal((uint32_t)c, a.coord, kStreamMomentum, (uint32_t)pp) / sqrtf(im[k]) : 0.0f;
    }
    const float H0 = kinetic(p, im) - a.logjoint[c];
    bool valid = own_finite(g, P);
    float out = -INFINITY;
    if (valid) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            p[k] = fmaf(half, g[k], p[k]);
            q[k] = fmaf(h * im[k], p[k], q[k]);
        }
        float lj = eval_lj<FAM, K, DMAX>(dm, q, g, qs, true);
        if (own_finite(g, P) && isfinite(lj)) {
#pragma unroll
            for (int k = 0; k < K; ++k) p[k] = -fmaf(half, g[k], p[k]);
            out = H0 - (kinetic(p, im) - lj);
        }
    }
    if (lane == 0) a.log_accept_ratio[c] = out;
}

// ---------------------------------------------------------------------------
// Persistent NUTS: one warp builds one chain's whole multinomial NUTS tree
// (persistent_nuts.jl:226-491).  Frontiers, subtree proposal and continuation
// proposal stay in registers; the dyadic checkpoint stack lives in a
// per-chain slice of global scratch (L2-resident, lane-contiguous).
// ---------------------------------------------------------------------------
struct NutsArgs {
    float* position;
    float* gradient;
    float* logjoint;
    const float* inverse_mass;
    const float* step;
    float* accept_prob;
    float* energy;
    float* energy_error;
    int32_t* tree_depth;
    int32_t* integration_steps;
    uint8_t* divergent;
    uint8_t* moved;
    float* ckpt;  // C x (max_depth + 1) x 2 x (32 K)
    int C;
    int max_depth;
    uint32_t coord;
    float thr;
};

__device__ __forceinline__ float logaddexp(float x, float y) {  // persistent_nuts.jl:83-92
    if (x == -INFINITY) return y;
    if (y == -INFINITY) return x;
    float hi = fmaxf(x, y);
    return hi + log1pf(expf(fminf(x, y) - hi));
}

template <int K>
__device__ __forceinline__ bool is_turning_lr(const float (&Lq)[K], const float (&Lp)[K], const float (&Rq)[K],
                                              const float (&Rp)[K], const float (&im)[K]) {
    float ld = 0.0f, rd = 0.0f;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        float delta = Rq[k] - Lq[k];
        ld = fmaf(delta * im[k], Lp[k], ld);
        rd = fmaf(delta * im[k], Rp[k], rd);
    }
    ld = warp_sum(ld);
    rd = warp_sum(rd);
    return ld <= 0.0f || rd <= 0.0f;
}

// One chain's state and outputs for one persistent-NUTS iteration: pointers to
// its position / gradient rows (P floats) and to its entry of each per-chain
// array.
struct NutsChainIO {
    float* position;
    float* gradient;
    float* logjoint;
    const float* inverse_mass;
    float step;
    float* accept_prob;
    float* energy;
    float* energy_error;
    int32_t* tree_depth;
    int32_t* integration_steps;
    uint8_t* divergent;
    uint8_t* moved;
};

// One persistent-NUTS iteration of one chain by one warp (persistent_nuts.jl:226-491).
// eval(q, g) returns the logjoint at q and writes its gradient to g; `chain`
// keys the chain's Philox streams, `it` is the iteration coordinate, ck the
// chain's checkpoint stack ((max_depth + 1) x 2 x 32K floats).
template <int K, class Eval>
__device__ __forceinline__ void nuts_chain(const Eval& eval, int P, const NutsChainIO& io, uint32_t chain,
                                           uint32_t it, int max_depth, float thr, float* ck) {
    const int lane = threadIdx.x & 31;
    const int VS = 32 * K;

    float q[K], g[K], p[K], im[K];
    float Lq[K], Lp[K], Lg[K], Rq[K], Rp[K], Rg[K], Sq[K], Sg[K], PPq[K], PPg[K], q0[K], g0[K];
    load_vec(q, io.position, P);
    load_vec(g, io.gradient, P);
    load_vec(im, io.inverse_mass, P);
    const float h = io.step;
    const float lj0 = *io.logjoint;

#pragma unroll
    for (int k = 0; k < K; ++k) {
        int pp = lane + 32 * k;
        p[k] = pp < P ? rand_normal(chain, it, kStreamMomentum, (uint32_t)pp) / sqrtf(im[k]) : 0.0f;
    }
    const float H0 = kinetic(p, im) - lj0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        q0[k] = q[k]; g0[k] = g[k];
        Lq[k] = q[k]; Lp[k] = p[k]; Lg[k] = g[k];
        Rq[k] = q[k]; Rp[k] = p[k]; Rg[k] = g[k];
        PPq[k] = q[k]; PPg[k] = g[k];
        Sq[k] = 0.0f; Sg[k] = 0.0f;
    }
    float ljL = lj0, ljR = lj0, ljS = 0.0f, prop_lj = lj0;
    float cont_w = -H0, accept_sum = 0.0f;
    int accept_count = 0, depth = 1, isteps = 0, leaf_counter = 0;
    bool divergent = false, turning = false;
    float prop_energy = H0, prop_error = 0.0f;

    // ---- first single-leaf trajectory (persistent_nuts.jl:284-338) ----
    {
        float u = rand_uniform(chain, it, kStreamDirection, 0u);
        float dir = u < 0.5f ? -1.0f : 1.0f;
        bool forward = dir > 0.0f;
        float hs = dir * h, half = hs * 0.5f;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            p[k] = fmaf(half, g[k], p[k]);
            q[k] = fmaf(hs, im[k] * p[k], q[k]);
        }
        float lj1 = eval(q, g);
        bool ok1 = isfinite(lj1) && own_finite(g, P);
        if (!ok1) {
            divergent = true;
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) p[k] = fmaf(half, g[k], p[k]);
            if (forward) {
#pragma unroll
                for (int k = 0; k < K; ++k) { Rq[k] = q[k]; Rp[k] = p[k]; Rg[k] = g[k]; }
                ljR = lj1;
            } else {
#pragma unroll
                for (int k = 0; k < K; ++k) { Lq[k] = q[k]; Lp[k] = p[k]; Lg[k] = g[k]; }
                ljL = lj1;
            }
            float pe = kinetic(p, im) - lj1;
            float delta = pe - H0;
            isteps = 1;
            if (!isfinite(delta) || delta > thr) {
                divergent = true;
            } else {
                accept_sum += fminf(1.0f, expf(fminf(0.0f, -delta)));
                accept_count += 1;
                float cand = -pe;
                float comb = logaddexp(cont_w, cand);
                float ul = rand_uniform(chain, it, kStreamLeaf, (uint32_t)leaf_counter);
                if (!isfinite(cont_w) || logf(ul) < cand - comb) {
#pragma unroll
                    for (int k = 0; k < K; ++k) { PPq[k] = q[k]; PPg[k] = g[k]; }
                    prop_lj = lj1; prop_energy = pe; prop_error = delta;
                }
                cont_w = comb;
                turning = is_turning_lr(Lq, Lp, Rq, Rp, im);
            }
            leaf_counter += 1;
        }
    }

    // ---- doubling loop (persistent_nuts.jl:341-475) ----
    while (depth < max_depth && !divergent && !turning) {
        const int round = depth;
        float ud = rand_uniform(chain, it, kStreamDirection, (uint32_t)round);
        float dir = ud < 0.5f ? -1.0f : 1.0f;
        const bool forward = dir > 0.0f;
        const float hs = dir * h, half = hs * 0.5f;
        float cur_lj;
        if (forward) {
#pragma unroll
            for (int k = 0; k < K; ++k) { q[k] = Rq[k]; p[k] = Rp[k]; g[k] = Rg[k]; }
            cur_lj = ljR;
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) { q[k] = Lq[k]; p[k] = Lp[k]; g[k] = Lg[k]; }
            cur_lj = ljL;
        }
        float sub_w = -INFINITY, sub_acc = 0.0f, sub_energy = 0.0f, sub_error = 0.0f;
        int sub_int = 0, sub_acc_n = 0;
        bool sub_div = false, sub_turn = false;
        const int nleaves = 1 << depth;
        for (int leaf = 0; leaf < nleaves; ++leaf) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                p[k] = fmaf(half, g[k], p[k]);
                q[k] = fmaf(hs, im[k] * p[k], q[k]);
            }
            float ljc = eval(q, g);
            if (!(isfinite(ljc) && own_finite(g, P))) { sub_div = true; break; }
#pragma unroll
            for (int k = 0; k < K; ++k) p[k] = fmaf(half, g[k], p[k]);
            cur_lj = ljc;
            sub_int += 1;
            float pe = kinetic(p, im) - ljc;
            float delta = pe - H0;
            if (!isfinite(delta) || delta > thr) { sub_div = true; break; }
            sub_acc += fminf(1.0f, expf(fminf(0.0f, -delta)));
            sub_acc_n += 1;
            float cand = -pe;
            float comb = logaddexp(sub_w, cand);
            float ul = rand_uniform(chain, it, kStreamLeaf, (uint32_t)leaf_counter);
            if (!isfinite(sub_w) || logf(ul) < cand - comb) {
#pragma unroll
                for (int k = 0; k < K; ++k) { Sq[k] = q[k]; Sg[k] = g[k]; }
                ljS = ljc; sub_energy = pe; sub_error = delta;
            }
            sub_w = comb;
            leaf_counter += 1;
            const int leaf_index = sub_int - 1;
            if ((leaf_index & 1) == 0) {
                // even leaf: checkpoint (position, momentum) at slot popcount(leaf_index)
                const int slot = __popc(leaf_index);
                float* dst = ck + (size_t)slot * 2 * VS;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    dst[32 * k + lane] = q[k];
                    dst[VS + 32 * k + lane] = p[k];
                }
            } else {
                // odd leaf: dyadic U-turn over the blocks ending here (persistent_nuts.jl:126-155)
                const int nt = __ffs(~leaf_index) - 1;  // trailing ones
                bool turned = false;
                for (int kk = 1; kk <= nt && !turned; ++kk) {
                    const int block_start = leaf_index - (1 << kk) + 1;
                    const int slot = __popc(block_start);
                    const float* src = ck + (size_t)slot * 2 * VS;
                    float ld = 0.0f, rd = 0.0f;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        float cp = src[32 * k + lane];
                        float cm = src[VS + 32 * k + lane];
                        if (forward) {
                            float d2 = (q[k] - cp) * im[k];
                            ld = fmaf(d2, cm, ld);
                            rd = fmaf(d2, p[k], rd);
                        } else {
                            float d2 = (cp - q[k]) * im[k];
                            ld = fmaf(d2, p[k], ld);
                            rd = fmaf(d2, cm, rd);
                        }
                    }
                    ld = warp_sum(ld);
                    rd = warp_sum(rd);
                    if (ld <= 0.0f || rd <= 0.0f) turned = true;
                }
                if (turned) { sub_turn = true; break; }
            }
        }
        depth += 1;
        if (sub_int == 0) { divergent = sub_div; break; }
        if (sub_turn || sub_div) {
            isteps += sub_int; accept_sum += sub_acc; accept_count += sub_acc_n;
            turning = sub_turn; divergent = sub_div;
            break;
        }
        if (forward) {
#pragma unroll
            for (int k = 0; k < K; ++k) { Rq[k] = q[k]; Rp[k] = p[k]; Rg[k] = g[k]; }
            ljR = cur_lj;
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) { Lq[k] = q[k]; Lp[k] = p[k]; Lg[k] = g[k]; }
            ljL = cur_lj;
        }
        float comb_cw = cont_w;
        if (isfinite(sub_w)) {
            comb_cw = logaddexp(cont_w, sub_w);
            float um = rand_uniform(chain, it, kStreamMerge, (uint32_t)round);
            if (logf(um) < sub_w - cont_w) {
#pragma unroll
                for (int k = 0; k < K; ++k) { PPq[k] = Sq[k]; PPg[k] = Sg[k]; }
                prop_lj = ljS; prop_energy = sub_energy; prop_error = sub_error;
            }
        }
        isteps += sub_int; accept_sum += sub_acc; accept_count += sub_acc_n;
        if (isfinite(sub_w)) cont_w = comb_cw;
        turning = sub_turn || is_turning_lr(Lq, Lp, Rq, Rp, im);
    }

    bool moved_l = false;
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (lane + 32 * k < P && PPq[k] != q0[k]) moved_l = true;
    const bool moved = __any_sync(UT_FULL_MASK, moved_l);
    if (moved) {
        store_vec(io.position, PPq, P);
        store_vec(io.gradient, PPg, P);
    }
    if (lane == 0) {
        if (moved) *io.logjoint = prop_lj;
        *io.moved = moved ? 1 : 0;
        *io.accept_prob = accept_count == 0 ? 0.0f : accept_sum / (float)accept_count;
        *io.energy = prop_energy;
        *io.energy_error = prop_error;
        *io.divergent = divergent ? 1 : 0;
        *io.tree_depth = depth;
        *io.integration_steps = isteps;
    }
    (void)g0;
}

template <int FAM, int K, int DMAX>
__global__ void __launch_bounds__(128) nuts_warp_kernel(DevModel dm, NutsArgs a) {
    extern __shared__ float smem[];
    stage_model<FAM>(dm, smem);
    const int warp = threadIdx.x >> 5;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= a.C) return;
    const int P = dm.P;
    NutsChainIO io;
    io.position = a.position + (size_t)c * P;
    io.gradient = a.gradient + (size_t)c * P;
    io.logjoint = a.logjoint + c;
    io.inverse_mass = a.inverse_mass;
    io.step = a.step[c];
    io.accept_prob = a.accept_prob + c;
    io.energy = a.energy + c;
    io.energy_error = a.energy_error + c;
    io.tree_depth = a.tree_depth + c;
    io.integration_steps = a.integration_steps + c;
    io.divergent = a.divergent + c;
    io.moved = a.moved + c;
    float* qs = smem + dm.staged_floats + warp * dm.Ppad;
    float* ck = a.ckpt + (size_t)c * (a.max_depth + 1) * 2 * (32 * K);
    auto eval = [&](const float (&qq)[K], float (&gg)[K]) { return eval_lj<FAM, K, DMAX>(dm, qq, gg, qs, true); };
    nuts_chain<K>(eval, P, io, (uint32_t)c, a.coord, a.max_depth, a.thr, ck);
}

}  // namespace ut
