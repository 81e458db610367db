// ut_nuts_lockstep.cuh -- lockstep ("masked") multinomial NUTS for models whose
// gradient is a batched kernel over all chains (the large GLM): every chain's
// tree is a resumable state machine in device memory, advanced one leaf per
// step between two batched gradient evaluations.  The tree decisions are those
// of nuts_chain (ut_warp_kernels.cuh, persistent_nuts.jl:226-491) in the same
// order with the same Philox draws, so on a model with a per-chain evaluator
// the two strategies give the same trees; the reference's device counterpart
// is the masked lockstep tree (src/device/nuts_kernels.jl:61-600).
//
// Per step (one warp per chain):
//   ls_step_kernel   consume the leaf just evaluated (logjoint + gradient at
//                    wq): leaf bookkeeping, multinomial choice, checkpoint /
//                    dyadic U-turn, round end (merge, frontier, full-tree
//                    U-turn), finalisation when the tree stops; otherwise drift
//                    to the next leaf and write its position to wq.
// ls_init_kernel draws the momentum and drifts to the first leaf.  When the
// gradient kernel can skip chains (the tensor-core path), the live chains are
// compacted before each evaluation (ls_compact / gather / scatter) so the trees
// still growing at the tail of an iteration cost only their own chain tiles.
#pragma once

#include "ut_warp_kernels.cuh"

namespace ut {

// Per-chain vectors of the state machine, each C x P (chain-major).
enum LsVec : int { kLsQ = 0, kLsP, kLsG, kLsLq, kLsLp, kLsLg, kLsRq, kLsRp, kLsRg, kLsSq, kLsSg, kLsPPq, kLsPPg,
                   kLsQ0, kLsNumVec };
// Per-chain float scalars.
enum LsF : int { kLsH0 = 0, kLsLjL, kLsLjR, kLsLjS, kLsPropLj, kLsContW, kLsAccSum, kLsPropE, kLsPropErr,
                 kLsStep, kLsSubW, kLsSubAcc, kLsSubE, kLsSubErr, kLsCurLj, kLsNumF };
// Per-chain int scalars.
enum LsI : int { kLsState = 0, kLsDepth, kLsIsteps, kLsLeafCtr, kLsAccCnt, kLsFlags, kLsRound, kLsLeaf,
                 kLsSubInt, kLsSubAccN, kLsNumI };
// kLsState values
constexpr int kLsFirst = 1, kLsInRound = 2, kLsDone = 3;
// kLsFlags bits
constexpr int kLsDivergent = 1, kLsTurning = 2, kLsForward = 4, kLsSubDiv = 8, kLsSubTurn = 16;

struct LsState {
    float* vec;      // kLsNumVec x C x P
    float* f;        // kLsNumF x C
    int32_t* i;      // kLsNumI x C
    float* ckpt;     // C x (max_depth + 1) x 2 x 32K
    float* wq;       // C x P   position to evaluate
    const float* wg; // C x P   gradient at wq
    const float* wlj;// C       logjoint at wq
    uint8_t* act;    // C       1 while the chain's tree is still growing (its next leaf is in wq)
};

struct LsArgs {
    NutsArgs n;  // caller state and outputs (position, gradient, logjoint, ... as for nuts_warp_kernel)
    LsState s;
    int P;
};

__device__ __forceinline__ float* ls_vec(const LsState& s, int v, int c, int C, int P) {
    return s.vec + ((size_t)v * C + c) * P;
}

// Drift to the next leaf from the current (q, p, g): p += h/2 g, q += h M^-1 p,
// and publish q for the batched evaluation.
template <int K>
__device__ __forceinline__ void ls_drift(float (&q)[K], float (&p)[K], const float (&g)[K], const float (&im)[K],
                                         float hs) {
    const float half = 0.5f * hs;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        p[k] = fmaf(half, g[k], p[k]);
        q[k] = fmaf(hs, im[k] * p[k], q[k]);
    }
}

template <int K>
__global__ void __launch_bounds__(128) ls_init_kernel(LsArgs a) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    const int C = a.n.C;
    if (c >= C) return;
    const LsState& s = a.s;
    const int PP = a.P;
    const uint32_t chain = (uint32_t)c, it = a.n.coord;
    float q[K], g[K], p[K], im[K];
    load_vec(q, a.n.position + (size_t)c * PP, PP);
    load_vec(g, a.n.gradient + (size_t)c * PP, PP);
    load_vec(im, a.n.inverse_mass, PP);
    const float h = a.n.step[c];
    const float lj0 = a.n.logjoint[c];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int pp = lane + 32 * k;
        p[k] = pp < PP ? rand_normal(chain, it, kStreamMomentum, (uint32_t)pp) / sqrtf(im[k]) : 0.0f;
    }
    const float H0 = kinetic(p, im) - lj0;
    store_vec(ls_vec(s, kLsQ0, c, C, PP), q, PP);
    store_vec(ls_vec(s, kLsLq, c, C, PP), q, PP);
    store_vec(ls_vec(s, kLsLp, c, C, PP), p, PP);
    store_vec(ls_vec(s, kLsLg, c, C, PP), g, PP);
    store_vec(ls_vec(s, kLsRq, c, C, PP), q, PP);
    store_vec(ls_vec(s, kLsRp, c, C, PP), p, PP);
    store_vec(ls_vec(s, kLsRg, c, C, PP), g, PP);
    store_vec(ls_vec(s, kLsPPq, c, C, PP), q, PP);
    store_vec(ls_vec(s, kLsPPg, c, C, PP), g, PP);
    // first single-leaf trajectory: direction, then drift
    const float u = rand_uniform(chain, it, kStreamDirection, 0u);
    const bool forward = !(u < 0.5f);
    const float hs = forward ? h : -h;
    ls_drift(q, p, g, im, hs);
    store_vec(ls_vec(s, kLsQ, c, C, PP), q, PP);
    store_vec(ls_vec(s, kLsP, c, C, PP), p, PP);
    store_vec(s.wq + (size_t)c * PP, q, PP);
    if (lane == 0) {
        s.act[c] = 1;
        float* F = s.f;
        int32_t* I = s.i;
        F[kLsH0 * C + c] = H0;
        F[kLsLjL * C + c] = lj0;
        F[kLsLjR * C + c] = lj0;
        F[kLsLjS * C + c] = 0.0f;
        F[kLsPropLj * C + c] = lj0;
        F[kLsContW * C + c] = -H0;
        F[kLsAccSum * C + c] = 0.0f;
        F[kLsPropE * C + c] = H0;
        F[kLsPropErr * C + c] = 0.0f;
        F[kLsStep * C + c] = h;
        I[kLsState * C + c] = kLsFirst;
        I[kLsDepth * C + c] = 1;
        I[kLsIsteps * C + c] = 0;
        I[kLsLeafCtr * C + c] = 0;
        I[kLsAccCnt * C + c] = 0;
        I[kLsFlags * C + c] = forward ? kLsForward : 0;
        I[kLsRound * C + c] = 0;
        I[kLsLeaf * C + c] = 0;
    }
}

template <int K>
__global__ void __launch_bounds__(128) ls_step_kernel(LsArgs a) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    const int C = a.n.C;
    if (c >= C) return;
    const LsState& s = a.s;
    float* F = s.f;
    int32_t* I = s.i;
    int state = I[kLsState * C + c];
    if (state == kLsDone) {
        if (lane == 0) s.act[c] = 0;
        return;
    }
    const int P = a.P;
    const int VS = 32 * K;
    const uint32_t chain = (uint32_t)c, it = a.n.coord;
    const float thr = a.n.thr;
    const int max_depth = a.n.max_depth;
    float* ck = s.ckpt + (size_t)c * (max_depth + 1) * 2 * VS;

    float q[K], p[K], g[K], im[K];
    load_vec(q, ls_vec(s, kLsQ, c, C, P), P);
    load_vec(p, ls_vec(s, kLsP, c, C, P), P);
    load_vec(g, s.wg + (size_t)c * P, P);
    load_vec(im, a.n.inverse_mass, P);
    const float lj = s.wlj[c];
    const float H0 = F[kLsH0 * C + c];
    const float h = F[kLsStep * C + c];
    int flags = I[kLsFlags * C + c];
    int depth = I[kLsDepth * C + c];
    int isteps = I[kLsIsteps * C + c];
    int leaf_counter = I[kLsLeafCtr * C + c];
    int accept_count = I[kLsAccCnt * C + c];
    float accept_sum = F[kLsAccSum * C + c];
    float cont_w = F[kLsContW * C + c];
    const bool forward = (flags & kLsForward) != 0;
    const float hs = forward ? h : -h, half = 0.5f * hs;
    bool tree_done = false;

    auto write_frontier = [&](float ljv) {
        if (forward) {
            store_vec(ls_vec(s, kLsRq, c, C, P), q, P);
            store_vec(ls_vec(s, kLsRp, c, C, P), p, P);
            store_vec(ls_vec(s, kLsRg, c, C, P), g, P);
            if (lane == 0) F[kLsLjR * C + c] = ljv;
        } else {
            store_vec(ls_vec(s, kLsLq, c, C, P), q, P);
            store_vec(ls_vec(s, kLsLp, c, C, P), p, P);
            store_vec(ls_vec(s, kLsLg, c, C, P), g, P);
            if (lane == 0) F[kLsLjL * C + c] = ljv;
        }
    };
    auto full_tree_turning = [&]() -> bool {
        float Lq[K], Lp[K], Rq[K], Rp[K];
        load_vec(Lq, ls_vec(s, kLsLq, c, C, P), P);
        load_vec(Lp, ls_vec(s, kLsLp, c, C, P), P);
        load_vec(Rq, ls_vec(s, kLsRq, c, C, P), P);
        load_vec(Rp, ls_vec(s, kLsRp, c, C, P), P);
        return is_turning_lr(Lq, Lp, Rq, Rp, im);
    };

    if (state == kLsFirst) {
        // ---- first single-leaf trajectory (persistent_nuts.jl:284-338) ----
        const bool ok1 = isfinite(lj) && own_finite(g, P);
        if (!ok1) {
            flags |= kLsDivergent;
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) p[k] = fmaf(half, g[k], p[k]);
            __syncwarp();
            write_frontier(lj);
            const float pe = kinetic(p, im) - lj;
            const float delta = pe - H0;
            isteps = 1;
            if (!isfinite(delta) || delta > thr) {
                flags |= kLsDivergent;
            } else {
                accept_sum += fminf(1.0f, expf(fminf(0.0f, -delta)));
                accept_count += 1;
                const float cand = -pe;
                const float comb = logaddexp(cont_w, cand);
                const float ul = rand_uniform(chain, it, kStreamLeaf, (uint32_t)leaf_counter);
                if (!isfinite(cont_w) || logf(ul) < cand - comb) {
                    store_vec(ls_vec(s, kLsPPq, c, C, P), q, P);
                    store_vec(ls_vec(s, kLsPPg, c, C, P), g, P);
                    if (lane == 0) {
                        F[kLsPropLj * C + c] = lj;
                        F[kLsPropE * C + c] = pe;
                        F[kLsPropErr * C + c] = delta;
                    }
                }
                cont_w = comb;
                __syncwarp();
                if (full_tree_turning()) flags |= kLsTurning;
            }
            leaf_counter += 1;
        }
        tree_done = true;  // the first trajectory is complete; continue with round 1 below
    } else {
        // ---- one leaf of a doubling round (persistent_nuts.jl:341-475) ----
        const int round = I[kLsRound * C + c];
        int leaf = I[kLsLeaf * C + c];
        int sub_int = I[kLsSubInt * C + c];
        int sub_acc_n = I[kLsSubAccN * C + c];
        float sub_w = F[kLsSubW * C + c];
        float sub_acc = F[kLsSubAcc * C + c];
        bool round_end = false;
        bool sub_div = (flags & kLsSubDiv) != 0, sub_turn = (flags & kLsSubTurn) != 0;
        float cur_lj = F[kLsCurLj * C + c];
        if (!(isfinite(lj) && own_finite(g, P))) {
            sub_div = true;
            round_end = true;
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) p[k] = fmaf(half, g[k], p[k]);
            cur_lj = lj;
            sub_int += 1;
            const float pe = kinetic(p, im) - lj;
            const float delta = pe - H0;
            if (!isfinite(delta) || delta > thr) {
                sub_div = true;
                round_end = true;
            } else {
                sub_acc += fminf(1.0f, expf(fminf(0.0f, -delta)));
                sub_acc_n += 1;
                const float cand = -pe;
                const float comb = logaddexp(sub_w, cand);
                const float ul = rand_uniform(chain, it, kStreamLeaf, (uint32_t)leaf_counter);
                if (!isfinite(sub_w) || logf(ul) < cand - comb) {
                    store_vec(ls_vec(s, kLsSq, c, C, P), q, P);
                    store_vec(ls_vec(s, kLsSg, c, C, P), g, P);
                    if (lane == 0) {
                        F[kLsLjS * C + c] = lj;
                        F[kLsSubE * C + c] = pe;
                        F[kLsSubErr * C + c] = delta;
                    }
                }
                sub_w = comb;
                leaf_counter += 1;
                const int leaf_index = sub_int - 1;
                if ((leaf_index & 1) == 0) {
                    const int slot = __popc(leaf_index);
                    float* dst = ck + (size_t)slot * 2 * VS;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        dst[32 * k + lane] = q[k];
                        dst[VS + 32 * k + lane] = p[k];
                    }
                } else {
                    const int nt = __ffs(~leaf_index) - 1;  // trailing ones (persistent_nuts.jl:126-155)
                    bool turned = false;
                    for (int kk = 1; kk <= nt && !turned; ++kk) {
                        const int block_start = leaf_index - (1 << kk) + 1;
                        const int slot = __popc(block_start);
                        const float* src = ck + (size_t)slot * 2 * VS;
                        float ld = 0.0f, rd = 0.0f;
#pragma unroll
                        for (int k = 0; k < K; ++k) {
                            const float cp = src[32 * k + lane];
                            const float cm = src[VS + 32 * k + lane];
                            if (forward) {
                                const float d2 = (q[k] - cp) * im[k];
                                ld = fmaf(d2, cm, ld);
                                rd = fmaf(d2, p[k], rd);
                            } else {
                                const float d2 = (cp - q[k]) * im[k];
                                ld = fmaf(d2, p[k], ld);
                                rd = fmaf(d2, cm, rd);
                            }
                        }
                        ld = warp_sum(ld);
                        rd = warp_sum(rd);
                        if (ld <= 0.0f || rd <= 0.0f) turned = true;
                    }
                    if (turned) {
                        sub_turn = true;
                        round_end = true;
                    }
                }
                if (!round_end && ++leaf == (1 << round)) round_end = true;
            }
        }
        if (!round_end) {
            // next leaf of this round: its opening half kick and drift
            ls_drift(q, p, g, im, hs);
            store_vec(ls_vec(s, kLsQ, c, C, P), q, P);
            store_vec(ls_vec(s, kLsP, c, C, P), p, P);
            store_vec(s.wq + (size_t)c * P, q, P);
            if (lane == 0) {
                I[kLsLeaf * C + c] = leaf;
                I[kLsSubInt * C + c] = sub_int;
                I[kLsSubAccN * C + c] = sub_acc_n;
                I[kLsLeafCtr * C + c] = leaf_counter;
                F[kLsSubW * C + c] = sub_w;
                F[kLsSubAcc * C + c] = sub_acc;
                F[kLsCurLj * C + c] = cur_lj;
            }
            if (lane == 0) s.act[c] = 1;
            return;
        }
        // ---- end of the round ----
        depth += 1;
        bool stop = false;
        if (sub_int == 0) {
            if (sub_div) flags |= kLsDivergent;
            stop = true;
        } else if (sub_turn || sub_div) {
            isteps += sub_int;
            accept_sum += sub_acc;
            accept_count += sub_acc_n;
            if (sub_turn) flags |= kLsTurning;
            if (sub_div) flags |= kLsDivergent;
            stop = true;
        } else {
            write_frontier(cur_lj);
            float comb_cw = cont_w;
            if (isfinite(sub_w)) {
                comb_cw = logaddexp(cont_w, sub_w);
                const float um = rand_uniform(chain, it, kStreamMerge, (uint32_t)round);
                if (logf(um) < sub_w - cont_w) {
                    float Sq[K], Sg[K];
                    load_vec(Sq, ls_vec(s, kLsSq, c, C, P), P);
                    load_vec(Sg, ls_vec(s, kLsSg, c, C, P), P);
                    store_vec(ls_vec(s, kLsPPq, c, C, P), Sq, P);
                    store_vec(ls_vec(s, kLsPPg, c, C, P), Sg, P);
                    if (lane == 0) {
                        F[kLsPropLj * C + c] = F[kLsLjS * C + c];
                        F[kLsPropE * C + c] = F[kLsSubE * C + c];
                        F[kLsPropErr * C + c] = F[kLsSubErr * C + c];
                    }
                }
            }
            isteps += sub_int;
            accept_sum += sub_acc;
            accept_count += sub_acc_n;
            if (isfinite(sub_w)) cont_w = comb_cw;
            __syncwarp();
            if (full_tree_turning()) flags |= kLsTurning;
        }
        tree_done = true;
        (void)stop;
    }

    // ---- either start the next doubling round or finalise ----
    if (tree_done) {
        const bool more = depth < max_depth && !(flags & kLsDivergent) && !(flags & kLsTurning);
        if (more) {
            const int round = depth;
            const float ud = rand_uniform(chain, it, kStreamDirection, (uint32_t)round);
            const bool fwd = !(ud < 0.5f);
            flags = (flags & ~(kLsForward | kLsSubDiv | kLsSubTurn)) | (fwd ? kLsForward : 0);
            const float hs2 = fwd ? h : -h;
            __syncwarp();
            load_vec(q, ls_vec(s, fwd ? kLsRq : kLsLq, c, C, P), P);
            load_vec(p, ls_vec(s, fwd ? kLsRp : kLsLp, c, C, P), P);
            load_vec(g, ls_vec(s, fwd ? kLsRg : kLsLg, c, C, P), P);
            const float cur = F[(fwd ? kLsLjR : kLsLjL) * C + c];
            ls_drift(q, p, g, im, hs2);
            store_vec(ls_vec(s, kLsQ, c, C, P), q, P);
            store_vec(ls_vec(s, kLsP, c, C, P), p, P);
            store_vec(s.wq + (size_t)c * P, q, P);
            if (lane == 0) {
                I[kLsState * C + c] = kLsInRound;
                I[kLsRound * C + c] = round;
                I[kLsLeaf * C + c] = 0;
                I[kLsSubInt * C + c] = 0;
                I[kLsSubAccN * C + c] = 0;
                F[kLsSubW * C + c] = -INFINITY;
                F[kLsSubAcc * C + c] = 0.0f;
                F[kLsSubE * C + c] = 0.0f;
                F[kLsSubErr * C + c] = 0.0f;
                F[kLsCurLj * C + c] = cur;
                I[kLsDepth * C + c] = depth;
                I[kLsIsteps * C + c] = isteps;
                I[kLsLeafCtr * C + c] = leaf_counter;
                I[kLsAccCnt * C + c] = accept_count;
                I[kLsFlags * C + c] = flags;
                F[kLsAccSum * C + c] = accept_sum;
                F[kLsContW * C + c] = cont_w;
            }
            if (lane == 0) s.act[c] = 1;
            return;
        }
        // finalise (the epilogue of nuts_chain)
        __syncwarp();
        float PPq[K], PPg[K], q0[K];
        load_vec(PPq, ls_vec(s, kLsPPq, c, C, P), P);
        load_vec(PPg, ls_vec(s, kLsPPg, c, C, P), P);
        load_vec(q0, ls_vec(s, kLsQ0, c, C, P), P);
        bool moved_l = false;
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (lane + 32 * k < P && PPq[k] != q0[k]) moved_l = true;
        const bool moved = __any_sync(UT_FULL_MASK, moved_l);
        if (moved) {
            store_vec(a.n.position + (size_t)c * P, PPq, P);
            store_vec(a.n.gradient + (size_t)c * P, PPg, P);
        }
        if (lane == 0) {
            if (moved) a.n.logjoint[c] = F[kLsPropLj * C + c];
            a.n.moved[c] = moved ? 1 : 0;
            a.n.accept_prob[c] = accept_count == 0 ? 0.0f : accept_sum / (float)accept_count;
            a.n.energy[c] = F[kLsPropE * C + c];
            a.n.energy_error[c] = F[kLsPropErr * C + c];
            a.n.divergent[c] = (flags & kLsDivergent) ? 1 : 0;
            a.n.tree_depth[c] = depth;
            a.n.integration_steps[c] = isteps;
            I[kLsState * C + c] = kLsDone;
            s.act[c] = 0;
        }
    }
}

// Stable compaction of the live chains (one CTA): idx[0, n) = the chains with
// act = 1 in chain order, *nact = n.
__global__ void __launch_bounds__(1024) ls_compact_kernel(const uint8_t* __restrict__ act, int C,
                                                          int32_t* __restrict__ idx, int32_t* __restrict__ nact) {
    __shared__ int sums[1024];
    const int t = threadIdx.x;
    const int per = (C + 1023) / 1024;
    const int b = min(C, t * per), e = min(C, b + per);
    int cnt = 0;
    for (int c = b; c < e; ++c) cnt += act[c];
    sums[t] = cnt;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {  // inclusive scan
        const int v = t >= off ? sums[t - off] : 0;
        __syncthreads();
        sums[t] += v;
        __syncthreads();
    }
    int pos = sums[t] - cnt;
    for (int c = b; c < e; ++c)
        if (act[c]) idx[pos++] = c;
    if (t == 1023) *nact = sums[1023];
}

// cq[j] = wq[idx[j]] for the live chains j < *nact (rows of P floats).
__global__ void ls_gather_kernel(const float* __restrict__ wq, const int32_t* __restrict__ idx,
                                 const int32_t* __restrict__ nact, int P, float* __restrict__ cq) {
    const long long total = (long long)(*nact) * P;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long j = i / P, k = i % P;
        cq[i] = wq[(long long)idx[j] * P + k];
    }
}

// wg[idx[j]] = cg[j], wlj[idx[j]] = clj[j] for j < *nact.
__global__ void ls_scatter_kernel(const float* __restrict__ cg, const float* __restrict__ clj,
                                  const int32_t* __restrict__ idx, const int32_t* __restrict__ nact, int P,
                                  float* __restrict__ wg, float* __restrict__ wlj) {
    const int n = *nact;
    const long long total = (long long)n * P;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long j = i / P, k = i % P;
        wg[(long long)idx[j] * P + k] = cg[i];
        if (k == 0) wlj[idx[j]] = clj[j];
    }
}

}  // namespace ut
