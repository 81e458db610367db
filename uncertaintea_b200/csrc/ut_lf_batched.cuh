// ut_lf_batched.cuh -- leapfrog/HMC pieces for models whose gradient is a
// batched (all-chains) kernel rather than a per-warp evaluation.  A trajectory
// of L steps is: lf_begin (momentum, H0, validity, half kick, first drift),
// then L x [batched gradient -> lf_step], where the last lf_step closes the
// trajectory (final half kick + flip, H1, Metropolis accept, column update).
// Same arithmetic, in the same order, as hmc_warp_kernel.
#pragma once

#include "ut_warp_kernels.cuh"

namespace ut {

struct LfScratch {
    float* wq;        // C x P working position (the batched gradient's input)
    float* wp;        // C x P working momentum
    float* wg;        // C x P gradient at wq
    float* wlj;       // C     logjoint at wq
    float* H0;        // C
    uint8_t* valid;   // C
};

template <int K>
__global__ void __launch_bounds__(256) lf_begin_kernel(HmcArgs a, LfScratch s, int P) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= a.C) return;
    float q[K], g[K], p[K], im[K];
    load_vec(q, a.position + (size_t)c * P, P);
    load_vec(g, a.gradient + (size_t)c * P, P);
    load_vec(im, a.inverse_mass, P);
    const float h = a.step[c], half = 0.5f * h;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        int pp = lane + 32 * k;
        p[k] = pp < P ? rand_normal((uint32_t)c, a.coord, kStreamMomentum, (uint32_t)pp) / sqrtf(im[k]) : 0.0f;
    }
    const float H0 = kinetic(p, im) - a.logjoint[c];
    const bool valid = own_finite(g, P);
    if (valid) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            p[k] = fmaf(half, g[k], p[k]);
            q[k] = fmaf(h * im[k], p[k], q[k]);
        }
    }
    store_vec(s.wq + (size_t)c * P, q, P);
    store_vec(s.wp + (size_t)c * P, p, P);
    if (lane == 0) {
        s.H0[c] = H0;
        s.valid[c] = valid ? 1 : 0;
    }
}

// After the batched gradient at wq (-> wg, wlj) for leapfrog step l of L.
template <int K>
__global__ void __launch_bounds__(256) lf_step_kernel(HmcArgs a, LfScratch s, int P, int l) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= a.C) return;
    bool valid = s.valid[c] != 0;
    float q[K], g[K], p[K], im[K];
    load_vec(q, s.wq + (size_t)c * P, P);
    load_vec(p, s.wp + (size_t)c * P, P);
    load_vec(g, s.wg + (size_t)c * P, P);
    load_vec(im, a.inverse_mass, P);
    const float h = a.step[c], half = 0.5f * h;
    const float lj = s.wlj[c];
    if (l < a.L) {
        if (valid) {
            if (!own_finite(g, P)) {
                valid = false;
            } else {
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    p[k] = fmaf(h, g[k], p[k]);
                    q[k] = fmaf(h * im[k], p[k], q[k]);
                }
                store_vec(s.wq + (size_t)c * P, q, P);
                store_vec(s.wp + (size_t)c * P, p, P);
            }
        }
        if (lane == 0) s.valid[c] = valid ? 1 : 0;
        return;
    }
    // final step: close the trajectory and run the accept
    if (valid) {
        if (!own_finite(g, P) || !isfinite(lj)) {
            valid = false;
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) p[k] = -fmaf(half, g[k], p[k]);
        }
    }
    const float H0 = s.H0[c];
    float ap = 0.0f, ee = INFINITY, H1 = INFINITY;
    bool acc = false, div = true;
    if (valid) {
        H1 = kinetic(p, im) - lj;
        float lar = H0 - H1;
        ee = H1 - H0;
        div = !isfinite(ee) || ee > a.thr;
        ap = !isfinite(lar) ? 0.0f : (lar >= 0.0f ? 1.0f : expf(lar));
        float u = rand_uniform((uint32_t)c, a.coord, kStreamAccept, 0u);
        acc = logf(u) < fminf(0.0f, lar);
    }
    if (lane == 0) {
        a.accept_prob[c] = ap;
        a.energy_error[c] = ee;
        a.accepted[c] = acc ? 1 : 0;
        a.divergent[c] = div ? 1 : 0;
        a.energy[c] = acc ? H1 : H0;
        if (acc) a.logjoint[c] = lj;
        s.valid[c] = valid ? 1 : 0;
    }
    if (a.proposal) store_vec(a.proposal + (size_t)c * P, q, P);
    if (a.endpoint_momentum) store_vec(a.endpoint_momentum + (size_t)c * P, p, P);
    if (acc) {
        store_vec(a.position + (size_t)c * P, q, P);
        store_vec(a.gradient + (size_t)c * P, g, P);
    }
}

// Probe: closes a one-step trajectory started by lf_begin (l = L = 1).
template <int K>
__global__ void __launch_bounds__(256) lf_probe_close_kernel(const float* inverse_mass, const float* trial_step,
                                                            LfScratch s, float* log_accept_ratio, int P, int C) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= C) return;
    float g[K], p[K], im[K];
    load_vec(p, s.wp + (size_t)c * P, P);
    load_vec(g, s.wg + (size_t)c * P, P);
    load_vec(im, inverse_mass, P);
    const float half = 0.5f * trial_step[c];
    const float lj = s.wlj[c];
    float out = -INFINITY;
    if (s.valid[c] && own_finite(g, P) && isfinite(lj)) {
#pragma unroll
        for (int k = 0; k < K; ++k) p[k] = -fmaf(half, g[k], p[k]);
        out = s.H0[c] - (kinetic(p, im) - lj);
    }
    if (lane == 0) log_accept_ratio[c] = out;
}

// ---------------------------------------------------------------------------
// ChEES cross-chain statistics (api_batched_chees.jl:158-228), float64.
// ---------------------------------------------------------------------------
struct CheesArgs {
    const float* initials;   // C x P
    const float* proposals;  // C x P
    const float* momenta;    // C x P
    const float* accept;     // C
    const uint8_t* divergent;// C
    const float* inverse_mass;
    uint8_t* flags;          // C: bit0 initials finite, bit1 proposals+momenta finite, bit2 proposals finite
    double* means;           // 2 x P: initials mean, proposal mean
    double* chain_terms;     // 2 x C: numerator term, denominator term
    double* out;             // 2
    int P, C;
};

__global__ void chees_flags_kernel(CheesArgs a) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= a.C) return;
    bool fi = true, fp = true, fm = true;
    for (int p = lane; p < a.P; p += 32) {
        fi &= isfinite(a.initials[(size_t)c * a.P + p]);
        fp &= isfinite(a.proposals[(size_t)c * a.P + p]);
        fm &= isfinite(a.momenta[(size_t)c * a.P + p]);
    }
    fi = warp_all(fi); fp = warp_all(fp); fm = warp_all(fm);
    if (lane == 0) a.flags[c] = (fi ? 1 : 0) | ((fp && fm) ? 2 : 0) | (fp ? 4 : 0);
}

// one block per parameter: the two cross-chain means (fixed-order block sum)
__global__ void __launch_bounds__(256) chees_means_kernel(CheesArgs a) {
    __shared__ double s0[256], s1[256], s2[256];
    __shared__ int sc[256];
    const int p = blockIdx.x;
    double si = 0.0, sp = 0.0, sw = 0.0;
    int cnt = 0;
    for (int c = threadIdx.x; c < a.C; c += 256) {
        uint8_t f = a.flags[c];
        if (f & 1) { si += a.initials[(size_t)c * a.P + p]; cnt++; }
        if (!a.divergent[c] && (f & 4)) {
            double w = a.accept[c];
            sw += w;
            sp += w * (double)a.proposals[(size_t)c * a.P + p];
        }
    }
    s0[threadIdx.x] = si; s1[threadIdx.x] = sp; s2[threadIdx.x] = sw; sc[threadIdx.x] = cnt;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s0[threadIdx.x] += s0[threadIdx.x + o];
            s1[threadIdx.x] += s1[threadIdx.x + o];
            s2[threadIdx.x] += s2[threadIdx.x + o];
            sc[threadIdx.x] += sc[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        a.means[p] = sc[0] > 0 ? s0[0] / sc[0] : 0.0;
        a.means[a.P + p] = s1[0] * (1.0 / (s2[0] + 1e-20));
    }
}

__global__ void chees_terms_kernel(CheesArgs a) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + warp;
    if (c >= a.C) return;
    const bool use = !a.divergent[c] && (a.flags[c] & 2);
    double se = 0.0, ss = 0.0, ev = 0.0;
    if (use) {
        for (int p = lane; p < a.P; p += 32) {
            double sigma = a.inverse_mass[p];
            double is = 1.0 / sqrt(sigma);
            double we = ((double)a.proposals[(size_t)c * a.P + p] - a.means[a.P + p]) * is;
            double ws = ((double)a.initials[(size_t)c * a.P + p] - a.means[p]) * is;
            double wv = (double)a.momenta[(size_t)c * a.P + p] * sigma * is;
            se += we * we; ss += ws * ws; ev += we * wv;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            se += __shfl_xor_sync(UT_FULL_MASK, se, o);
            ss += __shfl_xor_sync(UT_FULL_MASK, ss, o);
            ev += __shfl_xor_sync(UT_FULL_MASK, ev, o);
        }
    }
    if (lane == 0) {
        double pa = a.accept[c];
        a.chain_terms[c] = use ? pa * (se - ss) * ev : 0.0;
        a.chain_terms[a.C + c] = use ? pa + 1e-20 : 0.0;
    }
}

__global__ void __launch_bounds__(256) chees_final_kernel(CheesArgs a) {
    __shared__ double s0[256], s1[256];
    double n = 0.0, d = 0.0;
    for (int c = threadIdx.x; c < a.C; c += 256) { n += a.chain_terms[c]; d += a.chain_terms[a.C + c]; }
    s0[threadIdx.x] = n; s1[threadIdx.x] = d;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) { s0[threadIdx.x] += s0[threadIdx.x + o]; s1[threadIdx.x] += s1[threadIdx.x + o]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { a.out[0] = s0[0]; a.out[1] = s1[0]; }
}

// ---------------------------------------------------------------------------
// Philox batch kernels (host-facing ut_philox4x32 / ut_rand_*).
// ---------------------------------------------------------------------------
__global__ void philox_batch_kernel(const uint32_t* keys, const uint32_t* ctrs, int64_t n, uint32_t* out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    U4 c = {ctrs[4 * i], ctrs[4 * i + 1], ctrs[4 * i + 2], ctrs[4 * i + 3]};
    U4 r = philox4x32(keys[2 * i], keys[2 * i + 1], c);
    out[4 * i] = r.x; out[4 * i + 1] = r.y; out[4 * i + 2] = r.z; out[4 * i + 3] = r.w;
}

__global__ void rand_batch_kernel(uint32_t chain, uint32_t iter, uint32_t stream, uint32_t draw_start, int64_t n,
                                  int normal, float* out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t d = draw_start + (uint32_t)i;
    out[i] = normal ? rand_normal(chain, iter, stream, d) : rand_uniform(chain, iter, stream, d);
}

}  // namespace ut

namespace ut {

// ---------------------------------------------------------------------------
// Pooled running variance (adaptation.jl:83-101, 170-209): one CTA, one
// thread per parameter, chains folded strictly in index order so the result
// equals the reference's sequential column loop.  Positions are staged
// through shared memory 32 chains at a time.
// Constants: clip start 4, early/late clip scale 8/5, variance floor 1e-3
// (data_types.jl:189-193).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) running_variance_kernel(const float* __restrict__ pos,
                                                                const double* __restrict__ w, int P, int C,
                                                                double* state, int window_length) {
    extern __shared__ float stage[];  // 32 x P
    const int p = threadIdx.x;
    double mean = 0.0, m2 = 0.0;
    if (p < P) { mean = state[p]; m2 = state[P + p]; }
    double count = state[2 * P], wsum = state[2 * P + 1], wsq = state[2 * P + 2];
    for (int c0 = 0; c0 < C; c0 += 32) {
        const int nc = min(32, C - c0);
        __syncthreads();
        for (int i = threadIdx.x; i < nc * P; i += blockDim.x) stage[i] = pos[(size_t)c0 * P + i];
        __syncthreads();
        for (int cc = 0; cc < nc; ++cc) {
            const double wt = w[c0 + cc];
            if (wt == 0.0) continue;
            double x = p < P ? (double)stage[cc * P + p] : 0.0;
            if (count >= 4.0) {
                double scale;
                if (count <= 4.0) {
                    scale = 8.0;
                } else {
                    double prog = window_length <= 4 ? 1.0 : fmin(fmax(count - 4.0, 0.0) / (double)(window_length - 4), 1.0);
                    scale = 8.0 + (5.0 - 8.0) * prog;
                }
                double var = m2 / fmax(count - 1.0, 1.0);
                double bound = scale * sqrt(fmax(var, 1e-3));
                double delta = x - mean;
                x = mean + fmin(fmax(delta, -bound), bound);
            }
            count += 1.0;
            const double nws = wsum + wt;
            const double delta = x - mean;
            mean += (wt / nws) * delta;
            const double delta2 = x - mean;
            m2 += wt * delta * delta2;
            wsum = nws;
            wsq += wt * wt;
        }
    }
    if (p < P) { state[p] = mean; state[P + p] = m2; }
    __syncthreads();
    if (threadIdx.x == 0) { state[2 * P] = count; state[2 * P + 1] = wsum; state[2 * P + 2] = wsq; }
}

// One warmup iteration's adaptation on the device, so the single-model
// samplers copy nothing to the host between mass-window ends (one CTA):
//  * running-variance weights (adaptation.jl:225-260): 1 for an accepted
//    chain, 0 for a divergent one, else the rejection weight
//    1 + (clamp(accept_prob, 0, 1) - 1) * progress (0 when accept_prob is not
//    finite), with the window progress of adaptation.jl:56-65 taken from the
//    running-variance state's count (var[2P]);
//  * one dual-averaging update (adaptation.jl:1-28; gamma 0.05, t0 10, kappa
//    0.75) of each chain's state (per_chain) with the chain's statistic, 0 when
//    divergent, or of one shared state with the mean statistic over chains
//    (hmc_support.jl:635-652, summed in a fixed order); the new step sizes go
//    to step[C].  State: [mu, log step, log step avg, hbar, iteration] doubles.
__device__ __forceinline__ double dual_averaging_update(double* s, double stat, double target) {
    const double it = s[4] + 1.0;
    const double eta = 1.0 / (it + 10.0);
    s[3] = (1.0 - eta) * s[3] + eta * (target - stat);
    s[1] = s[0] - sqrt(it) / 0.05 * s[3];
    const double eta_bar = pow(it, -0.75);
    s[2] = eta_bar * s[1] + (1.0 - eta_bar) * s[2];
    s[4] = it;
    return s[1];
}

__global__ void __launch_bounds__(1024) warmup_adapt_kernel(const float* __restrict__ ap, const uint8_t* __restrict__ acc,
                                                            const uint8_t* __restrict__ div, int C, int P,
                                                            const double* __restrict__ var, int window_length,
                                                            double* weights, double* dual, int per_chain, int adapt,
                                                            double target, float* step) {
    __shared__ double red[1024];
    __shared__ float shared_step;
    const double count = var ? var[2 * P] : 0.0;
    const double prog = window_length <= 4 ? 1.0 : fmin(fmax(count - 4.0, 0.0) / (double)(window_length - 4), 1.0);
    double part = 0.0;
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        const double a = (double)ap[c];
        const bool dv = div[c] != 0;
        if (weights) {
            double w = isfinite(a) ? 1.0 + (fmin(fmax(a, 0.0), 1.0) - 1.0) * prog : 0.0;
            if (acc && acc[c]) w = 1.0;
            weights[c] = dv ? 0.0 : w;
        }
        const double stat = dv ? 0.0 : a;
        if (adapt && per_chain) step[c] = (float)exp(dual_averaging_update(dual + 5 * (size_t)c, stat, target));
        part += stat;
    }
    if (!adapt || per_chain) return;
    red[threadIdx.x] = part;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) shared_step = (float)exp(dual_averaging_update(dual, red[0] / (double)C, target));
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) step[c] = shared_step;
}

// Final warmup step sizes exp(log step avg) (adaptation.jl:25-28).
__global__ void dual_averaging_final_kernel(const double* dual, int C, int per_chain, float* step) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < C) step[c] = (float)exp(dual[per_chain ? 5 * (size_t)c + 2 : 2]);
}

}  // namespace ut
