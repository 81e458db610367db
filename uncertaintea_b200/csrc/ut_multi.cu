// ut_multi.cu -- uneven batching: many independent non-centred hierarchical
// normal models, each with its own group count, group sizes, priors and chain
// count, sampled together by batched persistent NUTS.
//
// Layout.  Every model's data is one contiguous pack -- sigma, start and
// count per group, then its observations group after group -- which a CTA
// either stages in shared memory (a data tile shared by the CTA's chains) or
// reads through L2; each model's chains own a contiguous C_m x P_m block of
// the position / gradient arrays.  Models are grouped into slot-count classes
// (K = parameter slots per lane, P_m <= 32 K); each class has a work list of
// (model, first chain, chain count) items ordered costliest first, one item
// per CTA, one warp per chain.
//
// One iteration = one persistent-NUTS launch per class (on forked streams, so
// the classes share the GPU), then one adaptation kernel (warmup: per-model
// dual averaging of the step size and windowed Welford estimates of the
// diagonal mass) or one draw-recording kernel (sampling), then a counter
// increment.  The iteration index lives in device memory, so one captured CUDA
// graph of kGraphIters iterations is replayed for the whole run.
//
// The autotuner times, per class, every (chains per CTA, shared-memory
// staging) candidate on the same iteration from a saved state and keeps the
// fastest; results do not depend on the choice (the trees and Philox streams
// are per chain).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/ut_b200.h"

namespace {  // the kernels below are private to this file
#include "ut_warp_kernels.cuh"
}

// Defined in ut_api.cu: stores the message that ut_last_error returns.
void ut_internal_set_last_error(const char* msg);

namespace {

using namespace ut;

constexpr int kNumClasses = 8;
constexpr int kClassK[kNumClasses] = {1, 2, 3, 4, 6, 8, 12, 17};
constexpr int kMaxParams = 32 * 17;
constexpr int kGraphIters = 8;
constexpr int kMaxWarps = 4;                    // chains per CTA at most (launch bound 128 threads)
constexpr int kStageMax = 200 * 1024;           // largest shared-memory staging we allow
constexpr int kCandW[3] = {1, 2, 4};
constexpr int kCandStage[2] = {0, kStageMax};

enum : uint8_t { kActWelford = 1, kActWindowEnd = 2, kActFinal = 4 };

struct MmModel {
    int32_t J, N, P, C;
    int64_t pack_off;     // first float of the model's data pack (a multiple of 4)
    int32_t pack_floats;  // pack length: 3 J + N rounded up to 4
    int32_t chain_off;    // first (global) chain of the model
    int64_t state_off;    // first float of the model's C x P block of position / gradient
    int32_t param_off;    // first float of the model's P inverse-mass entries
    int32_t klass;
    float mu_loc, mu_scale, tau_scale;
};

// The model's evaluator view of its pack [sigma (J), start (J), count (J), y (N)].
__device__ __forceinline__ HierModel mm_hier(const float* pack, const MmModel& m) {
    HierModel h;
    h.N = m.N;
    h.J = m.J;
    h.mu_loc = m.mu_loc;
    h.mu_scale = m.mu_scale;
    h.tau_scale = m.tau_scale;
    h.sig = pack;
    h.start = reinterpret_cast<const int32_t*>(pack + m.J);
    h.count = reinterpret_cast<const int32_t*>(pack + 2 * m.J);
    h.y = pack + 3 * m.J;
    return h;
}

// Copies the model's pack into shared memory (all threads of the CTA).
__device__ __forceinline__ const float* mm_stage(const float* src, int floats, float* smem) {
    const float4* s4 = reinterpret_cast<const float4*>(src);
    float4* d4 = reinterpret_cast<float4*>(smem);
    for (int i = threadIdx.x; i < floats / 4; i += blockDim.x) d4[i] = s4[i];
    __syncthreads();
    return smem;
}

struct MmItem {
    int32_t model, chain0, nchains, pad;
};

struct MmArgs {
    const MmModel* models;
    const MmItem* items;
    const float* packs;
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
    float* ckpt;               // this class's checkpoint stacks, indexed by class slot
    const int32_t* class_slot; // global chain -> index within its class
    const int32_t* counter;    // iteration index (device)
    uint32_t seed;             // Philox iteration coordinate = seed + *counter
    int max_depth;
    float thr;
    int stage_limit;           // stage a model in shared memory when its data fits in this many bytes
    // warmup: per-chain step search at the first iteration and after every mass window
    float* step_out;           // per chain (the search writes its result here)
    double* da;                // per chain dual-averaging state: mu, log_eps, log_eps_avg, hbar, t
    const uint8_t* actions;
    int num_warmup;
    const uint8_t* model_done; // per model: 1 = stopped (its items do nothing)
};

// log accept ratio H0 - H1 of one leapfrog step of size h from (q, g, lj)
// with momentum p (-Inf when the end point is not finite).
template <int K>
__device__ __forceinline__ float mm_probe(const float* pack, const MmModel& m, const float (&q)[K], const float (&g)[K],
                                          const float (&p)[K], const float (&im)[K], float lj, float h) {
    float qn[K], gn[K], pn[K];
    const float half = 0.5f * h;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        pn[k] = fmaf(half, g[k], p[k]);
        qn[k] = fmaf(h * im[k], pn[k], q[k]);
    }
    const float H0 = kinetic(p, im) - lj;
    const float lj1 = hier_lj_grad<K>(mm_hier(pack, m), m.P, qn, gn, true);
    if (!(isfinite(lj1) && own_finite(gn, m.P))) return -INFINITY;
#pragma unroll
    for (int k = 0; k < K; ++k) pn[k] = fmaf(half, gn[k], pn[k]);
    return H0 - (kinetic(pn, im) - lj1);
}

// Per-chain reasonable step size (adaptation.jl:438-514, as the single-model
// per-chain search): one momentum draw; double or halve the step until the
// one-step acceptance crosses 1/2, at most 20 times, within [1e-8, 1e3].
template <int K>
__device__ float mm_find_step(const float* pack, const MmModel& m, const NutsChainIO& io, float h, uint32_t chain,
                              uint32_t coord) {
    const int lane = threadIdx.x & 31;
    const int P = m.P;
    float q[K], g[K], p[K], im[K];
    load_vec(q, io.position, P);
    load_vec(g, io.gradient, P);
    load_vec(im, io.inverse_mass, P);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int pp = lane + 32 * k;
        p[k] = pp < P ? rand_normal(chain, coord, kStreamMomentum, (uint32_t)pp) / sqrtf(im[k]) : 0.0f;
    }
    const float lj = *io.logjoint;
    const float log_target = -0.6931471805599453f;
    double step = h;
    float lar = mm_probe<K>(pack, m, q, g, p, im, lj, (float)step);
    const double dir = lar > log_target ? 1.0 : -1.0;
    for (int t = 0; t < 20; ++t) {
        const double nxt = dir > 0 ? step * 2.0 : step * 0.5;
        if (nxt < 1e-8 || nxt > 1e3) break;
        lar = mm_probe<K>(pack, m, q, g, p, im, lj, (float)nxt);
        step = nxt;
        if ((dir > 0 && lar <= log_target) || (dir < 0 && lar >= log_target)) break;
    }
    return (float)fmin(fmax(step, 1e-8), 1e3);
}

// One NUTS iteration for every chain of one work item per CTA (preceded, at
// the first warmup iteration and after every mass window, by the chain's
// step-size search).
template <int K>
__global__ void __launch_bounds__(32 * kMaxWarps) mm_nuts_kernel(MmArgs a) {
    extern __shared__ float smem[];
    const MmItem item = a.items[blockIdx.x];
    if (a.model_done[item.model]) return;  // a stopped model's chains keep their state (uniform per CTA)
    const MmModel m = a.models[item.model];
    const float* pack = a.packs + m.pack_off;
    if ((int64_t)m.pack_floats * 4 <= (int64_t)a.stage_limit) pack = mm_stage(pack, m.pack_floats, smem);
    const int warp = threadIdx.x >> 5;
    if (warp >= item.nchains) return;
    const int local = item.chain0 + warp;
    const int c = m.chain_off + local;
    NutsChainIO io;
    io.position = a.position + m.state_off + (int64_t)local * m.P;
    io.gradient = a.gradient + m.state_off + (int64_t)local * m.P;
    io.logjoint = a.logjoint + c;
    io.inverse_mass = a.inverse_mass + m.param_off;
    io.step = a.step[c];
    io.accept_prob = a.accept_prob + c;
    io.energy = a.energy + c;
    io.energy_error = a.energy_error + c;
    io.tree_depth = a.tree_depth + c;
    io.integration_steps = a.integration_steps + c;
    io.divergent = a.divergent + c;
    io.moved = a.moved + c;
    const int it = *a.counter;
    if (it < a.num_warmup && (it == 0 || (a.actions[it - 1] & kActWindowEnd))) {
        const float h = mm_find_step<K>(pack, m, io, io.step, (uint32_t)c, a.seed + 0x80000000u + (uint32_t)it);
        io.step = h;
        if ((threadIdx.x & 31) == 0) {  // restart the chain's dual averaging at the new step
            a.step_out[c] = h;
            double* da = a.da + 5 * (size_t)c;
            const double ls = log((double)h);
            da[0] = log(10.0 * (double)h); da[1] = ls; da[2] = ls; da[3] = 0.0; da[4] = 0.0;
        }
    }
    float* ck = a.ckpt + (size_t)a.class_slot[c] * (a.max_depth + 1) * 2 * (32 * K);
    const uint32_t coord = a.seed + (uint32_t)it;
    const HierModel hm = mm_hier(pack, m);
    auto eval = [&](const float (&qq)[K], float (&gg)[K]) { return hier_lj_grad<K>(hm, m.P, qq, gg, true); };
    nuts_chain<K>(eval, m.P, io, (uint32_t)c, coord, a.max_depth, a.thr, ck);
}

// Logjoint + gradient at the current positions, one warp per chain.
template <int K>
__global__ void __launch_bounds__(32 * kMaxWarps) mm_density_kernel(MmArgs a) {
    const MmItem item = a.items[blockIdx.x];
    const MmModel m = a.models[item.model];
    const int warp = threadIdx.x >> 5;
    if (warp >= item.nchains) return;
    const int local = item.chain0 + warp;
    float q[K], g[K];
    load_vec(q, a.position + m.state_off + (int64_t)local * m.P, m.P);
    const float lj = hier_lj_grad<K>(mm_hier(a.packs + m.pack_off, m), m.P, q, g, true);
    store_vec(a.gradient + m.state_off + (int64_t)local * m.P, g, m.P);
    if ((threadIdx.x & 31) == 0) a.logjoint[m.chain_off + local] = lj;
}

// ---- warmup adaptation (one CTA per model) -----------------------------------
// The reference's default batched-NUTS warmup (a pooled diagonal mass per
// model and a dual-averaged step per chain, warmup.jl:362-473): every chain's
// step follows its own accept statistic (0 for a divergent transition,
// hmc_support.jl:635-652); the model's non-divergent positions feed its
// Welford window; at a window end the inverse mass becomes the window's
// variance shrunk towards 1e-3, and the next iteration re-searches every
// chain's step (mm_nuts_kernel).
struct MmAdaptArgs {
    const MmModel* models;
    const int32_t* counter;
    const uint8_t* actions;   // num_warmup entries
    int num_warmup;
    float target_accept;
    const float* accept_prob;
    const uint8_t* divergent;
    const float* position;
    float* inverse_mass;
    float* step;              // per chain
    double* da;               // per chain: mu, log_eps, log_eps_avg, hbar, t
    double* wmean;            // per parameter
    double* wm2;
    double* wcount;           // per model
    const uint8_t* model_done; // per model: 1 = stopped (its adaptation state stays)
};

constexpr double kDaGamma = 0.05, kDaT0 = 10.0, kDaKappa = 0.75;

__global__ void __launch_bounds__(256) mm_adapt_kernel(MmAdaptArgs a) {
    const int it = *a.counter;
    if (it >= a.num_warmup) return;
    if (a.model_done[blockIdx.x]) return;
    const MmModel m = a.models[blockIdx.x];
    const uint8_t act = a.actions[it];
    __shared__ int included;
    // per-chain dual averaging (DualAveraging.update / final)
    for (int lc = threadIdx.x; lc < m.C; lc += blockDim.x) {
        const int c = m.chain_off + lc;
        double* da = a.da + 5 * (size_t)c;
        const double accept = a.divergent[c] ? 0.0 : (double)a.accept_prob[c];
        const double t = da[4] + 1.0;
        const double eta = 1.0 / (t + kDaT0);
        const double hbar = (1.0 - eta) * da[3] + eta * ((double)a.target_accept - accept);
        const double log_eps = da[0] - sqrt(t) / kDaGamma * hbar;
        const double eta_bar = pow(t, -kDaKappa);
        const double log_avg = eta_bar * log_eps + (1.0 - eta_bar) * da[2];
        da[1] = log_eps; da[2] = log_avg; da[3] = hbar; da[4] = t;
        a.step[c] = (float)exp((act & kActFinal) ? log_avg : log_eps);
    }
    const double n0 = a.wcount[blockIdx.x];
    if (threadIdx.x == 0) {
        int n = 0;
        for (int lc = 0; lc < m.C; ++lc) n += a.divergent[m.chain_off + lc] ? 0 : 1;
        included = (act & kActWelford) ? n : 0;
    }
    if (act & kActWelford) {
        for (int p = threadIdx.x; p < m.P; p += blockDim.x) {
            double mean = a.wmean[m.param_off + p], m2 = a.wm2[m.param_off + p], n = n0;
            for (int lc = 0; lc < m.C; ++lc) {
                if (a.divergent[m.chain_off + lc]) continue;
                const double x = a.position[m.state_off + (int64_t)lc * m.P + p];
                n += 1.0;
                const double d = x - mean;
                mean += d / n;
                m2 += d * (x - mean);
            }
            a.wmean[m.param_off + p] = mean;
            a.wm2[m.param_off + p] = m2;
        }
    }
    __syncthreads();
    const double n1 = n0 + included;
    if (act & kActWindowEnd) {
        // regularised variance estimate, shrunk towards 1e-3 (windowed adaptation)
        for (int p = threadIdx.x; p < m.P; p += blockDim.x) {
            if (n1 > 1.0) {
                const double var = a.wm2[m.param_off + p] / (n1 - 1.0);
                a.inverse_mass[m.param_off + p] = (float)((n1 / (n1 + 5.0)) * var + 1e-3 * (5.0 / (n1 + 5.0)));
            }
            a.wmean[m.param_off + p] = 0.0;
            a.wm2[m.param_off + p] = 0.0;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) a.wcount[blockIdx.x] = (act & kActWindowEnd) ? 0.0 : n1;
}

// ---- sampling: draw recording and the iteration counter ------------------------
__global__ void mm_record_kernel(const int32_t* counter, int num_warmup, int capacity, const float* position,
                                 int64_t state_floats, float* draws, const float* accept_prob,
                                 const int32_t* tree_depth, const uint8_t* divergent, int64_t total_chains,
                                 float* draw_accept, int32_t* draw_depth, uint8_t* draw_div) {
    const int it = *counter;
    const int s = it - num_warmup;
    if (s < 0 || s >= capacity) return;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float* dst = draws + (int64_t)s * state_floats;
    for (int64_t i = i0; i < state_floats; i += stride) dst[i] = position[i];
    for (int64_t i = i0; i < total_chains; i += stride) {
        draw_accept[(int64_t)s * total_chains + i] = accept_prob[i];
        draw_depth[(int64_t)s * total_chains + i] = tree_depth[i];
        draw_div[(int64_t)s * total_chains + i] = divergent[i];
    }
}

__global__ void mm_counter_kernel(int32_t* counter) { *counter += 1; }

// ---- split R-hat of every model over its first S draws (one CTA per model) -----
// Each chain is split into halves of n = S / 2 draws (draws [0, n) and
// [n, 2n); an odd last draw is dropped), R-hat = sqrt(max(var+ / W, 1)) with
// W the mean within-half variance and var+ = (n-1)/n W + B/n
// (diagnostics.jl:461-528); the model's value is the max over its parameters.
__global__ void __launch_bounds__(256) mm_split_rhat_kernel(const MmModel* models, const float* draws,
                                                            int64_t state_floats, int S, float* out) {
    const MmModel m = models[blockIdx.x];
    __shared__ float red[256];
    const int n = S / 2;
    float worst = 0.0f;
    for (int p = threadIdx.x; p < m.P; p += blockDim.x) {
        double sum_mean = 0.0, sum_mean2 = 0.0, sum_var = 0.0;
        const int M2 = 2 * m.C;
        for (int c = 0; c < m.C; ++c) {
            const float* base = draws + m.state_off + (int64_t)c * m.P + p;
            for (int h = 0; h < 2; ++h) {
                const int s0 = h * n;
                double mu = 0.0;
                for (int s = 0; s < n; ++s) mu += base[(int64_t)(s0 + s) * state_floats];
                mu /= n;
                double v = 0.0;
                for (int s = 0; s < n; ++s) {
                    const double d = base[(int64_t)(s0 + s) * state_floats] - mu;
                    v += d * d;
                }
                v /= (n - 1);
                sum_mean += mu;
                sum_mean2 += mu * mu;
                sum_var += v;
            }
        }
        const double W = sum_var / M2;
        const double grand = sum_mean / M2;
        const double B_over_n = (sum_mean2 - M2 * grand * grand) / (M2 - 1);
        const double var_plus = (double)(n - 1) / n * W + B_over_n;
        double r;
        if (W == 0.0) r = var_plus == 0.0 ? 1.0 : INFINITY;
        else r = sqrt(fmax(var_plus / W, 1.0));
        worst = fmaxf(worst, (float)r);
    }
    red[threadIdx.x] = worst;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

int32_t mfail(int32_t code, const char* fmt, ...) {
    char buf[768];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ut_internal_set_last_error(buf);
    return code;
}

#define MM_CUDA(call)                                                                                    \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) return mfail(UT_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

#define MM_LAUNCHED()                                                                                    \
    do {                                                                                                 \
        cudaError_t e_ = cudaGetLastError();                                                             \
        if (e_ != cudaSuccess) return mfail(UT_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e_)); \
    } while (0)

int class_of(int P) {
    for (int i = 0; i < kNumClasses; ++i)
        if (P <= 32 * kClassK[i]) return i;
    return -1;
}

struct MmClass {
    int K = 0;
    std::vector<int> model_ids;
    int64_t chains = 0;
    int W = 4;                   // chains per CTA
    int stage_limit = kStageMax;
    int num_items = 0;
    MmItem* items = nullptr;     // capacity: one item per chain
    float* ckpt = nullptr;
    size_t smem = 0;             // dynamic shared memory of the current configuration
};

}  // namespace

struct ut_multi {
    int M = 0;
    int device = 0;
    int max_depth = 10;
    std::vector<MmModel> models_h;
    MmModel* models = nullptr;
    float* packs = nullptr;
    int64_t pack_total = 0;
    int64_t total_chains = 0, state_floats = 0, param_floats = 0;
    float *position = nullptr, *gradient = nullptr, *logjoint = nullptr, *inverse_mass = nullptr, *step = nullptr;
    float *accept_prob = nullptr, *energy = nullptr, *energy_error = nullptr;
    int32_t *tree_depth = nullptr, *integration_steps = nullptr;
    uint8_t *divergent = nullptr, *moved = nullptr;
    int32_t* class_slot = nullptr;
    MmClass classes[kNumClasses];
    // adaptation and run state
    double *da = nullptr, *wmean = nullptr, *wm2 = nullptr, *wcount = nullptr;
    uint8_t* actions = nullptr;
    uint8_t* model_done = nullptr;  // per model stop flags (device)
    int num_warmup = 0, num_samples = 0;
    float target_accept = 0.8f, thr = 1000.0f;
    uint32_t seed = 0;
    int32_t* counter = nullptr;
    float* draws = nullptr;
    float* draw_accept = nullptr;
    int32_t* draw_depth = nullptr;
    uint8_t* draw_div = nullptr;
    int draws_capacity = 0;
    bool begun = false;
    // streams and the captured graph
    cudaStream_t stream = nullptr;
    cudaStream_t side[kNumClasses] = {};
    cudaEvent_t fork = nullptr, join[kNumClasses] = {}, user_ev = nullptr, done_ev = nullptr;
    cudaGraphExec_t graph = nullptr;
    // autotune save area
    float* save = nullptr;
    double* save_da = nullptr;
    std::vector<void*> allocations;
    std::vector<void*> run_allocations;  // draws etc., replaced by every begin
};

namespace {

template <class T>
int32_t malloc_into(std::vector<void*>& list, T** p, size_t count) {
    void* v = nullptr;
    cudaError_t e = cudaMalloc(&v, (count ? count : 1) * sizeof(T));
    if (e != cudaSuccess)
        return mfail(UT_ERR_CUDA, "cudaMalloc(%zu bytes) failed: %s", count * sizeof(T), cudaGetErrorString(e));
    list.push_back(v);
    *p = static_cast<T*>(v);
    return UT_OK;
}

void drop_graph(ut_multi* mm) {
    if (mm->graph) cudaGraphExecDestroy(mm->graph);
    mm->graph = nullptr;
}

void release_all(ut_multi* mm) {
    drop_graph(mm);
    for (void* p : mm->run_allocations) cudaFree(p);
    for (void* p : mm->allocations) cudaFree(p);
    mm->run_allocations.clear();
    mm->allocations.clear();
    for (int k = 0; k < kNumClasses; ++k) {
        if (mm->side[k]) cudaStreamDestroy(mm->side[k]);
        if (mm->join[k]) cudaEventDestroy(mm->join[k]);
    }
    if (mm->stream) cudaStreamDestroy(mm->stream);
    if (mm->fork) cudaEventDestroy(mm->fork);
    if (mm->user_ev) cudaEventDestroy(mm->user_ev);
    if (mm->done_ev) cudaEventDestroy(mm->done_ev);
}

MmArgs base_args(const ut_multi* mm, const MmClass& cl) {
    MmArgs a;
    a.models = mm->models; a.items = cl.items;
    a.packs = mm->packs;
    a.position = mm->position; a.gradient = mm->gradient; a.logjoint = mm->logjoint;
    a.inverse_mass = mm->inverse_mass; a.step = mm->step;
    a.accept_prob = mm->accept_prob; a.energy = mm->energy; a.energy_error = mm->energy_error;
    a.tree_depth = mm->tree_depth; a.integration_steps = mm->integration_steps;
    a.divergent = mm->divergent; a.moved = mm->moved;
    a.ckpt = cl.ckpt; a.class_slot = mm->class_slot; a.counter = mm->counter; a.seed = mm->seed;
    a.max_depth = mm->max_depth; a.thr = mm->thr; a.stage_limit = cl.stage_limit;
    a.step_out = mm->step; a.da = mm->da; a.actions = mm->actions; a.num_warmup = mm->num_warmup;
    a.model_done = mm->model_done;
    return a;
}

#define MM_K_SWITCH(KV, ...)                                   \
    switch (KV) {                                              \
        case 1: { constexpr int K = 1; __VA_ARGS__; } break;   \
        case 2: { constexpr int K = 2; __VA_ARGS__; } break;   \
        case 3: { constexpr int K = 3; __VA_ARGS__; } break;   \
        case 4: { constexpr int K = 4; __VA_ARGS__; } break;   \
        case 6: { constexpr int K = 6; __VA_ARGS__; } break;   \
        case 8: { constexpr int K = 8; __VA_ARGS__; } break;   \
        case 12: { constexpr int K = 12; __VA_ARGS__; } break; \
        default: { constexpr int K = 17; __VA_ARGS__; } break; \
    }

// Rebuilds one class's work list for `W` chains per CTA (costliest items
// first: cost = chains x (N + J)) and its shared-memory size.
int32_t build_items(ut_multi* mm, MmClass& cl, int W, int stage_limit) {
    std::vector<MmItem> items;
    size_t smem = 0;
    for (int id : cl.model_ids) {
        const MmModel& m = mm->models_h[id];
        for (int c0 = 0; c0 < m.C; c0 += W) items.push_back(MmItem{id, c0, std::min(W, m.C - c0), 0});
        const size_t bytes = (size_t)m.pack_floats * 4;
        if (bytes <= (size_t)stage_limit) smem = std::max(smem, bytes);
    }
    auto cost = [&](const MmItem& it) {
        const MmModel& m = mm->models_h[it.model];
        return (double)it.nchains * (double)m.pack_floats;
    };
    std::stable_sort(items.begin(), items.end(), [&](const MmItem& a, const MmItem& b) { return cost(a) > cost(b); });
    if (!items.empty())
        MM_CUDA(cudaMemcpy(cl.items, items.data(), items.size() * sizeof(MmItem), cudaMemcpyHostToDevice));
    cl.num_items = (int)items.size();
    cl.W = W;
    cl.stage_limit = stage_limit;
    cl.smem = smem;
    // permission for the largest staging any configuration uses (reserves nothing)
    MM_K_SWITCH(cl.K, MM_CUDA(cudaFuncSetAttribute(mm_nuts_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   kStageMax)));
    return UT_OK;
}

int32_t launch_class_nuts(ut_multi* mm, const MmClass& cl, cudaStream_t st) {
    if (cl.num_items == 0) return UT_OK;
    MmArgs a = base_args(mm, cl);
    MM_K_SWITCH(cl.K, (mm_nuts_kernel<K><<<cl.num_items, 32 * cl.W, cl.smem, st>>>(a)));
    MM_LAUNCHED();
    return UT_OK;
}

// One iteration: the classes' NUTS launches forked onto the side streams, then
// adaptation / draw recording / counter on `st`.
int32_t enqueue_iteration(ut_multi* mm, cudaStream_t st) {
    int32_t rc;
    MM_CUDA(cudaEventRecord(mm->fork, st));
    for (int k = 0; k < kNumClasses; ++k) {
        MmClass& cl = mm->classes[k];
        if (cl.num_items == 0) continue;
        MM_CUDA(cudaStreamWaitEvent(mm->side[k], mm->fork, 0));
        if ((rc = launch_class_nuts(mm, cl, mm->side[k]))) return rc;
        MM_CUDA(cudaEventRecord(mm->join[k], mm->side[k]));
        MM_CUDA(cudaStreamWaitEvent(st, mm->join[k], 0));
    }
    MmAdaptArgs ad;
    ad.models = mm->models; ad.counter = mm->counter; ad.actions = mm->actions; ad.num_warmup = mm->num_warmup;
    ad.target_accept = mm->target_accept; ad.accept_prob = mm->accept_prob; ad.divergent = mm->divergent;
    ad.position = mm->position;
    ad.inverse_mass = mm->inverse_mass; ad.step = mm->step; ad.da = mm->da; ad.wmean = mm->wmean; ad.wm2 = mm->wm2;
    ad.wcount = mm->wcount;
    ad.model_done = mm->model_done;
    mm_adapt_kernel<<<mm->M, 256, 0, st>>>(ad);
    MM_LAUNCHED();
    if (mm->draws_capacity > 0) {
        mm_record_kernel<<<592, 256, 0, st>>>(mm->counter, mm->num_warmup, mm->draws_capacity, mm->position,
                                              mm->state_floats, mm->draws, mm->accept_prob, mm->tree_depth,
                                              mm->divergent, mm->total_chains, mm->draw_accept, mm->draw_depth,
                                              mm->draw_div);
        MM_LAUNCHED();
    }
    mm_counter_kernel<<<1, 1, 0, st>>>(mm->counter);
    MM_LAUNCHED();
    return UT_OK;
}

int32_t capture_graph(ut_multi* mm) {
    drop_graph(mm);
    MM_CUDA(cudaStreamBeginCapture(mm->stream, cudaStreamCaptureModeThreadLocal));
    int32_t rc = UT_OK;
    for (int i = 0; i < kGraphIters && rc == UT_OK; ++i) rc = enqueue_iteration(mm, mm->stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(mm->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return mfail(UT_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&mm->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        mm->graph = nullptr;
        return mfail(UT_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
    }
    return UT_OK;
}

int32_t check_mm(const ut_multi* mm) {
    if (!mm) return mfail(UT_ERR_ARGUMENT, "null multi-model handle");
    return UT_OK;
}

}  // namespace

extern "C" {

int32_t ut_multi_create(int32_t num_models, const ut_plan_desc* plans, const float* observed,
                        const int64_t* observed_offsets, const int32_t* trip_counts, const int32_t* loop_starts,
                        const int32_t* chains, int32_t max_tree_depth, ut_multi** out) {
    if (!out) return mfail(UT_ERR_ARGUMENT, "null output handle");
    *out = nullptr;
    if (num_models < 1) return mfail(UT_ERR_ARGUMENT, "num_models must be >= 1, got %d", (int)num_models);
    if (!plans || !observed || !observed_offsets || !trip_counts || !loop_starts || !chains)
        return mfail(UT_ERR_ARGUMENT, "null input array");
    if (max_tree_depth < 1 || max_tree_depth > 30)
        return mfail(UT_ERR_ARGUMENT, "max_tree_depth must be in 1..30, got %d", (int)max_tree_depth);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return mfail(UT_ERR_NO_DEVICE, "no CUDA device visible");
    }
    // ---- validate, lay out and pack every model's data (host) ----
    std::vector<MmModel> ms(num_models);
    int64_t grp_total = 0, chain_total = 0, state_total = 0, param_total = 0, pack_total = 0;
    if (observed_offsets[0] != 0) return mfail(UT_ERR_ARGUMENT, "observed_offsets[0] must be 0");
    for (int i = 0; i < num_models; ++i) {
        const ut_plan_desc& p = plans[i];
        if (p.family != UT_FAMILY_HIER_NORMAL_NONCENTERED)
            return mfail(UT_ERR_UNSUPPORTED, "model %d: only the non-centred hierarchical family is batched", i);
        if (p.num_groups < 1 || p.num_params != p.num_groups + 2 || p.num_params > kMaxParams)
            return mfail(UT_ERR_ARGUMENT, "model %d: needs 1 <= num_groups, num_params = num_groups + 2 <= %d", i,
                         kMaxParams);
        if (p.num_obs < 0) return mfail(UT_ERR_ARGUMENT, "model %d: num_obs must be >= 0", i);
        if (!(p.mu_scale > 0.0) || !(p.tau_scale > 0.0))
            return mfail(UT_ERR_ARGUMENT, "model %d: prior scales must be > 0", i);
        if (chains[i] < 1) return mfail(UT_ERR_ARGUMENT, "model %d: chain count must be >= 1", i);
        if (observed_offsets[i + 1] - observed_offsets[i] != (int64_t)p.num_obs + p.num_groups)
            return mfail(UT_ERR_DIMENSION, "model %d: observed block must hold num_obs + num_groups values", i);
        for (int j = 0; j < p.num_groups; ++j) {
            const int64_t s0 = loop_starts[grp_total + j], n = trip_counts[grp_total + j];
            if (s0 < 0 || n < 0 || s0 + n > p.num_obs)
                return mfail(UT_ERR_DIMENSION, "model %d group %d: rows [%lld, %lld) outside the model's %d observations",
                             i, j, (long long)s0, (long long)(s0 + n), p.num_obs);
        }
        const int64_t pack = (3 * (int64_t)p.num_groups + p.num_obs + 3) / 4 * 4;
        if (pack > INT32_MAX) return mfail(UT_ERR_ARGUMENT, "model %d: data too large", i);
        MmModel& m = ms[i];
        m.J = p.num_groups; m.N = p.num_obs; m.P = p.num_params; m.C = chains[i];
        m.pack_off = pack_total; m.pack_floats = (int32_t)pack;
        m.chain_off = (int32_t)chain_total;
        m.state_off = state_total; m.param_off = (int32_t)param_total;
        m.klass = class_of(m.P);
        m.mu_loc = (float)p.mu_loc; m.mu_scale = (float)p.mu_scale; m.tau_scale = (float)p.tau_scale;
        grp_total += m.J; chain_total += m.C; pack_total += pack;
        state_total += (int64_t)m.C * m.P; param_total += m.P;
        if (chain_total > INT32_MAX || grp_total > INT32_MAX || param_total > INT32_MAX)
            return mfail(UT_ERR_ARGUMENT, "too many chains / groups / parameters in one batch");
    }
    std::vector<float> packs((size_t)std::max<int64_t>(pack_total, 4), 0.0f);
    {
        int64_t goff = 0;
        for (int i = 0; i < num_models; ++i) {
            const MmModel& m = ms[i];
            const float* blk = observed + observed_offsets[i];  // y (N) then sigma (J)
            float* pk = packs.data() + m.pack_off;
            int32_t* st = reinterpret_cast<int32_t*>(pk + m.J);
            int32_t* ct = reinterpret_cast<int32_t*>(pk + 2 * m.J);
            for (int j = 0; j < m.J; ++j) {
                pk[j] = blk[m.N + j];
                st[j] = loop_starts[goff + j];
                ct[j] = trip_counts[goff + j];
            }
            std::copy(blk, blk + m.N, pk + 3 * m.J);
            goff += m.J;
        }
    }
    ut_multi* mm = new ut_multi();
    mm->M = num_models;
    mm->max_depth = max_tree_depth;
    mm->models_h = ms;
    mm->total_chains = chain_total;
    mm->state_floats = state_total;
    mm->param_floats = param_total;
    mm->pack_total = pack_total;
    cudaGetDevice(&mm->device);
    auto bail = [&](int32_t rc) {
        release_all(mm);
        delete mm;
        return rc;
    };
    int32_t rc;
    auto& L = mm->allocations;
    if ((rc = malloc_into(L, &mm->models, num_models)) || (rc = malloc_into(L, &mm->packs, packs.size())) ||
        (rc = malloc_into(L, &mm->position, state_total)) ||
        (rc = malloc_into(L, &mm->gradient, state_total)) || (rc = malloc_into(L, &mm->save, 2 * state_total + 2 * chain_total)) ||
        (rc = malloc_into(L, &mm->save_da, 5 * (size_t)chain_total)) ||
        (rc = malloc_into(L, &mm->logjoint, chain_total)) || (rc = malloc_into(L, &mm->inverse_mass, param_total)) ||
        (rc = malloc_into(L, &mm->step, chain_total)) || (rc = malloc_into(L, &mm->accept_prob, chain_total)) ||
        (rc = malloc_into(L, &mm->energy, chain_total)) || (rc = malloc_into(L, &mm->energy_error, chain_total)) ||
        (rc = malloc_into(L, &mm->tree_depth, chain_total)) || (rc = malloc_into(L, &mm->integration_steps, chain_total)) ||
        (rc = malloc_into(L, &mm->divergent, chain_total)) || (rc = malloc_into(L, &mm->moved, chain_total)) ||
        (rc = malloc_into(L, &mm->class_slot, chain_total)) || (rc = malloc_into(L, &mm->da, 5 * (size_t)chain_total)) ||
        (rc = malloc_into(L, &mm->wmean, param_total)) || (rc = malloc_into(L, &mm->wm2, param_total)) ||
        (rc = malloc_into(L, &mm->wcount, num_models)) || (rc = malloc_into(L, &mm->counter, 1)) ||
        (rc = malloc_into(L, &mm->model_done, num_models)))
        return bail(rc);
    std::vector<int32_t> slot((size_t)chain_total);
    for (int k = 0; k < kNumClasses; ++k) {
        MmClass& cl = mm->classes[k];
        cl.K = kClassK[k];
        for (int i = 0; i < num_models; ++i)
            if (ms[i].klass == k) {
                for (int c = 0; c < ms[i].C; ++c) slot[ms[i].chain_off + c] = (int32_t)(cl.chains + c);
                cl.model_ids.push_back(i);
                cl.chains += ms[i].C;
            }
        if (cl.chains == 0) continue;
        if ((rc = malloc_into(L, &cl.items, (size_t)cl.chains)) ||
            (rc = malloc_into(L, &cl.ckpt, (size_t)cl.chains * (max_tree_depth + 1) * 2 * 32 * cl.K)))
            return bail(rc);
    }
    if (cudaMemcpy(mm->models, ms.data(), ms.size() * sizeof(MmModel), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(mm->packs, packs.data(), packs.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(mm->class_slot, slot.data(), slot.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(mm->counter, 0, sizeof(int32_t)) != cudaSuccess)
        return bail(mfail(UT_ERR_CUDA, "multi-model upload failed: %s", cudaGetErrorString(cudaGetLastError())));
    for (int k = 0; k < kNumClasses; ++k) {
        MmClass& cl = mm->classes[k];
        if (cl.chains && (rc = build_items(mm, cl, 4, kStageMax))) return bail(rc);
    }
    if (cudaStreamCreateWithFlags(&mm->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&mm->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&mm->user_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&mm->done_ev, cudaEventDisableTiming) != cudaSuccess)
        return bail(mfail(UT_ERR_CUDA, "stream / event creation failed"));
    for (int k = 0; k < kNumClasses; ++k)
        if (cudaStreamCreateWithFlags(&mm->side[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&mm->join[k], cudaEventDisableTiming) != cudaSuccess)
            return bail(mfail(UT_ERR_CUDA, "stream / event creation failed"));
    *out = mm;
    return UT_OK;
}

int32_t ut_multi_destroy(ut_multi* mm) {
    if (!mm) return UT_OK;
    cudaDeviceSynchronize();
    release_all(mm);
    delete mm;
    return UT_OK;
}

int32_t ut_multi_layout(const ut_multi* mm, int64_t* state_offsets, int64_t* chain_offsets, int64_t* param_offsets) {
    int32_t rc = check_mm(mm);
    if (rc) return rc;
    for (int i = 0; i <= mm->M; ++i) {
        const bool end = i == mm->M;
        if (state_offsets) state_offsets[i] = end ? mm->state_floats : mm->models_h[i].state_off;
        if (chain_offsets) chain_offsets[i] = end ? mm->total_chains : mm->models_h[i].chain_off;
        if (param_offsets) param_offsets[i] = end ? mm->param_floats : mm->models_h[i].param_off;
    }
    return UT_OK;
}

int32_t ut_multi_class_info(const ut_multi* mm, int32_t* slot_counts, int32_t* num_models, int64_t* num_chains,
                            int32_t* chains_per_block, int32_t* stage_limit_bytes) {
    int32_t rc = check_mm(mm);
    if (rc) return rc;
    for (int k = 0; k < kNumClasses; ++k) {
        const MmClass& cl = mm->classes[k];
        if (slot_counts) slot_counts[k] = cl.K;
        if (num_models) num_models[k] = (int32_t)cl.model_ids.size();
        if (num_chains) num_chains[k] = cl.chains;
        if (chains_per_block) chains_per_block[k] = cl.W;
        if (stage_limit_bytes) stage_limit_bytes[k] = cl.stage_limit;
    }
    return UT_OK;
}

int32_t ut_multi_configure(ut_multi* mm, int32_t klass, int32_t chains_per_block, int32_t stage_limit_bytes) {
    int32_t rc = check_mm(mm);
    if (rc) return rc;
    if (klass < 0 || klass >= kNumClasses) return mfail(UT_ERR_ARGUMENT, "class must be in 0..%d", kNumClasses - 1);
    if (chains_per_block < 1 || chains_per_block > kMaxWarps)
        return mfail(UT_ERR_ARGUMENT, "chains_per_block must be in 1..%d", kMaxWarps);
    if (stage_limit_bytes < 0 || stage_limit_bytes > kStageMax)
        return mfail(UT_ERR_ARGUMENT, "stage_limit_bytes must be in 0..%d", kStageMax);
    MmClass& cl = mm->classes[klass];
    if (cl.chains == 0) return UT_OK;
    MM_CUDA(cudaDeviceSynchronize());
    if ((rc = build_items(mm, cl, chains_per_block, stage_limit_bytes))) return rc;
    drop_graph(mm);
    return UT_OK;
}

int32_t ut_multi_set_positions(ut_multi* mm, const float* d_positions, void* stream) {
    int32_t rc = check_mm(mm);
    if (rc) return rc;
    if (!d_positions) return mfail(UT_ERR_ARGUMENT, "null positions");
    cudaStream_t st = (cudaStream_t)stream;
    MM_CUDA(cudaMemcpyAsync(mm->position, d_positions, mm->state_floats * sizeof(float), cudaMemcpyDeviceToDevice, st));
    for (int k = 0; k < kNumClasses; ++k) {
        const MmClass& cl = mm->classes[k];
        if (cl.num_items == 0) continue;
        MmArgs a = base_args(mm, cl);
        MM_K_SWITCH(cl.K, (mm_density_kernel<K><<<cl.num_items, 32 * cl.W, 0, st>>>(a)));
        MM_LAUNCHED();
    }
    return UT_OK;
}

int32_t ut_multi_begin(ut_multi* mm, int32_t num_warmup, int32_t num_samples, uint32_t seed, float target_accept,
                       float initial_step, float divergence_threshold, const uint8_t* warmup_actions,
                       int32_t draws_capacity) {
    int32_t rc = check_mm(mm);
    if (rc) return rc;
    if (num_warmup < 0 || num_samples < 0) return mfail(UT_ERR_ARGUMENT, "iteration counts must be >= 0");
    if (num_warmup > 0 && !warmup_actions) return mfail(UT_ERR_ARGUMENT, "null warmup schedule");
    if (!(target_accept > 0.0f && target_accept < 1.0f)) return mfail(UT_ERR_ARGUMENT, "target_accept must be in (0, 1)");
    if (!(initial_step > 0.0f) || !std::isfinite(initial_step)) return mfail(UT_ERR_ARGUMENT, "initial_step must be > 0");
    if (draws_capacity < 0 || draws_capacity > num_samples)
        return mfail(UT_ERR_ARGUMENT, "draws_capacity must be in 0..num_samples");
    MM_CUDA(cudaDeviceSynchronize());
    drop_graph(mm);
    for (void* p : mm->run_allocations) cudaFree(p);
    mm->run_allocations.clear();
    mm->draws = nullptr; mm->draw_accept = nullptr; mm->draw_depth = nullptr; mm->draw_div = nullptr;
    mm->draws_capacity = 0;
    auto& R = mm->run_allocations;
    if ((rc = malloc_into(R, &mm->actions, std::max(num_warmup, 1)))) return rc;
    if (draws_capacity > 0) {
        if ((rc = malloc_into(R, &mm->draws, (size_t)draws_capacity * mm->state_floats)) ||
            (rc = malloc_into(R, &mm->draw_accept, (size_t)draws_capacity * mm->total_chains)) ||
            (rc = malloc_into(R, &mm->draw_depth, (size_t)draws_capacity * mm->total_chains)) ||
            (rc = malloc_into(R, &mm->draw_div, (size_t)draws_capacity * mm->total_chains)))
            return rc;
    }
    mm->draws_capacity = draws_capacity;
    if (num_warmup > 0)
        MM_CUDA(cudaMemcpy(mm->actions, warmup_actions, num_warmup, cudaMemcpyHostToDevice));
    mm->num_warmup = num_warmup;
    mm->num_samples = num_samples;
    mm->seed = seed;
    mm->target_accept = target_accept;
    mm->thr = divergence_threshold;
    std::vector<double> da(5 * (size_t)mm->total_chains);
    for (int64_t i = 0; i < mm->total_chains; ++i) {
        const double ls = std::log((double)initial_step);
        da[5 * i + 0] = std::log(10.0 * initial_step);
        da[5 * i + 1] = ls; da[5 * i + 2] = ls; da[5 * i + 3] = 0.0; da[5 * i + 4] = 0.0;
    }
    std::vector<float> ones((size_t)mm->param_floats, 1.0f), steps((size_t)mm->total_chains, initial_step);
    MM_CUDA(cudaMemcpy(mm->da, da.data(), da.size() * sizeof(double), cudaMemcpyHostToDevice));
    MM_CUDA(cudaMemcpy(mm->inverse_mass, ones.data(), ones.size() * sizeof(float), cudaMemcpyHostToDevice));
    MM_CUDA(cudaMemcpy(mm->step, steps.data(), steps.size() * sizeof(float), cudaMemcpyHostToDevice));
    MM_CUDA(cudaMemset(mm->wmean, 0, mm->param_floats * sizeof(double)));
    MM_CUDA(cudaMemset(mm->wm2, 0, mm->param_floats * sizeof(double)));
    MM_CUDA(cudaMemset(mm->wcount, 0, mm->M * sizeof(double)));
    MM_CUDA(cudaMemset(mm->counter, 0, sizeof(int32_t)));
    MM_CUDA(cudaMemset(mm->accept_prob, 0, mm->total_chains * sizeof(float)));
    MM_CUDA(cudaMemset(mm->model_done, 0, mm->M));
    mm->begun = true;
    return UT_OK;
}

int32_t ut_multi_set_stopped(ut_multi* mm, const uint8_t* stopped, void* stream) {
    int32_t rc = check_mm(mm);
    if (rc) return rc;
    if (!stopped) return mfail(UT_ERR_ARGUMENT, "null stop flags");
    if (!mm->begun) return mfail(UT_ERR_ARGUMENT, "call ut_multi_begin before ut_multi_set_stopped");
    MM_CUDA(cudaMemcpyAsync(mm->model_done, stopped, mm->M, cudaMemcpyHostToDevice, (cudaStream_t)stream));
    MM_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return UT_OK;
}

int32_t ut_multi_run(ut_multi* mm, int32_t num_iterations, int32_t use_graph, void* stream) {
    int32_t rc = check_mm(mm);
    if (rc) return rc;
    if (!mm->begun) return mfail(UT_ERR_ARGUMENT, "call ut_multi_begin before ut_multi_run");
    if (num_iterations < 0) return mfail(UT_ERR_ARGUMENT, "num_iterations must be >= 0");
    cudaStream_t user = (cudaStream_t)stream;
    MM_CUDA(cudaEventRecord(mm->user_ev, user));
    MM_CUDA(cudaStreamWaitEvent(mm->stream, mm->user_ev, 0));
    int left = num_iterations;
    if (use_graph) {
        if (left >= kGraphIters && !mm->graph && (rc = capture_graph(mm))) return rc;
        while (left >= kGraphIters) {
            MM_CUDA(cudaGraphLaunch(mm->graph, mm->stream));
            left -= kGraphIters;
        }
    }
    for (; left > 0; --left)
        if ((rc = enqueue_iteration(mm, mm->stream))) return rc;
    MM_CUDA(cudaEventRecord(mm->done_ev, mm->stream));
    MM_CUDA(cudaStreamWaitEvent(user, mm->done_ev, 0));
    return UT_OK;
}

int32_t ut_multi_autotune(ut_multi* mm, int32_t trials, float* timings_ms, void* stream) {
    int32_t rc = check_mm(mm);
    if (rc) return rc;
    if (!mm->begun) return mfail(UT_ERR_ARGUMENT, "call ut_multi_begin before ut_multi_autotune");
    if (trials < 1) return mfail(UT_ERR_ARGUMENT, "trials must be >= 1");
    (void)stream;
    MM_CUDA(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    MM_CUDA(cudaEventCreate(&e0));
    MM_CUDA(cudaEventCreate(&e1));
    const size_t sf = mm->state_floats * sizeof(float), cf = mm->total_chains * sizeof(float);
    float* sv_pos = mm->save;
    float* sv_grad = mm->save + mm->state_floats;
    float* sv_lj = mm->save + 2 * mm->state_floats;
    float* sv_step = sv_lj + mm->total_chains;
    const size_t df = 5 * mm->total_chains * sizeof(double);
    cudaStream_t st = mm->stream;
    // the trials may also run the step search, which writes steps and dual-averaging state
    auto save = [&]() -> int32_t {
        MM_CUDA(cudaMemcpyAsync(sv_pos, mm->position, sf, cudaMemcpyDeviceToDevice, st));
        MM_CUDA(cudaMemcpyAsync(sv_grad, mm->gradient, sf, cudaMemcpyDeviceToDevice, st));
        MM_CUDA(cudaMemcpyAsync(sv_lj, mm->logjoint, cf, cudaMemcpyDeviceToDevice, st));
        MM_CUDA(cudaMemcpyAsync(sv_step, mm->step, cf, cudaMemcpyDeviceToDevice, st));
        MM_CUDA(cudaMemcpyAsync(mm->save_da, mm->da, df, cudaMemcpyDeviceToDevice, st));
        return UT_OK;
    };
    auto restore = [&]() -> int32_t {
        MM_CUDA(cudaMemcpyAsync(mm->position, sv_pos, sf, cudaMemcpyDeviceToDevice, st));
        MM_CUDA(cudaMemcpyAsync(mm->gradient, sv_grad, sf, cudaMemcpyDeviceToDevice, st));
        MM_CUDA(cudaMemcpyAsync(mm->logjoint, sv_lj, cf, cudaMemcpyDeviceToDevice, st));
        MM_CUDA(cudaMemcpyAsync(mm->step, sv_step, cf, cudaMemcpyDeviceToDevice, st));
        MM_CUDA(cudaMemcpyAsync(mm->da, mm->save_da, df, cudaMemcpyDeviceToDevice, st));
        return UT_OK;
    };
    auto finish = [&](int32_t code) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return code;
    };
    if ((rc = save())) return finish(rc);
    for (int k = 0; k < kNumClasses; ++k) {
        MmClass& cl = mm->classes[k];
        float* row = timings_ms ? timings_ms + (size_t)k * 6 : nullptr;
        if (row) std::fill(row, row + 6, -1.0f);
        if (cl.chains == 0) continue;
        float best = INFINITY;
        int bw = cl.W, bs = cl.stage_limit;
        for (int wi = 0; wi < 3; ++wi)
            for (int si = 0; si < 2; ++si) {
                if ((rc = build_items(mm, cl, kCandW[wi], kCandStage[si]))) return finish(rc);
                float total = 0.0f;
                for (int t = 0; t < trials; ++t) {
                    if ((rc = restore())) return finish(rc);
                    MM_CUDA(cudaEventRecord(e0, st));
                    if ((rc = launch_class_nuts(mm, cl, st))) return finish(rc);
                    MM_CUDA(cudaEventRecord(e1, st));
                    MM_CUDA(cudaEventSynchronize(e1));
                    float ms = 0.0f;
                    MM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                    total += ms;
                }
                const float avg = total / trials;
                if (row) row[wi * 2 + si] = avg;
                if (avg < best) { best = avg; bw = kCandW[wi]; bs = kCandStage[si]; }
            }
        if ((rc = build_items(mm, cl, bw, bs))) return finish(rc);
    }
    if ((rc = restore())) return finish(rc);
    MM_CUDA(cudaStreamSynchronize(st));
    drop_graph(mm);
    return finish(UT_OK);
}

int32_t ut_multi_split_rhat(ut_multi* mm, int32_t num_draws, float* d_out, void* stream) {
    int32_t rc = check_mm(mm);
    if (rc) return rc;
    if (!d_out) return mfail(UT_ERR_ARGUMENT, "null output");
    if (num_draws < 4 || num_draws > mm->draws_capacity)
        return mfail(UT_ERR_ARGUMENT, "num_draws must be in 4..%d (the recorded draws)", mm->draws_capacity);
    mm_split_rhat_kernel<<<mm->M, 256, 0, (cudaStream_t)stream>>>(mm->models, mm->draws, mm->state_floats,
                                                                   num_draws, d_out);
    MM_LAUNCHED();
    return UT_OK;
}

int32_t ut_multi_buffers(const ut_multi* mm, ut_multi_view* v) {
    int32_t rc = check_mm(mm);
    if (rc) return rc;
    if (!v) return mfail(UT_ERR_ARGUMENT, "null output");
    v->position = mm->position; v->gradient = mm->gradient; v->logjoint = mm->logjoint;
    v->step = mm->step; v->inverse_mass = mm->inverse_mass; v->accept_prob = mm->accept_prob;
    v->tree_depth = mm->tree_depth; v->integration_steps = mm->integration_steps; v->divergent = mm->divergent;
    v->draws = mm->draws; v->draw_accept = mm->draw_accept; v->draw_tree_depth = mm->draw_depth;
    v->draw_divergent = mm->draw_div; v->iteration = mm->counter;
    v->state_floats = mm->state_floats; v->total_chains = mm->total_chains; v->param_floats = mm->param_floats;
    v->draws_capacity = mm->draws_capacity;
    return UT_OK;
}

}  // extern "C"
