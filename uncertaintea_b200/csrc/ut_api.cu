// ut_api.cu -- C ABI of the library (declared in include/ut_b200.h): workspace
// lifetime, kernel-description validation, and the launch sites of every
// kernel.  No CPU fallback: without a CUDA device every compute entry point
// returns UT_ERR_NO_DEVICE.
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <cmath>

#include "../../include/ut_b200.h"
#include "ut_warp_kernels.cuh"
#include "ut_glm_tiled.cuh"
#include "ut_lf_batched.cuh"
#include "ut_tc_glm.cuh"
#include "ut_glm_stream.cuh"
#include "ut_nuts_lockstep.cuh"
#include "ut_advi.cuh"
#include "ut_meads.cuh"

using namespace ut;

namespace {

thread_local std::string g_last_error;

int32_t fail(int32_t code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define UT_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail(UT_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

#define UT_LAUNCHED()                                                                          \
    do {                                                                                       \
        cudaError_t e_ = cudaGetLastError();                                                   \
        if (e_ != cudaSuccess) return fail(UT_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e_)); \
    } while (0)

enum Path { kPathWarp = 1, kPathTiled = 2 };

constexpr size_t kSmemBudget = 200 * 1024;  // dynamic shared memory per CTA we allow ourselves
constexpr int kWarpsDensity = 8;            // chains per CTA of the warp kernels
constexpr int kWarpsNuts = 4;

int inst_k(int P) {
    int k = (P + 31) / 32;
    const int ks[] = {1, 2, 3, 4, 8, 17};
    for (int v : ks)
        if (k <= v) return v;
    return -1;
}

}  // namespace

// Lets the library's other translation unit report through ut_last_error.
void ut_internal_set_last_error(const char* msg) { g_last_error = msg; }

struct ut_workspace {
    ut_plan_desc plan;
    int P = 0, C = 0, N = 0, device = 0;
    int path = 0;
    int K = 0, dmax = 16;
    DevModel dm;
    // device data
    float* d_XT = nullptr;   // GLM warp path: D x N
    float* d_Xa = nullptr;   // GLM tiled path: N x F (ones column first when intercept)
    float* d_y = nullptr;
    float* d_sig = nullptr;
    int32_t* d_start = nullptr;
    int32_t* d_count = nullptr;
    // tiled scratch
    int splits = 0, obs_per_split = 0, fpt = 1;
    float* d_part_ll = nullptr;
    float* d_part_g = nullptr;
    // tensor-core path (GLM, large N)
    TcGlmPlan tc;
    // streaming path (GLM, few chains)
    bool streaming = false;
    int stream_cb = 16, stream_splits = 0, stream_stages = 2, stream_slots = 1;
    size_t stream_smem = 0;
    float* d_ypad = nullptr;        // y rounded up to whole 32-row chunks, zero padded
    float* d_spart = nullptr;       // per-CTA partials
    float* d_sgpart = nullptr;      // per-group partials
    unsigned* d_stickets = nullptr; // fold tickets (zero between launches)
    int* d_serr = nullptr;          // sticky error word of the streaming kernel
    unsigned* d_sbar = nullptr;     // grid barrier of the one-launch trajectory: [arrivals, generation]
    // batched leapfrog scratch
    LfScratch lf = {};
    // NUTS checkpoint scratch
    float* d_ckpt = nullptr;
    int ckpt_depth = -1;
    // lockstep NUTS state machine
    float* ls_vec = nullptr;
    float* ls_f = nullptr;
    int32_t* ls_i = nullptr;
    float* ls_ckpt = nullptr;
    int32_t* ls_active = nullptr;  // live-chain count (device)
    int32_t* h_active = nullptr;   // pinned host copy of the live-chain count
    int32_t* h_err = nullptr;      // pinned host copies of the tensor-core / streaming error flags
    uint8_t* ls_act = nullptr;     // per-chain live flags
    int32_t* ls_idx = nullptr;     // compacted live chains
    float* ls_cq = nullptr;        // compacted positions / gradients / logjoints
    float* ls_cg = nullptr;
    float* ls_clj = nullptr;
    int ls_depth = -1;
    // MEADS fold scratch
    MeadsScratch meads = {};
    int meads_k = 0;
    // ChEES scratch
    uint8_t* d_flags = nullptr;
    double* d_means = nullptr;
    double* d_terms = nullptr;
    double* d_out = nullptr;
    // host-pointer entry buffers
    float* d_params = nullptr;
    float* d_totals = nullptr;
    float* d_grads = nullptr;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocations;
};

namespace {

template <class T>
int32_t dalloc(ut_workspace* ws, T** p, size_t count) {
    void* v = nullptr;
    cudaError_t e = cudaMalloc(&v, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return fail(UT_ERR_CUDA, "cudaMalloc(%zu bytes) failed: %s", count * sizeof(T), cudaGetErrorString(e));
    ws->allocations.push_back(v);
    *p = static_cast<T*>(v);
    return UT_OK;
}

std::string plan_issues(const ut_plan_desc* p) {
    std::string s;
    auto add = [&](const std::string& m) { s += (s.empty() ? "" : "\n") + m; };
    if (!p) { add("null kernel description"); return s; }
    // the kernels' observation index arithmetic is 32-bit: an observation
    // count of at most 2^30 keeps every split end and tile bound in range
    if (p->num_obs > UT_MAX_OBS) add("num_obs must be <= 2^30 (1073741824)");
    if (p->family == UT_FAMILY_GLM_BERNOULLI_LOGIT) {
        if (p->num_coefs < 1) add("GLM needs at least one covariate (num_coefs >= 1)");
        if (p->has_intercept != 0 && p->has_intercept != 1) add("has_intercept must be 0 or 1");
        if (p->num_params != p->num_coefs + (p->has_intercept ? 1 : 0))
            add("num_params must equal num_coefs + has_intercept");
        if (p->num_params > kGlmMaxF) add("GLM with more than 256 unconstrained parameters is not supported");
        if (!(p->coef_sigma > 0.0)) add("coefficient prior scale must be > 0");
        if (p->has_intercept && !(p->intercept_sigma > 0.0)) add("intercept prior scale must be > 0");
        if (p->num_obs < 0) add("num_obs must be >= 0");
    } else if (p->family == UT_FAMILY_HIER_NORMAL_NONCENTERED) {
        if (p->num_groups < 1) add("hierarchical model needs at least one group (num_groups >= 1)");
        if (p->num_params != p->num_groups + 2) add("num_params must equal num_groups + 2 (mu, log tau, z_1..z_J)");
        if (inst_k(p->num_params) < 0) add("hierarchical model with more than 544 parameters is not supported");
        if (!(p->mu_scale > 0.0)) add("mu prior scale must be > 0");
        if (!(p->tau_scale > 0.0)) add("tau prior scale must be > 0");
        if (p->num_obs < 0) add("num_obs must be >= 0");
    } else if (p->family == UT_FAMILY_NORMAL_LOCATION_SCALE) {
        if (p->num_params != 2) add("num_params must equal 2 (mu, log s)");
        if (!(p->mu_scale > 0.0)) add("mu prior scale must be > 0");
        if (!(p->scale_shape > 0.0) || !(p->scale_rate > 0.0)) add("gamma shape and rate must be > 0");
        if (p->num_obs < 0) add("num_obs must be >= 0");
    } else if (p->family == UT_FAMILY_NORMAL_KNOWN_SCALE) {
        if (p->num_params != 1) add("num_params must equal 1 (mu)");
        if (!(p->mu_scale > 0.0)) add("mu prior scale must be > 0");
        if (!(p->obs_scale > 0.0) || !std::isfinite(p->obs_scale)) add("observation scale must be finite and > 0");
        if (p->num_obs < 0) add("num_obs must be >= 0");
    } else if (p->family == UT_FAMILY_STUDENTT_HEAVY_TAIL) {
        if (p->num_params != 3) add("num_params must equal 3 (loc, log s, log w)");
        if (!(p->nu_prior > 0.0) || !(p->nu_obs > 0.0)) add("Student-t degrees of freedom must be > 0");
        if (!(p->mu_scale > 0.0)) add("Student-t prior scale must be > 0");
        if (!(p->scale_shape > 0.0) || !(p->scale_rate > 0.0)) add("inverse-gamma shape and scale must be > 0");
        if (!(p->weibull_shape > 0.0) || !(p->weibull_scale > 0.0)) add("Weibull shape and scale must be > 0");
        if (p->num_obs < 0) add("num_obs must be >= 0");
    } else if (p->family == UT_FAMILY_LOGNORMAL_GAMMA_NORMAL) {
        if (p->num_params != 2) add("num_params must equal 2 (log a, log b)");
        if (!(p->mu_scale > 0.0)) add("lognormal scale must be > 0");
        if (!(p->scale_shape > 0.0) || !(p->scale_rate > 0.0)) add("gamma shape and rate must be > 0");
        if (p->num_obs < 0) add("num_obs must be >= 0");
    } else if (p->family == UT_FAMILY_BERNOULLI_BETA) {
        if (p->num_params != 1) add("num_params must equal 1 (logit p)");
        if (!(p->prob_alpha > 0.0) || !(p->prob_beta > 0.0)) add("beta prior parameters must be > 0");
        if (p->num_obs < 0) add("num_obs must be >= 0");
    } else {
        char b[96];
        snprintf(b, sizeof(b), "unsupported kernel-description family %d", p->family);
        add(b);
    }
    return s;
}

size_t warp_smem_bytes(const ut_workspace* ws, int warps) {
    return (size_t)ws->dm.staged_floats * sizeof(float) + (size_t)warps * ws->dm.Ppad * sizeof(float);
}

int32_t need_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        return fail(UT_ERR_NO_DEVICE, "no CUDA device is visible; the B200 backend has no CPU fallback");
    return UT_OK;
}

// ---- kernel dispatch over the compile-time slot count K and GLM width DMAX ----
#define UT_DISPATCH_WARP(ws, KERNEL, ...)                                                                    \
    do {                                                                                                     \
        if ((ws)->dm.family == kFamGlm) {                                                                    \
            if ((ws)->K == 1 && (ws)->dmax == 16) { KERNEL(kFamGlm, 1, 16, __VA_ARGS__); }                   \
            else if ((ws)->K == 1) { KERNEL(kFamGlm, 1, 32, __VA_ARGS__); }                                  \
            else { KERNEL(kFamGlm, 2, 32, __VA_ARGS__); }                                                   \
        } else if ((ws)->dm.family == kFamGauss) {                                                           \
            KERNEL(kFamGauss, 1, 1, __VA_ARGS__);                                                            \
        } else if ((ws)->dm.family == kFamBern) {                                                            \
            KERNEL(kFamBern, 1, 1, __VA_ARGS__);                                                             \
        } else if ((ws)->dm.family == kFamLgn) {                                                             \
            KERNEL(kFamLgn, 1, 1, __VA_ARGS__);                                                              \
        } else if ((ws)->dm.family == kFamHt) {                                                              \
            KERNEL(kFamHt, 1, 1, __VA_ARGS__);                                                               \
        } else if ((ws)->dm.family == kFamProg) {                                                            \
            switch ((ws)->K) {                                                                               \
                case 1: KERNEL(kFamProg, 1, 1, __VA_ARGS__); break;                                          \
                case 2: KERNEL(kFamProg, 2, 1, __VA_ARGS__); break;                                          \
                case 3: KERNEL(kFamProg, 3, 1, __VA_ARGS__); break;                                          \
                case 4: KERNEL(kFamProg, 4, 1, __VA_ARGS__); break;                                          \
                default: KERNEL(kFamProg, 8, 1, __VA_ARGS__); break;                                         \
            }                                                                                                \
        } else {                                                                                             \
            switch ((ws)->K) {                                                                               \
                case 1: KERNEL(kFamHier, 1, 1, __VA_ARGS__); break;                                          \
                case 2: KERNEL(kFamHier, 2, 1, __VA_ARGS__); break;                                          \
                case 3: KERNEL(kFamHier, 3, 1, __VA_ARGS__); break;                                          \
                case 4: KERNEL(kFamHier, 4, 1, __VA_ARGS__); break;                                          \
                case 8: KERNEL(kFamHier, 8, 1, __VA_ARGS__); break;                                          \
                default: KERNEL(kFamHier, 17, 1, __VA_ARGS__); break;                                        \
            }                                                                                                \
        }                                                                                                    \
    } while (0)

// Lets `kern` take `smem` bytes of dynamic shared memory (needed above 48 KB).
template <class Kern>
cudaError_t allow_dynamic_smem(Kern kern, size_t smem) {
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

#define LAUNCH_DENSITY(FAM, K, DM, ws, params, totals, grads, st)                                           \
    {                                                                                                      \
        auto kern = density_warp_kernel<FAM, K, DM>;                                                        \
        size_t smem = warp_smem_bytes(ws, kWarpsDensity);                                                   \
        UT_CUDA(allow_dynamic_smem(kern, smem));                                                          \
        kern<<<((ws)->C + kWarpsDensity - 1) / kWarpsDensity, 32 * kWarpsDensity, smem, st>>>((ws)->dm, params, totals, grads, (ws)->C); \
    }

#define LAUNCH_HMC(FAM, K, DM, ws, args, st)                                                                \
    {                                                                                                      \
        auto kern = hmc_warp_kernel<FAM, K, DM>;                                                            \
        size_t smem = warp_smem_bytes(ws, kWarpsDensity);                                                   \
        UT_CUDA(allow_dynamic_smem(kern, smem));                                                          \
        kern<<<((ws)->C + kWarpsDensity - 1) / kWarpsDensity, 32 * kWarpsDensity, smem, st>>>((ws)->dm, args); \
    }

#define LAUNCH_PROBE(FAM, K, DM, ws, args, st)                                                              \
    {                                                                                                      \
        auto kern = probe_warp_kernel<FAM, K, DM>;                                                          \
        size_t smem = warp_smem_bytes(ws, kWarpsDensity);                                                   \
        UT_CUDA(allow_dynamic_smem(kern, smem));                                                          \
        kern<<<((ws)->C + kWarpsDensity - 1) / kWarpsDensity, 32 * kWarpsDensity, smem, st>>>((ws)->dm, args); \
    }

#define LAUNCH_NUTS(FAM, K, DM, ws, args, st)                                                               \
    {                                                                                                      \
        auto kern = nuts_warp_kernel<FAM, K, DM>;                                                           \
        size_t smem = warp_smem_bytes(ws, kWarpsNuts);                                                      \
        UT_CUDA(allow_dynamic_smem(kern, smem));                                                          \
        kern<<<((ws)->C + kWarpsNuts - 1) / kWarpsNuts, 32 * kWarpsNuts, smem, st>>>((ws)->dm, args);     \
    }

#define UT_K_SWITCH(KV, ...)                                        \
    switch (KV) {                                                   \
        case 1: { constexpr int K = 1; __VA_ARGS__; } break;        \
        case 2: { constexpr int K = 2; __VA_ARGS__; } break;        \
        case 3: { constexpr int K = 3; __VA_ARGS__; } break;        \
        case 4: { constexpr int K = 4; __VA_ARGS__; } break;        \
        default: { constexpr int K = 8; __VA_ARGS__; } break;       \
    }

size_t tiled_smem_bytes(int F) {
    return sizeof(float) * ((size_t)F * kGlmCT + (size_t)F * kGlmXS + (size_t)kGlmOT * kGlmRS + kGlmOT + 16 * kGlmCT);
}

template <bool GRAD>
int32_t launch_tiled_t(ut_workspace* ws, const float* params, float* totals, float* grads, cudaStream_t st) {
    GlmTiledArgs a;
    a.Xa = ws->d_Xa; a.y = ws->d_y; a.params = params;
    a.part_ll = ws->d_part_ll; a.part_g = ws->d_part_g;
    a.N = ws->N; a.F = ws->P; a.C = ws->C; a.obs_per_split = ws->obs_per_split;
    dim3 grid((ws->C + kGlmCT - 1) / kGlmCT, ws->splits);
    size_t smem = tiled_smem_bytes(ws->P);
#define TILED_CASE(FPTV)                                                                  \
    case FPTV: {                                                                          \
        auto kern = glm_tiled_kernel<GRAD, FPTV>;                                         \
        UT_CUDA(allow_dynamic_smem(kern, smem));                                        \
        kern<<<grid, 256, smem, st>>>(a);                                                 \
    } break;
    switch (ws->fpt) {
        TILED_CASE(1) TILED_CASE(2) TILED_CASE(4) TILED_CASE(7) TILED_CASE(8) TILED_CASE(12)
        default: TILED_CASE(16)
    }
#undef TILED_CASE
    UT_LAUNCHED();
    GlmReduceArgs r;
    r.params = params; r.part_ll = ws->d_part_ll; r.part_g = GRAD ? ws->d_part_g : nullptr;
    r.totals = totals; r.grads = GRAD ? grads : nullptr;
    r.S = ws->splits; r.C = ws->C; r.F = ws->P; r.off = ws->plan.has_intercept;
    r.icpt_mu = (float)ws->plan.intercept_mu; r.icpt_sigma = (float)ws->plan.intercept_sigma;
    r.coef_mu = (float)ws->plan.coef_mu; r.coef_sigma = (float)ws->plan.coef_sigma;
    glm_reduce_kernel<<<(ws->C + 7) / 8, 256, 0, st>>>(r);
    UT_LAUNCHED();
    return UT_OK;
}

int32_t launch_stream(ut_workspace* ws, const float* params, float* totals, float* grads, cudaStream_t st) {
    GlmStreamArgs a;
    a.Xa = ws->d_Xa; a.ypad = ws->d_ypad; a.params = params;
    a.part = ws->d_spart; a.gpart = ws->d_sgpart; a.tickets = ws->d_stickets; a.err = ws->d_serr;
    a.totals = totals; a.grads = grads;
    a.N = ws->N; a.F = ws->P; a.C = ws->C; a.stages = ws->stream_stages; a.slots = ws->stream_slots; a.off = ws->plan.has_intercept;
    a.icpt_mu = (float)ws->plan.intercept_mu; a.icpt_sigma = (float)ws->plan.intercept_sigma;
    a.coef_mu = (float)ws->plan.coef_mu; a.coef_sigma = (float)ws->plan.coef_sigma;
    const size_t smem = ws->stream_smem;
#define STREAM_CASE(CBV)                                                                            \
    case CBV: {                                                                                     \
        auto kern = grads ? glm_stream_kernel<CBV, true> : glm_stream_kernel<CBV, false>;          \
        UT_CUDA(allow_dynamic_smem(kern, smem));                                                  \
        kern<<<ws->stream_splits, kStreamThreads, smem, st>>>(a);                                   \
    } break;
    switch (ws->stream_cb) {
        STREAM_CASE(1) STREAM_CASE(2) STREAM_CASE(4) STREAM_CASE(8)
        default: STREAM_CASE(16)
    }
#undef STREAM_CASE
    UT_LAUNCHED();
    return UT_OK;
}

// Steps 1..L of a leapfrog trajectory on the streaming path in one cooperative
// launch (glm_stream_traj_kernel): the L evaluations at ws->lf.wq and the
// kicks and drifts between them; lf_begin_kernel runs before it and
// lf_step_kernel (l = L) after it.  UT_ERR_UNSUPPORTED when the launch cannot
// be made cooperative here (the caller then runs the steps one launch each).
int32_t launch_stream_traj(ut_workspace* ws, const HmcArgs& h, int L, cudaStream_t st) {
    int32_t rc;
    if (!ws->d_sbar) {
        if ((rc = dalloc(ws, &ws->d_sbar, 2))) return rc;
        UT_CUDA(cudaMemset(ws->d_sbar, 0, 2 * sizeof(unsigned)));
    }
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ws->device);
    if (!coop) return UT_ERR_UNSUPPORTED;
    GlmTrajArgs t;
    GlmStreamArgs& a = t.s;
    a.Xa = ws->d_Xa; a.ypad = ws->d_ypad; a.params = ws->lf.wq;
    a.part = ws->d_spart; a.gpart = ws->d_sgpart; a.tickets = ws->d_stickets; a.err = ws->d_serr;
    a.totals = ws->lf.wlj; a.grads = ws->lf.wg;
    a.N = ws->N; a.F = ws->P; a.C = ws->C; a.stages = ws->stream_stages; a.slots = ws->stream_slots;
    a.off = ws->plan.has_intercept;
    a.icpt_mu = (float)ws->plan.intercept_mu; a.icpt_sigma = (float)ws->plan.intercept_sigma;
    a.coef_mu = (float)ws->plan.coef_mu; a.coef_sigma = (float)ws->plan.coef_sigma;
    t.wq = ws->lf.wq; t.wp = ws->lf.wp; t.wg = ws->lf.wg; t.wlj = ws->lf.wlj; t.valid = ws->lf.valid;
    t.inverse_mass = h.inverse_mass; t.step = h.step; t.bar = ws->d_sbar; t.L = L;
    const size_t smem = ws->stream_smem;
    void* args[] = {&t};
#define TRAJ_CASE(CBV)                                                                                      case CBV: {                                                                                                 auto kern = glm_stream_traj_kernel<CBV>;                                                               UT_CUDA(allow_dynamic_smem(kern, smem));                                                              int per_sm = 0;                                                                                         UT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStreamThreads, smem));           int sms = 0;                                                                                            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws->device);                               if (per_sm < 1 || ws->stream_splits > per_sm * sms) return UT_ERR_UNSUPPORTED;                          UT_CUDA(cudaLaunchCooperativeKernel((const void*)kern, dim3(ws->stream_splits), dim3(kStreamThreads),                                             args, smem, st));                                              } break;
    switch (ws->stream_cb) {
        TRAJ_CASE(1) TRAJ_CASE(2) TRAJ_CASE(4) TRAJ_CASE(8)
        default: TRAJ_CASE(16)
    }
#undef TRAJ_CASE
    UT_LAUNCHED();
    return UT_OK;
}

// The streaming kernel over the first n (<= 16) rows of `params` of a GLM
// workspace that normally uses another path (the lockstep tail): buffers for 16
// chains are made on first use, the stage plan follows the chain bucket.
int32_t launch_stream_rows(ut_workspace* ws, const float* params, float* totals, float* grads, int n,
                           cudaStream_t st) {
    const int F = ws->P;
    int32_t rc;
    if (!ws->d_serr) {  // keyed on the last buffer made, so a failed attempt is redone
        int dev_sms = 148;
        cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ws->device);
        ws->stream_splits = dev_sms;
        const int chunks = (ws->N + kStreamRows - 1) / kStreamRows;
        const size_t ypad = (size_t)chunks * kStreamRows;
        const int groups = glm_stream_groups(dev_sms);
        if ((rc = dalloc(ws, &ws->d_ypad, ypad))) return rc;
        UT_CUDA(cudaMemset(ws->d_ypad, 0, ypad * sizeof(float)));
        UT_CUDA(cudaMemcpy(ws->d_ypad, ws->d_y, (size_t)ws->N * sizeof(float), cudaMemcpyDeviceToDevice));
        if ((rc = dalloc(ws, &ws->d_spart, (size_t)dev_sms * kStreamMaxC * (F + 1)))) return rc;
        if ((rc = dalloc(ws, &ws->d_sgpart, (size_t)groups * kStreamMaxC * (F + 1)))) return rc;
        if ((rc = dalloc(ws, &ws->d_stickets, (size_t)groups + 1))) return rc;
        if ((rc = dalloc(ws, &ws->d_serr, 1))) return rc;
        UT_CUDA(cudaMemset(ws->d_stickets, 0, ((size_t)groups + 1) * sizeof(unsigned)));
        UT_CUDA(cudaMemset(ws->d_serr, 0, sizeof(int)));
    }
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ws->device);
    const int CB = n <= 1 ? 1 : n <= 2 ? 2 : n <= 4 ? 4 : n <= 8 ? 8 : 16;
    int stages = 0, slots = 0;
    if (!glm_stream_plan(CB, F, (size_t)std::max(0, optin - 1024), &stages, &slots))
        return fail(UT_ERR_UNSUPPORTED, "streaming kernel: shared memory too small");
    GlmStreamArgs a;
    a.Xa = ws->d_Xa; a.ypad = ws->d_ypad; a.params = params;
    a.part = ws->d_spart; a.gpart = ws->d_sgpart; a.tickets = ws->d_stickets; a.err = ws->d_serr;
    a.totals = totals; a.grads = grads;
    a.N = ws->N; a.F = F; a.C = n; a.stages = stages; a.slots = slots; a.off = ws->plan.has_intercept;
    a.icpt_mu = (float)ws->plan.intercept_mu; a.icpt_sigma = (float)ws->plan.intercept_sigma;
    a.coef_mu = (float)ws->plan.coef_mu; a.coef_sigma = (float)ws->plan.coef_sigma;
    const size_t smem = glm_stream_smem(CB, F, stages);
#define STREAM_CASE(CBV)                                                                            \
    case CBV: {                                                                                     \
        auto kern = grads ? glm_stream_kernel<CBV, true> : glm_stream_kernel<CBV, false>;          \
        UT_CUDA(allow_dynamic_smem(kern, smem));                                                  \
        kern<<<ws->stream_splits, kStreamThreads, smem, st>>>(a);                                   \
    } break;
    switch (CB) {
        STREAM_CASE(1) STREAM_CASE(2) STREAM_CASE(4) STREAM_CASE(8)
        default: STREAM_CASE(16)
    }
#undef STREAM_CASE
    UT_LAUNCHED();
    return UT_OK;
}

// Batched density on device buffers, whichever path the workspace uses.
int32_t density(ut_workspace* ws, const float* params, float* totals, float* grads, cudaStream_t st) {
    if (ws->streaming) return launch_stream(ws, params, totals, grads, st);
    if (ws->path == kPathWarp) {
        UT_DISPATCH_WARP(ws, LAUNCH_DENSITY, ws, params, totals, grads, st);
        UT_LAUNCHED();
        return UT_OK;
    }
    if (ws->tc.enabled) return tc_glm_launch(ws->tc, params, totals, grads, st) == cudaSuccess
                                            ? UT_OK
                                            : fail(UT_ERR_CUDA, "tensor-core GLM launch failed: %s",
                                                   cudaGetErrorString(cudaGetLastError()));
    return grads ? launch_tiled_t<true>(ws, params, totals, grads, st) : launch_tiled_t<false>(ws, params, totals, nullptr, st);
}

// Lazily made buffer sets are keyed on the last buffer each makes: after a
// failed attempt (out of device memory) the next call makes the whole set again
// instead of finding it half made.  Buffers of a failed attempt stay in the
// workspace's allocation list and are freed with it.
int32_t ensure_lf(ut_workspace* ws) {
    if (ws->lf.valid) return UT_OK;
    size_t pc = (size_t)ws->P * ws->C;
    int32_t rc;
    if ((rc = dalloc(ws, &ws->lf.wq, pc))) return rc;
    if ((rc = dalloc(ws, &ws->lf.wp, pc))) return rc;
    if ((rc = dalloc(ws, &ws->lf.wg, pc))) return rc;
    if ((rc = dalloc(ws, &ws->lf.wlj, ws->C))) return rc;
    if ((rc = dalloc(ws, &ws->lf.H0, ws->C))) return rc;
    if ((rc = dalloc(ws, &ws->lf.valid, ws->C))) return rc;
    return UT_OK;
}

int32_t ensure_host_buffers(ut_workspace* ws) {
    if (ws->h_err) return UT_OK;
    size_t pc = (size_t)ws->P * ws->C;
    int32_t rc;
    if ((rc = dalloc(ws, &ws->d_params, pc))) return rc;
    if ((rc = dalloc(ws, &ws->d_totals, ws->C))) return rc;
    if ((rc = dalloc(ws, &ws->d_grads, pc))) return rc;
    void* hp = nullptr;
    UT_CUDA(cudaMallocHost(&hp, 2 * sizeof(int32_t)));
    ws->h_err = static_cast<int32_t*>(hp);
    return UT_OK;
}

// Enqueue the reads of the kernels' error flags on `st` (into pinned host words),
// so the host-array entry points need one stream synchronisation in all.
int32_t enqueue_error_reads(ut_workspace* ws, cudaStream_t st) {
    ws->h_err[0] = ws->h_err[1] = 0;
    if (ws->tc.err)
        UT_CUDA(cudaMemcpyAsync(&ws->h_err[0], ws->tc.err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    if (ws->d_serr)
        UT_CUDA(cudaMemcpyAsync(&ws->h_err[1], ws->d_serr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    return UT_OK;
}

// After the synchronisation: report (and clear) a flag the kernels raised.
int32_t error_reads_status(ut_workspace* ws) {
    if (ws->h_err[0]) {
        UT_CUDA(cudaMemset(ws->tc.err, 0, sizeof(int)));
        return fail(UT_ERR_DEVICE_TIMEOUT, "a bounded wait inside the tensor-core GLM kernel gave up; "
                                           "its results are invalid");
    }
    if (ws->h_err[1]) {
        const int code = ws->h_err[1];
        UT_CUDA(cudaMemset(ws->d_serr, 0, sizeof(int)));
        return fail(UT_ERR_DEVICE_TIMEOUT, "a bounded wait inside the streaming GLM kernel gave up (%s); "
                                           "its results are invalid", code == 2 ? "grid barrier" : "ring wait");
    }
    return UT_OK;
}

int32_t check_ws(const ut_workspace* ws) {
    if (!ws) return fail(UT_ERR_ARGUMENT, "null workspace handle");
    return UT_OK;
}

}  // namespace

// ===========================================================================
extern "C" {

const char* ut_version(void) { return "uncertaintea_b200 0.1.0 (sm_100a)"; }

int32_t ut_last_error(char* buf, size_t len) {
    if (buf && len > 0) {
        size_t n = std::min(len - 1, g_last_error.size());
        memcpy(buf, g_last_error.data(), n);
        buf[n] = '\0';
    }
    return (int32_t)g_last_error.size();
}

int32_t ut_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int32_t ut_lowering_report(const ut_plan_desc* plan, char* issues, size_t len) {
    std::string s = plan_issues(plan);
    if (issues && len > 0) {
        size_t n = std::min(len - 1, s.size());
        memcpy(issues, s.data(), n);
        issues[n] = '\0';
    }
    if (!s.empty()) return fail(UT_ERR_UNSUPPORTED, "kernel description cannot be lowered to the device path:\n%s", s.c_str());
    return UT_OK;
}

int32_t ut_workspace_create(const ut_plan_desc* plan, const float* observed, int64_t observed_rows,
                            int64_t observed_cols, const int32_t* trip_counts, const int32_t* loop_starts,
                            int32_t num_loops, int32_t batch_size, int32_t precision_bits, ut_workspace** out) {
    if (!out) return fail(UT_ERR_ARGUMENT, "null output handle");
    *out = nullptr;
    if (precision_bits != 32)
        return fail(UT_ERR_PRECISION,
                    "the B200 backend does not support Float%d arithmetic; request precision=Float32 instead",
                    (int)precision_bits);
    std::string issues = plan_issues(plan);
    if (!issues.empty()) return fail(UT_ERR_UNSUPPORTED, "kernel description cannot be lowered to the device path:\n%s", issues.c_str());
    if (batch_size < 1) return fail(UT_ERR_ARGUMENT, "batch size must be >= 1, got %d", (int)batch_size);
    if (observed_cols != 1)
        return fail(UT_ERR_UNSUPPORTED, "per-chain observation columns (observed_cols=%lld) are not supported; stage one shared column",
                    (long long)observed_cols);
    const int N = plan->num_obs;
    if (plan->family == UT_FAMILY_GLM_BERNOULLI_LOGIT) {
        int64_t want = (int64_t)N * (plan->num_coefs + 1);
        if (observed_rows != want)
            return fail(UT_ERR_DIMENSION, "expected %lld staged observation rows (N*(D+1)), got %lld", (long long)want,
                        (long long)observed_rows);
    } else if (plan->family == UT_FAMILY_NORMAL_LOCATION_SCALE || plan->family == UT_FAMILY_BERNOULLI_BETA ||
               plan->family == UT_FAMILY_LOGNORMAL_GAMMA_NORMAL || plan->family == UT_FAMILY_STUDENTT_HEAVY_TAIL ||
               plan->family == UT_FAMILY_NORMAL_KNOWN_SCALE) {
        if (observed_rows != N)
            return fail(UT_ERR_DIMENSION, "expected %d staged observation rows (N), got %lld", N,
                        (long long)observed_rows);
    } else {
        int64_t want = (int64_t)N + plan->num_groups;
        if (observed_rows != want)
            return fail(UT_ERR_DIMENSION, "expected %lld staged observation rows (N+J), got %lld", (long long)want,
                        (long long)observed_rows);
        if (num_loops != plan->num_groups || !trip_counts || !loop_starts)
            return fail(UT_ERR_DIMENSION, "expected %d trip counts / loop starts, got %d", plan->num_groups, (int)num_loops);
        int64_t total = 0;
        for (int j = 0; j < num_loops; ++j) {
            if (trip_counts[j] < 0 || loop_starts[j] < 0 || (int64_t)loop_starts[j] + trip_counts[j] > N)
                return fail(UT_ERR_ARGUMENT, "group %d has an out-of-range observation block", j);
            total += trip_counts[j];
        }
        if (total != N) return fail(UT_ERR_DIMENSION, "trip counts sum to %lld, expected %d", (long long)total, N);
    }
    if (N > 0 && !observed) return fail(UT_ERR_ARGUMENT, "null observation buffer");
    int32_t rc = need_device();
    if (rc) return rc;

    ut_workspace* ws = new ut_workspace();
    ws->plan = *plan;
    ws->P = plan->num_params;
    ws->C = batch_size;
    ws->N = N;
    cudaGetDevice(&ws->device);
    auto bail = [&](int32_t code) {
        ut_workspace_destroy(ws);
        return code;
    };
    if (cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(UT_ERR_CUDA, "cudaStreamCreate failed"));

    DevModel& dm = ws->dm;
    memset(&dm, 0, sizeof(dm));
    dm.P = ws->P;
    ws->K = inst_k(ws->P);
    dm.Ppad = 32 * ws->K;
    if (plan->family == UT_FAMILY_GLM_BERNOULLI_LOGIT) {
        const int D = plan->num_coefs, off = plan->has_intercept ? 1 : 0, F = ws->P;
        dm.family = kFamGlm;
        dm.glm.N = N; dm.glm.D = D; dm.glm.off = off;
        dm.glm.icpt_mu = (float)plan->intercept_mu; dm.glm.icpt_sigma = (float)plan->intercept_sigma;
        dm.glm.coef_mu = (float)plan->coef_mu; dm.glm.coef_sigma = (float)plan->coef_sigma;
        std::vector<float> y(N);
        for (int i = 0; i < N; ++i) y[i] = observed[(size_t)i * (D + 1) + D];
        if ((rc = dalloc(ws, &ws->d_y, N))) return bail(rc);
        UT_CUDA(cudaMemcpy(ws->d_y, y.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
        dm.glm.y = ws->d_y;
        size_t staged = (size_t)N * (D + 1);
        bool warp_ok = D <= 32 && (staged * 4 + (size_t)kWarpsDensity * dm.Ppad * 4) <= kSmemBudget;
        if (warp_ok) {
            ws->path = kPathWarp;
            ws->dmax = D <= 16 ? 16 : 32;
            std::vector<float> XT((size_t)D * N);
            for (int i = 0; i < N; ++i)
                for (int d = 0; d < D; ++d) XT[(size_t)d * N + i] = observed[(size_t)i * (D + 1) + d];
            if ((rc = dalloc(ws, &ws->d_XT, XT.size()))) return bail(rc);
            UT_CUDA(cudaMemcpy(ws->d_XT, XT.data(), sizeof(float) * XT.size(), cudaMemcpyHostToDevice));
            dm.glm.XT = ws->d_XT;
            dm.stage = 1;
            dm.staged_floats = (int)(((staged + 3) / 4) * 4);
        } else {
            ws->path = kPathTiled;
            std::vector<float> Xa((size_t)N * F);
            for (int i = 0; i < N; ++i) {
                if (off) Xa[(size_t)i * F] = 1.0f;
                for (int d = 0; d < D; ++d) Xa[(size_t)i * F + off + d] = observed[(size_t)i * (D + 1) + d];
            }
            if ((rc = dalloc(ws, &ws->d_Xa, Xa.size()))) return bail(rc);
            UT_CUDA(cudaMemcpy(ws->d_Xa, Xa.data(), sizeof(float) * Xa.size(), cudaMemcpyHostToDevice));
            int dev_sms = 148;
            cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ws->device);
            int ctiles = (ws->C + kGlmCT - 1) / kGlmCT;
            int target = 3 * dev_sms;
            int chunks = std::max(1, (N + kGlmOT - 1) / kGlmOT);
            int S = std::max(1, std::min(chunks, (target + ctiles - 1) / ctiles));
            int per = (chunks + S - 1) / S;
            ws->obs_per_split = per * kGlmOT;
            ws->splits = std::max(1, (N + ws->obs_per_split - 1) / ws->obs_per_split);
            int need = (F + 15) / 16;
            const int fpts[] = {1, 2, 4, 7, 8, 12, 16};
            for (int v : fpts) if (need <= v) { ws->fpt = v; break; }
            if ((rc = dalloc(ws, &ws->d_part_ll, (size_t)ws->splits * ws->C))) return bail(rc);
            if ((rc = dalloc(ws, &ws->d_part_g, (size_t)ws->splits * ws->C * F))) return bail(rc);
            // few chains: the HBM-streaming kernel (UT_DISABLE_STREAM_KERNEL=1 keeps the tiled one)
            const char* no_stream = getenv("UT_DISABLE_STREAM_KERNEL");
            if (ws->C <= kStreamMaxC && F % 4 == 0 && F <= kStreamMaxF && !(no_stream && no_stream[0] == '1')) {
                ws->streaming = true;
                const int C = ws->C;
                ws->stream_cb = C <= 1 ? 1 : C <= 2 ? 2 : C <= 4 ? 4 : C <= 8 ? 8 : 16;
                ws->stream_splits = dev_sms;  // one CTA per SM, each a contiguous range of 32-row chunks
                int optin = 0;
                cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ws->device);
                const int chunks = (N + kStreamRows - 1) / kStreamRows;
                if (!glm_stream_plan(ws->stream_cb, F, (size_t)std::max(0, optin - 1024), &ws->stream_stages,
                                     &ws->stream_slots))
                    return bail(fail(UT_ERR_UNSUPPORTED, "streaming kernel: shared memory too small"));
                ws->stream_smem = glm_stream_smem(ws->stream_cb, F, ws->stream_stages);
                const int groups = glm_stream_groups(ws->stream_splits);
                const size_t ypad = (size_t)chunks * kStreamRows;
                if ((rc = dalloc(ws, &ws->d_ypad, ypad))) return bail(rc);
                UT_CUDA(cudaMemset(ws->d_ypad, 0, ypad * sizeof(float)));
                UT_CUDA(cudaMemcpy(ws->d_ypad, ws->d_y, (size_t)N * sizeof(float), cudaMemcpyDeviceToDevice));
                if ((rc = dalloc(ws, &ws->d_spart, (size_t)ws->stream_splits * C * (F + 1)))) return bail(rc);
                if ((rc = dalloc(ws, &ws->d_sgpart, (size_t)groups * C * (F + 1)))) return bail(rc);
                if ((rc = dalloc(ws, &ws->d_stickets, (size_t)groups + 1))) return bail(rc);
                if ((rc = dalloc(ws, &ws->d_serr, 1))) return bail(rc);
                UT_CUDA(cudaMemset(ws->d_stickets, 0, ((size_t)groups + 1) * sizeof(unsigned)));
                UT_CUDA(cudaMemset(ws->d_serr, 0, sizeof(int)));
            } else if ((rc = tc_glm_setup(ws->tc, ws->d_Xa, ws->d_y, N, F, ws->C, off, (float)plan->intercept_mu,
                                          (float)plan->intercept_sigma, (float)plan->coef_mu,
                                          (float)plan->coef_sigma, dev_sms, &ws->allocations))) {
                return bail(fail(UT_ERR_CUDA, "tensor-core GLM setup failed: %s", tc_glm_last_error()));
            }
        }
    } else if (plan->family == UT_FAMILY_NORMAL_LOCATION_SCALE || plan->family == UT_FAMILY_NORMAL_KNOWN_SCALE) {
        dm.family = kFamGauss;
        dm.gauss.N = N;
        dm.gauss.mu_loc = (float)plan->mu_loc; dm.gauss.mu_scale = (float)plan->mu_scale;
        if (plan->family == UT_FAMILY_NORMAL_KNOWN_SCALE) {
            dm.gauss.known = 1;
            dm.gauss.sigma = (float)plan->obs_scale;
            dm.gauss.log_sigma = std::log((float)plan->obs_scale);
            dm.gauss.shape = dm.gauss.rate = 1.0f;
            dm.gauss.lgc = 0.0f;
        } else {
            dm.gauss.known = 0;
            dm.gauss.shape = (float)plan->scale_shape; dm.gauss.rate = (float)plan->scale_rate;
            dm.gauss.lgc = (float)(plan->scale_shape * std::log(plan->scale_rate) - std::lgamma(plan->scale_shape));
        }
        if ((rc = dalloc(ws, &ws->d_y, std::max(N, 1)))) return bail(rc);
        if (N > 0) UT_CUDA(cudaMemcpy(ws->d_y, observed, sizeof(float) * N, cudaMemcpyHostToDevice));
        dm.gauss.y = ws->d_y;
        ws->path = kPathWarp;
        dm.stage = ((size_t)N * 4 + (size_t)kWarpsDensity * dm.Ppad * 4) <= kSmemBudget ? 1 : 0;
        dm.staged_floats = dm.stage ? ((N + 3) / 4) * 4 : 0;
    } else if (plan->family == UT_FAMILY_STUDENTT_HEAVY_TAIL) {
        dm.family = kFamHt;
        HtModel& h = dm.ht;
        h.N = N;
        h.nu0 = (float)plan->nu_prior; h.mu0 = (float)plan->mu_loc; h.sigma0 = (float)plan->mu_scale;
        h.nu1 = (float)plan->nu_obs;
        h.ig_a = (float)plan->scale_shape; h.ig_b = (float)plan->scale_rate;
        h.wb_k = (float)plan->weibull_shape; h.wb_l = (float)plan->weibull_scale;
        auto tconst = [](double nu) {
            return std::lgamma((nu + 1.0) / 2.0) - std::lgamma(nu / 2.0) - 0.5 * (std::log(nu) + std::log(3.141592653589793));
        };
        h.c_prior = (float)(tconst(plan->nu_prior) - std::log(plan->mu_scale));
        h.c_obs = (float)tconst(plan->nu_obs);
        h.c_ig = (float)(plan->scale_shape * std::log(plan->scale_rate) - std::lgamma(plan->scale_shape));
        h.c_wb = (float)(std::log(plan->weibull_shape) - plan->weibull_shape * std::log(plan->weibull_scale));
        if ((rc = dalloc(ws, &ws->d_y, std::max(N, 1)))) return bail(rc);
        if (N > 0) UT_CUDA(cudaMemcpy(ws->d_y, observed, sizeof(float) * N, cudaMemcpyHostToDevice));
        h.y = ws->d_y;
        ws->path = kPathWarp;
        dm.stage = ((size_t)N * 4 + (size_t)kWarpsDensity * dm.Ppad * 4) <= kSmemBudget ? 1 : 0;
        dm.staged_floats = dm.stage ? ((N + 3) / 4) * 4 : 0;
    } else if (plan->family == UT_FAMILY_LOGNORMAL_GAMMA_NORMAL) {
        dm.family = kFamLgn;
        dm.lgn.N = N;
        dm.lgn.mu = (float)plan->mu_loc; dm.lgn.sigma = (float)plan->mu_scale;
        dm.lgn.shape = (float)plan->scale_shape; dm.lgn.rate = (float)plan->scale_rate;
        dm.lgn.lgc = (float)(plan->scale_shape * std::log(plan->scale_rate) - std::lgamma(plan->scale_shape));
        if ((rc = dalloc(ws, &ws->d_y, std::max(N, 1)))) return bail(rc);
        if (N > 0) UT_CUDA(cudaMemcpy(ws->d_y, observed, sizeof(float) * N, cudaMemcpyHostToDevice));
        dm.lgn.y = ws->d_y;
        ws->path = kPathWarp;
        dm.stage = ((size_t)N * 4 + (size_t)kWarpsDensity * dm.Ppad * 4) <= kSmemBudget ? 1 : 0;
        dm.staged_floats = dm.stage ? ((N + 3) / 4) * 4 : 0;
    } else if (plan->family == UT_FAMILY_BERNOULLI_BETA) {
        dm.family = kFamBern;
        dm.bern.N = N;
        dm.bern.a = (float)plan->prob_alpha;
        dm.bern.b = (float)plan->prob_beta;
        dm.bern.lbeta = (float)(std::lgamma(plan->prob_alpha) + std::lgamma(plan->prob_beta) -
                                std::lgamma(plan->prob_alpha + plan->prob_beta));
        if ((rc = dalloc(ws, &ws->d_y, std::max(N, 1)))) return bail(rc);
        if (N > 0) UT_CUDA(cudaMemcpy(ws->d_y, observed, sizeof(float) * N, cudaMemcpyHostToDevice));
        dm.bern.z = ws->d_y;
        ws->path = kPathWarp;
        dm.stage = ((size_t)N * 4 + (size_t)kWarpsDensity * dm.Ppad * 4) <= kSmemBudget ? 1 : 0;
        dm.staged_floats = dm.stage ? ((N + 3) / 4) * 4 : 0;
    } else {
        const int J = plan->num_groups;
        dm.family = kFamHier;
        dm.hier.N = N; dm.hier.J = J;
        dm.hier.mu_loc = (float)plan->mu_loc; dm.hier.mu_scale = (float)plan->mu_scale;
        dm.hier.tau_scale = (float)plan->tau_scale;
        if ((rc = dalloc(ws, &ws->d_y, N + J))) return bail(rc);
        UT_CUDA(cudaMemcpy(ws->d_y, observed, sizeof(float) * (N + J), cudaMemcpyHostToDevice));
        if ((rc = dalloc(ws, &ws->d_start, J))) return bail(rc);
        if ((rc = dalloc(ws, &ws->d_count, J))) return bail(rc);
        UT_CUDA(cudaMemcpy(ws->d_start, loop_starts, sizeof(int32_t) * J, cudaMemcpyHostToDevice));
        UT_CUDA(cudaMemcpy(ws->d_count, trip_counts, sizeof(int32_t) * J, cudaMemcpyHostToDevice));
        dm.hier.y = ws->d_y;
        dm.hier.sig = ws->d_y + N;
        dm.hier.start = ws->d_start;
        dm.hier.count = ws->d_count;
        ws->path = kPathWarp;
        size_t staged = (size_t)N + 3 * (size_t)J;
        dm.stage = (staged * 4 + (size_t)kWarpsDensity * dm.Ppad * 4) <= kSmemBudget ? 1 : 0;
        dm.staged_floats = dm.stage ? (int)(((staged + 3) / 4) * 4) : 0;
    }
    *out = ws;
    return UT_OK;
}

int32_t ut_program_report(const ut_program_step* steps, int32_t num_steps, const ut_expr_node* nodes,
                          int32_t num_nodes, int32_t num_slots, int32_t num_params, int64_t observed_rows,
                          char* issues, size_t len) {
    ProgCompiled pc;
    const std::string msg = ProgCompiler(steps, num_steps, nodes, num_nodes, num_slots, num_params, observed_rows).run(&pc);
    if (issues && len) {
        const size_t n = std::min(len - 1, msg.size());
        memcpy(issues, msg.data(), n);
        issues[n] = 0;
    }
    return msg.empty() ? UT_OK : UT_ERR_UNSUPPORTED;
}

int32_t ut_workspace_create_program(const ut_program_step* steps, int32_t num_steps, const ut_expr_node* nodes,
                                    int32_t num_nodes, int32_t num_slots, int32_t num_params, const float* observed,
                                    int64_t observed_rows, int32_t batch_size, int32_t precision_bits,
                                    ut_workspace** out) {
    if (!out) return fail(UT_ERR_ARGUMENT, "null output handle");
    *out = nullptr;
    if (precision_bits != 32)
        return fail(UT_ERR_PRECISION,
                    "the B200 backend does not support Float%d arithmetic; request precision=Float32 instead",
                    (int)precision_bits);
    ProgCompiled pc;
    const std::string issues =
        ProgCompiler(steps, num_steps, nodes, num_nodes, num_slots, num_params, observed_rows).run(&pc);
    if (!issues.empty())
        return fail(UT_ERR_UNSUPPORTED, "kernel description cannot be lowered to the device path:\n%s", issues.c_str());
    if (batch_size < 1) return fail(UT_ERR_ARGUMENT, "batch size must be >= 1, got %d", (int)batch_size);
    if (observed_rows > 0 && !observed) return fail(UT_ERR_ARGUMENT, "null observation buffer");
    int32_t rc = need_device();
    if (rc) return rc;

    ut_workspace* ws = new ut_workspace();
    memset(&ws->plan, 0, sizeof(ws->plan));
    ws->plan.family = UT_FAMILY_PROGRAM;
    ws->plan.num_params = num_params;
    ws->plan.num_obs = (int32_t)observed_rows;
    ws->P = num_params;
    ws->C = batch_size;
    ws->N = (int)observed_rows;
    cudaGetDevice(&ws->device);
    auto bail = [&](int32_t code) {
        ut_workspace_destroy(ws);
        return code;
    };
    if (cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(UT_ERR_CUDA, "cudaStreamCreate failed"));
    DevModel& dm = ws->dm;
    memset(&dm, 0, sizeof(dm));
    dm.family = kFamProg;
    dm.P = num_params;
    ws->K = inst_k(num_params);
    ws->path = kPathWarp;
    ProgModel& m = dm.prog;
    m.nsteps = (int)pc.steps.size();
    m.nnodes = (int)pc.nodes.size();
    m.nslots = pc.nslots;
    m.nobs = (int)observed_rows;
    m.P = num_params;
    m.pp = ((num_params + 31) / 32) * 32;
    dm.Ppad = prog_scratch_floats(num_params, pc.nslots);
    float* d_obs = nullptr;
    PStep* d_steps = nullptr;
    PNode* d_nodes = nullptr;
    if ((rc = dalloc(ws, &d_obs, (size_t)std::max<int64_t>(observed_rows, 1)))) return bail(rc);
    if ((rc = dalloc(ws, &d_steps, pc.steps.size()))) return bail(rc);
    if ((rc = dalloc(ws, &d_nodes, std::max<size_t>(pc.nodes.size(), 1)))) return bail(rc);
    if (observed_rows > 0)
        UT_CUDA(cudaMemcpy(d_obs, observed, sizeof(float) * (size_t)observed_rows, cudaMemcpyHostToDevice));
    UT_CUDA(cudaMemcpy(d_steps, pc.steps.data(), sizeof(PStep) * pc.steps.size(), cudaMemcpyHostToDevice));
    if (!pc.nodes.empty())
        UT_CUDA(cudaMemcpy(d_nodes, pc.nodes.data(), sizeof(PNode) * pc.nodes.size(), cudaMemcpyHostToDevice));
    m.obs = d_obs;
    m.steps = d_steps;
    m.nodes = d_nodes;
    ws->d_y = d_obs;
    // the program and its observations go to shared memory when they fit beside
    // the per-warp scratch of the widest launch
    const size_t staged = ((size_t)(observed_rows + 3) / 4) * 4 + pc.nodes.size() * (sizeof(PNode) / 4) +
                          pc.steps.size() * (sizeof(PStep) / 4);
    dm.stage = (staged * 4 + (size_t)kWarpsDensity * dm.Ppad * 4) <= kSmemBudget ? 1 : 0;
    dm.staged_floats = dm.stage ? (int)(((staged + 3) / 4) * 4) : 0;
    if ((size_t)dm.staged_floats * 4 + (size_t)kWarpsDensity * dm.Ppad * 4 > kSmemBudget)
        return bail(fail(UT_ERR_UNSUPPORTED, "the program's per-chain scratch does not fit shared memory"));
    *out = ws;
    return UT_OK;
}

int32_t ut_workspace_destroy(ut_workspace* ws) {
    if (!ws) return UT_OK;
    for (void* p : ws->allocations) cudaFree(p);
    if (ws->h_active) cudaFreeHost(ws->h_active);
    if (ws->h_err) cudaFreeHost(ws->h_err);
    if (ws->stream) cudaStreamDestroy(ws->stream);
    delete ws;
    return UT_OK;
}

int32_t ut_workspace_info(const ut_workspace* ws, int32_t* num_params, int32_t* batch_size) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (num_params) *num_params = ws->P;
    if (batch_size) *batch_size = ws->C;
    return UT_OK;
}

int32_t ut_workspace_path(const ut_workspace* ws) {
    if (!ws) return 0;
    if (ws->path == kPathWarp) return 1;
    if (ws->streaming) return 4;
    return ws->tc.enabled ? 3 : 2;
}

int32_t ut_workspace_check(ut_workspace* ws, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    UT_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    UT_CUDA(cudaStreamSynchronize(ws->stream));
    if (ws->tc.err) {
        int h = 0;
        UT_CUDA(cudaMemcpy(&h, ws->tc.err, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) {
            UT_CUDA(cudaMemset(ws->tc.err, 0, sizeof(int)));
            return fail(UT_ERR_DEVICE_TIMEOUT, "a bounded wait inside the tensor-core GLM kernel gave up; "
                                               "its results are invalid");
        }
    }
    if (ws->d_serr) {
        int h = 0;
        UT_CUDA(cudaMemcpy(&h, ws->d_serr, sizeof(int), cudaMemcpyDeviceToHost));
        if (h) {
            UT_CUDA(cudaMemset(ws->d_serr, 0, sizeof(int)));
            return fail(UT_ERR_DEVICE_TIMEOUT, "a bounded wait inside the streaming GLM kernel gave up (%s); "
                                               "its results are invalid", h == 2 ? "grid barrier" : "ring wait");
        }
    }
    return UT_OK;
}

// Test hook (not part of the C ABI in ut_b200.h): the tensor-core grid's
// observation split for num_obs observations, num_chains chains and sms SMs.
extern "C" int32_t ut_internal_tc_split_plan(int32_t num_obs, int32_t num_chains, int32_t sms, int32_t* splits,
                                             int32_t* tiles_per_split) {
    if (num_obs < 1 || num_chains < 1 || sms < 1 || !splits || !tiles_per_split) return UT_ERR_ARGUMENT;
    int S = 0, tps = 0;
    tc_choose_split((num_obs + kTcObs - 1) / kTcObs, (num_chains + kTcChains - 1) / kTcChains, sms, &S, &tps);
    *splits = S;
    *tiles_per_split = tps;
    return UT_OK;
}

// Test hook (not part of the C ABI in ut_b200.h): the streaming kernel's stage
// plan for a chain bucket CB and F features under smem_limit bytes; returns
// UT_ERR_UNSUPPORTED when fewer than 4 stages fit.
extern "C" int32_t ut_internal_stream_plan(int32_t CB, int32_t F, int64_t smem_limit, int32_t* stages,
                                           int32_t* slots, int64_t* smem_bytes) {
    if (CB < 1 || CB > kStreamMaxC || F < 1 || smem_limit < 0 || !stages || !slots || !smem_bytes)
        return UT_ERR_ARGUMENT;
    int st = 0, sl = 0;
    if (!glm_stream_plan(CB, F, (size_t)smem_limit, &st, &sl)) return UT_ERR_UNSUPPORTED;
    *stages = st;
    *slots = sl;
    *smem_bytes = (int64_t)glm_stream_smem(CB, F, st);
    return UT_OK;
}

// Test hook (not part of the C ABI in ut_b200.h): the tensor-core work split
// when only `live` chains are live (live < 0: no live count), as the kernels
// compute it; out = {chain tiles, splits, tiles per split, partial-row chains}.
extern "C" int32_t ut_internal_tc_live_split(int32_t num_obs, int32_t num_chains, int32_t sms, int32_t live,
                                             int32_t* out) {
    if (num_obs < 1 || num_chains < 1 || sms < 1 || !out || live > num_chains) return UT_ERR_ARGUMENT;
    TcGlmParams p = {};
    p.N = num_obs;
    p.C = num_chains;
    p.num_tiles = (num_obs + kTcObs - 1) / kTcObs;
    p.ctiles = (num_chains + kTcChains - 1) / kTcChains;
    p.sms = sms;
    tc_choose_split(p.num_tiles, p.ctiles, sms, &p.S, &p.tiles_per_split);
    int n = live;
    p.nact = live >= 0 ? &n : nullptr;
    const TcSplit r = tc_split(p);
    out[0] = r.nt; out[1] = r.S; out[2] = r.tps; out[3] = r.Cl;
    return UT_OK;
}

// Test hook (not part of the C ABI in ut_b200.h): the tensor-core kernel's TMEM
// column plan for F features: out = {KC, Fp, buffers, columns used}.
extern "C" int32_t ut_internal_tc_tmem_plan(int32_t F, int32_t* out) {
    if (F < 1 || F > kTcMaxFp || !out) return UT_ERR_ARGUMENT;
    const int KC = 8 * tc_kblocks_used(F), Fp = ((F + 15) / 16) * 16, nb = tc_nbuf(F, Fp);
    int cols[3];
    tc_columns(F, Fp, false, cols);
    out[0] = KC; out[1] = Fp; out[2] = nb; out[3] = cols[2] + 64 * nb;
    return UT_OK;
}

// Test hook (not part of the C ABI in ut_b200.h): the paired GEMM1's K-major copy
// and the MMAs that read it, for F features and N observations, from the
// kernel's own helpers: out = {K-blocks, box bytes of the 4-D copy, bytes of the
// stage's K-major region, end offset of the last N = 64 B-operand read (2 KB per
// K-block), hi/lo stride in bytes, innermost box bytes}.
extern "C" int32_t ut_internal_tc_pair_plan(int32_t F, int64_t N, int64_t* out) {
    if (F < 1 || F > kTcMaxFp || N < 1 || !out) return UT_ERR_ARGUMENT;
    const int Fp = ((F + 15) / 16) * 16, KB1 = tc_kblocks_used(F);
    out[0] = KB1;
    out[1] = (int64_t)8 * kTcObs * 2 * KB1 * (int64_t)sizeof(float);
    out[2] = 2 * (int64_t)tc_xk_bytes(Fp);
    out[3] = (int64_t)(KB1 - 1) * 2 * (kTcObs * 32) + 2 * kTcObs * 32;
    out[4] = N * Fp * (int64_t)sizeof(float);
    out[5] = 8 * (int64_t)sizeof(float);
    return UT_OK;
}

// Test hook (not part of the C ABI in ut_b200.h): one tensor-core evaluation of
// only the first *d_live chains of d_params -- the live-chain launch masked NUTS
// makes at every leaf, with its observation re-split -- on device buffers.
// Rows of chains at or past *d_live are left untouched.  d_grads may be NULL
// (logjoint only).  UT_ERR_UNSUPPORTED when the workspace is not on the
// tensor-core path.
extern "C" int32_t ut_internal_tc_glm_live(ut_workspace* ws, const float* d_params, float* d_totals, float* d_grads,
                                           const int32_t* d_live, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!ws->tc.enabled) return fail(UT_ERR_UNSUPPORTED, "the workspace is not on the tensor-core path");
    if (!d_params || !d_totals || !d_live) return fail(UT_ERR_ARGUMENT, "null device buffer");
    if (tc_glm_launch(ws->tc, d_params, d_totals, d_grads, (cudaStream_t)stream, d_live) != cudaSuccess)
        return fail(UT_ERR_CUDA, "tensor-core GLM launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    return UT_OK;
}

int32_t ut_logjoint_device(ut_workspace* ws, const float* d_params, float* d_totals, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!d_params || !d_totals) return fail(UT_ERR_ARGUMENT, "null device buffer");
    return density(ws, d_params, d_totals, nullptr, (cudaStream_t)stream);
}

int32_t ut_logjoint_gradient_device(ut_workspace* ws, const float* d_params, float* d_totals, float* d_gradients,
                                    void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!d_params || !d_totals || !d_gradients) return fail(UT_ERR_ARGUMENT, "null device buffer");
    return density(ws, d_params, d_totals, d_gradients, (cudaStream_t)stream);
}

int32_t ut_logjoint(ut_workspace* ws, const float* params, float* totals) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!params || !totals) return fail(UT_ERR_ARGUMENT, "null host buffer");
    if ((rc = ensure_host_buffers(ws))) return rc;
    size_t pc = (size_t)ws->P * ws->C;
    UT_CUDA(cudaMemcpyAsync(ws->d_params, params, pc * sizeof(float), cudaMemcpyHostToDevice, ws->stream));
    if ((rc = density(ws, ws->d_params, ws->d_totals, nullptr, ws->stream))) return rc;
    UT_CUDA(cudaMemcpyAsync(totals, ws->d_totals, ws->C * sizeof(float), cudaMemcpyDeviceToHost, ws->stream));
    if ((rc = enqueue_error_reads(ws, ws->stream))) return rc;
    UT_CUDA(cudaStreamSynchronize(ws->stream));
    return error_reads_status(ws);
}

int32_t ut_logjoint_gradient(ut_workspace* ws, const float* params, float* totals, float* gradients) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!params || !totals || !gradients) return fail(UT_ERR_ARGUMENT, "null host buffer");
    if ((rc = ensure_host_buffers(ws))) return rc;
    size_t pc = (size_t)ws->P * ws->C;
    UT_CUDA(cudaMemcpyAsync(ws->d_params, params, pc * sizeof(float), cudaMemcpyHostToDevice, ws->stream));
    if ((rc = density(ws, ws->d_params, ws->d_totals, ws->d_grads, ws->stream))) return rc;
    UT_CUDA(cudaMemcpyAsync(totals, ws->d_totals, ws->C * sizeof(float), cudaMemcpyDeviceToHost, ws->stream));
    UT_CUDA(cudaMemcpyAsync(gradients, ws->d_grads, pc * sizeof(float), cudaMemcpyDeviceToHost, ws->stream));
    if ((rc = enqueue_error_reads(ws, ws->stream))) return rc;
    UT_CUDA(cudaStreamSynchronize(ws->stream));
    return error_reads_status(ws);
}

// ---- Philox ---------------------------------------------------------------
int32_t ut_philox4x32(const uint32_t* keys, const uint32_t* counters, int64_t n, uint32_t* out) {
    if (n < 0 || (n > 0 && (!keys || !counters || !out))) return fail(UT_ERR_ARGUMENT, "invalid Philox batch");
    if (n == 0) return UT_OK;
    int32_t rc = need_device();
    if (rc) return rc;
    uint32_t *dk = nullptr, *dc = nullptr, *dout = nullptr;
    UT_CUDA(cudaMalloc(&dk, n * 2 * sizeof(uint32_t)));
    UT_CUDA(cudaMalloc(&dc, n * 4 * sizeof(uint32_t)));
    UT_CUDA(cudaMalloc(&dout, n * 4 * sizeof(uint32_t)));
    UT_CUDA(cudaMemcpy(dk, keys, n * 2 * sizeof(uint32_t), cudaMemcpyHostToDevice));
    UT_CUDA(cudaMemcpy(dc, counters, n * 4 * sizeof(uint32_t), cudaMemcpyHostToDevice));
    philox_batch_kernel<<<(unsigned)((n + 255) / 256), 256>>>(dk, dc, n, dout);
    UT_LAUNCHED();
    UT_CUDA(cudaMemcpy(out, dout, n * 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    cudaFree(dk); cudaFree(dc); cudaFree(dout);
    return UT_OK;
}

static int32_t rand_common(uint32_t chain, uint32_t iteration, uint32_t stream, uint32_t draw_start, int64_t n,
                           float* out, int normal) {
    if (n < 0 || (n > 0 && !out)) return fail(UT_ERR_ARGUMENT, "invalid draw batch");
    if (n == 0) return UT_OK;
    int32_t rc = need_device();
    if (rc) return rc;
    float* d = nullptr;
    UT_CUDA(cudaMalloc(&d, n * sizeof(float)));
    rand_batch_kernel<<<(unsigned)((n + 255) / 256), 256>>>(chain, iteration, stream, draw_start, n, normal, d);
    UT_LAUNCHED();
    UT_CUDA(cudaMemcpy(out, d, n * sizeof(float), cudaMemcpyDeviceToHost));
    cudaFree(d);
    return UT_OK;
}

int32_t ut_rand_uniform(uint32_t chain, uint32_t iteration, uint32_t stream, uint32_t draw_start, int64_t n,
                        float* out) {
    return rand_common(chain, iteration, stream, draw_start, n, out, 0);
}
int32_t ut_rand_normal(uint32_t chain, uint32_t iteration, uint32_t stream, uint32_t draw_start, int64_t n,
                       float* out) {
    return rand_common(chain, iteration, stream, draw_start, n, out, 1);
}

// ---- HMC ------------------------------------------------------------------
int32_t ut_hmc_iteration(ut_workspace* ws, const ut_hmc_buffers* buf, int32_t num_leapfrog_steps,
                         uint32_t iteration_coord, float divergence_threshold, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!buf || !buf->position || !buf->gradient || !buf->logjoint || !buf->inverse_mass || !buf->step ||
        !buf->accept_prob || !buf->energy || !buf->energy_error || !buf->accepted || !buf->divergent)
        return fail(UT_ERR_ARGUMENT, "null HMC buffer");
    if (num_leapfrog_steps < 1) return fail(UT_ERR_ARGUMENT, "num_leapfrog_steps must be >= 1, got %d", (int)num_leapfrog_steps);
    cudaStream_t st = (cudaStream_t)stream;
    HmcArgs a;
    a.position = buf->position; a.gradient = buf->gradient; a.logjoint = buf->logjoint;
    a.inverse_mass = buf->inverse_mass; a.step = buf->step;
    a.accept_prob = buf->accept_prob; a.energy = buf->energy; a.energy_error = buf->energy_error;
    a.accepted = buf->accepted; a.divergent = buf->divergent;
    a.proposal = buf->proposal; a.endpoint_momentum = buf->endpoint_momentum;
    a.C = ws->C; a.L = num_leapfrog_steps; a.coord = iteration_coord; a.thr = divergence_threshold;
    if (ws->path == kPathWarp) {
        UT_DISPATCH_WARP(ws, LAUNCH_HMC, ws, a, st);
        UT_LAUNCHED();
        return UT_OK;
    }
    if ((rc = ensure_lf(ws))) return rc;
    const int P = ws->P;
    const unsigned grid = (ws->C + 7) / 8;
    UT_K_SWITCH(ws->K, lf_begin_kernel<K><<<grid, 256, 0, st>>>(a, ws->lf, P));
    UT_LAUNCHED();
    // few chains on the streaming path: the L evaluations in one launch
    // (UT_DISABLE_STREAM_TRAJECTORY=1 keeps one launch per step; same values, bit for bit)
    const char* no_traj = getenv("UT_DISABLE_STREAM_TRAJECTORY");
    if (ws->streaming && !(no_traj && no_traj[0] == '1')) {
        rc = launch_stream_traj(ws, a, num_leapfrog_steps, st);
        if (rc == UT_OK) {
            UT_K_SWITCH(ws->K, lf_step_kernel<K><<<grid, 256, 0, st>>>(a, ws->lf, P, num_leapfrog_steps));
            UT_LAUNCHED();
            return UT_OK;
        }
        if (rc != UT_ERR_UNSUPPORTED) return rc;
    }
    for (int l = 1; l <= num_leapfrog_steps; ++l) {
        if ((rc = density(ws, ws->lf.wq, ws->lf.wlj, ws->lf.wg, st))) return rc;
        UT_K_SWITCH(ws->K, lf_step_kernel<K><<<grid, 256, 0, st>>>(a, ws->lf, P, l));
        UT_LAUNCHED();
    }
    return UT_OK;
}

int32_t ut_chees_iteration(ut_workspace* ws, const ut_hmc_buffers* buf, int32_t num_leapfrog_steps,
                           uint32_t iteration_coord, float divergence_threshold, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!buf || !buf->proposal || !buf->endpoint_momentum)
        return fail(UT_ERR_ARGUMENT, "a ChEES iteration needs non-null proposal and endpoint-momentum buffers");
    return ut_hmc_iteration(ws, buf, num_leapfrog_steps, iteration_coord, divergence_threshold, stream);
}

// Defined in ut_surrogate.cu (C++ linkage: not part of the exported C ABI).
extern "C++" int ut_internal_surrogate_num_params(const ut_surrogate* s);
extern "C++" int32_t ut_internal_surrogate_forward(const ut_surrogate* s, const float* x, int64_t n, float* out,
                                                   cudaStream_t st);

int32_t ut_surrogate_hmc_iteration(ut_workspace* ws, const ut_surrogate* s, const ut_hmc_buffers* buf,
                                   int32_t num_leapfrog_steps, uint32_t iteration_coord, float divergence_threshold,
                                   void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!s) return fail(UT_ERR_ARGUMENT, "null surrogate handle");
    if (ut_internal_surrogate_num_params(s) != ws->P)
        return fail(UT_ERR_DIMENSION, "surrogate has %d parameters, the model %d", ut_internal_surrogate_num_params(s),
                    ws->P);
    if (!buf || !buf->position || !buf->logjoint || !buf->inverse_mass || !buf->step || !buf->accept_prob ||
        !buf->energy || !buf->energy_error || !buf->accepted || !buf->divergent)
        return fail(UT_ERR_ARGUMENT, "null HMC buffer");
    if (num_leapfrog_steps < 1) return fail(UT_ERR_ARGUMENT, "num_leapfrog_steps must be >= 1, got %d", (int)num_leapfrog_steps);
    if ((rc = ensure_lf(ws))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    HmcArgs a;
    a.position = buf->position; a.logjoint = buf->logjoint;
    // the kicks read the surrogate gradient from lf.wg; the accept copies the
    // accepted row of lf.wg onto itself, so buf->gradient is never touched
    a.gradient = ws->lf.wg;
    a.inverse_mass = buf->inverse_mass; a.step = buf->step;
    a.accept_prob = buf->accept_prob; a.energy = buf->energy; a.energy_error = buf->energy_error;
    a.accepted = buf->accepted; a.divergent = buf->divergent;
    a.proposal = buf->proposal; a.endpoint_momentum = buf->endpoint_momentum;
    a.C = ws->C; a.L = num_leapfrog_steps; a.coord = iteration_coord; a.thr = divergence_threshold;
    const int P = ws->P;
    const unsigned grid = (ws->C + 7) / 8;
    if ((rc = ut_internal_surrogate_forward(s, buf->position, ws->C, ws->lf.wg, st))) return rc;
    UT_K_SWITCH(ws->K, lf_begin_kernel<K><<<grid, 256, 0, st>>>(a, ws->lf, P));
    UT_LAUNCHED();
    for (int l = 1; l <= num_leapfrog_steps; ++l) {
        if ((rc = ut_internal_surrogate_forward(s, ws->lf.wq, ws->C, ws->lf.wg, st))) return rc;
        if (l == num_leapfrog_steps && (rc = density(ws, ws->lf.wq, ws->lf.wlj, nullptr, st))) return rc;
        UT_K_SWITCH(ws->K, lf_step_kernel<K><<<grid, 256, 0, st>>>(a, ws->lf, P, l));
        UT_LAUNCHED();
    }
    return UT_OK;
}

int32_t ut_leapfrog_probe(ut_workspace* ws, const float* d_position, const float* d_gradient, const float* d_logjoint,
                          const float* d_inverse_mass, const float* d_trial_step, uint32_t iteration_coord,
                          float* d_log_accept_ratio, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!d_position || !d_gradient || !d_logjoint || !d_inverse_mass || !d_trial_step || !d_log_accept_ratio)
        return fail(UT_ERR_ARGUMENT, "null probe buffer");
    cudaStream_t st = (cudaStream_t)stream;
    if (ws->path == kPathWarp) {
        ProbeArgs a;
        a.position = d_position; a.gradient = d_gradient; a.logjoint = d_logjoint;
        a.inverse_mass = d_inverse_mass; a.trial_step = d_trial_step; a.log_accept_ratio = d_log_accept_ratio;
        a.C = ws->C; a.coord = iteration_coord;
        UT_DISPATCH_WARP(ws, LAUNCH_PROBE, ws, a, st);
        UT_LAUNCHED();
        return UT_OK;
    }
    if ((rc = ensure_lf(ws))) return rc;
    HmcArgs a = {};
    a.position = const_cast<float*>(d_position); a.gradient = const_cast<float*>(d_gradient);
    a.logjoint = const_cast<float*>(d_logjoint); a.inverse_mass = d_inverse_mass; a.step = d_trial_step;
    a.C = ws->C; a.L = 1; a.coord = iteration_coord;
    const int P = ws->P;
    const unsigned grid = (ws->C + 7) / 8;
    UT_K_SWITCH(ws->K, lf_begin_kernel<K><<<grid, 256, 0, st>>>(a, ws->lf, P));
    UT_LAUNCHED();
    if ((rc = density(ws, ws->lf.wq, ws->lf.wlj, ws->lf.wg, st))) return rc;
    UT_K_SWITCH(ws->K, lf_probe_close_kernel<K><<<grid, 256, 0, st>>>(d_inverse_mass, d_trial_step, ws->lf,
                                                                        d_log_accept_ratio, P, ws->C));
    UT_LAUNCHED();
    return UT_OK;
}

// ---- persistent NUTS --------------------------------------------------------
int32_t ut_persistent_nuts_iteration(ut_workspace* ws, const ut_nuts_buffers* buf, int32_t max_tree_depth,
                                     float divergence_threshold, uint32_t iteration_coord, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!buf || !buf->position || !buf->gradient || !buf->logjoint || !buf->inverse_mass || !buf->step ||
        !buf->accept_prob || !buf->energy || !buf->energy_error || !buf->tree_depth || !buf->integration_steps ||
        !buf->divergent || !buf->moved)
        return fail(UT_ERR_ARGUMENT, "null NUTS buffer");
    if (max_tree_depth < 1 || max_tree_depth > 30)
        return fail(UT_ERR_ARGUMENT, "max_tree_depth must be in 1..30, got %d", (int)max_tree_depth);
    if (ws->path != kPathWarp)
        return fail(UT_ERR_UNSUPPORTED,
                    "the persistent NUTS tree needs a per-chain (warp) evaluator; this model's observation data "
                    "does not fit the warp path (use batched_chees / batched_hmc for it)");
    if (ws->ckpt_depth < max_tree_depth) {
        if (ws->d_ckpt) {
            cudaFree(ws->d_ckpt);
            ws->allocations.erase(std::remove(ws->allocations.begin(), ws->allocations.end(), (void*)ws->d_ckpt),
                                  ws->allocations.end());
            ws->d_ckpt = nullptr;
        }
        if ((rc = dalloc(ws, &ws->d_ckpt, (size_t)ws->C * (max_tree_depth + 1) * 2 * 32 * ws->K))) return rc;
        ws->ckpt_depth = max_tree_depth;
    }
    NutsArgs a;
    a.position = buf->position; a.gradient = buf->gradient; a.logjoint = buf->logjoint;
    a.inverse_mass = buf->inverse_mass; a.step = buf->step;
    a.accept_prob = buf->accept_prob; a.energy = buf->energy; a.energy_error = buf->energy_error;
    a.tree_depth = buf->tree_depth; a.integration_steps = buf->integration_steps;
    a.divergent = buf->divergent; a.moved = buf->moved;
    a.ckpt = ws->d_ckpt; a.C = ws->C; a.max_depth = max_tree_depth; a.coord = iteration_coord;
    a.thr = divergence_threshold;
    cudaStream_t st = (cudaStream_t)stream;
    UT_DISPATCH_WARP(ws, LAUNCH_NUTS, ws, a, st);
    UT_LAUNCHED();
    return UT_OK;
}

// ---- MEADS -------------------------------------------------------------------
namespace {
int meads_k_slots(int P) { return P <= 32 ? 1 : P <= 64 ? 2 : P <= 96 ? 3 : P <= 128 ? 4 : P <= 256 ? 8 : 17; }
#define UT_MEADS_K_SWITCH(KV, ...)                                   \
    switch (KV) {                                                    \
        case 1: { constexpr int K = 1; __VA_ARGS__; } break;         \
        case 2: { constexpr int K = 2; __VA_ARGS__; } break;         \
        case 3: { constexpr int K = 3; __VA_ARGS__; } break;         \
        case 4: { constexpr int K = 4; __VA_ARGS__; } break;         \
        case 8: { constexpr int K = 8; __VA_ARGS__; } break;         \
        default: { constexpr int K = 17; __VA_ARGS__; } break;       \
    }

int32_t meads_check(ut_workspace* ws, const ut_meads_buffers* buf) {
    if (!buf || !buf->position || !buf->gradient || !buf->logjoint || !buf->momentum || !buf->slice ||
        !buf->accept_prob || !buf->energy || !buf->energy_error || !buf->accepted || !buf->divergent ||
        !buf->integration_steps)
        return fail(UT_ERR_ARGUMENT, "null MEADS buffer");
    if (ws->P > 544) return fail(UT_ERR_UNSUPPORTED, "MEADS supports up to 544 parameters");
    return UT_OK;
}

MeadsArgs meads_args(ut_workspace* ws, const ut_meads_buffers* buf, uint32_t coord, float thr, int skip) {
    MeadsArgs a;
    a.position = buf->position; a.gradient = buf->gradient; a.logjoint = buf->logjoint;
    a.momentum = buf->momentum; a.slice = buf->slice; a.accept_prob = buf->accept_prob; a.energy = buf->energy;
    a.energy_error = buf->energy_error; a.accepted = buf->accepted; a.divergent = buf->divergent;
    a.steps = buf->integration_steps;
    a.C = ws->C; a.P = ws->P; a.skip = skip; a.coord = coord; a.thr = thr;
    return a;
}
}  // namespace

int32_t ut_meads_init(ut_workspace* ws, const ut_meads_buffers* buf, uint32_t iteration_coord, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if ((rc = meads_check(ws, buf))) return rc;
    MeadsArgs a = meads_args(ws, buf, iteration_coord, 0.0f, -1);
    const unsigned grid = (unsigned)((ws->C + 7) / 8);
    UT_MEADS_K_SWITCH(meads_k_slots(ws->P), meads_init_kernel<K><<<grid, 256, 0, (cudaStream_t)stream>>>(a));
    UT_LAUNCHED();
    return UT_OK;
}

int32_t ut_meads_iteration(ut_workspace* ws, const ut_meads_buffers* buf, int32_t num_folds, int32_t iteration,
                           float divergence_threshold, uint32_t iteration_coord, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if ((rc = meads_check(ws, buf))) return rc;
    if (num_folds < 2 || num_folds > 32) return fail(UT_ERR_ARGUMENT, "num_folds must be in 2..32, got %d", (int)num_folds);
    if (ws->C < 2 * num_folds)
        return fail(UT_ERR_ARGUMENT, "MEADS needs num_chains >= 2 * num_folds; got num_chains=%d, num_folds=%d",
                    (int)ws->C, (int)num_folds);
    if (iteration < 1) return fail(UT_ERR_ARGUMENT, "iteration must be >= 1, got %d", (int)iteration);
    if ((rc = ensure_lf(ws))) return rc;
    const int P = ws->P, C = ws->C, K = num_folds;
    const int tx = (P + kMeadsTile - 1) / kMeadsTile;
    MeadsScratch& s = ws->meads;
    if (ws->meads_k != K) {  // (re)allocate for this fold count; earlier buffers are freed with the workspace
        s.ntiles = tx * tx;
        if ((rc = dalloc(ws, &s.mean, (size_t)K * P))) return rc;
        if ((rc = dalloc(ws, &s.sd, (size_t)K * P))) return rc;
        if ((rc = dalloc(ws, &s.tiles, (size_t)K * 2 * s.ntiles))) return rc;
        if ((rc = dalloc(ws, &s.norms, (size_t)K * 4))) return rc;
        if ((rc = dalloc(ws, &s.sdf, (size_t)K * P))) return rc;
        if ((rc = dalloc(ws, &s.fold, (size_t)K * 4))) return rc;
        if (!s.refreshed && (rc = dalloc(ws, &s.refreshed, (size_t)C * P))) return rc;
        ws->meads_k = K;
    }
    cudaStream_t st = (cudaStream_t)stream;
    MeadsFolds fo;
    fo.C = C; fo.P = P; fo.K = K;
    const int skip = (iteration - 1) % K;
    meads_stats_kernel<<<dim3(P, K), 256, 0, st>>>(fo, buf->position, s);
    meads_moment_kernel<<<dim3(tx, tx, 2 * K), dim3(kMeadsTile, kMeadsTile), 0, st>>>(fo, buf->position,
                                                                                       buf->gradient, s);
    meads_norm_kernel<<<2 * K, 256, 0, st>>>(fo, buf->position, buf->gradient, s);
    meads_params_kernel<<<1, 32, 0, st>>>(fo, s, (int)iteration);
    UT_LAUNCHED();
    MeadsArgs a = meads_args(ws, buf, iteration_coord, divergence_threshold, skip);
    const unsigned grid = (unsigned)((C + 7) / 8);
    const int KS = meads_k_slots(P);
    UT_MEADS_K_SWITCH(KS, meads_begin_kernel<K><<<grid, 256, 0, st>>>(a, fo, s, ws->lf));
    UT_LAUNCHED();
    if ((rc = density(ws, ws->lf.wq, ws->lf.wlj, ws->lf.wg, st))) return rc;
    UT_MEADS_K_SWITCH(KS, meads_end_kernel<K><<<grid, 256, 0, st>>>(a, fo, s, ws->lf));
    UT_LAUNCHED();
    if (buf->fold_parameters)
        UT_CUDA(cudaMemcpyAsync(buf->fold_parameters, s.fold, sizeof(float) * 4 * K, cudaMemcpyDeviceToDevice, st));
    return UT_OK;
}

// ---- mean-field ADVI step ---------------------------------------------------
int32_t ut_advi_step(ut_workspace* ws, const float* d_location, const float* d_scale, uint32_t iteration_coord,
                     float* d_particles, float* d_values, float* d_gradients, float* d_location_gradient,
                     float* d_scale_gradient, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!d_location || !d_scale || !d_particles || !d_values || !d_gradients || !d_location_gradient ||
        !d_scale_gradient)
        return fail(UT_ERR_ARGUMENT, "null ADVI buffer");
    cudaStream_t st = (cudaStream_t)stream;
    const int P = ws->P, M = ws->C;
    const long long n = (long long)P * M;
    const unsigned grid = (unsigned)std::min<long long>((n + 255) / 256, 4096);
    advi_particles_kernel<<<grid, 256, 0, st>>>(d_location, d_scale, iteration_coord, P, M, d_particles);
    UT_LAUNCHED();
    if ((rc = density(ws, d_particles, d_values, d_gradients, st))) return rc;
    advi_reduce_kernel<<<P, 256, 0, st>>>(d_gradients, d_scale, iteration_coord, P, M, d_location_gradient,
                                          d_scale_gradient);
    UT_LAUNCHED();
    return UT_OK;
}

// ---- lockstep (masked) NUTS ------------------------------------------------
// Leaves between the host's checks of the live-chain count: a check drains the
// stream, while a step with no live chain costs only its kernels' early exits.
constexpr int kLsCheckEvery = 16;

int32_t ut_lockstep_nuts_iteration(ut_workspace* ws, const ut_nuts_buffers* buf, int32_t max_tree_depth,
                                   float divergence_threshold, uint32_t iteration_coord, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!buf || !buf->position || !buf->gradient || !buf->logjoint || !buf->inverse_mass || !buf->step ||
        !buf->accept_prob || !buf->energy || !buf->energy_error || !buf->tree_depth || !buf->integration_steps ||
        !buf->divergent || !buf->moved)
        return fail(UT_ERR_ARGUMENT, "null NUTS buffer");
    if (max_tree_depth < 1 || max_tree_depth > 16)
        return fail(UT_ERR_ARGUMENT, "max_tree_depth must be in 1..16 for the lockstep tree, got %d",
                    (int)max_tree_depth);
    if (ws->P > 256) return fail(UT_ERR_UNSUPPORTED, "the lockstep NUTS tree supports up to 256 parameters");
    if ((rc = ensure_lf(ws))) return rc;
    const size_t C = ws->C, P = ws->P;
    const int K = ws->P <= 32 ? 1 : ws->P <= 64 ? 2 : ws->P <= 96 ? 3 : ws->P <= 128 ? 4 : 8;
    if (!ws->h_active) {  // keyed on the last buffer made
        if ((rc = dalloc(ws, &ws->ls_vec, (size_t)kLsNumVec * C * P))) return rc;
        if ((rc = dalloc(ws, &ws->ls_f, (size_t)kLsNumF * C))) return rc;
        if ((rc = dalloc(ws, &ws->ls_i, (size_t)kLsNumI * C))) return rc;
        if ((rc = dalloc(ws, &ws->ls_active, 1))) return rc;
        if ((rc = dalloc(ws, &ws->ls_act, C))) return rc;
        if ((rc = dalloc(ws, &ws->ls_idx, C))) return rc;
        if (ws->tc.enabled) {
            if ((rc = dalloc(ws, &ws->ls_cq, C * P))) return rc;
            if ((rc = dalloc(ws, &ws->ls_cg, C * P))) return rc;
            if ((rc = dalloc(ws, &ws->ls_clj, C))) return rc;
            UT_CUDA(cudaMemset(ws->ls_cq, 0, C * P * sizeof(float)));
        }
        void* hp = nullptr;
        UT_CUDA(cudaMallocHost(&hp, sizeof(int32_t)));
        ws->h_active = static_cast<int32_t*>(hp);
    }
    if (ws->ls_depth < max_tree_depth) {
        if (ws->ls_ckpt) {
            cudaFree(ws->ls_ckpt);
            ws->allocations.erase(std::remove(ws->allocations.begin(), ws->allocations.end(), (void*)ws->ls_ckpt),
                                  ws->allocations.end());
            ws->ls_ckpt = nullptr;
        }
        if ((rc = dalloc(ws, &ws->ls_ckpt, C * (max_tree_depth + 1) * 2 * 32 * K))) return rc;
        ws->ls_depth = max_tree_depth;
    }
    LsArgs a;
    a.n.position = buf->position; a.n.gradient = buf->gradient; a.n.logjoint = buf->logjoint;
    a.n.inverse_mass = buf->inverse_mass; a.n.step = buf->step;
    a.n.accept_prob = buf->accept_prob; a.n.energy = buf->energy; a.n.energy_error = buf->energy_error;
    a.n.tree_depth = buf->tree_depth; a.n.integration_steps = buf->integration_steps;
    a.n.divergent = buf->divergent; a.n.moved = buf->moved;
    a.n.ckpt = nullptr; a.n.C = ws->C; a.n.max_depth = max_tree_depth; a.n.coord = iteration_coord;
    a.n.thr = divergence_threshold;
    a.s.vec = ws->ls_vec; a.s.f = ws->ls_f; a.s.i = ws->ls_i; a.s.ckpt = ws->ls_ckpt;
    a.s.wq = ws->lf.wq; a.s.wg = ws->lf.wg; a.s.wlj = ws->lf.wlj; a.s.act = ws->ls_act;
    a.P = ws->P;
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned grid = (unsigned)((C + 3) / 4);
    UT_K_SWITCH(K, ls_init_kernel<K><<<grid, 128, 0, st>>>(a));
    UT_LAUNCHED();
    // at most 2^max_depth - 1 leaves per tree; every kLsCheckEvery leaves the host stops once no
    // chain is still growing
    const int max_steps = (1 << max_tree_depth) - 1;
    const bool compact = ws->tc.enabled;
    // once at most 16 trees still grow (known at a check; the count only falls
    // within an iteration), the remaining leaves are evaluated by the few-chain
    // streaming kernel over that many compacted rows
    const char* no_stream = getenv("UT_DISABLE_STREAM_KERNEL");
    const bool can_stream = compact && P % 4 == 0 && P <= (size_t)kStreamMaxF && !(no_stream && no_stream[0] == '1');
    int tail_rows = 0;
    const unsigned rows_grid = (unsigned)std::min<size_t>((C * P + 255) / 256, 4096);
    for (int step = 0; step < max_steps; ++step) {
        ls_compact_kernel<<<1, 1024, 0, st>>>(ws->ls_act, (int)C, ws->ls_idx, ws->ls_active);
        UT_LAUNCHED();
        if (step > 0 && step % kLsCheckEvery == 0) {
            UT_CUDA(cudaMemcpyAsync(ws->h_active, ws->ls_active, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            UT_CUDA(cudaStreamSynchronize(st));
            if (*ws->h_active == 0) break;
            if (can_stream && *ws->h_active <= kStreamMaxC) tail_rows = *ws->h_active;
        }
        if (compact) {
            ls_gather_kernel<<<rows_grid, 256, 0, st>>>(ws->lf.wq, ws->ls_idx, ws->ls_active, (int)P, ws->ls_cq);
            UT_LAUNCHED();
            if (tail_rows) {
                if ((rc = launch_stream_rows(ws, ws->ls_cq, ws->ls_clj, ws->ls_cg, tail_rows, st))) return rc;
            } else if (tc_glm_launch(ws->tc, ws->ls_cq, ws->ls_clj, ws->ls_cg, st, ws->ls_active) != cudaSuccess)
                return fail(UT_ERR_CUDA, "tensor-core GLM launch failed: %s", cudaGetErrorString(cudaGetLastError()));
            ls_scatter_kernel<<<rows_grid, 256, 0, st>>>(ws->ls_cg, ws->ls_clj, ws->ls_idx, ws->ls_active, (int)P,
                                                         ws->lf.wg, ws->lf.wlj);
            UT_LAUNCHED();
        } else if ((rc = density(ws, ws->lf.wq, ws->lf.wlj, ws->lf.wg, st))) {
            return rc;
        }
        UT_K_SWITCH(K, ls_step_kernel<K><<<grid, 128, 0, st>>>(a));
        UT_LAUNCHED();
    }
    return UT_OK;
}

// ---- ChEES ---------------------------------------------------------------
int32_t ut_chees_reduce(ut_workspace* ws, const float* d_initials, const float* d_proposals,
                        const float* d_endpoint_momentum, const float* d_accept_prob, const uint8_t* d_divergent,
                        const float* d_inverse_mass, double* out, void* stream) {
    int32_t rc = check_ws(ws);
    if (rc) return rc;
    if (!d_initials || !d_proposals || !d_endpoint_momentum || !d_accept_prob || !d_divergent || !d_inverse_mass || !out)
        return fail(UT_ERR_ARGUMENT, "null ChEES buffer");
    if (!ws->d_out) {  // keyed on the last buffer made
        if ((rc = dalloc(ws, &ws->d_flags, ws->C))) return rc;
        if ((rc = dalloc(ws, &ws->d_means, 2 * (size_t)ws->P))) return rc;
        if ((rc = dalloc(ws, &ws->d_terms, 2 * (size_t)ws->C))) return rc;
        if ((rc = dalloc(ws, &ws->d_out, 2))) return rc;
    }
    CheesArgs a;
    a.initials = d_initials; a.proposals = d_proposals; a.momenta = d_endpoint_momentum;
    a.accept = d_accept_prob; a.divergent = d_divergent; a.inverse_mass = d_inverse_mass;
    a.flags = ws->d_flags; a.means = ws->d_means; a.chain_terms = ws->d_terms; a.out = ws->d_out;
    a.P = ws->P; a.C = ws->C;
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned gw = (ws->C + 7) / 8;
    chees_flags_kernel<<<gw, 256, 0, st>>>(a);
    chees_means_kernel<<<ws->P, 256, 0, st>>>(a);
    chees_terms_kernel<<<gw, 256, 0, st>>>(a);
    chees_final_kernel<<<1, 256, 0, st>>>(a);
    UT_LAUNCHED();
    UT_CUDA(cudaMemcpyAsync(out, ws->d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    UT_CUDA(cudaStreamSynchronize(st));
    return UT_OK;
}

// ---- warmup adaptation ----------------------------------------------------
int32_t ut_running_variance_update(const float* d_positions, const double* d_weights, int32_t num_params,
                                   int32_t num_chains, double* d_state, int32_t window_length, void* stream) {
    if (!d_positions || !d_weights || !d_state) return fail(UT_ERR_ARGUMENT, "null running-variance buffer");
    if (num_params < 1 || num_params > 1024) return fail(UT_ERR_ARGUMENT, "num_params must be in 1..1024, got %d", (int)num_params);
    if (num_chains < 0) return fail(UT_ERR_ARGUMENT, "num_chains must be >= 0");
    if (window_length < 1) return fail(UT_ERR_ARGUMENT, "running variance state requires window_length > 0");
    if (num_chains == 0) return UT_OK;
    int threads = ((num_params + 31) / 32) * 32;
    size_t smem = (size_t)32 * num_params * sizeof(float);
    UT_CUDA(allow_dynamic_smem(running_variance_kernel, smem));
    running_variance_kernel<<<1, threads, smem, (cudaStream_t)stream>>>(d_positions, d_weights, num_params, num_chains,
                                                                      d_state, window_length);
    UT_LAUNCHED();
    return UT_OK;
}

int32_t ut_warmup_adapt(const float* d_accept_prob, const uint8_t* d_accepted, const uint8_t* d_divergent,
                        int32_t num_chains, int32_t num_params, const double* d_variance_state,
                        int32_t window_length, double* d_weights, double* d_dual, int32_t per_chain,
                        int32_t adapt_step, double target_accept, float* d_step, void* stream) {
    if (!d_accept_prob || !d_divergent) return fail(UT_ERR_ARGUMENT, "null accept / divergence buffer");
    if (num_chains < 1) return fail(UT_ERR_ARGUMENT, "num_chains must be >= 1, got %d", (int)num_chains);
    if (d_weights && (!d_variance_state || num_params < 1 || window_length < 1))
        return fail(UT_ERR_ARGUMENT, "weights need the running-variance state, num_params and window_length");
    if (adapt_step && (!d_dual || !d_step)) return fail(UT_ERR_ARGUMENT, "null dual-averaging state or step buffer");
    if (!(target_accept > 0.0 && target_accept < 1.0)) return fail(UT_ERR_ARGUMENT, "target_accept must be in (0, 1)");
    warmup_adapt_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(d_accept_prob, d_accepted, d_divergent, num_chains,
                                                              num_params, d_weights ? d_variance_state : nullptr,
                                                              window_length, d_weights, d_dual, per_chain ? 1 : 0,
                                                              adapt_step ? 1 : 0, target_accept, d_step);
    UT_LAUNCHED();
    return UT_OK;
}

int32_t ut_dual_averaging_final(const double* d_dual, int32_t num_chains, int32_t per_chain, float* d_step,
                                void* stream) {
    if (!d_dual || !d_step) return fail(UT_ERR_ARGUMENT, "null dual-averaging state or step buffer");
    if (num_chains < 1) return fail(UT_ERR_ARGUMENT, "num_chains must be >= 1, got %d", (int)num_chains);
    dual_averaging_final_kernel<<<(num_chains + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_dual, num_chains,
                                                                                           per_chain ? 1 : 0, d_step);
    UT_LAUNCHED();
    return UT_OK;
}

}  // extern "C"
