// ut_noalloc.cu -- Bernoulli-logit GLM logjoint + gradient that allocates no
// device memory.
//
// Some callers cannot call cudaMalloc / cudaFree at the moment they need a
// gradient: a host that owns all device memory through its own pool or
// allocator and forbids allocations after start-up (a serving process with a
// fixed memory budget, a Julia host whose GPU arrays all come from its own
// pool), or a latency-critical loop where the device-wide synchronisation that
// cudaMalloc / cudaFree can imply is not acceptable.  For them this file
// provides one entry point that takes every input and output as device
// pointers from the caller and keeps its only scratch memory -- the per-split
// partial sums of the observation-tiled CUDA-core kernel -- in a fixed,
// file-scope device array instead of allocating it.
//
// The scratch array (kNoAllocScratchFloats floats, 16 MiB) is held by every GPU
// that loads the library until the process exits.  All calls share it and it
// keeps the last call's contents; nothing in it has to start at zero (every
// partial the fold reads is written first by the same call).  Calls whose
// kernels overlap on the GPU (concurrent streams, threads or devices sharing a
// context) race on the array: serialise them.
#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <cuda_runtime.h>

#include "../../include/ut_b200.h"

namespace {  // the kernels below are private to this file
#include "ut_glm_tiled.cuh"
}

namespace {

constexpr size_t kNoAllocScratchFloats = 4u * 1024u * 1024u;  // 16 MiB
constexpr int kMaxDevices = 64;

// The scratch memory.  In host code this name is only a host-side stand-in for
// the device symbol; the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

std::mutex g_setup_mutex;
float* g_scratch_ptr[kMaxDevices] = {nullptr};
int g_sms[kMaxDevices] = {0};

}  // namespace

// Defined in ut_api.cu: stores the message that ut_last_error returns.
void ut_internal_set_last_error(const char* msg);

namespace {

int32_t noalloc_fail(int32_t code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ut_internal_set_last_error(buf);
    return code;
}

size_t tiled_smem(int F) {
    return sizeof(float) * ((size_t)F * ut::kGlmCT + (size_t)F * ut::kGlmXS + (size_t)ut::kGlmOT * ut::kGlmRS +
                            ut::kGlmOT + 16 * ut::kGlmCT);
}

template <class K>
cudaError_t opt_in(K kern, size_t smem) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// Once per device, with that device current: resolve the scratch array's device
// address and opt the kernel instantiations in to their shared-memory size.
// Done by the first call on each device.
int32_t setup_device(int dev, float** scratch, int* sms) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(UT_ERR_ARGUMENT, "device ordinal %d out of range", dev);
    if (!g_scratch_ptr[dev]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess)
            return noalloc_fail(UT_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess)
            return noalloc_fail(UT_ERR_CUDA, "cudaDeviceGetAttribute failed: %s", cudaGetErrorString(e));
        const size_t smem = tiled_smem(ut::kGlmMaxF);
        if ((e = opt_in(ut::glm_tiled_kernel<true, 1>, smem)) != cudaSuccess ||
            (e = opt_in(ut::glm_tiled_kernel<true, 2>, smem)) != cudaSuccess ||
            (e = opt_in(ut::glm_tiled_kernel<true, 4>, smem)) != cudaSuccess ||
            (e = opt_in(ut::glm_tiled_kernel<true, 8>, smem)) != cudaSuccess ||
            (e = opt_in(ut::glm_tiled_kernel<true, 16>, smem)) != cudaSuccess)
            return noalloc_fail(UT_ERR_CUDA, "shared-memory opt-in failed: %s", cudaGetErrorString(e));
        g_sms[dev] = n;
        g_scratch_ptr[dev] = static_cast<float*>(ptr);
    }
    *scratch = g_scratch_ptr[dev];
    *sms = g_sms[dev];
    return UT_OK;
}

}  // namespace

extern "C" int32_t ut_glm_logjoint_gradient_noalloc(const float* d_design, const float* d_y, int64_t num_obs,
                                                   int32_t num_params, int32_t has_intercept, double intercept_mu,
                                                   double intercept_sigma, double coef_mu, double coef_sigma,
                                                   const float* d_params, int32_t num_chains, float* d_totals,
                                                   float* d_gradients, void* stream) {
    if (!d_design || !d_y || !d_params || !d_totals || !d_gradients)
        return noalloc_fail(UT_ERR_ARGUMENT, "null device buffer");
    if (num_params < 1 || num_params > ut::kGlmMaxF)
        return noalloc_fail(UT_ERR_ARGUMENT, "num_params must be in 1..%d, got %d", ut::kGlmMaxF, (int)num_params);
    if (has_intercept != 0 && has_intercept != 1) return noalloc_fail(UT_ERR_ARGUMENT, "has_intercept must be 0 or 1");
    if (num_obs < 1 || num_obs > UT_MAX_OBS) return noalloc_fail(UT_ERR_ARGUMENT, "num_obs must be in 1..2^30");
    if (num_chains < 1) return noalloc_fail(UT_ERR_ARGUMENT, "num_chains must be >= 1, got %d", (int)num_chains);
    if (!(coef_sigma > 0.0) || (has_intercept && !(intercept_sigma > 0.0)))
        return noalloc_fail(UT_ERR_ARGUMENT, "prior scales must be > 0");
    // one split needs C * (P + 1) floats of scratch (log-likelihood + gradient partials)
    const size_t per_split = (size_t)num_chains * ((size_t)num_params + 1);
    if (per_split > kNoAllocScratchFloats)
        return noalloc_fail(UT_ERR_ARGUMENT,
                            "num_chains * (num_params + 1) = %zu exceeds the fixed scratch of %zu floats (16 MiB); "
                            "split the batch or use ut_logjoint_gradient_device",
                            per_split, kNoAllocScratchFloats);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(UT_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    float* scratch = nullptr;
    int sms = 0;
    int32_t rc = setup_device(dev, &scratch, &sms);
    if (rc) return rc;

    // The split plan in 64-bit arithmetic: S observation splits of whole chunks,
    // at most 3 CTAs per SM in all and at most what the scratch holds
    // (S * C * (P + 1) floats).  With N <= 2^30 every value fits the kernels' int.
    const int N = (int)num_obs, F = num_params, C = num_chains;
    const int ctiles = (C + ut::kGlmCT - 1) / ut::kGlmCT;
    const int64_t chunks = (num_obs + ut::kGlmOT - 1) / ut::kGlmOT;
    int64_t S64 = std::max<int64_t>(1, std::min<int64_t>(chunks, (3 * (int64_t)sms + ctiles - 1) / ctiles));
    S64 = std::max<int64_t>(1, std::min<int64_t>(S64, (int64_t)(kNoAllocScratchFloats / per_split)));
    const int64_t per = (chunks + S64 - 1) / S64;
    const int64_t ops64 = per * ut::kGlmOT;
    const int obs_per_split = (int)ops64;
    const int S = (int)((num_obs + ops64 - 1) / ops64);

    ut::GlmTiledArgs a;
    a.Xa = d_design; a.y = d_y; a.params = d_params;
    a.part_ll = scratch;
    a.part_g = scratch + (size_t)S * C;
    a.N = N; a.F = F; a.C = C; a.obs_per_split = obs_per_split;
    const dim3 grid(ctiles, S);
    const size_t smem = tiled_smem(F);
    const int need = (F + 15) / 16;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (need <= 1) ut::glm_tiled_kernel<true, 1><<<grid, 256, smem, st>>>(a);
    else if (need <= 2) ut::glm_tiled_kernel<true, 2><<<grid, 256, smem, st>>>(a);
    else if (need <= 4) ut::glm_tiled_kernel<true, 4><<<grid, 256, smem, st>>>(a);
    else if (need <= 8) ut::glm_tiled_kernel<true, 8><<<grid, 256, smem, st>>>(a);
    else ut::glm_tiled_kernel<true, 16><<<grid, 256, smem, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return noalloc_fail(UT_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));

    ut::GlmReduceArgs r;
    r.params = d_params; r.part_ll = a.part_ll; r.part_g = a.part_g;
    r.totals = d_totals; r.grads = d_gradients;
    r.S = S; r.C = C; r.F = F; r.off = has_intercept;
    r.icpt_mu = (float)intercept_mu; r.icpt_sigma = (float)intercept_sigma;
    r.coef_mu = (float)coef_mu; r.coef_sigma = (float)coef_sigma;
    ut::glm_reduce_kernel<<<(C + 7) / 8, 256, 0, st>>>(r);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return noalloc_fail(UT_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
    return UT_OK;
}
