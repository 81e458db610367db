// ut_surrogate.cu -- the learned gradient surrogate object: FP32 master
// weights, Adam moments, BF16 weight copies, input/output normalisation, and
// the entry points that initialise, normalise, train and evaluate it.  The
// kernels are in ut_mlp.cuh; the surrogate-driven HMC iteration that uses it
// is in ut_api.cu (it needs the workspace's batched density).
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/ut_b200.h"
#include "ut_mlp.cuh"
#include "ut_mlp_tc.cuh"

using namespace ut;

// Defined in ut_api.cu: stores the message that ut_last_error returns.
void ut_internal_set_last_error(const char* msg);

struct ut_surrogate {
    int P = 0;
    MlpLayout L;
    int device = 0;
    float* params = nullptr;   // FP32 master weights (L.total)
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    MlpBf16 wb = {};
    float* norm = nullptr;     // in_mean, in_scale, out_mean, out_scale (P each)
    float* partial = nullptr;  // parts x L.total
    float* part_loss = nullptr;
    int parts_capacity = 0;
    float* loss = nullptr;     // device scalar: loss of the last batch
    int* bad_index = nullptr;
    double* stats = nullptr;   // 2 x kStatChunks x P
    long long adam_step = 0;
    float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    // forward on the tcgen05 tensor cores (mlp_forward_tc_kernel): TMA maps of the BF16 weights
    bool tc = false;
    CUtensorMap map_w1, map_w2, map_w3;
    int* tc_err = nullptr;     // sticky error word of the tcgen05 forward (a bounded wait gave up)
    std::vector<void*> allocations;
};

namespace {

constexpr int kStatChunks = 512;

int32_t sfail(int32_t code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ut_internal_set_last_error(buf);
    return code;
}

#define US_CUDA(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return sfail(UT_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

#define US_LAUNCHED()                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = cudaGetLastError();                                                            \
        if (e_ != cudaSuccess) return sfail(UT_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e_)); \
    } while (0)

template <class T>
int32_t salloc(ut_surrogate* s, T** p, size_t count) {
    void* v = nullptr;
    cudaError_t e = cudaMalloc(&v, (count ? count : 1) * sizeof(T));
    if (e != cudaSuccess)
        return sfail(UT_ERR_CUDA, "cudaMalloc(%zu bytes) failed: %s", count * sizeof(T), cudaGetErrorString(e));
    s->allocations.push_back(v);
    *p = static_cast<T*>(v);
    return UT_OK;
}

void release(ut_surrogate* s) {
    for (void* p : s->allocations) cudaFree(p);
    s->allocations.clear();
}

MlpNorm norm_of(const ut_surrogate* s) {
    MlpNorm n;
    n.in_mean = s->norm;
    n.in_scale = s->norm + s->P;
    n.out_mean = s->norm + 2 * s->P;
    n.out_scale = s->norm + 3 * s->P;
    return n;
}

int32_t refresh_bf16(ut_surrogate* s, cudaStream_t st) {
    const int n = kMlpH * kMlpH;  // >= H * Pp since Pp <= 128 < H
    mlp_refresh_bf16_kernel<<<(n + 255) / 256, 256, 0, st>>>(s->params, s->wb, s->P);
    US_LAUNCHED();
    return UT_OK;
}

int32_t ensure_parts(ut_surrogate* s, int parts) {
    if (parts <= s->parts_capacity) return UT_OK;
    if (s->partial) {  // drop the old buffers (they are the last two allocations made for them)
        for (auto it = s->allocations.begin(); it != s->allocations.end();) {
            if (*it == s->partial || *it == s->part_loss) {
                cudaFree(*it);
                it = s->allocations.erase(it);
            } else {
                ++it;
            }
        }
        s->partial = nullptr;
        s->part_loss = nullptr;
        s->parts_capacity = 0;
    }
    int32_t rc;
    if ((rc = salloc(s, &s->partial, (size_t)parts * s->L.total))) return rc;
    if ((rc = salloc(s, &s->part_loss, (size_t)parts))) return rc;
    s->parts_capacity = parts;
    return UT_OK;
}

int32_t set_smem(const void* fn, size_t bytes) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return sfail(UT_ERR_CUDA, "shared-memory opt-in failed: %s", cudaGetErrorString(e));
    return UT_OK;
}

int32_t check_surrogate(const ut_surrogate* s) {
    if (!s) return sfail(UT_ERR_ARGUMENT, "null surrogate handle");
    return UT_OK;
}

// One forward + backward over `batch` pairs (rows from index, or drawn from
// Philox(seed, step) when index is NULL), folded into grad_out and/or an Adam step.
int32_t train_pass(ut_surrogate* s, const float* theta, const float* grad, long long n, const int32_t* index,
                   int batch, uint32_t seed, uint32_t step, float lr, bool adam, float* grad_out, float* loss_out,
                   cudaStream_t st) {
    const int parts = (batch + kMlpRows - 1) / kMlpRows;
    int32_t rc;
    if ((rc = ensure_parts(s, parts))) return rc;
    MlpTrainArgs a;
    a.params = s->params; a.wb = s->wb; a.nm = norm_of(s);
    a.x = theta; a.t = grad; a.n = n; a.index = index; a.seed = seed; a.step = step;
    a.batch = batch; a.P = s->P; a.partial = s->partial; a.partial_loss = s->part_loss;
    a.bad_index = s->bad_index;
    mlp_train_kernel<<<parts, kMlpThreads, mlp_train_smem(s->L.Pp), st>>>(a);
    US_LAUNCHED();
    float bc1 = 1.0f, bc2 = 1.0f;
    if (adam) {
        s->adam_step += 1;
        bc1 = (float)(1.0 / (1.0 - std::pow((double)s->beta1, (double)s->adam_step)));
        bc2 = (float)(1.0 / (1.0 - std::pow((double)s->beta2, (double)s->adam_step)));
    }
    const long long total = (long long)s->L.total;
    mlp_reduce_adam_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
        s->params, s->adam_m, s->adam_v, s->partial, parts, total, grad_out, s->part_loss,
        loss_out ? loss_out : s->loss, lr, s->beta1, s->beta2, s->eps, bc1, bc2, adam ? 1 : 0);
    US_LAUNCHED();
    if (adam) return refresh_bf16(s, st);
    return UT_OK;
}

int32_t check_pairs(const ut_surrogate* s, const float* theta, const float* grad, int64_t num_pairs, int32_t batch) {
    if (!theta || !grad) return sfail(UT_ERR_ARGUMENT, "null pair buffer");
    if (num_pairs < 1) return sfail(UT_ERR_ARGUMENT, "num_pairs must be >= 1, got %lld", (long long)num_pairs);
    if (batch < 1 || batch > 65536) return sfail(UT_ERR_ARGUMENT, "batch must be in 1..65536, got %d", (int)batch);
    (void)s;
    return UT_OK;
}

}  // namespace

// Internal entry used by the surrogate-driven HMC iteration in ut_api.cu.
int ut_internal_surrogate_num_params(const ut_surrogate* s) { return s ? s->P : 0; }

int32_t ut_internal_surrogate_forward(const ut_surrogate* s, const float* x, int64_t n, float* out, cudaStream_t st) {
    if (n <= 0) return UT_OK;
    if (s->tc) {
        const long long tblocks = (n + kMtRows - 1) / kMtRows;
        if (tblocks > 0x7fffffffLL) return sfail(UT_ERR_ARGUMENT, "too many rows for one surrogate evaluation");
        MlpTcArgs a;
        a.params = s->params; a.nm = norm_of(s); a.P = s->P; a.Pp = s->L.Pp; a.x = x; a.n = n; a.out = out;
        a.err = s->tc_err;
        mlp_forward_tc_kernel<<<(unsigned)tblocks, kMtThreads, mlp_tc_smem(s->L.Pp), st>>>(s->map_w1, s->map_w2,
                                                                                         s->map_w3, a);
        US_LAUNCHED();
        return UT_OK;
    }
    const long long blocks = (n + kMlpRows - 1) / kMlpRows;
    if (blocks > 0x7fffffffLL) return sfail(UT_ERR_ARGUMENT, "too many rows for one surrogate evaluation");
    mlp_forward_kernel<<<(unsigned)blocks, kMlpThreads, mlp_forward_smem(s->L.Pp), st>>>(s->params, s->wb,
                                                                                      norm_of(s), s->P, x, n, out);
    US_LAUNCHED();
    return UT_OK;
}

extern "C" {

int32_t ut_surrogate_create(int32_t num_params, uint32_t seed, ut_surrogate** out) {
    if (!out) return sfail(UT_ERR_ARGUMENT, "null output handle");
    *out = nullptr;
    if (num_params < 1 || num_params > kMlpMaxP)
        return sfail(UT_ERR_ARGUMENT, "the surrogate supports 1..%d parameters, got %d", kMlpMaxP, (int)num_params);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return sfail(UT_ERR_NO_DEVICE, "no CUDA device visible");
    }
    ut_surrogate* s = new ut_surrogate();
    s->P = num_params;
    s->L = MlpLayout::make(num_params);
    cudaGetDevice(&s->device);
    int32_t rc = UT_OK;
    const size_t total = s->L.total, Pp = s->L.Pp;
    __nv_bfloat16* bf = nullptr;
    const size_t nbf = 2 * (size_t)kMlpH * Pp + 2 * (size_t)kMlpH * kMlpH + (size_t)kMlpH * Pp;
    if ((rc = salloc(s, &s->params, total)) || (rc = salloc(s, &s->adam_m, total)) ||
        (rc = salloc(s, &s->adam_v, total)) || (rc = salloc(s, &bf, nbf)) || (rc = salloc(s, &s->norm, 4 * (size_t)num_params)) ||
        (rc = salloc(s, &s->loss, 1)) || (rc = salloc(s, &s->bad_index, 1)) ||
        (rc = salloc(s, &s->stats, 2 * (size_t)kStatChunks * num_params))) {
        release(s);
        delete s;
        return rc;
    }
    s->wb.w1 = bf;
    s->wb.w2 = s->wb.w1 + (size_t)kMlpH * Pp;
    s->wb.w2t = s->wb.w2 + (size_t)kMlpH * kMlpH;
    s->wb.w3 = s->wb.w2t + (size_t)kMlpH * kMlpH;
    s->wb.w3t = s->wb.w3 + Pp * kMlpH;
    {   // UT_MLP_TC=1: the forward pass on the tcgen05 tensor cores (128 rows per CTA).  The
        // warp-level kernel (32 rows per CTA) stays the default: at a few thousand rows it
        // spreads over 4x as many SMs and measured faster (27 vs 52 us for 4096 rows).
        int major = 0;
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, s->device);
        const char* want_tc = getenv("UT_MLP_TC");
        if (major == 10 && want_tc && want_tc[0] == '1' && (rc = salloc(s, &s->tc_err, 1)) == UT_OK &&
            cudaMemset(s->tc_err, 0, sizeof(int)) == cudaSuccess &&
            mlp_tc_make_map(&s->map_w1, s->wb.w1, kMlpH, (int)Pp, kMlpH) &&
            mlp_tc_make_map(&s->map_w2, s->wb.w2, kMlpH, kMlpH, kMlpH) &&
            mlp_tc_make_map(&s->map_w3, s->wb.w3, (int)Pp, kMlpH, (int)Pp) &&
            set_smem((const void*)mlp_forward_tc_kernel, mlp_tc_smem(kMlpMaxP)) == UT_OK)
            s->tc = true;
        if (rc) {
            release(s);
            delete s;
            return rc;
        }
    }
    auto fail_out = [&](int32_t code) {
        release(s);
        delete s;
        return code;
    };
    // opt in to the largest width's shared memory, so surrogates of any width can coexist
    if ((rc = set_smem((const void*)mlp_train_kernel, mlp_train_smem(kMlpMaxP)))) return fail_out(rc);
    if ((rc = set_smem((const void*)mlp_forward_kernel, mlp_forward_smem(kMlpMaxP)))) return fail_out(rc);
    std::vector<float> nrm(4 * (size_t)num_params, 0.0f);
    for (int j = 0; j < num_params; ++j) {
        nrm[num_params + j] = 1.0f;
        nrm[3 * num_params + j] = 1.0f;
    }
    if (cudaMemcpy(s->norm, nrm.data(), nrm.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(s->adam_m, 0, total * sizeof(float)) != cudaSuccess ||
        cudaMemset(s->adam_v, 0, total * sizeof(float)) != cudaSuccess ||
        cudaMemset(s->bad_index, 0, sizeof(int)) != cudaSuccess || cudaMemset(s->loss, 0, sizeof(float)) != cudaSuccess) {
        rc = sfail(UT_ERR_CUDA, "surrogate initialisation copy failed: %s", cudaGetErrorString(cudaGetLastError()));
        return fail_out(rc);
    }
    mlp_init_kernel<<<(unsigned)((total + 255) / 256), 256>>>(s->params, num_params, seed);
    if (cudaGetLastError() != cudaSuccess) return fail_out(sfail(UT_ERR_CUDA, "surrogate init launch failed"));
    if ((rc = refresh_bf16(s, nullptr))) return fail_out(rc);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail_out(sfail(UT_ERR_CUDA, "surrogate initialisation failed: %s", cudaGetErrorString(e)));
    *out = s;
    return UT_OK;
}

int32_t ut_surrogate_destroy(ut_surrogate* s) {
    if (!s) return UT_OK;
    cudaDeviceSynchronize();
    release(s);
    delete s;
    return UT_OK;
}

int32_t ut_surrogate_num_weights(const ut_surrogate* s, int64_t* out) {
    int32_t rc = check_surrogate(s);
    if (rc) return rc;
    if (!out) return sfail(UT_ERR_ARGUMENT, "null output");
    *out = (int64_t)s->L.total;
    return UT_OK;
}

int32_t ut_surrogate_get_weights(const ut_surrogate* s, float* out, int64_t n) {
    int32_t rc = check_surrogate(s);
    if (rc) return rc;
    if (!out) return sfail(UT_ERR_ARGUMENT, "null output");
    if (n != (int64_t)s->L.total)
        return sfail(UT_ERR_DIMENSION, "expected %zu weights, got %lld", s->L.total, (long long)n);
    US_CUDA(cudaDeviceSynchronize());
    US_CUDA(cudaMemcpy(out, s->params, s->L.total * sizeof(float), cudaMemcpyDeviceToHost));
    return UT_OK;
}

int32_t ut_surrogate_set_weights(ut_surrogate* s, const float* in, int64_t n) {
    int32_t rc = check_surrogate(s);
    if (rc) return rc;
    if (!in) return sfail(UT_ERR_ARGUMENT, "null input");
    if (n != (int64_t)s->L.total)
        return sfail(UT_ERR_DIMENSION, "expected %zu weights, got %lld", s->L.total, (long long)n);
    // padded rows / columns must stay zero
    const MlpLayout& L = s->L;
    for (int r = 0; r < kMlpH; ++r)
        for (int c = s->P; c < L.Pp; ++c)
            if (in[L.w1 + (size_t)r * L.Pp + c] != 0.0f || in[L.w3 + (size_t)c * kMlpH + r] != 0.0f)
                return sfail(UT_ERR_ARGUMENT, "padded weight entries (index >= num_params) must be zero");
    for (int c = s->P; c < L.Pp; ++c)
        if (in[L.b3 + c] != 0.0f) return sfail(UT_ERR_ARGUMENT, "padded bias entries must be zero");
    for (size_t i = 0; i < L.total; ++i)
        if (!std::isfinite(in[i])) return sfail(UT_ERR_ARGUMENT, "weights must be finite");
    US_CUDA(cudaDeviceSynchronize());
    US_CUDA(cudaMemcpy(s->params, in, L.total * sizeof(float), cudaMemcpyHostToDevice));
    US_CUDA(cudaMemset(s->adam_m, 0, L.total * sizeof(float)));
    US_CUDA(cudaMemset(s->adam_v, 0, L.total * sizeof(float)));
    s->adam_step = 0;
    if ((rc = refresh_bf16(s, nullptr))) return rc;
    US_CUDA(cudaDeviceSynchronize());
    return UT_OK;
}

int32_t ut_surrogate_get_normalization(const ut_surrogate* s, float* out) {
    int32_t rc = check_surrogate(s);
    if (rc) return rc;
    if (!out) return sfail(UT_ERR_ARGUMENT, "null output");
    US_CUDA(cudaDeviceSynchronize());
    US_CUDA(cudaMemcpy(out, s->norm, 4 * (size_t)s->P * sizeof(float), cudaMemcpyDeviceToHost));
    return UT_OK;
}

int32_t ut_surrogate_set_normalization(ut_surrogate* s, const float* in) {
    int32_t rc = check_surrogate(s);
    if (rc) return rc;
    if (!in) return sfail(UT_ERR_ARGUMENT, "null input");
    for (int k = 0; k < 4 * s->P; ++k)
        if (!std::isfinite(in[k])) return sfail(UT_ERR_ARGUMENT, "normalisation entries must be finite");
    for (int j = 0; j < s->P; ++j)
        if (!(in[s->P + j] > 0.0f) || !(in[3 * s->P + j] > 0.0f))
            return sfail(UT_ERR_ARGUMENT, "normalisation scales must be > 0");
    US_CUDA(cudaDeviceSynchronize());
    US_CUDA(cudaMemcpy(s->norm, in, 4 * (size_t)s->P * sizeof(float), cudaMemcpyHostToDevice));
    return UT_OK;
}

int32_t ut_surrogate_fit_normalization(ut_surrogate* s, const float* d_theta, const float* d_gradient,
                                       int64_t num_pairs, void* stream) {
    int32_t rc = check_surrogate(s);
    if (rc) return rc;
    if (!d_theta || !d_gradient) return sfail(UT_ERR_ARGUMENT, "null pair buffer");
    if (num_pairs < 2) return sfail(UT_ERR_ARGUMENT, "fitting the normalisation needs >= 2 pairs, got %lld", (long long)num_pairs);
    cudaStream_t st = (cudaStream_t)stream;
    const long long chunk = (num_pairs + kStatChunks - 1) / kStatChunks;
    const int chunks = (int)((num_pairs + chunk - 1) / chunk);
    const int P = s->P;
    double* psum = s->stats;
    double* psq = s->stats + (size_t)kStatChunks * P;
    const float* src[2] = {d_theta, d_gradient};
    for (int k = 0; k < 2; ++k) {
        mlp_stats_partial_kernel<<<chunks, kMlpMaxP, 0, st>>>(src[k], num_pairs, P, chunk, psum, psq);
        US_LAUNCHED();
        mlp_stats_final_kernel<<<1, kMlpMaxP, 0, st>>>(psum, psq, chunks, num_pairs, P, s->norm + 2 * k * P,
                                                       s->norm + (2 * k + 1) * P);
        US_LAUNCHED();
    }
    return UT_OK;
}

int32_t ut_surrogate_train(ut_surrogate* s, const float* d_theta, const float* d_gradient, int64_t num_pairs,
                           const int32_t* d_batch_index, int32_t batch, int32_t num_steps, float learning_rate,
                           float final_learning_rate, uint32_t seed, float* d_losses, void* stream) {
    int32_t rc = check_surrogate(s);
    if (rc) return rc;
    if ((rc = check_pairs(s, d_theta, d_gradient, num_pairs, batch))) return rc;
    if (num_steps < 1) return sfail(UT_ERR_ARGUMENT, "num_steps must be >= 1, got %d", (int)num_steps);
    if (!(learning_rate > 0.0f) || !(final_learning_rate > 0.0f) || !std::isfinite(learning_rate) ||
        !std::isfinite(final_learning_rate))
        return sfail(UT_ERR_ARGUMENT, "learning rates must be finite and > 0");
    cudaStream_t st = (cudaStream_t)stream;
    for (int k = 0; k < num_steps; ++k) {
        // geometric interpolation from learning_rate to final_learning_rate
        const double f = num_steps > 1 ? (double)k / (double)(num_steps - 1) : 0.0;
        const float lr = (float)(learning_rate * std::pow((double)final_learning_rate / learning_rate, f));
        const int32_t* idx = d_batch_index ? d_batch_index + (size_t)k * batch : nullptr;
        if ((rc = train_pass(s, d_theta, d_gradient, num_pairs, idx, batch, seed, (uint32_t)s->adam_step, lr, true,
                             nullptr, d_losses ? d_losses + k : nullptr, st)))
            return rc;
    }
    return UT_OK;
}

int32_t ut_surrogate_loss_gradient(ut_surrogate* s, const float* d_theta, const float* d_gradient, int64_t num_pairs,
                                   const int32_t* d_batch_index, int32_t batch, float* d_weight_gradient,
                                   float* d_loss, void* stream) {
    int32_t rc = check_surrogate(s);
    if (rc) return rc;
    if ((rc = check_pairs(s, d_theta, d_gradient, num_pairs, batch))) return rc;
    if (!d_batch_index || !d_weight_gradient || !d_loss) return sfail(UT_ERR_ARGUMENT, "null buffer");
    return train_pass(s, d_theta, d_gradient, num_pairs, d_batch_index, batch, 0u, 0u, 0.0f, false, d_weight_gradient,
                      d_loss, (cudaStream_t)stream);
}

int32_t ut_surrogate_gradient(const ut_surrogate* s, const float* d_theta, int64_t n, float* d_out, void* stream) {
    int32_t rc = check_surrogate(s);
    if (rc) return rc;
    if (!d_theta || !d_out) return sfail(UT_ERR_ARGUMENT, "null buffer");
    if (n < 0) return sfail(UT_ERR_ARGUMENT, "n must be >= 0");
    return ut_internal_surrogate_forward(s, d_theta, n, d_out, (cudaStream_t)stream);
}

int32_t ut_surrogate_check(ut_surrogate* s, void* stream) {
    int32_t rc = check_surrogate(s);
    if (rc) return rc;
    int bad = 0;
    cudaStream_t st = (cudaStream_t)stream;
    US_CUDA(cudaMemcpyAsync(&bad, s->bad_index, sizeof(int), cudaMemcpyDeviceToHost, st));
    US_CUDA(cudaStreamSynchronize(st));
    if (bad) {
        US_CUDA(cudaMemsetAsync(s->bad_index, 0, sizeof(int), st));
        US_CUDA(cudaStreamSynchronize(st));
        return sfail(UT_ERR_ARGUMENT, "a batch index was outside [0, num_pairs); those rows were skipped");
    }
    if (s->tc_err) {
        int terr = 0;
        US_CUDA(cudaMemcpyAsync(&terr, s->tc_err, sizeof(int), cudaMemcpyDeviceToHost, st));
        US_CUDA(cudaStreamSynchronize(st));
        if (terr) {
            US_CUDA(cudaMemsetAsync(s->tc_err, 0, sizeof(int), st));
            US_CUDA(cudaStreamSynchronize(st));
            return sfail(UT_ERR_DEVICE_TIMEOUT, "a bounded wait inside the tensor-core surrogate forward gave up; "
                                                "its results are invalid");
        }
    }
    return UT_OK;
}

}  // extern "C"
