// ut_advi.cuh -- device pieces of mean-field ADVI (reference device loop
// _run_device_batched_advi, src/device/advi_kernels.jl:45-209; reduction
// _device_advi_reduce!, :15-38; host semantics src/inference/vi.jl:314-520).
//
// One step for M particles and P unconstrained parameters:
//   eps[j, p]       = standard normal from Philox at (j, coord, kStreamAdvi, p)
//   particle[j, p]  = location[p] + scale[p] * eps[j, p]
//   (batched logjoint + gradient of the particles, the workspace's kernel)
//   loc_grad[p]     = mean_j grad[j, p]
//   scale_grad[p]   = mean_j grad[j, p] * scale[p] * eps[j, p]
// The reference draws eps on the host; here it comes from the device Philox
// stream (a replayable coordinate), and the reduction regenerates eps instead
// of reading a stored P x M noise matrix.  Sums over particles run in a fixed
// order (deterministic).
#pragma once

#include "ut_common.cuh"

namespace ut {

constexpr uint32_t kStreamAdvi = 5;

__global__ void advi_particles_kernel(const float* __restrict__ loc, const float* __restrict__ scale, uint32_t coord,
                                      int P, int M, float* __restrict__ particles) {
    const long long n = (long long)P * M;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(i / P), p = (int)(i % P);
        const float eps = rand_normal((uint32_t)j, coord, kStreamAdvi, (uint32_t)p);
        particles[i] = fmaf(scale[p], eps, loc[p]);
    }
}

// One CTA per parameter: thread t adds particles t, t + 256, ... in order, then
// a fixed tree over the 256 partial sums.
__global__ void __launch_bounds__(256) advi_reduce_kernel(const float* __restrict__ grads,
                                                          const float* __restrict__ scale, uint32_t coord, int P,
                                                          int M, float* __restrict__ loc_grad,
                                                          float* __restrict__ scale_grad) {
    __shared__ float sa[256], sb[256];
    const int p = blockIdx.x, t = threadIdx.x;
    const float s = scale[p];
    float a = 0.0f, b = 0.0f;
    for (int j = t; j < M; j += 256) {
        const float g = grads[(size_t)j * P + p];
        const float eps = rand_normal((uint32_t)j, coord, kStreamAdvi, (uint32_t)p);
        a += g;
        b += g * s * eps;
    }
    sa[t] = a;
    sb[t] = b;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w) {
            sa[t] += sa[t + w];
            sb[t] += sb[t + w];
        }
        __syncthreads();
    }
    if (t == 0) {
        const float inv = 1.0f / (float)M;
        loc_grad[p] = sa[0] * inv;
        scale_grad[p] = sb[0] * inv;
    }
}

}  // namespace ut
