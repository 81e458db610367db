// ut_mlp.cuh -- the learned gradient surrogate: an MLP  P -> H -> H -> P
// (SiLU hidden layers, H = 256) that maps an unconstrained position theta to
// the logjoint gradient.  FP32 master weights, BF16 matmul operands with FP32
// accumulation on the tensor cores through warp-level mma.sync m16n8k16 (each
// CTA multiplies 32 rows by at most 256 x 256 weights: tiles this small are
// latency-bound and too small to feed tcgen05), hand-written forward, backward
// and Adam kernels.
//
// Every GEMM is arranged as C[m][n] = sum_k A[m][k] * Bt[n][k] with both
// operands contiguous in k, so one fragment loader serves all of them:
//   forward  L1: A = x (s x in),     Bt = W1 (h x in)
//            L2: A = a1 (s x h),     Bt = W2 (h x h)
//            L3: A = a2 (s x h),     Bt = W3 (out x h)
//   backward dA2 = dY W3:   A = dY (s x out),   Bt = W3^T (h x out)
//            dA1 = dZ2 W2:  A = dZ2 (s x h),    Bt = W2^T (h x h)
//            dW3 = dY^T a2: A = dY^T (out x s), Bt = a2^T (h x s)
//            dW2 = dZ2^T a1, dW1 = dZ1^T x      (likewise)
// The transposed activations are written to shared memory when they are
// produced; W2^T and W3^T are kept as BF16 copies in global memory.
//
// Rounding points (the oracle's MLP restatement follows the same ones):
//   xb  = bf16((theta - in_mean) / in_scale)
//   z1  = xb W1b^T + b1;   a1b = bf16(silu(z1));  s1b = bf16(silu'(z1))
//   z2  = a1b W2b^T + b2;  a2b = bf16(silu(z2));  s2b = bf16(silu'(z2))
//   y   = a2b W3b^T + b3   (FP32);  output = y * out_scale + out_mean
//   t   = (g - out_mean) / out_scale;  loss = sum_rows sum_j (y - t)^2 / B
//   dyb = bf16(2 (y - t) / B)
//   dz2b = bf16((dyb W3b) * s2b);  dz1b = bf16((dz2b W2b) * s1b)
//   dW3 = dyb^T a2b, dW2 = dz2b^T a1b, dW1 = dz1b^T xb, db = column sums of dyb / dz2b / dz1b
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

#include "ut_common.cuh"

namespace ut {

constexpr int kMlpH = 256;        // hidden width
constexpr int kMlpMaxP = 128;     // input/output width (padded to a multiple of 16)
constexpr int kMlpRows = 32;      // samples per CTA
constexpr int kMlpMT = kMlpRows / 16;
constexpr int kMlpThreads = 256;  // 8 warps
constexpr int kMlpPad = 8;        // bf16 row padding of shared arrays (conflict-free fragment loads)

// FP32 parameter layout (one flat array), Pp = P rounded up to 16:
//   W1 [H][Pp]  b1 [H]  W2 [H][H]  b2 [H]  W3 [Pp][H]  b3 [Pp]
// Entries of padded rows/columns (index >= P) are zero and stay zero: their
// gradients are zero because the padded inputs and output errors are.
struct MlpLayout {
    int P, Pp;
    size_t w1, b1, w2, b2, w3, b3, total;
    __host__ __device__ static MlpLayout make(int P) {
        MlpLayout L;
        L.P = P;
        L.Pp = ((P + 15) / 16) * 16;
        L.w1 = 0;
        L.b1 = L.w1 + (size_t)kMlpH * L.Pp;
        L.w2 = L.b1 + kMlpH;
        L.b2 = L.w2 + (size_t)kMlpH * kMlpH;
        L.w3 = L.b2 + kMlpH;
        L.b3 = L.w3 + (size_t)L.Pp * kMlpH;
        L.total = L.b3 + L.Pp;
        return L;
    }
};

// BF16 copies used by the matmuls: W1 [H][Pp], W2 [H][H], W2^T [H][H], W3 [Pp][H], W3^T [H][Pp]
struct MlpBf16 {
    __nv_bfloat16 *w1, *w2, *w2t, *w3, *w3t;
};

// Per-coordinate affine normalisation of inputs and outputs (P entries each).
struct MlpNorm {
    const float *in_mean, *in_scale, *out_mean, *out_scale;
};

__device__ __forceinline__ float silu_f(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float dsilu_f(float z) {
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ uint32_t ld_pair(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// acc[mt][nt] += A[m0+16mt .. +16][0..K) * Bt[n0+8nt .. +8][0..K)^T   (one warp; K % 16 == 0)
// Fragment layout of m16n8k16 (row.col): lane = 4 g + t holds A rows g, g+8 at
// columns 2t, 2t+1, 2t+8, 2t+9 and B^T row g at columns 2t, 2t+1, 2t+8, 2t+9.
template <int MT, int NT>
__device__ __forceinline__ void warp_gemm(float (&acc)[MT][NT][4], const __nv_bfloat16* A, int lda, int m0,
                                          const __nv_bfloat16* Bt, int ldb, int n0, int K) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int k0 = 0; k0 < K; k0 += 16) {
        uint32_t b[NT][2];
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const __nv_bfloat16* bp = Bt + (size_t)(n0 + 8 * nt + g) * ldb + k0 + 2 * t;
            b[nt][0] = ld_pair(bp);
            b[nt][1] = ld_pair(bp + 8);
        }
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const __nv_bfloat16* ap = A + (size_t)(m0 + 16 * mt + g) * lda + k0 + 2 * t;
            const uint32_t a0 = ld_pair(ap), a1 = ld_pair(ap + 8 * lda), a2 = ld_pair(ap + 8),
                           a3 = ld_pair(ap + 8 * lda + 8);
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) mma_bf16(acc[mt][nt], a0, a1, a2, a3, b[nt][0], b[nt][1]);
        }
    }
}

template <int MT, int NT>
__device__ __forceinline__ void zero_acc(float (&acc)[MT][NT][4]) {
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.0f;
}

// Visit one warp's accumulator elements: f(row, col, value).
template <int MT, int NT, class F>
__device__ __forceinline__ void for_acc(const float (&acc)[MT][NT][4], int m0, int n0, F f) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int r = m0 + 16 * mt + g, c = n0 + 8 * nt + 2 * t;
            f(r, c, acc[mt][nt][0]);
            f(r, c + 1, acc[mt][nt][1]);
            f(r + 8, c, acc[mt][nt][2]);
            f(r + 8, c + 1, acc[mt][nt][3]);
        }
}

// One warp's 32-column block of C for rows [m0, m0 + min(rows, 64)), rows a
// multiple of 16; the number of 16-row tiles is picked at run time.
template <class F>
__device__ __forceinline__ void warp_gemm_rows(int rows, const __nv_bfloat16* A, int lda, int m0,
                                               const __nv_bfloat16* Bt, int ldb, int n0, int K, F f) {
    if (rows >= 64) {
        float acc[4][4][4]; zero_acc(acc); warp_gemm<4, 4>(acc, A, lda, m0, Bt, ldb, n0, K); for_acc(acc, m0, n0, f);
    } else if (rows >= 48) {
        float acc[3][4][4]; zero_acc(acc); warp_gemm<3, 4>(acc, A, lda, m0, Bt, ldb, n0, K); for_acc(acc, m0, n0, f);
    } else if (rows >= 32) {
        float acc[2][4][4]; zero_acc(acc); warp_gemm<2, 4>(acc, A, lda, m0, Bt, ldb, n0, K); for_acc(acc, m0, n0, f);
    } else {
        float acc[1][4][4]; zero_acc(acc); warp_gemm<1, 4>(acc, A, lda, m0, Bt, ldb, n0, K); for_acc(acc, m0, n0, f);
    }
}

// Row strides (bf16 elements) of the shared arrays.  Each is 4 (mod 8) words,
// so the 8 rows x 4 words of one fragment load hit 32 different banks.
__host__ __device__ constexpr int mlp_ldp(int Pp) { return Pp + kMlpPad; }
constexpr int kMlpLdh = kMlpH + kMlpPad;
constexpr int kMlpLds = kMlpRows + kMlpPad;

__host__ __device__ inline size_t mlp_forward_smem(int Pp) {
    return ((size_t)kMlpRows * mlp_ldp(Pp) + 2 * (size_t)kMlpRows * kMlpLdh) * sizeof(__nv_bfloat16);
}

// Work region 1 of the training kernel holds a1, later dY and dY^T.
__host__ __device__ inline size_t mlp_wk1_elems(int Pp) {
    const size_t a = (size_t)kMlpRows * kMlpLdh, b = (size_t)kMlpRows * mlp_ldp(Pp) + (size_t)Pp * kMlpLds;
    return a > b ? a : b;
}

__host__ __device__ inline size_t mlp_train_smem(int Pp) {
    const size_t e = (size_t)Pp * kMlpLds            // xT
                     + (size_t)kMlpH * kMlpLds       // a1T
                     + (size_t)kMlpRows * kMlpLdh    // s1
                     + (size_t)kMlpH * kMlpLds       // a2T
                     + (size_t)kMlpRows * kMlpLdh    // s2
                     + (size_t)kMlpRows * kMlpLdh    // wk0
                     + mlp_wk1_elems(Pp)             // wk1
                     + (size_t)kMlpH * kMlpLds;      // dz2T / dz1T
    return e * sizeof(__nv_bfloat16) + 8 * sizeof(float);
}

// ---------------------------------------------------------------------------
// Forward pass: out[r] = surrogate gradient at x[r], rows [32 b, 32 b + 32).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kMlpThreads) mlp_forward_kernel(const float* __restrict__ params, MlpBf16 wb,
                                                                   MlpNorm nm, int P, const float* __restrict__ x,
                                                                   long long n, float* __restrict__ out) {
    extern __shared__ __align__(16) __nv_bfloat16 sm_b[];
    const MlpLayout L = MlpLayout::make(P);
    const int Pp = L.Pp, ldp = mlp_ldp(Pp);
    __nv_bfloat16* xs = sm_b;                     // [32][ldp]
    __nv_bfloat16* a1 = xs + kMlpRows * ldp;      // [32][ldh]
    __nv_bfloat16* a2 = a1 + kMlpRows * kMlpLdh;  // [32][ldh]
    const long long r0 = (long long)blockIdx.x * kMlpRows;
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kMlpRows * Pp; i += kMlpThreads) {
        const int r = i / Pp, j = i % Pp;
        const long long row = r0 + r;
        float v = 0.0f;
        if (row < n && j < P) v = (x[row * P + j] - nm.in_mean[j]) / nm.in_scale[j];
        xs[r * ldp + j] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    {   // layer 1: 32 x 256, K = Pp; warp w -> columns [32 w, 32 w + 32)
        float acc[kMlpMT][4][4];
        zero_acc(acc);
        warp_gemm<kMlpMT, 4>(acc, xs, ldp, 0, wb.w1, Pp, 32 * warp, Pp);
        for_acc(acc, 0, 32 * warp, [&](int r, int c, float v) {
            a1[r * kMlpLdh + c] = __float2bfloat16_rn(silu_f(v + params[L.b1 + c]));
        });
    }
    __syncthreads();
    {   // layer 2
        float acc[kMlpMT][4][4];
        zero_acc(acc);
        warp_gemm<kMlpMT, 4>(acc, a1, kMlpLdh, 0, wb.w2, kMlpH, 32 * warp, kMlpH);
        for_acc(acc, 0, 32 * warp, [&](int r, int c, float v) {
            a2[r * kMlpLdh + c] = __float2bfloat16_rn(silu_f(v + params[L.b2 + c]));
        });
    }
    __syncthreads();
    // layer 3: 32 x Pp; 8-column tiles dealt to the warps round-robin
    for (int nt = warp; nt < Pp / 8; nt += 8) {
        float acc[kMlpMT][1][4];
        zero_acc(acc);
        warp_gemm<kMlpMT, 1>(acc, a2, kMlpLdh, 0, wb.w3, kMlpH, 8 * nt, kMlpH);
        for_acc(acc, 0, 8 * nt, [&](int r, int c, float v) {
            const long long row = r0 + r;
            if (row < n && c < P) out[row * P + c] = (v + params[L.b3 + c]) * nm.out_scale[c] + nm.out_mean[c];
        });
    }
}

// ---------------------------------------------------------------------------
// Forward + backward of one slice of 32 training pairs.  Writes this CTA's
// partial parameter gradient (MlpLayout order) and partial loss.
// ---------------------------------------------------------------------------
struct MlpTrainArgs {
    const float* params;
    MlpBf16 wb;
    MlpNorm nm;
    const float* x;        // pair positions, n x P
    const float* t;        // pair gradients, n x P
    long long n;           // number of pairs
    const int32_t* index;  // batch rows into the pairs; NULL = draw them from Philox(seed, step)
    uint32_t seed, step;
    int batch;             // B
    int P;
    float* partial;        // gridDim.x x layout.total
    float* partial_loss;   // gridDim.x
    int* bad_index;        // set to 1 when an index is outside [0, n)
};

// Row b of the batch drawn for Adam step `step`: multiply-shift of 64 Philox
// bits onto [0, n).
__device__ __forceinline__ long long mlp_draw_row(uint32_t seed, uint32_t step, int b, long long n) {
    const U4 w = philox4x32(seed, step, U4{(uint32_t)b, 0x53475452u, 0u, 0u});
    const unsigned long long r = ((unsigned long long)w.y << 32) | w.x;
    return (long long)__umul64hi(r, (unsigned long long)n);
}

__global__ void __launch_bounds__(kMlpThreads) mlp_train_kernel(MlpTrainArgs a) {
    extern __shared__ __align__(16) __nv_bfloat16 sm_b[];
    const MlpLayout L = MlpLayout::make(a.P);
    const int Pp = L.Pp, P = a.P, ldp = mlp_ldp(Pp);
    constexpr int ldh = kMlpLdh, lds = kMlpLds;
    const int warp = threadIdx.x >> 5;
    __nv_bfloat16* xT = sm_b;                       // [Pp][lds]  x^T       (until dW1)
    __nv_bfloat16* a1T = xT + Pp * lds;             // [H][lds]   a1^T      (until dW2)
    __nv_bfloat16* s1 = a1T + kMlpH * lds;          // [32][ldh]  silu'(z1) (until dZ1)
    __nv_bfloat16* a2T = s1 + kMlpRows * ldh;       // [H][lds]   a2^T      (until dW3)
    __nv_bfloat16* s2 = a2T + kMlpH * lds;          // [32][ldh]  silu'(z2) (until dZ2)
    __nv_bfloat16* wk0 = s2 + kMlpRows * ldh;       // [32][ldh]  x, then a2, then dZ2
    __nv_bfloat16* wk1 = wk0 + kMlpRows * ldh;      // a1, then dY [32][ldp] + dY^T [Pp][lds]
    __nv_bfloat16* dz2T = wk1 + mlp_wk1_elems(Pp);  // [H][lds]   dZ2^T, then dZ1^T
    float* red = reinterpret_cast<float*>(dz2T + kMlpH * lds);  // [8] loss partials
    __shared__ long long rows[kMlpRows];
    float* part = a.partial + (size_t)blockIdx.x * L.total;
    const int b0 = blockIdx.x * kMlpRows;
    const float inv_b = 1.0f / (float)a.batch;

    if (threadIdx.x < kMlpRows) {
        const int b = b0 + threadIdx.x;
        long long row = -1;
        if (b < a.batch) {
            if (a.index) {
                row = a.index[b];
                if (row < 0 || row >= a.n) { row = -1; *a.bad_index = 1; }
            } else {
                row = mlp_draw_row(a.seed, a.step, b, a.n);
            }
        }
        rows[threadIdx.x] = row;
    }
    __syncthreads();

    // ---- x: normalised, BF16, row-major into wk0 and transposed into xT
    __nv_bfloat16* xs = wk0;
    for (int i = threadIdx.x; i < kMlpRows * Pp; i += kMlpThreads) {
        const int r = i / Pp, j = i % Pp;
        const long long row = rows[r];
        float v = 0.0f;
        if (row >= 0 && j < P) v = (a.x[row * P + j] - a.nm.in_mean[j]) / a.nm.in_scale[j];
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        xs[r * ldp + j] = h;
        xT[j * lds + r] = h;
    }
    __syncthreads();
    // ---- layer 1 -> a1 (row-major in wk1), a1T, s1
    __nv_bfloat16* a1 = wk1;
    {
        float acc[kMlpMT][4][4];
        zero_acc(acc);
        warp_gemm<kMlpMT, 4>(acc, xs, ldp, 0, a.wb.w1, Pp, 32 * warp, Pp);
        for_acc(acc, 0, 32 * warp, [&](int r, int c, float v) {
            const float z = v + a.params[L.b1 + c];
            const __nv_bfloat16 h = __float2bfloat16_rn(silu_f(z));
            a1[r * ldh + c] = h;
            a1T[c * lds + r] = h;
            s1[r * ldh + c] = __float2bfloat16_rn(dsilu_f(z));
        });
    }
    __syncthreads();
    // ---- layer 2 -> a2 (row-major in wk0; x there is dead), a2T, s2
    __nv_bfloat16* a2 = wk0;
    {
        float acc[kMlpMT][4][4];
        zero_acc(acc);
        warp_gemm<kMlpMT, 4>(acc, a1, ldh, 0, a.wb.w2, kMlpH, 32 * warp, kMlpH);
        for_acc(acc, 0, 32 * warp, [&](int r, int c, float v) {
            const float z = v + a.params[L.b2 + c];
            const __nv_bfloat16 h = __float2bfloat16_rn(silu_f(z));
            a2[r * ldh + c] = h;
            a2T[c * lds + r] = h;
            s2[r * ldh + c] = __float2bfloat16_rn(dsilu_f(z));
        });
    }
    __syncthreads();
    // ---- layer 3 + squared error -> dY (wk1, a1 is dead) and dY^T
    __nv_bfloat16* dy = wk1;
    __nv_bfloat16* dyT = wk1 + kMlpRows * ldp;
    float lsum = 0.0f;
    for (int nt = warp; nt < Pp / 8; nt += 8) {
        float acc[kMlpMT][1][4];
        zero_acc(acc);
        warp_gemm<kMlpMT, 1>(acc, a2, ldh, 0, a.wb.w3, kMlpH, 8 * nt, kMlpH);
        for_acc(acc, 0, 8 * nt, [&](int r, int c, float v) {
            float d = 0.0f;
            const long long row = rows[r];
            if (row >= 0 && c < P) {
                const float tv = (a.t[row * P + c] - a.nm.out_mean[c]) / a.nm.out_scale[c];
                const float e = v + a.params[L.b3 + c] - tv;
                lsum = fmaf(e, e, lsum);
                d = 2.0f * e * inv_b;
            }
            const __nv_bfloat16 h = __float2bfloat16_rn(d);
            dy[r * ldp + c] = h;
            dyT[c * lds + r] = h;
        });
    }
    lsum = warp_sum(lsum);
    if ((threadIdx.x & 31) == 0) red[warp] = lsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float l = 0.0f;
        for (int w = 0; w < 8; ++w) l += red[w];
        a.partial_loss[blockIdx.x] = l * inv_b;
    }
    // ---- dW3 = dY^T a2 : [Pp][H]; warp -> 32 columns, rows in passes of 64
    for (int m0 = 0; m0 < Pp; m0 += 64)
        warp_gemm_rows(Pp - m0, dyT, lds, m0, a2T, lds, 32 * warp, kMlpRows, [&](int r, int c, float v) {
            part[L.w3 + (size_t)r * kMlpH + c] = v;
        });
    for (int c = threadIdx.x; c < Pp; c += kMlpThreads) {
        float s = 0.0f;
        for (int r = 0; r < kMlpRows; ++r) s += __bfloat162float(dy[r * ldp + c]);
        part[L.b3 + c] = s;
    }
    // ---- dA2 = dY W3 (Bt = W3^T [H][Pp]); dZ2 = dA2 * s2 -> wk0 (a2 is dead) and dz2T
    __nv_bfloat16* dz2 = wk0;
    {
        float acc[kMlpMT][4][4];
        zero_acc(acc);
        warp_gemm<kMlpMT, 4>(acc, dy, ldp, 0, a.wb.w3t, Pp, 32 * warp, Pp);
        for_acc(acc, 0, 32 * warp, [&](int r, int c, float v) {
            const __nv_bfloat16 h = __float2bfloat16_rn(v * __bfloat162float(s2[r * ldh + c]));
            dz2[r * ldh + c] = h;
            dz2T[c * lds + r] = h;
        });
    }
    __syncthreads();
    // ---- dW2 = dZ2^T a1 : [H][H]; warp -> 32 columns, 4 passes of 64 rows
    for (int m0 = 0; m0 < kMlpH; m0 += 64)
        warp_gemm_rows(64, dz2T, lds, m0, a1T, lds, 32 * warp, kMlpRows, [&](int r, int c, float v) {
            part[L.w2 + (size_t)r * kMlpH + c] = v;
        });
    for (int c = threadIdx.x; c < kMlpH; c += kMlpThreads) {
        float s = 0.0f;
        for (int r = 0; r < kMlpRows; ++r) s += __bfloat162float(dz2[r * ldh + c]);
        part[L.b2 + c] = s;
    }
    // ---- dA1 = dZ2 W2 (Bt = W2^T); dZ1 = dA1 * s1 -> dz1T (over dz2T once dW2 is done)
    {
        float acc[kMlpMT][4][4];
        zero_acc(acc);
        warp_gemm<kMlpMT, 4>(acc, dz2, ldh, 0, a.wb.w2t, kMlpH, 32 * warp, kMlpH);
        __syncthreads();  // every warp has finished reading dz2T (dW2) and dz2 (db2)
        for_acc(acc, 0, 32 * warp, [&](int r, int c, float v) {
            dz2T[c * lds + r] = __float2bfloat16_rn(v * __bfloat162float(s1[r * ldh + c]));
        });
    }
    __syncthreads();
    // ---- dW1 = dZ1^T x : [H][Pp]; 8-column tiles round-robin, 4 passes of 64 rows
    const __nv_bfloat16* dz1T = dz2T;
    for (int nt = warp; nt < Pp / 8; nt += 8)
        for (int m0 = 0; m0 < kMlpH; m0 += 64) {
            float acc[4][1][4];
            zero_acc(acc);
            warp_gemm<4, 1>(acc, dz1T, lds, m0, xT, lds, 8 * nt, kMlpRows);
            for_acc(acc, m0, 8 * nt, [&](int r, int c, float v) { part[L.w1 + (size_t)r * Pp + c] = v; });
        }
    for (int c = threadIdx.x; c < kMlpH; c += kMlpThreads) {
        float s = 0.0f;
        for (int r = 0; r < kMlpRows; ++r) s += __bfloat162float(dz1T[c * lds + r]);
        part[L.b1 + c] = s;
    }
}

// Fold the per-CTA partials in CTA order (deterministic), then one Adam step
// on the FP32 master weights (bias corrections bc1 = 1/(1-beta1^t),
// bc2 = 1/(1-beta2^t) from the host).  One thread per weight.  With
// adam == 0 only the folded gradient is written.
__global__ void mlp_reduce_adam_kernel(float* __restrict__ params, float* __restrict__ adam_m,
                                       float* __restrict__ adam_v, const float* __restrict__ partial, int nparts,
                                       long long total, float* __restrict__ grad_out,
                                       const float* __restrict__ part_loss, float* __restrict__ loss_out, float lr,
                                       float beta1, float beta2, float eps, float bc1, float bc2, int adam) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && loss_out) {
        float l = 0.0f;
        for (int p = 0; p < nparts; ++p) l += part_loss[p];
        *loss_out = l;
    }
    if (i >= total) return;
    float g = 0.0f;
    for (int p = 0; p < nparts; ++p) g += partial[(size_t)p * total + i];
    if (grad_out) grad_out[i] = g;
    if (!adam) return;
    const float m = beta1 * adam_m[i] + (1.0f - beta1) * g;
    const float v = beta2 * adam_v[i] + (1.0f - beta2) * g * g;
    adam_m[i] = m;
    adam_v[i] = v;
    params[i] -= lr * (m * bc1) / (sqrtf(v * bc2) + eps);
}

// BF16 copies (and the transposes the backward pass reads) of the FP32 weights.
__global__ void mlp_refresh_bf16_kernel(const float* __restrict__ params, MlpBf16 wb, int P) {
    const MlpLayout L = MlpLayout::make(P);
    const int Pp = L.Pp;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kMlpH * Pp) {
        wb.w1[i] = __float2bfloat16_rn(params[L.w1 + i]);  // W1 [H][Pp]
        const int r = i / Pp, c = i % Pp;                  // W3 [c][r] -> W3^T [r][c]
        const __nv_bfloat16 h = __float2bfloat16_rn(params[L.w3 + (size_t)c * kMlpH + r]);
        wb.w3[(size_t)c * kMlpH + r] = h;
        wb.w3t[(size_t)r * Pp + c] = h;
    }
    if (i < kMlpH * kMlpH) {
        const int r = i / kMlpH, c = i % kMlpH;
        const __nv_bfloat16 h = __float2bfloat16_rn(params[L.w2 + i]);
        wb.w2[i] = h;
        wb.w2t[(size_t)c * kMlpH + r] = h;
    }
}

// Initial weights U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from Philox (key = (seed,
// layer), counter = weight index), zero biases and zero padded entries.
__global__ void mlp_init_kernel(float* __restrict__ params, int P, uint32_t seed) {
    const MlpLayout L = MlpLayout::make(P);
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)L.total) return;
    uint32_t layer = 0;
    long long local = 0;
    int fan = 1;
    bool live = false;
    if (i < (long long)L.b1) {
        layer = 1; local = i - (long long)L.w1; fan = P; live = (local % L.Pp) < P;
    } else if (i >= (long long)L.w2 && i < (long long)L.b2) {
        layer = 2; local = i - (long long)L.w2; fan = kMlpH; live = true;
    } else if (i >= (long long)L.w3 && i < (long long)L.b3) {
        layer = 3; local = i - (long long)L.w3; fan = kMlpH; live = (local / kMlpH) < P;
    }
    float v = 0.0f;
    if (live) {
        const float u = u01(philox4x32(seed, layer, U4{(uint32_t)local, 0u, 0u, 0u}).x);
        v = (2.0f * u - 1.0f) * rsqrtf((float)fan);
    }
    params[i] = v;
}

// Column statistics of an n x P matrix: per-chunk sums and sums of squares in
// FP64 (thread j <-> column j over the rows of one chunk), folded in chunk
// order by mlp_stats_final_kernel.
__global__ void mlp_stats_partial_kernel(const float* __restrict__ x, long long n, int P, long long chunk_rows,
                                         double* __restrict__ part_sum, double* __restrict__ part_sq) {
    const int j = threadIdx.x;
    if (j >= P) return;
    const long long r0 = (long long)blockIdx.x * chunk_rows;
    const long long r1 = r0 + chunk_rows < n ? r0 + chunk_rows : n;
    double s = 0.0, q = 0.0;
    for (long long r = r0; r < r1; ++r) {
        const double v = x[r * P + j];
        s += v;
        q += v * v;
    }
    part_sum[(size_t)blockIdx.x * P + j] = s;
    part_sq[(size_t)blockIdx.x * P + j] = q;
}

// Mean and standard deviation per column; the deviation is floored at 1e-6 of
// the largest column's and at 1e-12, so constant columns do not divide by 0.
// One block of kMlpMaxP threads.
__global__ void mlp_stats_final_kernel(const double* __restrict__ part_sum, const double* __restrict__ part_sq,
                                       int chunks, long long n, int P, float* __restrict__ mean,
                                       float* __restrict__ scale) {
    __shared__ double sd[kMlpMaxP];
    __shared__ double top;
    const int j = threadIdx.x;
    double m = 0.0;
    if (j < P) {
        double s = 0.0, q = 0.0;
        for (int c = 0; c < chunks; ++c) {
            s += part_sum[(size_t)c * P + j];
            q += part_sq[(size_t)c * P + j];
        }
        m = s / (double)n;
        const double v = q / (double)n - m * m;
        sd[j] = sqrt(v > 0.0 ? v : 0.0);
    }
    __syncthreads();
    if (j == 0) {
        double t = 0.0;
        for (int k = 0; k < P; ++k) t = fmax(t, sd[k]);
        top = t;
    }
    __syncthreads();
    if (j < P) {
        mean[j] = (float)m;
        scale[j] = (float)fmax(fmax(sd[j], 1e-6 * top), 1e-12);
    }
}

}  // namespace ut
