// ut_mlp_tc.cuh -- the learned surrogate's forward pass on the 5th-generation
// tensor cores: 128 rows per CTA, the three layers as tcgen05.mma kind::f16
// (BF16 operands, FP32 accumulators in TMEM), the weights streamed by TMA in
// K-blocks of 16 through a shared-memory ring, and each layer's activations
// written back to shared memory (K-major, SWIZZLE_32B) as the next layer's A
// operand.  The rounding points are those of mlp_forward_kernel (ut_mlp.cuh):
//   xb = bf16((theta - in_mean) / in_scale)
//   a1b = bf16(silu(xb W1b^T + b1)),  a2b = bf16(silu(a1b W2b^T + b2))
//   out = (a2b W3b^T + b3) * out_scale + out_mean
// only the order of the FP32 accumulation inside each dot product differs.
//
// Warp roles (320 threads): warp 0 = TMA producer of the weight ring, warp 1 =
// MMA issuer (and TMEM owner), warps 2-9 = epilogue: thread = row (TMEM lane),
// two warps per lane quadrant, each taking half of a layer's columns.
// TMEM (512 columns): D1 [0, 256), D2 [256, 512), D3 [0, Pp) (D1 is consumed
// before layer 3 starts).  Shared memory: x tile (Pp/16 K-blocks of
// [128 rows][32 B]), one activation tile (16 K-blocks), 8 ring stages of
// [256 rows][32 B], barriers.  Every wait is bounded (mbar_wait).
#pragma once

#include <cuda_bf16.h>

#include "ut_mlp.cuh"
#include "ut_tc_glm.cuh"

namespace ut {

constexpr int kMtRows = 128;                 // rows per CTA (the MMA's M)
constexpr int kMtThreads = 320;              // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue
constexpr int kMtEpiWarps = 8;
constexpr int kMtStages = 8;                 // weight ring stages
constexpr int kMtStageBytes = kMlpH * 32;    // [256 rows][16 bf16]
constexpr int kMtBlockBytes = kMtRows * 32;  // one K-block of an A tile: [128 rows][16 bf16]
constexpr int kMtHBlocks = kMlpH / 16;       // K-blocks of a hidden activation

__host__ __device__ inline size_t mlp_tc_smem(int Pp) {
    return 1024 + (size_t)(Pp / 16) * kMtBlockBytes + (size_t)kMtHBlocks * kMtBlockBytes +
           (size_t)kMtStages * kMtStageBytes + 256;
}

// Instruction descriptor: D = F32, A = B = BF16, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem], kind::f16, issued by one elected lane of a converged warp.
__device__ __forceinline__ void mma_bf16_ss_warp(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p, e;\n\t.reg .b32 r;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "elect.sync r|e, 0xffffffff;\n\t"
        "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

// 8 consecutive K elements (k0 % 8 == 0) of row r into a K-major SWIZZLE_32B
// A tile of 128 rows: K-block k0 / 16, 16-byte chunk (k0 / 8) % 2, which the
// 32-byte swizzle exchanges on rows whose bit 2 is set.
__device__ __forceinline__ void mlp_tc_put8(uint8_t* tile, int r, int k0, const float (&v)[8]) {
    const int chunk = ((k0 >> 3) & 1) ^ ((r >> 2) & 1);
    uint4 w;
    __nv_bfloat162 p0 = __floats2bfloat162_rn(v[0], v[1]), p1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(v[4], v[5]), p3 = __floats2bfloat162_rn(v[6], v[7]);
    w.x = *reinterpret_cast<uint32_t*>(&p0);
    w.y = *reinterpret_cast<uint32_t*>(&p1);
    w.z = *reinterpret_cast<uint32_t*>(&p2);
    w.w = *reinterpret_cast<uint32_t*>(&p3);
    *reinterpret_cast<uint4*>(tile + (size_t)(k0 >> 4) * kMtBlockBytes + r * 32 + chunk * 16) = w;
}

struct MlpTcArgs {
    const float* params;  // FP32 master weights (for the biases)
    MlpNorm nm;
    int P, Pp;
    const float* x;       // n x P
    long long n;
    float* out;           // n x P
    int* err;             // sticky error word (a bounded wait gave up)
};

__global__ void __launch_bounds__(kMtThreads, 1)
    mlp_forward_tc_kernel(const __grid_constant__ CUtensorMap map_w1, const __grid_constant__ CUtensorMap map_w2,
                          const __grid_constant__ CUtensorMap map_w3, MlpTcArgs a) {
    extern __shared__ __align__(1024) uint8_t mt_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(mt_raw) + 1023) & ~uintptr_t(1023));
    const int Pp = a.Pp, KX = Pp / 16;
    uint8_t* xt = smem;                                       // [KX][128][32 B]
    uint8_t* act = xt + (size_t)KX * kMtBlockBytes;            // [16][128][32 B]
    uint8_t* ring = act + (size_t)kMtHBlocks * kMtBlockBytes;  // [8][256][32 B]
    uint64_t* bars = reinterpret_cast<uint64_t*>(ring + (size_t)kMtStages * kMtStageBytes);
    uint64_t* bar_full = bars;                 // [8]
    uint64_t* bar_empty = bars + 8;            // [8]
    uint64_t* bar_x = bars + 16;               // the x tile is in shared memory
    uint64_t* bar_a1 = bars + 17;              // layer-1 activations are in shared memory
    uint64_t* bar_a2 = bars + 18;
    uint64_t* bar_d = bars + 19;               // [3] layer d's accumulator is complete
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 22);
    const MlpLayout L = MlpLayout::make(a.P);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long r0 = (long long)blockIdx.x * kMtRows;
    // the weight blocks in the order the MMAs use them: W1 (KX), W2 (16), W3 (16)
    const int nblk = KX + 2 * kMtHBlocks;

    if (threadIdx.x == 0) {
        for (int i = 0; i < kMtStages; ++i) {
            mbar_init(bar_full + i, 1);
            mbar_init(bar_empty + i, 1);
        }
        mbar_init(bar_x, kMtEpiWarps);
        mbar_init(bar_a1, kMtEpiWarps);
        mbar_init(bar_a2, kMtEpiWarps);
        for (int i = 0; i < 3; ++i) mbar_init(bar_d + i, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(tmem_slot, 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    auto wwait = [&](uint64_t* bar, uint32_t parity) -> bool {
        return __all_sync(0xffffffffu, mbar_wait(bar, parity, a.err));
    };

    if (warp == 0) {
        // ---------------- TMA producer: the weight ring ----------------
        for (int j = 0; j < nblk; ++j) {
            const int s = j % kMtStages;
            if (j >= kMtStages && !wwait(bar_empty + s, ((j / kMtStages) - 1) & 1)) break;
            uint8_t* st = ring + (size_t)s * kMtStageBytes;
            if (j < KX) {
                mbar_expect_tx_warp(bar_full + s, kMlpH * 32);
                tma_load_2d_warp(st, &map_w1, bar_full + s, 16 * j, 0);
            } else if (j < KX + kMtHBlocks) {
                mbar_expect_tx_warp(bar_full + s, kMlpH * 32);
                tma_load_2d_warp(st, &map_w2, bar_full + s, 16 * (j - KX), 0);
            } else {
                mbar_expect_tx_warp(bar_full + s, Pp * 32);
                tma_load_2d_warp(st, &map_w3, bar_full + s, 16 * (j - KX - kMtHBlocks), 0);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        bool ok = true;
        int j = 0;
        // layer l: D += A (K-blocks of an A tile) x B (the ring's weight blocks)
        auto layer = [&](uint8_t* atile, int kblocks, uint32_t d, int N) {
            const uint32_t id = idesc_bf16(kMtRows, N);
            for (int kb = 0; ok && kb < kblocks; ++kb, ++j) {
                const int s = j % kMtStages;
                if (!wwait(bar_full + s, (j / kMtStages) & 1)) { ok = false; break; }
                tc_fence_after();
                const uint64_t ad = sdesc_sw32(smem_u32(atile + (size_t)kb * kMtBlockBytes), 16, 256);
                const uint64_t bd = sdesc_sw32(smem_u32(ring + (size_t)s * kMtStageBytes), 16, 256);
                mma_bf16_ss_warp(d, ad, bd, id, kb > 0 ? 1u : 0u);
                mma_commit_warp(bar_empty + s);
            }
        };
        if (wwait(bar_x, 0)) {
            tc_fence_after();
            layer(xt, KX, tmem, kMlpH);
            if (ok) mma_commit_warp(bar_d + 0);
        } else {
            ok = false;
        }
        if (ok && wwait(bar_a1, 0)) {
            tc_fence_after();
            layer(act, kMtHBlocks, tmem + kMlpH, kMlpH);
            if (ok) mma_commit_warp(bar_d + 1);
        } else {
            ok = false;
        }
        if (ok && wwait(bar_a2, 0)) {
            tc_fence_after();
            layer(act, kMtHBlocks, tmem, Pp);
            if (ok) mma_commit_warp(bar_d + 2);
        }
    } else {
        // ---------------- epilogue: thread = row ----------------
        const int q = warp & 3, half = (warp - 2) >> 2;
        const int r = q * 32 + lane;
        const long long row = r0 + r;
        const uint32_t lane_off = (uint32_t)(q * 32) << 16;
        auto warp_wait = [&](uint64_t* bar, uint32_t parity) -> bool {
            return __all_sync(0xffffffffu, mbar_wait(bar, parity, a.err));
        };
        auto arrive = [&](uint64_t* bar) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the tile is read by the tensor cores
            __syncwarp();
            if (lane == 0) mbar_arrive(bar);
        };
        // x tile: this half takes the K-blocks kb with kb % 2 == half
        for (int kb = half; kb < KX; kb += 2) {
#pragma unroll
            for (int c8 = 0; c8 < 2; ++c8) {
                float v[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const int k = 16 * kb + 8 * c8 + t;
                    v[t] = (row < a.n && k < a.P) ? (a.x[row * a.P + k] - a.nm.in_mean[k]) / a.nm.in_scale[k] : 0.0f;
                }
                mlp_tc_put8(xt, r, 16 * kb + 8 * c8, v);
            }
        }
        arrive(bar_x);
        // hidden layers: z = D + b, a = silu(z) into the activation tile; this half takes columns [128 half, +128)
        auto hidden = [&](int d, uint32_t dcol, size_t boff, uint64_t* done) -> bool {
            if (!warp_wait(bar_d + d, 0)) return false;
            tc_fence_after();
            for (int c16 = 0; c16 < 8; ++c16) {
                const int k0 = 128 * half + 16 * c16;
                float z[16];
                tmem_ld16(tmem + lane_off + dcol + k0, z);
#pragma unroll
                for (int c8 = 0; c8 < 2; ++c8) {
                    float v[8];
#pragma unroll
                    for (int t = 0; t < 8; ++t) v[t] = silu_f(z[8 * c8 + t] + a.params[boff + k0 + 8 * c8 + t]);
                    mlp_tc_put8(act, r, k0 + 8 * c8, v);
                }
            }
            tc_fence_before();
            arrive(done);
            return true;
        };
        bool ok = hidden(0, 0, L.b1, bar_a1);
        // the second layer's MMAs have read the first activations once its accumulator is complete
        ok = ok && hidden(1, kMlpH, L.b2, bar_a2);
        if (ok && warp_wait(bar_d + 2, 0)) {
            tc_fence_after();
            for (int c16 = half; c16 < Pp / 16; c16 += 2) {
                float yv[16];
                tmem_ld16(tmem + lane_off + 16 * c16, yv);
                if (row < a.n) {
#pragma unroll
                    for (int t = 0; t < 16; ++t) {
                        const int k = 16 * c16 + t;
                        if (k < a.P)
                            a.out[row * a.P + k] = (yv[t] + a.params[L.b3 + k]) * a.nm.out_scale[k] + a.nm.out_mean[k];
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, 512);
}

// A BF16 weight matrix [rows][cols] (row-major) as a TMA map of boxes
// [box_rows][16 columns], SWIZZLE_32B (the K-major B-operand layout).
inline bool mlp_tc_make_map(CUtensorMap* m, const __nv_bfloat16* base, int rows, int cols, int box_rows) {
    PFN_encodeTiled enc = tc_encode_fn();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * sizeof(__nv_bfloat16)};
    cuuint32_t box[2] = {16, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(base), dims, strides, box,
                     estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace ut
