// ut_tc_glm.cuh -- Bernoulli-logit GLM logjoint + gradient on the 5th-gen
// tensor cores (tcgen05, TF32 with FP32 accumulation in TMEM), FP32-accurate
// through the 3xTF32 split a*b ~ a_hi*b_hi + a_hi*b_lo + a_lo*b_hi, where
// hi = tf32_round(x) and lo = tf32_round(x - hi).
//
// One CTA owns a tile of 128 chains and a contiguous range of 32-observation
// tiles.  Per observation tile t:
//   GEMM1:  H^T[c, n]  = sum_f Theta[c, f] X[n, f]      M=128 chains, N=32 obs, K=Fp
//           A = Theta (hi/lo) resident in TMEM, B = X tile (K-major, SMEM)
//   epilogue (thread = chain c = TMEM lane c):
//           r = y_n - logistic(h),  ll_c += y_n h - log1p_exp(h)
//           r -> (r_hi, r_lo) written back into TMEM
//   GEMM2:  G^T[c, f] += sum_n R^T[c, n] X[n, f]         M=128, N=Fp, K=32 obs
//           A = R (TMEM), B = X tile (MN-major, SMEM)
// so the per-chain log-likelihood is a thread-local sum and the residual tile
// never touches shared memory.
//
// Warp roles (576 threads): warp 0 = TMA producer, warp 1 = MMA issuer (and
// TMEM owner), warps 2-17 = epilogue: four warps per TMEM lane quadrant, each
// owning 8 of a tile's observation columns and a quarter of the gradient columns.
// Pipelines: 3 X stages and up to 3 H/R TMEM buffers (as many as TMEM holds
// beside Theta and the gradient accumulator: 3 for 100 features), so GEMM1 of
// the next tiles runs on the tensor cores while the epilogue of tile t runs on
// the CUDA cores / SFUs.
// The tensor pipe stays busy while the epilogue's round trip (GEMM1(t) done ->
// R(t) in TMEM) is shorter than GEMM2(t-1) + GEMM1(t+1), so the epilogue keeps
// that path short: one mbarrier arrival per warp (not per thread), and the
// periodic drain of the gradient accumulator rides on the next tile's epilogue
// instead of stalling the MMA issuer.
//
// Every mbarrier wait is bounded (~2^31 clocks).  A wait that gives up sets the
// error word, the role stops issuing, all threads meet at the final barrier and
// the TMEM owner frees TMEM before the CTA exits.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "ut_common.cuh"

namespace ut {

constexpr int kTcChains = 128;          // M of both GEMMs (TMEM lanes)
constexpr int kTcObs = 32;              // observations per tile (N of GEMM1, K of GEMM2)
constexpr int kTcMaxFp = 128;           // padded feature count the TMEM plan holds (3 Fp + 128 <= 512)
constexpr int kTcThreads = 576;         // warp 0 TMA, warp 1 MMA, warps 2-17 epilogue
constexpr int kTcEpiThreads = 512;
constexpr int kTcEpiWarps = kTcEpiThreads / 32;   // arrivals per epilogue barrier phase
constexpr long long kTcWaitClocks = 1ll << 31;
// Per-CTA set-up (barriers, TMEM allocation, theta into TMEM, pipeline fill) in
// units of one 32-observation tile's time at one CTA per SM: ~27 us vs ~2.4 us
// per tile, fitted to timings of 8-, 4- and 2-wave grids on a 100000 x 100 design
// with 4096 chains.
constexpr int kTcCtaOverheadTiles = 11;

struct TcGlmParams {
    const float* y;        // N
    float* part_ll;        // S x C
    float* part_g;         // S x C x F
    int* err;              // device error word (1 = a bounded wait gave up)
    int N, F, Fp, C;
    int tiles_per_split;   // observation tiles per CTA
    int num_tiles;         // total observation tiles
    int want_grad;
    int ctiles, S, sms;    // chain tiles, observation splits of the full grid, SMs
    const int* nact;       // optional: only the first *nact chains are live
    int col_tlo, col_d2, col_buf;  // TMEM columns of Theta_lo, the accumulator, the first H/R buffer
    int xk3d;              // the K-major maps are 3-D (8 features, rows, K-blocks): one copy per tile
    int yvalid;            // every y is 0 or 1: tiles without padding skip the support check
    int xkpair;            // paired GEMM1: the K-major view is [K-block][hi | lo][rows] (one 4-D copy),
                           // Theta_hi meets X_hi and X_lo in one N = 64 MMA per K-block
};

// The epilogue works in base 2: Theta is scaled by log2(e) before it enters
// TMEM, so GEMM1 yields h' = log2(e) eta, and exp(-|eta|) = 2^-|h'|,
// log1p_exp(eta) = ln(2) (max(h', 0) + log2(1 + 2^-|h'|)): the hardware base-2
// exponential and logarithm apply directly, and the log-likelihood, summed in
// base-2 units, is multiplied by ln(2) once per chain.
constexpr float kTcLog2e = 1.4426950408889634f;
constexpr float kTcLn2 = 0.6931471805599453f;
__device__ __forceinline__ float tc_ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float tc_lg2(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float tc_rcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Work split of one launch.  Without nact: the (chain tile, split) grid of the
// plan and partial rows of C chains.  With nact: only ceil(nact / 128) chain
// tiles are live, and when they are few the observations are cut into more
// splits so the launch still fills the SMs (at most the plan's grid size
// CTAs); partial rows then hold nt * 128 chains.
struct TcSplit {
    int nt, S, tps, Cl;
};

__host__ __device__ __forceinline__ TcSplit tc_split(const TcGlmParams& p) {
    TcSplit r;
    if (!p.nact) {
        r.nt = p.ctiles; r.S = p.S; r.tps = p.tiles_per_split; r.Cl = p.C;
        return r;
    }
    const int n = *p.nact;
    r.nt = max(1, (n + kTcChains - 1) / kTcChains);
    int S = max(p.S, min(p.ctiles * p.S, p.sms) / r.nt);
    S = min(S, p.num_tiles);
    r.tps = (p.num_tiles + S - 1) / S;
    r.S = (p.num_tiles + r.tps - 1) / r.tps;
    r.Cl = r.nt * kTcChains;
    return r;
}

// ---------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Non-blocking test of a phase (no suspension, unlike try_wait).
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: returns false (and raises the error word) when it gives up.
// The clock and the (global) error word are only looked at every 1024 spins,
// so a wait that succeeds within a few polls costs no memory round trip.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 1023u) == 0) {
            if (clock64() - t0 > kTcWaitClocks) {
                atomicExch(err, 1);
                return false;
            }
            if (*((volatile int*)err)) return false;  // another role already gave up
        }
    }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// Plain (untiled) bulk copy global -> shared, completing on an mbarrier.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]
__device__ __forceinline__ void mma_ss(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

// D[tmem] (+)= A[tmem] * B[smem]
__device__ __forceinline__ void mma_ts(uint32_t d, uint32_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}"
        ::"r"(d), "r"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// Warp-wide forms: the whole (converged) warp runs the issuing code, so the
// descriptors and addresses are warp-uniform values, and one elected lane --
// always the same one, since tcgen05.commit tracks the MMAs of the thread that
// issues it -- issues the instruction.
__device__ __forceinline__ void mma_ts_warp(uint32_t d, uint32_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p, e;\n\t.reg .b32 r;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "elect.sync r|e, 0xffffffff;\n\t"
        "@e tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}"
        ::"r"(d), "r"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit_warp(uint64_t* bar) {
    asm volatile(
        "{\n\t.reg .pred e;\n\t.reg .b32 r;\n\t"
        "elect.sync r|e, 0xffffffff;\n\t"
        "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}"
        ::"r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_expect_tx_warp(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .pred e;\n\t.reg .b32 r;\n\t"
        "elect.sync r|e, 0xffffffff;\n\t"
        "@e mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n\t}"
        ::"r"(smem_u32(bar)), "r"(bytes)
        : "memory");
}

__device__ __forceinline__ void tma_load_2d_warp(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "{\n\t.reg .pred e;\n\t.reg .b32 r;\n\t"
        "elect.sync r|e, 0xffffffff;\n\t"
        "@e cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];\n\t}"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d_warp(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y,
                                                 int z) {
    asm volatile(
        "{\n\t.reg .pred e;\n\t.reg .b32 r;\n\t"
        "elect.sync r|e, 0xffffffff;\n\t"
        "@e cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];\n\t}"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ void tma_load_4d_warp(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y,
                                                 int z, int w) {
    asm volatile(
        "{\n\t.reg .pred e;\n\t.reg .b32 r;\n\t"
        "elect.sync r|e, 0xffffffff;\n\t"
        "@e cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], [%2];\n\t}"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
        : "memory");
}

__device__ __forceinline__ void bulk_load_warp(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "{\n\t.reg .pred e;\n\t.reg .b32 r;\n\t"
        "elect.sync r|e, 0xffffffff;\n\t"
        "@e cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n\t}"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool elect_one() {
    uint32_t is = 0;
    asm volatile(
        "{\n\t.reg .pred e;\n\t.reg .b32 r;\n\t"
        "elect.sync r|e, 0xffffffff;\n\t"
        "selp.u32 %0, 1, 0, e;\n\t}"
        : "=r"(is));
    return is != 0;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};"
        ::"r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
          "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]),
          "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]),
          "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
}

__device__ __forceinline__ uint32_t tf32_bits(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// Shared-memory matrix descriptor, SWIZZLE_32B layout.
__device__ __forceinline__ uint64_t sdesc_sw32(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version (sm_100)
    d |= (uint64_t)6 << 61;   // SWIZZLE_32B
    return d;
}

// Instruction descriptor: D=F32, A=B=TF32, dense, M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, int b_mn_major) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)b_mn_major << 16) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

// ---------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------
// TMEM columns (512 allocated), KC = features rounded up to 8 (GEMM1's K),
// Fp = features rounded up to 16 (GEMM2's N), both <= 128:
//   Theta_hi [0, KC)   Theta_lo [KC, 2KC)   D2 = G^T [2KC, 2KC + Fp)
//   buffer b (0 .. nbuf-1): H^T / R_hi [2KC + Fp + 64b, +32)   R_lo [.. + 32, +32)
//   (paired GEMM1: H^T is the sum of the buffer's two halves, Theta_hi X_hi in the
//   first, Theta_hi X_lo + Theta_lo X_hi in the second; R_hi / R_lo replace them)
// nbuf = min(3, (512 - 2KC - Fp) / 64): 3 for 100 features (208 + 112 + 192).
// Shared memory per pipeline stage (3 stages), Fp features x 32 observations:
//   XK_hi, XK_lo : K-major SWIZZLE_32B, Fp/8 blocks of [32 rows][32 B]     (GEMM1 B)
//                  (paired GEMM1: [K-block][XK_hi 32 rows, XK_lo 32 rows], 2 KB a K-block)
//   XM_hi, XM_lo : MN-major SWIZZLE_128B_BASE32B, Fp/32 atoms of [32 rows][128 B] (GEMM2 B)
// (TF32 operands that are MN-major must use the 128B_BASE32B layout, which no
// K-major layout shares, so each X tile is loaded twice, once per view.)
constexpr int kTcStages = 3;
constexpr int kTcMaxBufs = 3;      // H/R buffers: at most the X stages (GEMM1(i) needs stage i's
                                   // release after GEMM2(i - 3), which the same thread issues)
constexpr int kTcDrainTiles = 4;   // observation tiles per TMEM gradient accumulation run

__host__ __device__ inline int tc_kblocks(int Fp) { return Fp / 8; }
// K-blocks GEMM1 needs: the features rounded up to 8 (the TF32 MMA's K), not to
// the 16 of Fp (GEMM2's N); the blocks past it hold zero padding.
__host__ __device__ inline int tc_kblocks_used(int F) { return (F + 7) / 8; }
// H/R TMEM buffers the 512 columns hold beside Theta hi/lo and the accumulator.
__host__ __device__ inline int tc_nbuf(int F, int Fp) {
    const int n = (512 - 16 * tc_kblocks_used(F) - Fp) / 64;
    return n < kTcMaxBufs ? n : kTcMaxBufs;
}
// TMEM column plan {Theta_lo, D2, first H/R buffer} for nbuf buffers.  The
// compact plan packs Theta hi/lo at KC columns each; the wide plan (2 buffers
// only) spaces everything at Fp: Theta_lo at Fp, D2 at 2Fp, buffers at 3Fp.
__host__ __device__ inline void tc_columns(int F, int Fp, bool wide, int cols[3]) {
    const int KC = 8 * tc_kblocks_used(F);
    const int a = wide ? Fp : KC;
    cols[0] = a;
    cols[1] = 2 * a;
    cols[2] = 2 * a + Fp;
}
__host__ __device__ inline int tc_matoms(int Fp) { return (Fp + 31) / 32; }
__host__ __device__ inline int tc_xk_bytes(int Fp) { return tc_kblocks(Fp) * kTcObs * 32; }
__host__ __device__ inline int tc_xm_bytes(int Fp) { return tc_matoms(Fp) * kTcObs * 128; }
__host__ __device__ inline int tc_stage_bytes(int Fp) { return 2 * tc_xk_bytes(Fp) + 2 * tc_xm_bytes(Fp) + 1024; }  // + y tile (128 B used)

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
        ::"r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
          "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
                 ::"r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory descriptor, SWIZZLE_128B_BASE32B (layout type 1).
__device__ __forceinline__ uint64_t sdesc_sw128b32(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)1 << 61;
    return d;
}

// TMEM load of a warp's kCols (8 or 16) consecutive columns.
template <int kCols>
__device__ __forceinline__ void tmem_ld_cols(uint32_t taddr, float (&v)[kCols]) {
    if constexpr (kCols == 8) tmem_ld8(taddr, v);
    else tmem_ld16(taddr, v);
}

// The sum of two kCols-column TMEM ranges (both loads in flight, one wait).
template <int kCols>
__device__ __forceinline__ void tmem_ld_cols_sum(uint32_t ta, uint32_t tb, float (&v)[kCols]) {
    uint32_t ra[kCols], rb[kCols];
    if constexpr (kCols == 8) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(ra[0]), "=r"(ra[1]), "=r"(ra[2]), "=r"(ra[3]), "=r"(ra[4]), "=r"(ra[5]), "=r"(ra[6]),
                       "=r"(ra[7])
                     : "r"(ta));
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(rb[0]), "=r"(rb[1]), "=r"(rb[2]), "=r"(rb[3]), "=r"(rb[4]), "=r"(rb[5]), "=r"(rb[6]),
                       "=r"(rb[7])
                     : "r"(tb));
    } else {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                     : "=r"(ra[0]), "=r"(ra[1]), "=r"(ra[2]), "=r"(ra[3]), "=r"(ra[4]), "=r"(ra[5]), "=r"(ra[6]),
                       "=r"(ra[7]), "=r"(ra[8]), "=r"(ra[9]), "=r"(ra[10]), "=r"(ra[11]), "=r"(ra[12]), "=r"(ra[13]),
                       "=r"(ra[14]), "=r"(ra[15])
                     : "r"(ta));
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                     : "=r"(rb[0]), "=r"(rb[1]), "=r"(rb[2]), "=r"(rb[3]), "=r"(rb[4]), "=r"(rb[5]), "=r"(rb[6]),
                       "=r"(rb[7]), "=r"(rb[8]), "=r"(rb[9]), "=r"(rb[10]), "=r"(rb[11]), "=r"(rb[12]), "=r"(rb[13]),
                       "=r"(rb[14]), "=r"(rb[15])
                     : "r"(tb));
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < kCols; ++i) v[i] = __uint_as_float(ra[i]) + __uint_as_float(rb[i]);
}

// NBUF H/R TMEM buffers; G epilogue warp groups.  G = 1: all 16 epilogue
// warps work on every tile, 8 observation columns each.  G = 2: two groups of
// 8 warps take alternate tiles, 16 columns each, so two tiles' epilogues
// overlap (each warp's per-tile chain of waits, TMEM round trips and arrivals
// is paid once per 16 columns instead of once per 8); this needs 3 buffers,
// two tiles in the epilogue while GEMM1 of the next one runs.
template <int NBUF, int G>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_glm_kernel(const __grid_constant__ CUtensorMap map_xk_hi, const __grid_constant__ CUtensorMap map_xk_lo,
                  const __grid_constant__ CUtensorMap map_xm_hi, const __grid_constant__ CUtensorMap map_xm_lo,
                  const float* __restrict__ params, TcGlmParams p) {
    static_assert(G == 1 || (G == 2 && NBUF == 3), "two epilogue groups need three H/R buffers");
    constexpr int kGroupWarps = kTcEpiWarps / G;          // arrivals per tile
    constexpr int kCols = kTcObs / (kGroupWarps / 4);     // observation columns per warp and tile
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int Fp = p.Fp;
    const int KB1 = tc_kblocks_used(p.F), MA = tc_matoms(Fp);
    const int xk_bytes = tc_xk_bytes(Fp), xm_bytes = tc_xm_bytes(Fp), stage_bytes = tc_stage_bytes(Fp);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kTcStages * stage_bytes);
    uint64_t* bar_xfull = bars;                    // [3]
    uint64_t* bar_xempty = bars + 3;               // [3]
    uint64_t* bar_d1full = bars + 6;               // [kTcMaxBufs]
    uint64_t* bar_rfull = bars + 9;                // [kTcMaxBufs]
    uint64_t* bar_d2full = bars + 12;
    uint64_t* bar_theta = bars + 13;
    uint64_t* bar_drained = bars + 14;             // every epilogue warp has read the accumulator run
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 15);
    constexpr int nbuf = NBUF;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // chain tiles fastest: concurrent CTAs share X ranges in L2
    const TcSplit sp = tc_split(p);
    const int b = blockIdx.y * gridDim.x + blockIdx.x;
    // with nact, CTAs beyond the live work leave before any barrier or TMEM exists
    if (p.nact && (*p.nact <= 0 || b >= sp.S * sp.nt)) return;
    const int ctile = p.nact ? b % sp.nt : blockIdx.x;
    const int split = p.nact ? b / sp.nt : blockIdx.y;
    const int t_begin = split * sp.tps;
    const int t_end = min(p.num_tiles, t_begin + sp.tps);
    const int ntiles = max(0, t_end - t_begin);

    if (threadIdx.x == 0) {
        for (int i = 0; i < kTcStages; ++i) {
            mbar_init(bar_xfull + i, 1);
            mbar_init(bar_xempty + i, 1);
        }
        for (int i = 0; i < kTcMaxBufs; ++i) {
            mbar_init(bar_d1full + i, 1);
            mbar_init(bar_rfull + i, kGroupWarps);
        }
        mbar_init(bar_d2full, 1);
        mbar_init(bar_theta, kTcEpiWarps);
        mbar_init(bar_drained, kTcEpiWarps);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(tmem_slot, 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int KC = 8 * KB1;
    const uint32_t col_thi = 0, col_tlo = p.col_tlo, col_d2 = p.col_d2, col_buf = p.col_buf;

    // waits of the producer and issuer warps, with warp-uniform verdicts
    auto wwait = [&](uint64_t* bar, uint32_t parity) -> bool {
        return __all_sync(0xffffffffu, mbar_wait(bar, parity, p.err));
    };
    auto wtest = [&](uint64_t* bar, uint32_t parity) -> bool {
        return __all_sync(0xffffffffu, mbar_test_wait(bar, parity));
    };
    if (warp == 0) {
        // ---------------- TMA producer (the whole warp; an elected lane issues) ----------------
        for (int i = 0; i < ntiles; ++i) {
            const int s = i % kTcStages;
            if (i >= kTcStages && !wwait(bar_xempty + s, ((i / kTcStages) - 1) & 1)) break;
            uint8_t* st = smem + s * stage_bytes;
            mbar_expect_tx_warp(bar_xfull + s, 2 * KB1 * (kTcObs * 32) + 2 * xm_bytes + kTcObs * 4);
            const int n0 = (t_begin + i) * kTcObs;
            if (p.xkpair) {
                // [K-block][hi, lo][32 rows][8 features] in one copy
                tma_load_4d_warp(st, &map_xk_hi, bar_xfull + s, 0, n0, 0, 0);
            } else if (p.xk3d) {
                // [K-block][32 rows][8 features] in one copy per view
                tma_load_3d_warp(st, &map_xk_hi, bar_xfull + s, 0, n0, 0);
                tma_load_3d_warp(st + xk_bytes, &map_xk_lo, bar_xfull + s, 0, n0, 0);
            } else {
                for (int kb = 0; kb < KB1; ++kb) {
                    tma_load_2d_warp(st + kb * (kTcObs * 32), &map_xk_hi, bar_xfull + s, kb * 8, n0);
                    tma_load_2d_warp(st + xk_bytes + kb * (kTcObs * 32), &map_xk_lo, bar_xfull + s, kb * 8, n0);
                }
            }
            for (int a = 0; a < MA; ++a) {
                tma_load_2d_warp(st + 2 * xk_bytes + a * (kTcObs * 128), &map_xm_hi, bar_xfull + s, a * 32, n0);
                tma_load_2d_warp(st + 2 * xk_bytes + xm_bytes + a * (kTcObs * 128), &map_xm_lo, bar_xfull + s,
                                 a * 32, n0);
            }
            bulk_load_warp(st + 2 * xk_bytes + 2 * xm_bytes, p.y + n0, kTcObs * 4, bar_xfull + s);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer (the whole warp; an elected lane issues) ----------------
        if (ntiles > 0) {
            const uint32_t id1 = idesc_tf32(kTcChains, kTcObs, 0);
            const uint32_t id1p = idesc_tf32(kTcChains, 2 * kTcObs, 0);
            const uint32_t id2 = idesc_tf32(kTcChains, Fp, 1);
            bool ok = wwait(bar_theta, 0);
            tc_fence_after();
            // GEMM2 of tile j.  The G^T accumulator in TMEM restarts every
            // kTcDrainTiles tiles: the epilogue drains it into FP32 registers
            // (round-to-nearest adds) so only a short run of tensor-core
            // accumulations ever lands in one TMEM value.  A restart waits for
            // every epilogue warp's drain of the previous run (bar_drained).
            // descriptors advance by whole 1 KB blocks: +64 in the address field (addr >> 4)
            auto gemm2 = [&](int j) {
                const int s = j % kTcStages, b = j % nbuf;
                const uint32_t xm = smem_u32(smem + s * stage_bytes + 2 * xk_bytes);
                uint32_t rhi = tmem + col_buf + b * 64, rlo = rhi + 32;
                uint64_t bh = sdesc_sw128b32(xm, kTcObs * 128, 512);
                uint64_t bl = sdesc_sw128b32(xm + xm_bytes, kTcObs * 128, 512);
                const uint32_t d2 = tmem + col_d2;
#pragma unroll
                for (int kk = 0; kk < kTcObs / 8; ++kk) {
                    const uint32_t first = (j % kTcDrainTiles == 0 && kk == 0) ? 0u : 1u;
                    mma_ts_warp(d2, rhi, bh, id2, first);
                    mma_ts_warp(d2, rlo, bh, id2, 1u);
                    mma_ts_warp(d2, rhi, bl, id2, 1u);
                    bh += 64;
                    bl += 64;
                    rhi += 8;
                    rlo += 8;
                }
                if ((j + 1) % kTcDrainTiles == 0 || j == ntiles - 1) mma_commit_warp(bar_d2full);
            };
            // whether GEMM2(j) may restart the accumulator (1), not yet (0), or a wait gave up (-1)
            auto restart_ok = [&](int j, bool block) -> int {
                if (!p.want_grad || j == 0 || j % kTcDrainTiles) return 1;
                const uint32_t par = ((j / kTcDrainTiles) - 1) & 1;
                if (!block) return wtest(bar_drained, par) ? 1 : 0;
                return wwait(bar_drained, par) ? 1 : -1;
            };
            // GEMM2 of tile j (when the gradient is wanted), then the release of its X stage
            auto finish = [&](int j) {
                tc_fence_after();
                if (p.want_grad) gemm2(j);
                mma_commit_warp(bar_xempty + (j % kTcStages));
            };
            auto gemm1 = [&](int i) -> bool {
                const int s = i % kTcStages, b = i % nbuf;
                if (!wwait(bar_xfull + s, (i / kTcStages) & 1)) return false;
                tc_fence_after();
                const uint32_t xk = smem_u32(smem + s * stage_bytes);
                const uint32_t d1 = tmem + col_buf + b * 64;
                uint32_t ahi = tmem + col_thi, alo = tmem + col_tlo;
                if (p.xkpair) {
                    // per K-block (2 KB: 32 X_hi rows, then 32 X_lo rows): Theta_hi x [X_hi | X_lo]
                    // into columns [0, 64) in one N = 64 MMA -- an N = 32 MMA costs as much -- and
                    // Theta_lo x X_hi into [32, 64); H^T = columns [0, 32) + [32, 64)
                    uint64_t bp = sdesc_sw32(xk, 16, 256);
                    for (int kb = 0; kb < KB1; ++kb) {
                        mma_ts_warp(d1, ahi, bp, id1p, kb > 0 ? 1u : 0u);
                        mma_ts_warp(d1 + 32, alo, bp, id1, 1u);
                        bp += 128;
                        ahi += 8;
                        alo += 8;
                    }
                    mma_commit_warp(bar_d1full + b);
                    return true;
                }
                uint64_t bh = sdesc_sw32(xk, 16, 256), bl = sdesc_sw32(xk + xk_bytes, 16, 256);
                mma_ts_warp(d1, ahi, bh, id1, 0u);
                mma_ts_warp(d1, ahi, bl, id1, 1u);
                mma_ts_warp(d1, alo, bh, id1, 1u);
                for (int kb = 1; kb < KB1; ++kb) {
                    bh += 64;
                    bl += 64;
                    ahi += 8;
                    alo += 8;
                    mma_ts_warp(d1, ahi, bh, id1, 1u);
                    mma_ts_warp(d1, ahi, bl, id1, 1u);
                    mma_ts_warp(d1, alo, bh, id1, 1u);
                }
                mma_commit_warp(bar_d1full + b);
                return true;
            };
            int g2 = 0;  // next tile whose GEMM2 / stage release is due
            if (G == 1) {
                // GEMM1(i), then tile i-1's GEMM2 as soon as its residuals are in TMEM
                for (int i = 0; ok && i < ntiles; ++i) {
                    if (!gemm1(i)) { ok = false; break; }
                    if (i > 0) {
                        if (!wwait(bar_rfull + (g2 % nbuf), (g2 / nbuf) & 1) || restart_ok(g2, true) < 0) {
                            ok = false;
                            break;
                        }
                        finish(g2++);
                    }
                }
            } else {
                for (int i = 0; ok && i < ntiles; ++i) {
                    // buffer i % nbuf is reused: the epilogue has to be done with tile i - nbuf
                    while (g2 <= i - nbuf) {
                        if (!wwait(bar_rfull + (g2 % nbuf), (g2 / nbuf) & 1) || restart_ok(g2, true) < 0) {
                            ok = false;
                            break;
                        }
                        finish(g2++);
                    }
                    if (!ok) break;
                    // GEMM2s that are ready go ahead of the next GEMM1: they free X stages for the producer
                    while (g2 < i && wtest(bar_rfull + (g2 % nbuf), (g2 / nbuf) & 1) && restart_ok(g2, false) == 1)
                        finish(g2++);
                    if (!gemm1(i)) { ok = false; break; }
                }
            }
            while (ok && g2 < ntiles) {
                if (!wwait(bar_rfull + (g2 % nbuf), (g2 / nbuf) & 1) || restart_ok(g2, true) < 0) break;
                finish(g2++);
            }
        }
    } else {
        // ---------------- epilogue: thread = chain (TMEM lane) ----------------
        // Every wait's verdict is made warp-uniform (a lane that gave up makes
        // the whole warp give up), so the warp's lanes always meet at the same
        // __syncwarp and the single-lane arrivals stay matched.
        auto warp_wait = [&](uint64_t* bar, uint32_t parity) -> bool {
            const bool r = mbar_wait(bar, parity, p.err);
            return __all_sync(0xffffffffu, r);
        };
        const int q = warp & 3;                 // TMEM lane quadrant
        const int e = (warp - 2) >> 2;          // which of the quadrant's four warps
        const int grp = G == 1 ? 0 : (e & 1);   // the tiles i with i % G == grp are this warp's
        const int slot = G == 1 ? e : (e >> 1); // its kCols observation columns of such a tile
        const int c_local = q * 32 + lane;
        const int c = ctile * kTcChains + c_local;
        const uint32_t lane_off = (uint32_t)(q * 32) << 16;
        // Theta row of this chain -> TF32 hi / lo in TMEM (A operand of GEMM1):
        // 8-column chunks f0 = 8*e + 32*k < KC belong to this warp
        for (int f0 = 8 * e; f0 < KC; f0 += 32) {
            uint32_t hi[8], lo[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int f = f0 + j;
                const float x = (c < p.C && f < p.F) ? kTcLog2e * __ldg(params + (size_t)c * p.F + f) : 0.0f;
                hi[j] = tf32_bits(x);
                lo[j] = tf32_bits(x - __uint_as_float(hi[j]));
            }
            tmem_st8(tmem + lane_off + col_thi + f0, hi);
            tmem_st8(tmem + lane_off + col_tlo + f0, lo);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar_theta);

        float ll = 0.0f;
        constexpr int kOwnCols = kTcMaxFp / 4;     // gradient columns owned by this warp
        float gacc[kOwnCols];
#pragma unroll
        for (int f = 0; f < kOwnCols; ++f) gacc[f] = 0.0f;
        // the k-th 16-column chunk of the gradient this warp owns (G = 1: 16 e + 64 k;
        // G = 2: group grp owns [64 grp, 64 grp + 64), its warps 32 columns each)
        auto own_col = [&](int k) { return G == 1 ? 16 * e + 64 * k : 64 * grp + 32 * slot + 16 * k; };
        int drained = 0;  // accumulator runs this warp has drained
        // Drain the next run of the G^T accumulator into registers; arrive when
        // a later run will restart the accumulator after it.
        auto drain_next = [&](bool arrive) -> bool {
            if (!warp_wait(bar_d2full, drained & 1)) return false;
            tc_fence_after();
#pragma unroll
            for (int k = 0; k < kOwnCols / 16; ++k) {
                const int f0 = own_col(k);
                if (f0 < Fp) {
                    float gv[16];
                    tmem_ld16(tmem + lane_off + col_d2 + f0, gv);
#pragma unroll
                    for (int j = 0; j < 16; ++j) gacc[16 * k + j] += gv[j];
                }
            }
            ++drained;
            if (arrive) {
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(bar_drained);
            }
            return true;
        };
        bool ok = ntiles > 0;
        for (int i = grp; ok && i < ntiles; i += G) {
            const int b = i % nbuf, s = i % kTcStages;
            // the y tile arrived with the X stage; d1_full(i) implies GEMM1(i) consumed stage s,
            // which the producer only refills after GEMM2(i) -- after this tile's r_full
            if (!warp_wait(bar_d1full + b, (i / nbuf) & 1)) { ok = false; break; }
            tc_fence_after();
            const int c0 = kCols * slot;
            const int n0 = (t_begin + i) * kTcObs + c0;
            const float* ys = reinterpret_cast<const float*>(smem + s * stage_bytes + 2 * xk_bytes + 2 * xm_bytes) + c0;
            const uint32_t d1 = tmem + lane_off + col_buf + b * 64 + c0;
            float h[kCols];
            if (p.xkpair) tmem_ld_cols_sum<kCols>(d1, d1 + 32, h);
            else tmem_ld_cols<kCols>(d1, h);
            // a tile with all its observations present and y known to be 0 / 1 needs no checks
            const bool fast = p.yvalid && (t_begin + i + 1) * kTcObs <= p.N;
            // residuals in runs of 8 columns (few live registers beside the gradient accumulators)
#pragma unroll
            for (int j8 = 0; j8 < kCols; j8 += 8) {
                uint32_t rh[8], rl[8];
#pragma unroll
                for (int j0 = 0; j0 < 8; j0 += 4) {
                    const float4 y4 = *reinterpret_cast<const float4*>(ys + j8 + j0);
                    const float yt[4] = {y4.x, y4.y, y4.z, y4.w};
#pragma unroll
                    for (int jj = 0; jj < 4; ++jj) {
                        const int j = j0 + jj;
                        const float hv = h[j8 + j];   // log2(e) eta
                        // log1p_exp(eta) = max(eta,0) + log1p(exp(-|eta|)); logistic(eta) from the same exp
                        // (math.jl:202-224), in base 2
                        const float ex = tc_ex2(-fabsf(hv));
                        const float onepe = 1.0f + ex;
                        const float lpe = fmaxf(hv, 0.0f) + tc_lg2(onepe);
                        const float inv = tc_rcp(onepe);
                        const float sig = hv >= 0.0f ? inv : ex * inv;
                        float r;
                        if (fast) {
                            const float yv = yt[jj];
                            ll += fmaf(yv, hv, -lpe);
                            r = yv - sig;
                        } else {
                            const bool live = n0 + j8 + j < p.N;
                            const float yv = live ? yt[jj] : 0.0f;
                            const bool sup = (yv == 0.0f) | (yv == 1.0f);
                            ll += live ? (sup ? fmaf(yv, hv, -lpe) : -INFINITY) : 0.0f;
                            r = live ? yv - sig : 0.0f;
                        }
                        const uint32_t hb = tf32_bits(r);
                        rh[j] = hb;
                        rl[j] = tf32_bits(r - __uint_as_float(hb));
                    }
                }
                tmem_st8(d1 + j8, rh);        // R_hi overwrites the consumed H^T columns
                tmem_st8(d1 + 32 + j8, rl);
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            // the first tile of run g (g >= 1) that this warp's group takes: drain
            // run g-1 (its GEMM2s ran while this tile's residuals were computed)
            // before the residuals are signalled
            if (p.want_grad && i >= kTcDrainTiles && i % kTcDrainTiles == grp && !drain_next(true)) {
                ok = false;
                break;
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_rfull + b);
        }
        if (ok && p.want_grad) {
            const int last = (ntiles - 1) / kTcDrainTiles;
            while (ok && drained <= last) ok = drain_next(drained < last);
        }
        // combine the four column quarters' log-likelihoods through shared memory
        float* ll_part = reinterpret_cast<float*>(tmem_slot + 4);   // [4][128]
        ll_part[e * kTcChains + c_local] = ll;
        asm volatile("bar.sync 1, %0;" ::"n"(kTcEpiThreads));
        if (ok) {
            if (e == 0 && c < p.C)
                p.part_ll[(size_t)split * sp.Cl + c] =
                    kTcLn2 * (((ll_part[c_local] + ll_part[kTcChains + c_local]) + ll_part[2 * kTcChains + c_local]) +
                              ll_part[3 * kTcChains + c_local]);
            if (p.want_grad && c < p.C) {
                float* dst = p.part_g + ((size_t)split * sp.Cl + c) * p.F;
#pragma unroll
                for (int k = 0; k < kOwnCols / 16; ++k) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int f = own_col(k) + j;
                        if (f < p.F) dst[f] = gacc[16 * k + j];
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

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct TcGlmPlan {
    bool enabled = false;
    int N = 0, F = 0, Fp = 0, C = 0, S = 0, tiles_per_split = 0, num_tiles = 0, ctiles = 0, sms = 0;
    float* xhi = nullptr;
    float* xlo = nullptr;
    float* part_ll = nullptr;
    float* part_g = nullptr;
    int* err = nullptr;
    const float* y = nullptr;     // N rounded up to whole observation tiles, zero padded
    int off = 0;
    float icpt_mu = 0, icpt_sigma = 1, coef_mu = 0, coef_sigma = 1;
    CUtensorMap map_xk_hi, map_xk_lo, map_xm_hi, map_xm_lo;
    bool xk3d = false;   // the K-major maps are 3-D (tc_make_map_kblocks)
    bool xkpair = false; // paired GEMM1: map_xk_hi is the 4-D hi/lo map (tc_make_map_kblocks_pair)
    bool yvalid = false; // every y is 0 or 1
    size_t smem = 0;
    int nbuf = 2;        // H/R TMEM buffers
    int groups = 1;      // epilogue warp groups (2 needs 3 buffers)
    bool wide = false;   // TMEM column plan (tc_columns)
};

inline std::string& tc_err_string() {
    static thread_local std::string s;
    return s;
}
inline const char* tc_glm_last_error() { return tc_err_string().c_str(); }

typedef CUresult (*PFN_encodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline PFN_encodeTiled tc_encode_fn() {
    static PFN_encodeTiled fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_encodeTiled>(p);
    }
    return fn;
}

// 2D fp32 map over a rows x Fp row-major matrix with box = box_cols x box_rows.
inline bool tc_make_map(CUtensorMap* m, float* base, int rows, int Fp, int box_cols, int box_rows,
                        CUtensorMapSwizzle swz) {
    PFN_encodeTiled enc = tc_encode_fn();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)Fp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)Fp * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// The K-major view as a 3-D map: (8 features, rows, K-blocks), the K-block
// stride 32 bytes inside a row, so one box of (8, 32 rows, kblocks) lands as
// [K-block][row][8 features] -- the layout of kblocks separate 2-D copies.
inline bool tc_make_map_kblocks(CUtensorMap* m, float* base, int rows, int Fp, int kblocks, int box_rows) {
    PFN_encodeTiled enc = tc_encode_fn();
    if (!enc) return false;
    cuuint64_t dims[3] = {8, (cuuint64_t)rows, (cuuint64_t)kblocks};
    cuuint64_t strides[2] = {(cuuint64_t)Fp * sizeof(float), 8 * sizeof(float)};
    cuuint32_t box[3] = {8, (cuuint32_t)box_rows, (cuuint32_t)kblocks};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// The paired K-major view as a 4-D map over X_hi and X_lo in one allocation
// (X_lo = X_hi + hl_stride bytes): (8 features, rows, hi/lo, K-blocks), so one
// box of (8, 32 rows, 2, kblocks) lands as [K-block][hi, lo][row][8 features]:
// per K-block 32 X_hi rows and then 32 X_lo rows, one N = 64 B operand.
inline bool tc_make_map_kblocks_pair(CUtensorMap* m, float* base, int rows, int Fp, int kblocks, int box_rows,
                                     size_t hl_stride) {
    PFN_encodeTiled enc = tc_encode_fn();
    if (!enc) return false;
    cuuint64_t dims[4] = {8, (cuuint64_t)rows, 2, (cuuint64_t)kblocks};
    cuuint64_t strides[3] = {(cuuint64_t)Fp * sizeof(float), (cuuint64_t)hl_stride, 8 * sizeof(float)};
    cuuint32_t box[4] = {8, (cuuint32_t)box_rows, 2, (cuuint32_t)kblocks};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

static __global__ void tc_split_x_kernel(const float* __restrict__ Xa, float* __restrict__ hi, float* __restrict__ lo,
                                  long long N, int F, int Fp) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * Fp) return;
    const long long n = i / Fp;
    const int f = (int)(i % Fp);
    const float x = f < F ? Xa[n * F + f] : 0.0f;
    const uint32_t h = tf32_bits(x);
    hi[i] = __uint_as_float(h);
    lo[i] = __uint_as_float(tf32_bits(x - __uint_as_float(h)));
}

// Observation split count S of the (chain tile, split) grid, one CTA per SM:
// the S that minimises ceil(ctiles * S / sms) waves x (per-CTA set-up + tiles per
// CTA).  A grid whose last wave is nearly empty costs a whole wave, and every
// extra wave repeats the set-up.  S is at most num_tiles / 8 (at least 8 tiles a
// CTA) and is rounded to the split count its tiles-per-split gives.
inline void tc_choose_split(int num_tiles, int ctiles, int sms, int* S_out, int* tiles_per_split_out) {
    int best = 1;
    double best_cost = 1e300;
    for (int s_try = 1; s_try <= std::max(1, num_tiles / 8); ++s_try) {
        const int tps = (num_tiles + s_try - 1) / s_try;
        const int s_eff = (num_tiles + tps - 1) / tps;
        const double waves = std::ceil((double)ctiles * s_eff / sms);
        const double cost = waves * (double)(kTcCtaOverheadTiles + tps);
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best = s_eff;
        }
    }
    *tiles_per_split_out = (num_tiles + best - 1) / best;
    *S_out = (num_tiles + *tiles_per_split_out - 1) / *tiles_per_split_out;
}

inline int tc_glm_setup(TcGlmPlan& t, const float* d_Xa, const float* d_y, int N, int F, int C, int off,
                        float icpt_mu, float icpt_sigma, float coef_mu, float coef_sigma, int sms,
                        std::vector<void*>* allocs) {
    t.enabled = false;
    const char* env = getenv("UT_DISABLE_TENSOR_CORES");
    if (env && env[0] == '1') return 0;
    int dev = 0, major = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    const int Fp = ((F + 15) / 16) * 16;
    if (major != 10 || Fp > kTcMaxFp || N < 1 || C < 1) return 0;  // the CUDA-core tiled path serves the rest
    t.N = N; t.F = F; t.Fp = Fp; t.C = C; t.off = off;
    t.icpt_mu = icpt_mu; t.icpt_sigma = icpt_sigma; t.coef_mu = coef_mu; t.coef_sigma = coef_sigma;
    t.num_tiles = (N + kTcObs - 1) / kTcObs;
    const int ctiles = (C + kTcChains - 1) / kTcChains;
    tc_choose_split(t.num_tiles, ctiles, sms, &t.S, &t.tiles_per_split);
    t.ctiles = ctiles;
    t.sms = sms;
    // partial rows for every split plan tc_split can pick: at most ctiles * S CTAs of 128 chains
    const size_t part_rows = (size_t)ctiles * t.S * kTcChains;
    auto alloc = [&](void** p, size_t bytes) {
        if (cudaMalloc(p, bytes) != cudaSuccess) return false;
        allocs->push_back(*p);
        return true;
    };
    const size_t xbytes = (size_t)N * Fp * sizeof(float);
    // X_hi and X_lo in one allocation, X_lo right after X_hi (the paired map spans both)
    if (!alloc((void**)&t.xhi, 2 * xbytes)) {
        tc_err_string() = "cudaMalloc failed";
        return 1;
    }
    t.xlo = t.xhi + (size_t)N * Fp;
    if (!alloc((void**)&t.part_ll, part_rows * sizeof(float)) ||
        !alloc((void**)&t.part_g, part_rows * F * sizeof(float)) || !alloc((void**)&t.err, sizeof(int))) {
        tc_err_string() = "cudaMalloc failed";
        return 1;
    }
    cudaMemset(t.err, 0, sizeof(int));
    {
        float* yp = nullptr;
        const size_t ybytes = (size_t)t.num_tiles * kTcObs * sizeof(float);
        if (!alloc((void**)&yp, ybytes)) {
            tc_err_string() = "cudaMalloc failed";
            return 1;
        }
        cudaMemset(yp, 0, ybytes);
        cudaMemcpy(yp, d_y, (size_t)N * sizeof(float), cudaMemcpyDeviceToDevice);
        t.y = yp;
        std::vector<float> hy((size_t)N);
        if (cudaMemcpy(hy.data(), d_y, (size_t)N * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess) {
            bool ok = true;
            for (float v : hy) ok = ok && (v == 0.0f || v == 1.0f);
            t.yvalid = ok;
        }
    }
    const long long total = (long long)N * Fp;
    tc_split_x_kernel<<<(unsigned)((total + 255) / 256), 256>>>(d_Xa, t.xhi, t.xlo, N, F, Fp);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        tc_err_string() = "splitting X into TF32 hi/lo failed";
        return 1;
    }
    if (!tc_make_map(&t.map_xk_hi, t.xhi, N, Fp, 8, kTcObs, CU_TENSOR_MAP_SWIZZLE_32B) ||
        !tc_make_map(&t.map_xk_lo, t.xlo, N, Fp, 8, kTcObs, CU_TENSOR_MAP_SWIZZLE_32B) ||
        !tc_make_map(&t.map_xm_hi, t.xhi, N, Fp, 32, kTcObs, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B) ||
        !tc_make_map(&t.map_xm_lo, t.xlo, N, Fp, 32, kTcObs, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B)) {
        tc_err_string() = "cuTensorMapEncodeTiled failed";
        return 1;
    }
    // the K-major view in one copy per tile and view, where the driver takes the
    // 3-D map (UT_TC_XK2D=1 keeps the per-K-block copies: a tuning knob)
    {
        const char* e2 = getenv("UT_TC_XK2D");
        CUtensorMap k3h, k3l;
        if (!(e2 && e2[0] == '1') && tc_make_map_kblocks(&k3h, t.xhi, N, Fp, tc_kblocks_used(F), kTcObs) &&
            tc_make_map_kblocks(&k3l, t.xlo, N, Fp, tc_kblocks_used(F), kTcObs)) {
            t.map_xk_hi = k3h;
            t.map_xk_lo = k3l;
            t.xk3d = true;
        }
        // paired GEMM1 (UT_TC_PAIRED=0 keeps the three N = 32 MMAs per K-block: a tuning knob)
        const char* ep = getenv("UT_TC_PAIRED");
        CUtensorMap kp;
        if (t.xk3d && !(ep && ep[0] == '0') &&
            tc_make_map_kblocks_pair(&kp, t.xhi, N, Fp, tc_kblocks_used(F), kTcObs, xbytes)) {
            t.map_xk_hi = kp;
            t.xkpair = true;
        }
    }
    // H/R buffers: as many as TMEM holds (tc_nbuf); UT_TC_BUFFERS=2 keeps two (a tuning knob)
    t.nbuf = tc_nbuf(F, Fp);
    const char* nb_env = getenv("UT_TC_BUFFERS");
    if (nb_env && nb_env[0] == '2') t.nbuf = 2;
    // UT_TC_LAYOUT=wide: the wide column plan (2 buffers), a tuning knob
    const char* lay_env = getenv("UT_TC_LAYOUT");
    if (lay_env && lay_env[0] == 'w' && 3 * Fp + 128 <= 512) {
        t.wide = true;
        t.nbuf = 2;
    }
    // one epilogue group; UT_TC_GROUPS=2 splits it in two on alternate tiles when 3 buffers fit
    // (a tuning knob: measured slower on config 3)
    t.groups = 1;
    const char* g_env = getenv("UT_TC_GROUPS");
    if (g_env && g_env[0] == '2' && t.nbuf == 3) t.groups = 2;
    t.smem = 1024 + (size_t)kTcStages * tc_stage_bytes(Fp) + 128 + 16 + 4 * kTcChains * sizeof(float);
    if (cudaFuncSetAttribute(tc_glm_kernel<2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(tc_glm_kernel<3, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(tc_glm_kernel<3, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem) !=
            cudaSuccess) {
        tc_err_string() = "shared-memory opt-in failed";
        return 1;
    }
    t.enabled = true;
    return 0;
}

// Prior terms + deterministic fold of the split partials, one 128-thread CTA
// per chain (thread = feature; F <= 128 on this path), fixed summation order.
static __global__ void __launch_bounds__(128) tc_reduce_kernel(const float* params, float* totals, float* grads,
                                                        TcGlmParams p, int off, float icpt_mu, float icpt_sigma,
                                                        float coef_mu, float coef_sigma) {
    const int c = blockIdx.x;
    if (c >= p.C || (p.nact && c >= *p.nact)) return;
    const TcSplit sp = tc_split(p);
    const int f = threadIdx.x, warp = f >> 5, lane = f & 31;
    const int F = p.F;
    __shared__ float wsum[4];
    float prior = 0.0f;
    if (f < F) {
        const float th = params[(size_t)c * F + f];
        const bool icpt = off && f == 0;
        const float mu = icpt ? icpt_mu : coef_mu, sg = icpt ? icpt_sigma : coef_sigma;
        prior = normal_logpdf(mu, sg, th);
        if (grads) {
            const float* pg = p.part_g + (size_t)c * F + f;
            const size_t stride = (size_t)sp.Cl * F;
            float gs = 0.0f;
#pragma unroll 8
            for (int s = 0; s < sp.S; ++s) gs += pg[s * stride];
            grads[(size_t)c * F + f] = gs - (th - mu) / (sg * sg);
        }
    }
    prior = warp_sum(prior);
    if (lane == 0) wsum[warp] = prior;
    __syncthreads();
    if (warp == 0) {
        float ll = 0.0f;
        for (int s = lane; s < sp.S; s += 32) ll += p.part_ll[(size_t)s * sp.Cl + c];
        ll = warp_sum(ll);
        if (lane == 0) totals[c] = ll + (((wsum[0] + wsum[1]) + wsum[2]) + wsum[3]);
    }
}

// nact (optional, device): evaluate only the first *nact chains of params
// (the totals / gradients of later chains are left untouched).
inline cudaError_t tc_glm_launch(const TcGlmPlan& t, const float* params, float* totals, float* grads,
                                 cudaStream_t st, const int* nact = nullptr) {
    TcGlmParams p;
    p.y = t.y; p.part_ll = t.part_ll; p.part_g = t.part_g; p.err = t.err;
    p.N = t.N; p.F = t.F; p.Fp = t.Fp; p.C = t.C;
    p.tiles_per_split = t.tiles_per_split; p.num_tiles = t.num_tiles; p.want_grad = grads ? 1 : 0;
    p.ctiles = t.ctiles; p.S = t.S; p.sms = t.sms;
    p.nact = nact;
    int cols[3];
    tc_columns(t.F, t.Fp, t.wide, cols);
    p.col_tlo = cols[0]; p.col_d2 = cols[1]; p.col_buf = cols[2];
    p.xk3d = t.xk3d ? 1 : 0;
    p.xkpair = t.xkpair ? 1 : 0;
    p.yvalid = t.yvalid ? 1 : 0;
    dim3 grid(t.ctiles, t.S);
    if (t.nbuf == 3 && t.groups == 2)
        tc_glm_kernel<3, 2><<<grid, kTcThreads, t.smem, st>>>(t.map_xk_hi, t.map_xk_lo, t.map_xm_hi, t.map_xm_lo,
                                                              params, p);
    else if (t.nbuf == 3)
        tc_glm_kernel<3, 1><<<grid, kTcThreads, t.smem, st>>>(t.map_xk_hi, t.map_xk_lo, t.map_xm_hi, t.map_xm_lo,
                                                              params, p);
    else
        tc_glm_kernel<2, 1><<<grid, kTcThreads, t.smem, st>>>(t.map_xk_hi, t.map_xk_lo, t.map_xm_hi, t.map_xm_lo,
                                                              params, p);
    tc_reduce_kernel<<<t.C, 128, 0, st>>>(params, totals, grads, p, t.off, t.icpt_mu, t.icpt_sigma, t.coef_mu,
                                          t.coef_sigma);
    return cudaGetLastError();
}

}  // namespace ut
