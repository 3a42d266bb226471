// kernels_fused.cu -- fused 6-qubit gate blocks on the 5th-generation tensor
// cores (tcgen05, kind::f16) with split-FP16 (3 x FP16) products and FP32
// accumulation, for complex64 kets.
//
// No reference counterpart: Quantum++ applies one gate per pass
// (internal/kernels/qubit/apply.hpp:474-594 for k-qubit gates). Here runs of
// gates are fused on the host into one 64 x 64 complex block on six qubits
// and applied in a single read + write pass of the state.
//
// GEMM view of one pass: for every "group" g (the 64 amplitudes that differ
// only in the six target bits),
//     out_g[t] = sum_s U[t, s] in_g[s]
// written over reals with interleaved components k = 2 s + ri:
//     D[g, n] = sum_k A[g, k] B[k, n],   n = 2 t + ro,
//     B = [[Ur, Ui], [-Ui, Ur]] arranged so that D holds (re, im) pairs.
// Tile: 128 consecutive groups (M = 128), K = 128, N = 128.
//
// Split products. Every FP32 value x is written as hi + lo with hi = fp16(x)
// and lo = fp16(x - hi), and D = A_hi B_hi + A_hi B_lo + A_lo B_hi with FP32
// accumulation: 22 significant bits per operand, the same as the split-TF32
// form, at twice the tensor-core rate of kind::tf32. FP16 has a narrow
// exponent range, so the state is scaled by 2^eA with eA = 14 - ceil(log2
// |psi|) (every |amplitude| * 2^eA < 2^14; typical amplitudes of a 30-qubit
// state land near 2^-1, where both halves are normal numbers) and the block
// matrix by 2^6; the epilogue multiplies by 2^-(eA + 6). All scales are
// powers of two, so they are exact. |psi|^2 is an FP64 reduction on the
// device before the first block of a run (no host round trip, so a run can
// be captured in a CUDA graph).
//
// Layout per CTA (two CTAs per SM, 256 threads each):
//   A (state tile)  -> tensor memory: one TMEM lane per group; column m of
//                      [0, 64) holds amplitude m of the group as packed
//                      (re, im) fp16 hi halves, columns [64, 128) the lo
//                      halves;
//   B (block matrix) -> shared memory, K-major, 128-byte swizzle, hi and lo
//                      (2 x 32 KB);
//   D (accumulator) -> tensor memory columns [128, 256), FP32.
// 8 warps: warp w owns TMEM lane quarter w % 4 and half w / 4 of the 64
// amplitudes of each group; a thread loads its 32 complex inputs (one
// coalesced 256-byte row per warp and amplitude when the low state bits are
// not targets), and after the MMA reads back and stores the same 32 outputs,
// so every thread writes exactly the addresses it read (in place).
// Pipeline per CTA: the loads of tile i+1 are in flight while MMA(i) runs;
// the two co-resident CTAs of an SM interleave their load, MMA and epilogue
// phases.
//
// Every wait is bounded: on timeout the kernel records an error code in
// *err, waits (again bounded) for its own MMAs in flight, frees its tensor
// memory and returns.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "kernels.hpp"
#include "traj.hpp"

namespace qgpu {

struct Fused6Params {
    uint64_t ntiles;       // groups / 128
    int tb_sorted[6];      // target bit positions, ascending
    uint32_t off[64];      // element offset of block index m (big-endian over the block qubits)
    uint32_t loc_m[64];    // stage-local index of block index m
    uint32_t run_off[64];  // element offset of contiguous run j from the tile base
    uint32_t nruns;        // contiguous runs per tile (2^(13 - r))
    uint32_t run_bytes;    // bytes per run (2^r * 8, at least 1 KB)
    uint8_t g_pos[7];      // state bit of group bit i (the 7 lowest non-target bits)
    uint8_t g_loc[7];      // stage-local bit of group bit i
    const unsigned char* Bimg; // 64 KB shared-memory image of the block (fused6_images)
    const double* norm2;   // device word: |psi|^2 (sets the fp16 scale)
    int* err;              // error flag (0 = ok)
    uint32_t spin_limit;   // iterations of each wait
    uint32_t stall_first;  // test hook: the first wait is on a barrier nothing completes
};

constexpr uint32_t kSpinLimit = 1u << 26;
constexpr int kF6Threads = 384;      // 12 warps: producer, MMA, 2 idle, 4 converter, 4 epilogue
constexpr int kBScaleExp = 6;
constexpr uint32_t kStageBytes = 65536; // one tile: 128 groups x 64 amplitudes x 8 B
// B (64 KB, hi + lo) and two stages, 1 KB alignment slack: one CTA per SM,
// which then owns all 512 tensor-memory columns
constexpr size_t kF6Smem = 1024 + 65536 + 2 * size_t(kStageBytes);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of B element (n, k) in a K-major, 128B-swizzled tile of
// 128 rows (n) x 128 fp16 (k): two 64-element K atoms of 16 KB each.
__device__ __forceinline__ uint32_t b_swz16(int n, int k) {
    int ka = k >> 6, kk = k & 63;
    int chunk = (kk >> 3) ^ (n & 7);
    return uint32_t(ka * 16384 + n * 128 + chunk * 16 + (kk & 7) * 2);
}

__device__ __forceinline__ uint64_t b_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFF);        // start address
    d |= uint64_t(1) << 16;                      // leading byte offset (16 B, unused for SW128 K-major)
    d |= uint64_t(1024 >> 4) << 32;              // stride byte offset: 8 rows x 128 B
    d |= uint64_t(1) << 46;                      // descriptor version (sm_100)
    d |= uint64_t(2) << 61;                      // 128-byte swizzle
    return d;
}

// kind::f16, D fp32, A/B fp16, both K-major, M = 128, N = 128
constexpr uint32_t kIdescF16 = (1u << 4) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_f16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b,
                                           uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %3, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %4, p;\n\t}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b), "r"(accumulate), "r"(kIdescF16));
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, "
        "%10, %11, %12, %13, %14, %15, %16};\n" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]),
        "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]),
        "r"(v[15]));
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
        "%10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, "
        "%27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
          "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
          "=r"(v[31])
        : "r"(taddr));
}

// (x0, x1) -> packed fp16 hi halves and packed fp16 residuals; x0 in the low
// 16 bits (the even K element of the TMEM column).
__device__ __forceinline__ void split2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
    __half2 h = __floats2half2_rn(x0, x1);
    float2 hf = __half22float2(h);
    __half2 l = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
    hi = *reinterpret_cast<uint32_t*>(&h);
    lo = *reinterpret_cast<uint32_t*>(&l);
}

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity));
    return done != 0;
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_commit(uint32_t mbar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
        : "memory");
}

// Shared state of one CTA's pipeline. Barriers (phase k completes with the
// k-th event): full[s] stage s landed (bulk copies, tx bytes); empty[s] the
// converter warps released stage s; afull[a] the converter wrote A buffer a;
// aempty[a] the MMAs reading A buffer a finished; dfull[d] the MMAs writing D
// buffer d finished; dempty[d] the epilogue warps read D buffer d.
struct F6Shared {
    uint64_t full[2], empty[2], afull[2], aempty[2], dfull[2], dempty[2], drain, stall, bmat;
    uint32_t tmem_base;
    int abort;
};

// Bounded wait on phase `parity` of `bar`: false when the limit ran out (the
// CTA is then marked aborted and *err set) or another role aborted.
__device__ __forceinline__ bool f6_wait(F6Shared& S, uint32_t bar, uint32_t parity,
                                        uint32_t limit, int* err) {
    for (uint32_t it = 0; it < limit; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 255u) == 255u && *reinterpret_cast<volatile int*>(&S.abort)) return false;
    }
    *reinterpret_cast<volatile int*>(&S.abort) = 1;
    atomicExch(err, 1);
    return false;
}

__global__ void __launch_bounds__(kF6Threads, 1)
    k_fused6_tc(float2* __restrict__ psi, const __grid_constant__ Fused6Params p) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) F6Shared S;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    unsigned char* Bh = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* Bl = Bh + 32768;
    unsigned char* stage0 = Bh + 65536;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
            smem_u32(&S.tmem_base)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        S.abort = 0;
        for (int i = 0; i < 2; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.full[i])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&S.empty[i])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&S.afull[i])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.aempty[i])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.dfull[i])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&S.dempty[i])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.drain)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.stall)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bmat)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tbase = S.tmem_base;
    const uint64_t my_tiles =
        p.ntiles > blockIdx.x ? (p.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const uint32_t limit = p.spin_limit;

    // group index (tile * 128) with zero bits inserted at the target bits
    auto tile_base = [&](uint64_t tile) {
        uint64_t base = tile * 128;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            int b = p.tb_sorted[i];
            uint64_t low = (uint64_t(1) << b) - 1;
            base = ((base & ~low) << 1) | (base & low);
        }
        return base;
    };

    if (warp == 0) {
        // ---- producer: each tile is nruns contiguous runs, one bulk copy each
        if (lane == 0) {
            // the block matrix image (hi and lo halves, swizzled) in one copy
            const uint32_t bb = smem_u32(&S.bmat);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bb),
                         "r"(65536u)
                         : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                "[%0], [%1], %2, [%3];" ::"r"(smem_u32(Bh)),
                "l"(p.Bimg), "r"(65536u), "r"(bb)
                : "memory");
            uint64_t issued = 0;
            for (uint64_t i = 0; i < my_tiles; ++i) {
                const uint32_t st = uint32_t(i & 1), u = uint32_t(i >> 1);
                if (u >= 1 && !f6_wait(S, smem_u32(&S.empty[st]), (u - 1) & 1u, limit, p.err))
                    break;
                const uint64_t base = tile_base(blockIdx.x + i * gridDim.x);
                const uint32_t fb = smem_u32(&S.full[st]);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                             "r"(kStageBytes)
                             : "memory");
                const uint32_t dst = smem_u32(stage0) + st * kStageBytes;
                for (uint32_t j = 0; j < p.nruns; ++j)
                    asm volatile(
                        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                        "[%0], [%1], %2, [%3];" ::"r"(dst + j * p.run_bytes),
                        "l"(psi + base + p.run_off[j]), "r"(p.run_bytes), "r"(fb)
                        : "memory");
                ++issued;
            }
            // copies still in flight land before the CTA exits (bounded)
            f6_wait(S, bb, 0u, kSpinLimit, p.err);
            for (uint64_t i = issued > 2 ? issued - 2 : 0; i < issued; ++i)
                f6_wait(S, smem_u32(&S.full[i & 1]), uint32_t(i >> 1) & 1u, kSpinLimit, p.err);
        }
    } else if (warp == 1) {
        // ---- MMA issuer: D[d] = A_hi B_hi + A_hi B_lo + A_lo B_hi
        if (lane == 0) {
            const uint32_t bh = smem_u32(Bh), bl = smem_u32(Bl);
            const bool have_b = f6_wait(S, smem_u32(&S.bmat), 0u, limit, p.err);
            for (uint64_t i = 0; have_b && i < my_tiles; ++i) {
                const uint32_t b = uint32_t(i & 1), u = uint32_t(i >> 1);
                if (!f6_wait(S, smem_u32(&S.afull[b]), u & 1u, limit, p.err)) break;
                if (u >= 1 && !f6_wait(S, smem_u32(&S.dempty[b]), (u - 1) & 1u, limit, p.err))
                    break;
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t a = tbase + b * 128u, d = tbase + 256u + b * 128u;
#pragma unroll 1
                for (int ks = 0; ks < 8; ++ks) {
                    uint32_t koff = uint32_t((ks >> 2) * 16384 + (ks & 3) * 32);
                    uint64_t dh = b_desc(bh + koff), dl = b_desc(bl + koff);
                    mma_f16_ts(d, a + uint32_t(ks * 8), dh, ks > 0 ? 1u : 0u);
                    mma_f16_ts(d, a + uint32_t(ks * 8), dl, 1u);
                    mma_f16_ts(d, a + 64u + uint32_t(ks * 8), dh, 1u);
                }
                mbar_commit(smem_u32(&S.aempty[b]));
                mbar_commit(smem_u32(&S.dfull[b]));
            }
            // every MMA this thread issued has finished before TMEM is freed
            mbar_commit(smem_u32(&S.drain));
            f6_wait(S, smem_u32(&S.drain), 0u, kSpinLimit, p.err);
        }
    } else if (warp >= 4 && warp < 8) {
        // ---- converters: stage -> fp16 hi/lo -> A buffer (one TMEM lane per group)
        const int g = (warp & 3) * 32 + lane;
        uint32_t loc_g = 0;
#pragma unroll
        for (int i = 0; i < 7; ++i) loc_g |= uint32_t((g >> i) & 1) << p.g_loc[i];
        // scale from |psi|^2: |a| * 2^eA < 2^14 for every amplitude
        int eA = 14;
        {
            const double n2 = p.norm2 ? *p.norm2 : 1.0;
            if (n2 > 0.0 && n2 < 1e300) {
                int e2;
                frexp(n2, &e2); // n2 < 2^e2, so |psi| < 2^ceil(e2 / 2)
                eA = 14 - ((e2 + 1) >> 1);
            }
            eA = max(-100, min(100, eA));
        }
        const float sa = __int_as_float((127 + eA) << 23);
        const uint32_t lane_off = uint32_t((warp & 3) * 32) << 16;
        bool stall = p.stall_first != 0;
        for (uint64_t i = 0; i < my_tiles; ++i) {
            const uint32_t b = uint32_t(i & 1), u = uint32_t(i >> 1);
            if (stall) {
                f6_wait(S, smem_u32(&S.stall), 0u, limit, p.err); // never completes
                break;
            }
            if (!f6_wait(S, smem_u32(&S.full[b]), u & 1u, limit, p.err)) break;
            if (u >= 1 && !f6_wait(S, smem_u32(&S.aempty[b]), (u - 1) & 1u, limit, p.err)) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const float2* stg = reinterpret_cast<const float2*>(stage0 + b * kStageBytes);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                uint32_t hi[16], lo[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const float2 v = stg[loc_g + p.loc_m[c * 16 + j]];
                    split2(v.x * sa, v.y * sa, hi[j], lo[j]);
                }
                const uint32_t col = b * 128u + uint32_t(c * 16);
                tmem_st16(tbase + lane_off + col, hi);
                tmem_st16(tbase + lane_off + 64u + col, lo);
            }
            // the stage's reads are done: the producer may refill it
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&S.empty[b]));
            asm volatile("tcgen05.wait::st.sync.aligned;");
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&S.afull[b]));
        }
    } else if (warp >= 8) {
        // ---- epilogue: D buffer -> scaled FP32 -> the group's addresses in HBM
        const int g = (warp & 3) * 32 + lane;
        uint64_t base_low = 0;
#pragma unroll
        for (int i = 0; i < 7; ++i) base_low |= uint64_t((g >> i) & 1) << p.g_pos[i];
        int eA = 14;
        {
            const double n2 = p.norm2 ? *p.norm2 : 1.0;
            if (n2 > 0.0 && n2 < 1e300) {
                int e2;
                frexp(n2, &e2);
                eA = 14 - ((e2 + 1) >> 1);
            }
            eA = max(-100, min(100, eA));
        }
        const float inv = __int_as_float((127 - eA - kBScaleExp) << 23); // 2^-(eA + 6)
        const uint32_t lane_off = uint32_t((warp & 3) * 32) << 16;
        for (uint64_t i = 0; i < my_tiles; ++i) {
            const uint32_t b = uint32_t(i & 1), u = uint32_t(i >> 1);
            if (!f6_wait(S, smem_u32(&S.dfull[b]), u & 1u, limit, p.err)) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            float2* out = psi + tile_base(blockIdx.x + i * gridDim.x) + base_low;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                uint32_t dv[32];
                tmem_ld32(tbase + lane_off + 256u + b * 128u + uint32_t(c * 32), dv);
                asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    out[p.off[c * 16 + j]] = make_float2(__uint_as_float(dv[2 * j]) * inv,
                                                         __uint_as_float(dv[2 * j + 1]) * inv);
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&S.dempty[b]));
        }
    }
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tbase));
    }
}

// ------------------------------------------------------------- launcher
// Device words of the context: [0] the bounded-wait error flag, [8] the
// squared norm read by the fused kernel.
int* ctx_error_flag(qgpu_ctx* ctx) {
    if (!ctx->dev_flag) {
        QG_CUDA(cudaMalloc(&ctx->dev_flag, 64));
        QG_CUDA(cudaMemset(ctx->dev_flag, 0, 64));
    }
    return ctx->dev_flag;
}

double* ctx_norm_slot(qgpu_ctx* ctx) {
    return reinterpret_cast<double*>(reinterpret_cast<char*>(ctx_error_flag(ctx)) + 8);
}

// Builds B[n * 128 + k] from the 64 x 64 complex block U (column-major):
// n = 2 t + ro (output), k = 2 s + ri (input).
void fused6_matrix(const cd* U, float* B) {
    for (int t = 0; t < 64; ++t)
        for (int s = 0; s < 64; ++s) {
            cd u = U[t + 64 * s];
            float ur = float(u.real()), ui = float(u.imag());
            B[(2 * t) * 128 + 2 * s] = ur;       // re <- re
            B[(2 * t) * 128 + 2 * s + 1] = -ui;  // re <- im
            B[(2 * t + 1) * 128 + 2 * s] = ui;   // im <- re
            B[(2 * t + 1) * 128 + 2 * s + 1] = ur;
        }
}

// 64 KB shared-memory images of `nblocks` block matrices (fp32 128 x 128,
// fused6_matrix): each scaled by 2^6, split into fp16 hi and lo halves and
// laid out K-major with the 128-byte swizzle at the offsets the kernel's
// descriptors address (hi in the first 32 KB, lo in the second), so a pass
// loads its matrix with one bulk copy.
__global__ void __launch_bounds__(256)
    k_fused6_image(const float* __restrict__ B, unsigned char* __restrict__ img) {
    const float* b = B + size_t(blockIdx.x) * 128 * 128;
    unsigned char* o = img + size_t(blockIdx.x) * 65536;
    for (int e = threadIdx.x; e < 128 * 128; e += blockDim.x) {
        int n = e >> 7, k = e & 127;
        float x = b[e] * float(1 << kBScaleExp);
        __half hi = __float2half_rn(x);
        __half lo = __float2half_rn(x - __half2float(hi));
        uint32_t a = b_swz16(n, k);
        *reinterpret_cast<__half*>(o + a) = hi;
        *reinterpret_cast<__half*>(o + 32768 + a) = lo;
    }
}

void fused6_images(qgpu_ctx* ctx, const float* dB, void* dimg, int nblocks) {
    if (nblocks <= 0) return;
    k_fused6_image<<<nblocks, 256, 0, ctx->stream>>>(dB, static_cast<unsigned char*>(dimg));
    after_launch(ctx, "k_fused6_image");
}

// |psi|^2 of the complex64 ket into the context's norm slot (stream order;
// read by the fused passes that follow).
const double* fused_norm_prepare(qgpu_ctx* ctx, const void* data, uint64_t n) {
    double* slot = ctx_norm_slot(ctx);
    reduce_norm2_device(ctx, QGPU_C64, data, n, slot);
    return slot;
}

void launch_fused6_tc(qgpu_ctx* ctx, void* data, int nbits, const int* tbits,
                      const void* img, const double* norm2) {
    if (nbits < 13)
        raise(QGPU_ERR_NOT_SUPPORTED, "qgpu fused", "fused tensor-core blocks need n >= 13");
    Fused6Params p;
    std::memset(&p, 0, sizeof(p));
    p.ntiles = (uint64_t(1) << (nbits - 6)) / 128;
    int s[6];
    for (int i = 0; i < 6; ++i) s[i] = tbits[i];
    std::sort(s, s + 6);
    for (int i = 0; i < 6; ++i) p.tb_sorted[i] = s[i];
    // tile bits: the six targets and the seven lowest other bits, ascending;
    // stage-local bit i holds tile bit tpos[i]
    bool is_t[64] = {};
    for (int i = 0; i < 6; ++i) is_t[s[i]] = true;
    int tpos[13], nt = 0, ng = 0;
    for (int b = 0; b < nbits && nt < 13; ++b) {
        if (is_t[b]) {
            tpos[nt++] = b;
        } else if (ng < 7) {
            p.g_pos[ng] = uint8_t(b);
            p.g_loc[ng++] = uint8_t(nt);
            tpos[nt++] = b;
        }
    }
    int r = 0; // the low r tile bits are state bits 0..r-1: runs of 2^r amplitudes
    while (r < 13 && tpos[r] == r) ++r;
    p.nruns = 1u << (13 - r);
    p.run_bytes = (1u << r) * 8u;
    for (uint32_t j = 0; j < p.nruns; ++j) {
        uint32_t o = 0;
        for (int i = r; i < 13; ++i)
            if ((j >> (i - r)) & 1u) o |= 1u << tpos[i];
        p.run_off[j] = o;
    }
    auto local_of = [&](int bit) {
        for (int i = 0; i < 13; ++i)
            if (tpos[i] == bit) return i;
        return 0;
    };
    for (int m = 0; m < 64; ++m) {
        uint32_t o = 0, l = 0;
        for (int j = 0; j < 6; ++j)
            if ((m >> (5 - j)) & 1) {
                o |= uint32_t(1) << tbits[j];
                l |= uint32_t(1) << local_of(tbits[j]);
            }
        p.off[m] = o;
        p.loc_m[m] = l;
    }
    p.Bimg = static_cast<const unsigned char*>(img);
    p.norm2 = norm2;
    p.err = ctx_error_flag(ctx);
    p.spin_limit = ctx->wait_limit ? ctx->wait_limit : kSpinLimit;
    p.stall_first = ctx->stall_next ? 1u : 0u;
    ctx->stall_next = 0;
    ensure_smem(reinterpret_cast<const void*>(k_fused6_tc), kF6Smem);
    int grid = int(std::min<uint64_t>(p.ntiles, uint64_t(ctx->num_sms)));
    k_fused6_tc<<<grid, kF6Threads, kF6Smem, ctx->stream>>>(static_cast<float2*>(data), p);
    after_launch(ctx, "k_fused6_tc");
}

int fused_error(qgpu_ctx* ctx) {
    int h = 0;
    int* f = ctx_error_flag(ctx);
    QG_CUDA(cudaMemcpyAsync(&h, f, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    QG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h) QG_CUDA(cudaMemsetAsync(f, 0, sizeof(int), ctx->stream));
    return h;
}

} // namespace qgpu
