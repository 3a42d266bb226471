// kernels_fused.cu -- fused 6-qubit gate blocks on the 5th-generation tensor
// cores (tcgen05, kind::tf32) with split-TF32 (3xTF32) products and FP32
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
//   A (state tile)  -> tensor memory, one TMEM lane per group, hi and lo
//                      TF32 halves in columns [0,128) and [128,256);
//   B (block matrix) -> shared memory, K-major, 128-byte swizzle, hi and lo;
//   D (accumulator) -> tensor memory columns [256,384), FP32.
// D = A_hi B_hi + A_hi B_lo + A_lo B_hi (the dropped A_lo B_lo term and the
// TF32 rounding of the lo halves are ~2^-22 relative).
// Each of the 16 warps owns one TMEM lane quarter (warp % 4) and one quarter
// of the components (warp / 4): it loads 16 complex inputs per group, and
// after the MMA reads back and stores the same 16 outputs, so a thread
// writes exactly the addresses it read (in place, no staging).
//
// Every wait is bounded: on timeout the kernel records an error code in
// *err, skips the remaining tiles, frees its tensor memory and returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "kernels.hpp"

namespace qgpu {

struct Fused6Params {
    uint64_t ntiles;  // groups / 128
    int tb_sorted[6]; // target bit positions, ascending
    uint32_t off[64]; // element offset of block index m (big-endian over the block qubits)
    const float* B;   // 128 x 128 fp32, B[n * 128 + k]
    int* err;         // error flag (0 = ok)
};

constexpr uint32_t kSpinLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm volatile("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// byte offset of B element (n, k) in a K-major, 128B-swizzled tile of
// 128 rows (n) x 128 fp32 (k): four 32-element K atoms of 16 KB each.
__device__ __forceinline__ uint32_t b_swz(int n, int k) {
    int ka = k >> 5, kk = k & 31;
    int chunk = (kk >> 2) ^ (n & 7);
    return uint32_t(ka * 16384 + n * 128 + chunk * 16 + (kk & 3) * 4);
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

// kind::tf32, D fp32, A/B tf32, K-major, M = 128, N = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) |
                            ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %3, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %4, p;\n\t}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b), "r"(accumulate), "r"(kIdesc));
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, "
        "%10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, "
        "%27, %28, %29, %30, %31, %32};\n" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]),
        "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]),
        "r"(v[15]), "r"(v[16]), "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]),
        "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]),
        "r"(v[29]), "r"(v[30]), "r"(v[31]));
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

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (uint32_t it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity));
        if (done) return true;
    }
    return false;
}

__global__ void __launch_bounds__(512, 1)
    k_fused6_tc(float2* __restrict__ psi, const __grid_constant__ Fused6Params p) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int abort_sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quarter = warp & 3, kpart = warp >> 2;

    unsigned char* Bh = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* Bl = Bh + 65536;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
            smem_u32(&tmem_base_sh)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        abort_sh = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    // block matrix -> shared memory, split into TF32 hi and lo
    for (int e = tid; e < 128 * 128; e += blockDim.x) {
        int n = e >> 7, k = e & 127;
        float x = p.B[e];
        uint32_t hi = to_tf32(x);
        uint32_t lo = to_tf32(x - __uint_as_float(hi));
        uint32_t a = b_swz(n, k);
        *reinterpret_cast<uint32_t*>(Bh + a) = hi;
        *reinterpret_cast<uint32_t*>(Bl + a) = lo;
    }
    asm volatile("fence.proxy.async.shared::cta;");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tbase = tmem_base_sh;
    const uint32_t lane_off = uint32_t(quarter * 32) << 16;
    const uint32_t mb = smem_u32(&mbar);
    const uint32_t bh_addr = smem_u32(Bh), bl_addr = smem_u32(Bl);
    uint32_t parity = 0;

    // Software pipeline over this CTA's tiles (D double-buffered in TMEM
    // columns [256,384) and [384,512)):
    //   loads of tile i+1 are in flight while MMA(i) runs;
    //   MMA(i+1) runs while tile i is read back from TMEM and stored.
    auto tile_base = [&](uint64_t tile) {
        uint64_t base = tile * 128 + uint64_t(quarter * 32 + lane);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            int b = p.tb_sorted[i];
            uint64_t low = (uint64_t(1) << b) - 1;
            base = ((base & ~low) << 1) | (base & low);
        }
        return base;
    };
    auto load = [&](uint64_t base, float2 (&v)[16]) {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = psi[base + p.off[kpart * 16 + j]];
    };
    auto stage = [&](const float2 (&v)[16]) {
        uint32_t hi[32], lo[32];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            hi[2 * j] = to_tf32(v[j].x);
            lo[2 * j] = to_tf32(v[j].x - __uint_as_float(hi[2 * j]));
            hi[2 * j + 1] = to_tf32(v[j].y);
            lo[2 * j + 1] = to_tf32(v[j].y - __uint_as_float(hi[2 * j + 1]));
        }
        tmem_st32(tbase + lane_off + uint32_t(kpart * 32), hi);
        tmem_st32(tbase + lane_off + 128u + uint32_t(kpart * 32), lo);
        asm volatile("tcgen05.wait::st.sync.aligned;");
        asm volatile("tcgen05.fence::before_thread_sync;");
    };
    auto issue = [&](uint32_t dcol) { // after a __syncthreads
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t d = tbase + dcol;
#pragma unroll 1
            for (int ks = 0; ks < 16; ++ks) {
                uint32_t koff = uint32_t((ks >> 2) * 16384 + (ks & 3) * 32);
                uint64_t dh = b_desc(bh_addr + koff), dl = b_desc(bl_addr + koff);
                mma_tf32_ts(d, tbase + uint32_t(ks * 8), dh, ks > 0 ? 1u : 0u);
                mma_tf32_ts(d, tbase + uint32_t(ks * 8), dl, 1u);
                mma_tf32_ts(d, tbase + 128u + uint32_t(ks * 8), dh, 1u);
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    mb));
        }
    };

    uint64_t tile = blockIdx.x;
    if (tile < p.ntiles) {
        float2 v[16];
        uint64_t base_cur = tile_base(tile);
        load(base_cur, v);
        stage(v);
        __syncthreads();
        issue(256u);
        uint32_t dsel = 0;
        for (;;) {
            const uint64_t next = tile + gridDim.x;
            const bool has_next = next < p.ntiles;
            uint64_t base_next = 0;
            if (has_next) {
                base_next = tile_base(next);
                load(base_next, v);
            }
            bool ok = mbar_wait(mb, parity);
            if (!ok && lane == 0) {
                atomicExch(p.err, 1);
                abort_sh = 1;
            }
            __syncthreads();
            if (abort_sh) {
                // let MMAs still in flight drain (bounded) before freeing TMEM
                if (tid == 0) mbar_wait(mb, parity);
                break;
            }
            parity ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;");
            if (has_next) {
                stage(v);
                __syncthreads();
                issue(256u + 128u * (dsel ^ 1u));
            }
            uint32_t dv[32];
            tmem_ld32(tbase + lane_off + 256u + 128u * dsel + uint32_t(kpart * 32), dv);
            asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
            for (int j = 0; j < 16; ++j)
                psi[base_cur + p.off[kpart * 16 + j]] =
                    make_float2(__uint_as_float(dv[2 * j]), __uint_as_float(dv[2 * j + 1]));
            asm volatile("tcgen05.fence::before_thread_sync;");
            if (!has_next) break;
            tile = next;
            base_cur = base_next;
            dsel ^= 1u;
        }
    }
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tbase));
    }
}

// ------------------------------------------------------------- launcher
int* ctx_error_flag(qgpu_ctx* ctx) {
    if (!ctx->dev_flag) {
        QG_CUDA(cudaMalloc(&ctx->dev_flag, sizeof(int)));
        QG_CUDA(cudaMemset(ctx->dev_flag, 0, sizeof(int)));
    }
    return ctx->dev_flag;
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

void launch_fused6_tc(qgpu_ctx* ctx, void* data, int nbits, const int* tbits,
                      const float* dB) {
    if (nbits < 13)
        raise(QGPU_ERR_NOT_SUPPORTED, "qgpu fused", "fused tensor-core blocks need n >= 13");
    Fused6Params p;
    std::memset(&p, 0, sizeof(p));
    p.ntiles = (uint64_t(1) << (nbits - 6)) / 128;
    int s[6];
    for (int i = 0; i < 6; ++i) s[i] = tbits[i];
    std::sort(s, s + 6);
    for (int i = 0; i < 6; ++i) p.tb_sorted[i] = s[i];
    for (int m = 0; m < 64; ++m) {
        uint32_t o = 0;
        for (int j = 0; j < 6; ++j)
            if ((m >> (5 - j)) & 1) o |= uint32_t(1) << tbits[j];
        p.off[m] = o;
    }
    p.B = dB;
    p.err = ctx_error_flag(ctx);
    size_t smem = 2 * 65536 + 1024;
    static bool attr = false;
    if (!attr) {
        QG_CUDA(cudaFuncSetAttribute(k_fused6_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(smem)));
        attr = true;
    }
    int grid = int(std::min<uint64_t>(p.ntiles, uint64_t(ctx->num_sms)));
    k_fused6_tc<<<grid, 512, smem, ctx->stream>>>(static_cast<float2*>(data), p);
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
