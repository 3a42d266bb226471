// common.cuh -- device-side types shared by the kernels of libqpp_b200.
//
// Every op runs on a "virtual ket": a ket over dims is itself; a column-major
// D x D density matrix is a ket over the 2n subsystems [column digits, row
// digits] (column digit q has stride stride_q * D, row digit q stride_q).
// A gate group is the set of DA amplitudes that differ only in the target
// digits; its base offset comes from decomposing the group number over the
// "free" segments (runs of adjacent non-target, non-fixed subsystems merged
// into one mixed-radix digit).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace qgpu {

constexpr int kMaxSeg = 48; // merged free segments per plan

template <typename R>
struct CplxT;
template <>
struct CplxT<double> {
    using type = double2;
};
template <>
struct CplxT<float> {
    using type = float2;
};
template <typename R>
using Cplx = typename CplxT<R>::type;

// Decomposition of a dense group number g into a source offset:
// offset = fixed_off + sum_s digit_s(g) * stride[s], digits least significant
// first. When every size is a power of two, shift/mask replace div/mod.
struct SegPlan {
    uint64_t count;     // number of groups (product of sizes)
    uint64_t fixed_off; // offset contributed by fixed digits
    int nseg;
    int pow2;
    uint64_t size[kMaxSeg];
    uint64_t stride[kMaxSeg];
    uint8_t shift[kMaxSeg];
};

__host__ __device__ inline uint64_t seg_offset(const SegPlan& p, uint64_t g) {
    uint64_t off = p.fixed_off;
    if (p.pow2) {
        for (int s = 0; s < p.nseg; ++s) {
            off += (g & (p.size[s] - 1)) * p.stride[s];
            g >>= p.shift[s];
        }
    } else {
        for (int s = 0; s < p.nseg; ++s) {
            uint64_t q = g / p.size[s];
            off += (g - q * p.size[s]) * p.stride[s];
            g = q;
        }
    }
    return off;
}

// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11): 10 rounds of the
// published multipliers and Weyl key increments on a 128-bit counter.
__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = uint64_t(0xD2511F53u) * c[0];
        uint64_t p1 = uint64_t(0xCD9E8D57u) * c[2];
        uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
        uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Two uniforms in [0, 1) with 53 random bits each, for counter (a, b, c, d).
__host__ __device__ inline void philox_uniform2(uint64_t key, uint32_t a, uint32_t b,
                                                uint32_t c, uint32_t d, double& u0,
                                                double& u1) {
    uint32_t x[4] = {a, b, c, d};
    philox4x32_10(x, uint32_t(key), uint32_t(key >> 32));
    uint64_t m0 = (uint64_t(x[0]) << 21) ^ (uint64_t(x[1]) >> 11);
    uint64_t m1 = (uint64_t(x[2]) << 21) ^ (uint64_t(x[3]) >> 11);
    u0 = double(m0 & ((uint64_t(1) << 53) - 1)) * 0x1.0p-53;
    u1 = double(m1 & ((uint64_t(1) << 53) - 1)) * 0x1.0p-53;
}

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename C>
__device__ __forceinline__ C cfma(C a, C b, C acc) { // acc + a * b
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}

#ifdef __CUDACC__
// Asynchronous global -> shared copies of one amplitude (16 B for complex128
// through L2 only, 8 B for complex64) and their group fences.
template <typename C>
__device__ __forceinline__ void cp_async_elem(C* dst, const C* src) {
    const uint32_t a = uint32_t(__cvta_generic_to_shared(dst));
    if constexpr (sizeof(C) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(a), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
#endif

} // namespace qgpu
