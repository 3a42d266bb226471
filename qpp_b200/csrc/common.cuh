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

} // namespace qgpu
