// kernels_subsys.cu -- partial trace, partial transpose, subsystem
// permutation and state compaction.
//
// Replaces include/qpp/internal/kernels/qubit/{ptrace,ptranspose,syspermute}.hpp
// and the generic paths of operations.hpp:1908-2514. ptranspose and
// syspermute are pure digit permutations of the (virtual) index: the output
// is written densely and each element gathers its source through a merged
// segment plan, so the result is bit-exact. ptrace sums diagonal blocks in
// FP64 whatever the state precision.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "kernels.hpp"

namespace qgpu {

template <typename R>
__global__ void __launch_bounds__(256)
    k_gather(const Cplx<R>* __restrict__ in, Cplx<R>* __restrict__ out,
             const __grid_constant__ SegPlan map) {
    const uint64_t nth = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t o = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
         o < map.count; o += nth)
        out[o] = in[seg_offset(map, o)];
}

template <typename R>
__global__ void __launch_bounds__(256)
    k_gather_outer(const Cplx<R>* __restrict__ in, Cplx<R>* __restrict__ out,
                   const __grid_constant__ SegPlan ma,
                   const __grid_constant__ SegPlan mb) {
    const uint64_t nth = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t o = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
         o < ma.count; o += nth) {
        Cplx<R> a = in[seg_offset(ma, o)], b = in[seg_offset(mb, o)];
        Cplx<R> r;
        r.x = a.x * b.x + a.y * b.y; // a * conj(b)
        r.y = a.y * b.x - a.x * b.y;
        out[o] = r;
    }
}

template <typename R, bool KET>
__device__ __forceinline__ void ptrace_term(const Cplx<R>* in, uint64_t a0,
                                            uint64_t b0, uint64_t t,
                                            double& sr, double& si) {
    Cplx<R> x = in[a0 + t];
    if (KET) {
        Cplx<R> y = in[b0 + t];
        double xr = x.x, xi = x.y, yr = y.x, yi = y.y;
        sr += xr * yr + xi * yi;
        si += xi * yr - xr * yi;
    } else {
        sr += double(x.x);
        si += double(x.y);
    }
}

// one thread per output element (many outputs)
template <typename R, bool KET>
__global__ void __launch_bounds__(256)
    k_ptrace_thread(const Cplx<R>* __restrict__ in, Cplx<R>* __restrict__ out,
                    const __grid_constant__ SegPlan ma,
                    const __grid_constant__ SegPlan mb,
                    const uint64_t* __restrict__ toff, uint64_t DS) {
    const uint64_t nth = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t o = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
         o < ma.count; o += nth) {
        uint64_t a0 = seg_offset(ma, o), b0 = KET ? seg_offset(mb, o) : 0;
        double sr = 0, si = 0;
        for (uint64_t a = 0; a < DS; ++a)
            ptrace_term<R, KET>(in, a0, b0, __ldg(&toff[a]), sr, si);
        Cplx<R> r;
        r.x = R(sr);
        r.y = R(si);
        out[o] = r;
    }
}

// one warp per output element (few outputs, long sums)
template <typename R, bool KET>
__global__ void __launch_bounds__(256)
    k_ptrace_warp(const Cplx<R>* __restrict__ in, Cplx<R>* __restrict__ out,
                  const __grid_constant__ SegPlan ma,
                  const __grid_constant__ SegPlan mb,
                  const uint64_t* __restrict__ toff, uint64_t DS) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t o = warp; o < ma.count; o += nwarps) {
        uint64_t a0 = seg_offset(ma, o), b0 = KET ? seg_offset(mb, o) : 0;
        double sr = 0, si = 0;
        for (uint64_t a = lane; a < DS; a += 32)
            ptrace_term<R, KET>(in, a0, b0, __ldg(&toff[a]), sr, si);
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            sr += __shfl_down_sync(0xffffffffu, sr, s);
            si += __shfl_down_sync(0xffffffffu, si, s);
        }
        if (lane == 0) {
            Cplx<R> r;
            r.x = R(sr);
            r.y = R(si);
            out[o] = r;
        }
    }
}

// ------------------------------------------------------------- launchers
static int blocks_for(qgpu_ctx* ctx, uint64_t work, int per_sm) {
    int blocks = grid_blocks(ctx, per_sm);
    uint64_t need = (work + 255) / 256;
    if (need < uint64_t(blocks)) blocks = int(std::max<uint64_t>(need, 1));
    return blocks;
}

void launch_gather(qgpu_ctx* ctx, qgpu_prec prec, const void* in, void* out,
                   const SegPlan& map) {
    if (map.count == 0) return;
    int b = blocks_for(ctx, map.count, 8);
    if (prec == QGPU_C128)
        k_gather<double><<<b, 256, 0, ctx->stream>>>(
            static_cast<const double2*>(in), static_cast<double2*>(out), map);
    else
        k_gather<float><<<b, 256, 0, ctx->stream>>>(
            static_cast<const float2*>(in), static_cast<float2*>(out), map);
    after_launch(ctx, "k_gather");
}

void launch_gather_outer(qgpu_ctx* ctx, qgpu_prec prec, const void* in,
                         void* out, const SegPlan& ma, const SegPlan& mb) {
    if (ma.count == 0) return;
    int b = blocks_for(ctx, ma.count, 8);
    if (prec == QGPU_C128)
        k_gather_outer<double><<<b, 256, 0, ctx->stream>>>(
            static_cast<const double2*>(in), static_cast<double2*>(out), ma, mb);
    else
        k_gather_outer<float><<<b, 256, 0, ctx->stream>>>(
            static_cast<const float2*>(in), static_cast<float2*>(out), ma, mb);
    after_launch(ctx, "k_gather_outer");
}

template <typename R>
static void ptr(qgpu_ctx* ctx, const void* in, void* out, const SegPlan& ma,
                const SegPlan& mb, const std::vector<uint64_t>& toff,
                bool is_ket) {
    uint64_t DS = toff.size();
    uint64_t* dt = static_cast<uint64_t*>(ctx_scratch(ctx, DS * sizeof(uint64_t)));
    QG_CUDA(cudaMemcpyAsync(dt, toff.data(), DS * sizeof(uint64_t),
                            cudaMemcpyHostToDevice, ctx->stream));
    const Cplx<R>* i = static_cast<const Cplx<R>*>(in);
    Cplx<R>* o = static_cast<Cplx<R>*>(out);
    // few outputs with long sums: a warp per output
    bool warp = ma.count < uint64_t(ctx->num_sms) * 2048 && DS >= 32;
    if (warp) {
        int b = blocks_for(ctx, ma.count * 32, 8);
        if (is_ket)
            k_ptrace_warp<R, true><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, dt, DS);
        else
            k_ptrace_warp<R, false><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, dt, DS);
    } else {
        int b = blocks_for(ctx, ma.count, 8);
        if (is_ket)
            k_ptrace_thread<R, true><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, dt, DS);
        else
            k_ptrace_thread<R, false><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, dt, DS);
    }
    after_launch(ctx, "k_ptrace");
}

void launch_ptrace(qgpu_ctx* ctx, qgpu_prec prec, const void* in, void* out,
                   const SegPlan& ma, const SegPlan& mb,
                   const std::vector<uint64_t>& toff, bool is_ket) {
    if (ma.count == 0) return;
    if (prec == QGPU_C128) ptr<double>(ctx, in, out, ma, mb, toff, is_ket);
    else ptr<float>(ctx, in, out, ma, mb, toff, is_ket);
}

} // namespace qgpu
