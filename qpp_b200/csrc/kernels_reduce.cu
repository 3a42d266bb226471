// kernels_reduce.cu -- FP64 reductions, sampling search, projection,
// scaling, conversion and the seeded Gaussian generator.
//
// FP64 stays on the GPU for the three steps that need it whatever the state
// precision: norms / traces for renormalisation (functions.hpp:304-333), the
// probability prefix sums of measurement sampling (instruments.hpp:746-818)
// and the diagonal sums of ptrace. Every reduction is deterministic: a fixed
// grid, per-block tree sums into the context scratch, then one block summing
// the partials in order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "kernels.hpp"

namespace qgpu {

constexpr int kRedBlocks = 1184; // 148 SMs x 8
constexpr int kRedThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v += __shfl_down_sync(0xffffffffu, v, s);
    return v;
}

// Block-wide sum of NC values per thread; result valid in thread 0.
template <int NC>
__device__ __forceinline__ void block_sum(double (&v)[NC]) {
    __shared__ double sh[NC][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < NC; ++c) v[c] = warp_sum(v[c]);
    if (lane == 0)
#pragma unroll
        for (int c = 0; c < NC; ++c) sh[c][w] = v[c];
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            v[c] = lane < nw ? sh[c][lane] : 0.0;
            v[c] = warp_sum(v[c]);
        }
    }
    __syncthreads();
}

template <typename R>
__global__ void __launch_bounds__(kRedThreads)
    k_norm2_partial(const Cplx<R>* __restrict__ x, uint64_t n,
                    double* __restrict__ partial) {
    double v[1] = {0.0};
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += uint64_t(gridDim.x) * blockDim.x) {
        Cplx<R> a = x[i];
        v[0] += double(a.x) * a.x + double(a.y) * a.y;
    }
    block_sum<1>(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

template <typename R>
__global__ void __launch_bounds__(kRedThreads)
    k_strided_partial(const Cplx<R>* __restrict__ x, uint64_t n,
                      uint64_t stride, double* __restrict__ partial) {
    double v[2] = {0.0, 0.0};
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += uint64_t(gridDim.x) * blockDim.x) {
        Cplx<R> a = x[i * stride];
        v[0] += a.x;
        v[1] += a.y;
    }
    block_sum<2>(v);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = v[0];
        partial[2 * blockIdx.x + 1] = v[1];
    }
}

template <typename R>
__global__ void __launch_bounds__(kRedThreads)
    k_inner_partial(const Cplx<R>* __restrict__ a, const Cplx<R>* __restrict__ b,
                    uint64_t n, double* __restrict__ partial) {
    double v[2] = {0.0, 0.0};
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += uint64_t(gridDim.x) * blockDim.x) {
        Cplx<R> x = a[i], y = b[i];
        v[0] += double(x.x) * y.x + double(x.y) * y.y; // conj(x) * y
        v[1] += double(x.x) * y.y - double(x.y) * y.x;
    }
    block_sum<2>(v);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = v[0];
        partial[2 * blockIdx.x + 1] = v[1];
    }
}

// Sum `nb` partials of `nc` components each (component-major output).
__global__ void __launch_bounds__(kRedThreads)
    k_sum_partials(const double* __restrict__ partial, int nb, int nc,
                   double* __restrict__ out) {
    for (int c = 0; c < nc; ++c) {
        double v[1] = {0.0};
        for (int b = threadIdx.x; b < nb; b += blockDim.x) v[0] += partial[size_t(b) * nc + c];
        block_sum<1>(v);
        if (threadIdx.x == 0) out[c] = v[0];
    }
}

// Marginals: block (bx, m) sums the weights of element base(g) + off[m] over
// groups g = bx, bx + gridDim.x, ... ; partial[m * gridDim.x + bx].
template <typename R, bool DIAG>
__global__ void __launch_bounds__(kRedThreads)
    k_marginal_partial(const Cplx<R>* __restrict__ x,
                       const __grid_constant__ SegPlan outer,
                       const uint64_t* __restrict__ off, uint64_t diag_mul,
                       double* __restrict__ partial) {
    const int m = blockIdx.y;
    const uint64_t om = off[m];
    double v[1] = {0.0};
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
         g < outer.count; g += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t e = seg_offset(outer, g) + om;
        if (DIAG) {
            v[0] += double(x[e * diag_mul].x);
        } else {
            Cplx<R> a = x[e];
            v[0] += double(a.x) * a.x + double(a.y) * a.y;
        }
    }
    block_sum<1>(v);
    if (threadIdx.x == 0) partial[size_t(m) * gridDim.x + blockIdx.x] = v[0];
}

// Contiguous-chunk weight sums for the sampling search.
template <typename R, bool DIAG>
__global__ void __launch_bounds__(kRedThreads)
    k_chunk_sums(const Cplx<R>* __restrict__ x, uint64_t D, uint64_t chunk,
                 double* __restrict__ partial) {
    uint64_t lo = uint64_t(blockIdx.x) * chunk, hi = min(D, lo + chunk);
    double v[1] = {0.0};
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        if (DIAG) {
            v[0] += double(x[i * (D + 1)].x);
        } else {
            Cplx<R> a = x[i];
            v[0] += double(a.x) * a.x + double(a.y) * a.y;
        }
    }
    block_sum<1>(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

// Many draws at once: block b scans chunk [lo_b, lo_b + chunk) (clipped to D)
// for the first index whose running inclusive sum reaches thr[b]; the last
// index of the chunk holding weight if rounding leaves none.
template <typename R, bool DIAG>
__global__ void __launch_bounds__(256)
    k_chunk_scan_many(const Cplx<R>* __restrict__ x, uint64_t D, uint64_t chunk,
                      const uint64_t* __restrict__ lo_arr, const double* __restrict__ thr_arr,
                      unsigned long long* __restrict__ res) {
    __shared__ double sh[256];
    __shared__ double run;
    __shared__ unsigned long long found, last_pos;
    const uint64_t lo = lo_arr[blockIdx.x], hi = min(D, lo + chunk);
    const double thr = thr_arr[blockIdx.x];
    if (threadIdx.x == 0) {
        run = 0.0;
        found = ~0ull;
        last_pos = lo;
    }
    __syncthreads();
    for (uint64_t t0 = lo; t0 < hi; t0 += blockDim.x) {
        uint64_t i = t0 + threadIdx.x;
        double w = 0.0;
        if (i < hi) {
            if (DIAG) {
                w = double(x[i * (D + 1)].x);
            } else {
                Cplx<R> a = x[i];
                w = double(a.x) * a.x + double(a.y) * a.y;
            }
            if (w > 0) atomicMax(&last_pos, (unsigned long long)i);
        }
        sh[threadIdx.x] = w;
        __syncthreads();
        for (int s = 1; s < int(blockDim.x); s <<= 1) {
            double add = threadIdx.x >= unsigned(s) ? sh[threadIdx.x - s] : 0.0;
            __syncthreads();
            sh[threadIdx.x] += add;
            __syncthreads();
        }
        double incl = run + sh[threadIdx.x];
        if (i < hi && incl >= thr) atomicMin(&found, (unsigned long long)i);
        __syncthreads();
        if (found != ~0ull) break;
        if (threadIdx.x == blockDim.x - 1) run = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) res[blockIdx.x] = found == ~0ull ? last_pos : found;
}

// One block scans [lo, hi) in tiles of blockDim.x and writes the first index
// whose running inclusive sum reaches `thr` (hi - 1 if none).
template <typename R, bool DIAG>
__global__ void __launch_bounds__(1024)
    k_chunk_scan(const Cplx<R>* __restrict__ x, uint64_t D, uint64_t lo,
                 uint64_t hi, double thr, unsigned long long* __restrict__ res) {
    __shared__ double sh[1024];
    __shared__ double run;
    __shared__ unsigned long long found;
    if (threadIdx.x == 0) {
        run = 0.0;
        found = ~0ull;
    }
    __syncthreads();
    for (uint64_t t0 = lo; t0 < hi; t0 += blockDim.x) {
        uint64_t i = t0 + threadIdx.x;
        double w = 0.0;
        if (i < hi) {
            if (DIAG) {
                w = double(x[i * (D + 1)].x);
            } else {
                Cplx<R> a = x[i];
                w = double(a.x) * a.x + double(a.y) * a.y;
            }
        }
        sh[threadIdx.x] = w;
        __syncthreads();
        // Hillis-Steele inclusive scan
        for (int s = 1; s < int(blockDim.x); s <<= 1) {
            double add = threadIdx.x >= unsigned(s) ? sh[threadIdx.x - s] : 0.0;
            __syncthreads();
            sh[threadIdx.x] += add;
            __syncthreads();
        }
        double incl = run + sh[threadIdx.x];
        if (i < hi && incl >= thr) atomicMin(&found, (unsigned long long)i);
        __syncthreads();
        if (found != ~0ull) break;
        if (threadIdx.x == blockDim.x - 1) run = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *res = found == ~0ull ? (hi - 1) : found;
}

template <typename R>
__global__ void __launch_bounds__(256)
    k_scale(Cplx<R>* __restrict__ x, uint64_t n, double sr, double si) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += uint64_t(gridDim.x) * blockDim.x) {
        Cplx<R> a = x[i];
        double ar = a.x, ai = a.y;
        a.x = R(ar * sr - ai * si);
        a.y = R(ar * si + ai * sr);
        x[i] = a;
    }
}

// Keep elements whose digit (index / dig_stride) % dig_dim equals dig_val in
// the row (and, for rho, the column) index; zero the rest; scale the kept.
template <typename R>
__global__ void __launch_bounds__(256)
    k_project(Cplx<R>* __restrict__ x, uint64_t n, uint64_t D, int is_rho,
              uint64_t dig_stride, uint64_t dig_dim, uint64_t dig_val,
              double scale) {
    for (uint64_t e = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
         e += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t r = is_rho ? e % D : e;
        bool keep = (r / dig_stride) % dig_dim == dig_val;
        if (is_rho) keep = keep && ((e / D) / dig_stride) % dig_dim == dig_val;
        Cplx<R> a = x[e];
        if (keep) {
            a.x = R(double(a.x) * scale);
            a.y = R(double(a.y) * scale);
        } else {
            a.x = 0;
            a.y = 0;
        }
        x[e] = a;
    }
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): counter = element
// index, key = seed; Box-Muller on the first two words gives (re, im).
template <typename R>
__global__ void __launch_bounds__(256)
    k_fill_gaussian(Cplx<R>* __restrict__ x, uint64_t n, uint64_t seed) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t c[4] = {uint32_t(i), uint32_t(i >> 32), 0u, 0u};
        philox4x32_10(c, uint32_t(seed), uint32_t(seed >> 32));
        // 53-bit uniforms in (0, 1] and [0, 1)
        uint64_t a = (uint64_t(c[0]) << 21) ^ (uint64_t(c[1]) >> 11);
        uint64_t b = (uint64_t(c[2]) << 21) ^ (uint64_t(c[3]) >> 11);
        double u1 = (double(a & ((1ull << 53) - 1)) + 1.0) * 0x1.0p-53;
        double u2 = double(b & ((1ull << 53) - 1)) * 0x1.0p-53;
        double r = sqrt(-2.0 * log(u1));
        double s, co;
        sincospi(2.0 * u2, &s, &co);
        Cplx<R> v;
        v.x = R(r * co);
        v.y = R(r * s);
        x[i] = v;
    }
}

template <typename A, typename B>
__global__ void __launch_bounds__(256)
    k_convert(const A* __restrict__ in, B* __restrict__ out, uint64_t n) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += uint64_t(gridDim.x) * blockDim.x) {
        A a = in[i];
        B b;
        b.x = decltype(b.x)(a.x);
        b.y = decltype(b.y)(a.y);
        out[i] = b;
    }
}

// ------------------------------------------------------------- launchers
static int nblocks(qgpu_ctx* ctx, uint64_t n) {
    uint64_t need = (n + 255) / 256;
    uint64_t b = std::min<uint64_t>(need, uint64_t(ctx->num_sms) * 8);
    return int(std::max<uint64_t>(b, 1));
}

static void finish_partials(qgpu_ctx* ctx, double* partial, int nb, int nc,
                            double* host_out) {
    double* dout = partial + size_t(nb) * nc;
    k_sum_partials<<<1, kRedThreads, 0, ctx->stream>>>(partial, nb, nc, dout);
    after_launch(ctx, "k_sum_partials");
    double* pin = static_cast<double*>(ctx_pinned(ctx, nc * sizeof(double)));
    QG_CUDA(cudaMemcpyAsync(pin, dout, nc * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
    QG_CUDA(cudaStreamSynchronize(ctx->stream));
    std::memcpy(host_out, pin, nc * sizeof(double));
}

double reduce_norm2(qgpu_ctx* ctx, qgpu_prec prec, const void* data,
                    uint64_t n) {
    int nb = std::min(kRedBlocks, nblocks(ctx, n));
    double* part = static_cast<double*>(ctx_scratch(ctx, (nb + 1) * sizeof(double)));
    if (prec == QGPU_C128)
        k_norm2_partial<double><<<nb, kRedThreads, 0, ctx->stream>>>(
            static_cast<const double2*>(data), n, part);
    else
        k_norm2_partial<float><<<nb, kRedThreads, 0, ctx->stream>>>(
            static_cast<const float2*>(data), n, part);
    after_launch(ctx, "k_norm2_partial");
    double r;
    finish_partials(ctx, part, nb, 1, &r);
    return r;
}

void reduce_norm2_device(qgpu_ctx* ctx, qgpu_prec prec, const void* data, uint64_t n,
                         double* dev_out) {
    int nb = std::min(kRedBlocks, nblocks(ctx, n));
    double* part = static_cast<double*>(ctx_scratch(ctx, nb * sizeof(double)));
    if (prec == QGPU_C128)
        k_norm2_partial<double><<<nb, kRedThreads, 0, ctx->stream>>>(
            static_cast<const double2*>(data), n, part);
    else
        k_norm2_partial<float><<<nb, kRedThreads, 0, ctx->stream>>>(
            static_cast<const float2*>(data), n, part);
    after_launch(ctx, "k_norm2_partial");
    k_sum_partials<<<1, kRedThreads, 0, ctx->stream>>>(part, nb, 1, dev_out);
    after_launch(ctx, "k_sum_partials");
}

cd reduce_strided_sum(qgpu_ctx* ctx, qgpu_prec prec, const void* data,
                      uint64_t n, uint64_t stride) {
    int nb = std::min(kRedBlocks, nblocks(ctx, n));
    double* part = static_cast<double*>(ctx_scratch(ctx, (2 * nb + 2) * sizeof(double)));
    if (prec == QGPU_C128)
        k_strided_partial<double><<<nb, kRedThreads, 0, ctx->stream>>>(
            static_cast<const double2*>(data), n, stride, part);
    else
        k_strided_partial<float><<<nb, kRedThreads, 0, ctx->stream>>>(
            static_cast<const float2*>(data), n, stride, part);
    after_launch(ctx, "k_strided_partial");
    double r[2];
    finish_partials(ctx, part, nb, 2, r);
    return {r[0], r[1]};
}

cd reduce_inner(qgpu_ctx* ctx, qgpu_prec prec, const void* a, const void* b,
                uint64_t n) {
    int nb = std::min(kRedBlocks, nblocks(ctx, n));
    double* part = static_cast<double*>(ctx_scratch(ctx, (2 * nb + 2) * sizeof(double)));
    if (prec == QGPU_C128)
        k_inner_partial<double><<<nb, kRedThreads, 0, ctx->stream>>>(
            static_cast<const double2*>(a), static_cast<const double2*>(b), n, part);
    else
        k_inner_partial<float><<<nb, kRedThreads, 0, ctx->stream>>>(
            static_cast<const float2*>(a), static_cast<const float2*>(b), n, part);
    after_launch(ctx, "k_inner_partial");
    double r[2];
    finish_partials(ctx, part, nb, 2, r);
    return {r[0], r[1]};
}

void launch_scale(qgpu_ctx* ctx, qgpu_prec prec, void* data, uint64_t n,
                  cd s) {
    int nb = nblocks(ctx, n);
    if (prec == QGPU_C128)
        k_scale<double><<<nb, 256, 0, ctx->stream>>>(static_cast<double2*>(data), n,
                                                     s.real(), s.imag());
    else
        k_scale<float><<<nb, 256, 0, ctx->stream>>>(static_cast<float2*>(data), n,
                                                    s.real(), s.imag());
    after_launch(ctx, "k_scale");
}

std::vector<double> reduce_marginals(qgpu_ctx* ctx, qgpu_prec prec,
                                     const void* data, const SegPlan& outer,
                                     const std::vector<uint64_t>& off,
                                     bool diag_of_rho, uint64_t D) {
    int DA = int(off.size());
    int nbx = std::min(kRedBlocks / 4, nblocks(ctx, outer.count));
    nbx = std::max(nbx, 1);
    size_t off_bytes = (DA * sizeof(uint64_t) + 255) / 256 * 256;
    size_t part_elems = size_t(nbx) * DA;
    unsigned char* s = static_cast<unsigned char*>(
        ctx_scratch(ctx, off_bytes + (part_elems + DA) * sizeof(double)));
    uint64_t* doff = reinterpret_cast<uint64_t*>(s);
    double* part = reinterpret_cast<double*>(s + off_bytes);
    QG_CUDA(cudaMemcpyAsync(doff, off.data(), DA * sizeof(uint64_t),
                            cudaMemcpyHostToDevice, ctx->stream));
    dim3 grid(nbx, DA);
    uint64_t mul = D + 1;
    if (prec == QGPU_C128) {
        if (diag_of_rho)
            k_marginal_partial<double, true><<<grid, kRedThreads, 0, ctx->stream>>>(
                static_cast<const double2*>(data), outer, doff, mul, part);
        else
            k_marginal_partial<double, false><<<grid, kRedThreads, 0, ctx->stream>>>(
                static_cast<const double2*>(data), outer, doff, mul, part);
    } else {
        if (diag_of_rho)
            k_marginal_partial<float, true><<<grid, kRedThreads, 0, ctx->stream>>>(
                static_cast<const float2*>(data), outer, doff, mul, part);
        else
            k_marginal_partial<float, false><<<grid, kRedThreads, 0, ctx->stream>>>(
                static_cast<const float2*>(data), outer, doff, mul, part);
    }
    after_launch(ctx, "k_marginal_partial");
    // partial is m-major: component c = m, block b at [m * nbx + b]; reduce
    // each m's row with k_sum_partials using nc = 1 and an offset pointer.
    std::vector<double> res(DA);
    double* dout = part + part_elems;
    for (int m = 0; m < DA; ++m) {
        k_sum_partials<<<1, kRedThreads, 0, ctx->stream>>>(part + size_t(m) * nbx,
                                                           nbx, 1, dout + m);
        after_launch(ctx, "k_sum_partials");
    }
    double* pin = static_cast<double*>(ctx_pinned(ctx, DA * sizeof(double)));
    QG_CUDA(cudaMemcpyAsync(pin, dout, DA * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
    QG_CUDA(cudaStreamSynchronize(ctx->stream));
    std::memcpy(res.data(), pin, DA * sizeof(double));
    return res;
}

uint64_t prefix_search(qgpu_ctx* ctx, qgpu_prec prec, const void* data,
                       uint64_t D, bool diag, double fraction,
                       double* total_out) {
    int nb = std::min(kRedBlocks, nblocks(ctx, D));
    uint64_t chunk = (D + nb - 1) / nb;
    nb = int((D + chunk - 1) / chunk);
    double* part = static_cast<double*>(ctx_scratch(ctx, (nb + 2) * sizeof(double)));
    unsigned long long* dres = reinterpret_cast<unsigned long long*>(part + nb);
#define QG_CHUNK(R, T, DG)                                                     \
    k_chunk_sums<R, DG><<<nb, kRedThreads, 0, ctx->stream>>>(                  \
        static_cast<const T*>(data), D, chunk, part)
    if (prec == QGPU_C128) {
        if (diag) QG_CHUNK(double, double2, true);
        else QG_CHUNK(double, double2, false);
    } else {
        if (diag) QG_CHUNK(float, float2, true);
        else QG_CHUNK(float, float2, false);
    }
#undef QG_CHUNK
    after_launch(ctx, "k_chunk_sums");
    double* pin = static_cast<double*>(ctx_pinned(ctx, nb * sizeof(double) + 16));
    QG_CUDA(cudaMemcpyAsync(pin, part, nb * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
    QG_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<double> ps(pin, pin + nb);
    double total = 0;
    for (double p : ps) total += p;
    if (total_out) *total_out = total;
    double thr = fraction * total;
    double cum = 0;
    int b = 0;
    for (; b < nb; ++b) {
        if (cum + ps[b] >= thr && ps[b] > 0) break;
        cum += ps[b];
    }
    if (b == nb) { // rounding: take the last chunk holding weight
        b = nb - 1;
        while (b > 0 && ps[b] <= 0) --b;
        cum = 0;
        for (int j = 0; j < b; ++j) cum += ps[j];
    }
    uint64_t lo = uint64_t(b) * chunk, hi = std::min(D, lo + chunk);
#define QG_SCAN(R, T, DG)                                                      \
    k_chunk_scan<R, DG><<<1, 1024, 0, ctx->stream>>>(                          \
        static_cast<const T*>(data), D, lo, hi, thr - cum, dres)
    if (prec == QGPU_C128) {
        if (diag) QG_SCAN(double, double2, true);
        else QG_SCAN(double, double2, false);
    } else {
        if (diag) QG_SCAN(float, float2, true);
        else QG_SCAN(float, float2, false);
    }
#undef QG_SCAN
    after_launch(ctx, "k_chunk_scan");
    unsigned long long* pres = reinterpret_cast<unsigned long long*>(pin);
    QG_CUDA(cudaMemcpyAsync(pres, dres, sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, ctx->stream));
    QG_CUDA(cudaStreamSynchronize(ctx->stream));
    return uint64_t(*pres);
}

std::vector<uint64_t> prefix_search_many(qgpu_ctx* ctx, qgpu_prec prec, const void* data,
                                         uint64_t D, bool diag,
                                         const std::vector<double>& fractions) {
    std::vector<uint64_t> out(fractions.size());
    if (fractions.empty()) return out;
    // fixed chunks of 4096 weights: one pass for the chunk sums, then each
    // draw scans a single chunk
    const uint64_t chunk = 4096;
    const uint64_t nb64 = (D + chunk - 1) / chunk;
    if (nb64 > (uint64_t(1) << 31)) raise(QGPU_ERR_OUT_OF_RANGE, "prefix_search_many()", "D");
    const int nb = int(nb64);
    const size_t m = fractions.size();
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t b_part = al(nb * sizeof(double)), b_lo = al(m * sizeof(uint64_t)),
                 b_thr = al(m * sizeof(double)), b_res = al(m * sizeof(unsigned long long));
    unsigned char* buf = nullptr;
    QG_CUDA(ctx_malloc(ctx, reinterpret_cast<void**>(&buf), b_part + b_lo + b_thr + b_res));
    struct Free {
        qgpu_ctx* c;
        void* p;
        ~Free() { cudaFreeAsync(p, c->stream); }
    } fr{ctx, buf};
    double* part = reinterpret_cast<double*>(buf);
    uint64_t* dlo = reinterpret_cast<uint64_t*>(buf + b_part);
    double* dthr = reinterpret_cast<double*>(buf + b_part + b_lo);
    unsigned long long* dres =
        reinterpret_cast<unsigned long long*>(buf + b_part + b_lo + b_thr);
#define QG_CHUNK(R, T, DG)                                                     \
    k_chunk_sums<R, DG><<<nb, kRedThreads, 0, ctx->stream>>>(                  \
        static_cast<const T*>(data), D, chunk, part)
    if (prec == QGPU_C128) {
        if (diag) QG_CHUNK(double, double2, true);
        else QG_CHUNK(double, double2, false);
    } else {
        if (diag) QG_CHUNK(float, float2, true);
        else QG_CHUNK(float, float2, false);
    }
#undef QG_CHUNK
    after_launch(ctx, "k_chunk_sums");
    std::vector<double> ps(nb);
    QG_CUDA(cudaMemcpyAsync(ps.data(), part, nb * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream));
    QG_CUDA(cudaStreamSynchronize(ctx->stream));
    // inclusive chunk prefix (FP64, in order)
    std::vector<double> cp(nb);
    double acc = 0;
    int last = -1;
    for (int b = 0; b < nb; ++b) {
        acc += ps[b];
        cp[b] = acc;
        if (ps[b] > 0) last = b;
    }
    if (last < 0) raise(QGPU_ERR_DIVISION_BY_ZERO, "qpp::sample()", "zero weight");
    std::vector<uint64_t> lo(m);
    std::vector<double> thr(m);
    for (size_t j = 0; j < m; ++j) {
        const double t = fractions[j] * acc;
        int b = int(std::lower_bound(cp.begin(), cp.end(), t) - cp.begin());
        while (b < nb && ps[b] <= 0) ++b; // a chunk that holds weight
        if (b >= nb) b = last;
        lo[j] = uint64_t(b) * chunk;
        thr[j] = t - (b > 0 ? cp[b - 1] : 0.0);
    }
    QG_CUDA(cudaMemcpyAsync(dlo, lo.data(), m * sizeof(uint64_t), cudaMemcpyHostToDevice,
                            ctx->stream));
    QG_CUDA(cudaMemcpyAsync(dthr, thr.data(), m * sizeof(double), cudaMemcpyHostToDevice,
                            ctx->stream));
    for (size_t j0 = 0; j0 < m; j0 += 65535) {
        const unsigned g = unsigned(std::min<size_t>(65535, m - j0));
#define QG_SCAN(R, T, DG)                                                      \
    k_chunk_scan_many<R, DG><<<g, 256, 0, ctx->stream>>>(                      \
        static_cast<const T*>(data), D, chunk, dlo + j0, dthr + j0, dres + j0)
        if (prec == QGPU_C128) {
            if (diag) QG_SCAN(double, double2, true);
            else QG_SCAN(double, double2, false);
        } else {
            if (diag) QG_SCAN(float, float2, true);
            else QG_SCAN(float, float2, false);
        }
#undef QG_SCAN
        after_launch(ctx, "k_chunk_scan_many");
    }
    std::vector<unsigned long long> r(m);
    QG_CUDA(cudaMemcpyAsync(r.data(), dres, m * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, ctx->stream));
    QG_CUDA(cudaStreamSynchronize(ctx->stream));
    for (size_t j = 0; j < m; ++j) out[j] = uint64_t(r[j]);
    return out;
}

void launch_project(qgpu_ctx* ctx, qgpu_prec prec, void* data, uint64_t n,
                    uint64_t D, bool is_rho, uint64_t dig_stride,
                    uint64_t dig_dim, uint64_t dig_val, double scale) {
    int nb = nblocks(ctx, n);
    if (prec == QGPU_C128)
        k_project<double><<<nb, 256, 0, ctx->stream>>>(
            static_cast<double2*>(data), n, D, is_rho ? 1 : 0, dig_stride, dig_dim,
            dig_val, scale);
    else
        k_project<float><<<nb, 256, 0, ctx->stream>>>(
            static_cast<float2*>(data), n, D, is_rho ? 1 : 0, dig_stride, dig_dim,
            dig_val, scale);
    after_launch(ctx, "k_project");
}

void launch_fill_gaussian(qgpu_ctx* ctx, qgpu_prec prec, void* data,
                          uint64_t n, uint64_t seed) {
    int nb = nblocks(ctx, n);
    if (prec == QGPU_C128)
        k_fill_gaussian<double><<<nb, 256, 0, ctx->stream>>>(
            static_cast<double2*>(data), n, seed);
    else
        k_fill_gaussian<float><<<nb, 256, 0, ctx->stream>>>(
            static_cast<float2*>(data), n, seed);
    after_launch(ctx, "k_fill_gaussian");
}

void launch_convert(qgpu_ctx* ctx, const void* in, qgpu_prec in_prec,
                    void* out, qgpu_prec out_prec, uint64_t n) {
    int nb = nblocks(ctx, n);
    if (in_prec == QGPU_C128 && out_prec == QGPU_C64)
        k_convert<double2, float2><<<nb, 256, 0, ctx->stream>>>(
            static_cast<const double2*>(in), static_cast<float2*>(out), n);
    else if (in_prec == QGPU_C64 && out_prec == QGPU_C128)
        k_convert<float2, double2><<<nb, 256, 0, ctx->stream>>>(
            static_cast<const float2*>(in), static_cast<double2*>(out), n);
    else if (in_prec == QGPU_C128)
        k_convert<double2, double2><<<nb, 256, 0, ctx->stream>>>(
            static_cast<const double2*>(in), static_cast<double2*>(out), n);
    else
        k_convert<float2, float2><<<nb, 256, 0, ctx->stream>>>(
            static_cast<const float2*>(in), static_cast<float2*>(out), n);
    after_launch(ctx, "k_convert");
}

} // namespace qgpu
