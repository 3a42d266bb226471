// kernels_gate.cu -- in-place gate application on a (virtual) ket.
//
// Replaces the CPU loops of include/qpp/internal/kernels/qubit/apply.hpp
// (:57-594), apply_ctrl.hpp and the generic mixed-radix path of
// operations.hpp:182-371. qpp copies the state and writes a fresh result; here
// every group of amplitudes is read once and written back in place by the one
// thread that owns it, so a gate costs exactly one read and one write of the
// touched amplitudes (2 * 16 B per amplitude in c128).
//
//  k_qubit_1q  2x2 on one bit: pairs (i, i | 2^b), 128-bit accesses, U
//              independent pairs in flight per thread; grids are a multiple
//              of the SM count (persistent grid-stride).
//  k_qubit_2q  4x4 on two bits.
//  k_reg<DA>   any DA <= 16 (qudits, rho superoperators, Kraus channels),
//              matrix and offsets in the kernel parameter block.
//  k_smem      any DA <= 4096: groups staged in shared memory, one output row
//              per thread, the matrix read through L1.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "kernels.hpp"

namespace qgpu {

template <typename R>
struct M2 {
    Cplx<R> a00, a01, a10, a11;
};
template <typename R>
struct M4 {
    Cplx<R> a[16]; // row-major: a[4 * row + col]
};

template <typename R>
__device__ __forceinline__ Cplx<R> mk(R x, R y) {
    Cplx<R> c;
    c.x = x;
    c.y = y;
    return c;
}

template <typename R, typename I, int U>
__global__ void __launch_bounds__(256)
    k_qubit_1q(Cplx<R>* __restrict__ psi, I npairs, int b,
               const __grid_constant__ M2<R> m) {
    using C = Cplx<R>;
    const I low = (I(1) << b) - 1;
    const I step = I(1) << b;
    const I nth = I(gridDim.x) * blockDim.x;
    for (I p0 = I(blockIdx.x) * blockDim.x + threadIdx.x; p0 < npairs;
         p0 += nth * U) {
        C v0[U], v1[U];
        I i0[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            I p = p0 + I(u) * nth;
            i0[u] = ((p & ~low) << 1) | (p & low);
            if (p < npairs) {
                v0[u] = psi[i0[u]];
                v1[u] = psi[i0[u] + step];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            I p = p0 + I(u) * nth;
            if (p < npairs) {
                C r0 = cmul(m.a00, v0[u]);
                r0 = cfma(m.a01, v1[u], r0);
                C r1 = cmul(m.a10, v0[u]);
                r1 = cfma(m.a11, v1[u], r1);
                psi[i0[u]] = r0;
                psi[i0[u] + step] = r1;
            }
        }
    }
}

template <typename I>
__device__ __forceinline__ I insert_zero(I x, int b) {
    I low = (I(1) << b) - 1;
    return ((x & ~low) << 1) | (x & low);
}

template <typename R, typename I, int U>
__global__ void __launch_bounds__(256)
    k_qubit_2q(Cplx<R>* __restrict__ psi, I ngroups, int blo, int bhi,
               I s0, I s1, const __grid_constant__ M4<R> m) {
    using C = Cplx<R>;
    const I nth = I(gridDim.x) * blockDim.x;
    for (I g0 = I(blockIdx.x) * blockDim.x + threadIdx.x; g0 < ngroups;
         g0 += nth * U) {
        C v[U][4];
        I base[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            I g = g0 + I(u) * nth;
            base[u] = insert_zero(insert_zero(g, blo), bhi);
            if (g < ngroups) {
                v[u][0] = psi[base[u]];
                v[u][1] = psi[base[u] + s1];
                v[u][2] = psi[base[u] + s0];
                v[u][3] = psi[base[u] + s0 + s1];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            I g = g0 + I(u) * nth;
            if (g < ngroups) {
                C r[4];
#pragma unroll
                for (int row = 0; row < 4; ++row) {
                    C acc = cmul(m.a[4 * row], v[u][0]);
                    acc = cfma(m.a[4 * row + 1], v[u][1], acc);
                    acc = cfma(m.a[4 * row + 2], v[u][2], acc);
                    acc = cfma(m.a[4 * row + 3], v[u][3], acc);
                    r[row] = acc;
                }
                psi[base[u]] = r[0];
                psi[base[u] + s1] = r[1];
                psi[base[u] + s0] = r[2];
                psi[base[u] + s0 + s1] = r[3];
            }
        }
    }
}

template <typename R, int DA>
struct RegParams {
    SegPlan outer;
    uint64_t off[DA];
    Cplx<R> A[DA * DA]; // column-major
};

template <typename R, int DA>
__global__ void __launch_bounds__(256)
    k_reg(Cplx<R>* __restrict__ psi, const __grid_constant__ RegParams<R, DA> p) {
    using C = Cplx<R>;
    const uint64_t nth = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
         g < p.outer.count; g += nth) {
        const uint64_t base = seg_offset(p.outer, g);
        C v[DA];
#pragma unroll
        for (int c = 0; c < DA; ++c) v[c] = psi[base + p.off[c]];
#pragma unroll
        for (int m = 0; m < DA; ++m) {
            C acc = cmul(p.A[m], v[0]);
#pragma unroll
            for (int c = 1; c < DA; ++c) acc = cfma(p.A[m + c * DA], v[c], acc);
            psi[base + p.off[m]] = acc;
        }
    }
}

// A 16 x 16 operator that is a Kronecker product A (x) B of two 4 x 4 ones
// (a product channel's superoperator on two qubits): the group's element
// (i, j) sits at base + off[4 i + j]; A acts on i, B on j, both from the
// parameter bank. 128 complex MACs per group instead of 256.
template <typename R>
struct KronParams {
    SegPlan outer;
    uint64_t off[16];
    Cplx<R> A[16], B[16]; // column-major
};

// Complex128: a group split over two adjacent lanes (h = lane & 1). Lane h
// loads columns j = 2h, 2h + 1 (eight elements) and applies A along i; the
// pair then trades through shuffles so that lane h holds rows i = 2h, 2h + 1,
// applies B along j and stores them. Eight elements per lane instead of
// sixteen keep the kernel at two or more CTAs per SM without spills.
template <typename R>
__device__ __forceinline__ Cplx<R> shfl_pair(Cplx<R> v) {
    Cplx<R> r;
    r.x = __shfl_xor_sync(0xffffffffu, v.x, 1);
    r.y = __shfl_xor_sync(0xffffffffu, v.y, 1);
    return r;
}

template <typename R>
__global__ void __launch_bounds__(256, 2)
    k_reg_kron_pair(Cplx<R>* __restrict__ psi, const __grid_constant__ KronParams<R> p) {
    using C = Cplx<R>;
    const uint32_t h = threadIdx.x & 1u;
    const uint64_t pairs = uint64_t(gridDim.x) * (blockDim.x / 2);
    const uint64_t g_first = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 1;
    // every lane runs the same number of iterations (the shuffles need the
    // whole warp)
    const uint64_t iters = (p.outer.count + pairs - 1) / pairs;
    for (uint64_t it = 0; it < iters; ++it) {
        const uint64_t g = g_first + it * pairs;
        const bool valid = g < p.outer.count;
        const uint64_t base = valid ? seg_offset(p.outer, g) : 0;
        C v[4][2]; // v[i][jj]: element (i, 2h + jj)
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj) {
                const uint64_t o = h ? p.off[4 * i + 2 + jj] : p.off[4 * i + jj];
                if (valid) v[i][jj] = psi[base + o];
                else v[i][jj].x = v[i][jj].y = R(0);
            }
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
            C w[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                C acc = cmul(p.A[r], v[0][jj]);
#pragma unroll
                for (int c = 1; c < 4; ++c) acc = cfma(p.A[r + 4 * c], v[c][jj], acc);
                w[r] = acc;
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) v[r][jj] = w[r];
        }
        // mine[ii][j]: element (2h + ii, j)
        C mine[2][4];
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int jj = 0; jj < 2; ++jj) {
                const C keep = h ? v[2 + ii][jj] : v[ii][jj]; // (2h + ii, 2h + jj)
                const C send = h ? v[ii][jj] : v[2 + ii][jj]; // (2(1 - h) + ii, 2h + jj)
                const C recv = shfl_pair<R>(send);            // (2h + ii, 2(1 - h) + jj)
                mine[ii][jj] = h ? recv : keep;
                mine[ii][2 + jj] = h ? keep : recv;
            }
        if (!valid) continue;
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                C acc = cmul(p.B[r], mine[ii][0]);
#pragma unroll
                for (int c = 1; c < 4; ++c) acc = cfma(p.B[r + 4 * c], mine[ii][c], acc);
                const uint64_t o = h ? p.off[4 * (2 + ii) + r] : p.off[4 * ii + r];
                psi[base + o] = acc;
            }
    }
}

template <typename R>
__global__ void __launch_bounds__(256, 3)
    k_reg_kron(Cplx<R>* __restrict__ psi, const __grid_constant__ KronParams<R> p) {
    using C = Cplx<R>;
    const uint64_t nth = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < p.outer.count;
         g += nth) {
        const uint64_t base = seg_offset(p.outer, g);
        C v[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) v[e] = psi[base + p.off[e]];
        // A along i for each j
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            C w[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                C acc = cmul(p.A[r], v[j]);
#pragma unroll
                for (int c = 1; c < 4; ++c) acc = cfma(p.A[r + 4 * c], v[4 * c + j], acc);
                w[r] = acc;
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) v[4 * r + j] = w[r];
        }
        // B along j for each i, stored
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                C acc = cmul(p.B[r], v[4 * i]);
#pragma unroll
                for (int c = 1; c < 4; ++c) acc = cfma(p.B[r + 4 * c], v[4 * i + c], acc);
                psi[base + p.off[4 * i + r]] = acc;
            }
    }
}

// Output rows [P * DA / S, (P + 1) * DA / S) of one group, the matrix
// entries taken as compile-time offsets into the parameter bank.
template <typename R, int DA, int S, int P>
__device__ __forceinline__ void reg_rows(Cplx<R>* psi, const RegParams<R, DA>& p, uint64_t base,
                                         const Cplx<R> (&v)[DA]) {
    using C = Cplx<R>;
#pragma unroll
    for (int k = 0; k < DA / S; ++k) {
        constexpr int m0 = P * (DA / S);
        C acc = cmul(p.A[m0 + k], v[0]);
#pragma unroll
        for (int c = 1; c < DA; ++c) acc = cfma(p.A[m0 + k + c * DA], v[c], acc);
        psi[base + p.off[m0 + k]] = acc;
    }
}

// k_reg with each group shared by 2 warps: lane l of warps 2j and 2j + 1
// both load the group's DA inputs, and each forms half of the output rows,
// so a thread does half the arithmetic and holds half the partial results.
// A block barrier separates the loads of an iteration from its in-place
// stores.
template <typename R, int DA>
__global__ void __launch_bounds__(256)
    k_reg_split(Cplx<R>* __restrict__ psi, const __grid_constant__ RegParams<R, DA> p) {
    using C = Cplx<R>;
    const int warp = int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
    const int part = warp & 1; // uniform within a warp
    const uint64_t per_block = blockDim.x / 2;
    const uint64_t nth = uint64_t(gridDim.x) * per_block;
    const uint64_t g_first = uint64_t(blockIdx.x) * per_block + uint64_t(warp >> 1) * 32 + lane;
    // every thread of the block runs the same number of iterations
    const uint64_t iters = (p.outer.count + nth - 1) / nth;
    for (uint64_t it = 0; it < iters; ++it) {
        const uint64_t g = g_first + it * nth;
        const bool valid = g < p.outer.count;
        const uint64_t base = valid ? seg_offset(p.outer, g) : 0;
        C v[DA];
        if (valid) {
#pragma unroll
            for (int c = 0; c < DA; ++c) v[c] = psi[base + p.off[c]];
        }
        __syncthreads();
        if (valid) {
            if (part == 0) reg_rows<R, DA, 2, 0>(psi, p, base, v);
            else reg_rows<R, DA, 2, 1>(psi, p, base, v);
        }
    }
}

// Shared-memory variant for any DA: a block owns G groups at a time
// (G * DA <= blockDim.x when DA <= 256), stages them, then each thread forms
// output rows. A (column-major, state precision) and off live in global
// memory and are read through the read-only cache.
template <typename R>
__global__ void __launch_bounds__(256)
    k_smem(Cplx<R>* __restrict__ psi, const __grid_constant__ SegPlan outer,
           const uint64_t* __restrict__ off, const Cplx<R>* __restrict__ A,
           int DA, int G) {
    using C = Cplx<R>;
    extern __shared__ unsigned char smem_raw[];
    C* sv = reinterpret_cast<C*>(smem_raw);
    const int tid = threadIdx.x;
    const int per = G * DA;
    for (uint64_t g0 = uint64_t(blockIdx.x) * G; g0 < outer.count;
         g0 += uint64_t(gridDim.x) * G) {
        for (int e = tid; e < per; e += blockDim.x) {
            uint64_t g = g0 + e / DA;
            if (g < outer.count)
                sv[e] = psi[seg_offset(outer, g) + __ldg(&off[e % DA])];
        }
        __syncthreads();
        for (int e = tid; e < per; e += blockDim.x) {
            int gl = e / DA, m = e % DA;
            uint64_t g = g0 + gl;
            if (g < outer.count) {
                const C* v = sv + gl * DA;
                C acc;
                acc.x = 0;
                acc.y = 0;
                for (int c = 0; c < DA; ++c) acc = cfma(A[m + size_t(c) * DA], v[c], acc);
                psi[seg_offset(outer, g) + __ldg(&off[m])] = acc;
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------- launchers
int grid_blocks(qgpu_ctx* ctx, int blocks_per_sm) {
    return ctx->num_sms * blocks_per_sm;
}

template <typename R>
static Cplx<R> cv(const cd& z) {
    Cplx<R> c;
    c.x = static_cast<R>(z.real());
    c.y = static_cast<R>(z.imag());
    return c;
}

template <typename R>
static void q1(qgpu_ctx* ctx, void* data, int nbits, int bit, const cd* A) {
    M2<R> m{cv<R>(A[0]), cv<R>(A[2]), cv<R>(A[1]), cv<R>(A[3])};
    uint64_t np = uint64_t(1) << (nbits - 1);
    // one pair per thread over the whole state: on the 30-qubit sweep a grid
    // of one pair per thread moved 6.9 TB/s, a grid-stride loop over 8
    // blocks per SM 5.99 TB/s (fewer, longer-running blocks keep fewer
    // independent accesses in flight at the tail of each block)
    constexpr int U = sizeof(R) == 8 ? 2 : 4;
    const uint64_t need = (np + 255) / 256;
    const unsigned blocks = unsigned(std::min<uint64_t>(need, 0x7fffffffu));
    // 32-bit indices only while the loop's last step (p0 + nth * U, nth the
    // grid's threads) stays below 2^32; otherwise it would wrap and never end
    if (np + uint64_t(blocks) * 256 * U < (uint64_t(1) << 32))
        k_qubit_1q<R, uint32_t, U><<<blocks, 256, 0, ctx->stream>>>(
            static_cast<Cplx<R>*>(data), uint32_t(np), bit, m);
    else
        k_qubit_1q<R, uint64_t, U><<<blocks, 256, 0, ctx->stream>>>(
            static_cast<Cplx<R>*>(data), np, bit, m);
    after_launch(ctx, "k_qubit_1q");
}

void launch_qubit_1q(qgpu_ctx* ctx, qgpu_prec prec, void* data, int nbits,
                     int bit, const cd* A) {
    if (prec == QGPU_C128) q1<double>(ctx, data, nbits, bit, A);
    else q1<float>(ctx, data, nbits, bit, A);
}

template <typename R>
static void q2(qgpu_ctx* ctx, void* data, int nbits, int bit0, int bit1,
               const cd* A) {
    M4<R> m;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) m.a[4 * r + c] = cv<R>(A[r + 4 * c]);
    uint64_t ng = uint64_t(1) << (nbits - 2);
    int blo = std::min(bit0, bit1), bhi = std::max(bit0, bit1);
    // one group per thread over the whole state (as for one-qubit gates)
    constexpr int U = sizeof(R) == 8 ? 1 : 2;
    const uint64_t need = (ng + 255) / 256;
    const unsigned blocks = unsigned(std::min<uint64_t>(need, 0x7fffffffu));
    // 32-bit indices only while the loop's last step stays below 2^32
    if (ng + uint64_t(blocks) * 256 * U < (uint64_t(1) << 32))
        k_qubit_2q<R, uint32_t, U><<<blocks, 256, 0, ctx->stream>>>(
            static_cast<Cplx<R>*>(data), uint32_t(ng), blo, bhi,
            uint32_t(1) << bit0, uint32_t(1) << bit1, m);
    else
        k_qubit_2q<R, uint64_t, U><<<blocks, 256, 0, ctx->stream>>>(
            static_cast<Cplx<R>*>(data), ng, blo, bhi, uint64_t(1) << bit0,
            uint64_t(1) << bit1, m);
    after_launch(ctx, "k_qubit_2q");
}

void launch_qubit_2q(qgpu_ctx* ctx, qgpu_prec prec, void* data, int nbits,
                     int bit0, int bit1, const cd* A) {
    if (prec == QGPU_C128) q2<double>(ctx, data, nbits, bit0, bit1, A);
    else q2<float>(ctx, data, nbits, bit0, bit1, A);
}

template <typename R, int DA>
static void reg(qgpu_ctx* ctx, void* data, const SegPlan& outer,
                const std::vector<uint64_t>& off, const cd* A) {
    RegParams<R, DA> p;
    p.outer = outer;
    for (int i = 0; i < DA; ++i) p.off[i] = off[i];
    for (int i = 0; i < DA * DA; ++i) p.A[i] = cv<R>(A[i]);
    int blocks = grid_blocks(ctx, 4);
    uint64_t need = (outer.count + 255) / 256;
    if (need < uint64_t(blocks)) blocks = int(std::max<uint64_t>(need, 1));
    k_reg<R, DA><<<blocks, 256, 0, ctx->stream>>>(static_cast<Cplx<R>*>(data), p);
    after_launch(ctx, "k_reg");
}

template <typename R, int DA>
static void reg_split(qgpu_ctx* ctx, void* data, const SegPlan& outer,
                      const std::vector<uint64_t>& off, const cd* A) {
    RegParams<R, DA> p;
    p.outer = outer;
    for (int i = 0; i < DA; ++i) p.off[i] = off[i];
    for (int i = 0; i < DA * DA; ++i) p.A[i] = cv<R>(A[i]);
    int blocks = grid_blocks(ctx, 4);
    uint64_t need = (outer.count + 127) / 128;
    if (need < uint64_t(blocks)) blocks = int(std::max<uint64_t>(need, 1));
    k_reg_split<R, DA><<<blocks, 256, 0, ctx->stream>>>(static_cast<Cplx<R>*>(data), p);
    after_launch(ctx, "k_reg_split");
}

template <typename R>
static void smem(qgpu_ctx* ctx, void* data, const SegPlan& outer,
                 const std::vector<uint64_t>& off, const cd* A, uint64_t DA) {
    if (DA > 4096)
        raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_apply()",
              "gate dimension above 4096");
    // the staging copy below reads a host vector that a graph would read
    // only at its launch, after the vector is gone
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    QG_CUDA(cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone)
        raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_apply()",
              "gate dimension above 16 inside a stream capture");
    // staging: offsets then the matrix, in the context scratch
    size_t off_bytes = DA * sizeof(uint64_t);
    size_t a_off = (off_bytes + 255) / 256 * 256;
    size_t bytes = a_off + DA * DA * sizeof(Cplx<R>);
    std::vector<unsigned char> host(bytes);
    std::memcpy(host.data(), off.data(), off_bytes);
    Cplx<R>* ha = reinterpret_cast<Cplx<R>*>(host.data() + a_off);
    for (uint64_t i = 0; i < DA * DA; ++i) ha[i] = cv<R>(A[i]);
    unsigned char* dev = static_cast<unsigned char*>(ctx_scratch(ctx, bytes));
    QG_CUDA(cudaMemcpyAsync(dev, host.data(), bytes, cudaMemcpyHostToDevice,
                            ctx->stream));
    int G = DA >= 256 ? 1 : int(256 / DA);
    size_t sm = size_t(G) * DA * sizeof(Cplx<R>);
    ensure_smem(reinterpret_cast<const void*>(k_smem<R>), sm);
    int blocks = grid_blocks(ctx, 4);
    uint64_t need = (outer.count + G - 1) / G;
    if (need < uint64_t(blocks)) blocks = int(std::max<uint64_t>(need, 1));
    k_smem<R><<<blocks, 256, sm, ctx->stream>>>(
        static_cast<Cplx<R>*>(data), outer,
        reinterpret_cast<const uint64_t*>(dev),
        reinterpret_cast<const Cplx<R>*>(dev + a_off), int(DA), G);
    after_launch(ctx, "k_smem");
    // the host staging vector must outlive the (pageable) async copy's
    // staging step, which cudaMemcpyAsync completes before returning
}

template <typename R>
static void generic(qgpu_ctx* ctx, void* data, const SegPlan& outer,
                    const std::vector<uint64_t>& off, const cd* A,
                    uint64_t DA) {
    if (outer.count == 0) return;
    switch (DA) {
        case 2: return reg<R, 2>(ctx, data, outer, off, A);
        case 3: return reg<R, 3>(ctx, data, outer, off, A);
        case 4: return reg<R, 4>(ctx, data, outer, off, A);
        case 8: return reg<R, 8>(ctx, data, outer, off, A);
        case 9: return reg<R, 9>(ctx, data, outer, off, A);
        case 16:
            // complex128: two warps per group (a whole 16 x 16 per thread
            // needs over 250 registers)
            if (sizeof(R) == 8) return reg_split<R, 16>(ctx, data, outer, off, A);
            return reg<R, 16>(ctx, data, outer, off, A);
        default: return smem<R>(ctx, data, outer, off, A, DA);
    }
}

void launch_apply_generic(qgpu_ctx* ctx, qgpu_prec prec, void* data,
                          const SegPlan& outer,
                          const std::vector<uint64_t>& off, const cd* A,
                          uint64_t DA) {
    if (prec == QGPU_C128) generic<double>(ctx, data, outer, off, A, DA);
    else generic<float>(ctx, data, outer, off, A, DA);
}

template <typename R>
static void kron4(qgpu_ctx* ctx, void* data, const SegPlan& outer, const std::vector<uint64_t>& off,
                  const cd* A, const cd* B) {
    if (outer.count == 0) return;
    KronParams<R> p;
    p.outer = outer;
    for (int i = 0; i < 16; ++i) {
        p.off[i] = off[size_t(i)];
        p.A[i] = cv<R>(A[i]);
        p.B[i] = cv<R>(B[i]);
    }
    // one group (complex128: one pair of lanes) per thread over the whole
    // state: on the 12-qubit density matrix the channel pass took 0.085 ms
    // this way against 0.098 ms with one wave of resident CTAs looping
    if constexpr (sizeof(R) == 8) {
        const uint64_t need = std::max<uint64_t>((outer.count + 127) / 128, 1);
        const unsigned blocks = unsigned(std::min<uint64_t>(need, 0x7fffffffu));
        k_reg_kron_pair<R><<<blocks, 256, 0, ctx->stream>>>(static_cast<Cplx<R>*>(data), p);
        after_launch(ctx, "k_reg_kron_pair");
    } else {
        const uint64_t need = std::max<uint64_t>((outer.count + 255) / 256, 1);
        const unsigned blocks = unsigned(std::min<uint64_t>(need, 0x7fffffffu));
        k_reg_kron<R><<<blocks, 256, 0, ctx->stream>>>(static_cast<Cplx<R>*>(data), p);
        after_launch(ctx, "k_reg_kron");
    }
}

void launch_apply_kron4(qgpu_ctx* ctx, qgpu_prec prec, void* data, const SegPlan& outer,
                        const std::vector<uint64_t>& off, const cd* A, const cd* B) {
    if (prec == QGPU_C128) kron4<double>(ctx, data, outer, off, A, B);
    else kron4<float>(ctx, data, outer, off, A, B);
}

} // namespace qgpu
