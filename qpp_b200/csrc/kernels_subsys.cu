// kernels_subsys.cu -- partial trace, partial transpose, subsystem
// permutation and state compaction.
//
// Replaces include/qpp/internal/kernels/qubit/{ptrace,ptranspose,syspermute}.hpp
// and the generic paths of operations.hpp:1908-2514. ptranspose and
// syspermute are pure digit permutations of the (virtual) index, so the
// result is bit-exact: on qubit (power-of-two) digits a tiled bit
// permutation stages 2^10-element tiles in shared memory so reads and writes
// are both coalesced; otherwise the output is written densely and each
// element gathers its source through a merged segment plan. ptrace sums
// diagonal blocks in FP64 whatever the state precision.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

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

// The traced offsets: a device array, or (up to kPtraceTab of them) a table
// passed by value with the launch, which spares the copy to the device.
constexpr int kPtraceTab = 256;
struct PtraceTab {
    uint64_t t[kPtraceTab];
    __device__ __forceinline__ uint64_t operator[](uint64_t a) const { return t[a]; }
};

// one thread per output element (many outputs)
template <typename R, bool KET, typename TABLE>
__global__ void __launch_bounds__(256)
    k_ptrace_thread(const Cplx<R>* __restrict__ in, Cplx<R>* __restrict__ out,
                    const __grid_constant__ SegPlan ma,
                    const __grid_constant__ SegPlan mb,
                    const __grid_constant__ TABLE toff, uint64_t DS) {
    const uint64_t nth = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t o = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
         o < ma.count; o += nth) {
        uint64_t a0 = seg_offset(ma, o), b0 = KET ? seg_offset(mb, o) : 0;
        double sr = 0, si = 0;
        for (uint64_t a = 0; a < DS; ++a)
            ptrace_term<R, KET>(in, a0, b0, toff[a], sr, si);
        Cplx<R> r;
        r.x = R(sr);
        r.y = R(si);
        out[o] = r;
    }
}

// one warp per output element (few outputs, long sums)
template <typename R, bool KET, typename TABLE>
__global__ void __launch_bounds__(256)
    k_ptrace_warp(const Cplx<R>* __restrict__ in, Cplx<R>* __restrict__ out,
                  const __grid_constant__ SegPlan ma,
                  const __grid_constant__ SegPlan mb,
                  const __grid_constant__ TABLE toff, uint64_t DS) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t o = warp; o < ma.count; o += nwarps) {
        uint64_t a0 = seg_offset(ma, o), b0 = KET ? seg_offset(mb, o) : 0;
        double sr = 0, si = 0;
        for (uint64_t a = lane; a < DS; a += 32)
            ptrace_term<R, KET>(in, a0, b0, toff[a], sr, si);
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

// ------------------------------------------- tiled bit permutation
// When every digit's dimension is a power of two, a gather is a permutation
// of index bits: out[o] = in[foff + sum_j bit_j(o) * in_stride[j]]. A plain
// gather writes densely but reads with the stride of whatever input digit
// lands on the output's lowest bits. The tiled form moves 2^TB elements per
// tile through shared memory: the tile's bits are the output's lowest bits
// and the bits with the smallest input strides, so every warp access reads
// 32 consecutive input elements and writes 32 consecutive output elements.
// Every offset is a sum over index bits, split three ways: the lane's five
// bits and the warp's bits give per-thread constants, the remaining bits a
// small table shared by the CTA, and tile bases come from two 128-entry
// tables plus a short loop. The next tile is copied in with cp.async while
// the current one is written out. Tile positions are swizzled by the plan's
// linear map, which folds high position bits into the bank-selecting low
// bits wherever the warp's scattered stores would otherwise pile onto a few
// bank groups.

__device__ __forceinline__ uint32_t perm_swz(const PermPlan& P, uint32_t p, int tb) {
    uint32_t r = 0;
    for (int q = 0; q < tb; ++q)
        if ((p >> q) & 1u) r ^= P.swz_bit[q];
    return r;
}

template <typename R, typename OFF, int TB, int NTHR>
struct PermShape {
    static constexpr uint32_t NT = 1u << TB, NW = NTHR / 32, E = NT / NTHR;
    static constexpr int WB = NW == 8 ? 3 : NW == 16 ? 4 : 5; // warp bits
    static constexpr size_t kTile = size_t(2) * NT * sizeof(Cplx<R>);
    static constexpr size_t kSmem = kTile + 512 * sizeof(OFF) + E * (2 * sizeof(OFF) + 8);
};

template <typename R, typename OFF, int TB, int NTHR>
__global__ void __launch_bounds__(NTHR)
    k_permute_tiled(const Cplx<R>* __restrict__ in, Cplx<R>* __restrict__ out,
                    const __grid_constant__ PermPlan P) {
    using C = Cplx<R>;
    using S = PermShape<R, OFF, TB, NTHR>;
    constexpr uint32_t NT = S::NT, E = S::E;
    constexpr int LB = 5 + S::WB; // bits of the thread (lane, warp); the rest index u
    extern __shared__ __align__(16) unsigned char perm_smem[];
    C* tile = reinterpret_cast<C*>(perm_smem);                  // [2][NT]
    OFF* tb_in = reinterpret_cast<OFF*>(perm_smem + S::kTile);  // [2][128] tile number bits
    OFF* tb_out = tb_in + 256;                                  // [2][128]
    OFF* u_in = tb_out + 256;                                   // [E]
    OFF* u_out = u_in + E;                                      // [E]
    uint32_t* u_spos = reinterpret_cast<uint32_t*>(u_out + E);  // [E]
    uint32_t* u_rpos = u_spos + E;                              // [E]
    const int tid = threadIdx.x;
    const int r0 = P.nrest < 7 ? P.nrest : 7;
    const int r1 = P.nrest - r0 < 7 ? P.nrest - r0 : 7;
    for (int i = tid; i < 256; i += NTHR) {
        const int h = i >> 7, x = i & 127, lo = h ? r0 : 0, cnt = h ? r1 : r0;
        OFF bi = 0, bo = 0;
        for (int j = 0; j < cnt; ++j)
            if ((x >> j) & 1) {
                bi += OFF(P.in_stride[P.rest[lo + j]]);
                bo |= OFF(1) << P.rest[lo + j];
            }
        tb_in[i] = bi;
        tb_out[i] = bo;
    }
    // element l of a tile: bits [0, LB) are the thread (lane + 32 warp), bits
    // [LB, TB) the index u < E of its elements; in read order, l's bits are
    // the tile bits by ascending input stride (input offset, swizzled
    // position of the write-order element it is), in write order the tile
    // bits ascending (output offset, swizzled position)
    auto parts = [&](uint32_t l, int j0, int j1, OFF& io, OFF& oo, uint32_t& sp, uint32_t& rp) {
        io = 0;
        oo = 0;
        uint32_t po = 0;
        for (int j = j0; j < j1; ++j)
            if ((l >> j) & 1u) {
                io += OFF(P.in_stride[P.tin[j]]);
                po |= 1u << P.tin_pos[j];
                oo |= OFF(1) << P.tbits[j];
            }
        sp = perm_swz(P, po, TB);
        rp = perm_swz(P, l, TB);
    };
    if (tid < int(E)) {
        OFF io, oo;
        uint32_t sp, rp;
        parts(uint32_t(tid) << LB, LB, TB, io, oo, sp, rp);
        u_in[tid] = io;
        u_out[tid] = oo;
        u_spos[tid] = sp;
        u_rpos[tid] = rp;
    }
    OFF t_in, t_out;
    uint32_t t_spos, t_rpos;
    parts(uint32_t(tid), 0, LB, t_in, t_out, t_spos, t_rpos);
    __syncthreads();
    const uint64_t ntiles = uint64_t(1) << P.nrest;
    const uint64_t m0 = (uint64_t(1) << r0) - 1, m1 = (uint64_t(1) << r1) - 1;
    auto base = [&](uint64_t t, OFF& bi, OFF& bo) {
        bi = OFF(P.foff) + tb_in[t & m0] + tb_in[128 + ((t >> r0) & m1)];
        bo = tb_out[t & m0] | tb_out[128 + ((t >> r0) & m1)];
        for (int j = r0 + r1; j < P.nrest; ++j)
            if ((t >> j) & 1u) {
                bi += OFF(P.in_stride[P.rest[j]]);
                bo |= OFF(1) << P.rest[j];
            }
    };
    auto issue = [&](OFF bi, C* buf) {
        const C* src = in + bi + t_in;
#pragma unroll
        for (uint32_t u = 0; u < E; ++u) cp_async_elem(buf + (t_spos ^ u_spos[u]), src + u_in[u]);
        cp_async_commit();
    };
    uint64_t t = blockIdx.x;
    if (t >= ntiles) return; // uniform across the CTA
    OFF bi, bo;
    base(t, bi, bo);
    issue(bi, tile);
    for (int it = 0; t < ntiles; t += gridDim.x, ++it) {
        const C* cur = tile + (it & 1) * NT;
        const uint64_t tn = t + gridDim.x;
        OFF bin = 0, bon = 0;
        if (tn < ntiles) {
            base(tn, bin, bon);
            issue(bin, tile + ((it + 1) & 1) * NT);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        C* dst = out + bo + t_out;
#pragma unroll
        for (uint32_t u = 0; u < E; ++u) dst[u_out[u]] = cur[t_rpos ^ u_rpos[u]];
        __syncthreads();
        bo = bon;
    }
}

bool plan_permute(const std::vector<uint64_t>& out_dims, const std::vector<uint64_t>& src,
                  uint64_t fixed_off, PermPlan& P, int elem_bytes, int tile_bits, int out_low) {
    std::memset(&P, 0, sizeof(P));
    P.foff = fixed_off;
    if (tile_bits < kPermTileBits || tile_bits > 12 || out_low < 5 || out_low > tile_bits)
        return false;
    // output bits from the least significant digit up
    for (size_t v = out_dims.size(); v-- > 0;) {
        uint64_t d = out_dims[v];
        if (d == 0 || (d & (d - 1))) return false; // not a power of two
        for (uint64_t s = src[v]; d > 1; d >>= 1, s <<= 1) {
            if (P.nb >= 63) return false;
            P.in_stride[P.nb++] = s;
        }
    }
    if (P.nb < tile_bits + 1) return false;
    P.tb = tile_bits;
    uint64_t mask = (uint64_t(1) << out_low) - 1; // the lowest output bits
    std::vector<int> by_in(P.nb);
    for (int j = 0; j < P.nb; ++j) by_in[j] = j;
    std::stable_sort(by_in.begin(), by_in.end(),
                     [&](int a, int b) { return P.in_stride[a] < P.in_stride[b]; });
    for (int k = 0; k < P.nb && __builtin_popcountll(mask) < P.tb; ++k)
        mask |= uint64_t(1) << by_in[k];
    int c = 0, r = 0;
    for (int j = 0; j < P.nb; ++j) {
        if (mask >> j & 1u) P.tbits[c++] = uint8_t(j);
        else P.rest[r++] = uint8_t(j);
    }
    P.nrest = r;
    c = 0;
    for (int j : by_in)
        if (mask >> j & 1u) {
            P.tin[c] = uint8_t(j);
            for (int q = 0; q < P.tb; ++q)
                if (P.tbits[q] == uint8_t(j)) P.tin_pos[c] = uint8_t(q);
            ++c;
        }
    // Swizzle. A warp access of 128 bytes per wavefront covers 128 /
    // elem_bytes consecutive positions, so the low lb position bits pick the
    // bank group. The row reads vary positions 0-4 across the lanes, which
    // already covers the low lb bits. The scattered stores vary the positions
    // tin_pos[0..4]; each of the low lb bits that none of them is takes the
    // place of one of those positions above lb (folded in by XOR), so the
    // stores cover every bank group too. The map is unipotent, hence a
    // bijection of the tile.
    const int lb = elem_bytes >= 16 ? 3 : 4;
    bool have[4] = {false, false, false, false};
    for (int j = 0; j < 5; ++j)
        if (P.tin_pos[j] < lb) have[P.tin_pos[j]] = true;
    for (int q = 0; q < P.tb; ++q) P.swz_bit[q] = uint16_t(1u << q);
    int next = 0;
    for (int j = 0; j < 5; ++j) {
        const int q = P.tin_pos[j];
        if (q < lb) continue;
        while (next < lb && have[next]) ++next;
        if (next >= lb) break;
        P.swz_bit[q] = uint16_t((1u << q) | (1u << next));
        have[next] = true;
    }
    return true;
}

namespace {
template <typename R, typename OFF, int TB, int NTHR>
void permute_launch(qgpu_ctx* ctx, const void* in, void* out, const PermPlan& P) {
    using S = PermShape<R, OFF, TB, NTHR>;
    auto* kern = k_permute_tiled<R, OFF, TB, NTHR>;
    ensure_smem(reinterpret_cast<const void*>(kern), S::kSmem);
    // one tile per CTA: on a 2^24-element state the tiles moved 5.4 TB/s on
    // average over random permutations this way against 4.9 TB/s with one
    // wave of resident CTAs looping (the next tile's prefetch then has
    // nothing to overlap within a CTA; other CTAs do that)
    const uint64_t ntiles = uint64_t(1) << P.nrest;
    const int b = int(std::min<uint64_t>(ntiles, 0x7fffffffu));
    kern<<<b, NTHR, S::kSmem, ctx->stream>>>(static_cast<const Cplx<R>*>(in),
                                               static_cast<Cplx<R>*>(out), P);
}

template <typename R, typename OFF>
void permute_dispatch(qgpu_ctx* ctx, const void* in, void* out, const PermPlan& P) {
    switch (P.tb) {
    case 10: permute_launch<R, OFF, 10, 256>(ctx, in, out, P); break;
    case 11: permute_launch<R, OFF, 11, 512>(ctx, in, out, P); break;
    default: permute_launch<R, OFF, 12, 512>(ctx, in, out, P); break;
    }
}
} // namespace

// The tile shape: TB tile bits, the OUT lowest output bits among them.
constexpr int kPermTileTB = 10, kPermTileOut = 5;

bool launch_permute_tiled(qgpu_ctx* ctx, qgpu_prec prec, const void* in, void* out,
                          const std::vector<uint64_t>& out_dims,
                          const std::vector<uint64_t>& src, uint64_t fixed_off) {
    PermPlan P;
    if (!plan_permute(out_dims, src, fixed_off, P, prec == QGPU_C128 ? 16 : 8, kPermTileTB,
                      kPermTileOut))
        return false;
    // 32-bit offsets when every input and output offset fits (the output has
    // 2^nb elements; the input offsets are bounded by the fixed offset plus
    // every stride)
    uint64_t in_max = P.foff;
    for (int j = 0; j < P.nb; ++j) in_max += P.in_stride[j];
    const bool narrow = P.nb <= 31 && in_max < (uint64_t(1) << 31);
    if (prec == QGPU_C128) {
        if (narrow) permute_dispatch<double, uint32_t>(ctx, in, out, P);
        else permute_dispatch<double, uint64_t>(ctx, in, out, P);
    } else {
        if (narrow) permute_dispatch<float, uint32_t>(ctx, in, out, P);
        else permute_dispatch<float, uint64_t>(ctx, in, out, P);
    }
    after_launch(ctx, "k_permute_tiled");
    return true;
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

template <typename R, typename TABLE>
static void ptr_launch(qgpu_ctx* ctx, const Cplx<R>* i, Cplx<R>* o, const SegPlan& ma,
                       const SegPlan& mb, const TABLE& t, uint64_t DS, bool is_ket) {
    // few outputs with long sums: a warp per output
    bool warp = ma.count < uint64_t(ctx->num_sms) * 2048 && DS >= 32;
    if (warp) {
        int b = blocks_for(ctx, ma.count * 32, 8);
        if (is_ket)
            k_ptrace_warp<R, true, TABLE><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, t, DS);
        else
            k_ptrace_warp<R, false, TABLE><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, t, DS);
    } else {
        int b = blocks_for(ctx, ma.count, 8);
        if (is_ket)
            k_ptrace_thread<R, true, TABLE><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, t, DS);
        else
            k_ptrace_thread<R, false, TABLE><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, t, DS);
    }
    after_launch(ctx, "k_ptrace");
}

template <typename R>
static void ptr(qgpu_ctx* ctx, const void* in, void* out, const SegPlan& ma,
                const SegPlan& mb, const std::vector<uint64_t>& toff,
                bool is_ket) {
    uint64_t DS = toff.size();
    const Cplx<R>* i = static_cast<const Cplx<R>*>(in);
    Cplx<R>* o = static_cast<Cplx<R>*>(out);
    if (DS <= uint64_t(kPtraceTab)) {
        // small tables travel with the launch (no host-to-device copy)
        PtraceTab tab;
        std::memset(&tab, 0, sizeof(tab));
        std::copy(toff.begin(), toff.end(), tab.t);
        ptr_launch<R, PtraceTab>(ctx, i, o, ma, mb, tab, DS, is_ket);
        return;
    }
    uint64_t* dt = static_cast<uint64_t*>(ctx_scratch(ctx, DS * sizeof(uint64_t)));
    QG_CUDA(cudaMemcpyAsync(dt, toff.data(), DS * sizeof(uint64_t),
                            cudaMemcpyHostToDevice, ctx->stream));
    const uint64_t* cdt = dt;
    ptr_launch<R, const uint64_t*>(ctx, i, o, ma, mb, cdt, DS, is_ket);
}

void launch_ptrace(qgpu_ctx* ctx, qgpu_prec prec, const void* in, void* out,
                   const SegPlan& ma, const SegPlan& mb,
                   const std::vector<uint64_t>& toff, bool is_ket) {
    if (ma.count == 0) return;
    if (prec == QGPU_C128) ptr<double>(ctx, in, out, ma, mb, toff, is_ket);
    else ptr<float>(ctx, in, out, ma, mb, toff, is_ket);
}

} // namespace qgpu

// ======================================================================
// Allocation-free partial trace (qgpu_ptrace_noalloc).
//
// Some callers cannot allocate device memory at the moment they need a
// partial trace: a host application whose memory pool owns all of the
// GPU's free memory, or a latency-critical loop where the implicit device
// synchronisation of cudaMalloc/cudaFree is not acceptable. For them the
// table of traced offsets lives in a fixed array in device memory that the
// library reserves when it is loaded (512 KB on every GPU that loads it,
// held until the process exits), and the result goes to a buffer the caller
// already owns. Nothing is allocated on the device or the host on the
// success path.
// ======================================================================
#include <mutex>

#include "capi_common.hpp"

namespace qgpu {

constexpr uint64_t kNoAllocMaxTraced = 65536; // entries of the offset table

static __device__ __align__(256) uint64_t g_noalloc_toff[kNoAllocMaxTraced];

struct TraceDigits {
    int k;
    uint64_t dim[64];
    uint64_t stride[64]; // element stride of each traced digit (row + column for rho)
};

// toff[a] = sum_j digit_j(a) * stride[j], digits big-endian over the traced
// subsystems in the order given.
__global__ void __launch_bounds__(256)
    k_fill_toff(uint64_t* __restrict__ toff, uint64_t DS, const __grid_constant__ TraceDigits td) {
    for (uint64_t a = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; a < DS;
         a += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t r = a, o = 0;
        for (int j = td.k - 1; j >= 0; --j) {
            o += (r % td.dim[j]) * td.stride[j];
            r /= td.dim[j];
        }
        toff[a] = o;
    }
}

// Device address of g_noalloc_toff, looked up once per device with that
// device current (the host-side symbol is only a stand-in, never a device
// address), and looked up again after qgpu_ctx_create on the device
// (noalloc_forget), since a cudaDeviceReset in between reloads the module
// and can move the array.
static std::mutex g_noalloc_mu;
static uint64_t* g_noalloc_addr[64] = {nullptr};

void noalloc_forget(int device) {
    if (device < 0 || device >= 64) return;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    g_noalloc_addr[device] = nullptr;
}

static uint64_t* noalloc_table(int device) {
    uint64_t** addr = g_noalloc_addr;
    if (device < 0 || device >= 64)
        raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_ptrace_noalloc()", "device index above 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_toff);
        if (e != cudaSuccess)
            raise(QGPU_ERR_CUDA, "qgpu_ptrace_noalloc()", cudaGetErrorString(e));
        addr[device] = static_cast<uint64_t*>(p);
    }
    return addr[device];
}

// Merged gather plan over fixed-size arrays (same rule as plan_gather).
static void plan_gather_fixed(const uint64_t* od, const uint64_t* src, int n, SegPlan& p) {
    std::memset(&p, 0, sizeof(p));
    bool run = false;
    uint64_t cs = 1, cst = 0;
    auto push = [&](uint64_t size, uint64_t stride) {
        if (size == 1) return;
        if (p.nseg >= kMaxSeg)
            raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_ptrace_noalloc()", "too many index segments");
        p.size[p.nseg] = size;
        p.stride[p.nseg] = stride;
        ++p.nseg;
    };
    for (int v = n - 1; v >= 0; --v) {
        if (od[v] == 1) continue;
        if (!run) {
            cs = od[v];
            cst = src[v];
            run = true;
        } else if (src[v] == cst * cs) {
            cs *= od[v];
        } else {
            push(cs, cst);
            cs = od[v];
            cst = src[v];
        }
    }
    if (run) push(cs, cst);
    p.count = 1;
    p.pow2 = 1;
    for (int s = 0; s < p.nseg; ++s) {
        p.count *= p.size[s];
        if (p.size[s] & (p.size[s] - 1)) p.pow2 = 0;
        int sh = 0;
        while ((uint64_t(1) << sh) < p.size[s]) ++sh;
        p.shift[s] = uint8_t(sh);
    }
}

template <typename R>
static void noalloc_launch(qgpu_ctx* ctx, const void* in, void* out, const SegPlan& ma,
                           const SegPlan& mb, const uint64_t* toff, uint64_t DS, bool ket) {
    const Cplx<R>* i = static_cast<const Cplx<R>*>(in);
    Cplx<R>* o = static_cast<Cplx<R>*>(out);
    bool warp = ma.count < uint64_t(ctx->num_sms) * 2048 && DS >= 32;
    int b = blocks_for(ctx, warp ? ma.count * 32 : ma.count, 8);
    if (warp) {
        if (ket) k_ptrace_warp<R, true><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, toff, DS);
        else k_ptrace_warp<R, false><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, toff, DS);
    } else {
        if (ket) k_ptrace_thread<R, true><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, toff, DS);
        else k_ptrace_thread<R, false><<<b, 256, 0, ctx->stream>>>(i, o, ma, mb, toff, DS);
    }
    after_launch(ctx, "k_ptrace (no-alloc)");
}

} // namespace qgpu

extern "C" qgpu_status qgpu_ptrace_noalloc(const qgpu_state* s, const uint64_t* target,
                                           uint32_t k, void* d_out) {
    using namespace qgpu;
    return guarded([&] {
        const char* W = "qgpu_ptrace_noalloc()";
        need_handle(s);
        if (!d_out) raise(QGPU_ERR_INVALID_ARGUMENT, W, "d_out");
        const int n = int(s->dims.size());
        if (n > 64) raise(QGPU_ERR_NOT_SUPPORTED, W, "more than 64 subsystems");
        if (k > uint32_t(n) || (k > 0 && !target))
            raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
        bool traced[64] = {false};
        for (uint32_t j = 0; j < k; ++j) {
            if (target[j] >= uint64_t(n) || traced[target[j]])
                raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
            traced[target[j]] = true;
        }
        uint64_t stride[64];
        stride[n - 1] = 1;
        for (int q = n - 1; q > 0; --q) stride[q - 1] = stride[q] * s->dims[size_t(q)];
        const bool ket = s->kind == QGPU_KET;
        const uint64_t D = s->D;
        TraceDigits td;
        td.k = int(k);
        uint64_t DS = 1;
        for (uint32_t j = 0; j < k; ++j) {
            uint64_t q = target[j];
            td.dim[j] = s->dims[q];
            td.stride[j] = ket ? stride[q] : stride[q] * (D + 1);
            DS *= s->dims[q];
        }
        if (DS > kNoAllocMaxTraced)
            raise(QGPU_ERR_NOT_SUPPORTED, W,
                  "traced dimension above 65536 (the fixed offset table)");
        // output digits: [column digits of the kept subsystems, row digits]
        uint64_t od[128], sa[128], sb[128];
        int no = 0;
        for (int q = 0; q < n; ++q)
            if (!traced[q]) {
                od[no] = s->dims[size_t(q)];
                sa[no] = ket ? 0 : stride[q] * D;
                sb[no] = ket ? stride[q] : 0;
                ++no;
            }
        for (int q = 0; q < n; ++q)
            if (!traced[q]) {
                od[no] = s->dims[size_t(q)];
                sa[no] = stride[q];
                sb[no] = 0;
                ++no;
            }
        SegPlan ma, mb;
        plan_gather_fixed(od, sa, no, ma);
        plan_gather_fixed(od, sb, no, mb);
        int prev = 0;
        QG_CUDA(cudaGetDevice(&prev));
        QG_CUDA(cudaSetDevice(s->ctx->device));
        try {
            uint64_t* toff = noalloc_table(s->ctx->device);
            int fb = int(std::min<uint64_t>((DS + 255) / 256, 1024));
            k_fill_toff<<<fb, 256, 0, s->ctx->stream>>>(toff, DS, td);
            after_launch(s->ctx, "k_fill_toff");
            if (s->prec == QGPU_C128)
                noalloc_launch<double>(s->ctx, s->data, d_out, ma, mb, toff, DS, ket);
            else
                noalloc_launch<float>(s->ctx, s->data, d_out, ma, mb, toff, DS, ket);
        } catch (...) {
            cudaSetDevice(prev);
            throw;
        }
        QG_CUDA(cudaSetDevice(prev));
    });
}
