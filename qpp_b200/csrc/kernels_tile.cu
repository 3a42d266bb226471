// kernels_tile.cu -- cache-blocked tile passes: runs of 1- and 2-qubit gates
// (controlled or not) applied to a qubit ket in one read and one write of the
// state.
//
// Replaces, for runs of consecutive gates, the one-pass-per-gate loops of
// include/qpp/internal/kernels/qubit/apply.hpp:57-265 (apply_psi_1q/2q) and
// apply_ctrl.hpp:63-265 (apply_ctrl_psi_1q/2q). A pass owns a set of "tile
// bits": the L lowest state bits (contiguous runs of 2^L amplitudes, so loads
// and stores are coalesced) and up to T - L higher bits chosen by the host
// planner so that every target of every gate in the run is a tile bit. Each
// CTA copies a 2^T-amplitude tile (all values of the tile bits, the other
// bits fixed) into shared memory with cp.async, applies every gate of the
// run there -- a control on a tile bit is tested per amplitude, a control on
// any other bit once per tile -- and writes the tile back. The arithmetic per
// amplitude is the same as the one-gate kernels' (k_qubit_1q / k_qubit_2q:
// the same products and fused multiply-adds in the same order), so the
// results are those of applying the gates one pass at a time.
//
// Inside a tile the gates run in "sweeps": consecutive gates whose targets
// lie within three tile bits share one trip through shared memory. Every
// thread takes groups of up to 8 amplitudes (those that differ only in the
// sweep's bits) into registers, applies each gate of the sweep there (the
// group bit positions are compile-time constants, selected by a switch), and
// writes the group back; one barrier per sweep instead of one per gate. The
// tile is stored with its bank columns XOR-swizzled by its row number, which
// keeps the strided group accesses of sweeps on low tile bits within two
// wavefronts per phase.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "kernels.hpp"

namespace qgpu {

constexpr int kTileThreads = 512;
constexpr size_t kTileSmemMax = 227 * 1024; // the opt-in maximum per block

// Shared-memory position of tile element e: the element's bank column (the
// low CB bits; 2^CB elements per 128-byte row) XORed with every CB-bit chunk
// of its row number, so that elements whose indices differ in bits of
// distinct classes (bit mod CB) land in distinct columns.
template <int CB>
__device__ __forceinline__ uint32_t tswz(uint32_t e) {
    uint32_t r = e >> CB, h = 0;
#pragma unroll
    for (int k = 0; k < 16; k += CB) h ^= r >> k;
    return e ^ (h & ((1u << CB) - 1));
}

// The per-element control test selects between the new and the old values
// instead of branching around the arithmetic, so the pairs' multiply-add
// chains stay in one basic block and interleave; gates without tile-bit
// controls (CTRL = false) skip the test.
template <bool CTRL, typename C>
__device__ __forceinline__ C pick(bool ok, const C& nv, const C& ov) {
    if constexpr (!CTRL) return nv;
    C r;
    r.x = ok ? nv.x : ov.x;
    r.y = ok ? nv.y : ov.y;
    return r;
}

// 2 x 2 (row-major m) on group bit K of the registers v[0, 2^NB), for the
// elements whose tile index (b + off[j]) passes the tile-bit controls.
template <typename C, int NB, int K, bool CTRL>
__device__ __forceinline__ void group_1q(C (&v)[1 << NB], const C* m, uint32_t b,
                                         const uint32_t (&off)[1 << NB], uint32_t lmask,
                                         uint32_t lval) {
    const C a00 = m[0], a01 = m[1], a10 = m[2], a11 = m[3];
#pragma unroll
    for (int j = 0; j < (1 << NB); ++j) {
        if (j & (1 << K)) continue; // compile-time
        const bool ok = ((b + off[j]) & lmask) == lval;
        const int j1 = j | (1 << K);
        C r0 = cmul(a00, v[j]);
        r0 = cfma(a01, v[j1], r0);
        C r1 = cmul(a10, v[j]);
        r1 = cfma(a11, v[j1], r1);
        v[j] = pick<CTRL>(ok, r0, v[j]);
        v[j1] = pick<CTRL>(ok, r1, v[j1]);
    }
}

// 4 x 4 (row-major m, row index 2 * b(K0) + b(K1)) on group bits K0, K1.
template <typename C, int NB, int K0, int K1, bool CTRL>
__device__ __forceinline__ void group_2q(C (&v)[1 << NB], const C* m, uint32_t b,
                                         const uint32_t (&off)[1 << NB], uint32_t lmask,
                                         uint32_t lval) {
#pragma unroll
    for (int j = 0; j < (1 << NB); ++j) {
        if (j & ((1 << K0) | (1 << K1))) continue; // compile-time
        const bool ok = ((b + off[j]) & lmask) == lval;
        const int j1 = j | (1 << K1), j2 = j | (1 << K0), j3 = j | (1 << K0) | (1 << K1);
        const C x0 = v[j], x1 = v[j1], x2 = v[j2], x3 = v[j3];
        C r[4];
#pragma unroll
        for (int row = 0; row < 4; ++row) {
            C acc = cmul(m[4 * row], x0);
            acc = cfma(m[4 * row + 1], x1, acc);
            acc = cfma(m[4 * row + 2], x2, acc);
            acc = cfma(m[4 * row + 3], x3, acc);
            r[row] = acc;
        }
        v[j] = pick<CTRL>(ok, r[0], x0);
        v[j1] = pick<CTRL>(ok, r[1], x1);
        v[j2] = pick<CTRL>(ok, r[2], x2);
        v[j3] = pick<CTRL>(ok, r[3], x3);
    }
}

template <typename C, int NB, bool CTRL>
__device__ __forceinline__ void group_gate_c(C (&v)[1 << NB], const TileGate& g, const C* m,
                                             uint32_t b, const uint32_t (&off)[1 << NB]) {
#define QG_1Q(K)                                                                     \
    case K:                                                                          \
        if constexpr (NB > K) group_1q<C, NB, K, CTRL>(v, m, b, off, g.lmask, g.lval); \
        break;
#define QG_2Q(K0, K1)                                                                           \
    case K0 * 4 + K1:                                                                           \
        if constexpr (NB > K0 && NB > K1)                                                       \
            group_2q<C, NB, K0, K1, CTRL>(v, m, b, off, g.lmask, g.lval);                       \
        break;
    if (g.op == 1) {
        switch (g.k0) { QG_1Q(0) QG_1Q(1) QG_1Q(2) }
        return;
    }
    switch (g.k0 * 4 + g.k1) {
        QG_2Q(0, 1) QG_2Q(1, 0) QG_2Q(0, 2) QG_2Q(2, 0) QG_2Q(1, 2) QG_2Q(2, 1)
    }
#undef QG_1Q
#undef QG_2Q
}

template <typename C, int NB>
__device__ __forceinline__ void group_gate(C (&v)[1 << NB], const TileGate& g, const C* m,
                                           uint32_t b, const uint32_t (&off)[1 << NB]) {
    if (g.lmask) group_gate_c<C, NB, true>(v, g, m, b, off);
    else group_gate_c<C, NB, false>(v, g, m, b, off);
}

// One sweep over the tile: groups of 2^NB amplitudes through registers. The
// swizzle is linear over GF(2) and the group's element bits are disjoint from
// its base bits, so an element's position is swz(base) ^ swz(off[j]), with
// swz(off[j]) computed once per sweep.
template <typename C, int NB, int CB>
__device__ __forceinline__ void run_sweep(C* tile, int T, const TileSweep& gsw,
                                          const TileGate* sgates, const C* smat,
                                          uint32_t first_gate, uint32_t mat_first,
                                          uint64_t base) {
    constexpr int G = 1 << NB;
    const uint32_t ngates = gsw.ngates, first = gsw.first;
    int sbits[NB];
#pragma unroll
    for (int k = 0; k < NB; ++k) sbits[k] = gsw.b[k];
    uint32_t off[G], soff[G];
#pragma unroll
    for (int j = 0; j < G; ++j) {
        uint32_t o = 0;
#pragma unroll
        for (int k = 0; k < NB; ++k)
            if (j & (1 << k)) o |= 1u << sbits[k];
        off[j] = o;
        soff[j] = tswz<CB>(o);
    }
    int sorted[NB]; // the sweep's bits ascending, for the zero insertion
#pragma unroll
    for (int k = 0; k < NB; ++k) sorted[k] = sbits[k];
#pragma unroll
    for (int x = 0; x < NB; ++x)
#pragma unroll
        for (int y = x + 1; y < NB; ++y)
            if (sorted[y] < sorted[x]) {
                const int t = sorted[x];
                sorted[x] = sorted[y];
                sorted[y] = t;
            }
    const int nq = T - NB;
    for (uint32_t q = threadIdx.x; q < (1u << nq); q += kTileThreads) {
        uint32_t b = q;
#pragma unroll
        for (int k = 0; k < NB; ++k) {
            const uint32_t low = (1u << sorted[k]) - 1;
            b = ((b & ~low) << 1) | (b & low);
        }
        const uint32_t sb = tswz<CB>(b);
        C v[G];
#pragma unroll
        for (int j = 0; j < G; ++j) v[j] = tile[sb ^ soff[j]];
        for (uint32_t k = 0; k < ngates; ++k) {
            const TileGate& g = sgates[first - first_gate + k];
            if ((base & g.gmask) != g.gval) continue; // a control outside the tile
            group_gate<C, NB>(v, g, smat + (g.mat - mat_first), b, off);
        }
#pragma unroll
        for (int j = 0; j < G; ++j) tile[sb ^ soff[j]] = v[j];
    }
}

template <typename R>
__global__ void __launch_bounds__(kTileThreads, 1)
    k_tile_pass(Cplx<R>* __restrict__ psi, const __grid_constant__ TilePassParams p,
                const TileGate* __restrict__ gates, const TileSweep* __restrict__ sweeps,
                const Cplx<R>* __restrict__ mats) {
    using C = Cplx<R>;
    constexpr int NT = kTileThreads;
    constexpr int CB = sizeof(C) == 16 ? 3 : 4; // log2(elements per 128-byte row)
    extern __shared__ __align__(16) unsigned char tile_raw[];
    C* tile = reinterpret_cast<C*>(tile_raw);
    const int nhi = p.T - p.L;
    // after the tile: the offset table of the high tile bits, the pass's gate
    // descriptors and its matrices (read by every tile of this CTA)
    unsigned char* q = tile_raw + (sizeof(C) << p.T);
    uint64_t* hioff = reinterpret_cast<uint64_t*>(q);
    q += ((sizeof(uint64_t) << nhi) + 15) / 16 * 16;
    TileGate* sgates = reinterpret_cast<TileGate*>(q);
    q += (sizeof(TileGate) * p.ngates + 15) / 16 * 16;
    C* smat = reinterpret_cast<C*>(q);
    const int tid = threadIdx.x;
    const uint32_t nel = 1u << p.T, lmask = (1u << p.L) - 1;
    for (uint32_t j = tid; j < (1u << nhi); j += NT) {
        uint64_t o = 0;
        for (int i = 0; i < nhi; ++i)
            if ((j >> i) & 1u) o |= uint64_t(1) << p.hi[i];
        hioff[j] = o;
    }
    for (uint32_t j = tid; j < p.ngates; j += NT) sgates[j] = gates[p.first + j];
    for (uint32_t j = tid; j < p.mat_elems; j += NT) smat[j] = mats[p.mat_first + j];
    __syncthreads();
    for (uint64_t t = blockIdx.x; t < p.ntiles; t += gridDim.x) {
        // tile number -> base offset: zeros inserted at every tile bit
        uint64_t base = t << p.L;
        for (int i = 0; i < nhi; ++i) {
            const uint64_t low = (uint64_t(1) << p.hi[i]) - 1;
            base = ((base & ~low) << 1) | (base & low);
        }
        for (uint32_t e = tid; e < nel; e += NT)
            cp_async_elem(&tile[tswz<CB>(e)], &psi[base + hioff[e >> p.L] + (e & lmask)]);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        for (uint32_t s = 0; s < p.nsweeps; ++s) {
            const TileSweep& sw = sweeps[p.first_sweep + s];
            switch (sw.nb) {
                case 3: run_sweep<C, 3, CB>(tile, p.T, sw, sgates, smat, p.first, p.mat_first, base); break;
                case 2: run_sweep<C, 2, CB>(tile, p.T, sw, sgates, smat, p.first, p.mat_first, base); break;
                default: run_sweep<C, 1, CB>(tile, p.T, sw, sgates, smat, p.first, p.mat_first, base); break;
            }
            __syncthreads();
        }
        for (uint32_t e = tid; e < nel; e += NT)
            psi[base + hioff[e >> p.L] + (e & lmask)] = tile[tswz<CB>(e)];
        __syncthreads();
    }
}

size_t tile_pass_smem(qgpu_prec prec, const TilePassParams& p) {
    const size_t elem = prec == QGPU_C128 ? 16 : 8;
    return (elem << p.T) + ((sizeof(uint64_t) << (p.T - p.L)) + 15) / 16 * 16 +
           (sizeof(TileGate) * p.ngates + 15) / 16 * 16 + elem * p.mat_elems;
}

void launch_tile_pass(qgpu_ctx* ctx, qgpu_prec prec, void* data, const TilePassParams& p,
                      const TileGate* gates, const TileSweep* sweeps, const void* mats) {
    const size_t smem = tile_pass_smem(prec, p);
    if (smem > kTileSmemMax)
        raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_run_gates()", "tile above the shared memory");
    ensure_smem(prec == QGPU_C128 ? reinterpret_cast<const void*>(k_tile_pass<double>)
                                  : reinterpret_cast<const void*>(k_tile_pass<float>),
                kTileSmemMax);
    // residency per SM from shared memory (228 KB, 1 KB reserved per CTA)
    // and threads (2048)
    const int per_sm = std::max(1, std::min(2048 / kTileThreads, int(232448 / (smem + 1024))));
    const int grid = int(std::min<uint64_t>(p.ntiles, uint64_t(ctx->num_sms) * per_sm));
    if (prec == QGPU_C128)
        k_tile_pass<double><<<grid, kTileThreads, smem, ctx->stream>>>(
            static_cast<double2*>(data), p, gates, sweeps, static_cast<const double2*>(mats));
    else
        k_tile_pass<float><<<grid, kTileThreads, smem, ctx->stream>>>(
            static_cast<float2*>(data), p, gates, sweeps, static_cast<const float2*>(mats));
    after_launch(ctx, "k_tile_pass");
}

} // namespace qgpu
