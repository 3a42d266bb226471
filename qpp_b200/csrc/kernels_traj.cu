// kernels_traj.cu -- noisy circuit trajectories with the whole state in
// shared memory: one CTA runs one trajectory (one shot) of a QNoisyEngine
// request from start to finish, and one launch carries the trajectories of
// many requests (the serving loop's batched form).
//
// Semantics follow include/qpp/classes/qnoisy_engine.hpp:105-139: before every
// circuit step each non-measured qubit draws one Kraus index of the
// depolarising channel {I, X, Y, Z} with probabilities {1-p, p/3, p/3, p/3}
// (noise.hpp:388-412); Z-basis measurements follow measure_seq
// (instruments.hpp:985-1111) one qubit at a time; a destructively measured
// qubit stays in the register fixed at its outcome and is never touched
// again (equivalent to qpp removing it). After the last step one full-basis
// index is sampled from |psi|^2 (the shot's result).
//
// Arithmetic: amplitudes in complex64 with FP32 arithmetic; measurement
// probabilities, renormalisation factors and the final sampling prefix sums
// in FP64. Randomness: Philox4x32-10 keyed by the request seed with counter
// (shot, instruction, qubit, purpose), so every draw is reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

#include "common.cuh"
#include "kernels.hpp"
#include "traj.hpp"

namespace qgpu {

__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 c_fma(float2 a, float2 b, float2 c) {
    c.x = fmaf(a.x, b.x, c.x);
    c.x = fmaf(-a.y, b.y, c.x);
    c.y = fmaf(a.x, b.y, c.y);
    c.y = fmaf(a.y, b.x, c.y);
    return c;
}

__device__ __forceinline__ uint32_t ins0(uint32_t x, int b) {
    uint32_t low = (1u << b) - 1;
    return ((x & ~low) << 1) | (x & low);
}

// block-wide FP64 sum (256 threads), result broadcast to every thread
__device__ double block_sum_d(double v, double* red) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v += __shfl_down_sync(0xffffffffu, v, s);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double t = 0;
    for (int i = 0; i < int(blockDim.x >> 5); ++i) t += red[i];
    return t;
}

// kTG3: 8 x 8 on bits (b0, b1, b2 = cmask & 255), row index 4 b0 + 2 b1 + b2;
// each thread owns whole groups. The row loop stays rolled so that the 64
// matrix entries are read per row (L1) rather than held in registers.
__device__ __forceinline__ void tr_gate3(const TInstr& I, const float2* __restrict__ mats,
                                      float2* psi, uint32_t N, int tid, int nt) {
    const float2* m = mats + I.mat;
    const int b2 = int(I.cmask & 255u);
    int sb[3] = {I.b0, I.b1, b2};
    if (sb[0] > sb[1]) { const int t = sb[0]; sb[0] = sb[1]; sb[1] = t; }
    if (sb[1] > sb[2]) { const int t = sb[1]; sb[1] = sb[2]; sb[2] = t; }
    if (sb[0] > sb[1]) { const int t = sb[0]; sb[0] = sb[1]; sb[1] = t; }
    const uint32_t o4 = 1u << I.b0, o2 = 1u << I.b1, o1 = 1u << b2;
    for (uint32_t g = tid; g < N / 8; g += nt) {
        const uint32_t i = ins0(ins0(ins0(g, sb[0]), sb[1]), sb[2]);
        float2 v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c)
            v[c] = psi[i + ((c & 4) ? o4 : 0u) + ((c & 2) ? o2 : 0u) + ((c & 1) ? o1 : 0u)];
        // all eight inputs are in registers, so each row writes in place
#pragma unroll 1
        for (int row = 0; row < 8; ++row) {
            const float2* mr = m + row;
            float2 acc = c_mul(mr[0], v[0]);
#pragma unroll
            for (int c = 1; c < 8; ++c) acc = c_fma(mr[8 * c], v[c], acc);
            psi[i + ((row & 4) ? o4 : 0u) + ((row & 2) ? o2 : 0u) + ((row & 1) ? o1 : 0u)] = acc;
        }
    }
}

// One gate instruction (G1, CG1, G2, G3, G4) on a register of N amplitudes at
// psi (shared or global memory); every thread of the CTA calls it.
__device__ __forceinline__ void tr_gate(const TInstr& I, const float2* __restrict__ mats,
                                        float2* psi, uint32_t N, int tid, int nt) {
    switch (I.op) {
        case kTG1: {
            const float2* m = mats + I.mat; // column-major 2 x 2
            const float2 a00 = m[0], a10 = m[1], a01 = m[2], a11 = m[3];
            const uint32_t s = 1u << I.b0;
            for (uint32_t p = tid; p < N / 2; p += nt) {
                uint32_t i = ins0(p, I.b0);
                float2 v0 = psi[i], v1 = psi[i + s];
                psi[i] = c_fma(a01, v1, c_mul(a00, v0));
                psi[i + s] = c_fma(a11, v1, c_mul(a10, v0));
            }
            break;
        }
        case kTCG1: {
            const float2* m = mats + I.mat;
            const float2 a00 = m[0], a10 = m[1], a01 = m[2], a11 = m[3];
            const uint32_t s = 1u << I.b0;
            for (uint32_t p = tid; p < N / 2; p += nt) {
                uint32_t i = ins0(p, I.b0);
                if ((i & I.cmask) != I.cval) continue;
                float2 v0 = psi[i], v1 = psi[i + s];
                psi[i] = c_fma(a01, v1, c_mul(a00, v0));
                psi[i + s] = c_fma(a11, v1, c_mul(a10, v0));
            }
            break;
        }
        case kTG2: {
            const float2* m = mats + I.mat; // column-major 4 x 4
            const int lo = min(I.b0, I.b1), hi = max(I.b0, I.b1);
            const uint32_t s0 = 1u << I.b0, s1 = 1u << I.b1;
            for (uint32_t p = tid; p < N / 4; p += nt) {
                uint32_t i = ins0(ins0(p, lo), hi);
                float2 v[4] = {psi[i], psi[i + s1], psi[i + s0], psi[i + s0 + s1]};
                float2 r[4];
#pragma unroll
                for (int row = 0; row < 4; ++row) {
                    float2 acc = c_mul(m[row], v[0]);
                    acc = c_fma(m[row + 4], v[1], acc);
                    acc = c_fma(m[row + 8], v[2], acc);
                    acc = c_fma(m[row + 12], v[3], acc);
                    r[row] = acc;
                }
                psi[i] = r[0];
                psi[i + s1] = r[1];
                psi[i + s0] = r[2];
                psi[i + s0 + s1] = r[3];
            }
            break;
        }
        case kTG3:
            tr_gate3(I, mats, psi, N, tid, nt);
            break;
        case kTG4: {
            // 16 x 16 on bits (b0, b1, b2, b3) = (b0, b1, cmask & 255,
            // cmask >> 8 & 255); row index 8 b0 + 4 b1 + 2 b2 + b3
            const float2* m = mats + I.mat;
            const int bb[4] = {I.b0, I.b1, int(I.cmask & 255u), int((I.cmask >> 8) & 255u)};
            int sb[4] = {bb[0], bb[1], bb[2], bb[3]};
#pragma unroll
            for (int x = 0; x < 3; ++x)
#pragma unroll
                for (int y = 0; y < 3 - x; ++y)
                    if (sb[y] > sb[y + 1]) {
                        int tmp = sb[y];
                        sb[y] = sb[y + 1];
                        sb[y + 1] = tmp;
                    }
            auto off = [&](int r) {
                return ((uint32_t(r) >> 3 & 1u) << bb[0]) | ((uint32_t(r) >> 2 & 1u) << bb[1]) |
                       ((uint32_t(r) >> 1 & 1u) << bb[2]) | ((uint32_t(r) & 1u) << bb[3]);
            };
            // one output row per thread (16 groups per round): read
            // everything, barrier, then write in place
            const int row = tid & 15;
            const uint32_t gpp = uint32_t(nt) >> 4;
            for (uint32_t g0 = 0; g0 < N / 16; g0 += gpp) {
                const uint32_t g = g0 + (uint32_t(tid) >> 4);
                const bool valid = g < N / 16;
                uint32_t i = 0;
                float2 acc = make_float2(0.f, 0.f);
                if (valid) {
                    i = ins0(ins0(ins0(ins0(g, sb[0]), sb[1]), sb[2]), sb[3]);
#pragma unroll 4
                    for (int c = 0; c < 16; ++c) acc = c_fma(m[row + 16 * c], psi[i + off(c)], acc);
                }
                __syncthreads();
                if (valid) psi[i + off(row)] = acc;
                __syncthreads();
            }
            break;
        }
        default:
            break;
    }
}

// Depolarising draws of one circuit step (counter `ins` = the instruction's
// index in the untiled program): thread b <-> qubit b. Returns whether any
// qubit drew a Pauli (uniform over the CTA). With `apply`, the Pauli string is
// recorded and applied to all N amplitudes at psi.
__device__ bool tr_noise(const TWork& W, uint32_t ins, int n, uint32_t alive, bool apply,
                         float2* psi, uint32_t N, TEvent* events, int max_events,
                         uint32_t* sh /* xm, zm, ny, nev */) {
    const int tid = threadIdx.x, nt = blockDim.x;
    int pk = 0;
    if (tid < n && ((alive >> tid) & 1u)) {
        double u0, u1;
        philox_uniform2(W.seed, W.shot, ins, uint32_t(tid), 0x6e6f6973u, u0, u1);
        if (u0 < double(W.p_noise)) pk = 1 + min(int(u1 * 3.0), 2); // 1 X, 2 Y, 3 Z
    }
    if (!__syncthreads_or(pk != 0)) return false;
    if (!apply) return true;
    if (tid == 0) sh[0] = sh[1] = sh[2] = 0;
    __syncthreads();
    if (pk) {
        if (pk != 3) atomicOr(&sh[0], 1u << tid);
        if (pk != 1) atomicOr(&sh[1], 1u << tid);
        if (pk == 2) atomicAdd(&sh[2], 1u);
        if (events) {
            uint32_t e = atomicAdd(&sh[3], 1u);
            if (int(e) < max_events)
                events[size_t(W.out) * max_events + e] = TEvent{ins, uint16_t(tid), uint16_t(pk)};
        }
    }
    __syncthreads();
    const uint32_t xm = sh[0], zm = sh[1], ny = sh[2];
    // P|i> = i^ny (-1)^popc(i & zm) |i ^ xm>
    const float2 gph = ny % 4 == 0 ? make_float2(1, 0)
                     : ny % 4 == 1 ? make_float2(0, 1)
                     : ny % 4 == 2 ? make_float2(-1, 0) : make_float2(0, -1);
    if (xm == 0) {
        for (uint32_t i = tid; i < N; i += nt) {
            float2 a = c_mul(gph, psi[i]);
            if (__popc(i & zm) & 1) a = make_float2(-a.x, -a.y);
            psi[i] = a;
        }
    } else {
        int hb = 31 - __clz(xm); // pair (i, i ^ xm) with bit hb of i clear
        for (uint32_t p = tid; p < N / 2; p += nt) {
            uint32_t i = ins0(p, hb), j = i ^ xm;
            float2 a = c_mul(gph, psi[i]), b = c_mul(gph, psi[j]);
            if (__popc(i & zm) & 1) a = make_float2(-a.x, -a.y);
            if (__popc(j & zm) & 1) b = make_float2(-b.x, -b.y);
            psi[j] = a;
            psi[i] = b;
        }
    }
    __syncthreads();
    return true;
}

// A tile pass (kTTile header H at program position k): the m instructions
// after it act on the T bits listed at mats + H.mat (bits 0..4 first); each
// tile of 2^T amplitudes (fixed values of the other n - T bits) is gathered
// into shared memory, the instructions run there on local bit positions,
// and the tile is written back. Noise of a step inside the pass splits it:
// the instructions before run tiled, the Pauli string is applied to the
// whole register, and the pass resumes. `orig0` = untiled index of the first
// instruction of the pass.
__device__ void tr_tile_pass(const TWork& W, uint32_t k, uint32_t orig0, int n, uint32_t alive,
                             float2* psi, float2* tile, uint32_t* offh, TEvent* events,
                             int max_events, uint32_t* sh) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const TInstr H = W.prog[k];
    const int T = H.b0;
    const uint32_t m = H.cmask;
    const uint32_t* tb = reinterpret_cast<const uint32_t*>(W.mats + H.mat);
    const uint32_t NT = 1u << T, NH = NT >> 5;
    // global offset of local index (lh << 5 | ll) = offh[lh] + ll
    for (uint32_t lh = tid; lh < NH; lh += nt) {
        uint32_t o = 0;
        for (int j = 5; j < T; ++j) o |= ((lh >> (j - 5)) & 1u) << tb[j];
        offh[lh] = o;
    }
    uint32_t tilebits = 0;
    for (int j = 0; j < T; ++j) tilebits |= 1u << tb[j];
    const uint32_t rest = (n == 32 ? 0xffffffffu : ((1u << n) - 1)) & ~tilebits;
    const uint32_t ntiles = 1u << (n - T);
    __syncthreads();
    uint32_t start = k + 1;
    const uint32_t end = k + 1 + m;
    bool start_done = false; // noise before `start` already applied
    while (start < end) {
        uint32_t stop = end;
        if (W.p_noise > 0.f)
            for (uint32_t i = start; i < end; ++i) {
                if (!(W.prog[i].flags & kTNewStep) || (i == start && start_done)) continue;
                if (tr_noise(W, orig0 + (i - k - 1), n, alive, false, psi, 0, events, max_events, sh)) {
                    stop = i;
                    break;
                }
            }
        if (stop > start) {
            for (uint32_t t = 0; t < ntiles; ++t) {
                // deposit t into the bits outside the tile
                uint32_t base = 0, r = rest, tt = t;
                while (r) {
                    const uint32_t low = r & (0u - r);
                    if (tt & 1u) base |= low;
                    tt >>= 1;
                    r ^= low;
                }
                for (uint32_t l0 = 0; l0 < NT; l0 += 4u * nt) {
                    float2 v[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const uint32_t l = l0 + u * nt + tid;
                        v[u] = l < NT ? psi[base + offh[l >> 5] + (l & 31u)] : make_float2(0.f, 0.f);
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const uint32_t l = l0 + u * nt + tid;
                        if (l < NT) tile[l] = v[u];
                    }
                }
                __syncthreads();
                for (uint32_t i = start; i < stop; ++i) {
                    tr_gate(W.prog[i], W.mats, tile, NT, tid, nt);
                    __syncthreads();
                }
                for (uint32_t l = tid; l < NT; l += nt) psi[base + offh[l >> 5] + (l & 31u)] = tile[l];
                __syncthreads();
            }
        }
        if (stop < end) {
            tr_noise(W, orig0 + (stop - k - 1), n, alive, true, psi, 1u << n, events, max_events, sh);
            start = stop;
            start_done = true;
        } else {
            start = end;
        }
    }
}

__global__ void __launch_bounds__(256, 4)
    k_traj(const TWork* __restrict__ work, int nwork, uint32_t* __restrict__ dits,
           int maxcreg, uint64_t* __restrict__ samples, float2* __restrict__ dump,
           TEvent* __restrict__ events, int max_events, float2* __restrict__ gscratch,
           uint64_t gslot, int tile_bits) {
    extern __shared__ __align__(16) unsigned char sm[];
    // registers of up to 2^14 amplitudes live in shared memory; larger ones
    // in this CTA's own slot of a global scratch buffer or in place in their
    // own state (L2 / HBM), which __syncthreads makes coherent between the
    // block's threads; their tile passes use the shared memory as the tile
    float2* const base = gscratch ? gscratch + uint64_t(blockIdx.x) * gslot
                                  : reinterpret_cast<float2*>(sm);
    float2* const tile = reinterpret_cast<float2*>(sm);
    uint32_t* const offh = reinterpret_cast<uint32_t*>(sm + (size_t(1) << tile_bits) * sizeof(float2));
    __shared__ double red[8];
    __shared__ double part[256];
    __shared__ uint32_t nsh[4]; // noise: xm, zm, ny, events so far
    __shared__ int outcome_sh;
    const int tid = threadIdx.x, nt = blockDim.x;

    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const TWork W = work[w];
        const int n = W.n;
        const uint32_t N = 1u << n;
        // in place: the CTA works directly on the instance's own state;
        // an item without a buffer that can hold it is skipped (uniform
        // across the CTA, before any barrier of this iteration)
        if (W.inplace ? W.fin == nullptr : (!gscratch && n > kTrajMaxQubits)) continue;
        float2* const psi = W.inplace ? W.fin : base;
        if (W.inplace) {
        } else if (W.init)
            for (uint32_t i = tid; i < N; i += nt) psi[i] = W.init[i];
        else
            for (uint32_t i = tid; i < N; i += nt) psi[i] = make_float2(i == 0 ? 1.f : 0.f, 0.f);
        uint32_t alive = (n == 32) ? 0xffffffffu : ((1u << n) - 1);
        if (tid == 0) nsh[3] = 0;
        __syncthreads();
        uint32_t nhdr = 0; // tile headers so far: untiled index = k - nhdr
        for (uint32_t k = 0; k < W.nins; ++k) {
            const TInstr I = W.prog[k];
            if (I.op == kTTile) {
                // headers appear only in programs of registers above 2^14
                // amplitudes, launched with a tile buffer of 2^tile_bits
                if (int(I.b0) <= tile_bits && n > kTrajMaxQubits)
                    tr_tile_pass(W, k, k - nhdr, n, alive, psi, tile, offh, events, max_events, nsh);
                ++nhdr;
                k += I.cmask;
                __syncthreads();
                continue;
            }
            const uint32_t orig = k - nhdr;
            if ((I.flags & kTNewStep) && W.p_noise > 0.f)
                tr_noise(W, orig, n, alive, true, psi, N, events, max_events, nsh);
            switch (I.op) {
                case kTG1:
                case kTCG1:
                case kTG2:
                case kTG3:
                case kTG4:
                    tr_gate(I, W.mats, psi, N, tid, nt);
                    break;
                case kTMeas: {
                    const uint32_t bit = 1u << I.b0;
                    double p1 = 0, tot = 0;
                    for (uint32_t i = tid; i < N; i += nt) {
                        double w2 = double(psi[i].x) * psi[i].x + double(psi[i].y) * psi[i].y;
                        tot += w2;
                        if (i & bit) p1 += w2;
                    }
                    tot = block_sum_d(tot, red);
                    p1 = block_sum_d(p1, red);
                    if (tid == 0) {
                        double u0, u1;
                        philox_uniform2(W.seed, W.shot, orig, 0xffffu, 0x6d656173u, u0, u1);
                        // first outcome whose cumulative probability reaches u
                        outcome_sh = (u0 * tot <= tot - p1 && tot - p1 > 0) ? 0 : 1;
                        if (I.mat < uint32_t(maxcreg))
                            dits[size_t(W.out) * maxcreg + I.mat] = uint32_t(outcome_sh);
                    }
                    __syncthreads();
                    const int o = outcome_sh;
                    const double pk = o ? p1 : tot - p1;
                    const float sc = float(1.0 / sqrt(pk));
                    for (uint32_t i = tid; i < N; i += nt) {
                        bool keep = (((i & bit) != 0) == (o == 1));
                        float2 a = psi[i];
                        psi[i] = keep ? make_float2(a.x * sc, a.y * sc) : make_float2(0.f, 0.f);
                    }
                    if (I.flags & kTDestructive) alive &= ~bit;
                    break;
                }
                default:
                    break;
            }
            __syncthreads();
        }
        if (W.diag) {
            // density matrix over n/2 qubits: its diagonal, for the shots
            const uint32_t Dh = 1u << (n / 2);
            for (uint32_t i = tid; i < Dh; i += nt) W.diag[i] = double(psi[i * (Dh + 1)].x);
        }
        // final full-basis sample: FP64 prefix sums over thread chunks
        if (!W.diag) {
            const uint32_t chunk = (N + nt - 1) / nt;
            double s = 0;
            const uint32_t lo = tid * chunk, hi = min(N, lo + chunk);
            for (uint32_t i = lo; i < hi; ++i)
                s += double(psi[i].x) * psi[i].x + double(psi[i].y) * psi[i].y;
            part[tid] = s;
            __syncthreads();
            if (tid == 0) {
                double tot = 0;
                for (int t = 0; t < nt; ++t) tot += part[t];
                double u0, u1;
                philox_uniform2(W.seed, W.shot, 0xffffffffu, 0u, 0x66696e6cu, u0, u1);
                double thr = u0 * tot, cum = 0;
                uint64_t idx = N - 1;
                int t = 0;
                for (; t < nt; ++t) {
                    if (cum + part[t] >= thr && part[t] > 0) break;
                    cum += part[t];
                }
                if (t < nt) {
                    for (uint32_t i = t * chunk; i < min(N, (t + 1) * chunk); ++i) {
                        cum += double(psi[i].x) * psi[i].x + double(psi[i].y) * psi[i].y;
                        if (cum >= thr) {
                            idx = i;
                            break;
                        }
                    }
                }
                samples[W.out] = idx;
            }
            __syncthreads();
        }
        if (dump)
            for (uint32_t i = tid; i < N; i += nt) dump[size_t(W.out) * N + i] = psi[i];
        if (W.fin && !W.inplace)
            for (uint32_t i = tid; i < N; i += nt) W.fin[i] = psi[i];
        __syncthreads();
    }
}

// One tile pass of many registers at once (layer-synchronous batches): the
// launch covers pass k of every register that has one. A CTA takes a
// contiguous range of items; an item is tiles_per_item consecutive tiles of
// one register. Tiles move by bulk copies (the copy engine, untiled
// cp.async.bulk; rows = runs of >= 32 consecutive amplitudes, 16-byte
// aligned): warp 0 loads tile i + 1 into the second buffer (completion
// counted on an mbarrier) while all warps apply tile i's gates in shared
// memory, and writes tile i back with bulk stores. Every mbarrier wait is
// bounded; a timeout sets *err, waits once more (bounded) for the copies in
// flight and ends the CTA. Registers are independent, and the kernel
// boundary orders pass k before pass k + 1.
constexpr uint32_t kPassSpinLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool pass_mbar_wait(uint32_t mbar, uint32_t parity) {
    for (uint32_t it = 0; it < kPassSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

struct PassCursor {
    int j;          // register (PassInst) index
    uint32_t it;    // item
    uint32_t t, t1; // tile and end of the item's tiles
};

__device__ __forceinline__ void cursor_item(const PassInst* insts, PassCursor& c) {
    const PassInst& P = insts[c.j];
    c.t = (c.it - P.first_item) * P.tiles_per_item;
    c.t1 = min(c.t + P.tiles_per_item, 1u << (P.n - P.T));
}

// false when the CTA's range is exhausted
__device__ __forceinline__ bool cursor_next(const PassInst* insts, int ninst, uint32_t it1,
                                            PassCursor& c) {
    if (++c.t < c.t1) return true;
    if (++c.it >= it1) return false;
    while (c.j + 1 < ninst && insts[c.j + 1].first_item <= c.it) ++c.j;
    cursor_item(insts, c);
    return true;
}

// Geometry of one register's tile pass, cached in shared memory by the CTA
// while it works on that register: row offsets (rows = runs of 2^crow
// consecutive amplitudes) and the bits outside the tile.
struct PassGeom {
    uint32_t nrows, rowbytes, rest;
    int j; // register the table belongs to (-1: none)
};

// every thread fills rows; thread 0 writes the header (call between
// barriers)
__device__ void pass_geom(const PassInst& P, int j, PassGeom* g, uint32_t* rowoff) {
    const uint32_t* tb = reinterpret_cast<const uint32_t*>(P.mats + P.tb_off);
    const int T = P.T, n = P.n;
    int crow = 0;
    while (crow < T && tb[crow] == uint32_t(crow)) ++crow;
    const uint32_t nrows = 1u << (T - crow);
    if (threadIdx.x == 0) {
        uint32_t tilebits = 0;
        for (int q = 0; q < T; ++q) tilebits |= 1u << tb[q];
        g->rest = (n == 32 ? 0xffffffffu : ((1u << n) - 1)) & ~tilebits;
        g->nrows = nrows;
        g->rowbytes = (1u << crow) * uint32_t(sizeof(float2));
        g->j = j;
    }
    for (uint32_t row = threadIdx.x; row < nrows; row += blockDim.x) {
        uint32_t off = 0;
        for (int q = crow; q < T; ++q) off |= ((row >> (q - crow)) & 1u) << tb[q];
        rowoff[row] = off;
    }
}

__device__ __forceinline__ uint32_t tile_base(uint32_t rest, uint32_t t) {
    uint32_t base = 0;
    while (rest) {
        const uint32_t low = rest & (0u - rest);
        if (t & 1u) base |= low;
        t >>= 1;
        rest ^= low;
    }
    return base;
}

// warp 0: bulk-load tile t into buf, completion on mbar
__device__ __forceinline__ void pass_issue_load(const PassInst& P, const PassGeom& g,
                                                const uint32_t* rowoff, uint32_t t, float2* buf,
                                                uint32_t mbar, int lane) {
    const float2* src = P.psi + tile_base(g.rest, t);
    if (lane == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar),
                     "r"(g.nrows * g.rowbytes)
                     : "memory");
    __syncwarp();
    const uint32_t rowlen = g.rowbytes / uint32_t(sizeof(float2));
    for (uint32_t row = lane; row < g.nrows; row += 32)
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
                "r"(smem_addr(buf + row * rowlen)),
            "l"(src + rowoff[row]), "r"(g.rowbytes), "r"(mbar)
            : "memory");
}

// warp 0: bulk-store tile t from buf back into its register
__device__ __forceinline__ void pass_issue_store(const PassInst& P, const PassGeom& g,
                                                 const uint32_t* rowoff, uint32_t t,
                                                 const float2* buf, int lane) {
    float2* dst = P.psi + tile_base(g.rest, t);
    const uint32_t rowlen = g.rowbytes / uint32_t(sizeof(float2));
    for (uint32_t row = lane; row < g.nrows; row += 32)
        asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(
                         dst + rowoff[row]),
                     "r"(smem_addr(buf + row * rowlen)), "r"(g.rowbytes)
                     : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

__global__ void __launch_bounds__(256, 3)
    k_pass_batch(const PassInst* __restrict__ insts, int ninst, uint32_t nitems, int tile_bits,
                 int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char sm[];
    float2* const buf0 = reinterpret_cast<float2*>(sm);
    float2* const buf1 = reinterpret_cast<float2*>(sm + (size_t(1) << tile_bits) * sizeof(float2));
    // row tables of the registers of the current and the next tile (at
    // most 2^(tile_bits - 5) rows each)
    uint32_t* const rows0 = reinterpret_cast<uint32_t*>(sm + (size_t(2) << tile_bits) * sizeof(float2));
    uint32_t* const rows1 = rows0 + (size_t(1) << (tile_bits - 5));
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ int abort_sh;
    __shared__ PassGeom geom[2];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t per = (nitems + gridDim.x - 1) / gridDim.x;
    const uint32_t it0 = blockIdx.x * per, it1 = min(nitems, it0 + per);
    if (it0 >= it1) return; // uniform across the CTA
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_sh = 0;
        geom[0].j = geom[1].j = -1;
    }
    PassCursor cur;
    {
        int lo = 0, hi = ninst - 1; // last register with first_item <= it0
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (insts[mid].first_item <= it0) lo = mid;
            else hi = mid - 1;
        }
        cur.j = lo;
        cur.it = it0;
        cursor_item(insts, cur);
    }
    __syncthreads();
    // geometry slot x belongs to buffer x
    pass_geom(insts[cur.j], cur.j, &geom[0], rows0);
    __syncthreads();
    uint32_t parity[2] = {0u, 0u};
    bool pending[2] = {true, false}; // a load in flight into buffer x
    int b = 0;
    if (warp == 0)
        pass_issue_load(insts[cur.j], geom[0], rows0, cur.t, buf0, smem_addr(&mbar[0]), lane);
    bool more = true;
    while (more) {
        float2* const bc = b ? buf1 : buf0;
        float2* const bn = b ? buf0 : buf1;
        uint32_t* const rc = b ? rows1 : rows0;
        uint32_t* const rn = b ? rows0 : rows1;
        PassCursor nxt = cur;
        more = cursor_next(insts, ninst, it1, nxt);
        if (more) {
            // rebuilt only when the register changes; nothing writes the
            // slot before the first barrier, so every thread takes the
            // same branch
            if (geom[b ^ 1].j != nxt.j) {
                __syncthreads();
                pass_geom(insts[nxt.j], nxt.j, &geom[b ^ 1], rn);
                __syncthreads();
            }
            if (warp == 0) {
                // the other buffer's last bulk store must have read it
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                __syncwarp();
                pass_issue_load(insts[nxt.j], geom[b ^ 1], rn, nxt.t, bn, smem_addr(&mbar[b ^ 1]),
                                lane);
            }
            pending[b ^ 1] = true;
        }
        if (pass_mbar_wait(smem_addr(&mbar[b]), parity[b])) {
            parity[b] ^= 1u;
            pending[b] = false;
        } else {
            atomicExch(err, 1);
            abort_sh = 1;
        }
        __syncthreads();
        if (abort_sh) break;
        const PassInst& P = insts[cur.j];
        const uint32_t NT = 1u << P.T;
        for (uint32_t i = 0; i < P.nins; ++i) {
            tr_gate(P.ins[i], P.mats, bc, NT, tid, nt);
            __syncthreads();
        }
        // the threads' shared-memory writes, visible to the bulk stores
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (warp == 0) pass_issue_store(P, geom[b], rc, cur.t, bc, lane);
        cur = nxt;
        b ^= 1;
    }
    // after a timeout: wait once more (bounded) for the loads in flight
    for (int x = 0; x < 2; ++x)
        if (pending[x]) pass_mbar_wait(smem_addr(&mbar[x]), parity[x]);
    if (warp == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

void launch_pass_batch(qgpu_ctx* ctx, const PassInst* dinsts, int ninst, uint32_t nitems,
                       int tile_bits, int* err, cudaStream_t stream) {
    if (ninst == 0 || nitems == 0) return;
    if (tile_bits < 9 || tile_bits > 13)
        raise(QGPU_ERR_INVALID_ARGUMENT, "launch_pass_batch()", "tile_bits");
    ensure_smem(reinterpret_cast<const void*>(k_pass_batch),
                (size_t(2) << 13) * sizeof(float2) + (size_t(2) << 8) * sizeof(uint32_t));
    // two tile buffers and two row tables
    const size_t smem = (size_t(2) << tile_bits) * sizeof(float2) +
                        (size_t(2) << (tile_bits - 5)) * sizeof(uint32_t);
    int per_sm = 0;
    QG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pass_batch, 256, smem));
    per_sm = std::max(1, per_sm);
    const uint32_t grid = std::min<uint32_t>(nitems, uint32_t(ctx->num_sms) * uint32_t(per_sm));
    k_pass_batch<<<grid, 256, smem, stream ? stream : ctx->stream>>>(dinsts, ninst, nitems,
                                                                      tile_bits, err);
    after_launch(ctx, "k_pass_batch");
}

// Block-layered launches (no reference counterpart): each thread takes two
// groups of 2^K amplitudes of one block (g0 and g0 + 256) at once (both loaded before any
// arithmetic, so twice the loads are in flight), keeps all inputs in
// registers before the in-place writes, and computes rows in pairs, so that
// each matrix load is one float4 (entries (row, c) and (row + 1, c) are
// adjacent in column-major order) feeding both groups. No barriers: a group
// belongs to one thread, and a launch holds at most one block per register.
template <int K>
__device__ __forceinline__ void block_groups(const BlockInst& B, uint32_t g0, bool two) {
    constexpr int D = 1 << K;
    int sb[K];
#pragma unroll
    for (int j = 0; j < K; ++j) sb[j] = B.b[j];
#pragma unroll
    for (int x = 0; x < K - 1; ++x)
#pragma unroll
        for (int y = 0; y < K - 1 - x; ++y)
            if (sb[y] > sb[y + 1]) {
                const int t = sb[y];
                sb[y] = sb[y + 1];
                sb[y + 1] = t;
            }
    uint32_t i0 = g0, i1 = g0 + 256;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        i0 = ins0(i0, sb[j]);
        i1 = ins0(i1, sb[j]);
    }
    uint32_t o[K];
#pragma unroll
    for (int j = 0; j < K; ++j) o[j] = 1u << B.b[j];
    auto off = [&](int r) {
        uint32_t x = 0;
#pragma unroll
        for (int j = 0; j < K; ++j) x += ((r >> (K - 1 - j)) & 1) ? o[j] : 0u;
        return x;
    };
    float2* psi = B.psi;
    if (!two) i1 = i0; // the second group repeats the first; only one is written
    float2 v[D], w[D];
#pragma unroll
    for (int c = 0; c < D; ++c) {
        v[c] = psi[i0 + off(c)];
        w[c] = psi[i1 + off(c)];
    }
    const float4* m4 = reinterpret_cast<const float4*>(B.m);
#pragma unroll(K == 4 ? 1 : D / 2)
    for (int row = 0; row < D; row += 2) {
        float2 a0 = make_float2(0.f, 0.f), a1 = a0, b0 = a0, b1 = a0;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const float4 e = m4[(row + D * c) >> 1];
            const float2 e0 = make_float2(e.x, e.y), e1 = make_float2(e.z, e.w);
            a0 = c_fma(e0, v[c], a0);
            a1 = c_fma(e1, v[c], a1);
            b0 = c_fma(e0, w[c], b0);
            b1 = c_fma(e1, w[c], b1);
        }
        psi[i0 + off(row)] = a0;
        psi[i0 + off(row + 1)] = a1;
        if (two) {
            psi[i1 + off(row)] = b0;
            psi[i1 + off(row + 1)] = b1;
        }
    }
}

// Items of 512 groups (thread t takes groups t and t + 256 of the item); the
// blocks' first items sit in shared memory (up to kBlockSmemInsts of them),
// so that finding an item's block is a short search there rather than a
// chain of dependent global loads.
constexpr int kBlockSmemInsts = 4096;

__global__ void __launch_bounds__(256, 2)
    k_block_batch(const BlockInst* __restrict__ insts, int ninst, uint32_t nitems) {
    __shared__ uint32_t first[kBlockSmemInsts];
    const bool in_smem = ninst <= kBlockSmemInsts;
    if (in_smem)
        for (int j = threadIdx.x; j < ninst; j += blockDim.x) first[j] = insts[j].first_item;
    __syncthreads();
    for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        int lo = 0, hi = ninst - 1; // last block with first_item <= it
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if ((in_smem ? first[mid] : insts[mid].first_item) <= it) lo = mid;
            else hi = mid - 1;
        }
        const BlockInst B = insts[lo];
        const uint32_t ngroups = 1u << (B.n - B.k);
        const uint32_t g = (it - B.first_item) * 512u + threadIdx.x;
        if (g >= ngroups) continue;
        const bool two = g + 256 < ngroups;
        switch (B.k) {
            case 1: block_groups<1>(B, g, two); break;
            case 2: block_groups<2>(B, g, two); break;
            case 3: block_groups<3>(B, g, two); break;
            default: block_groups<4>(B, g, two); break;
        }
    }
}

void launch_block_batch(qgpu_ctx* ctx, const BlockInst* dinsts, int ninst, uint32_t nitems,
                        cudaStream_t stream) {
    if (ninst <= 0 || nitems == 0) return;
    static int per_sm = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        QG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_block_batch, 256, 0));
        per_sm = std::max(1, per_sm);
    });
    const uint32_t grid = std::min<uint32_t>(nitems, uint32_t(ctx->num_sms) * uint32_t(per_sm));
    k_block_batch<<<grid, 256, 0, stream ? stream : ctx->stream>>>(dinsts, ninst, nitems);
    after_launch(ctx, "k_block_batch");
}

void traj_prepare() {
    // a 2^14-amplitude register, or a tile of up to 2^14 amplitudes with its
    // offset table
    ensure_smem(reinterpret_cast<const void*>(k_traj),
                (size_t(1) << kTrajMaxQubits) * sizeof(float2) + 4096);
}

int traj_global_grid(qgpu_ctx* ctx, int nwork, int n) {
    const uint64_t slot = (uint64_t(1) << n) * sizeof(float2);
    const uint64_t by_mem = std::max<uint64_t>(1, (uint64_t(4) << 30) / slot);
    return int(std::min<uint64_t>(std::min<uint64_t>(nwork, uint64_t(ctx->num_sms) * 8), by_mem));
}

// resident CTAs per SM for a dynamic shared-memory size (cached)
static int traj_per_sm(size_t smem) {
    static std::mutex mu;
    static std::map<size_t, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(smem);
    if (it != cache.end()) return it->second;
    int b = 0;
    QG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_traj, 256, smem));
    b = std::max(1, std::min(b, 8));
    cache[smem] = b;
    return b;
}

int traj_resident_slots(qgpu_ctx* ctx, int n) {
    traj_prepare();
    return ctx->num_sms * traj_per_sm((size_t(1) << n) * sizeof(float2));
}

void launch_traj(qgpu_ctx* ctx, const TWork* dwork, int nwork, int nmax, uint32_t* ddits,
                 int maxcreg, uint64_t* dsamples, float2* ddump, TEvent* devents,
                 int max_events, float2* gscratch, cudaStream_t stream, int tile_bits) {
    if (nwork == 0) return;
    cudaStream_t st = stream ? stream : ctx->stream;
    traj_prepare();
    if (nmax > kTrajMaxQubits) {
        if (tile_bits && (tile_bits < 9 || tile_bits > kTrajMaxQubits))
            raise(QGPU_ERR_INVALID_ARGUMENT, "launch_traj()", "tile_bits");
        const size_t smem = tile_bits ? (size_t(1) << tile_bits) * sizeof(float2) +
                                            (size_t(1) << (tile_bits - 5)) * sizeof(uint32_t)
                                      : 0;
        const int cap = ctx->num_sms * traj_per_sm(smem);
        // no scratch: the caller promises in-place work items (own states)
        int grid = gscratch ? std::min(traj_global_grid(ctx, nwork, nmax), cap)
                            : std::min(nwork, cap);
        k_traj<<<grid, 256, smem, st>>>(dwork, nwork, ddits, maxcreg, dsamples, ddump, devents,
                                        max_events, gscratch, uint64_t(1) << nmax, tile_bits);
        after_launch(ctx, "k_traj (global)");
        return;
    }
    size_t smem = (size_t(1) << nmax) * sizeof(float2);
    int grid = std::min(nwork, ctx->num_sms * traj_per_sm(smem));
    k_traj<<<grid, 256, smem, st>>>(dwork, nwork, ddits, maxcreg, dsamples, ddump, devents,
                                    max_events, nullptr, 0, 0);
    after_launch(ctx, "k_traj");
}

} // namespace qgpu
