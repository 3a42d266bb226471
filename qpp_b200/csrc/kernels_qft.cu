// kernels_qft.cu -- qudit quantum Fourier transform passes (sm_100a).
//
// qpp::applyQFT (operations.hpp:2565-2676) runs, for i = 0..k-1, the Fourier
// gate F (H for qubits, Fd(d) otherwise) on target[i] followed by the
// controlled phases R_j = diag(exp(2 pi i m / d^j)) with control
// target[i+j-1] (j = 2..k-i) on target[i], and then reverses the order of
// the targets with SWAPs; applyTFQ (:2680-2787) runs the adjoint steps in the
// reverse order. The phases of step i commute with each other: together they
// are the diagonal exp(s 2 pi i m_i Y_i / d^(k-i)), where m_i is target digit
// i, Y_i the integer spelled by digits i+1..k-1 (most significant first) and
// s = +1 (QFT) or -1 (TFQ). So step i is "F on digit i, then that diagonal".
//
// A pass applies the steps of M consecutive targets [a, a + M) to tiles that
// hold every value of those M digits, plus the lowest other digits in memory
// order so that reads and writes run over >= 128 contiguous bytes, staged in
// shared memory. The part of each step's phase that depends on digits
// outside the group is one constant per tile, step and value of the later
// targets inside the tile (at most 4 of them). A pass reads and
// writes every amplitude once, so a k-digit transform costs ceil(k / M)
// passes over the state instead of the k(k+1)/2 gate passes of the gate
// sequence. The pass that also reverses the targets reads one buffer and
// writes another with permuted digit strides.
//
// Qubit butterflies omit the 1/sqrt(2) of H; the store multiplies by
// 2^(-M/2) once.
#include <cstdio>

#include "kernels.hpp"

namespace qgpu {

namespace {

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
    return {a.x + b.x, a.y + b.y};
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
    return {a.x - b.x, a.y - b.y};
}

// Tile offsets of index e (tile digits in read order) or of store index f
// (tile digits in write order): sum over the digits of digit * stride.
__device__ inline uint64_t tile_sum(const QftPlan& p, uint32_t idx, bool write_order,
                                    int what) {
    uint64_t acc = 0;
    for (int q = 0; q < p.ntd; ++q) {
        const int td = write_order ? p.wperm[q] : q;
        const uint32_t pitch = write_order ? p.fpitch[q] : p.tpitch[q];
        const uint32_t dg = (idx / pitch) % p.tdim[td];
        const uint64_t w = what == 0 ? p.trs[td] : what == 1 ? p.tws[td] : p.tpitch[td];
        acc += uint64_t(dg) * w;
    }
    return acc;
}

} // namespace

// One CTA per tile (grid-stride over tiles). Dynamic shared memory: the tile
// (E amplitudes), the per-tile step constants (M * d * d^nzr), and the read /
// write offset tables split into a low and a high half.
template <typename R, bool QB>
__global__ void __launch_bounds__(256, 4)
    k_qft_pass(const Cplx<R>* in, Cplx<R>* out, const __grid_constant__ QftPlan p,
               const Cplx<R>* __restrict__ W, const Cplx<R>* __restrict__ F) {
    using C = Cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tile = reinterpret_cast<C*>(smem_raw);
    C* cst = tile + p.E;
    uint64_t* rlo = reinterpret_cast<uint64_t*>(cst + p.M * p.d * p.CZ);
    uint64_t* rhi = rlo + p.Elo;
    uint64_t* wlo = rhi + p.E / p.Elo;
    uint64_t* whi = wlo + p.Flo;
    uint32_t* elo = reinterpret_cast<uint32_t*>(whi + p.E / p.Flo);
    uint32_t* ehi = elo + p.Flo;

    const int tid = threadIdx.x, nt = blockDim.x;
    for (uint32_t i = tid; i < p.Elo; i += nt) rlo[i] = tile_sum(p, i, false, 0);
    for (uint32_t i = tid; i < p.E / p.Elo; i += nt) rhi[i] = tile_sum(p, i * p.Elo, false, 0);
    for (uint32_t i = tid; i < p.Flo; i += nt) {
        wlo[i] = tile_sum(p, i, true, 1);
        elo[i] = uint32_t(tile_sum(p, i, true, 2));
    }
    for (uint32_t i = tid; i < p.E / p.Flo; i += nt) {
        whi[i] = tile_sum(p, i * p.Flo, true, 1);
        ehi[i] = uint32_t(tile_sum(p, i * p.Flo, true, 2));
    }
    __syncthreads();

    const int M = p.M, d = p.d;
    const R sg = R(p.sigma);
    for (uint64_t t = blockIdx.x; t < p.ntiles; t += gridDim.x) {
        // base offsets and Z (the value of the later targets outside the tile)
        uint64_t rb = 0, wb = 0, z = 0;
        for (int q = 0; q < p.nod; ++q) {
            const uint64_t dg = p.pow2 ? (t >> p.oshift[q]) & (p.odim[q] - 1)
                                       : (t / p.opitch[q]) % p.odim[q];
            rb += dg * p.ors[q];
            wb += dg * p.ows[q];
            z += dg * p.ozw[q];
        }
        // step constants exp(s 2 pi i r (Z + Zr(c)) / d^(k-i)), i = a + j, for
        // every value c of the phase digits; r (Z + Zr) < d^(k-i)
        for (int i = tid; i < M * d * int(p.CZ); i += nt) {
            const int c = i % int(p.CZ), jr = i / int(p.CZ);
            const int j = jr / d, r = jr % d;
            uint64_t zz = z;
            for (int q = 0, cc = c; q < p.nzr; ++q, cc /= d) zz += uint64_t(cc % d) * p.zrw[q];
            const uint64_t N = p.dpow[p.k - p.a - j];
            double sn, cs;
            sincospi(2.0 * (double(uint64_t(r) * zz) / double(N)), &sn, &cs);
            cst[i] = C{R(cs), R(p.sigma * sn)};
        }
        for (uint32_t e = tid; e < p.E; e += nt) {
            const uint32_t lo = QB ? (e & (p.Elo - 1)) : e % p.Elo;
            const uint32_t hi = QB ? (e >> p.elo_shift) : e / p.Elo;
            tile[e] = in[rb + rlo[lo] + rhi[hi]];
        }
        __syncthreads();

        for (int s = 0; s < M; ++s) {
            const int j = p.inverse ? M - 1 - s : s;
            if constexpr (QB) {
                const int g = p.gpos[j]; // tile bit of digit j
                const uint32_t lm = (1u << g) - 1;
                const C* cj = cst + (j * 2 + 1) * p.CZ;
                for (uint32_t pr = tid; pr < p.E / 2; pr += nt) {
                    const uint32_t e0 = ((pr & ~lm) << 1) | (pr & lm);
                    const uint32_t e1 = e0 | (1u << g);
                    uint32_t L = 0, c = 0;
                    for (int l = j + 1; l < M; ++l) L = (L << 1) | ((e0 >> p.gpos[l]) & 1u);
                    for (int q = 0; q < p.nzr; ++q) c |= ((e0 >> p.zpos[q]) & 1u) << q;
                    C w = W[(L << j) * p.wmul];
                    w.y *= sg;
                    const C ph = cmul(w, cj[c]);
                    const C x = tile[e0];
                    C y = tile[e1];
                    if (!p.inverse) {
                        tile[e0] = cadd(x, y);
                        tile[e1] = cmul(csub(x, y), ph);
                    } else {
                        y = cmul(y, ph);
                        tile[e0] = cadd(x, y);
                        tile[e1] = csub(x, y);
                    }
                }
            } else {
                const uint32_t pj = p.tpitch[p.gpos[j]];
                const uint64_t dj = p.dpow[j];
                for (uint32_t fb = tid; fb < p.E / d; fb += nt) {
                    const uint32_t hi = fb / pj, lo = fb - hi * pj;
                    const uint32_t e0 = hi * pj * d + lo;
                    uint64_t L = 0;
                    uint32_t c = 0;
                    for (int l = j + 1; l < M; ++l)
                        L = L * d + (e0 / p.tpitch[p.gpos[l]]) % d;
                    for (int q = p.nzr; q-- > 0;) c = c * d + (e0 / p.tpitch[p.zpos[q]]) % d;
                    C v[kQftMaxD], o[kQftMaxD];
                    for (int r = 0; r < d; ++r) v[r] = tile[e0 + r * pj];
                    auto phase = [&](int r) {
                        C w = W[(uint64_t(r) * L * dj) * p.wmul]; // r L d^j < d^M
                        w.y *= sg;
                        return cmul(w, cst[(j * d + r) * p.CZ + c]);
                    };
                    if (p.inverse)
                        for (int r = 1; r < d; ++r) v[r] = cmul(v[r], phase(r));
                    for (int x = 0; x < d; ++x) {
                        C acc{R(0), R(0)};
                        for (int y = 0; y < d; ++y) acc = cfma(F[x + y * d], v[y], acc);
                        o[x] = acc;
                    }
                    if (!p.inverse)
                        for (int r = 1; r < d; ++r) o[r] = cmul(o[r], phase(r));
                    for (int r = 0; r < d; ++r) tile[e0 + r * pj] = o[r];
                }
            }
            __syncthreads();
        }

        const R sc = R(p.scale);
        for (uint32_t f = tid; f < p.E; f += nt) {
            const uint32_t lo = QB ? (f & (p.Flo - 1)) : f % p.Flo;
            const uint32_t hi = QB ? (f >> p.flo_shift) : f / p.Flo;
            C v = tile[elo[lo] + ehi[hi]];
            if (QB) {
                v.x *= sc;
                v.y *= sc;
            }
            out[wb + wlo[lo] + whi[hi]] = v;
        }
        __syncthreads();
    }
}

size_t qft_smem_bytes(const QftPlan& p, size_t elem_bytes) {
    return p.E * elem_bytes + size_t(p.M) * p.d * p.CZ * elem_bytes +
           (p.Elo + p.E / p.Elo + p.Flo + p.E / p.Flo) * sizeof(uint64_t) +
           (p.Flo + p.E / p.Flo) * sizeof(uint32_t);
}

template <typename R>
static void qft_launch(qgpu_ctx* ctx, const void* in, void* out, const QftPlan& p,
                       const void* W, const void* F) {
    using C = Cplx<R>;
    const size_t sm = qft_smem_bytes(p, sizeof(C));
    uint64_t blocks = uint64_t(grid_blocks(ctx, 4));
    if (p.ntiles < blocks) blocks = p.ntiles;
    if (p.d == 2) {
        if (sm > 48 * 1024)
            QG_CUDA(cudaFuncSetAttribute(k_qft_pass<R, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        k_qft_pass<R, true><<<unsigned(blocks), 256, sm, ctx->stream>>>(
            static_cast<const C*>(in), static_cast<C*>(out), p, static_cast<const C*>(W),
            static_cast<const C*>(F));
    } else {
        if (sm > 48 * 1024)
            QG_CUDA(cudaFuncSetAttribute(k_qft_pass<R, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        k_qft_pass<R, false><<<unsigned(blocks), 256, sm, ctx->stream>>>(
            static_cast<const C*>(in), static_cast<C*>(out), p, static_cast<const C*>(W),
            static_cast<const C*>(F));
    }
    after_launch(ctx, "k_qft_pass");
}

void launch_qft_pass(qgpu_ctx* ctx, qgpu_prec prec, const void* in, void* out,
                     const QftPlan& p, const void* W, const void* F) {
    if (p.ntiles == 0) return;
    if (prec == QGPU_C128) qft_launch<double>(ctx, in, out, p, W, F);
    else qft_launch<float>(ctx, in, out, p, W, F);
}

} // namespace qgpu
