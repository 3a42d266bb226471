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
// shared memory. In the tile index the run digits come first and the group
// digits follow with step M - 1 lowest, so the phase of step j splits into
// W[L << j] (L = the group digits after j: a shift and mask of the index),
// a constant per tile and step for the later targets outside the tile, and a
// factor for the later targets among the run digits (the lowest index
// digits). For qubits the last two are a per-block table over the run
// digits' values times one base per tile and step; for qudits they are
// tabulated per tile. A pass reads and writes every amplitude once, so a
// k-digit transform costs ceil(k / M) passes over the state instead of the
// k(k+1)/2 gate passes of the gate sequence. The pass that also reverses the
// targets reads one buffer and writes another with permuted digit strides.
//
// Qubit steps run three at a time in registers (a thread holds the 8
// amplitudes of a base); the next tile is copied in with cp.async while the
// current one is transformed. Qubit butterflies omit the 1/sqrt(2) of H; the
// store multiplies by 2^(-M/2) once.
#include <algorithm>

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

// Memory offset (what = 0 read, 1 write) or tile index (what = 2) of the
// element at position idx of the read (write_order = false) or write order.
__device__ inline uint64_t order_sum(const QftPlan& p, uint32_t idx, bool write_order, int what) {
    uint64_t acc = 0;
    for (int q = 0; q < p.ntd; ++q) {
        const int td = write_order ? p.wperm[q] : p.rperm[q];
        const uint32_t pitch = write_order ? p.wpitch[q] : p.rpitch[q];
        const uint32_t dg = (idx / pitch) % p.tdim[td];
        const uint64_t w = what == 0 ? p.trs[td] : what == 1 ? p.tws[td] : p.tpitch[td];
        acc += uint64_t(dg) * w;
    }
    return acc;
}

// G consecutive qubit steps starting at step jf (forward: jf, jf + 1, ...;
// inverse: jf, jf - 1, ...) on every base of the tile, in registers. Step j
// sits on tile bit nr + M - 1 - j: the round's bits are [lo, lo + G) and step
// u of the round (u = 0 first) is on bit lo + G - 1 - u (forward) or lo + u
// (inverse).
template <typename R, int G, bool INV>
__device__ __forceinline__ void qubit_round(const QftPlan& p, Cplx<R>* tile,
                                            const Cplx<R>* T, const Cplx<R>* B, const Cplx<R>* W,
                                            int jf) {
    using C = Cplx<R>;
    const int M = p.M;
    const uint32_t CZ = p.CZ;
    const int jlow = INV ? jf : jf + G - 1; // the step on the lowest bit
    const int lo = p.nr + M - 1 - jlow;
    const uint32_t lom = (1u << lo) - 1;
    for (uint32_t q = threadIdx.x; q < (p.E >> G); q += blockDim.x) {
        const uint32_t eb = ((q & ~lom) << G) | (q & lom);
        const C* cc = T + (eb & (CZ - 1));
        C v[1 << G];
#pragma unroll
        for (int m = 0; m < (1 << G); ++m) v[m] = tile[eb | (uint32_t(m) << lo)];
#pragma unroll
        for (int u = 0; u < G; ++u) {
            const int j = INV ? jf - u : jf + u;
            const int rel = INV ? u : G - 1 - u;
            const uint32_t Lmask = (1u << (M - 1 - j)) - 1;
            const C cj = cmul(B[j], cc[j * CZ]);
            // the phase depends on the round bits below the step's bit only
            C ph[1 << (G - 1)];
#pragma unroll
            for (int lb = 0; lb < (1 << rel); ++lb) {
                const uint32_t L = ((eb >> p.nr) + (uint32_t(lb) << (lo - p.nr))) & Lmask;
                ph[lb] = cmul(W[(L << j) * p.wmul], cj);
            }
#pragma unroll
            for (int m = 0; m < (1 << G); ++m) {
                if ((m >> rel) & 1) continue;
                const int m1 = m | (1 << rel);
                const C phm = ph[m & ((1 << rel) - 1)];
                if (!INV) {
                    const C x = v[m], y = v[m1];
                    v[m] = cadd(x, y);
                    v[m1] = cmul(csub(x, y), phm);
                } else {
                    const C x = v[m], y = cmul(v[m1], phm);
                    v[m] = cadd(x, y);
                    v[m1] = csub(x, y);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < (1 << G); ++m) tile[eb | (uint32_t(m) << lo)] = v[m];
    }
}

// The same rounds with the pass shape known at compile time (M steps, NR run
// bits, a tile of E = 2^(M + NR) amplitudes, roots W[e * 2^WS]): every bit
// position, mask and trip count folds into the instructions. Used for the
// shapes that full transforms of up to 30+ qubits consist of.
template <typename R, int G, bool INV, int M, int NR, int WS, int JF, int NTHR>
__device__ __forceinline__ void qubit_round_ct(Cplx<R>* tile, const Cplx<R>* T,
                                               const Cplx<R>* B, const Cplx<R>* W,
                                               uint32_t CZ) {
    using C = Cplx<R>;
    constexpr int JLOW = INV ? JF : JF + G - 1; // the step on the lowest bit
    constexpr int LO = NR + M - 1 - JLOW;
    constexpr uint32_t LOM = (1u << LO) - 1;
    constexpr uint32_t NB = (1u << (M + NR)) >> G; // bases per tile
    static_assert(NB % NTHR == 0, "bases per thread");
    C cj[G];
#pragma unroll
    for (int u = 0; u < G; ++u) cj[u] = B[INV ? JF - u : JF + u];
#pragma unroll
    for (uint32_t q0 = 0; q0 < NB; q0 += NTHR) {
        const uint32_t q = q0 + threadIdx.x;
        const uint32_t eb = ((q & ~LOM) << G) | (q & LOM);
        const C* cc = T + (eb & (CZ - 1));
        const uint32_t grp = eb >> NR; // the group digits of the base
        C v[1 << G];
#pragma unroll
        for (int m = 0; m < (1 << G); ++m) v[m] = tile[eb | (uint32_t(m) << LO)];
#pragma unroll
        for (int u = 0; u < G; ++u) {
            const int j = INV ? JF - u : JF + u;
            const int rel = INV ? u : G - 1 - u;
            const uint32_t Lmask = (1u << (M - 1 - j)) - 1;
            const C cju = cmul(cj[u], cc[j * CZ]);
            C ph[1 << (G - 1)];
#pragma unroll
            for (int lb = 0; lb < (1 << (G - 1)); ++lb) {
                if (lb >= (1 << rel)) break;
                const uint32_t L = (grp + (uint32_t(lb) << (LO - NR))) & Lmask;
                ph[lb] = cmul(W[(L << j) << WS], cju);
            }
#pragma unroll
            for (int m = 0; m < (1 << G); ++m) {
                if ((m >> rel) & 1) continue;
                const int m1 = m | (1 << rel);
                const C phm = ph[m & ((1 << rel) - 1)];
                if (!INV) {
                    const C x = v[m], y = v[m1];
                    v[m] = cadd(x, y);
                    v[m1] = cmul(csub(x, y), phm);
                } else {
                    const C x = v[m], y = cmul(v[m1], phm);
                    v[m] = cadd(x, y);
                    v[m1] = csub(x, y);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < (1 << G); ++m) tile[eb | (uint32_t(m) << LO)] = v[m];
    }
}

// All rounds of a pass of shape (M, NR): three steps per round, the last
// round takes the remainder; a barrier after each round.
template <typename R, bool INV, int M, int NR, int WS, int S0, int NTHR>
__device__ __forceinline__ void qubit_rounds_ct(Cplx<R>* tile, const Cplx<R>* T,
                                                const Cplx<R>* B, const Cplx<R>* W,
                                                uint32_t CZ) {
    if constexpr (S0 < M) {
        constexpr int G = M - S0 < 3 ? M - S0 : 3;
        constexpr int JF = INV ? M - 1 - S0 : S0;
        qubit_round_ct<R, G, INV, M, NR, WS, JF, NTHR>(tile, T, B, W, CZ);
        __syncthreads();
        qubit_rounds_ct<R, INV, M, NR, WS, S0 + 3, NTHR>(tile, T, B, W, CZ);
    }
}

// the compile-time pass shapes: (M, NR) with E = 2^(M + NR) amplitudes per
// tile (4096 in complex64, 2048 in complex128) and Mmax = 8
template <typename R>
struct QftShapes {
    static constexpr int kE = sizeof(R) == 4 ? 12 : 11; // log2 of the tile
    static constexpr int kNR8 = kE - 8, kNR6 = kE - 6;
};

} // namespace

// One CTA per tile (grid-stride over tiles); the next tile's amplitudes are
// copied into the second tile buffer while the current one is transformed.
// Dynamic shared memory: two tile buffers (E amplitudes each), the per-tile
// step constants (M * d * CZ), the roots of unity W (nW, conjugated for
// s = -1), and the offset / tile-index tables of the read and write orders
// split into a low and a high half.
template <typename R, bool QB>
__global__ void __launch_bounds__(256, 2)
    k_qft_pass(const Cplx<R>* in, Cplx<R>* out, const __grid_constant__ QftPlan p,
               const Cplx<R>* __restrict__ Wg, const Cplx<R>* __restrict__ F) {
    using C = Cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int M = p.M, d = p.d;
    const uint32_t ncst = uint32_t(M) * d * p.CZ;
    C* bufs = reinterpret_cast<C*>(smem_raw);
    C* cst = bufs + 2 * p.E; // qubits: T (M x CZ), then B (M); qudits: M x d x CZ
    C* W = cst + ncst + M;
    uint64_t* goff_lo = reinterpret_cast<uint64_t*>(W + p.nW);
    uint64_t* goff_hi = goff_lo + p.Glo;
    uint64_t* woff_lo = goff_hi + p.E / p.Glo;
    uint64_t* woff_hi = woff_lo + p.Flo;
    uint32_t* ge_lo = reinterpret_cast<uint32_t*>(woff_hi + p.E / p.Flo);
    uint32_t* ge_hi = ge_lo + p.Glo;
    uint32_t* we_lo = ge_hi + p.E / p.Glo;
    uint32_t* we_hi = we_lo + p.Flo;

    const int tid = threadIdx.x, nt = blockDim.x;
    for (uint32_t i = tid; i < p.Glo; i += nt) {
        goff_lo[i] = order_sum(p, i, false, 0);
        ge_lo[i] = uint32_t(order_sum(p, i, false, 2));
    }
    for (uint32_t i = tid; i < p.E / p.Glo; i += nt) {
        goff_hi[i] = order_sum(p, i * p.Glo, false, 0);
        ge_hi[i] = uint32_t(order_sum(p, i * p.Glo, false, 2));
    }
    for (uint32_t i = tid; i < p.Flo; i += nt) {
        woff_lo[i] = order_sum(p, i, true, 1);
        we_lo[i] = uint32_t(order_sum(p, i, true, 2));
    }
    for (uint32_t i = tid; i < p.E / p.Flo; i += nt) {
        woff_hi[i] = order_sum(p, i * p.Flo, true, 1);
        we_hi[i] = uint32_t(order_sum(p, i * p.Flo, true, 2));
    }
    for (uint32_t i = tid; i < p.nW; i += nt) {
        C w = Wg[i];
        w.y *= R(p.sigma);
        W[i] = w;
    }
    if constexpr (QB) {
        // T[j][c] = exp(s 2 pi i Zr(c) / 2^(k-i)), i = a + j: the later
        // targets among the run digits (value c); the same for every tile
        for (uint32_t i = tid; i < uint32_t(M) * p.CZ; i += nt) {
            const uint32_t c = i % p.CZ;
            const int j = int(i / p.CZ);
            uint64_t zz = 0;
            for (int q = 0; q < p.nz; ++q) zz += uint64_t((c >> q) & 1u) * p.tzw[q];
            double sn, cs;
            sincospi(ldexp(double(zz), 1 - (p.k - p.a - j)), &sn, &cs);
            cst[i] = C{R(cs), R(p.sigma * sn)};
        }
    }
    __syncthreads();

    // base offsets and Z (the later targets outside the tile) of tile t
    auto tile_base = [&](uint64_t t, uint64_t& rb, uint64_t& wb, uint64_t& z) {
        rb = wb = z = 0;
        for (int q = 0; q < p.nod; ++q) {
            const uint64_t dg = p.pow2 ? (t >> p.oshift[q]) & (p.odim[q] - 1)
                                       : (t / p.opitch[q]) % p.odim[q];
            rb += dg * p.ors[q];
            wb += dg * p.ows[q];
            z += dg * p.ozw[q];
        }
    };
    // qubit tiles split their orders at the block size: a thread's low
    // table entries are the same for every element it moves
    const bool fixed_lo = QB && p.Glo == uint32_t(nt) && p.Flo == uint32_t(nt);
    // async copies of a tile's amplitudes, walked in read order
    auto issue_loads = [&](uint64_t rb, C* dst) {
        if (fixed_lo) {
            const C* src = in + rb + goff_lo[tid];
            C* d0 = dst + ge_lo[tid];
            for (uint32_t h = 0; h < p.E / uint32_t(nt); ++h)
                cp_async_elem(d0 + ge_hi[h], src + goff_hi[h]);
        } else {
            for (uint32_t g = tid; g < p.E; g += nt) {
                const uint32_t lo = QB ? (g & (p.Glo - 1)) : g % p.Glo;
                const uint32_t hi = QB ? (g >> p.glo_shift) : g / p.Glo;
                cp_async_elem(dst + ge_lo[lo] + ge_hi[hi], in + rb + goff_lo[lo] + goff_hi[hi]);
            }
        }
        cp_async_commit();
    };

    const uint32_t Rs = p.Rsize, CZ = p.CZ;
    // a compile-time pass shape (1: M = 8, 2: M = 6 with roots every 4th
    // entry) when the plan is one, else 0: the runtime rounds
    int shape = 0;
    if constexpr (QB) {
        using SH = QftShapes<R>;
        if (nt == 256 && p.E == (1u << SH::kE)) {
            if (p.M == 8 && p.nr == SH::kNR8 && p.wmul == 1) shape = 1;
            else if (p.M == 6 && p.nr == SH::kNR6 && p.wmul == 4) shape = 2;
        }
    }
    uint64_t t = blockIdx.x;
    if (t >= p.ntiles) return;
    uint64_t rb, wb, z;
    tile_base(t, rb, wb, z);
    issue_loads(rb, bufs);
    for (int it = 0; t < p.ntiles; t += gridDim.x, ++it) {
        C* tile = bufs + (it & 1) * p.E;
        // step constants exp(s 2 pi i r (Z + Zr(c)) / d^(k-i)), i = a + j, for
        // every value c of the later targets among the run digits (Zr: their
        // value); r (Z + Zr) < d^(k-i)
        if constexpr (QB) {
            // B[j] = exp(s 2 pi i Z / 2^(k-i)); the step constant of run
            // value c is B[j] T[j][c]
            if (tid < M) {
                double sn, cs;
                sincospi(ldexp(double(z), 1 - (p.k - p.a - tid)), &sn, &cs);
                cst[uint32_t(M) * CZ + tid] = C{R(cs), R(p.sigma * sn)};
            }
        } else
        for (uint32_t i = tid; i < ncst; i += nt) {
            const uint32_t c = i % CZ, jr = i / CZ;
            const int j = int(jr) / d, r = int(jr) % d;
            uint64_t zz = z;
            for (int q = 0; q < p.nz; ++q) zz += uint64_t((c / p.tpitch[q]) % p.tdim[q]) * p.tzw[q];
            const uint64_t N = p.dpow[p.k - p.a - j];
            double sn, cs;
            sincospi(2.0 * (double(uint64_t(r) * zz) / double(N)), &sn, &cs);
            cst[i] = C{R(cs), R(p.sigma * sn)};
        }
        const uint64_t tn = t + gridDim.x;
        uint64_t rbn = 0, wbn = 0, zn = 0;
        if (tn < p.ntiles) {
            tile_base(tn, rbn, wbn, zn);
            issue_loads(rbn, bufs + ((it + 1) & 1) * p.E);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();

        if constexpr (QB) {
            // up to three consecutive steps per round in registers: step j
            // sits on tile bit nr + M - 1 - j, so the round's bits are
            // contiguous; each thread takes the 2^G amplitudes of a base
            using SH = QftShapes<R>;
            const C* Tc = cst;
            const C* Bc = cst + M * CZ;
            if (shape == 1) {
                if (p.inverse) qubit_rounds_ct<R, true, 8, SH::kNR8, 0, 0, 256>(tile, Tc, Bc, W, CZ);
                else qubit_rounds_ct<R, false, 8, SH::kNR8, 0, 0, 256>(tile, Tc, Bc, W, CZ);
            } else if (shape == 2) {
                if (p.inverse) qubit_rounds_ct<R, true, 6, SH::kNR6, 2, 0, 256>(tile, Tc, Bc, W, CZ);
                else qubit_rounds_ct<R, false, 6, SH::kNR6, 2, 0, 256>(tile, Tc, Bc, W, CZ);
            } else
            for (int s0 = 0; s0 < M; s0 += 3) {
                const int G = M - s0 < 3 ? M - s0 : 3;
                const int jf = p.inverse ? M - 1 - s0 : s0;
                if (p.inverse) {
                    if (G == 3) qubit_round<R, 3, true>(p, tile, cst, cst + M * CZ, W, jf);
                    else if (G == 2) qubit_round<R, 2, true>(p, tile, cst, cst + M * CZ, W, jf);
                    else qubit_round<R, 1, true>(p, tile, cst, cst + M * CZ, W, jf);
                } else {
                    if (G == 3) qubit_round<R, 3, false>(p, tile, cst, cst + M * CZ, W, jf);
                    else if (G == 2) qubit_round<R, 2, false>(p, tile, cst, cst + M * CZ, W, jf);
                    else qubit_round<R, 1, false>(p, tile, cst, cst + M * CZ, W, jf);
                }
                __syncthreads();
            }
        } else {
            for (int s = 0; s < M; ++s) {
                const int j = p.inverse ? M - 1 - s : s;
                const uint32_t pj = Rs * uint32_t(p.dpow[M - 1 - j]);
                const uint64_t Ld = p.dpow[M - 1 - j], dj = p.dpow[j];
                for (uint32_t fb = tid; fb < p.E / d; fb += nt) {
                    const uint32_t hi = fb / pj, lo = fb - hi * pj;
                    const uint32_t e0 = hi * pj * d + lo;
                    const uint64_t L = (e0 / Rs) % Ld;
                    const uint32_t c = e0 % CZ;
                    C v[kQftMaxD], o[kQftMaxD];
                    for (int r = 0; r < d; ++r) v[r] = tile[e0 + r * pj];
                    auto phase = [&](int r) {
                        return cmul(W[(uint64_t(r) * L * dj) * p.wmul], // r L d^j < d^M
                                    cst[(j * d + r) * CZ + c]);
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
                __syncthreads();
            }
        }

        const R sc = R(p.scale);
        if (fixed_lo) {
            C* dst = out + wb + woff_lo[tid];
            const C* t0 = tile + we_lo[tid];
            for (uint32_t h = 0; h < p.E / uint32_t(nt); ++h) {
                C v = t0[we_hi[h]];
                v.x *= sc;
                v.y *= sc;
                dst[woff_hi[h]] = v;
            }
        } else {
            for (uint32_t f = tid; f < p.E; f += nt) {
                const uint32_t lo = QB ? (f & (p.Flo - 1)) : f % p.Flo;
                const uint32_t hi = QB ? (f >> p.flo_shift) : f / p.Flo;
                C v = tile[we_lo[lo] + we_hi[hi]];
                if (QB) {
                    v.x *= sc;
                    v.y *= sc;
                }
                out[wb + woff_lo[lo] + woff_hi[hi]] = v;
            }
        }
        __syncthreads();
        wb = wbn;
        z = zn;
    }
}

// Qubit passes of M = 8 or 6 steps over tiles of 2^EB amplitudes (EB = 12
// in complex64, 11 in complex128; EB - M run bits): two rounds of G = M / 2
// steps in registers. Each thread copies the amplitudes of its round-A bases
// (cp.async, one tile ahead) into the tile buffer at the positions it will
// read them from, transforms them, writes them back to the same positions
// (no other thread reads those in round A), and after one barrier reads its
// round-B bases, transforms them and stores them straight to global memory.
// Round A holds the steps on the tile bits [loA, loA + G), round B the rest
// (forward: steps 0..G-1 then G..M-1; inverse: M-1..G then G-1..0). A
// thread's index bits pick the other tile bits in ascending read stride for
// round A and in ascending write stride for round B, so the copies and the
// stores run over the smallest strides, also in the pass that reverses the
// targets (reading one buffer, writing another). The buffer is swizzled (tile
// bits 4-7 and 8-11 folded into 0-3) so that either order hits distinct banks,
// also when the lanes run over the tile's highest bits (the group digits are
// the lowest in memory). The phases are those of qubit_round_ct.
namespace {

__device__ __forceinline__ uint32_t q8_swz(uint32_t e) {
    return e ^ ((e >> 4) & 15u) ^ ((e >> 8) & 15u);
}

// G steps of a round on the 2^G amplitudes of base eb (round bits [lo, lo+G))
template <typename R, bool INV, int G, int M, int EB>
__device__ __forceinline__ void q8_round(Cplx<R>* v, uint32_t eb, int lo, int jf,
                                         const Cplx<R>* T, const Cplx<R>* B,
                                         const Cplx<R>* W, uint32_t CZ) {
    using C = Cplx<R>;
    constexpr int NR = EB - M, WS = 8 - M; // roots: W[e * 2^WS], 2^8 of them
    const C* cc = T + (eb & (CZ - 1));
    const uint32_t grp = eb >> NR;
#pragma unroll
    for (int u = 0; u < G; ++u) {
        const int j = INV ? jf - u : jf + u;
        const int rel = INV ? u : G - 1 - u;
        const uint32_t Lmask = (1u << (M - 1 - j)) - 1;
        const C cju = cmul(B[j], cc[j * CZ]);
        // one phase per value lb of the round bits below the step's bit,
        // applied to the pairs with that value before the next is formed
#pragma unroll
        for (int lb = 0; lb < (1 << (G - 1)); ++lb) {
            if (lb >= (1 << rel)) break;
            const uint32_t L = (grp + (uint32_t(lb) << (lo - NR))) & Lmask;
            const C phm = cmul(W[(L << j) << WS], cju);
#pragma unroll
            for (int m = 0; m < (1 << G); ++m) {
                if (((m >> rel) & 1) || (m & ((1 << rel) - 1)) != lb) continue;
                const int m1 = m | (1 << rel);
                if (!INV) {
                    const C x = v[m], y = v[m1];
                    v[m] = cadd(x, y);
                    v[m1] = cmul(csub(x, y), phm);
                } else {
                    const C x = v[m], y = cmul(v[m1], phm);
                    v[m] = cadd(x, y);
                    v[m1] = csub(x, y);
                }
            }
        }
    }
}

// the register-round pass shapes: tile bits and threads per CTA
template <typename R>
struct Q8Shape {
    static constexpr int EB = sizeof(R) == 4 ? 12 : 11;
    static constexpr int NTHR = sizeof(R) == 4 ? 256 : 128;
    static constexpr int MINB = sizeof(R) == 4 ? 2 : 3; // resident CTAs per SM
};
} // namespace

template <typename R, bool INV, typename OFF, int M>
__global__ void __launch_bounds__(Q8Shape<R>::NTHR, Q8Shape<R>::MINB)
    k_qft_pass8(const Cplx<R>* in, Cplx<R>* out, const __grid_constant__ QftPlan p,
                const Cplx<R>* __restrict__ Wg) {
    using C = Cplx<R>;
    constexpr int EB = Q8Shape<R>::EB, NTHR = Q8Shape<R>::NTHR;
    constexpr int G = M / 2, NR = EB - M;
    constexpr int NQ = EB - G;                   // tile bits outside a round
    constexpr int BPT = (1 << NQ) / NTHR;        // bases per thread per round
    static_assert(BPT >= 1, "bases per thread");
    constexpr uint32_t E = 1u << EB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* bufs = reinterpret_cast<C*>(smem_raw);                // [2][E]
    C* T = bufs + 2 * E;                                     // M x CZ
    const uint32_t CZ = p.CZ;
    C* Bs = T + M * CZ;                                      // [2][M] per-tile constants
    C* W = Bs + 2 * M;                                       // 2^8 roots
    const int tid = threadIdx.x;
    for (uint32_t i = tid; i < 256u; i += NTHR) {
        C w = Wg[i];
        w.y *= R(p.sigma);
        W[i] = w;
    }
    for (uint32_t i = tid; i < uint32_t(M) * CZ; i += NTHR) {
        const uint32_t c = i % CZ;
        const int j = int(i / CZ);
        uint64_t zz = 0;
        for (int q = 0; q < p.nz; ++q) zz += uint64_t((c >> q) & 1u) * p.tzw[q];
        double sn, cs;
        sincospi(ldexp(double(zz), 1 - (p.k - p.a - j)), &sn, &cs);
        T[i] = C{R(cs), R(p.sigma * sn)};
    }
    auto tile_base = [&](uint64_t t, OFF& rb, OFF& wb, uint64_t& z) {
        rb = wb = 0;
        z = 0;
        for (int q = 0; q < p.nod; ++q) {
            const uint64_t dg = (t >> p.oshift[q]) & (p.odim[q] - 1);
            rb += OFF(dg * p.ors[q]);
            wb += OFF(dg * p.ows[q]);
            z += dg * p.ozw[q];
        }
    };
    auto set_b = [&](uint64_t z, C* b) {
        if (tid < M) {
            double sn, cs;
            sincospi(ldexp(double(z), 1 - (p.k - p.a - tid)), &sn, &cs);
            b[tid] = C{R(cs), R(p.sigma * sn)};
        }
    };
    constexpr int loA = INV ? NR : NR + G, loB = INV ? NR + G : NR;
    constexpr int jfA = INV ? M - 1 : 0, jfB = INV ? G - 1 : G;
    // the thread's bases (index tid + NTHR c, c < BPT) in each round
    uint32_t ebA[BPT], ebB[BPT];
    OFF oA[BPT], oB[BPT];
#pragma unroll
    for (int c = 0; c < BPT; ++c) {
        const uint32_t q = uint32_t(tid) + uint32_t(c) * NTHR;
        uint32_t ea = 0, ew = 0;
        for (int i = 0; i < NQ; ++i) {
            ea |= ((q >> i) & 1u) << p.q8a[i];
            ew |= ((q >> i) & 1u) << p.q8b[i];
        }
        OFF a = 0, w = 0;
        for (int b = 0; b < EB; ++b) {
            if ((ea >> b) & 1u) a += OFF(p.trs[b]);
            if ((ew >> b) & 1u) w += OFF(p.tws[b]);
        }
        ebA[c] = ea;
        ebB[c] = ew;
        oA[c] = a;
        oB[c] = w;
    }
    auto m_off = [&](const uint64_t* st, int lo, int m) {
        OFF o = 0;
#pragma unroll
        for (int b = 0; b < G; ++b)
            if ((m >> b) & 1) o += OFF(st[lo + b]);
        return o;
    };
    // copies of a tile's round-A amplitudes into buffer `buf`
    auto issue = [&](OFF rb, C* buf) {
#pragma unroll
        for (int c = 0; c < BPT; ++c)
#pragma unroll
            for (int m = 0; m < (1 << G); ++m)
                cp_async_elem(buf + q8_swz(ebA[c] | (uint32_t(m) << loA)),
                              in + rb + oA[c] + m_off(p.trs, loA, m));
        cp_async_commit();
    };
    __syncthreads();

    uint64_t t = blockIdx.x;
    if (t >= p.ntiles) return;
    OFF rb, wb;
    uint64_t z;
    tile_base(t, rb, wb, z);
    set_b(z, Bs);
    issue(rb, bufs);
    const R sc = R(p.scale);
    for (int it = 0; t < p.ntiles; t += gridDim.x, ++it) {
        const C* B = Bs + (it & 1) * M;
        C* buf = bufs + (it & 1) * E;
        cp_async_wait<0>();
        // every thread is past the previous tile's round B: the other buffer
        // and the other constant slot are free for the next tile
        __syncthreads();
        const uint64_t tn = t + gridDim.x;
        OFF wbn = 0;
        if (tn < p.ntiles) {
            OFF rbn;
            uint64_t zn;
            tile_base(tn, rbn, wbn, zn);
            set_b(zn, Bs + ((it + 1) & 1) * M);
            issue(rbn, bufs + ((it + 1) & 1) * E);
        }
#pragma unroll
        for (int c = 0; c < BPT; ++c) {
            C v[1 << G];
#pragma unroll
            for (int m = 0; m < (1 << G); ++m) v[m] = buf[q8_swz(ebA[c] | (uint32_t(m) << loA))];
            q8_round<R, INV, G, M, EB>(v, ebA[c], loA, jfA, T, B, W, CZ);
#pragma unroll
            for (int m = 0; m < (1 << G); ++m) buf[q8_swz(ebA[c] | (uint32_t(m) << loA))] = v[m];
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < BPT; ++c) {
            C v[1 << G];
#pragma unroll
            for (int m = 0; m < (1 << G); ++m) v[m] = buf[q8_swz(ebB[c] | (uint32_t(m) << loB))];
            q8_round<R, INV, G, M, EB>(v, ebB[c], loB, jfB, T, B, W, CZ);
#pragma unroll
            for (int m = 0; m < (1 << G); ++m) {
                C x = v[m];
                x.x *= sc;
                x.y *= sc;
                out[wb + oB[c] + m_off(p.tws, loB, m)] = x;
            }
        }
        wb = wbn;
    }
}

int qft_pass8_tile_bits(qgpu_prec prec) {
    return prec == QGPU_C64 ? Q8Shape<float>::EB : Q8Shape<double>::EB;
}

// whether k_qft_pass8 applies: qubits, 8 or 6 steps over tiles of 2^EB
// amplitudes; in place, or (the pass that reverses the targets) into another
// buffer
bool qft_pass8_applies(qgpu_prec prec, const void* in, const void* out, const QftPlan& p) {
    const int EB = qft_pass8_tile_bits(prec);
    if (p.d != 2 || (p.M != 8 && p.M != 6) || p.nr != EB - p.M || p.E != (1u << EB) ||
        p.wmul != (1u << (8 - p.M)) || p.ntd != EB || p.nW != 256u || !p.pow2)
        return false;
    bool same = true;
    for (int q = 0; q < p.ntd; ++q) {
        if (p.tdim[q] != 2 || p.tpitch[q] != (1u << q)) return false;
        same = same && p.trs[q] == p.tws[q];
    }
    for (int q = 0; q < p.nod; ++q) same = same && p.ors[q] == p.ows[q];
    if (in == out && !same) return false;
    // both rounds must reach 128-byte runs across a warp's lanes: when the
    // lowest memory digits are a round's own bits (the pass whose targets
    // are the lowest digits, without the reversal), each thread would hold
    // a contiguous run itself and the lanes' accesses would scatter; such a
    // pass stays with the shared-memory rounds, which write in memory order
    QftPlan q = p;
    qft_pass8_maps(q, EB);
    const int NQ = EB - p.M / 2;
    const uint32_t run = prec == QGPU_C64 ? 16 : 8;
    for (int r = 0; r < 2; ++r) {
        const uint8_t* map = r ? q.q8b : q.q8a;
        const uint64_t* st = r ? q.tws : q.trs;
        for (uint32_t l = 1; l < run; ++l) {
            uint64_t o = 0;
            for (int i = 0; i < NQ; ++i)
                if ((l >> i) & 1u) o += st[map[i]];
            if (o != l) return false;
        }
    }
    return true;
}

// the thread-to-base maps of k_qft_pass8: the tile bits outside a round's
// [lo, lo + G), by ascending stride
void qft_pass8_maps(QftPlan& p, int EB) {
    const int G = p.M / 2, NR = EB - p.M;
    const int loA = p.inverse ? NR : NR + G, loB = p.inverse ? NR + G : NR;
    auto fill = [&](int lo, const uint64_t* st, uint8_t* out) {
        int bits[16], c = 0;
        for (int b = 0; b < EB; ++b)
            if (b < lo || b >= lo + G) bits[c++] = b;
        std::stable_sort(bits, bits + c, [&](int x, int y) { return st[x] < st[y]; });
        for (int i = 0; i < c; ++i) out[i] = uint8_t(bits[i]);
    };
    fill(loA, p.trs, p.q8a);
    fill(loB, p.tws, p.q8b);
}

template <typename R>
static void qft_pass8_launch(qgpu_ctx* ctx, const void* in, void* out, const QftPlan& p0,
                             const void* W) {
    using C = Cplx<R>;
    using S = Q8Shape<R>;
    QftPlan q = p0;
    qft_pass8_maps(q, S::EB);
    const size_t sm = (2 * (size_t(1) << S::EB) + size_t(q.M) * q.CZ + 2 * size_t(q.M) + 256) *
                      sizeof(C);
    // 64 CTAs per SM, several tiles each: at 30 qubits complex128 TFQ took
    // 26.7 ms this way, 30.4 ms with one resident wave and 32.3 ms with one
    // tile per CTA (each CTA builds its step tables once)
    uint64_t blocks = uint64_t(grid_blocks(ctx, 64));
    if (q.ntiles < blocks) blocks = q.ntiles;
    // 32-bit offsets when the state has fewer than 2^31 amplitudes
    const bool narrow = q.ntiles <= (uint64_t(1) << (31 - S::EB));
    using K = void (*)(const C*, C*, const QftPlan, const C*);
    K kern;
    if (q.M == 8)
        kern = narrow ? (q.inverse ? K(k_qft_pass8<R, true, uint32_t, 8>) : K(k_qft_pass8<R, false, uint32_t, 8>))
                      : (q.inverse ? K(k_qft_pass8<R, true, uint64_t, 8>) : K(k_qft_pass8<R, false, uint64_t, 8>));
    else
        kern = narrow ? (q.inverse ? K(k_qft_pass8<R, true, uint32_t, 6>) : K(k_qft_pass8<R, false, uint32_t, 6>))
                      : (q.inverse ? K(k_qft_pass8<R, true, uint64_t, 6>) : K(k_qft_pass8<R, false, uint64_t, 6>));
    ensure_smem(reinterpret_cast<const void*>(kern), sm);
    kern<<<unsigned(blocks), S::NTHR, sm, ctx->stream>>>(static_cast<const C*>(in),
                                                         static_cast<C*>(out), q,
                                                         static_cast<const C*>(W));
}

size_t qft_smem_bytes(const QftPlan& p, size_t elem_bytes) {
    return (2 * size_t(p.E) + size_t(p.M) * p.d * p.CZ + p.M + p.nW) * elem_bytes +
           (p.Glo + p.E / p.Glo + p.Flo + p.E / p.Flo) * (sizeof(uint64_t) + sizeof(uint32_t));
}

template <typename R>
static void qft_launch(qgpu_ctx* ctx, const void* in, void* out, const QftPlan& p,
                       const void* W, const void* F) {
    using C = Cplx<R>;
    const size_t sm = qft_smem_bytes(p, sizeof(C));
    uint64_t blocks = uint64_t(grid_blocks(ctx, 2));
    if (p.ntiles < blocks) blocks = p.ntiles;
    if (p.d == 2) {
        ensure_smem(reinterpret_cast<const void*>(k_qft_pass<R, true>), sm);
        k_qft_pass<R, true><<<unsigned(blocks), 256, sm, ctx->stream>>>(
            static_cast<const C*>(in), static_cast<C*>(out), p, static_cast<const C*>(W),
            static_cast<const C*>(F));
    } else {
        ensure_smem(reinterpret_cast<const void*>(k_qft_pass<R, false>), sm);
        k_qft_pass<R, false><<<unsigned(blocks), 256, sm, ctx->stream>>>(
            static_cast<const C*>(in), static_cast<C*>(out), p, static_cast<const C*>(W),
            static_cast<const C*>(F));
    }
    after_launch(ctx, "k_qft_pass");
}

void launch_qft_pass(qgpu_ctx* ctx, qgpu_prec prec, const void* in, void* out,
                     const QftPlan& p, const void* W, const void* F) {
    if (p.ntiles == 0) return;
    if (qft_pass8_applies(prec, in, out, p)) {
        if (prec == QGPU_C64) qft_pass8_launch<float>(ctx, in, out, p, W);
        else qft_pass8_launch<double>(ctx, in, out, p, W);
        after_launch(ctx, "k_qft_pass8");
        return;
    }
    if (prec == QGPU_C128) qft_launch<double>(ctx, in, out, p, W, F);
    else qft_launch<float>(ctx, in, out, p, W, F);
}

} // namespace qgpu
