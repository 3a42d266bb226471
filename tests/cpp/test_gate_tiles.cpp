// CPU check of the plain form's tile passes (qgpu::gate_desc_of,
// qgpu::plan_gate_tiles and the addressing of k_tile_pass, its swizzled
// shared-memory layout and its sweeps of register groups): random sequences
// of 1- and 2-qubit gates, fan gates and controlled gates (1-3 controls, with
// and without shifts) on kets of 1-16 qubits, for several tile sizes. A host
// model of the kernel (the same tile-base insertion, offset table, per-tile
// and per-amplitude control tests and arithmetic) must reproduce, bit for
// bit, the gates applied one at a time over the whole state; every pass must
// respect its tile budget, visit every amplitude exactly once and read and
// write only inside the state. Built and run by tests/test_gate_tiles.py.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "circuit.hpp"
#include "tile_gates.hpp"

using namespace qgpu;
using C = std::complex<double>;

static int fails = 0;
#define EXPECT(c)                                                                     \
    do {                                                                              \
        if (!(c)) {                                                                   \
            if (fails < 20) std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c);   \
            ++fails;                                                                  \
        }                                                                             \
    } while (0)

// the kernels' complex product and fused multiply-add, in the same order
static C cmul(C a, C b) {
    return {a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real()};
}
static C cfma(C a, C b, C acc) {
    double x = std::fma(a.real(), b.real(), acc.real());
    x = std::fma(-a.imag(), b.imag(), x);
    double y = std::fma(a.real(), b.imag(), acc.imag());
    y = std::fma(a.imag(), b.real(), y);
    return {x, y};
}

// the kernel's complex128 tile layout (3 column bits): column XOR the
// folded row number
static uint32_t tswz(uint32_t e) {
    uint32_t r = e >> 3, h = 0;
    for (int k = 0; k < 16; k += 3) h ^= r >> k;
    return e ^ (h & 7u);
}

static bool ctrl_ok(const GateDesc& g, uint64_t i) {
    for (auto& c : g.ctrl)
        if (int((i >> c.first) & 1) != c.second) return false;
    return true;
}

// one gate over the whole state (what the one-gate kernels compute)
static void apply_direct(std::vector<C>& psi, int nbits, const GateDesc& g) {
    const uint64_t N = uint64_t(1) << nbits;
    if (g.op == 1) {
        const C a00 = g.A[0], a01 = g.A[2], a10 = g.A[1], a11 = g.A[3];
        const uint64_t s = uint64_t(1) << g.b0;
        for (uint64_t i0 = 0; i0 < N; ++i0) {
            if (i0 & s) continue;
            if (!ctrl_ok(g, i0)) continue;
            const C v0 = psi[i0], v1 = psi[i0 + s];
            C r0 = cmul(a00, v0);
            r0 = cfma(a01, v1, r0);
            C r1 = cmul(a10, v0);
            r1 = cfma(a11, v1, r1);
            psi[i0] = r0;
            psi[i0 + s] = r1;
        }
    } else {
        const uint64_t s0 = uint64_t(1) << g.b0, s1 = uint64_t(1) << g.b1;
        for (uint64_t b = 0; b < N; ++b) {
            if ((b & s0) || (b & s1)) continue;
            if (!ctrl_ok(g, b)) continue;
            const C v[4] = {psi[b], psi[b + s1], psi[b + s0], psi[b + s0 + s1]};
            C r[4];
            for (int row = 0; row < 4; ++row) {
                C acc = cmul(g.A[row], v[0]);
                acc = cfma(g.A[row + 4], v[1], acc);
                acc = cfma(g.A[row + 8], v[2], acc);
                acc = cfma(g.A[row + 12], v[3], acc);
                r[row] = acc;
            }
            psi[b] = r[0];
            psi[b + s1] = r[1];
            psi[b + s0] = r[2];
            psi[b + s0 + s1] = r[3];
        }
    }
}

// host model of k_tile_pass over every tile of one pass: sweeps of groups of
// 2^nb amplitudes, the gates of a sweep applied to each group in order
static void apply_pass(std::vector<C>& psi, const TilePassParams& p,
                       const std::vector<TileGate>& gates, const std::vector<TileSweep>& sweeps,
                       const std::vector<cd>& mats, std::vector<int>& visits) {
    const uint32_t nel = 1u << p.T, lmask = (1u << p.L) - 1;
    const int nhi = p.T - p.L;
    std::vector<uint64_t> hioff(size_t(1) << nhi);
    for (uint32_t j = 0; j < hioff.size(); ++j) {
        uint64_t o = 0;
        for (int i = 0; i < nhi; ++i)
            if ((j >> i) & 1u) o |= uint64_t(1) << p.hi[i];
        hioff[j] = o;
    }
    std::vector<C> tile(nel);
    for (uint64_t t = 0; t < p.ntiles; ++t) {
        uint64_t base = t << p.L;
        for (int i = 0; i < nhi; ++i) {
            const uint64_t low = (uint64_t(1) << p.hi[i]) - 1;
            base = ((base & ~low) << 1) | (base & low);
        }
        for (uint32_t e = 0; e < nel; ++e) {
            const uint64_t a = base + hioff[e >> p.L] + (e & lmask);
            EXPECT(a < psi.size());
            if (a >= psi.size()) return;
            tile[tswz(e)] = psi[a];
            ++visits[a];
        }
        for (uint32_t s = 0; s < p.nsweeps; ++s) {
            const TileSweep& sw = sweeps[p.first_sweep + s];
            const int NB = int(sw.nb), G = 1 << NB;
            std::vector<uint32_t> off(G);
            for (int j = 0; j < G; ++j) {
                uint32_t o = 0;
                for (int k = 0; k < NB; ++k)
                    if (j & (1 << k)) o |= 1u << sw.b[k];
                off[j] = o;
            }
            std::vector<int> seen(nel, 0);
            std::vector<int> sb(sw.b, sw.b + NB);
            std::sort(sb.begin(), sb.end());
            const int nq = p.T - NB;
            for (uint32_t q = 0; q < (1u << nq); ++q) {
                uint32_t b = q;
                for (int k = 0; k < NB; ++k) {
                    const uint32_t low = (1u << sb[k]) - 1;
                    b = ((b & ~low) << 1) | (b & low);
                }
                std::vector<C> v(G);
                for (int j = 0; j < G; ++j) {
                    EXPECT(b + off[j] < nel && tswz(b + off[j]) < nel);
                    EXPECT(tswz(b + off[j]) == (tswz(b) ^ tswz(off[j]))); // the kernel's form
                    v[j] = tile[tswz(b + off[j])];
                    ++seen[b + off[j]];
                }
                for (uint32_t k = 0; k < sw.ngates; ++k) {
                    const TileGate& g = gates[sw.first + k];
                    if ((base & g.gmask) != g.gval) continue;
                    const cd* m = mats.data() + g.mat;
                    if (g.op == 1) {
                        const int K = int(g.k0);
                        for (int j = 0; j < G; ++j) {
                            if (j & (1 << K)) continue;
                            if (((b + off[j]) & g.lmask) != g.lval) continue;
                            const int j1 = j | (1 << K);
                            C r0 = cmul(m[0], v[j]);
                            r0 = cfma(m[1], v[j1], r0);
                            C r1 = cmul(m[2], v[j]);
                            r1 = cfma(m[3], v[j1], r1);
                            v[j] = r0;
                            v[j1] = r1;
                        }
                    } else {
                        const int K0 = int(g.k0), K1 = int(g.k1);
                        for (int j = 0; j < G; ++j) {
                            if (j & ((1 << K0) | (1 << K1))) continue;
                            if (((b + off[j]) & g.lmask) != g.lval) continue;
                            const int j1 = j | (1 << K1), j2 = j | (1 << K0), j3 = j2 | (1 << K1);
                            const C x[4] = {v[j], v[j1], v[j2], v[j3]};
                            C r[4];
                            for (int row = 0; row < 4; ++row) {
                                C acc = cmul(m[4 * row], x[0]);
                                acc = cfma(m[4 * row + 1], x[1], acc);
                                acc = cfma(m[4 * row + 2], x[2], acc);
                                acc = cfma(m[4 * row + 3], x[3], acc);
                                r[row] = acc;
                            }
                            v[j] = r[0];
                            v[j1] = r[1];
                            v[j2] = r[2];
                            v[j3] = r[3];
                        }
                    }
                }
                for (int j = 0; j < G; ++j) tile[tswz(b + off[j])] = v[j];
            }
            for (uint32_t e = 0; e < nel; ++e) EXPECT(seen[e] == 1);
        }
        for (uint32_t e = 0; e < nel; ++e) psi[base + hioff[e >> p.L] + (e & lmask)] = tile[tswz(e)];
    }
}

static std::vector<cd> rand_mat(std::mt19937_64& rng, int D) {
    std::normal_distribution<double> nd;
    std::vector<cd> U(size_t(D) * D);
    for (auto& x : U) x = cd(nd(rng), nd(rng));
    return U;
}

int main() {
    std::mt19937_64 rng(7);
    int cases = 0;
    for (int nbits = 1; nbits <= 16; ++nbits) {
        for (int Tmax : {5, 8, 11, 12, 13}) {
            for (int rep = 0; rep < 3; ++rep) {
                // random steps -> gate descriptors
                std::vector<GateDesc> gates;
                std::uniform_int_distribution<int> q(0, nbits - 1);
                for (int k = 0; k < 60; ++k) {
                    Step st;
                    const int kind = int(rng() % 5);
                    std::vector<int> perm(nbits);
                    for (int i = 0; i < nbits; ++i) perm[i] = i;
                    std::shuffle(perm.begin(), perm.end(), rng);
                    if (kind == 0 || nbits < 2) {
                        st.kind = StepKind::Gate;
                        st.target = {uint64_t(perm[0])};
                        st.DU = 2;
                    } else if (kind == 1) {
                        st.kind = StepKind::Gate;
                        st.target = {uint64_t(perm[0]), uint64_t(perm[1])};
                        st.DU = 4;
                    } else if (kind == 2) {
                        st.kind = StepKind::Fan;
                        const int nt = 1 + int(rng() % std::min(3, nbits));
                        for (int i = 0; i < nt; ++i) st.target.push_back(uint64_t(perm[i]));
                        st.DU = 2;
                    } else {
                        const int nt = (kind == 4 && nbits >= 3) ? 2 : 1;
                        const int nc = 1 + int(rng() % std::max(1, std::min(3, nbits - nt)));
                        if (nt + nc > nbits) {
                            st.kind = StepKind::Gate;
                            st.target = {uint64_t(perm[0])};
                            st.DU = 2;
                        } else {
                            st.kind = StepKind::Ctrl;
                            for (int i = 0; i < nc; ++i) st.ctrl.push_back(uint64_t(perm[i]));
                            for (int i = 0; i < nt; ++i) st.target.push_back(uint64_t(perm[nc + i]));
                            st.DU = uint64_t(1) << nt;
                            if (rng() % 2) {
                                st.has_shift = true;
                                for (int i = 0; i < nc; ++i) st.shift.push_back(rng() % 2);
                            }
                        }
                    }
                    st.U = rand_mat(rng, int(st.DU));
                    const size_t before = gates.size();
                    EXPECT(gate_desc_of(st, nbits, gates));
                    EXPECT(gates.size() > before);
                }
                std::vector<TilePassParams> passes;
                std::vector<TileGate> dev;
                std::vector<TileSweep> sweeps;
                std::vector<cd> mats;
                plan_gate_tiles(gates, nbits, Tmax, passes, dev, sweeps, mats);
                EXPECT(dev.size() == gates.size());
                std::normal_distribution<double> nd;
                const uint64_t N = uint64_t(1) << nbits;
                std::vector<C> a(N), b;
                for (auto& x : a) x = C(nd(rng), nd(rng));
                b = a;
                for (const auto& g : gates) apply_direct(a, nbits, g);
                uint32_t covered = 0;
                for (const auto& p : passes) {
                    EXPECT(p.T <= std::min(nbits, Tmax) && p.L <= 5 && p.L <= p.T);
                    EXPECT(p.first == covered && p.ngates >= 1 && p.ngates <= 256);
                    EXPECT(p.mat_first == dev[p.first].mat);
                    covered += p.ngates;
                    // the pass's sweeps cover its gates in order; every gate's
                    // targets are its sweep's bits k0 (and k1)
                    uint32_t next = p.first;
                    for (uint32_t s = 0; s < p.nsweeps; ++s) {
                        const TileSweep& sw = sweeps[p.first_sweep + s];
                        EXPECT(sw.first == next && sw.ngates >= 1 && sw.nb >= 1 && sw.nb <= 3);
                        for (uint32_t k = sw.first; k < sw.first + sw.ngates; ++k) {
                            const TileGate& g = dev[k];
                            EXPECT(g.k0 < sw.nb && sw.b[g.k0] == g.t0);
                            if (g.op == 2) EXPECT(g.k1 < sw.nb && sw.b[g.k1] == g.t1 && g.k1 != g.k0);
                        }
                        next += sw.ngates;
                    }
                    EXPECT(next == p.first + p.ngates);
                    std::vector<int> visits(N, 0);
                    apply_pass(b, p, dev, sweeps, mats, visits);
                    for (uint64_t i = 0; i < N; ++i) EXPECT(visits[i] == 1);
                }
                EXPECT(covered == gates.size());
                for (uint64_t i = 0; i < N; ++i) EXPECT(a[i] == b[i]);
                ++cases;
            }
        }
    }
    // steps that are not 1- or 2-qubit unitaries are left to the per-step path
    {
        std::vector<GateDesc> g;
        Step st;
        st.kind = StepKind::Gate;
        st.target = {0, 1, 2};
        st.DU = 8;
        st.U.assign(64, cd(0));
        EXPECT(!gate_desc_of(st, 5, g) && g.empty());
        st.kind = StepKind::Measure;
        st.target = {0};
        EXPECT(!gate_desc_of(st, 5, g) && g.empty());
    }
    if (fails) {
        std::printf("%d failures\n", fails);
        return 1;
    }
    std::printf("gate tiles ok: %d cases\n", cases);
    return 0;
}
