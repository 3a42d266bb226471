// CPU check of the trajectory kernel's cache blocking (qgpu::plan_tiles and
// the tile-pass index arithmetic of k_traj): random gate programs over
// 15-18 qubits are run untiled and tiled by a host interpreter that uses the
// kernel's gate arithmetic (complex64, the same operation order) and its
// gather / scatter addressing (offset table for the tile bits above 4, bits
// of the tile number deposited into the other bits). Checks: every address
// is inside the register, every amplitude is gathered exactly once per tile
// pass, and the tiled result equals the untiled one bit for bit.
// Built and run by tests/test_tiles.py.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "traj.hpp"

using namespace qgpu;
using f2 = std::complex<float>;

static int fails = 0;
#define EXPECT(c)                                                            \
    do {                                                                     \
        if (!(c)) {                                                          \
            if (fails < 20) std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c); \
            ++fails;                                                         \
        }                                                                    \
    } while (0)

static uint32_t ins0(uint32_t x, int b) {
    uint32_t low = (1u << b) - 1;
    return ((x & ~low) << 1) | (x & low);
}
// the kernel's c_mul / c_fma (fmaf order)
static f2 cmul(f2 a, f2 b) {
    return f2(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}
static f2 cfma(f2 a, f2 b, f2 c) {
    float x = std::fma(a.real(), b.real(), c.real());
    x = std::fma(-a.imag(), b.imag(), x);
    float y = std::fma(a.real(), b.imag(), c.imag());
    y = std::fma(a.imag(), b.real(), y);
    return f2(x, y);
}

static void gate(const TInstr& I, const float* mats, f2* psi, uint32_t N) {
    const f2* m = reinterpret_cast<const f2*>(mats) + I.mat;
    switch (I.op) {
        case kTG1:
        case kTCG1:
            for (uint32_t p = 0; p < N / 2; ++p) {
                uint32_t i = ins0(p, I.b0), s = 1u << I.b0;
                if (I.op == kTCG1 && (i & I.cmask) != I.cval) continue;
                f2 v0 = psi[i], v1 = psi[i + s];
                psi[i] = cfma(m[2], v1, cmul(m[0], v0));
                psi[i + s] = cfma(m[3], v1, cmul(m[1], v0));
            }
            break;
        case kTG3: {
            // 8 x 8 on (b0, b1, cmask & 255), row index 4 b0 + 2 b1 + b2
            int sb[3] = {I.b0, I.b1, int(I.cmask & 255u)};
            std::sort(sb, sb + 3);
            const uint32_t o4 = 1u << I.b0, o2 = 1u << I.b1, o1 = 1u << (I.cmask & 255u);
            for (uint32_t p = 0; p < N / 8; ++p) {
                const uint32_t i = ins0(ins0(ins0(p, sb[0]), sb[1]), sb[2]);
                auto at = [&](int r) {
                    return i + ((r & 4) ? o4 : 0u) + ((r & 2) ? o2 : 0u) + ((r & 1) ? o1 : 0u);
                };
                f2 v[8];
                for (int c = 0; c < 8; ++c) v[c] = psi[at(c)];
                for (int row = 0; row < 8; ++row) {
                    f2 acc = cmul(m[row], v[0]);
                    for (int c = 1; c < 8; ++c) acc = cfma(m[row + 8 * c], v[c], acc);
                    psi[at(row)] = acc;
                }
            }
            break;
        }
        case kTG2: {
            int lo = std::min(I.b0, I.b1), hi = std::max(I.b0, I.b1);
            uint32_t s0 = 1u << I.b0, s1 = 1u << I.b1;
            for (uint32_t p = 0; p < N / 4; ++p) {
                uint32_t i = ins0(ins0(p, lo), hi);
                f2 v[4] = {psi[i], psi[i + s1], psi[i + s0], psi[i + s0 + s1]}, r[4];
                for (int row = 0; row < 4; ++row) {
                    f2 acc = cmul(m[row], v[0]);
                    acc = cfma(m[row + 4], v[1], acc);
                    acc = cfma(m[row + 8], v[2], acc);
                    acc = cfma(m[row + 12], v[3], acc);
                    r[row] = acc;
                }
                psi[i] = r[0];
                psi[i + s1] = r[1];
                psi[i + s0] = r[2];
                psi[i + s0 + s1] = r[3];
            }
            break;
        }
        case kTG4: {
            int bb[4] = {I.b0, I.b1, int(I.cmask & 255u), int((I.cmask >> 8) & 255u)};
            int sb[4] = {bb[0], bb[1], bb[2], bb[3]};
            std::sort(sb, sb + 4);
            auto off = [&](int r) {
                return ((uint32_t(r) >> 3 & 1u) << bb[0]) | ((uint32_t(r) >> 2 & 1u) << bb[1]) |
                       ((uint32_t(r) >> 1 & 1u) << bb[2]) | ((uint32_t(r) & 1u) << bb[3]);
            };
            for (uint32_t g = 0; g < N / 16; ++g) {
                uint32_t i = ins0(ins0(ins0(ins0(g, sb[0]), sb[1]), sb[2]), sb[3]);
                f2 out[16];
                for (int row = 0; row < 16; ++row) {
                    f2 acc(0.f, 0.f);
                    for (int c = 0; c < 16; ++c) acc = cfma(m[row + 16 * c], psi[i + off(c)], acc);
                    out[row] = acc;
                }
                for (int row = 0; row < 16; ++row) psi[i + off(row)] = out[row];
            }
            break;
        }
        default:
            break;
    }
}

// The kernel's tile pass (no noise): offset table, deposit, gather, local
// gates, scatter.
static void tile_pass(const std::vector<TInstr>& prog, const float* mats, size_t k, int n,
                      f2* psi) {
    const TInstr H = prog[k];
    const int T = H.b0;
    const uint32_t m = H.cmask;
    std::vector<uint32_t> tb(T);
    std::memcpy(tb.data(), mats + 2 * size_t(H.mat), T * sizeof(uint32_t));
    EXPECT(T >= 9 && T <= 14);
    for (int j = 0; j < 5; ++j) EXPECT(tb[j] == uint32_t(j));
    for (int j = 1; j < T; ++j) EXPECT(tb[j] > tb[j - 1] && tb[j] < uint32_t(n));
    const uint32_t NT = 1u << T, NH = NT >> 5, N = 1u << n;
    std::vector<uint32_t> offh(NH);
    for (uint32_t lh = 0; lh < NH; ++lh) {
        uint32_t o = 0;
        for (int j = 5; j < T; ++j) o |= ((lh >> (j - 5)) & 1u) << tb[j];
        offh[lh] = o;
    }
    uint32_t tilebits = 0;
    for (int j = 0; j < T; ++j) tilebits |= 1u << tb[j];
    const uint32_t rest = ((1u << n) - 1) & ~tilebits;
    std::vector<uint8_t> seen(N, 0);
    std::vector<f2> tile(NT);
    for (uint32_t t = 0; t < (1u << (n - T)); ++t) {
        uint32_t base = 0, r = rest, tt = t;
        while (r) {
            const uint32_t low = r & (0u - r);
            if (tt & 1u) base |= low;
            tt >>= 1;
            r ^= low;
        }
        for (uint32_t l = 0; l < NT; ++l) {
            const uint32_t a = base + offh[l >> 5] + (l & 31u);
            EXPECT(a < N);
            if (a < N) {
                EXPECT(seen[a] == 0);
                seen[a] = 1;
                tile[l] = psi[a];
            }
        }
        for (uint32_t i = k + 1; i < k + 1 + m; ++i) {
            const TInstr& I = prog[i];
            // local bits inside the tile
            EXPECT(I.b0 < T);
            if (I.op == kTG2 || I.op == kTG3 || I.op == kTG4) EXPECT(I.b1 < T);
            if (I.op == kTG3) EXPECT((I.cmask & 255u) < uint32_t(T));
            if (I.op == kTCG1) EXPECT((I.cmask >> T) == 0);
            gate(I, mats, tile.data(), NT);
        }
        for (uint32_t l = 0; l < NT; ++l) {
            const uint32_t a = base + offh[l >> 5] + (l & 31u);
            if (a < N) psi[a] = tile[l];
        }
    }
    for (uint32_t a = 0; a < N; ++a) EXPECT(seen[a] == 1);
}

static void run(const TProgram& P, std::vector<f2>& psi) {
    const uint32_t N = 1u << P.n;
    for (size_t k = 0; k < P.ins.size(); ++k) {
        const TInstr& I = P.ins[k];
        if (I.op == kTTile) {
            tile_pass(P.ins, P.mats.data(), k, int(P.n), psi.data());
            k += I.cmask;
        } else {
            gate(I, P.mats.data(), psi.data(), N);
        }
    }
}

// The layer kernel's traversal (k_pass_batch: contiguous item ranges per
// CTA, a cursor over (register, item, tile)) with the launch layout of the
// batch runner (items of 2^15 amplitudes): every tile of every register of
// the launch is visited exactly once, whatever the grid.
static void check_layer_cursor(std::mt19937& rng) {
    for (int trial = 0; trial < 50; ++trial) {
        const int ninst = 1 + int(rng() % 40);
        std::vector<PassInst> insts(ninst);
        uint32_t items = 0;
        for (int j = 0; j < ninst; ++j) {
            PassInst& q = insts[j];
            q.n = uint8_t(15 + rng() % 8);
            q.T = uint8_t(rng() & 1 ? 12 : 13);
            const uint32_t ntiles = 1u << (q.n - q.T);
            q.tiles_per_item = std::min<uint32_t>(ntiles, std::max<uint32_t>(1, (1u << 15) >> q.T));
            q.first_item = items;
            items += (ntiles + q.tiles_per_item - 1) / q.tiles_per_item;
        }
        std::vector<std::vector<int>> seen(ninst);
        for (int j = 0; j < ninst; ++j) seen[j].assign(1u << (insts[j].n - insts[j].T), 0);
        const uint32_t grid = 1 + rng() % 300;
        const uint32_t per = (items + grid - 1) / grid;
        for (uint32_t bx = 0; bx < grid; ++bx) {
            const uint32_t it0 = bx * per, it1 = std::min(items, it0 + per);
            if (it0 >= it1) continue;
            int lo = 0, hi = ninst - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (insts[mid].first_item <= it0) lo = mid;
                else hi = mid - 1;
            }
            int j = lo;
            uint32_t it = it0;
            auto item = [&](uint32_t& t, uint32_t& t1) {
                const PassInst& P = insts[j];
                t = (it - P.first_item) * P.tiles_per_item;
                t1 = std::min(t + P.tiles_per_item, 1u << (P.n - P.T));
            };
            uint32_t t, t1;
            item(t, t1);
            for (;;) {
                EXPECT(t < seen[j].size());
                if (t < seen[j].size()) ++seen[j][t];
                if (++t < t1) continue;
                if (++it >= it1) break;
                while (j + 1 < ninst && insts[j + 1].first_item <= it) ++j;
                item(t, t1);
            }
        }
        for (int j = 0; j < ninst; ++j)
            for (int c : seen[j]) EXPECT(c == 1);
    }
}

int main() {
    std::mt19937 rng(12345);
    check_layer_cursor(rng);
    std::normal_distribution<float> g(0.f, 1.f);
    for (int trial = 0; trial < 8; ++trial) {
        const int n = 15 + trial % 4; // 15..18
        TProgram P;
        P.n = uint32_t(n);
        // random matrices: 2x2, 4x4, 16x16 (not unitary: exercises arithmetic)
        auto add = [&](int D) {
            uint32_t off = uint32_t(P.mats.size() / 2);
            for (int i = 0; i < D * D; ++i) {
                P.mats.push_back(g(rng) * 0.3f);
                P.mats.push_back(g(rng) * 0.3f);
            }
            return off;
        };
        std::uniform_int_distribution<int> qb(0, n - 1), op(0, 9);
        const int len = 30 + trial * 3;
        for (int i = 0; i < len; ++i) {
            TInstr I{};
            int o = op(rng);
            I.flags = (i % 5 == 0) ? kTNewStep : 0;
            int a = qb(rng), b = qb(rng), c = qb(rng), d = qb(rng);
            while (b == a) b = qb(rng);
            if (o < 4) {
                I.op = kTG1;
                I.b0 = uint8_t(a);
                I.mat = add(2);
            } else if (o < 7) {
                I.op = kTG2;
                I.b0 = uint8_t(a);
                I.b1 = uint8_t(b);
                I.mat = add(4);
            } else if (o < 8) {
                I.op = kTCG1;
                I.b0 = uint8_t(a);
                I.cmask = 1u << b;
                I.cval = (trial & 1) ? (1u << b) : 0u;
                I.mat = add(2);
            } else if (o < 9) {
                while (c == a || c == b) c = qb(rng);
                while (d == a || d == b || d == c) d = qb(rng);
                I.op = kTG4;
                I.b0 = uint8_t(a);
                I.b1 = uint8_t(b);
                I.cmask = uint32_t(c) | (uint32_t(d) << 8);
                I.mat = add(16);
            } else {
                I.op = kTMeas; // not tileable: splits runs (not executed here)
                I.b0 = uint8_t(a);
            }
            P.ins.push_back(I);
        }
        // measurements split the runs; the interpreter skips them
        const TProgram U = P;
        {
            // folding 1-qubit gates into their next gate: same result up to
            // complex64 rounding, no more instructions than before
            TProgram F = U;
            fold_1q_gates(F);
            EXPECT(F.ins.size() <= U.ins.size());
            const uint32_t N = 1u << n;
            std::vector<f2> a(N), c(N);
            for (uint32_t i = 0; i < N; ++i) a[i] = c[i] = f2(g(rng), g(rng));
            run(U, a);
            run(F, c);
            double num = 0, den = 0;
            for (uint32_t i = 0; i < N; ++i) {
                num = std::max(num, double(std::abs(a[i] - c[i])));
                den = std::max(den, double(std::abs(a[i])));
            }
            EXPECT(num <= 1e-4 * den);
        }
        for (int w = 2; w <= kFuseMaxWidth; ++w) {
            // dense blocks of at most w bits (wider gates pass as they are):
            // same result up to complex64 rounding, also after tiling
            TProgram F = U;
            fuse_blocks(F, w);
            size_t gates = 0, gates_u = 0;
            for (const auto& I : F.ins) {
                const int k = I.op == kTG1 ? 1 : I.op == kTG2 ? 2 : I.op == kTG3 ? 3 : I.op == kTG4 ? 4 : 0;
                if (k) ++gates;
                EXPECT(k <= w || I.op == kTG4);
            }
            for (const auto& I : U.ins) gates_u += I.op != kTMeas;
            EXPECT(gates <= gates_u);
            const uint32_t N = 1u << n;
            std::vector<f2> a(N), c(N), t(N);
            for (uint32_t i = 0; i < N; ++i) a[i] = c[i] = t[i] = f2(g(rng), g(rng));
            run(U, a);
            run(F, c);
            TProgram FT = F;
            plan_tiles(FT, 12, 1);
            run(FT, t);
            double num = 0, numt = 0, den = 0;
            for (uint32_t i = 0; i < N; ++i) {
                num = std::max(num, double(std::abs(a[i] - c[i])));
                numt = std::max(numt, double(std::abs(c[i] - t[i])));
                den = std::max(den, double(std::abs(a[i])));
            }
            EXPECT(num <= 1e-4 * den);
            EXPECT(numt == 0.0); // tiling reorders nothing
        }
        const uint32_t N = 1u << n;
        std::vector<f2> x0(N);
        for (auto& v : x0) v = f2(g(rng), g(rng));
        std::vector<f2> ref = x0;
        run(U, ref);
        for (int mode = 0; mode < 4; ++mode) {
            const int T = mode == 3 ? 12 : (mode == 0 ? 9 : (mode == 1 ? 12 : 14));
            const size_t min_run = mode == 3 ? 1 : 2; // 1: every gate in a pass
            if (T >= n) continue;
            TProgram Q = U;
            plan_tiles(Q, T, min_run);
            size_t headers = 0, inner = 0;
            for (size_t k = 0; k < Q.ins.size(); ++k)
                if (Q.ins[k].op == kTTile) {
                    ++headers;
                    inner += Q.ins[k].cmask;
                    EXPECT(Q.ins[k].cmask >= min_run);
                }
            EXPECT(Q.ins.size() == U.ins.size() + headers);
            EXPECT(headers > 0);
            if (min_run == 1) { // every gate inside a pass
                size_t gates = 0;
                for (const auto& I : U.ins) gates += I.op != kTMeas;
                EXPECT(inner == gates);
            }
            std::vector<f2> got = x0;
            run(Q, got);
            EXPECT(std::memcmp(got.data(), ref.data(), N * sizeof(f2)) == 0);
            // untiled index of every instruction: position minus headers so
            // far (the kernel's noise / measurement counter)
            size_t nh = 0;
            for (size_t k = 0; k < Q.ins.size(); ++k) {
                if (Q.ins[k].op == kTTile) {
                    ++nh;
                    for (uint32_t j = 1; j <= Q.ins[k].cmask; ++j)
                        EXPECT(Q.ins[k + j].flags == U.ins[k + j - nh].flags &&
                               Q.ins[k + j].op == U.ins[k + j - nh].op &&
                               Q.ins[k + j].mat == U.ins[k + j - nh].mat);
                    k += Q.ins[k].cmask;
                } else {
                    EXPECT(std::memcmp(&Q.ins[k], &U.ins[k - nh], sizeof(TInstr)) == 0);
                }
            }
        }
    }
    std::printf(fails ? "tiles FAILED (%d)\n" : "tiles ok\n", fails);
    return fails ? 1 : 0;
}
