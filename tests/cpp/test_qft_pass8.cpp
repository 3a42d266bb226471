// CPU check of the addressing of the register-round QFT passes
// (k_qft_pass8, kernels_qft.cu) on the plans of whole transforms: for kets
// of 22-30 qubits, complex64 and complex128, forward and inverse, with and
// without the target reversal, every pass the launcher gives to k_qft_pass8
// (all but the pass on the lowest digits of a transform without the
// reversal) must
//  * have one-bit tile digits at tile positions 2^q (position p <-> memory
//    offset sum_b bit_b(p) * stride[b], as the kernel computes it);
//  * cover each tile position exactly once in round A and in round B through
//    the thread-to-base maps (q8a, q8b) and the round bits;
//  * keep the shared-memory swizzle a bijection whose warp accesses in both
//    rounds touch every bank group equally;
//  * read (round A) and write (round B) runs of at least 128 contiguous bytes
//    per warp access;
//  * stay inside the state for every tile.
// Built and run by tests/test_qft_pass8.py.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "kernels.hpp"

using namespace qgpu;

static int fails = 0;
#define EXPECT(c)                                                                     \
    do {                                                                              \
        if (!(c)) {                                                                   \
            if (fails < 20) std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c); \
            ++fails;                                                                  \
        }                                                                             \
    } while (0)

static uint32_t swz(uint32_t e) { return e ^ ((e >> 4) & 15u) ^ ((e >> 8) & 15u); }

static int checked = 0;

static void check_pass(qgpu_prec prec, const QftPlan& p0, bool fold, int n) {
    const void* in = reinterpret_cast<const void*>(uintptr_t(0x1000));
    const void* out = fold ? reinterpret_cast<const void*>(uintptr_t(0x2000)) : in;
    if (!qft_pass8_applies(prec, in, out, p0)) return;
    ++checked;
    const int EB = qft_pass8_tile_bits(prec);
    const size_t elem = prec == QGPU_C64 ? 8 : 16;
    const int NTHR = prec == QGPU_C64 ? 256 : 128;
    QftPlan p = p0;
    qft_pass8_maps(p, EB);
    const int M = p.M, G = M / 2, NR = EB - M, NQ = EB - G;
    const uint32_t E = 1u << EB;
    for (int q = 0; q < p.ntd; ++q) EXPECT(p.tdim[q] == 2 && p.tpitch[q] == (1u << q));
    const int loA = p.inverse ? NR : NR + G, loB = p.inverse ? NR + G : NR;
    auto pos_of = [&](const uint8_t* map, uint32_t qq) {
        uint32_t e = 0;
        for (int i = 0; i < NQ; ++i) e |= ((qq >> i) & 1u) << map[i];
        return e;
    };
    auto off = [&](const uint64_t* st, uint32_t e) {
        uint64_t o = 0;
        for (int b = 0; b < EB; ++b)
            if ((e >> b) & 1u) o += st[b];
        return o;
    };
    // maps: the bits outside each round, each once
    for (int r = 0; r < 2; ++r) {
        const uint8_t* map = r ? p.q8b : p.q8a;
        const int lo = r ? loB : loA;
        std::vector<int> seen(EB, 0);
        for (int i = 0; i < NQ; ++i) {
            EXPECT(map[i] < EB && (map[i] < lo || map[i] >= lo + G));
            if (map[i] < EB) seen[map[i]]++;
        }
        for (int b = 0; b < EB; ++b) EXPECT(seen[b] == ((b >= lo && b < lo + G) ? 0 : 1));
    }
    // coverage of the tile in both rounds
    for (int r = 0; r < 2; ++r) {
        const uint8_t* map = r ? p.q8b : p.q8a;
        const int lo = r ? loB : loA;
        std::vector<int> hit(E, 0);
        for (uint32_t qq = 0; qq < (1u << NQ); ++qq)
            for (uint32_t m = 0; m < (1u << G); ++m) hit[pos_of(map, qq) | (m << lo)]++;
        for (uint32_t e = 0; e < E; ++e) EXPECT(hit[e] == 1);
    }
    // swizzle: a bijection; each warp access spreads over the bank groups
    {
        std::vector<int> hit(E, 0);
        for (uint32_t e = 0; e < E; ++e) hit[swz(e)]++;
        for (uint32_t e = 0; e < E; ++e) EXPECT(hit[e] == 1);
        const uint32_t groups = uint32_t(128 / elem), best = 32 / groups;
        for (int r = 0; r < 2; ++r) {
            const uint8_t* map = r ? p.q8b : p.q8a;
            const int lo = r ? loB : loA;
            for (uint32_t w0 = 0; w0 < (1u << NQ); w0 += 32)
                for (uint32_t m = 0; m < (1u << G); ++m) {
                    std::vector<uint32_t> cnt(groups, 0);
                    for (uint32_t l = 0; l < 32; ++l)
                        cnt[swz(pos_of(map, w0 + l) | (m << lo)) % groups]++;
                    for (uint32_t g = 0; g < groups; ++g) EXPECT(cnt[g] == best);
                }
        }
    }
    // contiguous runs of >= 128 bytes per warp access: the first 128 / elem
    // lanes of each warp read (round A) and write (round B) consecutive
    // elements
    {
        const uint32_t run = uint32_t(128 / elem);
        for (int r = 0; r < 2; ++r) {
            const uint8_t* map = r ? p.q8b : p.q8a;
            const uint64_t* st = r ? p.tws : p.trs;
            for (uint32_t w0 = 0; w0 < (1u << NQ); w0 += 32)
                for (uint32_t l = 1; l < run; ++l)
                    EXPECT(off(st, pos_of(map, w0 + l)) == off(st, pos_of(map, w0)) + l);
        }
    }
    // every tile stays inside the state (the outer digits' largest offsets)
    {
        uint64_t rmax = 0, wmax = 0;
        for (int q = 0; q < p.nod; ++q) {
            rmax += (p.odim[q] - 1) * p.ors[q];
            wmax += (p.odim[q] - 1) * p.ows[q];
        }
        const uint64_t D = uint64_t(1) << n;
        EXPECT(rmax + off(p.trs, E - 1) < D);
        EXPECT(wmax + off(p.tws, E - 1) < D);
        EXPECT(p.ntiles * E == D);
    }
    (void)NTHR;
}

int main() {
    for (qgpu_prec prec : {QGPU_C64, QGPU_C128}) {
        const size_t eb = prec == QGPU_C64 ? 8 : 16;
        for (int n : {22, 24, 26, 27, 30})
            for (int inverse = 0; inverse < 2; ++inverse)
                for (int fold = 0; fold < 2; ++fold) {
                    std::vector<uint64_t> t(static_cast<size_t>(n));
                    for (int i = 0; i < n; ++i) t[size_t(i)] = uint64_t(i);
                    QftSchedule S;
                    EXPECT(plan_qft(false, uint64_t(1) << n, 2, eb, t, inverse != 0, fold != 0, S));
                    int applied_before = checked;
                    for (size_t i = 0; i < S.plans.size(); ++i)
                        check_pass(prec, S.plans[i], S.fold[i] != 0, n);
                    // whole transforms of >= 22 qubits with the reversal run
                    // every pass of 8 or 6 targets in register rounds (the
                    // partial group of n mod 8 targets otherwise stays with
                    // the shared-memory rounds); without the reversal, the
                    // pass on the lowest digits stays there too
                    int expect = 0;
                    for (const QftPlan& p : S.plans) expect += (p.M == 8 || p.M == 6) ? 1 : 0;
                    if (!fold) --expect;
                    EXPECT(checked - applied_before == expect);
                }
    }
    std::printf("%d passes checked\n", checked);
    std::printf(fails ? "qft pass8 FAILED (%d)\n" : "qft pass8 ok\n", fails);
    return fails ? 1 : 0;
}
