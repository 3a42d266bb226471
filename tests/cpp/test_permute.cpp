// CPU check of the tiled bit permutation behind ptranspose / syspermute
// (qgpu::plan_permute and the addressing of k_permute_tiled): for density
// matrices of 6-9 qubits with random targets / permutations and for kets of
// 11-16 qubits, the kernel's tiles must write every output exactly once,
// read only inside the input, and read for output o the element the plain
// gather reads (the digit formula sum_v digit_v(o) * src[v]).
// Built and run by tests/test_permute.py.
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

#include "kernels.hpp"

using namespace qgpu;

static int fails = 0;
#define EXPECT(c)                                                            \
    do {                                                                     \
        if (!(c)) {                                                          \
            if (fails < 20) std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c); \
            ++fails;                                                         \
        }                                                                    \
    } while (0)

static void check_shape(const std::vector<uint64_t>& od, const std::vector<uint64_t>& src,
                        uint64_t in_count, int tb, int wl) {
    PermPlan P;
    uint64_t count = 1;
    for (uint64_t d : od) count *= d;
    if (count < (uint64_t(2) << tb)) {
        EXPECT(!plan_permute(od, src, 0, P, 16, tb, wl));
        return;
    }
    EXPECT(plan_permute(od, src, 0, P, 16, tb, wl));
    EXPECT((uint64_t(1) << P.nb) == count);
    EXPECT(P.tb == tb && P.nrest == P.nb - P.tb);
    // the wl lowest output bits are in the tile
    for (int j = 0; j < wl; ++j) EXPECT(P.tbits[j] == j);
    const uint32_t NT = 1u << P.tb;
    std::vector<uint64_t> in_off(NT), out_off(NT);
    std::vector<uint32_t> pos_of(NT);
    for (uint32_t l = 0; l < NT; ++l) {
        uint64_t io = 0, oo = 0;
        uint32_t lo = 0;
        for (int j = 0; j < P.tb; ++j)
            if ((l >> j) & 1u) {
                io += P.in_stride[P.tin[j]];
                lo |= 1u << P.tin_pos[j];
                oo |= uint64_t(1) << P.tbits[j];
            }
        in_off[l] = io;
        out_off[l] = oo;
        pos_of[l] = lo;
    }
    // the kernel's split: every offset is a sum (or an OR) over index bits,
    // so the lane's five bits and the rest of a tile index combine exactly
    {
        const uint32_t NH = NT >> 5;
        std::vector<uint64_t> in_lo(32), in_hi(NH), out_lo(32), out_hi(NH);
        std::vector<uint32_t> pos_lo(32), pos_hi(NH);
        for (int h = 0; h < 2; ++h)
            for (uint32_t i = 0; i < (h ? NH : 32u); ++i) {
                uint64_t io = 0, oo = 0;
                uint32_t po = 0;
                for (int j = 0; j < (h ? P.tb - 5 : 5); ++j)
                    if ((i >> j) & 1) {
                        io += P.in_stride[P.tin[5 * h + j]];
                        po |= 1u << P.tin_pos[5 * h + j];
                        oo |= uint64_t(1) << P.tbits[5 * h + j];
                    }
                (h ? in_hi : in_lo)[i] = io;
                (h ? pos_hi : pos_lo)[i] = po;
                (h ? out_hi : out_lo)[i] = oo;
            }
        for (uint32_t l = 0; l < NT; ++l) {
            EXPECT(in_lo[l & 31] + in_hi[l >> 5] == in_off[l]);
            EXPECT((pos_lo[l & 31] | pos_hi[l >> 5]) == pos_of[l]);
            EXPECT((out_lo[l & 31] | out_hi[l >> 5]) == out_off[l]);
        }
        // the tile-position swizzle is a bijection, and every warp access of
        // the kernel touches each bank group equally: 4 wavefronts for 16-byte
        // elements (8 bank groups), 2 for 8-byte ones (16), for the scattered
        // stores in read order (lanes over pos_lo) and the row reads in write
        // order (lanes over positions 0-4)
        for (int eb : {16, 8}) {
            PermPlan Q;
            EXPECT(plan_permute(od, src, 0, Q, eb, tb, wl));
            auto swz = [&](uint32_t p) {
                uint32_t r = 0;
                for (int q = 0; q < Q.tb; ++q)
                    if ((p >> q) & 1u) r ^= Q.swz_bit[q];
                return r;
            };
            std::vector<uint8_t> hit(NT, 0);
            for (uint32_t p = 0; p < NT; ++p) hit[swz(p)]++;
            for (uint8_t x : hit) EXPECT(x == 1);
            const uint32_t groups = eb == 16 ? 8 : 16, best = 32 / groups;
            for (uint32_t h = 0; h < NH; ++h) {
                std::vector<uint32_t> st(groups, 0), rd(groups, 0);
                for (int lane = 0; lane < 32; ++lane) {
                    st[swz(pos_lo[lane] | pos_hi[h]) % groups]++;
                    rd[swz((uint32_t(h) << 5) | uint32_t(lane)) % groups]++;
                }
                for (uint32_t g = 0; g < groups; ++g) EXPECT(st[g] == best && rd[g] == best);
            }
        }
        // tile-number bases: two 7-bit tables plus the remaining bits
        const int r0 = std::min(P.nrest, 7), r1 = std::min(P.nrest - r0, 7);
        for (uint64_t t = 0; t < (uint64_t(1) << P.nrest); t += 1 + (t % 5)) {
            uint64_t bi = 0, bo = 0, ci = 0, co = 0;
            for (int j = 0; j < P.nrest; ++j)
                if ((t >> j) & 1u) {
                    bo |= uint64_t(1) << P.rest[j];
                    bi += P.in_stride[P.rest[j]];
                    if (j < r0 + r1) {
                        co |= uint64_t(1) << P.rest[j];
                        ci += P.in_stride[P.rest[j]];
                    }
                }
            uint64_t ti = 0, to = 0;
            for (int h = 0; h < 2; ++h) {
                const uint64_t x = h ? (t >> r0) & ((uint64_t(1) << r1) - 1) : t & ((uint64_t(1) << r0) - 1);
                const int lo = h ? r0 : 0, cnt = h ? r1 : r0;
                for (int j = 0; j < cnt; ++j)
                    if ((x >> j) & 1) {
                        ti += P.in_stride[P.rest[lo + j]];
                        to |= uint64_t(1) << P.rest[lo + j];
                    }
            }
            EXPECT(ti == ci && to == co);
            (void)bi;
            (void)bo;
        }
    }
    std::vector<uint8_t> written(count, 0);
    for (uint64_t t = 0; t < (uint64_t(1) << P.nrest); ++t) {
        uint64_t bo = 0, bi = P.foff;
        for (int j = 0; j < P.nrest; ++j)
            if ((t >> j) & 1u) {
                bo |= uint64_t(1) << P.rest[j];
                bi += P.in_stride[P.rest[j]];
            }
        for (uint32_t l = 0; l < NT; ++l) {
            const uint64_t ia = bi + in_off[l];
            const uint64_t oa = bo + out_off[pos_of[l]];
            EXPECT(ia < in_count && oa < count);
            if (oa >= count) continue;
            EXPECT(written[oa] == 0);
            written[oa] = 1;
            // the plain gather's source of output oa
            uint64_t r = oa, want = 0;
            for (size_t v = od.size(); v-- > 0;) {
                want += (r % od[v]) * src[v];
                r /= od[v];
            }
            EXPECT(ia == want);
        }
    }
    for (uint64_t o = 0; o < count; ++o) EXPECT(written[o] == 1);
}

// the tile shapes the kernel supports: 10 bits with the 5 lowest output
// bits (the launcher's), and wider tiles that keep more of them
static void check(const std::vector<uint64_t>& od, const std::vector<uint64_t>& src,
                  uint64_t in_count) {
    const int shapes[][2] = {{10, 5}, {10, 7}, {11, 6}, {12, 7}, {12, 5}};
    for (const auto& sh : shapes) check_shape(od, src, in_count, sh[0], sh[1]);
}

int main() {
    std::mt19937 rng(7);
    for (int trial = 0; trial < 12; ++trial) {
        const int n = 6 + trial % 4; // density matrices of 6..9 qubits
        const uint64_t D = uint64_t(1) << n;
        std::vector<uint64_t> strides(n);
        for (int q = 0; q < n; ++q) strides[q] = uint64_t(1) << (n - 1 - q);
        // syspermute: out column digits then row digits, permuted
        std::vector<uint64_t> perm(n);
        for (int q = 0; q < n; ++q) perm[q] = uint64_t(q);
        std::shuffle(perm.begin(), perm.end(), rng);
        std::vector<uint64_t> od, sa;
        for (int q = 0; q < n; ++q) {
            od.push_back(2);
            sa.push_back(strides[perm[q]] * D);
        }
        for (int q = 0; q < n; ++q) {
            od.push_back(2);
            sa.push_back(strides[perm[q]]);
        }
        check(od, sa, D * D);
        // ptranspose over a random subset
        std::vector<char> inT(n);
        for (auto& x : inT) x = char(rng() & 1u);
        od.clear();
        sa.clear();
        for (int q = 0; q < n; ++q) {
            od.push_back(2);
            sa.push_back(inT[q] ? strides[q] : strides[q] * D);
        }
        for (int q = 0; q < n; ++q) {
            od.push_back(2);
            sa.push_back(inT[q] ? strides[q] * D : strides[q]);
        }
        check(od, sa, D * D);
    }
    for (int n = 11; n <= 16; ++n) { // ket syspermute, mixed power-of-two dims
        std::vector<uint64_t> dims;
        int bits = 0;
        while (bits < n) {
            const int b = (bits + 2 <= n && (rng() & 1u)) ? 2 : 1;
            dims.push_back(uint64_t(1) << b);
            bits += b;
        }
        const size_t m = dims.size();
        std::vector<uint64_t> st(m);
        uint64_t s = 1;
        for (size_t q = m; q-- > 0;) {
            st[q] = s;
            s *= dims[q];
        }
        std::vector<uint64_t> perm(m);
        for (size_t q = 0; q < m; ++q) perm[q] = q;
        std::shuffle(perm.begin(), perm.end(), rng);
        std::vector<uint64_t> od, sa;
        for (size_t q = 0; q < m; ++q) {
            od.push_back(dims[perm[q]]);
            sa.push_back(st[perm[q]]);
        }
        check(od, sa, s);
    }
    // not applicable: a qutrit, or too few bits
    PermPlan P;
    EXPECT(!plan_permute({3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2}, {1, 3, 6, 12, 24, 48, 96, 192, 384, 768, 1536}, 0, P));
    EXPECT(!plan_permute({2, 2, 2}, {1, 2, 4}, 0, P));
    std::printf(fails ? "permute FAILED (%d)\n" : "permute ok\n", fails);
    return fails ? 1 : 0;
}
