// CPU check of the QFT pass plans behind qgpu_apply_qft (qgpu::plan_qft) and
// of the arithmetic of k_qft_pass: a host model of the kernel (same tables,
// tile loop, step order and phases, in FP64) runs every pass of the plan,
// and the result must equal the transform's definition within 1e-12:
//   QFT with swap = the DFT on the register spelled by the targets
//   (target[0] most significant): out[y] = sum_x w^(x y) in[x] / sqrt(N),
//   w = exp(2 pi i / N), N = d^k; without swap the output digits are then
//   reversed; TFQ is the adjoint. A density matrix gets U rho U^dagger.
// It also checks that each pass reads and writes inside the state and writes
// every element exactly once, and that the shared memory fits.
// Built and run by tests/test_qft_plan.py.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <random>
#include <vector>

#include "kernels.hpp"
#include "ops.hpp"

using namespace qgpu;
using cdd = std::complex<double>;

static int fails = 0;
#define EXPECT(c)                                                                     \
    do {                                                                              \
        if (!(c)) {                                                                   \
            if (fails < 20) std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c); \
            ++fails;                                                                  \
        }                                                                             \
    } while (0)

static uint64_t order_sum(const QftPlan& p, uint32_t idx, bool write_order, int what) {
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

static size_t max_smem = 0;

// Host model of one k_qft_pass launch (kernels_qft.cu), FP64.
static void run_pass(const QftPlan& p, size_t eb, const std::vector<cdd>& Wg,
                     const std::vector<cdd>& F, const std::vector<cdd>& in,
                     std::vector<cdd>& out) {
    const bool QB = p.d == 2;
    EXPECT(p.Glo && p.Flo && p.E / p.Glo <= 256 && p.Glo <= 256 && p.E / p.Flo <= 256 &&
           p.Flo <= 256);
    EXPECT(p.E * eb <= 32768);
    EXPECT(p.nW == Wg.size());
    for (int q = 0; q < p.nr; ++q) EXPECT((p.tzw[q] != 0) == (q < p.nz));
    max_smem = std::max(max_smem, qft_smem_bytes(p, eb));
    // two CTAs per SM (the kernel's launch bounds)
    EXPECT(qft_smem_bytes(p, eb) <= 110 * 1024);
    const uint32_t Glo = p.Glo, Flo = p.Flo;
    std::vector<uint64_t> goff_lo(Glo), goff_hi(p.E / Glo), woff_lo(Flo), woff_hi(p.E / Flo);
    std::vector<uint32_t> ge_lo(Glo), ge_hi(p.E / Glo), we_lo(Flo), we_hi(p.E / Flo);
    for (uint32_t i = 0; i < Glo; ++i) {
        goff_lo[i] = order_sum(p, i, false, 0);
        ge_lo[i] = uint32_t(order_sum(p, i, false, 2));
    }
    for (uint32_t i = 0; i < p.E / Glo; ++i) {
        goff_hi[i] = order_sum(p, i * Glo, false, 0);
        ge_hi[i] = uint32_t(order_sum(p, i * Glo, false, 2));
    }
    for (uint32_t i = 0; i < Flo; ++i) {
        woff_lo[i] = order_sum(p, i, true, 1);
        we_lo[i] = uint32_t(order_sum(p, i, true, 2));
    }
    for (uint32_t i = 0; i < p.E / Flo; ++i) {
        woff_hi[i] = order_sum(p, i * Flo, true, 1);
        we_hi[i] = uint32_t(order_sum(p, i * Flo, true, 2));
    }
    std::vector<cdd> W(p.nW);
    for (uint32_t i = 0; i < p.nW; ++i) W[i] = p.sigma < 0 ? std::conj(Wg[i]) : Wg[i];
    std::vector<int> written(out.size(), 0), loaded(p.E);
    const int M = p.M, d = p.d;
    const uint32_t Rs = p.Rsize, CZ = p.CZ, ncst = uint32_t(M) * d * CZ;
    std::vector<cdd> tile(p.E), cst(ncst);
    // qubits: the kernel's per-block table T[j][c] and per-tile bases B[j]
    std::vector<cdd> Tq(size_t(M) * CZ), Bq(static_cast<size_t>(M));
    if (QB)
        for (uint32_t i = 0; i < uint32_t(M) * CZ; ++i) {
            const uint32_t c = i % CZ;
            const int j = int(i / CZ);
            uint64_t zz = 0;
            for (int q = 0; q < p.nz; ++q) zz += uint64_t((c >> q) & 1u) * p.tzw[q];
            const double x = std::ldexp(double(zz), 1 - (p.k - p.a - j));
            Tq[i] = cdd(std::cos(M_PI * x), p.sigma * std::sin(M_PI * x));
        }
    for (uint64_t t = 0; t < p.ntiles; ++t) {
        uint64_t rb = 0, wb = 0, z = 0;
        for (int q = 0; q < p.nod; ++q) {
            const uint64_t dg = p.pow2 ? (t >> p.oshift[q]) & (p.odim[q] - 1)
                                       : (t / p.opitch[q]) % p.odim[q];
            rb += dg * p.ors[q];
            wb += dg * p.ows[q];
            z += dg * p.ozw[q];
        }
        for (uint32_t i = 0; i < ncst; ++i) {
            const uint32_t c = i % CZ, jr = i / CZ;
            const int j = int(jr) / d, r = int(jr) % d;
            uint64_t zz = z;
            for (int q = 0; q < p.nz; ++q) zz += uint64_t((c / p.tpitch[q]) % p.tdim[q]) * p.tzw[q];
            const uint64_t N = p.dpow[p.k - p.a - j];
            EXPECT(uint64_t(r) * zz < N || r == 0);
            const double x = 2.0 * (double(uint64_t(r) * zz) / double(N));
            cst[i] = cdd(std::cos(M_PI * x), p.sigma * std::sin(M_PI * x));
        }
        if (QB)
            for (int j = 0; j < M; ++j) {
                const double x = std::ldexp(double(z), 1 - (p.k - p.a - j));
                Bq[size_t(j)] = cdd(std::cos(M_PI * x), p.sigma * std::sin(M_PI * x));
            }
        std::fill(loaded.begin(), loaded.end(), 0);
        for (uint32_t g = 0; g < p.E; ++g) {
            const uint32_t lo = QB ? (g & (Glo - 1)) : g % Glo;
            const uint32_t hi = QB ? (g >> p.glo_shift) : g / Glo;
            const uint32_t e = ge_lo[lo] + ge_hi[hi];
            const uint64_t a = rb + goff_lo[lo] + goff_hi[hi];
            EXPECT(a < in.size() && e < p.E);
            if (a < in.size() && e < p.E) {
                tile[e] = in[a];
                loaded[e]++;
            }
        }
        for (int x : loaded) EXPECT(x == 1);
        if (QB) {
            // the kernel's rounds of up to three steps (qubit_round)
            for (int s0 = 0; s0 < M; s0 += 3) {
                const int G = M - s0 < 3 ? M - s0 : 3;
                const bool INV = p.inverse;
                const int jf = INV ? M - 1 - s0 : s0;
                const int jlow = INV ? jf : jf + G - 1;
                const int lo = p.nr + M - 1 - jlow;
                const uint32_t lom = (1u << lo) - 1;
                std::vector<int> touched(p.E, 0);
                for (uint32_t q = 0; q < (p.E >> G); ++q) {
                    const uint32_t eb = ((q & ~lom) << G) | (q & lom);
                    const cdd* cc = Tq.data() + (eb & (CZ - 1));
                    cdd v[8];
                    for (int m = 0; m < (1 << G); ++m) {
                        const uint32_t e = eb | (uint32_t(m) << lo);
                        EXPECT(e < p.E);
                        v[m] = tile[e];
                        touched[e]++;
                    }
                    for (int u = 0; u < G; ++u) {
                        const int j = INV ? jf - u : jf + u;
                        const int rel = INV ? u : G - 1 - u;
                        EXPECT(p.nr + M - 1 - j == lo + rel);
                        const uint32_t Lmask = (1u << (M - 1 - j)) - 1;
                        const cdd cj = Bq[size_t(j)] * cc[size_t(j) * CZ];
                        EXPECT(std::abs(cj - cst[size_t(j * 2 + 1) * CZ + (eb & (CZ - 1))]) < 1e-14);
                        for (int m = 0; m < (1 << G); ++m) {
                            if ((m >> rel) & 1) continue;
                            const int m1 = m | (1 << rel);
                            // the kernel's per-round phase: round bits below rel
                            const uint32_t lb = uint32_t(m) & ((1u << rel) - 1);
                            const uint32_t L = ((eb >> p.nr) + (lb << (lo - p.nr))) & Lmask;
                            EXPECT(L == (((eb | (uint32_t(m) << lo)) >> p.nr) & Lmask));
                            const uint64_t wi = uint64_t(L << j) * p.wmul;
                            EXPECT(wi < W.size());
                            const cdd ph = W[wi] * cj;
                            if (!INV) {
                                const cdd x = v[m], y = v[m1];
                                v[m] = x + y;
                                v[m1] = (x - y) * ph;
                            } else {
                                const cdd x = v[m], y = v[m1] * ph;
                                v[m] = x + y;
                                v[m1] = x - y;
                            }
                        }
                    }
                    for (int m = 0; m < (1 << G); ++m) tile[eb | (uint32_t(m) << lo)] = v[m];
                }
                for (int x : touched) EXPECT(x == 1);
            }
        } else {
        for (int s = 0; s < M; ++s) {
            const int j = p.inverse ? M - 1 - s : s;
            {
                const uint32_t pj = Rs * uint32_t(p.dpow[M - 1 - j]);
                const uint64_t Ld = p.dpow[M - 1 - j], dj = p.dpow[j];
                for (uint32_t fb = 0; fb < p.E / d; ++fb) {
                    const uint32_t hi = fb / pj, lo = fb - hi * pj;
                    const uint32_t e0 = hi * pj * d + lo;
                    const uint64_t L = (e0 / Rs) % Ld;
                    const uint32_t c = e0 % CZ;
                    cdd v[kQftMaxD], o[kQftMaxD];
                    for (int r = 0; r < d; ++r) v[r] = tile[e0 + r * pj];
                    auto phase = [&](int r) {
                        const uint64_t wi = (uint64_t(r) * L * dj) * p.wmul;
                        EXPECT(wi < W.size());
                        return W[wi] * cst[(size_t(j) * d + r) * CZ + c];
                    };
                    if (p.inverse)
                        for (int r = 1; r < d; ++r) v[r] *= phase(r);
                    for (int x = 0; x < d; ++x) {
                        cdd acc = 0;
                        for (int y = 0; y < d; ++y) acc += F[x + y * d] * v[y];
                        o[x] = acc;
                    }
                    if (!p.inverse)
                        for (int r = 1; r < d; ++r) o[r] *= phase(r);
                    for (int r = 0; r < d; ++r) tile[e0 + r * pj] = o[r];
                }
            }
        }
        }
        for (uint32_t f = 0; f < p.E; ++f) {
            const uint32_t lo = QB ? (f & (Flo - 1)) : f % Flo;
            const uint32_t hi = QB ? (f >> p.flo_shift) : f / Flo;
            const uint32_t e = we_lo[lo] + we_hi[hi];
            EXPECT(e < p.E);
            const uint64_t a = wb + woff_lo[lo] + woff_hi[hi];
            EXPECT(a < out.size());
            if (a < out.size() && e < p.E) {
                out[a] = tile[e] * (QB ? p.scale : 1.0);
                written[a]++;
            }
        }
    }
    for (int w : written) EXPECT(w == 1);
}

// The transform's definition on virtual digits vt (all of dimension d) of a
// vector over nv digits; conj_u applies conj(U) instead of U.
static void reference(std::vector<cdd>& v, size_t nv, uint64_t d, const std::vector<size_t>& vt,
                      bool swap, bool inverse, bool conj_u) {
    const size_t k = vt.size();
    uint64_t N = 1;
    for (size_t i = 0; i < k; ++i) N *= d;
    std::vector<uint64_t> stride(nv);
    uint64_t s = 1;
    for (size_t q = nv; q-- > 0;) {
        stride[q] = s;
        s *= d;
    }
    std::vector<char> is_t(nv, 0);
    for (size_t t : vt) is_t[t] = 1;
    auto reg_off = [&](uint64_t x) { // offset of register value x
        uint64_t o = 0;
        for (size_t a = k; a-- > 0;) {
            o += (x % d) * stride[vt[a]];
            x /= d;
        }
        return o;
    };
    auto rev = [&](uint64_t x) {
        uint64_t r = 0;
        for (size_t a = 0; a < k; ++a) {
            r = r * d + x % d;
            x /= d;
        }
        return r;
    };
    const double sgn = (inverse ? -1.0 : 1.0) * (conj_u ? -1.0 : 1.0);
    std::vector<cdd> root(N);
    for (uint64_t e = 0; e < N; ++e) root[e] = std::polar(1.0, sgn * 2.0 * M_PI * double(e) / double(N));
    std::vector<cdd> reg(N), res(N);
    for (uint64_t base = 0; base < v.size(); ++base) {
        bool zero = true; // bases with every target digit 0
        for (size_t q = 0; q < nv; ++q)
            if (is_t[q] && (base / stride[q]) % d) zero = false;
        if (!zero) continue;
        for (uint64_t x = 0; x < N; ++x) reg[x] = v[base + reg_off(x)];
        if (inverse && !swap) {
            std::vector<cdd> t(N);
            for (uint64_t x = 0; x < N; ++x) t[rev(x)] = reg[x];
            reg = t;
        }
        for (uint64_t y = 0; y < N; ++y) {
            cdd acc = 0;
            for (uint64_t x = 0; x < N; ++x) {
                acc += root[(x * y) % N] * reg[x];
            }
            res[y] = acc / std::sqrt(double(N));
        }
        if (!inverse && !swap) {
            std::vector<cdd> t(N);
            for (uint64_t x = 0; x < N; ++x) t[rev(x)] = res[x];
            res = t;
        }
        for (uint64_t y = 0; y < N; ++y) v[base + reg_off(y)] = res[y];
    }
}

static double check_case(bool rho, size_t n, uint64_t d, const std::vector<uint64_t>& target,
                         bool swap, bool inverse, size_t eb, std::mt19937_64& rng) {
    uint64_t D = 1;
    for (size_t i = 0; i < n; ++i) D *= d;
    const uint64_t elems = rho ? D * D : D;
    std::normal_distribution<double> g;
    std::vector<cdd> v(elems);
    for (auto& x : v) x = cdd(g(rng), g(rng));
    std::vector<cdd> ref = v;
    if (!rho) {
        std::vector<size_t> vt(target.begin(), target.end());
        reference(ref, n, d, vt, swap, inverse, false);
    } else {
        std::vector<size_t> rows, cols;
        for (uint64_t t : target) {
            rows.push_back(n + t);
            cols.push_back(t);
        }
        reference(ref, 2 * n, d, rows, swap, inverse, false);
        reference(ref, 2 * n, d, cols, swap, inverse, true);
    }
    const bool rev = swap && target.size() >= 2;
    QftSchedule S;
    const bool ok = plan_qft(rho, D, d, eb, target, inverse, rev, S);
    EXPECT(ok);
    if (!ok) return 1e300;
    int nfold = 0;
    for (char f : S.fold) nfold += f;
    EXPECT(nfold == (rev ? 1 : 0));
    const std::vector<cdd> W = qft_roots(S.nW);
    const std::vector<cdd> Fd = fourier_gate(d);
    std::vector<cdd> Fc(Fd.size());
    for (size_t i = 0; i < Fd.size(); ++i) Fc[i] = std::conj(Fd[i]);
    std::vector<cdd> cur = v, other(elems);
    for (size_t i = 0; i < S.plans.size(); ++i) {
        const QftPlan& p = S.plans[i];
        EXPECT(p.ntiles * p.E == elems);
        const std::vector<cdd>& F = p.sigma > 0 ? Fd : Fc;
        if (S.fold[i]) {
            run_pass(p, eb, W, F, cur, other);
            std::swap(cur, other);
        } else {
            std::vector<cdd> tmp(elems);
            run_pass(p, eb, W, F, cur, tmp);
            cur.swap(tmp);
        }
    }
    double num = 0, den = 0;
    for (uint64_t i = 0; i < elems; ++i) {
        num = std::max(num, std::abs(cur[i] - ref[i]));
        den = std::max(den, std::abs(ref[i]));
    }
    return num / den;
}

int main() {
    std::mt19937_64 rng(12345);
    int cases = 0;
    double worst = 0;
    struct Cfg {
        bool rho;
        size_t n;
        uint64_t d;
    };
    std::vector<Cfg> cfgs = {{false, 1, 2},  {false, 2, 2}, {false, 5, 2},  {false, 9, 2},
                             {false, 12, 2}, {false, 14, 2}, {false, 3, 3}, {false, 6, 3},
                             {false, 4, 4},  {false, 3, 5}, {false, 2, 16}, {true, 1, 2},
                             {true, 3, 2},   {true, 5, 2},  {true, 6, 2},   {true, 2, 3},
                             {true, 3, 3}};
    for (const Cfg& c : cfgs) {
        for (int rep = 0; rep < 6; ++rep) {
            // random target subset in random order (all digits on rep 0)
            std::vector<uint64_t> all(c.n);
            for (size_t i = 0; i < c.n; ++i) all[i] = i;
            std::shuffle(all.begin(), all.end(), rng);
            size_t k = rep == 0 ? c.n : 1 + rng() % c.n;
            if (rep == 0) std::sort(all.begin(), all.end());
            std::vector<uint64_t> t(all.begin(), all.begin() + long(k));
            const bool swap = rep % 3 != 2, inverse = rep % 2 == 1;
            for (size_t eb : {size_t(16), size_t(8)}) {
                double e = check_case(c.rho, c.n, c.d, t, swap, inverse, eb, rng);
                worst = std::max(worst, e);
                if (e > 1e-12 && fails < 20) {
                    std::printf("FAIL rho=%d n=%zu d=%llu k=%zu swap=%d inv=%d eb=%zu err=%g\n",
                                int(c.rho), c.n, (unsigned long long)c.d, k, int(swap),
                                int(inverse), eb, e);
                    ++fails;
                }
                ++cases;
            }
        }
    }
    std::printf("%d cases, worst relative error %.3g, shared memory up to %zu B\n", cases,
                worst, max_smem);
    if (fails) return 1;
    std::printf("qft plans ok\n");
    return 0;
}
