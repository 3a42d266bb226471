// qft.cpp -- planning of qpp::applyQFT / applyTFQ onto k_qft_pass.
//
// qpp::applyQFT(A, target, d, swap) (operations.hpp:2565-2676) and applyTFQ
// (:2680-2787) treat A as n qudits of dimension d. On a ket the transform acts
// on the target digits; on a density matrix rho -> U rho U^dagger is U on the
// row digits and conj(U) on the column digits (conj(QFT) is the same step
// sequence with every phase and F conjugated). The targets of a ket, or of
// each half of rho, are cut into groups of at most Mmax consecutive targets,
// one pass each; forward transforms take the groups in increasing order,
// inverse ones in decreasing order. With swap (k >= 2) the target reversal
// is folded into the last pass of a forward transform or the first pass of an
// inverse one, which writes a new buffer. Dimensions above kQftMaxD, or a
// failed allocation of that buffer, take qpp's own gate sequence instead
// (Fd / H, controlled R_j, SWAPd) through the gate kernels.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "kernels.hpp"
#include "ops.hpp"

namespace qgpu {

namespace {
constexpr double kPi = 3.141592653589793238462643383279502884;
} // namespace

std::vector<cd> fourier_gate(uint64_t d) {
    std::vector<cd> F(d * d);
    if (d == 2) {
        const double h = 1.0 / std::sqrt(2.0);
        F = {h, h, h, -h};
        return F;
    }
    const cd omega = std::exp(2.0 * kPi * cd(0, 1) / static_cast<double>(d));
    for (uint64_t j = 0; j < d; ++j)
        for (uint64_t i = 0; i < d; ++i)
            F[i + j * d] = 1.0 / std::sqrt(static_cast<double>(d)) *
                           std::pow(omega, static_cast<double>(i * j));
    return F;
}

std::vector<cd> qft_phase(uint64_t d, size_t j, bool inverse) {
    std::vector<cd> Rj(d * d, 0.0);
    const double sgn = inverse ? -1.0 : 1.0;
    for (uint64_t m = 0; m < d; ++m)
        Rj[m + m * d] = std::exp(sgn * 2.0 * kPi * static_cast<double>(m) * cd(0, 1) /
                                 std::pow(static_cast<double>(d), static_cast<double>(j)));
    return Rj;
}

std::vector<cd> swap_gate(uint64_t d) {
    std::vector<cd> SW(d * d * d * d, 0.0); // |a b> -> |b a>
    for (uint64_t a = 0; a < d; ++a)
        for (uint64_t b = 0; b < d; ++b) SW[(b * d + a) + (a * d + b) * d * d] = 1.0;
    return SW;
}

namespace {

// qpp's gate sequence (operations.hpp:2611-2672, :2722-2784) on the dims
// n x d, through op_apply / op_apply_ctrl.
void qft_gate_sequence(qgpu_state* s, const std::vector<uint64_t>& target, uint64_t d,
                       bool swap, bool inverse, bool do_main, bool do_swap) {
    const size_t k = target.size();
    const std::vector<cd> F = fourier_gate(d);
    std::vector<cd> Fa(d * d); // adjoint
    for (uint64_t i = 0; i < d; ++i)
        for (uint64_t j = 0; j < d; ++j) Fa[i + j * d] = std::conj(F[j + i * d]);
    const std::vector<cd> SW = swap_gate(d);
    const std::vector<uint64_t> noshift(1, 0);
    auto swaps = [&](bool forward) {
        if (!(swap && do_swap)) return;
        if (forward) {
            for (size_t i = 0; i < k / 2; ++i)
                op_apply(s, SW.data(), d * d, {target[i], target[k - i - 1]});
        } else {
            for (size_t i = k / 2; i-- > 0;)
                op_apply(s, SW.data(), d * d, {target[i], target[k - i - 1]});
        }
    };
    if (!inverse) {
        if (do_main)
            for (size_t i = 0; i < k; ++i) {
                op_apply(s, F.data(), d, {target[i]});
                for (size_t j = 2; j <= k - i; ++j) {
                    std::vector<cd> R = qft_phase(d, j, false);
                    op_apply_ctrl(s, R.data(), d, {target[i + j - 1]}, {target[i]}, noshift,
                                  false);
                }
            }
        swaps(true);
    } else {
        swaps(false);
        if (do_main)
            for (size_t i = k; i-- > 0;) {
                for (size_t j = k - i + 1; j-- > 2;) {
                    std::vector<cd> R = qft_phase(d, j, true);
                    op_apply_ctrl(s, R.data(), d, {target[i + j - 1]}, {target[i]}, noshift,
                                  false);
                }
                op_apply(s, Fa.data(), d, {target[i]});
            }
    }
}

struct PassSpec {
    std::vector<int> group; // virtual digits of targets a .. a + M - 1
    int a = 0, M = 0, sigma = 1;
    const std::vector<int>* half = nullptr; // the half's virtual targets
    bool fold = false;
};

// The prefix product p of dims (in order) with p <= 256 and E / p <= 256
// closest to sqrt(E); 0 when there is none.
uint32_t split_prefix(const std::vector<uint32_t>& dims, uint32_t E) {
    uint32_t p = 1, best = 0;
    double bestd = 1e300;
    for (size_t i = 0; i <= dims.size(); ++i) {
        if (p <= 256 && E / p <= 256) {
            double dd = std::fabs(std::log2(double(p)) - 0.5 * std::log2(double(E)));
            if (dd < bestd) {
                bestd = dd;
                best = p;
            }
        }
        if (i < dims.size()) p *= dims[i];
    }
    return best;
}

int log2u(uint64_t x) {
    int s = 0;
    while ((uint64_t(1) << s) < x) ++s;
    return s;
}

// Builds the launch plan of one pass; false when it does not fit the kernel's
// limits (too many tile or outer digits, or tables too large).
bool build_pass(const VSpace& vs, const PassSpec& ps, uint64_t d, size_t k,
                const std::vector<uint64_t>& rs, const std::vector<uint64_t>& ws,
                uint32_t Emax, uint32_t Rt, int Mmax, uint64_t nW, QftPlan& P) {
    std::memset(&P, 0, sizeof(P));
    const size_t N = vs.dims.size();
    std::vector<char> in_tile(N, 0);
    uint64_t E = 1;
    for (int v : ps.group) {
        in_tile[size_t(v)] = 1;
        E *= vs.dims[size_t(v)];
    }
    // run digits: the lowest digits in read order, then in write order, until
    // each order's contiguous run reaches Rt elements
    std::vector<int> run;
    auto add_run = [&](const std::vector<uint64_t>& st) {
        std::vector<int> order(N);
        std::iota(order.begin(), order.end(), 0);
        std::sort(order.begin(), order.end(), [&](int x, int y) { return st[x] < st[y]; });
        uint64_t len = 1;
        for (int v : order) {
            if (len >= Rt || st[size_t(v)] != len) break;
            if (!in_tile[size_t(v)]) {
                if (E * vs.dims[size_t(v)] > Emax) break;
                in_tile[size_t(v)] = 1;
                E *= vs.dims[size_t(v)];
                run.push_back(v);
            }
            len *= vs.dims[size_t(v)];
        }
    };
    add_run(rs);
    add_run(ws);
    std::vector<int> qidx(N, -1); // QFT index of this half's targets
    for (size_t l = 0; l < ps.half->size(); ++l) qidx[size_t((*ps.half)[l])] = int(l);
    const int b = ps.a + ps.M;
    // the step constants are tabulated over the values of the later targets
    // among the run digits (CZ of them): M * d * CZ entries; tile filling
    // keeps that at most 256
    uint64_t CZ = 1;
    for (int v : run)
        if (qidx[size_t(v)] >= b) CZ *= vs.dims[size_t(v)];
    // then the next lowest digits in read order while the tile fits: larger
    // tiles spread the per-tile work over more amplitudes. The step-constant
    // table stays within 256 entries, or 768 for qubits, whose 6-step passes
    // then still fill whole tiles (k_qft_pass8)
    const uint64_t cz_cap = d == 2 ? 768 : 256;
    {
        std::vector<int> order(N);
        std::iota(order.begin(), order.end(), 0);
        std::sort(order.begin(), order.end(), [&](int x, int y) { return rs[x] < rs[y]; });
        for (int v : order) {
            if (in_tile[size_t(v)]) continue;
            const uint64_t dim = vs.dims[size_t(v)];
            if (E * dim > Emax) break;
            const bool later = qidx[size_t(v)] >= b;
            if (later && uint64_t(ps.M) * d * CZ * dim > cz_cap) break;
            if (later) CZ *= dim;
            in_tile[size_t(v)] = 1;
            E *= dim;
            run.push_back(v);
        }
    }
    // run digits: the later targets first (lowest tile index digits), each
    // part by read stride
    std::sort(run.begin(), run.end(), [&](int x, int y) {
        const bool lx = qidx[size_t(x)] >= b, ly = qidx[size_t(y)] >= b;
        if (lx != ly) return lx;
        return rs[x] < rs[y];
    });
    auto zweight = [&](int l) {
        uint64_t w = 1;
        for (size_t e = 0; e + 1 + size_t(l) < k; ++e) w *= d; // d^(k-1-l)
        return w;
    };

    // tile order: run digits, then group steps M - 1 .. 0
    std::vector<int> tdig = run;
    for (int j = ps.M; j-- > 0;) tdig.push_back(ps.group[size_t(j)]);
    if (tdig.size() > size_t(kQftMaxTile)) return false;
    P.ntd = int(tdig.size());
    P.nr = int(run.size());
    P.E = uint32_t(E);
    uint32_t pitch = 1;
    for (int q = 0; q < P.ntd; ++q) {
        const size_t v = size_t(tdig[size_t(q)]);
        P.tdim[q] = uint32_t(vs.dims[v]);
        P.tpitch[q] = pitch;
        pitch *= P.tdim[q];
        P.trs[q] = rs[v];
        P.tws[q] = ws[v];
        const int l = qidx[v];
        P.tzw[q] = (q < P.nr && l >= b) ? zweight(l) : 0;
        if (P.tzw[q]) ++P.nz;
    }
    P.Rsize = P.nr > 0 ? P.tpitch[P.nr - 1] * P.tdim[P.nr - 1] : 1;
    P.CZ = P.nz > 0 ? P.tpitch[P.nz - 1] * P.tdim[P.nz - 1] : 1;
    if (size_t(ps.M) * d * P.CZ > 1024) return false; // the run digits alone stay within this
    // memory orders of the tile digits
    auto order_of = [&](const uint64_t* st, int* perm, uint32_t* mp) {
        std::vector<int> o(size_t(P.ntd));
        std::iota(o.begin(), o.end(), 0);
        std::sort(o.begin(), o.end(), [&](int x, int y) { return st[x] < st[y]; });
        std::vector<uint32_t> dims;
        uint32_t pp = 1;
        for (int q = 0; q < P.ntd; ++q) {
            perm[q] = o[size_t(q)];
            mp[q] = pp;
            pp *= P.tdim[o[size_t(q)]];
            dims.push_back(P.tdim[o[size_t(q)]]);
        }
        return split_prefix(dims, P.E);
    };
    P.Glo = order_of(P.trs, P.rperm, P.rpitch);
    P.Flo = order_of(P.tws, P.wperm, P.wpitch);
    // qubit tiles of 256 to 65536 amplitudes split both orders at the kernel's
    // block size (256 threads): each thread's low table entries stay fixed
    if (d == 2 && P.E >= 256 && P.E / 256 <= 256) P.Glo = P.Flo = 256;
    if (P.Glo == 0 || P.Flo == 0) return false;
    P.glo_shift = log2u(P.Glo);
    P.flo_shift = log2u(P.Flo);

    // outer digits by ascending read stride, merged where read stride, write
    // stride and Z weight all continue
    std::vector<int> od;
    for (size_t v = 0; v < N; ++v)
        if (!in_tile[v]) od.push_back(int(v));
    std::sort(od.begin(), od.end(), [&](int x, int y) { return rs[x] < rs[y]; });
    P.pow2 = (d & (d - 1)) == 0;
    uint64_t opitch = 1;
    P.nod = 0;
    for (int v : od) {
        const uint64_t dim = vs.dims[size_t(v)];
        const int l = qidx[size_t(v)];
        const uint64_t zw = l >= b ? zweight(l) : 0;
        if (P.nod > 0) {
            const int q = P.nod - 1;
            const bool zok = (zw == 0 && P.ozw[q] == 0) || (zw != 0 && zw == P.ozw[q] * P.odim[q]);
            if (rs[size_t(v)] == P.ors[q] * P.odim[q] && ws[size_t(v)] == P.ows[q] * P.odim[q] &&
                zok) {
                P.odim[q] *= dim;
                opitch *= dim;
                continue;
            }
        }
        if (P.nod >= kQftMaxOuter) return false;
        const int q = P.nod++;
        P.odim[q] = dim;
        P.opitch[q] = opitch;
        P.oshift[q] = uint8_t(log2u(opitch));
        P.ors[q] = rs[size_t(v)];
        P.ows[q] = ws[size_t(v)];
        P.ozw[q] = zw;
        opitch *= dim;
    }
    P.ntiles = opitch;
    P.dpow[0] = 1;
    for (size_t e = 1; e <= k && e < 65; ++e) P.dpow[e] = P.dpow[e - 1] * d;
    P.M = ps.M;
    P.a = ps.a;
    P.k = int(k);
    P.d = int(d);
    P.sigma = ps.sigma;
    P.wmul = 1;
    for (int e = ps.M; e < Mmax; ++e) P.wmul *= uint32_t(d);
    P.nW = uint32_t(nW);
    P.scale = d == 2 ? std::ldexp(1.0, -(ps.M / 2)) * ((ps.M & 1) ? 1.0 / std::sqrt(2.0) : 1.0)
                     : 1.0;
    return true;
}

} // namespace

std::vector<cd> qft_roots(uint64_t nW) {
    std::vector<cd> W(nW);
    for (uint64_t e = 0; e < nW; ++e) {
        const double ang = 2.0 * kPi * static_cast<double>(e) / static_cast<double>(nW);
        W[e] = cd(std::cos(ang), std::sin(ang));
    }
    return W;
}

bool plan_qft(bool rho, uint64_t D, uint64_t d, size_t elem_bytes,
              const std::vector<uint64_t>& target, bool inverse, bool fold, QftSchedule& S) {
    S = QftSchedule();
    const size_t k = target.size();
    if (d > uint64_t(kQftMaxD) || d < 2) return false;
    size_t n = 0;
    for (uint64_t x = 1; x < D; x *= d) ++n;
    const std::vector<uint64_t> dims(n, d);
    const VSpace vs = rho ? vspace_rho(dims) : vspace_ket(dims);
    const size_t NV = vs.dims.size();
    const int sg = inverse ? -1 : 1;
    std::vector<std::vector<int>> halves;
    std::vector<int> hsig, vt;
    for (uint64_t t : target) vt.push_back(int(rho ? n + t : t));
    halves.push_back(vt); // kets, or the row digits of rho: U
    hsig.push_back(sg);
    if (rho) {
        vt.clear();
        for (uint64_t t : target) vt.push_back(int(t));
        halves.push_back(vt); // the column digits of rho: conj(U)
        hsig.push_back(-sg);
    }
    // the reversal of every half's targets, as a map of virtual digits
    std::vector<int> revmap(NV);
    std::iota(revmap.begin(), revmap.end(), 0);
    for (auto& h : halves)
        for (size_t a = 0; a < k; ++a) revmap[size_t(h[a])] = h[k - 1 - a];

    const uint32_t Emax = uint32_t(32768 / elem_bytes), Rt = uint32_t(128 / elem_bytes);
    int Mmax = 0;
    for (uint64_t p = d; p * Rt <= Emax; p *= d) ++Mmax;
    if (Mmax == 0) return false;
    S.Mmax = Mmax;
    S.nW = 1;
    for (int e = 0; e < Mmax; ++e) S.nW *= d;
    // groups of consecutive targets; for qubits the partial one (k mod Mmax
    // targets) comes first, so that the pass carrying the reversal (the last
    // forward pass, the first inverse one) is a full one, which the
    // register-round kernel takes: group g covers targets [start(g),
    // start(g + 1))
    const size_t npass_half = (k + size_t(Mmax) - 1) / size_t(Mmax);
    const size_t part = d == 2 ? k % size_t(Mmax) : 0;
    auto start = [&](size_t g) {
        if (g == 0) return size_t(0);
        return std::min(k, (part ? part : size_t(Mmax)) + (g - 1) * size_t(Mmax));
    };
    // (with part = 0 this is g * Mmax, capped at k)
    std::vector<PassSpec> passes;
    for (size_t h = 0; h < halves.size(); ++h) {
        for (size_t gi = 0; gi < npass_half; ++gi) {
            const size_t g = inverse ? npass_half - 1 - gi : gi;
            PassSpec ps;
            ps.a = int(start(g));
            ps.M = int(start(g + 1) - start(g));
            for (int j = 0; j < ps.M; ++j) ps.group.push_back(halves[h][size_t(ps.a + j)]);
            ps.sigma = hsig[h];
            ps.half = &halves[h];
            passes.push_back(ps);
        }
    }
    if (fold && !passes.empty()) (inverse ? passes.front() : passes.back()).fold = true;
    std::vector<uint64_t> nat(vs.strides), perm(NV);
    for (size_t v = 0; v < NV; ++v) perm[v] = nat[size_t(revmap[v])];
    S.plans.resize(passes.size());
    for (size_t i = 0; i < passes.size(); ++i) {
        const PassSpec& ps = passes[i];
        const std::vector<uint64_t>& rs = (ps.fold && inverse) ? perm : nat;
        const std::vector<uint64_t>& ws = (ps.fold && !inverse) ? perm : nat;
        if (!build_pass(vs, ps, d, k, rs, ws, Emax, Rt, Mmax, S.nW, S.plans[i])) return false;
        S.plans[i].inverse = inverse ? 1 : 0;
        S.fold.push_back(ps.fold ? 1 : 0);
    }
    return true;
}

void op_apply_qft(qgpu_state* s, const std::vector<uint64_t>& target, uint64_t d, bool swap,
                  bool inverse) {
    const size_t k = target.size();
    if (k == 0) return;
    // qpp: dims = n copies of d (the state's own dims may group digits)
    size_t n = 0;
    for (uint64_t x = 1; x < s->D; x *= d) ++n;
    const std::vector<uint64_t> saved = s->dims;
    struct Restore {
        qgpu_state* s;
        const std::vector<uint64_t>& dims;
        ~Restore() { s->dims = dims; }
    } restore{s, saved};
    s->dims.assign(n, d);

    const bool rev = swap && k >= 2;
    const bool rho = s->kind == QGPU_RHO;
    const size_t eb = s->elem_bytes();
    QftSchedule S;
    if (!plan_qft(rho, s->D, d, eb, target, inverse, false, S)) {
        qft_gate_sequence(s, target, d, swap, inverse, true, true);
        return;
    }
    // the reversal rides on one pass, which needs a second buffer
    void* other = nullptr;
    if (rev) {
        if (ctx_malloc(s->ctx, &other, s->bytes()) == cudaSuccess) {
            if (!plan_qft(rho, s->D, d, eb, target, inverse, true, S)) {
                cudaFreeAsync(other, s->ctx->stream);
                qft_gate_sequence(s, target, d, swap, inverse, true, true);
                return;
            }
        } else {
            cudaGetLastError();
            other = nullptr;
        }
    }
    // W (the d^Mmax roots of unity) and F / conj(F) in the state precision,
    // staged through the context scratch
    const std::vector<cd> Fd = fourier_gate(d);
    std::vector<cd> tabs = qft_roots(S.nW);
    for (uint64_t i = 0; i < d * d; ++i) tabs.push_back(Fd[i]);
    for (uint64_t i = 0; i < d * d; ++i) tabs.push_back(std::conj(Fd[i]));
    unsigned char* dev = static_cast<unsigned char*>(ctx_scratch(s->ctx, tabs.size() * eb));
    if (s->prec == QGPU_C128) {
        QG_CUDA(cudaMemcpyAsync(dev, tabs.data(), tabs.size() * eb, cudaMemcpyHostToDevice,
                                s->ctx->stream));
    } else {
        std::vector<float> f(2 * tabs.size());
        for (size_t i = 0; i < tabs.size(); ++i) {
            f[2 * i] = float(tabs[i].real());
            f[2 * i + 1] = float(tabs[i].imag());
        }
        QG_CUDA(cudaMemcpyAsync(dev, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice,
                                s->ctx->stream));
    }
    const unsigned char* dW = dev;
    const unsigned char* dF = dev + S.nW * eb;
    const unsigned char* dFc = dev + (S.nW + d * d) * eb;

    if (rev && !other && inverse) qft_gate_sequence(s, target, d, swap, inverse, false, true);
    for (size_t i = 0; i < S.plans.size(); ++i) {
        const void* F = S.plans[i].sigma > 0 ? static_cast<const void*>(dF)
                                             : static_cast<const void*>(dFc);
        if (S.fold[i]) {
            launch_qft_pass(s->ctx, s->prec, s->data, other, S.plans[i], dW, F);
            std::swap(s->data, other);
            cudaFreeAsync(other, s->ctx->stream);
            other = nullptr;
        } else {
            launch_qft_pass(s->ctx, s->prec, s->data, s->data, S.plans[i], dW, F);
        }
    }
    if (rev && !other && !inverse && !std::count(S.fold.begin(), S.fold.end(), 1))
        qft_gate_sequence(s, target, d, swap, inverse, false, true);
}

} // namespace qgpu
