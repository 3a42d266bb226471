// traj.cpp -- compile qgpu_circuit steps into shared-memory trajectory
// programs, and run all shots of one request in one launch.
#include "traj.hpp"

#include <algorithm>
#include <array>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "capi_common.hpp"
#include "circuit.hpp"

namespace qgpu {

uint32_t MatPool::add(const std::vector<cd>& U) {
    std::string key(U.size() * 2 * sizeof(float), '\0');
    float* k = reinterpret_cast<float*>(&key[0]);
    for (size_t i = 0; i < U.size(); ++i) {
        k[2 * i] = float(U[i].real());
        k[2 * i + 1] = float(U[i].imag());
    }
    auto it = seen.find(key);
    if (it != seen.end()) return it->second;
    // every matrix starts on a 16-byte boundary (two complex64 entries), so
    // that a kernel may read adjacent rows as one float4
    while (P.mats.size() % 4) P.mats.push_back(0.f);
    const uint32_t off = uint32_t(P.mats.size() / 2);
    P.mats.insert(P.mats.end(), k, k + 2 * U.size());
    seen.emplace(std::move(key), off);
    return off;
}

// false when the circuit needs a step the kernel does not execute (gates on
// more than two qubits, controlled multi-qubit gates, classical control) or
// the register does not fit shared memory.
bool compile_traj(const qgpu_circuit* c, TProgram& P) {
    if (c->d != 2 || c->nq > uint32_t(kTrajMaxGlobalQubits)) return false;
    P = TProgram{};
    P.n = c->nq;
    P.ncreg = c->nc;
    const int n = int(c->nq);
    auto bit = [&](uint64_t q) { return uint8_t(n - 1 - int(q)); };
    MatPool pool(P);
    auto add_mat = [&](const std::vector<cd>& U) { return pool.add(U); };
    for (const Step& s : c->steps) {
        uint8_t first = kTNewStep;
        switch (s.kind) {
            case StepKind::Gate: {
                if (s.target.size() > 2) return false;
                TInstr I{};
                I.op = s.target.size() == 1 ? kTG1 : kTG2;
                I.b0 = bit(s.target[0]);
                I.b1 = s.target.size() == 2 ? bit(s.target[1]) : 0;
                I.flags = first;
                I.mat = add_mat(s.U);
                P.ins.push_back(I);
                break;
            }
            case StepKind::Fan: {
                uint32_t m = add_mat(s.U);
                for (uint64_t t : s.target) {
                    TInstr I{};
                    I.op = kTG1;
                    I.b0 = bit(t);
                    I.flags = first;
                    I.mat = m;
                    P.ins.push_back(I);
                    first = 0;
                }
                break;
            }
            case StepKind::Ctrl:
            case StepKind::CtrlFan: {
                if (s.kind == StepKind::Ctrl && s.target.size() != 1) return false;
                uint32_t cmask = 0, cval = 0;
                for (size_t i = 0; i < s.ctrl.size(); ++i) {
                    uint32_t b = 1u << bit(s.ctrl[i]);
                    uint64_t sh = s.has_shift ? s.shift[i] % 2 : 0;
                    cmask |= b;
                    if (sh == 0) cval |= b; // active on |1> unless shifted
                }
                uint32_t m = add_mat(s.U);
                for (uint64_t t : s.target) {
                    TInstr I{};
                    I.op = kTCG1;
                    I.b0 = bit(t);
                    I.flags = first;
                    I.mat = m;
                    I.cmask = cmask;
                    I.cval = cval;
                    P.ins.push_back(I);
                    first = 0;
                }
                break;
            }
            case StepKind::Measure: {
                for (size_t i = 0; i < s.target.size(); ++i) {
                    TInstr I{};
                    I.op = kTMeas;
                    I.b0 = bit(s.target[i]);
                    I.flags = uint8_t(first | (s.destructive ? kTDestructive : 0));
                    I.mat = uint32_t(s.c_reg + i);
                    P.ins.push_back(I);
                    first = 0;
                }
                break;
            }
            case StepKind::Nop:
                break;
            default:
                return false;
        }
    }
    return true;
}

namespace {

bool tileable(const TInstr& I) {
    return I.op == kTG1 || I.op == kTCG1 || I.op == kTG2 || I.op == kTG3 || I.op == kTG4;
}

// bits an instruction reads or writes (controls included)
uint32_t ins_bits(const TInstr& I) {
    switch (I.op) {
        case kTG1: return 1u << I.b0;
        case kTCG1: return (1u << I.b0) | I.cmask;
        case kTG2: return (1u << I.b0) | (1u << I.b1);
        case kTG3: return (1u << I.b0) | (1u << I.b1) | (1u << (I.cmask & 255u));
        case kTG4:
            return (1u << I.b0) | (1u << I.b1) | (1u << (I.cmask & 255u)) |
                   (1u << ((I.cmask >> 8) & 255u));
        default: return 0;
    }
}

} // namespace

void fold_1q_gates(TProgram& P) {
    using C = std::complex<double>;
    using M2 = std::array<C, 4>;
    using M4 = std::array<C, 16>;
    auto ld = [&](uint32_t off, C* m, int count) {
        for (int i = 0; i < count; ++i)
            m[i] = C(P.mats[2 * (size_t(off) + i)], P.mats[2 * (size_t(off) + i) + 1]);
    };
    MatPool pool(P);
    auto store = [&](const C* m, int count) {
        return pool.add(std::vector<C>(m, m + count));
    };
    std::vector<TInstr> out;
    out.reserve(P.ins.size());
    M2 g1[32];
    int pending[32];
    std::fill(pending, pending + 32, -1);
    auto flush = [&](uint32_t bits) {
        for (int b = 0; b < 32; ++b)
            if ((bits >> b & 1u) && pending[b] >= 0) {
                out[pending[b]].mat = store(g1[b].data(), 4);
                pending[b] = -1;
            }
    };
    for (const TInstr& I : P.ins) {
        if (I.op == kTG1) {
            const int b = I.b0;
            M2 G;
            ld(I.mat, G.data(), 4);
            if (pending[b] >= 0) { // the later gate acts second: G * g1
                const M2 A = g1[b];
                for (int r = 0; r < 2; ++r)
                    for (int c = 0; c < 2; ++c)
                        g1[b][r + 2 * c] = G[r] * A[2 * c] + G[r + 2] * A[1 + 2 * c];
            } else {
                pending[b] = int(out.size());
                g1[b] = G;
                out.push_back(I);
            }
        } else if (I.op == kTG2) {
            M4 M;
            ld(I.mat, M.data(), 16);
            for (int side = 0; side < 2; ++side) {
                const int b = side == 0 ? I.b0 : I.b1;
                if (pending[b] < 0) continue;
                // M * (G on the row index's high bit (side 0) or low bit)
                const M2& G = g1[b];
                M4 R;
                for (int r = 0; r < 4; ++r)
                    for (int c = 0; c < 4; ++c) {
                        C acc = 0.0;
                        for (int k = 0; k < 4; ++k) {
                            const bool hi = side == 0;
                            const int kh = k >> 1, kl = k & 1, ch = c >> 1, cl = c & 1;
                            C lk = hi ? (kl == cl ? G[kh + 2 * ch] : C(0.0))
                                      : (kh == ch ? G[kl + 2 * cl] : C(0.0));
                            acc += M[r + 4 * k] * lk;
                        }
                        R[r + 4 * c] = acc;
                    }
                M = R;
                out[pending[b]].op = 0; // folded into this gate
                pending[b] = -1;
            }
            TInstr J = I;
            J.mat = store(M.data(), 16);
            out.push_back(J);
        } else {
            flush(ins_bits(I) | (I.op == kTMeas ? (1u << I.b0) : 0u) |
                  (I.op == kTTile ? 0xffffffffu : 0u));
            out.push_back(I);
        }
    }
    flush(0xffffffffu);
    std::vector<TInstr> kept;
    kept.reserve(out.size());
    for (const TInstr& I : out)
        if (I.op != 0) kept.push_back(I);
    P.ins.swap(kept);
}

void plan_tiles(TProgram& P, int T, size_t min_run) {
    const int n = int(P.n);
    if (T < 9 || n <= kTrajMaxQubits || T >= n) return;
    const uint32_t low = 31u; // bits 0..4: 32 consecutive amplitudes per tile row
    std::vector<TInstr> out;
    out.reserve(P.ins.size() + P.ins.size() / 4 + 1);
    size_t i = 0;
    while (i < P.ins.size()) {
        if (!tileable(P.ins[i])) {
            out.push_back(P.ins[i++]);
            continue;
        }
        // the longest run of gates whose bits outside 0..4 number <= T - 5
        uint32_t S = 0;
        size_t j = i;
        while (j < P.ins.size() && tileable(P.ins[j])) {
            const uint32_t S2 = S | ins_bits(P.ins[j]);
            if (__builtin_popcount(S2 & ~low) > T - 5) break;
            S = S2;
            ++j;
        }
        if (j - i < std::max<size_t>(min_run, 1)) {
            out.push_back(P.ins[i++]);
            continue;
        }
        uint32_t tb = S | low;
        for (int b = 5; b < n && __builtin_popcount(tb) < T; ++b) tb |= 1u << b;
        int loc[32];
        std::fill(loc, loc + 32, 0);
        uint32_t cnt = 0;
        const uint32_t off = uint32_t(P.mats.size() / 2);
        for (int b = 0; b < n; ++b)
            if (tb >> b & 1u) {
                loc[b] = int(cnt++);
                const uint32_t w = uint32_t(b);
                float f;
                std::memcpy(&f, &w, sizeof f);
                P.mats.push_back(f);
            }
        if (cnt % 2) P.mats.push_back(0.f); // keep whole complex entries
        TInstr H{};
        H.op = kTTile;
        H.b0 = uint8_t(T);
        H.mat = off;
        H.cmask = uint32_t(j - i);
        out.push_back(H);
        auto remap = [&](uint32_t mask) {
            uint32_t r = 0;
            for (int b = 0; b < 32; ++b)
                if (mask >> b & 1u) r |= 1u << loc[b];
            return r;
        };
        for (size_t k = i; k < j; ++k) {
            TInstr I = P.ins[k];
            I.b0 = uint8_t(loc[I.b0]);
            if (I.op == kTG2 || I.op == kTG3 || I.op == kTG4) I.b1 = uint8_t(loc[I.b1]);
            if (I.op == kTG3) I.cmask = uint32_t(loc[I.cmask & 255u]);
            if (I.op == kTCG1) {
                I.cmask = remap(I.cmask);
                I.cval = remap(I.cval);
            }
            if (I.op == kTG4)
                I.cmask = uint32_t(loc[I.cmask & 255u]) | (uint32_t(loc[(I.cmask >> 8) & 255u]) << 8);
            out.push_back(I);
        }
        i = j;
    }
    P.ins.swap(out);
}

namespace {
std::mutex g_tile_mu;
std::map<std::pair<int, int>, int> g_tile_chosen; // (device, n) -> T
} // namespace

void set_tile_width(qgpu_ctx* ctx, int n, int T) {
    std::lock_guard<std::mutex> lock(g_tile_mu);
    if (T < 0) g_tile_chosen.erase({ctx->device, n});
    else g_tile_chosen[{ctx->device, n}] = T;
}

namespace {

// The calibration program of a register of n qubits: two layers of 1-qubit
// gates on every qubit and 2-qubit gates on (0,1), (2,3), ... or, with
// `matching`, on a fixed random matching (what fusion sees in layered
// circuits). Matrix values do not change the time; one layer under-rates
// the narrower tiles.
TProgram calibration_program(int n, bool matching) {
    TProgram P;
    P.n = uint32_t(n);
    const float h = 0.70710678f;
    const float g1[8] = {h, 0, h, 0, h, 0, -h, 0};
    for (float v : g1) P.mats.push_back(v);
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            P.mats.push_back(r == c ? 0.5f : 0.5f * float((r + c) % 2));
            P.mats.push_back(0.f);
        }
    uint32_t x = 12345u; // fixed matching sequence
    for (int layer = 0; layer < 2; ++layer) {
        for (int q = 0; q < n; ++q) {
            TInstr I{};
            I.op = kTG1;
            I.b0 = uint8_t(q);
            I.flags = q == 0 ? kTNewStep : 0;
            P.ins.push_back(I);
        }
        std::vector<int> perm(static_cast<size_t>(n));
        for (int q = 0; q < n; ++q) perm[size_t(q)] = q;
        for (int q = n - 1; q > 0 && matching; --q) {
            x = x * 1664525u + 1013904223u;
            std::swap(perm[size_t(q)], perm[size_t(x % uint32_t(q + 1))]);
        }
        for (int q = 0; q + 1 < n; q += 2) {
            TInstr I{};
            I.op = kTG2;
            I.b0 = uint8_t(perm[size_t(q)]);
            I.b1 = uint8_t(perm[size_t(q + 1)]);
            I.mat = 4;
            P.ins.push_back(I);
        }
    }
    return P;
}

// Device time (ms) of one launch of K registers of n qubits running each
// program of `forms` with its tile width; -1 for forms too large to stage.
std::vector<float> time_forms(qgpu_ctx* ctx, int n, const std::vector<std::pair<TProgram, int>>& forms) {
    const uint64_t N = uint64_t(1) << n;
    const int K = int(std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(ctx->num_sms) * 4,
                                                               (uint64_t(1) << 29) / (N * 8))));
    const size_t b_state = size_t(K) * N * sizeof(float2);
    const size_t b_prog = 4096 * sizeof(TInstr), b_mat = 262144, b_work = K * sizeof(TWork);
    unsigned char* buf = nullptr;
    QG_CUDA(qgpu::ctx_malloc(ctx, reinterpret_cast<void**>(&buf),
                             b_state + b_prog + b_mat + b_work + 64 * K));
    struct Free {
        qgpu_ctx* c;
        void* p;
        ~Free() { cudaFreeAsync(p, c->stream); }
    } fr{ctx, buf};
    auto* dstate = reinterpret_cast<float2*>(buf);
    auto* dins = reinterpret_cast<TInstr*>(buf + b_state);
    auto* dmat = reinterpret_cast<float2*>(buf + b_state + b_prog);
    auto* dwork = reinterpret_cast<TWork*>(buf + b_state + b_prog + b_mat);
    auto* dsamp = reinterpret_cast<uint64_t*>(buf + b_state + b_prog + b_mat + b_work);
    QG_CUDA(cudaMemsetAsync(dstate, 0, b_state, ctx->stream));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    QG_CUDA(cudaEventCreate(&e0));
    QG_CUDA(cudaEventCreate(&e1));
    struct Ev {
        cudaEvent_t a, b;
        ~Ev() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } ev{e0, e1};
    std::vector<float> out;
    for (const auto& f : forms) {
        const TProgram& Q = f.first;
        const int T = f.second;
        if (Q.ins.size() > 4096 || Q.mats.size() * sizeof(float) > b_mat) {
            out.push_back(-1.f);
            continue;
        }
        QG_CUDA(cudaMemcpyAsync(dins, Q.ins.data(), Q.ins.size() * sizeof(TInstr),
                                cudaMemcpyHostToDevice, ctx->stream));
        QG_CUDA(cudaMemcpyAsync(dmat, Q.mats.data(), Q.mats.size() * sizeof(float),
                                cudaMemcpyHostToDevice, ctx->stream));
        std::vector<TWork> work(static_cast<size_t>(K));
        for (int k = 0; k < K; ++k) {
            TWork w{};
            w.prog = dins;
            w.mats = dmat;
            w.nins = uint32_t(Q.ins.size());
            w.n = uint8_t(n);
            w.out = uint32_t(k);
            w.init = dstate + size_t(k) * N;
            w.fin = dstate + size_t(k) * N;
            w.inplace = n > kTrajMaxQubits ? 1 : 0;
            w.diag = nullptr;
            work[size_t(k)] = w;
        }
        QG_CUDA(cudaMemcpyAsync(dwork, work.data(), K * sizeof(TWork), cudaMemcpyHostToDevice,
                                ctx->stream));
        launch_traj(ctx, dwork, K, n, nullptr, 0, dsamp, nullptr, nullptr, 0, nullptr, nullptr, T);
        QG_CUDA(cudaEventRecord(e0, ctx->stream));
        launch_traj(ctx, dwork, K, n, nullptr, 0, dsamp, nullptr, nullptr, 0, nullptr, nullptr, T);
        QG_CUDA(cudaEventRecord(e1, ctx->stream));
        QG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        QG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        out.push_back(ms);
    }
    return out;
}

std::map<std::pair<int, int>, int> g_fuse_chosen; // (device, n) -> fusion width

} // namespace

void fuse_blocks(TProgram& P, int w) {
    using C = std::complex<double>;
    // plain complex products (std::complex's operator* also handles infinities
    // and NaNs through a library call)
    auto mul = [](C a, C b) {
        return C(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
    };
    w = std::max(1, std::min(w, kFuseMaxWidth));
    // a block of nb <= 4 bits: bits[0] is the most significant digit of its
    // index; U column-major (2^nb x 2^nb)
    struct Blk {
        int nb;
        int bits[4];
        C U[256];
    };
    MatPool pool(P);
    std::vector<TInstr> out;
    out.reserve(P.ins.size());
    std::vector<Blk> open; // acting on disjoint bits, so they commute
    auto emit = [&](const Blk& B) {
        TInstr I{};
        I.op = B.nb == 1 ? kTG1 : B.nb == 2 ? kTG2 : B.nb == 3 ? kTG3 : kTG4;
        I.b0 = uint8_t(B.bits[0]);
        if (B.nb >= 2) I.b1 = uint8_t(B.bits[1]);
        if (B.nb == 3) I.cmask = uint32_t(B.bits[2]);
        if (B.nb == 4) I.cmask = uint32_t(B.bits[2]) | (uint32_t(B.bits[3]) << 8);
        const size_t D = size_t(1) << B.nb;
        I.mat = pool.add(std::vector<C>(B.U, B.U + D * D));
        out.push_back(I);
    };
    auto bits_of = [](const Blk& B) {
        uint32_t m = 0;
        for (int t = 0; t < B.nb; ++t) m |= 1u << B.bits[t];
        return m;
    };
    // emit (in order) the open blocks that touch `mask`, keep the rest
    auto flush = [&](uint32_t mask) {
        size_t keep = 0;
        for (size_t i = 0; i < open.size(); ++i) {
            if (bits_of(open[i]) & mask) emit(open[i]);
            else {
                if (keep != i) open[keep] = open[i];
                ++keep;
            }
        }
        open.resize(keep);
    };
    Blk nb{};
    for (const TInstr& I : P.ins) {
        int gb[4], k = 0;
        switch (I.op) {
            case kTG1: gb[0] = I.b0; k = 1; break;
            case kTG2: gb[0] = I.b0; gb[1] = I.b1; k = 2; break;
            case kTG3: gb[0] = I.b0; gb[1] = I.b1; gb[2] = int(I.cmask & 255u); k = 3; break;
            case kTG4:
                gb[0] = I.b0;
                gb[1] = I.b1;
                gb[2] = int(I.cmask & 255u);
                gb[3] = int((I.cmask >> 8) & 255u);
                k = 4;
                break;
            default: break;
        }
        if (!k) { // not a dense gate: keep it, after the blocks it touches
            flush(ins_bits(I) | (I.op == kTMeas ? (1u << I.b0) : 0u) |
                  (I.op == kTTile ? 0xffffffffu : 0u));
            out.push_back(I);
            continue;
        }
        uint32_t gmask = 0;
        for (int t = 0; t < k; ++t) gmask |= 1u << gb[t];
        // union of the gate's bits and the open blocks it touches: the gate's
        // bits first, then each touched block's, in the blocks' order
        int ub[32], nu = 0;
        for (int t = 0; t < k; ++t) ub[nu++] = gb[t];
        size_t touched[32];
        int nt = 0;
        for (size_t bi = 0; bi < open.size(); ++bi) {
            if (!(bits_of(open[bi]) & gmask)) continue;
            touched[nt++] = bi;
            for (int t = 0; t < open[bi].nb; ++t)
                if (!((gmask >> open[bi].bits[t]) & 1u) &&
                    std::find(ub, ub + nu, open[bi].bits[t]) == ub + nu)
                    ub[nu++] = open[bi].bits[t];
        }
        if (nu > w) {
            flush(gmask); // emit the touched blocks, then start over with G
            nu = k;
            nt = 0;
            if (k > w) { // wider than the fusion width: as is
                out.push_back(I);
                continue;
            }
        }
        // position of register bit b in the new block's index
        int pos[32];
        for (int t = 0; t < nu; ++t) pos[ub[t]] = nu - 1 - t;
        const uint32_t D = 1u << nu;
        // M = the touched blocks' Kronecker product on ub (identity on the
        // gate's bits that no block held)
        uint32_t idm = 0;
        for (int t = 0; t < k; ++t) idm |= 1u << pos[gb[t]];
        uint32_t proj[32][16];
        for (int j = 0; j < nt; ++j) {
            const Blk& B = open[touched[j]];
            for (int t = 0; t < B.nb; ++t) idm &= ~(1u << pos[B.bits[t]]);
            for (uint32_t r = 0; r < D; ++r) {
                uint32_t x = 0;
                for (int t = 0; t < B.nb; ++t) x |= ((r >> pos[B.bits[t]]) & 1u) << (B.nb - 1 - t);
                proj[j][r] = x;
            }
        }
        C* M = nb.U;
        for (uint32_t c = 0; c < D; ++c)
            for (uint32_t r = 0; r < D; ++r) {
                C v = ((r ^ c) & idm) ? C(0.0) : C(1.0);
                for (int j = 0; j < nt && v != C(0.0); ++j) {
                    const Blk& B = open[touched[j]];
                    v = mul(v, B.U[proj[j][r] + (size_t(proj[j][c]) << B.nb)]);
                }
                M[r + size_t(c) * D] = v;
            }
        // M <- G M: G acts on the row digits at the gate's positions
        const uint32_t g = 1u << k;
        C G[256];
        for (uint32_t e = 0; e < g * g; ++e)
            G[e] = C(P.mats[2 * (size_t(I.mat) + e)], P.mats[2 * (size_t(I.mat) + e) + 1]);
        uint32_t spread[16];
        for (uint32_t j = 0; j < g; ++j) {
            uint32_t x = 0;
            for (int t = 0; t < k; ++t) x |= ((j >> (k - 1 - t)) & 1u) << pos[gb[t]];
            spread[j] = x;
        }
        uint32_t gpos = 0;
        for (int t = 0; t < k; ++t) gpos |= 1u << pos[gb[t]];
        C x[16];
        for (uint32_t c = 0; c < D; ++c)
            for (uint32_t r0 = 0; r0 < D; ++r0) {
                if (r0 & gpos) continue;
                C* col = M + size_t(c) * D;
                for (uint32_t j = 0; j < g; ++j) x[j] = col[r0 | spread[j]];
                for (uint32_t i = 0; i < g; ++i) {
                    C acc = 0.0;
                    for (uint32_t j = 0; j < g; ++j) acc += mul(G[i + j * g], x[j]);
                    col[r0 | spread[i]] = acc;
                }
            }
        nb.nb = nu;
        for (int t = 0; t < nu; ++t) nb.bits[t] = ub[t];
        // drop the touched blocks (ascending indices), add the new one
        for (int j = nt - 1; j >= 0; --j) open.erase(open.begin() + std::ptrdiff_t(touched[j]));
        open.push_back(nb);
    }
    flush(0xffffffffu);
    P.ins.swap(out);
}

int tile_width(qgpu_ctx* ctx, int n) {
    if (n <= kTrajMaxQubits) return 0;
    {
        std::lock_guard<std::mutex> lock(g_tile_mu);
        auto it = g_tile_chosen.find({ctx->device, n});
        if (it != g_tile_chosen.end()) return it->second;
    }
    const TProgram P = calibration_program(n, false);
    std::vector<std::pair<TProgram, int>> forms;
    for (int T : {0, 10, 11, 12, 13}) {
        // from 17 qubits on the untiled form (one register pass per gate)
        // is never competitive and the slowest to time
        if (T >= n || (T == 0 && n >= 17)) continue;
        TProgram Q = P;
        plan_tiles(Q, T);
        forms.emplace_back(std::move(Q), T);
    }
    const std::vector<float> ms = time_forms(ctx, n, forms);
    int best = 0;
    float best_ms = 0;
    for (size_t i = 0; i < forms.size(); ++i)
        if (ms[i] >= 0 && (best_ms == 0 || ms[i] < best_ms)) {
            best = forms[i].second;
            best_ms = ms[i];
        }
    std::lock_guard<std::mutex> lock(g_tile_mu);
    g_tile_chosen[{ctx->device, n}] = best;
    return best;
}

void set_fusion_width(qgpu_ctx* ctx, int n, int w) {
    std::lock_guard<std::mutex> lock(g_tile_mu);
    if (w < 0) g_fuse_chosen.erase({ctx->device, n});
    else g_fuse_chosen[{ctx->device, n}] = w;
}

int fusion_width(qgpu_ctx* ctx, int n) {
    {
        std::lock_guard<std::mutex> lock(g_tile_mu);
        auto it = g_fuse_chosen.find({ctx->device, n});
        if (it != g_fuse_chosen.end()) return it->second;
    }
    const int T = tile_width(ctx, n);
    const TProgram P = calibration_program(n, true);
    std::vector<std::pair<TProgram, int>> forms;
    for (int w = 2; w <= kFuseMaxWidth; ++w) {
        TProgram Q = P;
        fuse_blocks(Q, w);
        if (T) plan_tiles(Q, T);
        forms.emplace_back(std::move(Q), T);
    }
    const std::vector<float> ms = time_forms(ctx, n, forms);
    int best = 2;
    float best_ms = 0;
    for (size_t i = 0; i < forms.size(); ++i)
        if (ms[i] >= 0 && (best_ms == 0 || ms[i] < best_ms)) {
            best = int(i) + 2;
            best_ms = ms[i];
        }
    std::lock_guard<std::mutex> lock(g_tile_mu);
    g_fuse_chosen[{ctx->device, n}] = best;
    return best;
}

} // namespace qgpu

using qgpu::guarded;
using qgpu::need_handle;
using qgpu::raise;

extern "C" qgpu_status qgpu_trajectories(qgpu_ctx* ctx, qgpu_circuit* c, double p_depol,
                                         uint64_t shots, uint64_t seed, uint64_t* samples,
                                         uint32_t* dits, double* dump, uint32_t* events,
                                         uint32_t max_events) {
    return guarded(__func__, [&] {
        need_handle(ctx);
        need_handle(c);
        const char* W = "qgpu_trajectories()";
        qgpu::TProgram P;
        if (!qgpu::compile_traj(c, P))
            raise(QGPU_ERR_NOT_SUPPORTED, W,
                  "circuit needs the engine (> 20 qubits, > 2-qubit or classically controlled gates)");
        if (shots == 0) raise(QGPU_ERR_OUT_OF_RANGE, W, "shots");
        const int T = qgpu::tile_width(ctx, int(P.n));
        qgpu::plan_tiles(P, T);
        const uint32_t maxcreg = std::max<uint32_t>(P.ncreg, 1);
        const uint64_t N = uint64_t(1) << P.n;
        // device buffers: program, matrices, work, outputs
        size_t b_ins = P.ins.size() * sizeof(qgpu::TInstr);
        size_t b_mat = std::max<size_t>(P.mats.size() * sizeof(float), 8);
        size_t b_work = shots * sizeof(qgpu::TWork);
        size_t b_dits = shots * maxcreg * sizeof(uint32_t);
        size_t b_samp = shots * sizeof(uint64_t);
        size_t b_dump = dump ? shots * N * sizeof(float2) : 0;
        size_t b_ev = events ? shots * size_t(max_events) * sizeof(qgpu::TEvent) : 0;
        size_t b_g = P.n > uint32_t(qgpu::kTrajMaxQubits)
                         ? size_t(qgpu::traj_global_grid(ctx, int(shots), int(P.n))) * N *
                               sizeof(float2)
                         : 0;
        auto al = [](size_t x) { return (x + 255) / 256 * 256; };
        size_t total = al(b_ins) + al(b_mat) + al(b_work) + al(b_dits) + al(b_samp) + al(b_dump) +
                       al(b_ev) + al(b_g);
        unsigned char* buf = nullptr;
        QG_CUDA(qgpu::ctx_malloc(ctx, reinterpret_cast<void**>(&buf), total));
        unsigned char* p = buf;
        auto take = [&](size_t b) {
            unsigned char* r = p;
            p += al(b);
            return r;
        };
        auto* dins = reinterpret_cast<qgpu::TInstr*>(take(b_ins));
        auto* dmat = reinterpret_cast<float2*>(take(b_mat));
        auto* dwork = reinterpret_cast<qgpu::TWork*>(take(b_work));
        auto* ddits = reinterpret_cast<uint32_t*>(take(b_dits));
        auto* dsamp = reinterpret_cast<uint64_t*>(take(b_samp));
        auto* ddump = reinterpret_cast<float2*>(dump ? take(b_dump) : nullptr);
        auto* dev = reinterpret_cast<qgpu::TEvent*>(events ? take(b_ev) : nullptr);
        auto* dg = reinterpret_cast<float2*>(b_g ? take(b_g) : nullptr);
        std::vector<qgpu::TWork> work(shots);
        for (uint64_t s = 0; s < shots; ++s) {
            qgpu::TWork w{};
            w.prog = dins;
            w.mats = dmat;
            w.nins = uint32_t(P.ins.size());
            w.n = uint8_t(P.n);
            w.p_noise = float(p_depol);
            w.shot = uint32_t(s);
            w.out = uint32_t(s);
            w.seed = seed;
            work[s] = w;
        }
        QG_CUDA(cudaMemcpyAsync(dins, P.ins.data(), b_ins, cudaMemcpyHostToDevice, ctx->stream));
        if (!P.mats.empty())
            QG_CUDA(cudaMemcpyAsync(dmat, P.mats.data(), P.mats.size() * sizeof(float),
                                    cudaMemcpyHostToDevice, ctx->stream));
        QG_CUDA(cudaMemcpyAsync(dwork, work.data(), b_work, cudaMemcpyHostToDevice, ctx->stream));
        QG_CUDA(cudaMemsetAsync(ddits, 0, b_dits, ctx->stream));
        if (dev) QG_CUDA(cudaMemsetAsync(dev, 0xff, b_ev, ctx->stream));
        qgpu::launch_traj(ctx, dwork, int(shots), int(P.n), ddits, int(maxcreg), dsamp, ddump,
                          dev, int(max_events), dg, nullptr, T);
        if (samples)
            QG_CUDA(cudaMemcpyAsync(samples, dsamp, b_samp, cudaMemcpyDeviceToHost, ctx->stream));
        if (dits)
            QG_CUDA(cudaMemcpyAsync(dits, ddits, b_dits, cudaMemcpyDeviceToHost, ctx->stream));
        std::vector<float> dumpf;
        if (dump) {
            dumpf.resize(shots * N * 2);
            QG_CUDA(cudaMemcpyAsync(dumpf.data(), ddump, b_dump, cudaMemcpyDeviceToHost,
                                    ctx->stream));
        }
        if (events)
            QG_CUDA(cudaMemcpyAsync(events, dev, b_ev, cudaMemcpyDeviceToHost, ctx->stream));
        QG_CUDA(cudaFreeAsync(buf, ctx->stream));
        QG_CUDA(cudaStreamSynchronize(ctx->stream));
        if (dump)
            for (size_t i = 0; i < dumpf.size(); ++i) dump[i] = double(dumpf[i]);
    });
}

extern "C" qgpu_status qgpu_traj_fusion_width(qgpu_ctx* ctx, uint32_t n, int set_w, int* chosen) {
    return guarded(__func__, [&] {
        need_handle(ctx);
        const char* W = "qgpu_traj_fusion_width()";
        if (n < 1 || n > uint32_t(qgpu::kTrajMaxGlobalQubits))
            raise(QGPU_ERR_OUT_OF_RANGE, W, "n");
        if (set_w > qgpu::kFuseMaxWidth || set_w == 0 || set_w == 1 || set_w < -2)
            raise(QGPU_ERR_OUT_OF_RANGE, W, "set_w");
        if (set_w >= 2) qgpu::set_fusion_width(ctx, int(n), set_w);
        if (set_w == -2) qgpu::set_fusion_width(ctx, int(n), -1);
        if (chosen) *chosen = qgpu::fusion_width(ctx, int(n));
    });
}

extern "C" qgpu_status qgpu_traj_tile_width(qgpu_ctx* ctx, uint32_t n, int set_T, int* chosen) {
    return guarded(__func__, [&] {
        need_handle(ctx);
        const char* W = "qgpu_traj_tile_width()";
        if (n == 0 || n > uint32_t(qgpu::kTrajMaxGlobalQubits)) raise(QGPU_ERR_OUT_OF_RANGE, W, "n");
        if (set_T != -1 && set_T != -2 && set_T != 0 && (set_T < 9 || set_T > qgpu::kTrajMaxQubits ||
                                                         set_T >= int(n)))
            raise(QGPU_ERR_OUT_OF_RANGE, W, "T");
        if (set_T >= 0) qgpu::set_tile_width(ctx, int(n), set_T);
        if (set_T == -2) qgpu::set_tile_width(ctx, int(n), -1);
        if (chosen) *chosen = qgpu::tile_width(ctx, int(n));
    });
}
