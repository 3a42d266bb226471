// tile_gates.cpp -- the plain form of qgpu_run_gates on qubit kets as
// cache-blocked tile passes (kernels_tile.cu).
//
// qpp applies every gate of a circuit as its own pass over the state
// (QEngine::visit_gate_step_, qengine.hpp:551-578 -> apply / applyCTRL). Here
// consecutive 1- and 2-qubit gates (plain, fan, controlled with any number of
// controls) are grouped into passes: a pass keeps the L lowest state bits and
// up to T - L other bits in shared memory, and takes gates in circuit order
// while the union of their target bits outside the low L stays within T - L
// (controls may be anywhere). Each pass reads and writes the state once,
// however many gates it holds, and applies each gate with the one-gate
// kernels' arithmetic, so the result is the gate-by-gate result.
#include "tile_gates.hpp"

#include <algorithm>
#include <cstring>
#include <set>

#include "circuit.hpp"
#include "kernels.hpp"
#include "ops.hpp"

namespace qgpu {

// gates per pass, so that the pass's matrices (<= 16 complex each) stay
// within 64 KB of shared memory next to a 128 KB tile
constexpr size_t kTileMaxGates = 256;
// tile bits a sweep may span (groups of up to 8 amplitudes in registers)
constexpr int kSweepBits = 3;

bool gate_desc_of(const Step& st, int nbits, std::vector<GateDesc>& out) {
    auto bit_of = [&](uint64_t q) { return nbits - 1 - int(q); };
    auto ctrl_list = [&](std::vector<std::pair<int, int>>& c) {
        for (size_t i = 0; i < st.ctrl.size(); ++i) {
            // the gate acts when control i reads (shift_inv + 1) % 2, with
            // shift_inv = (2 - shift) % 2 (operations.hpp:727-735, :777-821)
            const uint64_t sh = st.has_shift ? st.shift[i] % 2 : 0;
            const uint64_t inv = (2 - sh) % 2;
            c.push_back({bit_of(st.ctrl[i]), int((inv + 1) % 2)});
        }
    };
    switch (st.kind) {
        case StepKind::Gate: {
            if (st.target.size() == 1 && st.DU == 2) {
                GateDesc g;
                g.op = 1;
                g.b0 = bit_of(st.target[0]);
                std::copy(st.U.begin(), st.U.end(), g.A);
                out.push_back(g);
                return true;
            }
            if (st.target.size() == 2 && st.DU == 4) {
                GateDesc g;
                g.op = 2;
                g.b0 = bit_of(st.target[0]);
                g.b1 = bit_of(st.target[1]);
                std::copy(st.U.begin(), st.U.end(), g.A);
                out.push_back(g);
                return true;
            }
            return false;
        }
        case StepKind::Fan: {
            if (st.DU != 2) return false;
            for (uint64_t t : st.target) {
                GateDesc g;
                g.op = 1;
                g.b0 = bit_of(t);
                std::copy(st.U.begin(), st.U.end(), g.A);
                out.push_back(g);
            }
            return true;
        }
        case StepKind::Ctrl: {
            if (st.target.size() == 1 && st.DU == 2) {
                GateDesc g;
                g.op = 1;
                g.b0 = bit_of(st.target[0]);
                ctrl_list(g.ctrl);
                std::copy(st.U.begin(), st.U.end(), g.A);
                out.push_back(g);
                return true;
            }
            if (st.target.size() == 2 && st.DU == 4) {
                GateDesc g;
                g.op = 2;
                g.b0 = bit_of(st.target[0]);
                g.b1 = bit_of(st.target[1]);
                ctrl_list(g.ctrl);
                std::copy(st.U.begin(), st.U.end(), g.A);
                out.push_back(g);
                return true;
            }
            return false;
        }
        case StepKind::CtrlFan: {
            if (st.DU != 2) return false;
            for (uint64_t t : st.target) {
                GateDesc g;
                g.op = 1;
                g.b0 = bit_of(t);
                ctrl_list(g.ctrl);
                std::copy(st.U.begin(), st.U.end(), g.A);
                out.push_back(g);
            }
            return true;
        }
        default:
            return false;
    }
}

// Tile of at most Tmax bits on an nbits-qubit ket: the L lowest state bits
// (five: coalesced runs; fewer when the tile must still hold the two targets
// of any 2-qubit gate above them) and up to nfree = T - L others.
static void tile_split(int nbits, int Tmax, int& L, int& nfree) {
    const int T = std::min(nbits, Tmax);
    L = std::min(T, 5);
    if (T < nbits && T - L < 2) L = std::max(0, T - 2);
    nfree = T - L;
}

std::vector<GateDesc> schedule_gates(const std::vector<GateDesc>& gates, int nbits, int Tmax) {
    int L = 0, nfree = 0;
    tile_split(nbits, Tmax, L, nfree);
    const size_t N = gates.size();
    // gate j waits for the last earlier gate on each of its bits (targets
    // and controls)
    std::vector<uint32_t> npred(N, 0);
    std::vector<std::vector<uint32_t>> succ(N);
    std::vector<int64_t> last(size_t(std::max(nbits, 1)), -1);
    for (size_t j = 0; j < N; ++j) {
        const GateDesc& g = gates[j];
        std::vector<int> bits{g.b0};
        if (g.op == 2) bits.push_back(g.b1);
        for (const auto& c : g.ctrl) bits.push_back(c.first);
        std::vector<int64_t> pred;
        for (int b : bits) {
            if (last[size_t(b)] >= 0) pred.push_back(last[size_t(b)]);
            last[size_t(b)] = int64_t(j);
        }
        std::sort(pred.begin(), pred.end());
        pred.erase(std::unique(pred.begin(), pred.end()), pred.end());
        for (int64_t p : pred) succ[size_t(p)].push_back(uint32_t(j));
        npred[j] = uint32_t(pred.size());
    }
    std::set<uint32_t> ready; // in circuit order
    for (size_t j = 0; j < N; ++j)
        if (!npred[j]) ready.insert(uint32_t(j));
    std::vector<GateDesc> out;
    out.reserve(N);
    while (!ready.empty()) {
        // one pass: ready gates while their targets above the low L bits fit
        // in nfree bits, those that extend the current sweep (<= 3 target
        // bits) first
        uint64_t hi = 0;
        int sw[kSweepBits], nsw = 0;
        size_t in_pass = 0;
        while (in_pass < kTileMaxGates) {
            int64_t pick = -1;
            bool pick_in_sweep = false;
            for (uint32_t j : ready) {
                const GateDesc& g = gates[j];
                uint64_t h2 = hi;
                for (int b : {g.b0, g.op == 2 ? g.b1 : -1})
                    if (b >= L) h2 |= uint64_t(1) << b;
                if (__builtin_popcountll(h2) > nfree) continue;
                int n2 = nsw;
                for (int b : {g.b0, g.op == 2 ? g.b1 : -1}) {
                    bool have = false;
                    for (int x = 0; x < nsw; ++x) have |= sw[x] == b;
                    if (b >= 0 && !have) ++n2;
                }
                if (n2 <= kSweepBits) {
                    pick = j;
                    pick_in_sweep = true;
                    break;
                }
                if (pick < 0) pick = j;
            }
            if (pick < 0) break;
            const GateDesc& g = gates[size_t(pick)];
            if (!pick_in_sweep) nsw = 0;
            for (int b : {g.b0, g.op == 2 ? g.b1 : -1}) {
                if (b < 0) continue;
                if (b >= L) hi |= uint64_t(1) << b;
                bool have = false;
                for (int x = 0; x < nsw; ++x) have |= sw[x] == b;
                if (!have) sw[nsw++] = b;
            }
            out.push_back(g);
            ++in_pass;
            ready.erase(uint32_t(pick));
            for (uint32_t s2 : succ[size_t(pick)])
                if (--npred[s2] == 0) ready.insert(s2);
        }
    }
    return out;
}

void plan_gate_tiles(const std::vector<GateDesc>& gates, int nbits, int Tmax,
                     std::vector<TilePassParams>& passes, std::vector<TileGate>& dev,
                     std::vector<TileSweep>& sweeps, std::vector<cd>& mats) {
    passes.clear();
    dev.clear();
    sweeps.clear();
    mats.clear();
    int L = 0, nfree = 0;
    tile_split(nbits, Tmax, L, nfree);
    size_t i = 0;
    while (i < gates.size()) {
        // greedy run: targets outside the low L bits within nfree bits
        std::vector<int> hi;
        size_t j = i;
        for (; j < gates.size() && j - i < kTileMaxGates; ++j) {
            std::vector<int> h2 = hi;
            const GateDesc& g = gates[j];
            for (int b : {g.b0, g.op == 2 ? g.b1 : -1})
                if (b >= L && std::find(h2.begin(), h2.end(), b) == h2.end()) h2.push_back(b);
            if (int(h2.size()) > nfree) break;
            hi.swap(h2);
        }
        if (j == i) raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_run_gates()", "tile too small");
        std::sort(hi.begin(), hi.end());
        TilePassParams p;
        std::memset(&p, 0, sizeof(p));
        p.T = L + int(hi.size());
        p.L = L;
        for (size_t k = 0; k < hi.size(); ++k) p.hi[k] = hi[k];
        p.ntiles = uint64_t(1) << (nbits - p.T);
        p.first = uint32_t(dev.size());
        p.ngates = uint32_t(j - i);
        p.mat_first = uint32_t(mats.size());
        auto local = [&](int b) {
            if (b < L) return b;
            return L + int(std::find(hi.begin(), hi.end(), b) - hi.begin());
        };
        for (size_t k = i; k < j; ++k) {
            const GateDesc& g = gates[k];
            TileGate d;
            std::memset(&d, 0, sizeof(d));
            d.op = uint32_t(g.op);
            d.t0 = local(g.b0);
            d.t1 = g.op == 2 ? local(g.b1) : 0;
            for (auto& c : g.ctrl) {
                const bool in_tile =
                    c.first < L || std::find(hi.begin(), hi.end(), c.first) != hi.end();
                if (in_tile) {
                    d.lmask |= 1u << local(c.first);
                    if (c.second) d.lval |= 1u << local(c.first);
                } else {
                    d.gmask |= uint64_t(1) << c.first;
                    if (c.second) d.gval |= uint64_t(1) << c.first;
                }
            }
            d.mat = uint32_t(mats.size());
            const int D = g.op == 1 ? 2 : 4;
            for (int r = 0; r < D; ++r)
                for (int c = 0; c < D; ++c) mats.push_back(g.A[r + D * c]); // row-major
            dev.push_back(d);
        }
        p.mat_elems = uint32_t(mats.size()) - p.mat_first;
        // sweeps: consecutive gates whose targets fit in three tile bits
        p.first_sweep = uint32_t(sweeps.size());
        for (size_t k = p.first; k < dev.size();) {
            TileSweep sw;
            std::memset(&sw, 0, sizeof(sw));
            sw.first = uint32_t(k);
            int nb = 0;
            for (; k < dev.size(); ++k) {
                TileGate& d = dev[k];
                int bits[3], n2 = nb;
                for (int x = 0; x < nb; ++x) bits[x] = sw.b[x];
                bool fits = true;
                for (int t : {d.t0, d.op == 2 ? d.t1 : -1}) {
                    if (t < 0 || std::find(bits, bits + n2, t) != bits + n2) continue;
                    if (n2 == kSweepBits) {
                        fits = false;
                        break;
                    }
                    bits[n2++] = t;
                }
                if (!fits) break;
                nb = n2;
                for (int x = 0; x < nb; ++x) sw.b[x] = bits[x];
                d.k0 = uint32_t(std::find(bits, bits + nb, d.t0) - bits);
                d.k1 = d.op == 2 ? uint32_t(std::find(bits, bits + nb, d.t1) - bits) : 0;
                ++sw.ngates;
            }
            sw.nb = uint32_t(nb);
            sweeps.push_back(sw);
        }
        p.nsweeps = uint32_t(sweeps.size()) - p.first_sweep;
        passes.push_back(p);
        i = j;
    }
}

int tile_bits_max(const qgpu_ctx* ctx, qgpu_prec prec) {
    // 128 KB tiles by default (one CTA per SM), and at most
    const int cap = prec == QGPU_C128 ? 13 : 14;
    if (ctx->tile_bits > 0) return std::min(ctx->tile_bits, cap);
    return cap;
}

void plan_tile_program(const std::vector<GateDesc>& gates, int nbits, int Tmax, TileProgram& P) {
    P.nbits = nbits;
    P.Tmax = Tmax;
    P.gates = gates;
    plan_gate_tiles(gates, nbits, Tmax, P.passes, P.dev, P.sweeps, P.mats);
}

void run_tile_program(qgpu_state* s, const TileProgram& P) {
    if (P.gates.empty()) return;
    if (P.nbits != int(s->dims.size()))
        raise(QGPU_ERR_DIMS_MISMATCH_CVECTOR, "qgpu_run_gates()", "tile program / state");
    const int nbits = P.nbits;
    const auto& passes = P.passes;
    const auto& dev = P.dev;
    const auto& sweeps = P.sweeps;
    const auto& mats = P.mats;
    // a pass of one uncontrolled gate runs on the one-gate kernels
    bool any_tiled = false;
    for (const auto& p : passes)
        if (p.ngates > 1 || dev[p.first].lmask || dev[p.first].gmask) any_tiled = true;
    unsigned char* buf = nullptr;
    const size_t eb = s->prec == QGPU_C128 ? 16 : 8;
    const size_t b_gates = (dev.size() * sizeof(TileGate) + 255) / 256 * 256;
    const size_t b_sweeps = (sweeps.size() * sizeof(TileSweep) + 255) / 256 * 256;
    const size_t o_mats = b_gates + b_sweeps;
    if (any_tiled) {
        QG_CUDA(ctx_malloc(s->ctx, reinterpret_cast<void**>(&buf), o_mats + mats.size() * eb));
        QG_CUDA(cudaMemcpyAsync(buf, dev.data(), dev.size() * sizeof(TileGate),
                                cudaMemcpyHostToDevice, s->ctx->stream));
        QG_CUDA(cudaMemcpyAsync(buf + b_gates, sweeps.data(), sweeps.size() * sizeof(TileSweep),
                                cudaMemcpyHostToDevice, s->ctx->stream));
        if (s->prec == QGPU_C128) {
            QG_CUDA(cudaMemcpyAsync(buf + o_mats, mats.data(), mats.size() * sizeof(cd),
                                    cudaMemcpyHostToDevice, s->ctx->stream));
        } else {
            std::vector<float> mf(2 * mats.size());
            for (size_t k = 0; k < mats.size(); ++k) {
                mf[2 * k] = float(mats[k].real());
                mf[2 * k + 1] = float(mats[k].imag());
            }
            QG_CUDA(cudaMemcpyAsync(buf + o_mats, mf.data(), mf.size() * sizeof(float),
                                    cudaMemcpyHostToDevice, s->ctx->stream));
        }
    }
    size_t gi = 0;
    for (const auto& p : passes) {
        const GateDesc& g0 = P.gates[gi];
        if (p.ngates == 1 && g0.ctrl.empty()) {
            if (g0.op == 1) launch_qubit_1q(s->ctx, s->prec, s->data, nbits, g0.b0, g0.A);
            else launch_qubit_2q(s->ctx, s->prec, s->data, nbits, g0.b0, g0.b1, g0.A);
        } else {
            launch_tile_pass(s->ctx, s->prec, s->data, p, reinterpret_cast<TileGate*>(buf),
                             reinterpret_cast<TileSweep*>(buf + b_gates), buf + o_mats);
        }
        gi += p.ngates;
    }
    if (buf) QG_CUDA(cudaFreeAsync(buf, s->ctx->stream));
}

void run_tiled_gates(qgpu_state* s, const std::vector<GateDesc>& gates) {
    if (gates.empty()) return;
    TileProgram P;
    plan_tile_program(gates, int(s->dims.size()), tile_bits_max(s->ctx, s->prec), P);
    run_tile_program(s, P);
}

} // namespace qgpu
