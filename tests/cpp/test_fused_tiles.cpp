// CPU check of the fused complex128 form's tile-pass runs (qgpu::fuse with
// blocks of <= 2 qubits, then qgpu::tiled_runs): random circuits on qubit
// kets of 1-12 qubits mixing 1- and 2-qubit gates, fan gates, controlled
// gates with 1-3 controls (with and without shifts) and 3-qubit gates. The
// runs' gate descriptors applied one by one on the host, with the runs' steps
// in between, must equal the circuit's steps applied one by one within 1e-12
// (relative, max-norm): the blocks' qubit order, their column-major matrices
// and the cut into runs and steps are what the tile passes execute. Each run
// list-scheduled (qgpu::schedule_gates, tiles of 5-13 bits) must give the
// same product within 1e-12 and plan into no more passes than circuit order.
// On kets of 20-30 qubits the schedule keeps every bit's gates in circuit
// order. The tile passes' own addressing is checked against gate-by-gate
// application by test_gate_tiles.cpp. Built and run by
// tests/test_fused_tiles.py.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
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

// a gate descriptor over the whole state: op 1 on bit b0, op 2 on bits
// (b0, b1) with row index 2 * b(b0) + b(b1); controls (bit, value)
static void apply_desc(std::vector<C>& psi, const GateDesc& g) {
    const uint64_t N = psi.size();
    auto ok = [&](uint64_t i) {
        for (auto& c : g.ctrl)
            if (int((i >> c.first) & 1) != c.second) return false;
        return true;
    };
    const int D = g.op == 1 ? 2 : 4;
    std::vector<uint64_t> off(D);
    for (int r = 0; r < D; ++r)
        off[r] = g.op == 1 ? (r ? uint64_t(1) << g.b0 : 0)
                           : (((r >> 1) & 1 ? uint64_t(1) << g.b0 : 0) |
                              ((r & 1) ? uint64_t(1) << g.b1 : 0));
    const uint64_t mask = off[D - 1] | (g.op == 1 ? 0 : off[1] | off[2]);
    std::vector<C> v(D);
    for (uint64_t b = 0; b < N; ++b) {
        if ((b & mask) || !ok(b)) continue;
        for (int r = 0; r < D; ++r) v[r] = psi[b + off[r]];
        for (int r = 0; r < D; ++r) {
            C acc = 0;
            for (int c = 0; c < D; ++c) acc += g.A[r + D * c] * v[c];
            psi[b + off[r]] = acc;
        }
    }
}

// a dense gate U (column-major, big-endian over `target`) on an n-qubit ket
static void apply_dense(std::vector<C>& psi, int n, const std::vector<cd>& U,
                        const std::vector<uint64_t>& target) {
    const int k = int(target.size());
    const uint64_t D = uint64_t(1) << k, N = psi.size();
    std::vector<uint64_t> off(D);
    uint64_t mask = 0;
    for (uint64_t r = 0; r < D; ++r) {
        uint64_t o = 0;
        for (int j = 0; j < k; ++j)
            if ((r >> (k - 1 - j)) & 1) o |= uint64_t(1) << (n - 1 - int(target[size_t(j)]));
        off[r] = o;
        mask |= o;
    }
    std::vector<C> v(D);
    for (uint64_t b = 0; b < N; ++b) {
        if (b & mask) continue;
        for (uint64_t r = 0; r < D; ++r) v[r] = psi[b + off[r]];
        for (uint64_t r = 0; r < D; ++r) {
            C acc = 0;
            for (uint64_t c = 0; c < D; ++c) acc += U[r + D * c] * v[c];
            psi[b + off[r]] = acc;
        }
    }
}

// one step as qpp applies it: 1- and 2-qubit steps through their gate
// descriptors, 3-qubit gates densely
static void apply_step_host(std::vector<C>& psi, int n, const Step& st) {
    std::vector<GateDesc> g;
    if (gate_desc_of(st, n, g)) {
        for (const GateDesc& d : g) apply_desc(psi, d);
        return;
    }
    EXPECT(st.kind == StepKind::Gate);
    apply_dense(psi, n, st.U, st.target);
}

static std::vector<cd> haar(std::mt19937_64& rng, int D) {
    // Gram-Schmidt on a complex Gaussian matrix (column-major)
    std::normal_distribution<double> nd;
    std::vector<cd> M(size_t(D) * D);
    for (auto& x : M) x = cd(nd(rng), nd(rng));
    for (int c = 0; c < D; ++c) {
        for (int p = 0; p < c; ++p) {
            cd dot = 0;
            for (int r = 0; r < D; ++r) dot += std::conj(M[r + D * p]) * M[r + D * c];
            for (int r = 0; r < D; ++r) M[r + D * c] -= dot * M[r + D * p];
        }
        double nrm = 0;
        for (int r = 0; r < D; ++r) nrm += std::norm(M[r + D * c]);
        nrm = std::sqrt(nrm);
        for (int r = 0; r < D; ++r) M[r + D * c] /= nrm;
    }
    return M;
}

static std::vector<uint64_t> distinct(std::mt19937_64& rng, int n, int k) {
    std::vector<uint64_t> all(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) all[size_t(i)] = uint64_t(i);
    std::shuffle(all.begin(), all.end(), rng);
    all.resize(size_t(k));
    return all;
}

// Large runs (kets of 20-30 qubits, 2000 gates; too large to simulate here):
// the schedule is a permutation of the gates in which the gates on each bit
// (targets and controls) keep their circuit order, and it plans into no more
// passes than circuit order.
static void check_large_schedules(std::mt19937_64& rng) {
    for (int n : {20, 24, 30})
        for (int Tmax : {10, 13}) {
            std::vector<GateDesc> g;
            for (int i = 0; i < 2000; ++i) {
                GateDesc d;
                d.op = (rng() % 10 < 7) ? 1 : 2;
                d.b0 = int(rng() % uint64_t(n));
                if (d.op == 2)
                    do d.b1 = int(rng() % uint64_t(n));
                    while (d.b1 == d.b0);
                if (rng() % 10 == 0) {
                    int c;
                    do c = int(rng() % uint64_t(n));
                    while (c == d.b0 || (d.op == 2 && c == d.b1));
                    d.ctrl.push_back({c, int(rng() % 2)});
                }
                d.A[0] = cd(double(i), 0.0); // the gate's identity
                g.push_back(d);
            }
            const std::vector<GateDesc> s = schedule_gates(g, n, Tmax);
            EXPECT(s.size() == g.size());
            std::vector<int> seen(g.size(), 0);
            std::vector<std::vector<int>> on_bit(static_cast<size_t>(n));
            for (const GateDesc& d : s) {
                const int id = int(d.A[0].real());
                EXPECT(id >= 0 && id < int(g.size()));
                if (id < 0 || id >= int(g.size())) return;
                ++seen[size_t(id)];
                std::vector<int> bits{d.b0};
                if (d.op == 2) bits.push_back(d.b1);
                for (const auto& c : d.ctrl) bits.push_back(c.first);
                for (int b : bits) on_bit[size_t(b)].push_back(id);
            }
            for (int x : seen) EXPECT(x == 1);
            for (const auto& v : on_bit) EXPECT(std::is_sorted(v.begin(), v.end()));
            std::vector<TilePassParams> p0, p1;
            std::vector<TileGate> dv;
            std::vector<TileSweep> sw;
            std::vector<cd> m;
            plan_gate_tiles(g, n, Tmax, p0, dv, sw, m);
            plan_gate_tiles(s, n, Tmax, p1, dv, sw, m);
            EXPECT(p1.size() <= p0.size());
            std::printf("n=%d tiles of %d bits: %zu passes in circuit order, %zu scheduled\n", n,
                        Tmax, p0.size(), p1.size());
        }
}

int main() {
    std::mt19937_64 rng(7);
    check_large_schedules(rng);
    int cases = 0, with_steps = 0;
    size_t passes_in_order = 0, passes_scheduled = 0, sweeps_in_order = 0, sweeps_scheduled = 0;
    for (int n = 1; n <= 12; ++n)
        for (int rep = 0; rep < 4; ++rep) {
            qgpu_circuit* c = nullptr;
            EXPECT(qgpu_circuit_create(uint32_t(n), 2, 0, &c) == QGPU_OK);
            const int ngates = 20 + int(rng() % 60);
            for (int i = 0; i < ngates; ++i) {
                const int kind = int(rng() % 10);
                if (kind < 5 || n < 2) { // 1-qubit gate
                    auto t = distinct(rng, n, 1);
                    auto U = haar(rng, 2);
                    EXPECT(qgpu_circuit_gate(c, reinterpret_cast<double*>(U.data()), 2, t.data(),
                                             1) == QGPU_OK);
                } else if (kind < 8) { // 2-qubit gate
                    auto t = distinct(rng, n, 2);
                    auto U = haar(rng, 4);
                    EXPECT(qgpu_circuit_gate(c, reinterpret_cast<double*>(U.data()), 4, t.data(),
                                             2) == QGPU_OK);
                } else if (kind == 8) { // controlled 1-qubit gate, 1-3 controls
                    const int nc = std::min(n - 1, 1 + int(rng() % 3));
                    auto q = distinct(rng, n, nc + 1);
                    std::vector<uint64_t> ctrl(q.begin(), q.begin() + nc), tgt{q.back()};
                    std::vector<uint64_t> shift(static_cast<size_t>(nc));
                    for (auto& x : shift) x = rng() % 2;
                    auto U = haar(rng, 2);
                    EXPECT(qgpu_circuit_ctrl(c, reinterpret_cast<double*>(U.data()), 2,
                                             ctrl.data(), uint32_t(nc), tgt.data(), 1,
                                             (rng() % 2) ? shift.data() : nullptr,
                                             0) == QGPU_OK);
                } else if (n >= 3 && (rng() % 2)) { // 3-qubit gate
                    auto t = distinct(rng, n, 3);
                    auto U = haar(rng, 8);
                    EXPECT(qgpu_circuit_gate(c, reinterpret_cast<double*>(U.data()), 8, t.data(),
                                             3) == QGPU_OK);
                } else { // fan gate
                    const int k = std::min(n, 1 + int(rng() % 3));
                    auto t = distinct(rng, n, k);
                    auto U = haar(rng, 2);
                    EXPECT(qgpu_circuit_gate_fan(c, reinterpret_cast<double*>(U.data()), 2,
                                                 t.data(), uint32_t(k)) == QGPU_OK);
                }
            }
            std::vector<C> psi(size_t(1) << n);
            std::normal_distribution<double> nd;
            for (auto& x : psi) x = C(nd(rng), nd(rng));
            std::vector<C> ref = psi, got = psi, sch = psi;
            for (const Step& st : c->steps) apply_step_host(ref, n, st);
            c->plan = fuse(c->steps, c->nq, 2);
            c->plan_k = 2;
            std::vector<TiledRun> runs;
            tiled_runs(c, runs);
            size_t gates = 0;
            const int Tmax = 5 + int(rng() % 9); // tiles of 5-13 bits
            for (const TiledRun& r : runs) {
                if (r.step >= 0) {
                    EXPECT(r.gates.empty());
                    apply_step_host(got, n, c->steps[size_t(r.step)]);
                    apply_step_host(sch, n, c->steps[size_t(r.step)]);
                    ++with_steps;
                    continue;
                }
                for (const GateDesc& g : r.gates) {
                    EXPECT(g.op == 1 || g.op == 2);
                    EXPECT(g.b0 >= 0 && g.b0 < n && (g.op == 1 || (g.b1 >= 0 && g.b1 < n)));
                    EXPECT(g.op == 1 || g.b0 != g.b1);
                    apply_desc(got, g);
                    ++gates;
                }
                // the list-scheduled order: the same gates, no more passes
                // than circuit order, the same product up to rounding
                const std::vector<GateDesc> s2 = schedule_gates(r.gates, n, Tmax);
                EXPECT(s2.size() == r.gates.size());
                for (const GateDesc& g : s2) apply_desc(sch, g);
                std::vector<TilePassParams> p0, p1;
                std::vector<TileGate> d;
                std::vector<TileSweep> sw0, sw1;
                std::vector<cd> m;
                plan_gate_tiles(r.gates, n, Tmax, p0, d, sw0, m);
                plan_gate_tiles(s2, n, Tmax, p1, d, sw1, m);
                EXPECT(p1.size() <= p0.size());
                passes_in_order += p0.size();
                passes_scheduled += p1.size();
                sweeps_in_order += sw0.size();
                sweeps_scheduled += sw1.size();
            }
            EXPECT(gates <= c->steps.size() * 3); // fan gates expand, blocks merge
            double err = 0, err_s = 0, scale = 0;
            for (size_t i = 0; i < ref.size(); ++i) {
                err = std::max(err, std::abs(got[i] - ref[i]));
                err_s = std::max(err_s, std::abs(sch[i] - ref[i]));
                scale = std::max(scale, std::abs(ref[i]));
            }
            EXPECT(err <= 1e-12 * scale);
            EXPECT(err_s <= 1e-12 * scale);
            if (err > 1e-12 * scale || err_s > 1e-12 * scale)
                std::printf("n=%d rep=%d: rel err %.3e, scheduled %.3e\n", n, rep, err / scale,
                            err_s / scale);
            qgpu_circuit_destroy(c);
            ++cases;
        }
    std::printf("%d circuits, %d steps run as they are\n", cases, with_steps);
    std::printf("tile passes %zu in circuit order, %zu scheduled; sweeps %zu / %zu\n",
                passes_in_order, passes_scheduled, sweeps_in_order, sweeps_scheduled);
    std::printf(fails ? "fused tiles FAILED (%d)\n" : "fused tiles ok\n", fails);
    return fails ? 1 : 0;
}
