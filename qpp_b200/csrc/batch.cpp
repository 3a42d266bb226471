// batch.cpp -- many independent instances (kets and density matrices of
// uneven sizes, each with its own circuit) in one CUDA-graph launch.
//
// No reference counterpart: Quantum++ runs one state per call. The batched
// form compiles every instance into a trajectory program (a density matrix
// as a ket over 2n virtual qubits, see compile_traj_rho), groups instances
// by register size, and captures everything into a single CUDA graph, so the
// whole batch is one graph launch. Registers of up to 2^14 amplitudes: one
// CTA per instance with the register in shared memory, one trajectory-kernel
// launch per size on its own graph branch. Larger registers whose programs
// are all gates: cache-blocked tile passes at the tuned width, run
// layer-synchronously on one more branch -- graph node k applies pass k of
// every such register, all tiles in parallel, in place in the instances' own
// states. Larger registers with measurements keep one CTA per instance.
// Registers of at least 2^18 amplitudes whose programs are all dense gates
// (kets of 18-22 qubits, density matrices of 9-15 qubits) run block-layered
// on one more branch instead: every program fused into blocks of <= 4
// (virtual) qubits, launch j applies block j of every such register. The
// plain form loops over the instances with one kernel launch per gate
// (qgpu_run_gates, QGPU_FORM_PLAIN).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <exception>
#include <functional>
#include <map>
#include <mutex>
#include <set>
#include <thread>

#include "capi_common.hpp"
#include "circuit.hpp"
#include "ops.hpp"
#include "traj.hpp"

namespace qgpu {

// Register bits (kets: qubits; density matrices: twice the qubits) from which
// batched instances run block-layered.
constexpr int kBlockMinBits = 18;

bool compile_traj_rho(const qgpu_circuit* c, TProgram& P, int max_nv) {
    const int nq = int(c->nq), nv = 2 * nq;
    if (c->d != 2 || nv > std::min(max_nv, 31)) return false;
    P = TProgram{};
    P.n = uint32_t(nv);
    P.ncreg = c->nc;
    auto vbit = [&](int v) { return uint8_t(nv - 1 - v); };
    MatPool pool(P);
    auto add_mat = [&](const std::vector<cd>& U) { return pool.add(U); };
    auto super1 = [&](int t, const std::vector<cd>& S, uint8_t flags) {
        TInstr I{};
        I.op = kTG2;
        I.b0 = vbit(t);      // column digit t
        I.b1 = vbit(nq + t); // row digit t
        I.flags = flags;
        I.mat = add_mat(S);
        P.ins.push_back(I);
    };
    for (const Step& s : c->steps) {
        uint8_t first = kTNewStep;
        switch (s.kind) {
            case StepKind::Gate:
            case StepKind::Fan: {
                if (s.kind == StepKind::Gate && s.target.size() == 2) {
                    int a = int(s.target[0]), b = int(s.target[1]);
                    TInstr R{};
                    R.op = kTG2;
                    R.b0 = vbit(nq + a);
                    R.b1 = vbit(nq + b);
                    R.flags = first;
                    R.mat = add_mat(s.U);
                    P.ins.push_back(R);
                    TInstr Cc = R;
                    Cc.b0 = vbit(a);
                    Cc.b1 = vbit(b);
                    Cc.flags = 0;
                    Cc.mat = add_mat(conj_mat(s.U));
                    P.ins.push_back(Cc);
                    break;
                }
                if (s.kind == StepKind::Gate && s.target.size() != 1) return false;
                std::vector<cd> S = kron_mat(conj_mat(s.U), 2, s.U, 2);
                for (uint64_t t : s.target) {
                    super1(int(t), S, first);
                    first = 0;
                }
                break;
            }
            case StepKind::Channel: {
                const uint64_t DK = s.DU;
                if (!((s.target.size() == 1 && DK == 2) || (s.target.size() == 2 && DK == 4)))
                    return false;
                const uint64_t DS = DK * DK;
                std::vector<cd> S(DS * DS, 0.0);
                for (uint32_t i = 0; i < s.nK; ++i) {
                    std::vector<cd> K(s.U.begin() + DK * DK * i, s.U.begin() + DK * DK * (i + 1));
                    std::vector<cd> t = kron_mat(conj_mat(K), DK, K, DK);
                    for (size_t j = 0; j < t.size(); ++j) S[j] += t[j];
                }
                if (s.target.size() == 1) {
                    super1(int(s.target[0]), S, first);
                } else {
                    // sum_i conj(K_i) (x) K_i on (col a, col b, row a, row b)
                    int a = int(s.target[0]), b = int(s.target[1]);
                    TInstr I{};
                    I.op = kTG4;
                    I.b0 = vbit(a);
                    I.b1 = vbit(b);
                    I.cmask = uint32_t(vbit(nq + a)) | (uint32_t(vbit(nq + b)) << 8);
                    I.flags = first;
                    I.mat = add_mat(S);
                    P.ins.push_back(I);
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

} // namespace qgpu

using qgpu::guarded;
using qgpu::need_handle;
using qgpu::raise;

extern "C" qgpu_status qgpu_run_batch(qgpu_ctx* ctx, uint32_t n_inst, qgpu_circuit* const* circuits,
                                      qgpu_state* const* states, int form,
                                      uint64_t* graph_kernels) {
    return guarded(__func__, [&] {
        need_handle(ctx);
        const char* W = "qgpu_run_batch()";
        using clk = std::chrono::steady_clock;
        auto ms_since = [](clk::time_point t) {
            return std::chrono::duration<double, std::milli>(clk::now() - t).count();
        };
        for (double& x : ctx->batch_ms) x = 0;
        auto t_check = clk::now();
        if (n_inst && (!circuits || !states)) raise(QGPU_ERR_INVALID_ARGUMENT, W, "arrays");
        std::set<const qgpu_state*> seen;
        for (uint32_t i = 0; i < n_inst; ++i) {
            need_handle(circuits[i]);
            need_handle(states[i]);
            // instances run concurrently, each in its own state
            if (!seen.insert(states[i]).second) raise(QGPU_ERR_DUPLICATES, W, "states");
            const qgpu_state* s = states[i];
            if (s->dims.size() != circuits[i]->nq)
                raise(QGPU_ERR_DIMS_MISMATCH_CVECTOR, W, "state/circuit");
            for (uint64_t d : s->dims)
                if (d != circuits[i]->d) raise(QGPU_ERR_DIMS_MISMATCH_CVECTOR, W, "state/circuit");
        }
        if (graph_kernels) *graph_kernels = 0;
        ctx->batch_ms[4] = ms_since(t_check);
        auto t_compile = clk::now();
        std::vector<uint32_t> plain;
        std::vector<std::pair<uint32_t, qgpu::TProgram>> prog;
        // compile (and fold, tile, stage) every instance; the programs are
        // independent, so host threads share the work
        auto pfor = [](size_t count, const std::function<void(size_t)>& fn) {
            const size_t nth = std::min<size_t>(
                std::max(1u, std::thread::hardware_concurrency()), std::max<size_t>(1, count / 16));
            std::atomic<size_t> next{0};
            std::exception_ptr first;
            std::mutex emu;
            auto body = [&] {
                try {
                    for (size_t i; (i = next.fetch_add(1)) < count;) fn(i);
                } catch (...) {
                    std::lock_guard<std::mutex> lock(emu);
                    if (!first) first = std::current_exception();
                    next = count;
                }
            };
            std::vector<std::thread> th;
            for (size_t t = 1; t < nth; ++t) th.emplace_back(body);
            body();
            for (auto& t : th) t.join();
            if (first) std::rethrow_exception(first);
        };
        std::vector<qgpu::TProgram> progs(n_inst);
        std::vector<char> ok(n_inst, 0);
        pfor(n_inst, [&](size_t i) {
            qgpu::TProgram& P = progs[i];
            ok[i] = form == 1 && states[i]->prec == QGPU_C64 &&
                    (states[i]->kind == QGPU_KET ? qgpu::compile_traj(circuits[i], P)
                                                 : qgpu::compile_traj_rho(circuits[i], P));
        });
        auto all_gates = [](const qgpu::TProgram& P) {
            for (const auto& I : P.ins)
                if (I.op != qgpu::kTG1 && I.op != qgpu::kTCG1 && I.op != qgpu::kTG2 &&
                    I.op != qgpu::kTG3 && I.op != qgpu::kTG4)
                    return false;
            return true;
        };
        // Block-layered registers (no reference counterpart): density matrices
        // of at least kBlockMinBits virtual qubits (up to 15 qubits) and kets
        // of at least kBlockMinBits qubits whose programs are dense gates. Each
        // program is fused into blocks of <= 4 qubits (virtual qubits for a
        // density matrix: a layer's gates and channels on one qubit pair
        // become one block), and launch j of one chain applies block j of
        // every such register, one HBM pass per block with one thread per
        // group (k_block_batch). Above 2^18 amplitudes this beats the layered
        // tile passes, whose per-gate barriers held them to about a quarter of
        // HBM bandwidth there.
        std::vector<uint32_t> blocked;
        std::vector<char> on_block(n_inst, 0);
        std::vector<qgpu::TProgram> bprog(n_inst); // kets' block programs
        if (form == 1) {
            std::vector<uint32_t> cand;
            std::map<qgpu_circuit*, uint32_t> first_of; // one build per circuit
            for (uint32_t i = 0; i < n_inst; ++i) {
                const qgpu_state* s = states[i];
                if (s->kind != QGPU_RHO || s->prec != QGPU_C64 || s->ctx != ctx ||
                    circuits[i]->d != 2 || 2 * circuits[i]->nq < uint32_t(qgpu::kBlockMinBits))
                    continue;
                cand.push_back(i);
                first_of.emplace(circuits[i], i);
            }
            std::vector<uint32_t> reps;
            for (auto& kv : first_of) reps.push_back(kv.second);
            std::vector<char> good(n_inst, 0);
            pfor(reps.size(), [&](size_t k) {
                try {
                    qgpu::rho_program_prepare(states[reps[k]], circuits[reps[k]]);
                    good[reps[k]] = 1;
                } catch (const qgpu::Exc&) {
                    // not expressible in the fused form: stays as compiled
                }
            });
            for (uint32_t i : cand) {
                if (!good[first_of.at(circuits[i])]) continue;
                ok[i] = 0;
                on_block[i] = 1;
                blocked.push_back(i);
            }
            std::vector<uint32_t> kets;
            for (uint32_t i = 0; i < n_inst; ++i) {
                if (!ok[i] || states[i]->kind != QGPU_KET || states[i]->ctx != ctx ||
                    progs[i].n < uint32_t(qgpu::kBlockMinBits) || !all_gates(progs[i]))
                    continue;
                bool dense = true;
                for (const auto& I : progs[i].ins) dense = dense && I.op != qgpu::kTCG1;
                if (dense) kets.push_back(i);
            }
            pfor(kets.size(), [&](size_t k) {
                bprog[kets[k]] = std::move(progs[kets[k]]);
                qgpu::fuse_blocks(bprog[kets[k]], 4);
            });
            for (uint32_t i : kets) {
                ok[i] = 0;
                on_block[i] = 1;
                blocked.push_back(i);
            }
        }
        // batch programs carry no noise: gates fuse into dense blocks of the
        // width tuned for each register size (timed serially on the GPU)
        std::map<uint32_t, int> width_of;
        for (uint32_t i = 0; i < n_inst; ++i)
            if (ok[i] && !width_of.count(progs[i].n))
                width_of.emplace(progs[i].n, qgpu::fusion_width(ctx, int(progs[i].n)));
        pfor(n_inst, [&](size_t i) {
            if (ok[i]) qgpu::fuse_blocks(progs[i], width_of.at(progs[i].n));
        });
        for (uint32_t i = 0; i < n_inst; ++i) {
            if (ok[i]) prog.emplace_back(i, std::move(progs[i]));
            else if (!on_block[i]) plain.push_back(i);
        }
        if (!prog.empty() || !blocked.empty()) {
            // Registers above shared-memory size whose programs are all gates
            // run layer-synchronously: every gate belongs to a tile pass of
            // the tuned width, and launch k runs pass k of every such
            // register, all tiles in parallel. Programs with measurements keep
            // one CTA per register (tile passes inside k_traj).
            std::map<uint32_t, int> tile_of; // tuned serially (it times on the GPU)
            for (auto& pr : prog) {
                const uint32_t n = pr.second.n;
                if (n > uint32_t(qgpu::kTrajMaxQubits) && !tile_of.count(n))
                    tile_of.emplace(n, qgpu::tile_width(ctx, int(n)));
            }
            std::vector<char> layered(prog.size(), 0);
            pfor(prog.size(), [&](size_t k) {
                qgpu::TProgram& P = prog[k].second;
                const uint32_t n = P.n;
                if (n > uint32_t(qgpu::kTrajMaxQubits)) {
                    const int tw = tile_of.at(n);
                    if (all_gates(P) && !P.ins.empty()) {
                        // two 2^T tiles per CTA: T = 12 keeps three CTAs per SM
                        qgpu::plan_tiles(P, std::min(tw ? tw : 12, 12), 1);
                        layered[k] = 1;
                    } else {
                        qgpu::plan_tiles(P, tw);
                    }
                }
            });
            int layer_bits = 0;
            for (size_t k = 0; k < prog.size(); ++k)
                if (layered[k]) layer_bits = std::max(layer_bits, std::min(tile_of.at(prog[k].second.n) ? tile_of.at(prog[k].second.n) : 12, 12));
            ctx->batch_ms[0] = ms_since(t_compile);
            auto t_build = clk::now();
            // device copies of all programs, per-CTA work items grouped by size
            std::map<uint32_t, std::vector<size_t>> by_n;
            std::vector<qgpu::TInstr> ins;
            std::vector<float> mats;
            std::vector<std::pair<size_t, size_t>> ofs(prog.size());
            for (size_t k = 0; k < prog.size(); ++k) {
                ofs[k] = {ins.size(), mats.size() / 2};
                ins.insert(ins.end(), prog[k].second.ins.begin(), prog[k].second.ins.end());
                mats.insert(mats.end(), prog[k].second.mats.begin(), prog[k].second.mats.end());
                if (!layered[k]) by_n[prog[k].second.n].push_back(k);
            }
            // the passes of each layered register, in program order
            struct Pass {
                uint32_t pos, nins, tb_off;
                uint8_t T;
            };
            std::vector<std::vector<Pass>> passes(prog.size());
            size_t kmax = 0;
            for (size_t k = 0; k < prog.size(); ++k) {
                if (!layered[k]) continue;
                const auto& P = prog[k].second;
                for (size_t i = 0; i < P.ins.size(); ++i)
                    if (P.ins[i].op == qgpu::kTTile) {
                        passes[k].push_back({uint32_t(i + 1), P.ins[i].cmask, P.ins[i].mat,
                                             P.ins[i].b0});
                        i += P.ins[i].cmask;
                    }
                kmax = std::max(kmax, passes[k].size());
            }
            // block-layered registers: their programs' matrices (each program
            // once, on a 16-byte boundary), then launch j's blocks
            std::unique_ptr<float[]> bmats; // not zero-filled: every float is copied in
            size_t nbfloat = 0;
            std::map<const qgpu::TProgram*, size_t> bbase; // float2 offset
            std::vector<qgpu::BlockInst> binst;
            std::vector<size_t> bmoff; // float2 offset of each block's matrix
            std::vector<std::pair<size_t, std::pair<int, uint32_t>>> blaunch; // offset, (count, items)
            {
                std::vector<const qgpu::TProgram*> bp, uniq;
                size_t jmax = 0, nfloat = 0;
                for (uint32_t i : blocked) {
                    const qgpu::TProgram* P =
                        states[i]->kind == QGPU_KET ? &bprog[i] : circuits[i]->rho_prog.get();
                    bp.push_back(P);
                    jmax = std::max(jmax, P->ins.size());
                    if (bbase.count(P)) continue;
                    bbase[P] = nfloat / 2;
                    uniq.push_back(P);
                    nfloat += (P->mats.size() + 3) / 4 * 4; // next one 16-byte aligned
                }
                // one allocation, filled by host threads (about 200 MB for
                // config 4's registers)
                nbfloat = nfloat;
                bmats.reset(new float[std::max<size_t>(nfloat, 1)]);
                pfor(uniq.size(), [&](size_t u) {
                    const qgpu::TProgram* P = uniq[u];
                    float* dst = bmats.get() + 2 * bbase.at(P);
                    std::copy(P->mats.begin(), P->mats.end(), dst);
                    std::fill(dst + P->mats.size(), dst + (P->mats.size() + 3) / 4 * 4, 0.f);
                });
                for (size_t j = 0; j < jmax; ++j) {
                    const size_t off = binst.size();
                    uint32_t items = 0;
                    for (size_t k = 0; k < blocked.size(); ++k) {
                        const qgpu::TProgram& P = *bp[k];
                        if (j >= P.ins.size()) continue;
                        const qgpu::TInstr& I = P.ins[j];
                        qgpu::BlockInst B{};
                        B.k = I.op == qgpu::kTG1 ? 1 : I.op == qgpu::kTG2 ? 2
                            : I.op == qgpu::kTG3 ? 3 : I.op == qgpu::kTG4 ? 4 : 0;
                        if (!B.k) raise(QGPU_ERR_NOT_SUPPORTED, W, "block program");
                        const uint8_t bits[4] = {I.b0, I.b1, uint8_t(I.cmask & 255u),
                                                 uint8_t((I.cmask >> 8) & 255u)};
                        uint32_t seen_bits = 0;
                        for (int t = 0; t < B.k; ++t) {
                            if (bits[t] >= P.n || (seen_bits >> bits[t] & 1u))
                                raise(QGPU_ERR_NOT_SUPPORTED, W, "block bits");
                            seen_bits |= 1u << bits[t];
                            B.b[t] = bits[t];
                        }
                        const size_t moff = bbase.at(&P) + I.mat;
                        if (moff % 2) raise(QGPU_ERR_NOT_SUPPORTED, W, "block matrix alignment");
                        B.psi = static_cast<float2*>(states[blocked[k]]->data);
                        if (reinterpret_cast<uintptr_t>(B.psi) % 16)
                            raise(QGPU_ERR_INVALID_ARGUMENT, W, "state not 16-byte aligned");
                        B.n = uint8_t(P.n);
                        B.first_item = items;
                        items += uint32_t(((uint64_t(1) << (P.n - B.k)) + 511) / 512);
                        binst.push_back(B);
                        bmoff.push_back(moff);
                    }
                    blaunch.push_back({off, {int(binst.size() - off), items}});
                }
            }
            auto al = [](size_t x) { return (x + 255) / 256 * 256; };
            size_t npass_total = 0;
            for (auto& v : passes) npass_total += v.size();
            size_t b_ins = std::max<size_t>(ins.size() * sizeof(qgpu::TInstr), 16);
            size_t b_mat = std::max<size_t>(mats.size() * sizeof(float), 16);
            size_t b_work = std::max<size_t>(prog.size() * sizeof(qgpu::TWork), 16);
            size_t b_pass = std::max<size_t>(npass_total * sizeof(qgpu::PassInst), 16);
            // every region is taken on its own 256-byte boundary below
            size_t b_samp = std::max<size_t>(prog.size() * sizeof(uint64_t), 16);
            size_t b_dits = std::max<size_t>(prog.size() * sizeof(uint32_t) * 8, 16);
            size_t b_bmat = std::max<size_t>(nbfloat * sizeof(float), 16);
            size_t b_binst = std::max<size_t>(binst.size() * sizeof(qgpu::BlockInst), 16);
            size_t total = al(b_ins) + al(b_mat) + al(b_work) + al(b_pass) + al(b_samp) +
                           al(b_dits) + al(b_bmat) + al(b_binst);
            unsigned char* buf = nullptr;
            QG_CUDA(qgpu::ctx_malloc(ctx, reinterpret_cast<void**>(&buf), total));
            unsigned char* p = buf;
            auto take = [&](size_t b) {
                unsigned char* q = p;
                p += al(b);
                if (size_t(p - buf) > total) raise(QGPU_ERR_CUDA, W, "batch buffer layout");
                return q;
            };
            auto* dins = reinterpret_cast<qgpu::TInstr*>(take(b_ins));
            auto* dmat = reinterpret_cast<float2*>(take(b_mat));
            auto* dwork = reinterpret_cast<qgpu::TWork*>(take(b_work));
            auto* dpass = reinterpret_cast<qgpu::PassInst*>(take(b_pass));
            auto* dsamp = reinterpret_cast<uint64_t*>(take(b_samp));
            auto* ddits = reinterpret_cast<uint32_t*>(take(b_dits));
            auto* dbmat = reinterpret_cast<float2*>(take(b_bmat));
            auto* dbinst = reinterpret_cast<qgpu::BlockInst*>(take(b_binst));
            for (size_t k = 0; k < binst.size(); ++k) binst[k].m = dbmat + bmoff[k];
            std::vector<qgpu::TWork> work;
            std::vector<std::pair<uint32_t, std::pair<size_t, size_t>>> ranges; // n -> [lo, hi)
            for (auto& kv : by_n) {
                size_t lo = work.size();
                for (size_t k : kv.second) {
                    qgpu::TWork w{};
                    w.prog = dins + ofs[k].first;
                    w.mats = dmat + ofs[k].second;
                    w.nins = uint32_t(prog[k].second.ins.size());
                    w.n = uint8_t(kv.first);
                    w.p_noise = 0.f;
                    w.shot = 0;
                    w.out = uint32_t(work.size());
                    w.seed = prog[k].first;
                    w.init = static_cast<const float2*>(states[prog[k].first]->data);
                    w.fin = static_cast<float2*>(states[prog[k].first]->data);
                    // above shared-memory size the CTA works in the state itself
                    w.inplace = kv.first > uint32_t(qgpu::kTrajMaxQubits) ? 1 : 0;
                    work.push_back(w);
                }
                ranges.push_back({kv.first, {lo, work.size()}});
            }
            // launch k: pass k of every layered register; an item is 2^15
            // amplitudes of one register (equal work per item)
            std::vector<qgpu::PassInst> pinst;
            pinst.reserve(npass_total);
            std::vector<std::pair<size_t, std::pair<int, uint32_t>>> launches; // offset, (count, items)
            for (size_t kk = 0; kk < kmax; ++kk) {
                const size_t off = pinst.size();
                uint32_t items = 0;
                for (size_t k = 0; k < prog.size(); ++k) {
                    if (!layered[k] || kk >= passes[k].size()) continue;
                    const Pass& ps = passes[k][kk];
                    const uint32_t n = prog[k].second.n;
                    const uint32_t ntiles = 1u << (n - ps.T);
                    const uint32_t tpi =
                        std::min<uint32_t>(ntiles, std::max<uint32_t>(1, (1u << 15) >> ps.T));
                    qgpu::PassInst q{};
                    q.psi = static_cast<float2*>(states[prog[k].first]->data);
                    if (reinterpret_cast<uintptr_t>(q.psi) % 16)
                        raise(QGPU_ERR_INVALID_ARGUMENT, W, "state not 16-byte aligned");
                    q.mats = dmat + ofs[k].second;
                    q.ins = dins + ofs[k].first + ps.pos;
                    q.nins = ps.nins;
                    q.tb_off = ps.tb_off;
                    q.first_item = items;
                    q.tiles_per_item = tpi;
                    q.n = uint8_t(n);
                    q.T = ps.T;
                    pinst.push_back(q);
                    items += (ntiles + tpi - 1) / tpi;
                }
                launches.push_back({off, {int(pinst.size() - off), items}});
            }
            QG_CUDA(cudaMemcpyAsync(dins, ins.data(), ins.size() * sizeof(qgpu::TInstr),
                                    cudaMemcpyHostToDevice, ctx->stream));
            if (!mats.empty())
                QG_CUDA(cudaMemcpyAsync(dmat, mats.data(), mats.size() * sizeof(float),
                                        cudaMemcpyHostToDevice, ctx->stream));
            if (!work.empty())
                QG_CUDA(cudaMemcpyAsync(dwork, work.data(), work.size() * sizeof(qgpu::TWork),
                                        cudaMemcpyHostToDevice, ctx->stream));
            if (!pinst.empty())
                QG_CUDA(cudaMemcpyAsync(dpass, pinst.data(), pinst.size() * sizeof(qgpu::PassInst),
                                        cudaMemcpyHostToDevice, ctx->stream));
            if (!binst.empty()) {
                QG_CUDA(cudaMemcpyAsync(dbmat, bmats.get(), nbfloat * sizeof(float),
                                        cudaMemcpyHostToDevice, ctx->stream));
                QG_CUDA(cudaMemcpyAsync(dbinst, binst.data(), binst.size() * sizeof(qgpu::BlockInst),
                                        cudaMemcpyHostToDevice, ctx->stream));
            }
            int* dflag = launches.empty() ? nullptr : qgpu::ctx_error_flag(ctx);
            // one graph: a k_traj launch per register size on its own branch,
            // and the chain of layer launches on one more branch (all touch
            // disjoint states)
            qgpu::traj_prepare();
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            const size_t nbr = ranges.size() + (launches.empty() ? 0 : 1) + (blaunch.empty() ? 0 : 1);
            std::vector<cudaStream_t> side(nbr, nullptr);
            std::vector<cudaEvent_t> ev(nbr + 1, nullptr);
            struct Rel {
                std::vector<cudaStream_t>& s;
                std::vector<cudaEvent_t>& e;
                ~Rel() {
                    for (cudaStream_t x : s)
                        if (x) cudaStreamDestroy(x);
                    for (cudaEvent_t x : e)
                        if (x) cudaEventDestroy(x);
                }
            } rel{side, ev};
            for (auto& x : side) QG_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
            for (auto& x : ev) QG_CUDA(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
            QG_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            try {
                QG_CUDA(cudaEventRecord(ev[0], ctx->stream));
                size_t g = 0;
                if (!launches.empty()) { // longest chain first
                    QG_CUDA(cudaStreamWaitEvent(side[g], ev[0], 0));
                    for (auto& L : launches)
                        qgpu::launch_pass_batch(ctx, dpass + L.first, L.second.first,
                                                L.second.second, layer_bits, dflag, side[g]);
                    QG_CUDA(cudaEventRecord(ev[g + 1], side[g]));
                    QG_CUDA(cudaStreamWaitEvent(ctx->stream, ev[g + 1], 0));
                    ++g;
                }
                if (!blaunch.empty()) {
                    QG_CUDA(cudaStreamWaitEvent(side[g], ev[0], 0));
                    for (auto& L : blaunch)
                        qgpu::launch_block_batch(ctx, dbinst + L.first, L.second.first,
                                                 L.second.second, side[g]);
                    QG_CUDA(cudaEventRecord(ev[g + 1], side[g]));
                    QG_CUDA(cudaStreamWaitEvent(ctx->stream, ev[g + 1], 0));
                    ++g;
                }
                for (const auto& rg : ranges) {
                    QG_CUDA(cudaStreamWaitEvent(side[g], ev[0], 0));
                    auto tt = tile_of.find(rg.first);
                    qgpu::launch_traj(ctx, dwork + rg.second.first,
                                      int(rg.second.second - rg.second.first), int(rg.first), ddits, 1,
                                      dsamp, nullptr, nullptr, 0, nullptr, side[g],
                                      tt == tile_of.end() ? 0 : tt->second);
                    QG_CUDA(cudaEventRecord(ev[g + 1], side[g]));
                    QG_CUDA(cudaStreamWaitEvent(ctx->stream, ev[g + 1], 0));
                    ++g;
                }
            } catch (...) {
                cudaStreamEndCapture(ctx->stream, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            QG_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
            QG_CUDA(cudaGraphInstantiate(&exec, graph, 0));
            QG_CUDA(cudaStreamSynchronize(ctx->stream)); // uploads done
            ctx->batch_ms[1] = ms_since(t_build);
            // the graph's device time, on timing events of its own
            cudaEvent_t g0 = nullptr, g1 = nullptr;
            QG_CUDA(cudaEventCreate(&g0));
            QG_CUDA(cudaEventCreate(&g1));
            struct DelEv {
                cudaEvent_t a, b;
                ~DelEv() {
                    cudaEventDestroy(a);
                    cudaEventDestroy(b);
                }
            } delev{g0, g1};
            QG_CUDA(cudaEventRecord(g0, ctx->stream));
            QG_CUDA(cudaGraphLaunch(exec, ctx->stream));
            QG_CUDA(cudaEventRecord(g1, ctx->stream));
            QG_CUDA(cudaFreeAsync(buf, ctx->stream));
            QG_CUDA(cudaStreamSynchronize(ctx->stream));
            float gms = 0;
            QG_CUDA(cudaEventElapsedTime(&gms, g0, g1));
            ctx->batch_ms[2] = gms;
            auto t_tear = clk::now();
            cudaGraphExecDestroy(exec);
            cudaGraphDestroy(graph);
            if (dflag && qgpu::fused_error(ctx))
                raise(QGPU_ERR_TIMEOUT, W, "a bounded wait of a batch kernel gave up");
            ctx->batch_ms[5] = ms_since(t_tear);
            if (graph_kernels) *graph_kernels = ranges.size() + launches.size() + blaunch.size();
        }
        auto t_plain = clk::now();
        for (uint32_t i : plain) qgpu::run_gates(states[i], circuits[i], 0, 0, circuits[i]->steps.size());
        QG_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->batch_ms[3] = ms_since(t_plain);
    });
}

extern "C" qgpu_status qgpu_batch_last_phases(qgpu_ctx* ctx, double* phases_ms) {
    return guarded(__func__, [&] {
        need_handle(ctx);
        if (phases_ms) std::copy(ctx->batch_ms, ctx->batch_ms + 6, phases_ms);
    });
}
