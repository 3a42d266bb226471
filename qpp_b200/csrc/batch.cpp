// batch.cpp -- many independent instances (kets and density matrices of
// uneven sizes, each with its own circuit) in one CUDA-graph launch.
//
// No reference counterpart: Quantum++ runs one state per call. The batched
// form compiles every instance into a trajectory program (a density matrix
// as a ket over 2n virtual qubits, see compile_traj_rho), groups instances
// by register size, and captures one trajectory-kernel launch per size into
// a single CUDA graph (one parallel branch per size), so the whole batch is
// one graph launch. One CTA runs one instance: registers of up to 2^14
// amplitudes are copied into shared memory and back to the instance's own
// qgpu_state; larger ones are worked on in place in that state (HBM). The
// plain form loops over the instances with one kernel launch per gate
// (qgpu_run_gates, QGPU_FORM_PLAIN).
#include <algorithm>
#include <cstring>
#include <map>
#include <set>

#include "capi_common.hpp"
#include "circuit.hpp"
#include "ops.hpp"
#include "traj.hpp"

namespace qgpu {

bool compile_traj_rho(const qgpu_circuit* c, TProgram& P) {
    const int nq = int(c->nq), nv = 2 * nq;
    if (c->d != 2 || nv > kTrajMaxGlobalQubits) return false;
    P = TProgram{};
    P.n = uint32_t(nv);
    P.ncreg = c->nc;
    auto vbit = [&](int v) { return uint8_t(nv - 1 - v); };
    auto add_mat = [&](const std::vector<cd>& U) {
        uint32_t off = uint32_t(P.mats.size() / 2);
        for (const cd& z : U) {
            P.mats.push_back(float(z.real()));
            P.mats.push_back(float(z.imag()));
        }
        return off;
    };
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
    return guarded([&] {
        need_handle(ctx);
        const char* W = "qgpu_run_batch()";
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
        std::vector<uint32_t> plain;
        std::vector<std::pair<uint32_t, qgpu::TProgram>> prog;
        for (uint32_t i = 0; i < n_inst; ++i) {
            qgpu::TProgram P;
            bool ok = form == 1 && states[i]->prec == QGPU_C64 &&
                      (states[i]->kind == QGPU_KET ? qgpu::compile_traj(circuits[i], P)
                                                   : qgpu::compile_traj_rho(circuits[i], P));
            if (ok) prog.emplace_back(i, std::move(P));
            else plain.push_back(i);
        }
        if (!prog.empty()) {
            // registers above shared-memory size: cache-blocked tile passes
            // at the tuned width of their size class (timed before capture)
            std::map<uint32_t, int> tile_of;
            for (auto& pr : prog) {
                const uint32_t n = pr.second.n;
                if (n <= uint32_t(qgpu::kTrajMaxQubits)) continue;
                auto it = tile_of.find(n);
                if (it == tile_of.end()) it = tile_of.emplace(n, qgpu::tile_width(ctx, int(n))).first;
                qgpu::plan_tiles(pr.second, it->second);
            }
            // device copies of all programs, work items grouped by size
            std::map<uint32_t, std::vector<size_t>> by_n;
            std::vector<qgpu::TInstr> ins;
            std::vector<float> mats;
            std::vector<std::pair<size_t, size_t>> ofs(prog.size());
            for (size_t k = 0; k < prog.size(); ++k) {
                ofs[k] = {ins.size(), mats.size() / 2};
                ins.insert(ins.end(), prog[k].second.ins.begin(), prog[k].second.ins.end());
                mats.insert(mats.end(), prog[k].second.mats.begin(), prog[k].second.mats.end());
                by_n[prog[k].second.n].push_back(k);
            }
            auto al = [](size_t x) { return (x + 255) / 256 * 256; };
            size_t b_ins = std::max<size_t>(ins.size() * sizeof(qgpu::TInstr), 16);
            size_t b_mat = std::max<size_t>(mats.size() * sizeof(float), 16);
            size_t b_work = prog.size() * sizeof(qgpu::TWork);
            size_t b_out = prog.size() * (sizeof(uint64_t) + sizeof(uint32_t) * 8);
            size_t total = al(b_ins) + al(b_mat) + al(b_work) + al(b_out);
            unsigned char* buf = nullptr;
            QG_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&buf), total, ctx->stream));
            unsigned char* p = buf;
            auto take = [&](size_t b) {
                unsigned char* q = p;
                p += al(b);
                return q;
            };
            auto* dins = reinterpret_cast<qgpu::TInstr*>(take(b_ins));
            auto* dmat = reinterpret_cast<float2*>(take(b_mat));
            auto* dwork = reinterpret_cast<qgpu::TWork*>(take(b_work));
            auto* dsamp = reinterpret_cast<uint64_t*>(take(prog.size() * sizeof(uint64_t)));
            auto* ddits = reinterpret_cast<uint32_t*>(take(prog.size() * sizeof(uint32_t) * 8));
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
            QG_CUDA(cudaMemcpyAsync(dins, ins.data(), ins.size() * sizeof(qgpu::TInstr),
                                    cudaMemcpyHostToDevice, ctx->stream));
            if (!mats.empty())
                QG_CUDA(cudaMemcpyAsync(dmat, mats.data(), mats.size() * sizeof(float),
                                        cudaMemcpyHostToDevice, ctx->stream));
            QG_CUDA(cudaMemcpyAsync(dwork, work.data(), b_work, cudaMemcpyHostToDevice,
                                    ctx->stream));
            // one graph: a launch per register size, each on its own branch
            // (the groups touch disjoint states), so the small-register
            // launches fill the SMs that the few large instances leave idle
            qgpu::traj_prepare();
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            std::vector<cudaStream_t> side(ranges.size(), nullptr);
            std::vector<cudaEvent_t> ev(ranges.size() + 1, nullptr);
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
                for (size_t g = 0; g < ranges.size(); ++g) {
                    const auto& rg = ranges[g];
                    QG_CUDA(cudaStreamWaitEvent(side[g], ev[0], 0));
                    auto tt = tile_of.find(rg.first);
                    qgpu::launch_traj(ctx, dwork + rg.second.first,
                                      int(rg.second.second - rg.second.first), int(rg.first), ddits, 1,
                                      dsamp, nullptr, nullptr, 0, nullptr, side[g],
                                      tt == tile_of.end() ? 0 : tt->second);
                    QG_CUDA(cudaEventRecord(ev[g + 1], side[g]));
                    QG_CUDA(cudaStreamWaitEvent(ctx->stream, ev[g + 1], 0));
                }
            } catch (...) {
                cudaStreamEndCapture(ctx->stream, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            QG_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
            QG_CUDA(cudaGraphInstantiate(&exec, graph, 0));
            QG_CUDA(cudaGraphLaunch(exec, ctx->stream));
            QG_CUDA(cudaFreeAsync(buf, ctx->stream));
            QG_CUDA(cudaStreamSynchronize(ctx->stream));
            cudaGraphExecDestroy(exec);
            cudaGraphDestroy(graph);
            if (graph_kernels) *graph_kernels = ranges.size();
        }
        for (uint32_t i : plain) qgpu::run_gates(states[i], circuits[i], 0, 0, circuits[i]->steps.size());
        QG_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}
