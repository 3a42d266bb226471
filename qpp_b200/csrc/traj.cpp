// traj.cpp -- compile qgpu_circuit steps into shared-memory trajectory
// programs, and run all shots of one request in one launch.
#include "traj.hpp"

#include <algorithm>
#include <cstring>

#include "capi_common.hpp"
#include "circuit.hpp"

namespace qgpu {

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
    auto add_mat = [&](const std::vector<cd>& U) {
        uint32_t off = uint32_t(P.mats.size() / 2);
        for (const cd& z : U) {
            P.mats.push_back(float(z.real()));
            P.mats.push_back(float(z.imag()));
        }
        return off;
    };
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

} // namespace qgpu

using qgpu::guarded;
using qgpu::need_handle;
using qgpu::raise;

extern "C" qgpu_status qgpu_trajectories(qgpu_ctx* ctx, qgpu_circuit* c, double p_depol,
                                         uint64_t shots, uint64_t seed, uint64_t* samples,
                                         uint32_t* dits, double* dump, uint32_t* events,
                                         uint32_t max_events) {
    return guarded([&] {
        need_handle(ctx);
        need_handle(c);
        const char* W = "qgpu_trajectories()";
        qgpu::TProgram P;
        if (!qgpu::compile_traj(c, P))
            raise(QGPU_ERR_NOT_SUPPORTED, W,
                  "circuit needs the engine (> 20 qubits, > 2-qubit or classically controlled gates)");
        if (shots == 0) raise(QGPU_ERR_OUT_OF_RANGE, W, "shots");
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
        QG_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&buf), total, ctx->stream));
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
                          dev, int(max_events), dg);
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
