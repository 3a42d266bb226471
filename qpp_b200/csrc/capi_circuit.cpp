// capi_circuit.cpp -- extern "C" entry points for circuits, the fused form
// and single tensor-core blocks.
#include <algorithm>
#include <cstring>
#include <string>

#include "capi_common.hpp"
#include "circuit.hpp"
#include "kernels.hpp"
#include "ops.hpp"
#include "traj.hpp"

using qgpu::cd;
using qgpu::guarded;
using qgpu::need_handle;
using qgpu::raise;
using qgpu::vec_of;

namespace qgpu {
void fused6_matrix(const cd* U, float* B);
} // namespace qgpu

namespace {

std::string ctx_of(const qgpu_circuit* c) {
    return "Step " + std::to_string(c->steps.size()) + ": ";
}

// QCircuit::gate target checks (qcircuit.hpp:1453-1483)
void check_targets(const qgpu_circuit* c, const char* W,
                   const std::vector<uint64_t>& t, const char* what,
                   const std::vector<char>& measured) {
    if (t.empty()) raise(QGPU_ERR_ZERO_SIZE, W, ctx_of(c) + what);
    for (uint64_t x : t) {
        if (x >= c->nq) raise(QGPU_ERR_OUT_OF_RANGE, W, ctx_of(c) + what);
        if (measured[x]) raise(QGPU_ERR_QUDIT_ALREADY_MEASURED, W, ctx_of(c) + what);
    }
    std::vector<uint64_t> s = t;
    std::sort(s.begin(), s.end());
    if (std::adjacent_find(s.begin(), s.end()) != s.end())
        raise(QGPU_ERR_DUPLICATES, W, ctx_of(c) + what);
}

std::vector<char> measured_of(const qgpu_circuit* c) {
    std::vector<char> m(c->nq, 0);
    for (auto& s : c->steps)
        if (s.kind == qgpu::StepKind::Measure && s.destructive)
            for (uint64_t t : s.target) m[t] = 1;
    return m;
}

uint64_t ipow(uint64_t d, size_t k) {
    uint64_t r = 1;
    for (size_t i = 0; i < k; ++i) r *= d;
    return r;
}

} // namespace

extern "C" {

qgpu_status qgpu_circuit_create(uint32_t nq, uint64_t d, uint32_t nc,
                                qgpu_circuit** out) {
    return guarded(__func__, [&] {
        if (!out) raise(QGPU_ERR_INVALID_ARGUMENT, "qgpu_circuit_create()", "out");
        if (nq == 0) raise(QGPU_ERR_ZERO_SIZE, "qpp::QCircuit::QCircuit()", "nq");
        if (d < 2) raise(QGPU_ERR_DIMS_INVALID, "qpp::QCircuit::QCircuit()", "d");
        auto* c = new qgpu_circuit;
        c->nq = nq;
        c->d = d;
        c->nc = nc;
        *out = c;
    });
}

qgpu_status qgpu_circuit_destroy(qgpu_circuit* c) {
    return guarded(__func__, [&] { delete c; });
}

qgpu_status qgpu_circuit_gate(qgpu_circuit* c, const double* U, uint64_t DU,
                              const uint64_t* target, uint32_t k) {
    return guarded(__func__, [&] {
        need_handle(c);
        const char* W = "qpp::QCircuit::gate()";
        auto t = vec_of(target, k);
        check_targets(c, W, t, "target", measured_of(c));
        if (DU != ipow(c->d, t.size()))
            raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, ctx_of(c) + "U");
        qgpu::Step s;
        s.kind = qgpu::StepKind::Gate;
        s.U.assign(reinterpret_cast<const cd*>(U), reinterpret_cast<const cd*>(U) + DU * DU);
        s.DU = DU;
        s.target = t;
        c->steps.push_back(std::move(s));
        c->plan_k = 0;
    });
}

qgpu_status qgpu_circuit_gate_fan(qgpu_circuit* c, const double* U, uint64_t DU,
                                  const uint64_t* target, uint32_t k) {
    return guarded(__func__, [&] {
        need_handle(c);
        const char* W = "qpp::QCircuit::gate_fan()";
        auto t = vec_of(target, k);
        check_targets(c, W, t, "target", measured_of(c));
        if (DU != c->d) raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, ctx_of(c) + "U");
        qgpu::Step s;
        s.kind = qgpu::StepKind::Fan;
        s.U.assign(reinterpret_cast<const cd*>(U), reinterpret_cast<const cd*>(U) + DU * DU);
        s.DU = DU;
        s.target = t;
        c->steps.push_back(std::move(s));
        c->plan_k = 0;
    });
}

qgpu_status qgpu_circuit_ctrl(qgpu_circuit* c, const double* U, uint64_t DU,
                              const uint64_t* ctrl, uint32_t nc,
                              const uint64_t* target, uint32_t k,
                              const uint64_t* shift, int fan) {
    return guarded(__func__, [&] {
        need_handle(c);
        const char* W = fan ? "qpp::QCircuit::CTRL_fan()" : "qpp::QCircuit::CTRL()";
        auto cv = vec_of(ctrl, nc), t = vec_of(target, k);
        auto meas = measured_of(c);
        check_targets(c, W, cv, "ctrl", meas);
        check_targets(c, W, t, "target", meas);
        for (uint64_t x : cv)
            if (std::find(t.begin(), t.end(), x) != t.end())
                raise(QGPU_ERR_OUT_OF_RANGE, W, ctx_of(c) + "ctrl/target");
        uint64_t want = fan ? c->d : ipow(c->d, t.size());
        if (DU != want) raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, ctx_of(c) + "U");
        qgpu::Step s;
        s.kind = fan ? qgpu::StepKind::CtrlFan : qgpu::StepKind::Ctrl;
        s.U.assign(reinterpret_cast<const cd*>(U), reinterpret_cast<const cd*>(U) + DU * DU);
        s.DU = DU;
        s.ctrl = cv;
        s.target = t;
        if (shift) {
            s.has_shift = true;
            s.shift = vec_of(shift, nc);
            for (uint64_t x : s.shift)
                if (x >= c->d) raise(QGPU_ERR_OUT_OF_RANGE, W, ctx_of(c) + "shift");
        }
        c->steps.push_back(std::move(s));
        c->plan_k = 0;
    });
}

qgpu_status qgpu_circuit_cctrl(qgpu_circuit* c, const double* U, uint64_t DU,
                               const uint64_t* ctrl_dits, uint32_t nc,
                               const uint64_t* target, uint32_t k,
                               const uint64_t* shift, int fan) {
    return guarded(__func__, [&] {
        need_handle(c);
        const char* W = fan ? "qpp::QCircuit::cCTRL_fan()" : "qpp::QCircuit::cCTRL()";
        auto cv = vec_of(ctrl_dits, nc), t = vec_of(target, k);
        if (cv.empty()) raise(QGPU_ERR_ZERO_SIZE, W, ctx_of(c) + "ctrl_dits");
        for (uint64_t x : cv)
            if (x >= c->nc) raise(QGPU_ERR_OUT_OF_RANGE, W, ctx_of(c) + "ctrl_dits");
        check_targets(c, W, t, "target", measured_of(c));
        uint64_t want = fan ? c->d : ipow(c->d, t.size());
        if (DU != want) raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, ctx_of(c) + "U");
        qgpu::Step s;
        s.kind = fan ? qgpu::StepKind::CCtrlFan : qgpu::StepKind::CCtrl;
        s.U.assign(reinterpret_cast<const cd*>(U), reinterpret_cast<const cd*>(U) + DU * DU);
        s.DU = DU;
        s.ctrl = cv;
        s.target = t;
        if (shift) {
            s.has_shift = true;
            s.shift = vec_of(shift, nc);
        }
        c->steps.push_back(std::move(s));
        c->plan_k = 0;
    });
}

qgpu_status qgpu_circuit_measure(qgpu_circuit* c, const uint64_t* target, uint32_t k,
                                 uint64_t c_reg, int destructive) {
    return guarded(__func__, [&] {
        need_handle(c);
        const char* W = k > 1 ? "qpp::QCircuit::measure_many()" : "qpp::QCircuit::measure()";
        auto t = vec_of(target, k);
        check_targets(c, W, t, "target", measured_of(c));
        if (c_reg >= c->nc) raise(QGPU_ERR_OUT_OF_RANGE, W, ctx_of(c) + "c_reg");
        qgpu::Step s;
        s.kind = qgpu::StepKind::Measure;
        s.target = t;
        s.c_reg = c_reg;
        s.destructive = destructive != 0;
        c->steps.push_back(std::move(s));
        c->plan_k = 0;
    });
}

// QCircuit::reset (qcircuit.hpp): RESET / RESET_MANY measurement steps.
qgpu_status qgpu_circuit_reset(qgpu_circuit* c, const uint64_t* target, uint32_t k) {
    return guarded(__func__, [&] {
        need_handle(c);
        const char* W = k > 1 ? "qpp::QCircuit::reset_many()" : "qpp::QCircuit::reset()";
        auto t = vec_of(target, k);
        check_targets(c, W, t, "target", measured_of(c));
        qgpu::Step s;
        s.kind = qgpu::StepKind::Reset;
        s.target = t;
        c->steps.push_back(std::move(s));
        c->plan_k = 0;
    });
}

// QCircuit::cond_if / cond_end: the steps added in between run only when
// the dits (dits[0] the least significant bit) spell `value`.
qgpu_status qgpu_circuit_cond_if(qgpu_circuit* c, const uint64_t* dits, uint32_t n,
                                 uint64_t value) {
    return guarded(__func__, [&] {
        need_handle(c);
        const char* W = "qpp::QCircuit::cond_if()";
        for (const auto& st : c->steps)
            if (st.kind == qgpu::StepKind::CondIf && st.nK == 0)
                raise(QGPU_ERR_INVALID_ARGUMENT, W, "nested conditionals are not supported");
        auto d = vec_of(dits, n);
        if (d.empty() || d.size() > 63) raise(QGPU_ERR_OUT_OF_RANGE, W, ctx_of(c) + "dits");
        for (uint64_t x : d)
            if (x >= c->nc) raise(QGPU_ERR_OUT_OF_RANGE, W, ctx_of(c) + "dits");
        qgpu::Step s;
        s.kind = qgpu::StepKind::CondIf;
        s.ctrl = d;
        s.c_reg = value;
        s.nK = 0; // open
        c->steps.push_back(std::move(s));
        c->plan_k = 0;
    });
}

// QCircuit::QFT / TFQ (qcircuit.hpp:1514-1617, :1628-1732): qpp's gate
// sequence as steps (H or Fd on target i, CTRL R_j from target i + j - 1,
// SWAP / SWAPd; the adjoint sequence in the reverse order for TFQ);
// target == NULL takes every qudit not yet measured (QFT(bool swap)).
qgpu_status qgpu_circuit_qft(qgpu_circuit* c, const uint64_t* target, uint32_t k, int swap,
                             int inverse) {
    return guarded(__func__, [&] {
        need_handle(c);
        const char* W = inverse ? "qpp::QCircuit::TFQ()" : "qpp::QCircuit::QFT()";
        auto meas = measured_of(c);
        std::vector<uint64_t> t;
        if (target) {
            t = vec_of(target, k);
        } else {
            for (uint64_t q = 0; q < c->nq; ++q)
                if (!meas[q]) t.push_back(q);
        }
        check_targets(c, W, t, "target", meas);
        const uint64_t d = c->d;
        const size_t n = t.size();
        std::vector<cd> F = qgpu::fourier_gate(d);
        if (inverse) {
            std::vector<cd> Fa(d * d);
            for (uint64_t i = 0; i < d; ++i)
                for (uint64_t j = 0; j < d; ++j) Fa[i + j * d] = std::conj(F[j + i * d]);
            F = Fa;
        }
        const std::vector<cd> SW = qgpu::swap_gate(d);
        const size_t first = c->steps.size();
        auto gate = [&](const std::vector<cd>& U, uint64_t DU, std::vector<uint64_t> tg) {
            qgpu::Step s;
            s.kind = qgpu::StepKind::Gate;
            s.U = U;
            s.DU = DU;
            s.target = std::move(tg);
            c->steps.push_back(std::move(s));
        };
        auto ctrl = [&](size_t i, size_t j) {
            qgpu::Step s;
            s.kind = qgpu::StepKind::Ctrl;
            s.U = qgpu::qft_phase(d, j, inverse != 0);
            s.DU = d;
            s.ctrl = {t[i + j - 1]};
            s.target = {t[i]};
            c->steps.push_back(std::move(s));
        };
        if (!inverse) {
            for (size_t i = 0; i < n; ++i) {
                gate(F, d, {t[i]});
                for (size_t j = 2; j <= n - i; ++j) ctrl(i, j);
            }
            if (swap)
                for (size_t i = 0; i < n / 2; ++i) gate(SW, d * d, {t[i], t[n - i - 1]});
        } else {
            if (swap)
                for (size_t i = n / 2; i-- > 0;) gate(SW, d * d, {t[i], t[n - i - 1]});
            for (size_t i = n; i-- > 0;) {
                for (size_t j = n - i + 1; j-- > 2;) ctrl(i, j);
                gate(F, d, {t[i]});
            }
        }
        qgpu::Step& b = c->steps[first];
        b.block_len = uint32_t(c->steps.size() - first);
        b.block_inverse = inverse != 0;
        b.block_swap = swap != 0;
        b.block_target = t;
        c->plan_k = 0;
    });
}

qgpu_status qgpu_circuit_cond_end(qgpu_circuit* c) {
    return guarded(__func__, [&] {
        need_handle(c);
        size_t open = c->steps.size();
        for (size_t i = c->steps.size(); i-- > 0;)
            if (c->steps[i].kind == qgpu::StepKind::CondIf && c->steps[i].nK == 0) {
                open = i;
                break;
            }
        if (open == c->steps.size())
            raise(QGPU_ERR_INVALID_ARGUMENT, "qpp::QCircuit::cond_end()", "no open cond_if");
        qgpu::Step s;
        s.kind = qgpu::StepKind::CondEnd;
        c->steps.push_back(std::move(s));
        c->steps[open].nK = uint32_t(c->steps.size() - 1 - open); // the block and the END
        c->plan_k = 0;
    });
}

qgpu_status qgpu_circuit_channel(qgpu_circuit* c, const double* Ks, uint32_t nK, uint64_t DK,
                                 const uint64_t* target, uint32_t k) {
    return guarded(__func__, [&] {
        need_handle(c);
        const char* W = "qgpu_circuit_channel()";
        auto t = vec_of(target, k);
        check_targets(c, W, t, "target", measured_of(c));
        if (nK == 0) raise(QGPU_ERR_ZERO_SIZE, W, ctx_of(c) + "Ks");
        if (DK != ipow(c->d, t.size())) raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, ctx_of(c) + "Ks");
        qgpu::Step s;
        s.kind = qgpu::StepKind::Channel;
        const cd* K = reinterpret_cast<const cd*>(Ks);
        s.U.assign(K, K + size_t(nK) * DK * DK);
        s.DU = DK;
        s.nK = nK;
        s.target = t;
        c->steps.push_back(std::move(s));
        c->plan_k = 0;
    });
}

qgpu_status qgpu_circuit_info(const qgpu_circuit* c, uint32_t* nq, uint64_t* n_steps) {
    return guarded(__func__, [&] {
        need_handle(c);
        if (nq) *nq = c->nq;
        if (n_steps) *n_steps = c->steps.size();
    });
}

qgpu_status qgpu_circuit_shape(const qgpu_circuit* c, uint32_t* nq, uint64_t* d, uint32_t* nc) {
    return guarded(__func__, [&] {
        need_handle(c);
        if (nq) *nq = c->nq;
        if (d) *d = c->d;
        if (nc) *nc = c->nc;
    });
}

qgpu_status qgpu_circuit_fuse(qgpu_circuit* c, uint32_t max_k, uint64_t* n_passes) {
    return guarded(__func__, [&] {
        need_handle(c);
        if (c->d != 2) raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_circuit_fuse()", "qubit circuits only");
        if (max_k < 1 || max_k > 12)
            raise(QGPU_ERR_OUT_OF_RANGE, "qgpu_circuit_fuse()", "max_k");
        auto plan = qgpu::fuse(c->steps, c->nq, max_k);
        if (n_passes) *n_passes = plan.size();
    });
}

qgpu_status qgpu_run_gates(qgpu_state* s, qgpu_circuit* c, int form) {
    return guarded(__func__, [&] {
        need_handle(s);
        need_handle(c);
        if (s->dims.size() != c->nq)
            raise(QGPU_ERR_DIMS_MISMATCH_CVECTOR, "qgpu_run_gates()", "state/circuit");
        for (uint64_t x : s->dims)
            if (x != c->d) raise(QGPU_ERR_DIMS_MISMATCH_CVECTOR, "qgpu_run_gates()", "state/circuit");
        qgpu::run_gates(s, c, form, 0, c->steps.size());
    });
}

qgpu_status qgpu_apply_tc(qgpu_state* s, const double* U, const uint64_t* target, uint32_t k) {
    return guarded(__func__, [&] {
        need_handle(s);
        const char* W = "qgpu_apply_tc()";
        auto t = vec_of(target, k);
        if (s->kind != QGPU_KET || s->prec != QGPU_C64)
            raise(QGPU_ERR_NOT_SUPPORTED, W, "complex64 kets only");
        for (uint64_t x : s->dims)
            if (x != 2) raise(QGPU_ERR_NOT_SUPPORTED, W, "qubits only");
        int n = int(s->dims.size());
        if (n < 13) raise(QGPU_ERR_NOT_SUPPORTED, W, "needs at least 13 qubits");
        if (t.empty() || t.size() > 6) raise(QGPU_ERR_OUT_OF_RANGE, W, "target");
        std::vector<int> q;
        for (uint64_t x : t) {
            if (x >= uint64_t(n)) raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
            q.push_back(int(x));
        }
        std::vector<int> q6 = q;
        for (int x = 0; q6.size() < 6; ++x)
            if (std::find(q6.begin(), q6.end(), x) == q6.end()) q6.push_back(x);
        uint64_t DA = uint64_t(1) << q.size();
        std::vector<cd> G(reinterpret_cast<const cd*>(U), reinterpret_cast<const cd*>(U) + DA * DA);
        std::vector<cd> U6 = qgpu::embed(G, q, q6);
        std::vector<float> B(128 * 128);
        qgpu::fused6_matrix(U6.data(), B.data());
        // |psi|^2 first: its block partials use the context scratch, which
        // the block matrix takes over after them in stream order
        const double* norm2 = qgpu::fused_norm_prepare(s->ctx, s->data, s->elems);
        auto* scr = static_cast<unsigned char*>(qgpu::ctx_scratch(s->ctx, 2 * 65536));
        float* dB = reinterpret_cast<float*>(scr);
        QG_CUDA(cudaMemcpyAsync(dB, B.data(), B.size() * sizeof(float), cudaMemcpyHostToDevice,
                                s->ctx->stream));
        qgpu::fused6_images(s->ctx, dB, scr + 65536, 1);
        int tb[6];
        for (int j = 0; j < 6; ++j) tb[j] = n - 1 - q6[size_t(j)];
        qgpu::launch_fused6_tc(s->ctx, s->data, n, tb, scr + 65536, norm2);
        if (qgpu::fused_error(s->ctx))
            raise(QGPU_ERR_TIMEOUT, W, "tensor-core pass timed out");
    });
}

} // extern "C"
