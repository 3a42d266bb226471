// engine.cpp -- device-resident circuit engines: QEngine / QDensityEngine /
// QNoisyEngine semantics over a qgpu_circuit.
//
// Follows include/qpp/classes/qengine.hpp (execute(reps) :1341-1405,
// execute(it) :1271-1316, visit_gate_step_ :533-631, visit_measurement_step_
// :639-823, relative positions after destructive measurements) and
// qnoisy_engine.hpp:105-139 (before every step, one Kraus pick per
// non-measured qudit, recorded per step). The state stays in HBM between
// steps; only measurement probabilities (FP64 sums) cross to the host.
//
// Randomness: one std::mt19937 per engine, drawn in qpp's order -- a
// measurement draws one full-basis index from the |amplitude|^2 (or
// diagonal) distribution exactly like std::discrete_distribution
// (generate_canonical<double, 53> then the first index whose prefix sum
// reaches u * total; prefix sums in FP64 on the device), and noise draws one
// Kraus index per qudit per step. Every outcome and Kraus index is recorded;
// a replay list forces them instead (parity against the oracle).
//
// Noise speed-up (exact up to rounding): a Kraus operator proportional to
// the identity is skipped; one proportional to a unitary is applied as that
// unitary without the renormalisation pass.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <random>

#include "capi_common.hpp"
#include "circuit.hpp"
#include "kernels.hpp"
#include "ops.hpp"

using qgpu::cd;

struct qgpu_engine {
    qgpu_ctx* ctx = nullptr;
    qgpu_circuit* circ = nullptr;
    qgpu_kind kind = QGPU_KET;
    qgpu_prec prec = QGPU_C128;
    std::mt19937 gen;
    // noise model (one Kraus set on a single qudit of dimension d)
    bool noisy = false;
    bool state_dependent = false;
    std::vector<std::vector<cd>> Ks;
    std::vector<double> kprobs;
    std::vector<int> kclass; // 0 general, 1 identity-like, 2 unitary-like
    std::vector<std::vector<cd>> kunit; // normalised unitary for class 2
    // optional initial state
    qgpu_state* init = nullptr;
    // run state
    qgpu_state* st = nullptr;
    std::vector<uint64_t> dits;
    std::vector<double> probs;
    std::vector<char> measured; // original qudit measured destructively
    std::map<std::vector<uint64_t>, uint64_t> stats;
    std::vector<std::vector<uint64_t>> noise_results; // per step
    std::vector<uint64_t> rec_outcomes, rec_noise;
    bool replay = false;
    std::vector<uint64_t> forced_outcomes, forced_noise;
    size_t fo_pos = 0, fn_pos = 0;
    ~qgpu_engine() {
        qgpu::free_state(st);
        qgpu::free_state(init);
    }
};

namespace qgpu {
namespace {

const char* kExec = "qpp::QEngineT::execute()";

uint64_t rel_pos(const qgpu_engine* e, uint64_t q) {
    if (e->measured[q])
        raise(QGPU_ERR_QUDIT_ALREADY_MEASURED, kExec, "qudit measured destructively");
    uint64_t r = 0;
    for (uint64_t i = 0; i < q; ++i)
        if (!e->measured[i]) ++r;
    return r;
}

void reset_state(qgpu_engine* e) {
    free_state(e->st);
    e->st = nullptr;
    std::vector<uint64_t> dims(e->circ->nq, e->circ->d);
    if (e->init) {
        e->st = new_state(e->ctx, e->init->kind, e->prec, e->init->dims, false);
        QG_CUDA(cudaMemcpyAsync(e->st->data, e->init->data, e->init->bytes(),
                                cudaMemcpyDeviceToDevice, e->ctx->stream));
    } else {
        e->st = new_state(e->ctx, e->kind, e->prec, dims, true);
        if (e->prec == QGPU_C128) {
            static const double one[2] = {1.0, 0.0};
            QG_CUDA(cudaMemcpyAsync(e->st->data, one, sizeof(one), cudaMemcpyHostToDevice,
                                    e->ctx->stream));
        } else {
            static const float one[2] = {1.0f, 0.0f};
            QG_CUDA(cudaMemcpyAsync(e->st->data, one, sizeof(one), cudaMemcpyHostToDevice,
                                    e->ctx->stream));
        }
    }
    e->dits.assign(e->circ->nc, 0);
    e->probs.assign(e->circ->nc, 0.0);
    e->measured.assign(e->circ->nq, 0);
    e->noise_results.assign(e->circ->steps.size(), {});
}

// Draw from weights w with std::discrete_distribution semantics.
uint64_t draw(std::mt19937& gen, const std::vector<double>& w) {
    std::discrete_distribution<uint64_t> dd(w.begin(), w.end());
    return dd(gen);
}

// weight of digit `val` of subsystem t (probability of that outcome)
double digit_weight(qgpu_state* s, uint64_t t, uint64_t val) {
    VSpace k = vspace_ket(s->dims);
    SegPlan outer = plan_free(k, {int(t)}, 0);
    std::vector<uint64_t> off = target_offsets(k, {int(t)});
    std::vector<double> m = reduce_marginals(s->ctx, s->prec, s->data, outer, off,
                                             s->kind == QGPU_RHO, s->D);
    return m[val];
}

// project subsystem t of s on digit val and renormalise by the kept weight
double project(qgpu_state* s, uint64_t t, uint64_t val) {
    double p = digit_weight(s, t, val);
    if (p <= 0) raise(QGPU_ERR_DIVISION_BY_ZERO, "qpp::measure_seq()", "zero probability");
    VSpace k = vspace_ket(s->dims);
    double scale = s->kind == QGPU_KET ? 1.0 / std::sqrt(p) : 1.0 / p;
    launch_project(s->ctx, s->prec, s->data, s->elems, s->D, s->kind == QGPU_RHO,
                   k.strides[t], s->dims[t], val, scale);
    return p;
}

// remove subsystems `ts` fixed at digits `vals` (the state is already
// projected there): a gather into a smaller state of the same kind
qgpu_state* drop(qgpu_state* s, const std::vector<uint64_t>& ts,
                 const std::vector<uint64_t>& vals) {
    VSpace k = vspace_ket(s->dims);
    std::vector<char> gone(s->dims.size(), 0);
    uint64_t foff = 0;
    for (size_t i = 0; i < ts.size(); ++i) {
        gone[ts[i]] = 1;
        foff += vals[i] * k.strides[ts[i]] * (s->kind == QGPU_RHO ? s->D + 1 : 1);
    }
    std::vector<uint64_t> nd;
    for (size_t q = 0; q < s->dims.size(); ++q)
        if (!gone[q]) nd.push_back(s->dims[q]);
    if (nd.empty()) nd.push_back(1);
    qgpu_state* out = new_state(s->ctx, s->kind, s->prec, nd, false);
    std::vector<uint64_t> od, src;
    if (s->kind == QGPU_RHO)
        for (size_t q = 0; q < s->dims.size(); ++q)
            if (!gone[q]) {
                od.push_back(s->dims[q]);
                src.push_back(k.strides[q] * s->D);
            }
    for (size_t q = 0; q < s->dims.size(); ++q)
        if (!gone[q]) {
            od.push_back(s->dims[q]);
            src.push_back(k.strides[q]);
        }
    launch_gather(s->ctx, s->prec, s->data, out->data, plan_gather(od, src, foff));
    return out;
}

// qpp::measure_seq on the engine state (instruments.hpp:985-1111).
void measure_seq(qgpu_engine* e, const std::vector<uint64_t>& rel, bool destructive,
                 std::vector<uint64_t>& res, std::vector<double>& ps) {
    qgpu_state* s = e->st;
    const size_t k = rel.size();
    res.assign(k, 0);
    ps.assign(k, 0.0);
    if (e->replay) {
        if (e->fo_pos + k > e->forced_outcomes.size())
            raise(QGPU_ERR_OUT_OF_RANGE, kExec, "replay list exhausted (outcomes)");
        for (size_t i = 0; i < k; ++i) res[i] = e->forced_outcomes[e->fo_pos++];
    } else {
        double u = std::generate_canonical<double, std::numeric_limits<double>::digits>(e->gen);
        uint64_t idx = prefix_search(s->ctx, s->prec, s->data, s->D, s->kind == QGPU_RHO, u,
                                     nullptr);
        uint64_t r = idx;
        std::vector<uint64_t> dg(s->dims.size());
        for (size_t q = s->dims.size(); q-- > 0;) {
            dg[q] = r % s->dims[q];
            r /= s->dims[q];
        }
        for (size_t i = 0; i < k; ++i) res[i] = dg[rel[i]];
    }
    for (uint64_t v : res) e->rec_outcomes.push_back(v);
    bool small_rho = s->kind == QGPU_RHO && s->dims.size() <= 10;
    std::vector<size_t> order(k);
    for (size_t i = 0; i < k; ++i) order[i] = i;
    if (destructive && !small_rho)
        std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return rel[a] > rel[b]; });
    for (size_t c = 0; c < k; ++c) {
        size_t i = order[c];
        ps[i] = project(e->st, rel[i], res[i]);
        if (destructive && !small_rho) {
            qgpu_state* nxt = drop(e->st, {rel[i]}, {res[i]});
            free_state(e->st);
            e->st = nxt;
        }
    }
    if (destructive && small_rho) {
        qgpu_state* nxt = drop(e->st, rel, res);
        free_state(e->st);
        e->st = nxt;
    }
}

void apply_noise(qgpu_engine* e, size_t step_idx) {
    const uint64_t nq = e->circ->nq;
    for (uint64_t q = 0; q < nq; ++q) {
        if (e->measured[q]) continue;
        uint64_t r = rel_pos(e, q);
        uint64_t kidx;
        if (e->replay) {
            if (e->fn_pos >= e->forced_noise.size())
                raise(QGPU_ERR_OUT_OF_RANGE, kExec, "replay list exhausted (noise)");
            kidx = e->forced_noise[e->fn_pos++];
        } else if (!e->state_dependent) {
            kidx = draw(e->gen, e->kprobs);
        } else {
            // noise.hpp:100-121: p_i = tr(K_i rho_q K_i^dagger) from the
            // reduced state of the qudit
            std::vector<uint64_t> comp;
            for (uint64_t i = 0; i < e->st->dims.size(); ++i)
                if (i != r) comp.push_back(i);
            qgpu_state* red = op_ptrace(e->st, comp);
            uint64_t d = e->st->dims[r];
            std::vector<cd> rho(d * d);
            std::vector<double> tmp(2 * d * d);
            if (red->prec == QGPU_C128) {
                QG_CUDA(cudaMemcpyAsync(tmp.data(), red->data, red->bytes(),
                                        cudaMemcpyDeviceToHost, e->ctx->stream));
                QG_CUDA(cudaStreamSynchronize(e->ctx->stream));
                for (uint64_t i = 0; i < d * d; ++i) rho[i] = cd(tmp[2 * i], tmp[2 * i + 1]);
            } else {
                std::vector<float> tf(2 * d * d);
                QG_CUDA(cudaMemcpyAsync(tf.data(), red->data, red->bytes(),
                                        cudaMemcpyDeviceToHost, e->ctx->stream));
                QG_CUDA(cudaStreamSynchronize(e->ctx->stream));
                for (uint64_t i = 0; i < d * d; ++i) rho[i] = cd(tf[2 * i], tf[2 * i + 1]);
            }
            free_state(red);
            std::vector<double> w(e->Ks.size());
            for (size_t i = 0; i < e->Ks.size(); ++i) {
                const auto& K = e->Ks[i];
                double tr = 0;
                for (uint64_t a = 0; a < d; ++a)      // (K rho K^dagger)(a, a)
                    for (uint64_t b = 0; b < d; ++b)
                        for (uint64_t c = 0; c < d; ++c)
                            tr += (K[a + b * d] * rho[b + c * d] * std::conj(K[a + c * d])).real();
                w[i] = tr;
            }
            kidx = draw(e->gen, w);
        }
        e->rec_noise.push_back(kidx);
        e->noise_results[step_idx].push_back(kidx);
        int cls = e->kclass[kidx];
        uint64_t d = e->st->dims[r];
        if (cls == 1) continue;
        if (cls == 2) {
            op_apply(e->st, e->kunit[kidx].data(), d, {r});
        } else {
            op_apply(e->st, e->Ks[kidx].data(), d, {r});
            if (!op_normalize(e->st))
                raise(QGPU_ERR_DIVISION_BY_ZERO, "qpp::normalize()", "Division by zero!");
        }
    }
}

void run_step(qgpu_engine* e, const Step& st, size_t idx) {
    if (e->noisy) apply_noise(e, idx);
    auto relv = [&](const std::vector<uint64_t>& v) {
        std::vector<uint64_t> r;
        for (uint64_t q : v) r.push_back(rel_pos(e, q));
        return r;
    };
    switch (st.kind) {
        case StepKind::Gate:
        case StepKind::Fan:
        case StepKind::Ctrl:
        case StepKind::CtrlFan: {
            Step s2 = st;
            s2.target = relv(st.target);
            if (st.kind == StepKind::Ctrl || st.kind == StepKind::CtrlFan) s2.ctrl = relv(st.ctrl);
            apply_step(e->st, s2);
            break;
        }
        case StepKind::CCtrl:
        case StepKind::CCtrlFan: {
            // qengine.hpp:582-630: apply U^first when all shifted dits agree
            uint64_t d = e->circ->d;
            auto val = [&](size_t m) {
                uint64_t v = e->dits[st.ctrl[m]];
                return st.has_shift ? (v + st.shift[m]) % d : v;
            };
            uint64_t first = val(0);
            for (size_t m = 1; m < st.ctrl.size(); ++m)
                if (val(m) != first) return;
            if (first == 0) return; // U^0 = identity
            std::vector<cd> Up = mat_pow(st.U, st.DU, first);
            auto t = relv(st.target);
            if (st.kind == StepKind::CCtrlFan) {
                for (uint64_t x : t) op_apply(e->st, Up.data(), st.DU, {x});
            } else {
                op_apply(e->st, Up.data(), st.DU, t);
            }
            break;
        }
        case StepKind::Channel: {
            Step s2 = st;
            s2.target = relv(st.target);
            if (e->st->kind == QGPU_RHO) {
                apply_step(e->st, s2);
                break;
            }
            // ket: pick branch i with probability ||K_i psi||^2 (one draw),
            // then psi <- K_i psi / ||K_i psi|| (noise.hpp:132-160)
            const uint64_t DK = st.DU;
            std::vector<double> w(st.nK);
            for (uint32_t i = 0; i < st.nK; ++i) {
                qgpu_state* tmp = new_state(e->ctx, e->st->kind, e->st->prec, e->st->dims, false);
                QG_CUDA(cudaMemcpyAsync(tmp->data, e->st->data, e->st->bytes(),
                                        cudaMemcpyDeviceToDevice, e->ctx->stream));
                op_apply(tmp, st.U.data() + size_t(i) * DK * DK, DK, s2.target);
                w[i] = op_norm2(tmp);
                free_state(tmp);
            }
            uint64_t k;
            if (e->replay) {
                if (e->fn_pos >= e->forced_noise.size())
                    raise(QGPU_ERR_OUT_OF_RANGE, kExec, "replay list exhausted (noise)");
                k = e->forced_noise[e->fn_pos++];
            } else {
                k = draw(e->gen, w);
            }
            e->rec_noise.push_back(k);
            op_apply(e->st, st.U.data() + size_t(k) * DK * DK, DK, s2.target);
            if (!op_normalize(e->st))
                raise(QGPU_ERR_DIVISION_BY_ZERO, "qpp::normalize()", "Division by zero!");
            break;
        }
        case StepKind::Measure: {
            std::vector<uint64_t> res;
            std::vector<double> ps;
            measure_seq(e, relv(st.target), st.destructive, res, ps);
            for (size_t i = 0; i < res.size() && st.c_reg + i < e->dits.size(); ++i) {
                e->dits[st.c_reg + i] = res[i];
                e->probs[st.c_reg + i] = ps[i];
            }
            if (st.destructive)
                for (uint64_t q : st.target) e->measured[q] = 1;
            break;
        }
        default:
            break;
    }
}

int classify(const std::vector<cd>& K, uint64_t d, std::vector<cd>& unit) {
    // K^dagger K = c I ?
    double c = 0;
    for (uint64_t a = 0; a < d; ++a) c += std::norm(K[a]);
    bool iso = c > 0;
    for (uint64_t i = 0; i < d && iso; ++i)
        for (uint64_t j = 0; j < d && iso; ++j) {
            cd s = 0;
            for (uint64_t a = 0; a < d; ++a) s += std::conj(K[a + i * d]) * K[a + j * d];
            cd want = i == j ? cd(c) : cd(0.0);
            if (std::abs(s - want) > 1e-14 * std::max(1.0, c)) iso = false;
        }
    if (!iso) return 0;
    double sc = 1.0 / std::sqrt(c);
    unit.resize(d * d);
    for (uint64_t i = 0; i < d * d; ++i) unit[i] = K[i] * sc;
    // identity up to a global phase?
    cd ph = unit[0];
    bool idl = std::abs(std::abs(ph) - 1.0) < 1e-14;
    for (uint64_t i = 0; i < d && idl; ++i)
        for (uint64_t j = 0; j < d && idl; ++j) {
            cd want = i == j ? ph : cd(0.0);
            if (std::abs(unit[i + j * d] - want) > 1e-14) idl = false;
        }
    return idl ? 1 : 2;
}

} // namespace
} // namespace qgpu

using qgpu::guarded;
using qgpu::need_handle;
using qgpu::raise;

extern "C" {

qgpu_status qgpu_engine_create(qgpu_ctx* ctx, qgpu_circuit* c, qgpu_kind kind,
                               qgpu_prec prec, qgpu_engine** out) {
    return guarded([&] {
        need_handle(ctx);
        need_handle(c);
        if (!out) raise(QGPU_ERR_INVALID_ARGUMENT, "qgpu_engine_create()", "out");
        auto* e = new qgpu_engine;
        e->ctx = ctx;
        e->circ = c;
        e->kind = kind;
        e->prec = prec;
        e->gen.seed(std::mt19937::default_seed);
        *out = e;
    });
}

qgpu_status qgpu_engine_destroy(qgpu_engine* e) {
    return guarded([&] { delete e; });
}

qgpu_status qgpu_engine_set_seed(qgpu_engine* e, uint64_t seed) {
    return guarded([&] {
        need_handle(e);
        e->gen.seed(static_cast<std::mt19937::result_type>(seed));
    });
}

qgpu_status qgpu_engine_set_noise(qgpu_engine* e, const double* Ks, uint32_t nK, uint64_t d,
                                  const double* probs) {
    return guarded([&] {
        need_handle(e);
        if (nK == 0) {
            e->noisy = false;
            return;
        }
        if (d != e->circ->d)
            raise(QGPU_ERR_DIMS_MISMATCH_MATRIX, "qpp::QNoisyEngineT::QNoisyEngineT()", "noise/d");
        const cd* K = reinterpret_cast<const cd*>(Ks);
        e->Ks.clear();
        e->kclass.clear();
        e->kunit.clear();
        for (uint32_t i = 0; i < nK; ++i) {
            std::vector<cd> k(K + size_t(i) * d * d, K + size_t(i + 1) * d * d);
            std::vector<cd> u;
            e->kclass.push_back(qgpu::classify(k, d, u));
            e->kunit.push_back(u);
            e->Ks.push_back(k);
        }
        e->state_dependent = probs == nullptr;
        e->kprobs.clear();
        if (probs) e->kprobs.assign(probs, probs + nK);
        e->noisy = true;
    });
}

qgpu_status qgpu_engine_set_state(qgpu_engine* e, const qgpu_state* s) {
    return guarded([&] {
        need_handle(e);
        need_handle(s);
        qgpu::free_state(e->init);
        e->init = nullptr;
        e->init = qgpu::new_state(e->ctx, s->kind, e->prec, s->dims, false);
        if (s->prec == e->prec)
            QG_CUDA(cudaMemcpyAsync(e->init->data, s->data, s->bytes(),
                                    cudaMemcpyDeviceToDevice, e->ctx->stream));
        else
            qgpu::launch_convert(e->ctx, s->data, s->prec, e->init->data, e->prec, s->elems);
    });
}

qgpu_status qgpu_engine_set_replay(qgpu_engine* e, const uint64_t* outcomes, uint64_t n_out,
                                   const uint64_t* noise, uint64_t n_noise) {
    return guarded([&] {
        need_handle(e);
        e->replay = outcomes != nullptr || noise != nullptr;
        e->forced_outcomes.assign(outcomes, outcomes ? outcomes + n_out : outcomes);
        e->forced_noise.assign(noise, noise ? noise + n_noise : noise);
        e->fo_pos = e->fn_pos = 0;
    });
}

qgpu_status qgpu_engine_execute(qgpu_engine* e, uint64_t reps) {
    return guarded([&] {
        need_handle(e);
        if (reps == 0) raise(QGPU_ERR_OUT_OF_RANGE, "qpp::QEngineT::execute()", "reps");
        e->stats.clear();
        e->rec_outcomes.clear();
        e->rec_noise.clear();
        e->fo_pos = e->fn_pos = 0;
        for (uint64_t rep = 0; rep < reps; ++rep) {
            qgpu::reset_state(e);
            for (size_t i = 0; i < e->circ->steps.size(); ++i)
                qgpu::run_step(e, e->circ->steps[i], i);
            e->stats[e->dits] += 1;
        }
        QG_CUDA(cudaStreamSynchronize(e->ctx->stream));
    });
}

qgpu_status qgpu_engine_get_dits(const qgpu_engine* e, uint64_t* dits, double* probs) {
    return guarded([&] {
        need_handle(e);
        if (dits) std::copy(e->dits.begin(), e->dits.end(), dits);
        if (probs) std::copy(e->probs.begin(), e->probs.end(), probs);
    });
}

qgpu_status qgpu_engine_get_state(const qgpu_engine* e, qgpu_state** out) {
    return guarded([&] {
        need_handle(e);
        if (!e->st) raise(QGPU_ERR_INVALID_HANDLE, "qpp::QEngineT::get_state()", "not executed");
        qgpu_state* c = qgpu::new_state(e->ctx, e->st->kind, e->st->prec, e->st->dims, false);
        QG_CUDA(cudaMemcpyAsync(c->data, e->st->data, e->st->bytes(), cudaMemcpyDeviceToDevice,
                                e->ctx->stream));
        *out = c;
    });
}

// number of distinct outcome vectors, then (counts, dits) when arrays given
qgpu_status qgpu_engine_get_stats(const qgpu_engine* e, uint64_t* n_distinct,
                                  uint64_t* counts, uint64_t* outcomes) {
    return guarded([&] {
        need_handle(e);
        if (n_distinct) *n_distinct = e->stats.size();
        size_t i = 0, nc = e->circ->nc;
        for (auto& kv : e->stats) {
            if (counts) counts[i] = kv.second;
            if (outcomes) std::copy(kv.first.begin(), kv.first.end(), outcomes + i * nc);
            ++i;
        }
    });
}

// recorded random choices of the last execute(): measurement outcome dits
// (in execution order) and Kraus indices (step by step, qudit by qudit)
qgpu_status qgpu_engine_get_record(const qgpu_engine* e, uint64_t* n_out, uint64_t* outcomes,
                                   uint64_t* n_noise, uint64_t* noise) {
    return guarded([&] {
        need_handle(e);
        if (n_out) *n_out = e->rec_outcomes.size();
        if (outcomes) std::copy(e->rec_outcomes.begin(), e->rec_outcomes.end(), outcomes);
        if (n_noise) *n_noise = e->rec_noise.size();
        if (noise) std::copy(e->rec_noise.begin(), e->rec_noise.end(), noise);
    });
}

} // extern "C"
