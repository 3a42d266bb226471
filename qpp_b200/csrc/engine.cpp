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
#include <set>

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
    // engine state (qengine_state.hpp:52-157): the current state (null:
    // |0...0> not materialised yet), dits, probabilities, and which qudits
    // were measured destructively
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
    ~qgpu_engine() { qgpu::free_state(st); }
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

// dits, probabilities and measured flags back to their initial values
// (QEngineState::reset, qengine_state.hpp:115-157)
void clear_registers(qgpu_engine* e) {
    e->dits.assign(e->circ->nc, 0);
    e->probs.assign(e->circ->nc, 0.0);
    e->measured.assign(e->circ->nq, 0);
}

// materialise |0...0> (ket) or |0...0><0...0| when the engine has no state
void ensure_state(qgpu_engine* e) {
    if (e->dits.size() != e->circ->nc || e->measured.size() != e->circ->nq) clear_registers(e);
    if (e->noise_results.size() != e->circ->steps.size())
        e->noise_results.resize(e->circ->steps.size());
    if (e->st) return;
    std::vector<uint64_t> dims(e->circ->nq, e->circ->d);
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

qgpu_state* copy_state(const qgpu_state* s) {
    qgpu_state* c = new_state(s->ctx, s->kind, s->prec, s->dims, false);
    QG_CUDA(cudaMemcpyAsync(c->data, s->data, s->bytes(), cudaMemcpyDeviceToDevice,
                            s->ctx->stream));
    return c;
}

// A copy of the engine state (qeng_st_ copies in qengine.hpp:316-345).
struct Snapshot {
    qgpu_state* st = nullptr;
    std::vector<uint64_t> dits;
    std::vector<double> probs;
    std::vector<char> measured;
    void take(qgpu_engine* e) { // move the engine's state in
        st = e->st;
        e->st = nullptr;
        dits = e->dits;
        probs = e->probs;
        measured = e->measured;
    }
    void copy_from(const qgpu_engine* e) {
        st = copy_state(e->st);
        dits = e->dits;
        probs = e->probs;
        measured = e->measured;
    }
    void restore_copy(qgpu_engine* e) const {
        free_state(e->st);
        e->st = copy_state(st);
        e->dits = dits;
        e->probs = probs;
        e->measured = measured;
    }
    void restore_move(qgpu_engine* e) {
        free_state(e->st);
        e->st = st;
        st = nullptr;
        e->dits = dits;
        e->probs = probs;
        e->measured = measured;
    }
    ~Snapshot() { free_state(st); }
};

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
// big-endian mixed-radix digits of a full-basis index (util.hpp:58-84)
std::vector<uint64_t> digits_of(uint64_t idx, const std::vector<uint64_t>& dims) {
    std::vector<uint64_t> dg(dims.size());
    for (size_t q = dims.size(); q-- > 0;) {
        dg[q] = idx % dims[q];
        idx /= dims[q];
    }
    return dg;
}

double canonical(std::mt19937& gen) {
    return std::generate_canonical<double, std::numeric_limits<double>::digits>(gen);
}

} // namespace

// The collapse of qpp::measure_seq (instruments.hpp:1024-1093) for given
// outcomes: project each target on its outcome and renormalise (ps = the
// conditional probabilities); destructive: drop the targets (one at a time
// in descending order, or all at the end for density matrices of <= 10
// subsystems, as qpp does). `s` may be replaced by a smaller state.
void collapse_seq(qgpu_state*& s, const std::vector<uint64_t>& tgt, bool destructive,
                  const std::vector<uint64_t>& res, std::vector<double>& ps) {
    const size_t k = tgt.size();
    ps.assign(k, 0.0);
    const bool small_rho = s->kind == QGPU_RHO && s->dims.size() <= 10;
    std::vector<size_t> order(k);
    for (size_t i = 0; i < k; ++i) order[i] = i;
    if (destructive && !small_rho)
        std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return tgt[a] > tgt[b]; });
    for (size_t c = 0; c < k; ++c) {
        size_t i = order[c];
        ps[i] = project(s, tgt[i], res[i]);
        if (destructive && !small_rho) {
            qgpu_state* nxt = drop(s, {tgt[i]}, {res[i]});
            free_state(s);
            s = nxt;
        }
    }
    if (destructive && small_rho) {
        qgpu_state* nxt = drop(s, tgt, res);
        free_state(s);
        s = nxt;
    }
}

// One full-basis draw (qpp::sample, instruments.hpp:746-818): the digits of
// the targets.
std::vector<uint64_t> sample_once(const qgpu_state* s, const std::vector<uint64_t>& tgt,
                                  double u) {
    uint64_t idx =
        prefix_search(s->ctx, s->prec, s->data, s->D, s->kind == QGPU_RHO, u, nullptr);
    std::vector<uint64_t> dg = digits_of(idx, s->dims), res(tgt.size());
    for (size_t i = 0; i < tgt.size(); ++i) res[i] = dg[tgt[i]];
    return res;
}

namespace {

void measure_seq(qgpu_engine* e, const std::vector<uint64_t>& rel, bool destructive,
                 std::vector<uint64_t>& res, std::vector<double>& ps) {
    const size_t k = rel.size();
    res.assign(k, 0);
    if (e->replay) {
        if (e->fo_pos + k > e->forced_outcomes.size())
            raise(QGPU_ERR_OUT_OF_RANGE, kExec, "replay list exhausted (outcomes)");
        for (size_t i = 0; i < k; ++i) res[i] = e->forced_outcomes[e->fo_pos++];
    } else {
        res = sample_once(e->st, rel, canonical(e->gen));
    }
    for (uint64_t v : res) e->rec_outcomes.push_back(v);
    collapse_seq(e->st, rel, destructive, res, ps);
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

// Executes one step; returns how many following steps to skip (a runtime IF
// that is false jumps past its block and its END, qengine.hpp:853-861).
uint32_t run_step(qgpu_engine* e, const Step& st, size_t idx) {
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
                if (val(m) != first) return 0;
            if (first == 0) return 0; // U^0 = identity
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
        case StepKind::CondIf: {
            uint64_t v = 0;
            for (size_t i = 0; i < st.ctrl.size(); ++i)
                v |= (e->dits[st.ctrl[i]] & 1u) << i;
            return v == st.c_reg ? 0u : st.nK;
        }
        case StepKind::CondEnd:
            break;
        case StepKind::Reset: {
            // qpp::reset (instruments.hpp:1148-1206) on the relative
            // positions: measure_seq without destruction (one draw), then
            // Xd^(d - r) on each target
            const std::vector<uint64_t> rel = relv(st.target);
            std::vector<uint64_t> res;
            std::vector<double> ps;
            measure_seq(e, rel, false, res, ps);
            const uint64_t d = e->circ->d;
            for (size_t i = 0; i < rel.size(); ++i) {
                std::vector<cd> X(d * d, 0.0);
                for (uint64_t j = 0; j < d; ++j) X[((j + d - res[i]) % d) + j * d] = 1.0;
                op_apply(e->st, X.data(), d, {rel[i]});
            }
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
    return 0;
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

bool is_measurement(const Step& s) { return s.kind == StepKind::Measure || s.kind == StepKind::Reset; }
bool is_runtime(const Step& s) { return s.kind == StepKind::CondIf || s.kind == StepKind::CondEnd; }
bool is_cctrl(const Step& s) { return s.kind == StepKind::CCtrl || s.kind == StepKind::CCtrlFan; }

// (ctrl, target, c_reg) of a step as qpp's
// extract_ctrl_target_ps_vals_c_reg sees them (qcircuit.hpp:7371-7440)
void step_sets(const Step& s, std::vector<uint64_t>& ctrl, std::vector<uint64_t>& target,
               std::vector<uint64_t>& creg) {
    ctrl.clear();
    creg.clear();
    target = s.target;
    switch (s.kind) {
        case StepKind::Measure:
            for (size_t i = 0; i < s.target.size(); ++i) creg.push_back(s.c_reg + i);
            break;
        case StepKind::CCtrl:
        case StepKind::CCtrlFan:
            creg = s.ctrl;
            break;
        case StepKind::Ctrl:
        case StepKind::CtrlFan:
            ctrl = s.ctrl;
            break;
        default:
            break;
    }
}

bool overlap(const std::vector<uint64_t>& a, const std::vector<uint64_t>& b) {
    for (uint64_t x : a)
        if (std::find(b.begin(), b.end(), x) != b.end()) return true;
    return false;
}

// qpp::internal::can_swap (qcircuit.hpp:7465-7492): controls, targets and
// classical dits pairwise disjoint (a control may meet a target)
bool can_swap(const Step& a, const Step& b) {
    std::vector<uint64_t> c1, t1, r1, c2, t2, r2;
    step_sets(a, c1, t1, r1);
    step_sets(b, c2, t2, r2);
    return !overlap(c1, c2) && !overlap(t1, t2) && !overlap(r1, r2);
}

// qpp::internal::canonical_form (qcircuit.hpp:7556-7631): from the first
// measurement on, classically controlled steps and then measurements are
// bubbled towards the end past the steps they can swap with (stable: two
// steps of the same class are never exchanged). Only for reps > 1.
std::vector<size_t> canonical_order(const qgpu_circuit* c, bool canonical) {
    const size_t ns = c->steps.size();
    std::vector<size_t> order(ns);
    for (size_t i = 0; i < ns; ++i) order[i] = i;
    if (!canonical) return order;
    for (const Step& s : c->steps) // runtime steps: the circuit as it is
        if (is_runtime(s)) return order;
    size_t first = 0;
    while (first < ns && !is_measurement(c->steps[first])) ++first;
    auto push_back_class = [&](bool (*cls)(const Step&)) {
        for (size_t r = ns; r-- > first;) {
            if (!cls(c->steps[order[r]])) continue;
            for (size_t j = r; j + 1 < ns; ++j) {
                const Step& cur = c->steps[order[j]];
                const Step& nxt = c->steps[order[j + 1]];
                if (can_swap(cur, nxt) && !cls(nxt)) std::swap(order[j], order[j + 1]);
                else break;
            }
        }
    };
    push_back_class(is_cctrl);
    push_back_class(is_measurement);
    return order;
}

// A QCircuit::QFT / TFQ block met in its own step order by a noiseless
// engine runs as one transform (op_apply_qft) instead of its k(k+1)/2 gate
// steps; returns the steps consumed, 0 when the block does not apply.
size_t run_block(qgpu_engine* e, const std::vector<size_t>& order, size_t i) {
    const Step& st = e->circ->steps[order[i]];
    if (e->noisy || st.block_len < 2 || i + st.block_len > order.size()) return 0;
    for (size_t m = 1; m < st.block_len; ++m)
        if (order[i + m] != order[i] + m) return 0;
    std::vector<uint64_t> rel;
    for (uint64_t q : st.block_target) {
        if (e->measured[q]) return 0;
        rel.push_back(rel_pos(e, q));
    }
    op_apply_qft(e->st, rel, e->circ->d, st.block_swap, st.block_inverse);
    return st.block_len;
}

// qengine.hpp:240-345: steps order[pos..] executed reps times, each from
// the engine state at entry; the statistics count every repetition that
// measured something; the engine keeps the first repetition's state.
void repeat_steps(qgpu_engine* e, const std::vector<size_t>& order, size_t pos, uint64_t reps) {
    Snapshot entry, first;
    if (reps > 1) entry.copy_from(e);
    for (uint64_t rep = 0; rep < reps; ++rep) {
        bool measured = false;
        for (size_t i = pos; i < order.size(); ++i) {
            const Step& s = e->circ->steps[order[i]];
            if (is_measurement(s)) measured = true;
            if (size_t b = run_block(e, order, i)) {
                i += b - 1;
                continue;
            }
            i += run_step(e, s, order[i]); // a false IF skips its block
        }
        if (measured) e->stats[e->dits] += 1;
        if (reps == 1) break;
        if (rep == 0) {
            first.take(e);
            entry.restore_copy(e);
        } else if (rep + 1 < reps) {
            entry.restore_copy(e);
        }
    }
    if (reps > 1) first.restore_move(e);
}

// qengine.hpp:374-481 (no post-selection steps here): the steps from pos on
// are all projective measurements, so the measurement steps run once (the
// engine's state and dits) and every further repetition is one full-basis
// sample of the pre-measurement state, written into the dits that the
// measurements would fill. The RNG is consumed in qpp's order: one sample,
// the measurement steps, then one sample per further repetition. Returns
// false (nothing done) when two classical dits read the same qudit, where
// qpp's fill loop reads past its sample.
bool sample_steps(qgpu_engine* e, const std::vector<size_t>& order, size_t pos, uint64_t reps) {
    std::map<uint64_t, uint64_t> c_q; // dit -> qudit
    for (size_t i = pos; i < order.size(); ++i) {
        const Step& s = e->circ->steps[order[i]];
        for (size_t q = 0; q < s.target.size(); ++q) c_q[s.c_reg + q] = s.target[q];
    }
    if (c_q.empty()) return false;
    std::set<uint64_t> from_set;
    for (auto& kv : c_q) from_set.insert(kv.second);
    if (from_set.size() != c_q.size()) return false;
    std::vector<uint64_t> sample_from(from_set.begin(), from_set.end());
    qgpu_state* pre = copy_state(e->st);
    struct Del {
        qgpu_state* s;
        ~Del() { free_state(s); }
    } del{pre};
    (void)canonical(e->gen); // rep 0's sample (it only checks post-selection)
    for (size_t i = pos; i < order.size(); ++i) run_step(e, e->circ->steps[order[i]], order[i]);
    e->stats[e->dits] += 1;
    if (reps == 1) return true;
    std::vector<double> us(reps - 1);
    for (auto& u : us) u = canonical(e->gen);
    const bool rho = pre->kind == QGPU_RHO;
    std::vector<uint64_t> idx = prefix_search_many(pre->ctx, pre->prec, pre->data, pre->D, rho, us);
    std::vector<uint64_t> res;
    for (uint64_t x : idx) {
        std::vector<uint64_t> dg = digits_of(x, pre->dims);
        res = e->dits;
        size_t i = 0;
        // qpp fills the dits in increasing dit order from the samples of
        // the qudits in increasing qudit order
        for (auto& kv : c_q)
            if (kv.first < res.size()) res[kv.first] = dg[sample_from[i++]];
            else ++i;
        e->stats[res] += 1;
    }
    return true;
}

} // namespace
} // namespace qgpu

using qgpu::guarded;
using qgpu::need_handle;
using qgpu::raise;

extern "C" {

qgpu_status qgpu_engine_create(qgpu_ctx* ctx, qgpu_circuit* c, qgpu_kind kind,
                               qgpu_prec prec, qgpu_engine** out) {
    return guarded(__func__, [&] {
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
    return guarded(__func__, [&] { delete e; });
}

qgpu_status qgpu_engine_set_seed(qgpu_engine* e, uint64_t seed) {
    return guarded(__func__, [&] {
        need_handle(e);
        e->gen.seed(static_cast<std::mt19937::result_type>(seed));
    });
}

qgpu_status qgpu_engine_set_noise(qgpu_engine* e, const double* Ks, uint32_t nK, uint64_t d,
                                  const double* probs) {
    return guarded(__func__, [&] {
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
    return guarded(__func__, [&] {
        need_handle(e);
        need_handle(s);
        // QEngineT::set_state (qengine.hpp:1191-1214): the state must match
        // the qudits not yet measured destructively
        const char* W = "qpp::QEngineT::set_state()";
        qgpu::ensure_state(e);
        uint64_t n = 0, D = 1;
        for (char m : e->measured)
            if (!m) ++n;
        for (uint64_t i = 0; i < n; ++i) D *= e->circ->d;
        if (s->kind != e->kind) raise(QGPU_ERR_TYPE_MISMATCH, W, "state");
        if (s->D != D) raise(QGPU_ERR_DIMS_NOT_EQUAL, W, "state");
        std::vector<uint64_t> dims(n, e->circ->d);
        if (dims.empty()) dims.push_back(1);
        qgpu_state* c = qgpu::new_state(e->ctx, e->kind, e->prec, dims, false);
        if (s->prec == e->prec)
            QG_CUDA(cudaMemcpyAsync(c->data, s->data, s->bytes(), cudaMemcpyDeviceToDevice,
                                    e->ctx->stream));
        else
            qgpu::launch_convert(e->ctx, s->data, s->prec, c->data, e->prec, s->elems);
        qgpu::free_state(e->st);
        e->st = c;
    });
}

qgpu_status qgpu_engine_reset(qgpu_engine* e, int reset_stats) {
    return guarded(__func__, [&] {
        need_handle(e);
        // QEngineT::reset (qengine.hpp:1251-1260) / QNoisyEngineT::reset
        qgpu::free_state(e->st);
        e->st = nullptr;
        qgpu::clear_registers(e);
        e->noise_results.assign(e->circ->steps.size(), {});
        if (reset_stats) e->stats.clear();
    });
}

qgpu_status qgpu_engine_set_replay(qgpu_engine* e, const uint64_t* outcomes, uint64_t n_out,
                                   const uint64_t* noise, uint64_t n_noise) {
    return guarded(__func__, [&] {
        need_handle(e);
        e->replay = outcomes != nullptr || noise != nullptr;
        e->forced_outcomes.assign(outcomes, outcomes ? outcomes + n_out : outcomes);
        e->forced_noise.assign(noise, noise ? noise + n_noise : noise);
        e->fo_pos = e->fn_pos = 0;
    });
}

qgpu_status qgpu_engine_execute(qgpu_engine* e, uint64_t reps) {
    return guarded(__func__, [&] {
        need_handle(e);
        if (reps == 0)
            raise(QGPU_ERR_OUT_OF_RANGE,
                  e->noisy ? "qpp::QNoisyEngineT::execute()" : "qpp::QEngineT::execute()", "reps");
        qgpu::ensure_state(e);
        e->rec_outcomes.clear();
        e->rec_noise.clear();
        e->fo_pos = e->fn_pos = 0;
        const size_t ns = e->circ->steps.size();
        if (e->noisy) {
            // QNoisyEngineT::execute (qnoisy_engine.hpp:129-139): every step,
            // reps times from the current engine state
            std::vector<size_t> order(ns);
            for (size_t i = 0; i < ns; ++i) order[i] = i;
            qgpu::repeat_steps(e, order, 0, reps);
        } else {
            // QEngineT::execute (qengine.hpp:1341-1405)
            std::vector<uint64_t> full(e->circ->nq, e->circ->d);
            uint64_t D = 1;
            for (uint64_t x : full) D *= x;
            if (e->st->D != D)
                raise(QGPU_ERR_DIMS_NOT_EQUAL, "qpp::internal::QEngineState::reset()", "state");
            qgpu::clear_registers(e);
            std::vector<size_t> order = qgpu::canonical_order(e->circ, reps > 1);
            size_t pos = 0; // the first measurement, reset or runtime step
            while (pos < order.size() && !qgpu::is_measurement(e->circ->steps[order[pos]]) &&
                   !qgpu::is_runtime(e->circ->steps[order[pos]]))
                ++pos;
            for (size_t i = 0; i < pos; ++i) {
                if (size_t b = qgpu::run_block(e, order, i)) {
                    i += b - 1;
                    continue;
                }
                qgpu::run_step(e, e->circ->steps[order[i]], order[i]);
            }
            bool can_sample = reps > 1 && !e->replay && pos < order.size();
            for (size_t i = pos; i < order.size() && can_sample; ++i)
                if (e->circ->steps[order[i]].kind != qgpu::StepKind::Measure) can_sample = false;
            if (!(can_sample && qgpu::sample_steps(e, order, pos, reps)))
                qgpu::repeat_steps(e, order, pos, reps);
        }
        QG_CUDA(cudaStreamSynchronize(e->ctx->stream));
    });
}

qgpu_status qgpu_engine_get_dits(const qgpu_engine* e, uint64_t* dits, double* probs) {
    return guarded(__func__, [&] {
        need_handle(e);
        if (dits) std::copy(e->dits.begin(), e->dits.end(), dits);
        if (probs) std::copy(e->probs.begin(), e->probs.end(), probs);
    });
}

qgpu_status qgpu_engine_get_state(const qgpu_engine* e, qgpu_state** out) {
    return guarded(__func__, [&] {
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
    return guarded(__func__, [&] {
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
    return guarded(__func__, [&] {
        need_handle(e);
        if (n_out) *n_out = e->rec_outcomes.size();
        if (outcomes) std::copy(e->rec_outcomes.begin(), e->rec_outcomes.end(), outcomes);
        if (n_noise) *n_noise = e->rec_noise.size();
        if (noise) std::copy(e->rec_noise.begin(), e->rec_noise.end(), noise);
    });
}


namespace {
bool targets_ok(const std::vector<uint64_t>& t, size_t n) {
    if (t.size() > n) return false;
    std::vector<uint64_t> u = t;
    std::sort(u.begin(), u.end());
    if (std::adjacent_find(u.begin(), u.end()) != u.end()) return false;
    for (uint64_t x : t)
        if (x >= n) return false;
    return true;
}
} // namespace

// qpp::sample(num_samples, A, target, dims) (instruments.hpp:856-940):
// num_samples full-basis draws of |A_i|^2 (ket) or Re A(i, i) (density
// matrix), each reported as the digits of `target`.
qgpu_status qgpu_sample(const qgpu_state* s, const uint64_t* target, uint32_t k,
                        uint64_t num_samples, uint64_t seed, const double* u,
                        uint64_t* results) {
    return guarded(__func__, [&] {
        need_handle(s);
        const char* W = "qpp::sample()";
        std::vector<uint64_t> tgt = qgpu::vec_of(target, k);
        if (!targets_ok(tgt, s->dims.size())) raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
        if (num_samples == 0) raise(QGPU_ERR_OUT_OF_RANGE, W, "num_samples");
        if (!results && k) raise(QGPU_ERR_INVALID_ARGUMENT, W, "results");
        std::vector<double> us(num_samples);
        if (u) {
            for (uint64_t i = 0; i < num_samples; ++i) {
                if (!(u[i] >= 0.0 && u[i] < 1.0)) raise(QGPU_ERR_OUT_OF_RANGE, W, "u");
                us[i] = u[i];
            }
        } else {
            std::mt19937 gen(static_cast<std::mt19937::result_type>(seed));
            for (auto& x : us) x = qgpu::canonical(gen);
        }
        std::vector<uint64_t> idx =
            qgpu::prefix_search_many(s->ctx, s->prec, s->data, s->D, s->kind == QGPU_RHO, us);
        for (uint64_t i = 0; i < num_samples; ++i) {
            std::vector<uint64_t> dg = qgpu::digits_of(idx[i], s->dims);
            for (uint32_t j = 0; j < k; ++j) results[i * k + j] = dg[tgt[j]];
        }
    });
}

// qpp::measure_seq(A, target, dims, destructive) (instruments.hpp:985-1111)
// with value semantics: `s` is unchanged, the post-measurement state is a
// new handle.
qgpu_status qgpu_measure_seq(const qgpu_state* s, const uint64_t* target, uint32_t k,
                             int destructive, uint64_t seed, const uint64_t* forced,
                             uint64_t* results, double* probs, qgpu_state** out) {
    return guarded(__func__, [&] {
        need_handle(s);
        const char* W = "qpp::measure_seq()";
        if (!out) raise(QGPU_ERR_INVALID_ARGUMENT, W, "out");
        std::vector<uint64_t> tgt = qgpu::vec_of(target, k);
        if (!targets_ok(tgt, s->dims.size())) raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
        std::vector<uint64_t> res(k);
        if (forced) {
            for (uint32_t i = 0; i < k; ++i) {
                if (forced[i] >= s->dims[tgt[i]]) raise(QGPU_ERR_OUT_OF_RANGE, W, "forced");
                res[i] = forced[i];
            }
        } else if (k) {
            std::mt19937 gen(static_cast<std::mt19937::result_type>(seed));
            res = qgpu::sample_once(s, tgt, qgpu::canonical(gen));
        }
        qgpu_state* c = qgpu::copy_state(s);
        std::vector<double> ps;
        try {
            qgpu::collapse_seq(c, tgt, destructive != 0, res, ps);
        } catch (...) {
            qgpu::free_state(c);
            throw;
        }
        QG_CUDA(cudaStreamSynchronize(s->ctx->stream));
        if (results) std::copy(res.begin(), res.end(), results);
        if (probs) std::copy(ps.begin(), ps.end(), probs);
        *out = c;
    });
}


namespace {

// one std::discrete_distribution draw from std::mt19937(seed)
uint64_t draw_seeded(const std::vector<double>& w, uint64_t seed) {
    std::mt19937 gen(static_cast<std::mt19937::result_type>(seed));
    return qgpu::draw(gen, w);
}

void scale_state(qgpu_state* s, double f) {
    qgpu::launch_scale(s->ctx, s->prec, s->data, s->elems, qgpu::cd(f, 0.0));
}

const char* kMeasure = "qpp::measure()";

void check_kraus_shape(const qgpu_state* s, const std::vector<uint64_t>& tgt, uint32_t nK,
                       uint64_t DK) {
    if (!targets_ok(tgt, s->dims.size()))
        raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, kMeasure, "dims/target");
    uint64_t Dsub = 1;
    for (uint64_t t : tgt) Dsub *= s->dims[t];
    if (nK == 0) raise(QGPU_ERR_ZERO_SIZE, kMeasure, "Ks");
    if (DK != Dsub) raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, kMeasure, "Ks[0]");
}

// instruments.hpp:429-486 for operators Ks (nK consecutive DK x DK)
void measure_ops(const qgpu_state* s, const qgpu::cd* Ks, uint32_t nK, uint64_t DK,
                 const std::vector<uint64_t>& tgt, bool destructive, std::vector<double>& probs,
                 std::vector<qgpu_state*>& outs) {
    probs.assign(nK, 0.0);
    outs.assign(nK, nullptr);
    try {
        for (uint32_t i = 0; i < nK; ++i) {
            qgpu_state* c = qgpu::copy_state(s);
            qgpu::op_apply(c, Ks + size_t(i) * DK * DK, DK, tgt);
            if (s->kind == QGPU_KET) {
                const double p = qgpu::op_norm2(c);
                probs[i] = p;
                if (p > 0) {
                    scale_state(c, 1.0 / std::sqrt(p));
                    if (destructive) {
                        qgpu_state* r = qgpu::op_ptrace(c, tgt);
                        qgpu::free_state(c);
                        c = r;
                    }
                    outs[i] = c;
                } else {
                    qgpu::free_state(c);
                }
            } else {
                if (destructive) {
                    qgpu_state* r = qgpu::op_ptrace(c, tgt);
                    qgpu::free_state(c);
                    c = r;
                }
                const double p = std::abs(qgpu::op_trace(c));
                probs[i] = p;
                if (p > 0) {
                    scale_state(c, 1.0 / p);
                    outs[i] = c;
                } else {
                    qgpu::free_state(c);
                }
            }
        }
    } catch (...) {
        for (auto*& o : outs) qgpu::free_state(o);
        throw;
    }
}

void finish_measure(const std::vector<double>& probs, std::vector<qgpu_state*>& outs,
                    uint64_t seed, uint64_t* result, double* probs_out, qgpu_state** outs_out) {
    bool any = false;
    for (double p : probs) any = any || p > 0;
    if (!any) {
        for (auto*& o : outs) qgpu::free_state(o);
        raise(QGPU_ERR_DIVISION_BY_ZERO, kMeasure, "all outcome probabilities are zero");
    }
    const uint64_t r = draw_seeded(probs, seed);
    if (result) *result = r;
    if (probs_out) std::copy(probs.begin(), probs.end(), probs_out);
    for (size_t i = 0; i < outs.size(); ++i) {
        if (outs_out) outs_out[i] = outs[i];
        else qgpu::free_state(outs[i]);
    }
}

} // namespace

// qpp::measure(A, Ks, target, dims, destructive) (instruments.hpp:371-494).
qgpu_status qgpu_measure_kraus(const qgpu_state* s, const double* Ks, uint32_t nK, uint64_t DK,
                               const uint64_t* target, uint32_t k, int destructive,
                               uint64_t seed, uint64_t* result, double* probs,
                               qgpu_state** outs) {
    return guarded(__func__, [&] {
        need_handle(s);
        std::vector<uint64_t> tgt = qgpu::vec_of(target, k);
        check_kraus_shape(s, tgt, nK, DK);
        if (!Ks) raise(QGPU_ERR_INVALID_ARGUMENT, kMeasure, "Ks");
        std::vector<double> pr;
        std::vector<qgpu_state*> os;
        measure_ops(s, reinterpret_cast<const qgpu::cd*>(Ks), nK, DK, tgt, destructive != 0, pr,
                    os);
        QG_CUDA(cudaStreamSynchronize(s->ctx->stream));
        finish_measure(pr, os, seed, result, probs, outs);
    });
}

// qpp::measure(A, V, target, dims, destructive) (instruments.hpp:587-712):
// the M columns of V (Dsub x M, column-major) as rank-1 projectors.
qgpu_status qgpu_measure_basis(const qgpu_state* s, const double* V, uint64_t rows, uint64_t M,
                               const uint64_t* target, uint32_t k, int destructive,
                               uint64_t seed, uint64_t* result, double* probs,
                               qgpu_state** outs) {
    return guarded(__func__, [&] {
        need_handle(s);
        std::vector<uint64_t> tgt = qgpu::vec_of(target, k);
        if (!targets_ok(tgt, s->dims.size()))
            raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, kMeasure, "dims/target");
        uint64_t Dsub = 1;
        for (uint64_t t : tgt) Dsub *= s->dims[t];
        if (rows * M == 0 || !V) raise(QGPU_ERR_ZERO_SIZE, kMeasure, "V");
        if (rows != Dsub) raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, kMeasure, "V");
        const qgpu::cd* v = reinterpret_cast<const qgpu::cd*>(V);
        std::vector<qgpu::cd> Ks(size_t(M) * Dsub * Dsub);
        for (uint64_t i = 0; i < M; ++i) // K_i = v_i v_i^dagger
            for (uint64_t c = 0; c < Dsub; ++c)
                for (uint64_t r = 0; r < Dsub; ++r)
                    Ks[i * Dsub * Dsub + r + c * Dsub] = v[i * Dsub + r] * std::conj(v[i * Dsub + c]);
        std::vector<double> pr;
        std::vector<qgpu_state*> os;
        if (s->kind == QGPU_KET && destructive) {
            // <v_i| psi> over the targets (qpp::ip): E = |0><v_i| on the
            // targets, then the targets dropped at digit 0 -- a ket
            pr.assign(M, 0.0);
            os.assign(M, nullptr);
            try {
                std::vector<uint64_t> zeros(tgt.size(), 0);
                for (uint64_t i = 0; i < M; ++i) {
                    std::vector<qgpu::cd> E(Dsub * Dsub, 0.0);
                    for (uint64_t c = 0; c < Dsub; ++c) E[0 + c * Dsub] = std::conj(v[i * Dsub + c]);
                    qgpu_state* c0 = qgpu::copy_state(s);
                    qgpu::op_apply(c0, E.data(), Dsub, tgt);
                    qgpu_state* o = qgpu::drop(c0, tgt, zeros);
                    qgpu::free_state(c0);
                    const double p = qgpu::op_norm2(o);
                    pr[i] = p;
                    if (p > 0) {
                        scale_state(o, 1.0 / std::sqrt(p));
                        os[i] = o;
                    } else {
                        qgpu::free_state(o);
                    }
                }
            } catch (...) {
                for (auto*& o : os) qgpu::free_state(o);
                throw;
            }
        } else {
            measure_ops(s, Ks.data(), uint32_t(M), Dsub, tgt, destructive != 0, pr, os);
        }
        QG_CUDA(cudaStreamSynchronize(s->ctx->stream));
        finish_measure(pr, os, seed, result, probs, outs);
    });
}

// qpp::reset(A, target, dims) (instruments.hpp:1148-1206): measure_seq
// without destruction, then Xd^(d - result) on each target, d = dims[i] for
// the i-th target as qpp indexes it.
qgpu_status qgpu_reset(const qgpu_state* s, const uint64_t* target, uint32_t k, uint64_t seed,
                       qgpu_state** out) {
    return guarded(__func__, [&] {
        need_handle(s);
        const char* W = "qpp::reset()";
        if (!out) raise(QGPU_ERR_INVALID_ARGUMENT, W, "out");
        std::vector<uint64_t> tgt = qgpu::vec_of(target, k);
        if (!targets_ok(tgt, s->dims.size())) raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
        std::vector<uint64_t> res;
        if (k) {
            std::mt19937 gen(static_cast<std::mt19937::result_type>(seed));
            res = qgpu::sample_once(s, tgt, qgpu::canonical(gen));
        }
        qgpu_state* c = qgpu::copy_state(s);
        try {
            std::vector<double> ps;
            qgpu::collapse_seq(c, tgt, false, res, ps);
            for (uint32_t i = 0; i < k; ++i) {
                const uint64_t d = s->dims[i];
                if (d != s->dims[tgt[i]])
                    raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, "qpp::apply()", "A/dims/target");
                // Xd^(d - r): |j> -> |j + d - r mod d>
                std::vector<qgpu::cd> X(d * d, 0.0);
                for (uint64_t j = 0; j < d; ++j) X[((j + d - res[i]) % d) + j * d] = 1.0;
                qgpu::op_apply(c, X.data(), d, {tgt[i]});
            }
        } catch (...) {
            qgpu::free_state(c);
            throw;
        }
        QG_CUDA(cudaStreamSynchronize(s->ctx->stream));
        *out = c;
    });
}

// qpp::discard(A, target, dims) (instruments.hpp:1243-1292): measure_seq
// with destruction, keeping only the post-measurement state.
qgpu_status qgpu_discard(const qgpu_state* s, const uint64_t* target, uint32_t k, uint64_t seed,
                         qgpu_state** out) {
    return guarded(__func__, [&] {
        need_handle(s);
        const char* W = "qpp::discard()";
        if (!out) raise(QGPU_ERR_INVALID_ARGUMENT, W, "out");
        std::vector<uint64_t> tgt = qgpu::vec_of(target, k);
        if (!targets_ok(tgt, s->dims.size())) raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
        std::vector<uint64_t> res;
        if (k) {
            std::mt19937 gen(static_cast<std::mt19937::result_type>(seed));
            res = qgpu::sample_once(s, tgt, qgpu::canonical(gen));
        }
        qgpu_state* c = qgpu::copy_state(s);
        try {
            std::vector<double> ps;
            qgpu::collapse_seq(c, tgt, true, res, ps);
        } catch (...) {
            qgpu::free_state(c);
            throw;
        }
        QG_CUDA(cudaStreamSynchronize(s->ctx->stream));
        *out = c;
    });
}

} // extern "C"
