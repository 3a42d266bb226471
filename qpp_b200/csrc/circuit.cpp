// circuit.cpp -- gate fusion planner and the plain / fused execution forms.
#include "circuit.hpp"

#include <algorithm>
#include <cstring>
#include <map>

#include "kernels.hpp"
#include "ops.hpp"
#include "tile_gates.hpp"
#include "traj.hpp"

namespace qgpu {

// Makes `dev` the current device for a scope and then restores the caller's
// (a circuit may run on states of several GPUs in one process, and its
// device images live on the device they were built for).
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int dev) {
        if (dev < 0 || cudaGetDevice(&prev) != cudaSuccess || prev == dev ||
            cudaSetDevice(dev) != cudaSuccess)
            prev = -1;
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Frees a circuit's device image on the device that holds it.
static void free_image(unsigned char*& p, int dev) {
    if (!p) return;
    DeviceScope on(dev);
    cudaFree(p);
    p = nullptr;
}

} // namespace qgpu

qgpu_circuit::~qgpu_circuit() {
    qgpu::free_image(dB, dB_dev);
    qgpu::free_image(rho_dB, rho_dB_dev);
}

namespace qgpu {

void fused6_matrix(const cd* U, float* B);

// E on block qubits bq (big-endian), with G acting on gq (subset of bq).
std::vector<cd> embed(const std::vector<cd>& G, const std::vector<int>& gq,
                      const std::vector<int>& bq) {
    int kb = int(bq.size()), kg = int(gq.size());
    uint64_t Db = uint64_t(1) << kb, Dg = uint64_t(1) << kg;
    std::vector<int> pos(kg); // bit of the block index holding gq[j]
    uint64_t mask = 0;
    for (int j = 0; j < kg; ++j) {
        int p = int(std::find(bq.begin(), bq.end(), gq[j]) - bq.begin());
        pos[j] = kb - 1 - p;
        mask |= uint64_t(1) << pos[j];
    }
    std::vector<cd> E(Db * Db, 0.0);
    for (uint64_t c = 0; c < Db; ++c) {
        uint64_t gc = 0;
        for (int j = 0; j < kg; ++j) gc |= ((c >> pos[j]) & 1) << (kg - 1 - j);
        for (uint64_t gr = 0; gr < Dg; ++gr) {
            uint64_t r = c & ~mask;
            for (int j = 0; j < kg; ++j) r |= ((gr >> (kg - 1 - j)) & 1) << pos[j];
            E[r + c * Db] = G[gr + gc * Dg];
        }
    }
    return E;
}

static std::vector<cd> matmul(const std::vector<cd>& A, const std::vector<cd>& B,
                              uint64_t m) {
    std::vector<cd> C(m * m, 0.0);
    for (uint64_t j = 0; j < m; ++j)
        for (uint64_t l = 0; l < m; ++l) {
            cd b = B[l + j * m];
            if (b == cd(0.0)) continue;
            for (uint64_t i = 0; i < m; ++i) C[i + j * m] += A[i + l * m] * b;
        }
    return C;
}

static std::vector<cd> kron_pow(const std::vector<cd>& U, int m) {
    std::vector<cd> R{cd(1.0)};
    uint64_t dr = 1;
    for (int i = 0; i < m; ++i) {
        R = kron_mat(R, dr, U, 2);
        dr *= 2;
    }
    return R;
}

bool step_dense(const Step& s, uint32_t max_k, std::vector<int>& qubits,
                std::vector<cd>& U) {
    qubits.clear();
    switch (s.kind) {
        case StepKind::Gate:
            for (uint64_t t : s.target) qubits.push_back(int(t));
            if (qubits.size() > max_k) return false;
            U = s.U;
            return true;
        case StepKind::Fan:
            for (uint64_t t : s.target) qubits.push_back(int(t));
            if (qubits.size() > max_k) return false;
            U = kron_pow(s.U, int(s.target.size()));
            return true;
        case StepKind::Ctrl:
        case StepKind::CtrlFan: {
            for (uint64_t c : s.ctrl) qubits.push_back(int(c));
            for (uint64_t t : s.target) qubits.push_back(int(t));
            if (qubits.size() > max_k) return false;
            int nc = int(s.ctrl.size()), nt = int(s.target.size());
            std::vector<cd> G = s.kind == StepKind::Ctrl ? s.U : kron_pow(s.U, nt);
            uint64_t Dt = uint64_t(1) << nt, D = uint64_t(1) << (nc + nt);
            // control pattern: the gate acts when every control bit equals
            // (shift_inv + 1) % 2 with shift_inv = (2 - shift) % 2 = shift
            uint64_t want = 0;
            for (int i = 0; i < nc; ++i) {
                uint64_t sh = s.has_shift ? s.shift[i] % 2 : 0;
                if (((sh + 1) % 2) == 1) want |= uint64_t(1) << (nc - 1 - i);
            }
            U.assign(D * D, 0.0);
            for (uint64_t c = 0; c < D; ++c) {
                uint64_t cc = c >> nt, ct = c & (Dt - 1);
                if (cc != want) {
                    U[c + c * D] = 1.0;
                    continue;
                }
                for (uint64_t rt = 0; rt < Dt; ++rt) U[(cc << nt | rt) + c * D] = G[rt + ct * Dt];
            }
            return true;
        }
        default:
            return false;
    }
}

std::vector<Block> fuse(const std::vector<Step>& steps, uint32_t nq, uint32_t max_k) {
    std::vector<Block> plan;
    std::vector<Block> open;
    std::vector<int> owner(nq, -1); // qubit -> index in `open`, -1 none
    auto rebuild_owner = [&] {
        std::fill(owner.begin(), owner.end(), -1);
        for (size_t b = 0; b < open.size(); ++b)
            for (int q : open[b].qubits) owner[size_t(q)] = int(b);
    };
    // Emitted blocks act on disjoint qubits, so they commute: pack them
    // first-fit (largest first) into passes of at most max_k qubits.
    auto emit = [&](std::vector<int> ids) {
        std::sort(ids.begin(), ids.end());
        ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
        std::vector<Block> out;
        for (int id : ids) out.push_back(open[size_t(id)]);
        std::stable_sort(out.begin(), out.end(), [](const Block& a, const Block& b) {
            return a.qubits.size() > b.qubits.size();
        });
        std::vector<std::vector<Block>> bins;
        for (auto& b : out) {
            bool placed = false;
            for (auto& bin : bins) {
                size_t w = 0;
                for (auto& x : bin) w += x.qubits.size();
                if (w + b.qubits.size() <= max_k) {
                    bin.push_back(b);
                    placed = true;
                    break;
                }
            }
            if (!placed) bins.push_back({b});
        }
        for (auto& bin : bins) {
            if (bin.size() == 1) {
                plan.push_back(bin[0]);
                continue;
            }
            Block m;
            for (auto& x : bin) m.qubits.insert(m.qubits.end(), x.qubits.begin(), x.qubits.end());
            uint64_t Dm = uint64_t(1) << m.qubits.size();
            m.U.assign(Dm * Dm, 0.0);
            for (uint64_t j = 0; j < Dm; ++j) m.U[j + j * Dm] = 1.0;
            for (auto& x : bin) m.U = matmul(embed(x.U, x.qubits, m.qubits), m.U, Dm);
            plan.push_back(m);
        }
        for (size_t i = ids.size(); i-- > 0;) open.erase(open.begin() + ids[i]);
        rebuild_owner();
    };
    for (size_t i = 0; i < steps.size(); ++i) {
        std::vector<int> q;
        std::vector<cd> G;
        if (!step_dense(steps[i], max_k, q, G)) {
            std::vector<int> all(open.size());
            for (size_t b = 0; b < open.size(); ++b) all[b] = int(b);
            emit(all);
            Block pass;
            pass.step = int(i);
            plan.push_back(pass);
            continue;
        }
        std::vector<int> touched;
        for (int x : q)
            if (owner[size_t(x)] >= 0) touched.push_back(owner[size_t(x)]);
        std::sort(touched.begin(), touched.end());
        touched.erase(std::unique(touched.begin(), touched.end()), touched.end());
        std::vector<int> uq;
        for (int b : touched)
            for (int x : open[size_t(b)].qubits) uq.push_back(x);
        for (int x : q)
            if (std::find(uq.begin(), uq.end(), x) == uq.end()) uq.push_back(x);
        Block nb;
        if (uq.size() <= max_k) {
            nb.qubits = uq;
            uint64_t Db = uint64_t(1) << uq.size();
            std::vector<cd> M(Db * Db, 0.0);
            for (uint64_t j = 0; j < Db; ++j) M[j + j * Db] = 1.0;
            for (int b : touched) M = matmul(embed(open[size_t(b)].U, open[size_t(b)].qubits, uq), M, Db);
            nb.U = matmul(embed(G, q, uq), M, Db);
            std::vector<int> rm = touched;
            for (size_t r = rm.size(); r-- > 0;) open.erase(open.begin() + rm[r]);
        } else {
            emit(touched);
            nb.qubits = q;
            nb.U = G;
        }
        open.push_back(nb);
        rebuild_owner();
    }
    std::vector<int> all(open.size());
    for (size_t b = 0; b < open.size(); ++b) all[b] = int(b);
    emit(all);
    return plan;
}

void apply_step(qgpu_state* s, const Step& st) {
    auto shift_inv = [&](uint64_t d) {
        std::vector<uint64_t> r(st.ctrl.size(), 0);
        if (st.has_shift)
            for (size_t i = 0; i < r.size(); ++i) r[i] = (d - st.shift[i] % d) % d;
        return r;
    };
    switch (st.kind) {
        case StepKind::Gate:
            op_apply(s, st.U.data(), st.DU, st.target);
            break;
        case StepKind::Fan:
            for (uint64_t t : st.target) op_apply(s, st.U.data(), st.DU, {t});
            break;
        case StepKind::Ctrl:
        case StepKind::CtrlFan: {
            uint64_t d = s->dims[st.ctrl[0]];
            op_apply_ctrl(s, st.U.data(), st.DU, st.ctrl, st.target, shift_inv(d),
                          st.kind == StepKind::CtrlFan);
            break;
        }
        case StepKind::Channel:
            if (s->kind != QGPU_RHO)
                raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_run_gates()",
                      "a channel on a ket needs the engine (sampled branch)");
            op_apply_kraus(s, st.U.data(), st.nK, st.DU, st.target);
            break;
        case StepKind::Nop:
            break;
        default:
            raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_run_gates()",
                  "measurement or classically controlled step: use the engine");
    }
}

// Tensor-core images of the plan's blocks of 3-6 qubits (each executed as a
// 6-qubit block, padded with identity on the lowest free qubits), uploaded
// once: slot[i] >= 0 is block i's image in *dB (65536 bytes each).
constexpr uint32_t kRhoTcMinQubits = 11;

static void upload_tc_blocks(qgpu_ctx* ctx, std::vector<Block>& plan, uint32_t nq,
                             unsigned char** dB, std::vector<int64_t>& slot) {
    DeviceScope on(ctx->device);
    slot.assign(plan.size(), -1);
    int64_t nslot = 0;
    for (size_t i = 0; i < plan.size(); ++i)
        if (plan[i].step < 0 && plan[i].qubits.size() >= 3) slot[i] = nslot++;
    if (nslot == 0) return;
    std::vector<float> host(size_t(nslot) * 128 * 128);
    for (size_t i = 0; i < plan.size(); ++i) {
        if (slot[i] < 0) continue;
        const Block& b = plan[i];
        std::vector<int> q6 = b.qubits;
        for (int x = 0; int(q6.size()) < 6 && x < int(nq); ++x)
            if (std::find(q6.begin(), q6.end(), x) == q6.end()) q6.push_back(x);
        std::vector<cd> U6 = embed(b.U, b.qubits, q6);
        plan[i].qubits = q6; // executed as a 6-qubit block
        plan[i].U = U6;
        fused6_matrix(U6.data(), host.data() + size_t(slot[i]) * 128 * 128);
    }
    float* tmp = nullptr;
    QG_CUDA(cudaMalloc(&tmp, host.size() * sizeof(float)));
    struct FreeTmp {
        float* p;
        ~FreeTmp() { cudaFree(p); }
    } free_tmp{tmp};
    QG_CUDA(cudaMemcpy(tmp, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice));
    QG_CUDA(cudaMalloc(dB, size_t(nslot) * 65536));
    fused6_images(ctx, tmp, *dB, int(nslot));
    QG_CUDA(cudaStreamSynchronize(ctx->stream));
}

static void prepare_plan(qgpu_state* s, qgpu_circuit* c, uint32_t k) {
    // block images held by another device are rebuilt on this one
    if (c->dB && c->dB_dev != s->ctx->device) c->plan_k = 0;
    if (c->plan_k != k) {
        c->plan = fuse(c->steps, c->nq, k);
        c->plan_k = k;
        free_image(c->dB, c->dB_dev);
        c->block_slot.clear();
    }
    bool tc = s->prec == QGPU_C64 && c->nq >= 13 && k == 6;
    if (!tc || c->dB || !c->block_slot.empty()) return;
    upload_tc_blocks(s->ctx, c->plan, c->nq, &c->dB, c->block_slot);
    c->dB_dev = s->ctx->device;
    c->plan_ctx = s->ctx;
}

// Runs a fused plan on a complex64 (virtual) qubit ket of nb bits: blocks with
// an image on the tensor cores, the rest as dense passes, unfused steps as
// they are. Launches only.
static void launch_blocks(qgpu_state* s, const VSpace& vs, int nb, const std::vector<Block>& plan,
                          const unsigned char* dB, const std::vector<int64_t>& slot,
                          const std::vector<Step>& steps) {
    const double* norm2 = nullptr; // |psi|^2 for the tensor-core passes' fp16 scale
    for (size_t i = 0; i < plan.size(); ++i) {
        const Block& b = plan[i];
        if (b.step >= 0) {
            apply_step(s, steps[size_t(b.step)]);
            continue;
        }
        if (!slot.empty() && slot[i] >= 0) {
            int tb[6];
            for (int j = 0; j < 6; ++j) tb[j] = nb - 1 - b.qubits[size_t(j)];
            if (!norm2) norm2 = fused_norm_prepare(s->ctx, s->data, s->elems);
            launch_fused6_tc(s->ctx, s->data, nb, tb, dB + size_t(slot[i]) * 65536, norm2);
            continue;
        }
        vapply(s, vs, b.qubits, {}, b.U.data(), uint64_t(1) << b.qubits.size());
    }
}

// A density-matrix circuit as dense gates on the 2n virtual qubits [column
// digits, row digits] of the column-major matrix (FP64): a 1-qubit gate U is
// conj(U) (x) U on (column t, row t); a 2-qubit gate is conj(U) on the two
// column digits and U on the two row digits; a 1- or 2-qubit channel is its
// superoperator sum_i conj(K_i) (x) K_i on (column digits, row digits). False
// when the circuit holds anything else.
static bool rho_virtual_steps(const qgpu_circuit* c, std::vector<Step>& out) {
    const uint64_t n = c->nq;
    auto gate = [&](std::vector<uint64_t> t, std::vector<cd> U) {
        Step v;
        v.kind = StepKind::Gate;
        v.target = std::move(t);
        v.DU = uint64_t(1) << v.target.size();
        v.U = std::move(U);
        out.push_back(std::move(v));
    };
    for (const Step& st : c->steps) {
        if (st.kind == StepKind::Nop) continue;
        if (st.kind == StepKind::Gate && st.target.size() == 1 && st.DU == 2) {
            gate({st.target[0], n + st.target[0]}, kron_mat(conj_mat(st.U), 2, st.U, 2));
        } else if (st.kind == StepKind::Gate && st.target.size() == 2 && st.DU == 4) {
            gate({st.target[0], st.target[1]}, conj_mat(st.U));
            gate({n + st.target[0], n + st.target[1]}, st.U);
        } else if (st.kind == StepKind::Channel && (st.target.size() == 1 || st.target.size() == 2) &&
                   st.DU == (uint64_t(1) << st.target.size())) {
            const uint64_t DA = st.DU, DS = DA * DA;
            std::vector<cd> S(DS * DS, 0.0);
            for (uint32_t i = 0; i < st.nK; ++i) {
                std::vector<cd> K(st.U.begin() + ptrdiff_t(i * DA * DA),
                                  st.U.begin() + ptrdiff_t((i + 1) * DA * DA));
                std::vector<cd> t = kron_mat(conj_mat(K), DA, K, DA);
                for (size_t j = 0; j < t.size(); ++j) S[j] += t[j];
            }
            std::vector<uint64_t> vt = st.target;
            for (uint64_t q : st.target) vt.push_back(n + q);
            gate(vt, S);
        } else {
            return false;
        }
    }
    return true;
}

// The tensor-core form of a complex64 density matrix of n >= 11 qubits (no
// reference counterpart): the virtual gates merged
// into blocks of <= 6 virtual qubits (fuse), each block one split-FP16
// tcgen05 pass over the matrix. Built once per circuit (and again after steps
// are added). False when the circuit does not qualify.
static bool rho_tc_prepare(qgpu_state* s, qgpu_circuit* c) {
    // from 11 qubits on; below, the launch-bound passes of the 4-virtual-qubit
    // form are as fast (depth-30 serving circuits, one B200: 8 qubits 0.65 vs
    // 0.77 ms, 10 qubits 1.01 vs 1.06 ms, 12 qubits 9.4 vs 6.9 ms)
    if (s->prec != QGPU_C64 || c->d != 2 || c->nq < kRhoTcMinQubits || 2 * c->nq > 62)
        return false;
    if (c->rho_tc_steps != c->steps.size() || (c->rho_dB && c->rho_dB_dev != s->ctx->device)) {
        free_image(c->rho_dB, c->rho_dB_dev);
        c->rho_slot.clear();
        c->rho_plan.clear();
        std::vector<Step> vsteps;
        c->rho_tc_ok = rho_virtual_steps(c, vsteps);
        if (c->rho_tc_ok) {
            c->rho_plan = fuse(vsteps, 2 * c->nq, 6);
            for (const Block& b : c->rho_plan)
                if (b.step >= 0) c->rho_tc_ok = false; // every virtual step is a gate
        }
        if (c->rho_tc_ok) upload_tc_blocks(s->ctx, c->rho_plan, 2 * c->nq, &c->rho_dB, c->rho_slot);
        c->rho_dB_dev = s->ctx->device;
        c->rho_tc_steps = c->steps.size();
    }
    return c->rho_tc_ok;
}

// Fused form of a complex64 qubit density matrix (no reference counterpart).
// The circuit compiles into superoperators on the 2n virtual qubits [column
// digits, row digits] of the column-major matrix (compile_traj_rho: a 1-qubit
// gate or channel is 4 x 4 on (column t, row t), a 2-qubit gate U on the row
// digits and conj(U) on the column digits, a 2-qubit channel 16 x 16 on all
// four). Consecutive superoperators merge into blocks of at most 4 virtual
// qubits (fuse_blocks: FP64 products, rounded to complex64 once), so the
// 1-qubit gates, 2-qubit gate and pair channel that a layer puts on one qubit
// pair become a single 16 x 16 block, and every block is one in-place pass
// over the matrix. Plain form: one pass per gate and per channel.
// The program is built once per circuit (and again after steps are added).
void rho_program_prepare(qgpu_state* s, qgpu_circuit* c) {
    if (c->rho_steps != c->steps.size()) {
        auto P = std::make_shared<TProgram>();
        if (compile_traj_rho(c, *P, 30)) fuse_blocks(*P, 4);
        else P.reset();
        c->rho_prog = P;
        c->rho_steps = c->steps.size();
    }
    if (s->prec != QGPU_C64 || !c->rho_prog)
        raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_run_gates()",
              "fused form of a density matrix needs complex64, qubits, at most 15 of them, and "
              "only gates and 1- or 2-qubit channels");
}

void launch_program(qgpu_state* s, const TProgram& P) {
    const VSpace vs = vspace_of(s);
    const int nv = int(P.n);
    std::vector<cd> A;
    for (const TInstr& I : P.ins) {
        if (I.op != kTG1 && I.op != kTG2 && I.op != kTG3 && I.op != kTG4)
            raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_run_gates()", "dense block program");
        std::vector<int> vt;
        vt.push_back(nv - 1 - I.b0);
        if (I.op != kTG1) vt.push_back(nv - 1 - I.b1);
        if (I.op == kTG3 || I.op == kTG4) vt.push_back(nv - 1 - int(I.cmask & 255u));
        if (I.op == kTG4) vt.push_back(nv - 1 - int((I.cmask >> 8) & 255u));
        const uint64_t DA = uint64_t(1) << vt.size();
        A.resize(DA * DA);
        for (uint64_t j = 0; j < DA * DA; ++j)
            A[j] = cd(P.mats[2 * (I.mat + j)], P.mats[2 * (I.mat + j) + 1]);
        vapply(s, vs, vt, {}, A.data(), DA);
    }
}

// Complex128 qubit kets of up to 22 qubits (64 MiB, half the L2) run the
// fused form as tile passes over blocks of <= 2 qubits. Such a state is read
// from the L2, so a pass's time follows its FP64 work per amplitude, and
// blocks of <= 2 qubits keep that work lowest: a 1-qubit gate merged into a
// neighbouring 2-qubit block costs nothing, where a 3-qubit block costs as
// much as two 2-qubit gates. Larger complex128 kets are HBM-bound and take
// blocks of <= 3 qubits as dense passes, fewer trips through HBM.
constexpr size_t kFusedTileQubitsC128 = 22;

static bool fused_tiles(const qgpu_state* s) {
    return s->kind == QGPU_KET && s->prec == QGPU_C128 && !s->dims.empty() &&
           s->dims.size() <= kFusedTileQubitsC128;
}

void tiled_runs(const qgpu_circuit* c, std::vector<TiledRun>& out) {
    out.clear();
    const int nq = int(c->nq);
    out.emplace_back();
    for (const Block& b : c->plan) {
        if (b.step >= 0) {
            const Step& st = c->steps[size_t(b.step)];
            if (gate_desc_of(st, nq, out.back().gates)) continue;
            out.emplace_back();
            out.back().step = b.step;
            out.emplace_back();
            continue;
        }
        GateDesc g;
        g.op = int(b.qubits.size());
        g.b0 = nq - 1 - b.qubits[0];
        if (g.op == 2) g.b1 = nq - 1 - b.qubits[1];
        std::copy(b.U.begin(), b.U.end(), g.A);
        out.back().gates.push_back(g);
    }
}

// Plans the fused plan's blocks (<= 2 qubits, c->plan) and its unfused
// steps as tile programs once per circuit (again after steps are added or
// the tile size changes): each run list-scheduled into fewer passes and
// sweeps, then cut into passes.
static void prepare_tiled_blocks(qgpu_state* s, qgpu_circuit* c) {
    const int Tmax = tile_bits_max(s->ctx, s->prec);
    if (c->ftiles && c->ftiles->nsteps == c->steps.size() && c->ftiles->Tmax == Tmax) return;
    auto F = std::make_shared<FusedTiles>();
    F->nsteps = c->steps.size();
    F->Tmax = Tmax;
    std::vector<TiledRun> runs;
    tiled_runs(c, runs);
    for (const TiledRun& r : runs) {
        if (r.step >= 0) {
            F->runs.push_back({r.step, TileProgram{}});
        } else if (!r.gates.empty()) {
            TileProgram P;
            plan_tile_program(schedule_gates(r.gates, int(c->nq), Tmax), int(c->nq), Tmax, P);
            F->runs.push_back({-1, std::move(P)});
        }
    }
    c->ftiles = std::move(F);
}

// The planned tile programs in order, a step the passes do not take run as
// it is between them.
static void launch_tiled_blocks(qgpu_state* s, qgpu_circuit* c) {
    prepare_plan(s, c, 2); // both no-ops after fused_prepare
    prepare_tiled_blocks(s, c);
    for (const auto& r : c->ftiles->runs) {
        if (r.first >= 0) apply_step(s, c->steps[size_t(r.first)]);
        else run_tile_program(s, r.second);
    }
}

// Kets: qubits only; blocks of up to 6 qubits (complex64: 3-6 qubit blocks on
// the tensor cores from 13 qubits on); in complex128, 2 (as tile passes) up to
// 22 qubits and 3 above.
void fused_prepare(qgpu_state* s, qgpu_circuit* c) {
    if (s->kind == QGPU_RHO) {
        if (rho_tc_prepare(s, c)) {
            ctx_error_flag(s->ctx); // allocated outside any capture
            return;
        }
        return rho_program_prepare(s, c);
    }
    if (c->d != 2)
        raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_run_gates()", "fused form needs a qubit ket");
    prepare_plan(s, c, s->prec == QGPU_C64 ? 6 : fused_tiles(s) ? 2 : 3);
    if (fused_tiles(s)) prepare_tiled_blocks(s, c);
    if (!c->block_slot.empty()) ctx_error_flag(s->ctx); // allocated outside any capture
}

void fused_launch(qgpu_state* s, qgpu_circuit* c) {
    if (s->kind == QGPU_RHO) {
        if (c->rho_tc_ok && c->rho_tc_steps == c->steps.size()) {
            launch_blocks(s, vspace_of(s), int(2 * c->nq), c->rho_plan, c->rho_dB, c->rho_slot,
                          c->steps);
            return;
        }
        return launch_program(s, *c->rho_prog);
    }
    if (fused_tiles(s)) return launch_tiled_blocks(s, c);
    launch_blocks(s, vspace_ket(s->dims), int(c->nq), c->plan, c->dB, c->block_slot, c->steps);
}

void run_gates(qgpu_state* s, qgpu_circuit* c, int form, uint64_t first, uint64_t count) {
    for (const Step& st : c->steps)
        if (st.kind == StepKind::CondIf)
            raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_run_gates()",
                  "classical conditionals need an engine (qgpu_engine_execute)");
    if (form == 0) {
        // qubit kets: runs of 1- and 2-qubit gates as tile passes
        const bool tiles = s->kind == QGPU_KET && c->d == 2 && !s->dims.empty();
        std::vector<GateDesc> run;
        for (uint64_t i = first; i < first + count && i < c->steps.size(); ++i) {
            if (tiles && gate_desc_of(c->steps[i], int(c->nq), run)) continue;
            run_tiled_gates(s, run);
            run.clear();
            apply_step(s, c->steps[i]);
        }
        run_tiled_gates(s, run);
        return;
    }
    if (first != 0 || count < c->steps.size())
        raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_run_gates()", "fused form runs whole circuits");
    fused_prepare(s, c);
    fused_launch(s, c);
    const bool tc = s->kind == QGPU_KET ? !c->block_slot.empty()
                                        : c->rho_tc_ok && !c->rho_slot.empty();
    if (tc && fused_error(s->ctx))
        raise(QGPU_ERR_TIMEOUT, "qgpu_run_gates()", "tensor-core pass timed out");
}

} // namespace qgpu
