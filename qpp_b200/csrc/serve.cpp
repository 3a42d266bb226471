// serve.cpp -- the serving loop: QNoisyEngine requests executed on one GPU
// with continuous batching.
//
// A request is a circuit (ket of n qubits or density matrix), a depolarising
// probability per qubit per step (kets, stochastic trajectories as in
// qnoisy_engine.hpp:105-139), a shot count and a seed; its result is one
// classical register (the measurement dits) and one final full-basis sample
// per shot. Requests are queued by any thread and routed to one of three
// lanes, each with its own worker thread and CUDA stream, so small requests
// never wait behind large ones:
//
//   lane 0  kets of <= 14 qubits: trajectories with the state in shared
//           memory; every request that arrived while the lane's previous
//           launch ran is admitted (in arrival order, by an estimate of its
//           HBM footprint against the budget) into the next launch;
//   lane 1  kets of 15-20 qubits: the same kernel with each CTA on its own
//           slot of global scratch (L2 / HBM), batched the same way;
//   lane 2  everything the kernel cannot run (density matrices, > 20 qubits,
//           wider gates, classical control): the resident engine, one
//           request at a time.
//   plain mode: every request on lane 2 in complex128, one at a time (the
//           comparison form: one kernel launch per gate).
//
// Latency is measured from submit to the moment the lane has the result on
// the host.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <thread>
#include <unordered_map>

#include "capi_common.hpp"
#include "circuit.hpp"
#include "kernels.hpp"
#include "ops.hpp"
#include "traj.hpp"

using Clock = std::chrono::steady_clock;

namespace qgpu {

struct Request {
    uint64_t id = 0;
    qgpu_circuit* c = nullptr;
    qgpu_kind kind = QGPU_KET;
    double p = 0;
    uint64_t shots = 1;
    uint64_t seed = 0;
    const TProgram* prog = nullptr; // compiled trajectory program, or null
    Clock::time_point t_submit, t_done;
    bool done = false;
    qgpu_status status = QGPU_OK;
    std::string err;
    std::vector<uint32_t> dits;    // shots x max(nc, 1)
    std::vector<uint64_t> samples; // shots
};

struct Lane {
    qgpu_ctx* ctx = nullptr;
    std::deque<Request*> q;
    std::thread th;
};

} // namespace qgpu

struct qgpu_server {
    int mode = 0;
    uint64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    qgpu::Lane lanes[3];
    std::unordered_map<uint64_t, qgpu::Request*> all;
    bool stop = false;
    uint64_t next_id = 1;
    uint64_t batches = 0, launched_traj = 0, engine_runs = 0;
    double busy_s = 0;
    std::unordered_map<const qgpu_circuit*, std::pair<bool, qgpu::TProgram>> progs;
};

namespace qgpu {
namespace {

// Engine path: trajectories one shot at a time on the resident engine; a
// density matrix evolves once (its noise is in the circuit's channels) and
// the shots sample the final diagonal.
void run_engine(qgpu_ctx* ctx, Request* r, qgpu_prec prec) {
    const uint32_t nc = std::max<uint32_t>(r->c->nc, 1);
    r->dits.assign(r->shots * nc, 0);
    r->samples.assign(r->shots, 0);
    qgpu_engine* e = nullptr;
    qgpu_status st = qgpu_engine_create(ctx, r->c, r->kind, prec, &e);
    if (st != QGPU_OK) raise(st, "qgpu_server", "engine create");
    struct Del {
        qgpu_engine* e;
        ~Del() { qgpu_engine_destroy(e); }
    } del{e};
    qgpu_engine_set_seed(e, r->seed);
    if (r->kind == QGPU_KET && r->p > 0) {
        const double s = std::sqrt(r->p / 3);
        const double Ks[4][8] = {{std::sqrt(1 - r->p), 0, 0, 0, 0, 0, std::sqrt(1 - r->p), 0},
                                 {0, 0, s, 0, s, 0, 0, 0},
                                 {0, 0, 0, s, 0, -s, 0, 0},
                                 {s, 0, 0, 0, 0, 0, -s, 0}};
        const double pr[4] = {1 - r->p, r->p / 3, r->p / 3, r->p / 3};
        if ((st = qgpu_engine_set_noise(e, &Ks[0][0], 4, 2, pr)) != QGPU_OK)
            raise(st, "qgpu_server", "noise");
    }
    std::mt19937 gen(uint32_t(r->seed ^ 0x5eed));
    const uint64_t runs = r->kind == QGPU_KET ? r->shots : 1;
    std::vector<uint64_t> dv(nc);
    std::vector<double> pv(nc);
    for (uint64_t s = 0; s < runs; ++s) {
        if ((st = qgpu_engine_execute(e, 1)) != QGPU_OK) raise(st, "qgpu_server", "execute");
        qgpu_engine_get_dits(e, dv.data(), pv.data());
        qgpu_state* fin = nullptr;
        if ((st = qgpu_engine_get_state(e, &fin)) != QGPU_OK) raise(st, "qgpu_server", "state");
        struct DelS {
            qgpu_state* s;
            ~DelS() { qgpu_state_destroy(s); }
        } dels{fin};
        std::uniform_real_distribution<double> U(0.0, 1.0);
        const uint64_t nsamp = r->kind == QGPU_KET ? 1 : r->shots;
        for (uint64_t k = 0; k < nsamp; ++k) {
            uint64_t idx = prefix_search(fin->ctx, fin->prec, fin->data, fin->D,
                                         fin->kind == QGPU_RHO, U(gen), nullptr);
            uint64_t slot = r->kind == QGPU_KET ? s : k;
            r->samples[slot] = idx;
            for (uint32_t i = 0; i < nc; ++i) r->dits[slot * nc + i] = uint32_t(dv[i]);
        }
    }
}

// caller holds S->mu
const TProgram* program_of(qgpu_server* S, qgpu_circuit* c, qgpu_kind kind) {
    if (kind != QGPU_KET) return nullptr;
    auto it = S->progs.find(c);
    if (it == S->progs.end()) {
        TProgram P;
        bool ok = compile_traj(c, P);
        it = S->progs.emplace(c, std::make_pair(ok, std::move(P))).first;
    }
    return it->second.first ? &it->second.second : nullptr;
}

void finish(qgpu_server* S, Request* r) {
    std::lock_guard<std::mutex> lock(S->mu);
    r->t_done = Clock::now();
    r->done = true;
    S->cv_done.notify_all();
}

void fail(qgpu_server* S, Request* r, qgpu_status code, const std::string& msg) {
    r->status = code;
    r->err = msg;
    finish(S, r);
}

// One launch per register size for all trajectories of `batch`; each size
// class is finished as soon as its results are on the host.
void run_batch(qgpu_server* S, qgpu_ctx* ctx, std::vector<Request*>& batch) {
    std::map<uint32_t, std::vector<Request*>> by_n;
    for (Request* r : batch) by_n[r->prog->n].push_back(r);
    for (auto& kv : by_n) {
        const uint32_t n = kv.first;
        auto& rs = kv.second;
        uint32_t maxcreg = 1;
        uint64_t nwork = 0;
        std::vector<TInstr> ins;
        std::vector<float> mats;
        std::vector<std::pair<size_t, size_t>> pofs; // (ins offset, mat offset) per request
        for (Request* r : rs) {
            const TProgram* P = r->prog;
            pofs.push_back({ins.size(), mats.size() / 2});
            ins.insert(ins.end(), P->ins.begin(), P->ins.end());
            mats.insert(mats.end(), P->mats.begin(), P->mats.end());
            maxcreg = std::max<uint32_t>(maxcreg, std::max<uint32_t>(P->ncreg, 1));
            nwork += r->shots;
        }
        const uint64_t N = uint64_t(1) << n;
        auto al = [](size_t x) { return (x + 255) / 256 * 256; };
        size_t b_ins = std::max<size_t>(ins.size() * sizeof(TInstr), 16);
        size_t b_mat = std::max<size_t>(mats.size() * sizeof(float), 16);
        size_t b_work = nwork * sizeof(TWork);
        size_t b_dits = nwork * maxcreg * sizeof(uint32_t);
        size_t b_samp = nwork * sizeof(uint64_t);
        size_t b_g = n > uint32_t(kTrajMaxQubits)
                         ? size_t(traj_global_grid(ctx, int(nwork), int(n))) * N * sizeof(float2)
                         : 0;
        size_t total = al(b_ins) + al(b_mat) + al(b_work) + al(b_dits) + al(b_samp) + al(b_g);
        unsigned char* buf = nullptr;
        QG_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&buf), total, ctx->stream));
        unsigned char* p = buf;
        auto take = [&](size_t b) {
            unsigned char* q = p;
            p += al(b);
            return q;
        };
        auto* dins = reinterpret_cast<TInstr*>(take(b_ins));
        auto* dmat = reinterpret_cast<float2*>(take(b_mat));
        auto* dwork = reinterpret_cast<TWork*>(take(b_work));
        auto* ddits = reinterpret_cast<uint32_t*>(take(b_dits));
        auto* dsamp = reinterpret_cast<uint64_t*>(take(b_samp));
        auto* dg = reinterpret_cast<float2*>(b_g ? take(b_g) : nullptr);
        std::vector<TWork> work;
        work.reserve(nwork);
        uint32_t out = 0;
        for (size_t i = 0; i < rs.size(); ++i) {
            const TProgram* P = rs[i]->prog;
            for (uint64_t s = 0; s < rs[i]->shots; ++s) {
                TWork w{};
                w.prog = dins + pofs[i].first;
                w.mats = dmat + pofs[i].second;
                w.nins = uint32_t(P->ins.size());
                w.n = uint8_t(n);
                w.p_noise = float(rs[i]->p);
                w.shot = uint32_t(s);
                w.out = out++;
                w.seed = rs[i]->seed;
                work.push_back(w);
            }
        }
        QG_CUDA(cudaMemcpyAsync(dins, ins.data(), ins.size() * sizeof(TInstr),
                                cudaMemcpyHostToDevice, ctx->stream));
        if (!mats.empty())
            QG_CUDA(cudaMemcpyAsync(dmat, mats.data(), mats.size() * sizeof(float),
                                    cudaMemcpyHostToDevice, ctx->stream));
        QG_CUDA(cudaMemcpyAsync(dwork, work.data(), b_work, cudaMemcpyHostToDevice, ctx->stream));
        QG_CUDA(cudaMemsetAsync(ddits, 0, b_dits, ctx->stream));
        launch_traj(ctx, dwork, int(nwork), int(n), ddits, int(maxcreg), dsamp, nullptr,
                    nullptr, 0, dg);
        std::vector<uint32_t> hd(nwork * maxcreg);
        std::vector<uint64_t> hs(nwork);
        QG_CUDA(cudaMemcpyAsync(hd.data(), ddits, b_dits, cudaMemcpyDeviceToHost, ctx->stream));
        QG_CUDA(cudaMemcpyAsync(hs.data(), dsamp, b_samp, cudaMemcpyDeviceToHost, ctx->stream));
        QG_CUDA(cudaFreeAsync(buf, ctx->stream));
        QG_CUDA(cudaStreamSynchronize(ctx->stream));
        out = 0;
        for (Request* r : rs) {
            const uint32_t nc = std::max<uint32_t>(r->c->nc, 1);
            r->dits.assign(r->shots * nc, 0);
            r->samples.assign(r->shots, 0);
            for (uint64_t s = 0; s < r->shots; ++s, ++out) {
                r->samples[s] = hs[out];
                for (uint32_t i = 0; i < nc; ++i) r->dits[s * nc + i] = hd[size_t(out) * maxcreg + i];
            }
            finish(S, r);
        }
        std::lock_guard<std::mutex> lock(S->mu);
        S->launched_traj += nwork;
    }
}

void lane_loop(qgpu_server* S, int li) {
    Lane& L = S->lanes[li];
    cudaSetDevice(L.ctx->device);
    const bool batching = li < 2;
    for (;;) {
        std::vector<Request*> got;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            S->cv_work.wait(lock, [&] { return S->stop || !L.q.empty(); });
            if (S->stop && L.q.empty()) return;
            if (!batching) {
                got.push_back(L.q.front());
                L.q.pop_front();
            } else {
                // admit in arrival order while the estimated footprint fits:
                // per-CTA slots for >= 15 qubits, outputs otherwise
                uint64_t used = 0;
                while (!L.q.empty()) {
                    Request* r = L.q.front();
                    uint64_t need = r->shots * 64 + (r->prog->n > uint32_t(kTrajMaxQubits)
                                                          ? (uint64_t(8) << r->prog->n) * 8
                                                          : 0);
                    if (!got.empty() && used + need > S->budget) break;
                    used += need;
                    got.push_back(r);
                    L.q.pop_front();
                }
            }
        }
        auto t0 = Clock::now();
        if (batching) {
            try {
                run_batch(S, L.ctx, got);
            } catch (const Exc& e) {
                for (Request* r : got)
                    if (!r->done) fail(S, r, e.code, e.where + ": " + e.what);
            }
        } else {
            for (Request* r : got) {
                try {
                    run_engine(L.ctx, r, S->mode == 1 ? QGPU_C128 : QGPU_C64);
                    finish(S, r);
                } catch (const Exc& e) {
                    fail(S, r, e.code, e.where + ": " + e.what);
                }
            }
        }
        std::lock_guard<std::mutex> lock(S->mu);
        if (batching) ++S->batches;
        else S->engine_runs += got.size();
        S->busy_s += std::chrono::duration<double>(Clock::now() - t0).count();
    }
}

} // namespace
} // namespace qgpu

using qgpu::guarded;
using qgpu::need_handle;
using qgpu::raise;

extern "C" {

qgpu_status qgpu_server_create(int device, uint64_t hbm_budget, int mode, qgpu_server** out) {
    return guarded([&] {
        if (!out) raise(QGPU_ERR_INVALID_ARGUMENT, "qgpu_server_create()", "out");
        if (mode != 0 && mode != 1)
            raise(QGPU_ERR_INVALID_ARGUMENT, "qgpu_server_create()", "mode");
        auto* S = new qgpu_server;
        S->mode = mode;
        S->budget = hbm_budget;
        for (auto& L : S->lanes) {
            qgpu_status st = qgpu_ctx_create(device, &L.ctx);
            if (st != QGPU_OK) {
                for (auto& M : S->lanes)
                    if (M.ctx) qgpu_ctx_destroy(M.ctx);
                delete S;
                raise(st, "qgpu_server_create()", "context");
            }
        }
        for (int i = 0; i < 3; ++i) S->lanes[i].th = std::thread(qgpu::lane_loop, S, i);
        *out = S;
    });
}

qgpu_status qgpu_server_submit(qgpu_server* S, qgpu_circuit* c, qgpu_kind kind, double p,
                               uint64_t shots, uint64_t seed, uint64_t* id) {
    return guarded([&] {
        need_handle(S);
        need_handle(c);
        if (shots == 0) raise(QGPU_ERR_OUT_OF_RANGE, "qgpu_server_submit()", "shots");
        auto* r = new qgpu::Request;
        r->c = c;
        r->kind = kind;
        r->p = p;
        r->shots = shots;
        r->seed = seed;
        r->t_submit = Clock::now();
        {
            std::lock_guard<std::mutex> lock(S->mu);
            r->id = S->next_id++;
            S->all[r->id] = r;
            int lane = 2;
            if (S->mode == 0) {
                r->prog = qgpu::program_of(S, c, kind);
                if (r->prog) lane = r->prog->n > uint32_t(qgpu::kTrajMaxQubits) ? 1 : 0;
            }
            S->lanes[lane].q.push_back(r);
        }
        S->cv_work.notify_all();
        if (id) *id = r->id;
    });
}

// Waits up to timeout_s (negative: forever) for request `id`; latency in
// seconds from submit to result; samples / dits copied when given; the
// request is released after a successful wait.
qgpu_status qgpu_server_wait(qgpu_server* S, uint64_t id, double timeout_s, double* latency_s,
                             uint64_t* samples, uint32_t* dits) {
    return guarded([&] {
        need_handle(S);
        qgpu::Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            auto it = S->all.find(id);
            if (it == S->all.end()) raise(QGPU_ERR_INVALID_HANDLE, "qgpu_server_wait()", "id");
            r = it->second;
            auto pred = [&] { return r->done; };
            if (timeout_s < 0)
                S->cv_done.wait(lock, pred);
            else if (!S->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), pred))
                raise(QGPU_ERR_TIMEOUT, "qgpu_server_wait()", "request not finished");
            S->all.erase(it);
        }
        std::unique_ptr<qgpu::Request> own(r);
        if (r->status != QGPU_OK) raise(r->status, "qgpu_server", r->err);
        if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
        if (samples) std::copy(r->samples.begin(), r->samples.end(), samples);
        if (dits) std::copy(r->dits.begin(), r->dits.end(), dits);
    });
}

qgpu_status qgpu_server_stats(qgpu_server* S, uint64_t* batches, uint64_t* trajectories,
                              uint64_t* engine_runs, double* busy_s) {
    return guarded([&] {
        need_handle(S);
        std::lock_guard<std::mutex> lock(S->mu);
        if (batches) *batches = S->batches;
        if (trajectories) *trajectories = S->launched_traj;
        if (engine_runs) *engine_runs = S->engine_runs;
        if (busy_s) *busy_s = S->busy_s;
    });
}

qgpu_status qgpu_server_destroy(qgpu_server* S) {
    return guarded([&] {
        if (!S) return;
        {
            std::lock_guard<std::mutex> lock(S->mu);
            S->stop = true;
        }
        S->cv_work.notify_all();
        for (auto& L : S->lanes)
            if (L.th.joinable()) L.th.join();
        for (auto& kv : S->all) delete kv.second;
        for (auto& L : S->lanes) qgpu_ctx_destroy(L.ctx);
        delete S;
    });
}

} // extern "C"
