// serve.cpp -- the serving loop: QNoisyEngine requests executed on one GPU
// with continuous batching.
//
// A request is a circuit (ket of n qubits or density matrix), a depolarising
// probability per qubit per step (kets, stochastic trajectories as in
// qnoisy_engine.hpp:105-139), a shot count and a seed; its result is one
// classical register (the measurement dits) and one final full-basis sample
// per shot. Requests are queued by any thread; one worker thread drains the
// queue:
//
//   batched mode  every request that arrived while the previous launch ran
//                 is admitted (by an estimate of its HBM footprint against the
//                 budget) and all their trajectories go into the next launch
//                 of the shared-memory / per-CTA-slot trajectory kernel, one
//                 launch per register size. Requests the kernel cannot run
//                 (density matrices, > 20 qubits, wider gates) run on the
//                 resident engine on a second stream, overlapping the batch.
//   plain mode    one request at a time on the resident engine, one kernel
//                 launch per gate, complex128 (the comparison form).
//
// Latency is measured from submit to the moment the worker has the result
// on the host.
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
    Clock::time_point t_submit, t_done;
    bool done = false;
    qgpu_status status = QGPU_OK;
    std::string err;
    std::vector<uint32_t> dits;    // shots x max(nc, 1)
    std::vector<uint64_t> samples; // shots
};

} // namespace qgpu

struct qgpu_server {
    qgpu_ctx* ctx = nullptr;  // batches
    qgpu_ctx* ctx2 = nullptr; // engine path
    int mode = 0;
    uint64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<qgpu::Request*> queue;
    std::unordered_map<uint64_t, qgpu::Request*> all;
    std::thread worker;
    bool stop = false;
    uint64_t next_id = 1;
    uint64_t batches = 0, launched_traj = 0, engine_runs = 0;
    double busy_s = 0;
    std::unordered_map<const qgpu_circuit*, std::pair<bool, qgpu::TProgram>> progs;
};

namespace qgpu {
namespace {

uint64_t state_bytes(const Request* r, qgpu_prec prec) {
    uint64_t D = 1;
    for (uint32_t i = 0; i < r->c->nq; ++i) D *= r->c->d;
    uint64_t e = prec == QGPU_C128 ? 16 : 8;
    return r->kind == QGPU_KET ? D * e : D * D * e;
}

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

const TProgram* program_of(qgpu_server* S, Request* r) {
    auto it = S->progs.find(r->c);
    if (it == S->progs.end()) {
        TProgram P;
        bool ok = r->kind == QGPU_KET && compile_traj(r->c, P);
        it = S->progs.emplace(r->c, std::make_pair(ok, std::move(P))).first;
    }
    return it->second.first ? &it->second.second : nullptr;
}

// One launch (per register size) for all trajectories of `batch`.
void run_batch(qgpu_server* S, std::vector<Request*>& batch) {
    qgpu_ctx* ctx = S->ctx;
    // group by register size
    std::map<uint32_t, std::vector<Request*>> by_n;
    for (Request* r : batch) by_n[program_of(S, r)->n].push_back(r);
    for (auto& kv : by_n) {
        const uint32_t n = kv.first;
        auto& rs = kv.second;
        uint32_t maxcreg = 1;
        uint64_t nwork = 0;
        std::vector<TInstr> ins;
        std::vector<float> mats;
        std::vector<std::pair<size_t, size_t>> pofs; // (ins offset, mat offset) per request
        for (Request* r : rs) {
            const TProgram* P = program_of(S, r);
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
                         ? size_t(traj_global_grid(ctx, int(nwork))) * N * sizeof(float2)
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
            const TProgram* P = program_of(S, rs[i]);
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
        S->launched_traj += nwork;
        out = 0;
        for (Request* r : rs) {
            const uint32_t nc = std::max<uint32_t>(r->c->nc, 1);
            r->dits.assign(r->shots * nc, 0);
            r->samples.assign(r->shots, 0);
            for (uint64_t s = 0; s < r->shots; ++s, ++out) {
                r->samples[s] = hs[out];
                for (uint32_t i = 0; i < nc; ++i) r->dits[s * nc + i] = hd[size_t(out) * maxcreg + i];
            }
        }
    }
}

void finish(qgpu_server* S, Request* r) {
    std::lock_guard<std::mutex> lock(S->mu);
    r->t_done = Clock::now();
    r->done = true;
    S->cv_done.notify_all();
}

void worker_loop(qgpu_server* S) {
    cudaSetDevice(S->ctx->device);
    for (;;) {
        std::vector<Request*> got;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            S->cv_work.wait(lock, [&] { return S->stop || !S->queue.empty(); });
            if (S->stop && S->queue.empty()) return;
            if (S->mode == 1) {
                got.push_back(S->queue.front());
                S->queue.pop_front();
            } else {
                // admit in arrival order while the estimated footprint fits
                uint64_t used = 0;
                while (!S->queue.empty()) {
                    Request* r = S->queue.front();
                    uint64_t need = program_of(S, r) ? r->shots * 64 : 2 * state_bytes(r, QGPU_C64);
                    if (!got.empty() && used + need > S->budget) break;
                    used += need;
                    got.push_back(r);
                    S->queue.pop_front();
                }
            }
        }
        auto t0 = Clock::now();
        std::vector<Request*> batch, rest;
        for (Request* r : got) (S->mode == 0 && program_of(S, r) ? batch : rest).push_back(r);
        try {
            if (!batch.empty()) {
                std::thread side;
                std::vector<std::pair<Request*, std::string>> side_err;
                // engine-path requests overlap the batch on the second stream
                if (!rest.empty())
                    side = std::thread([&] {
                        cudaSetDevice(S->ctx2->device);
                        for (Request* r : rest) {
                            try {
                                run_engine(S->ctx2, r, QGPU_C64);
                            } catch (const Exc& e) {
                                r->status = e.code;
                                r->err = e.where + ": " + e.what;
                            }
                            finish(S, r);
                        }
                    });
                try {
                    run_batch(S, batch);
                } catch (const Exc& e) {
                    for (Request* r : batch) {
                        r->status = e.code;
                        r->err = e.where + ": " + e.what;
                    }
                }
                for (Request* r : batch) finish(S, r);
                if (side.joinable()) side.join();
                ++S->batches;
            } else {
                for (Request* r : rest) {
                    try {
                        run_engine(S->ctx2, r, S->mode == 1 ? QGPU_C128 : QGPU_C64);
                    } catch (const Exc& e) {
                        r->status = e.code;
                        r->err = e.where + ": " + e.what;
                    }
                    ++S->engine_runs;
                    finish(S, r);
                }
            }
        } catch (...) {
            for (Request* r : got)
                if (!r->done) {
                    r->status = QGPU_ERR_CUDA;
                    finish(S, r);
                }
        }
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
        qgpu_status st = qgpu_ctx_create(device, &S->ctx);
        if (st == QGPU_OK) st = qgpu_ctx_create(device, &S->ctx2);
        if (st != QGPU_OK) {
            if (S->ctx) qgpu_ctx_destroy(S->ctx);
            delete S;
            raise(st, "qgpu_server_create()", "context");
        }
        S->mode = mode;
        S->budget = hbm_budget;
        S->worker = std::thread(qgpu::worker_loop, S);
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
            S->queue.push_back(r);
        }
        S->cv_work.notify_one();
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
        if (S->worker.joinable()) S->worker.join();
        for (auto& kv : S->all) delete kv.second;
        qgpu_ctx_destroy(S->ctx2);
        qgpu_ctx_destroy(S->ctx);
        delete S;
    });
}

} // extern "C"
