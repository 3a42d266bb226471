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
//   lane 0  kets of <= 14 qubits and density matrices of <= 7 qubits (14
//           virtual qubits, one exact run): trajectories with the state in
//           shared memory; every request that arrived while the lane's
//           previous launch ran is admitted (in arrival order, by an estimate
//           of its HBM footprint against the budget) into the next launch;
//   lane 1  kets of 15-20 qubits: the same kernel with each CTA on its own
//           slot of global scratch (HBM), batched the same way;
//   lane 2  everything else, one request at a time: density matrices above
//           7 qubits whose circuits are gates and channels only run in the
//           fused superoperator form (qgpu_run_gates, QGPU_FORM_FUSED: a
//           layer's gates and channel on one qubit pair are one 16 x 16 pass
//           over the matrix; one CTA per matrix would take seconds); the rest
//           (density matrices with measurements, kets above 20 qubits, whose
//           one-at-a-time engine run keeps the state in L2 and beats an
//           HBM-bound slot per shot, wider gates, classical control) run on
//           the resident engine.
//   plain mode: every request on lane 2 in complex128, one at a time (the
//           comparison form: one kernel launch per gate).
//
// Lanes 0 and 1 admit work at shot granularity: a launch takes, in arrival
// order, at most kChunkShots shots of each waiting request, up to a launch
// budget, and a request that arrives meanwhile joins the next launch. A
// request with more shots spans several launches and finishes when its last
// shot lands. Every shot draws from its own Philox counter (request seed,
// shot index), so the results do not depend on how the shots were split.
// Each of these lanes keeps two launches in flight: the host builds and
// enqueues the next batch while the current one runs, and collects results
// from pinned memory.
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
    bool fused_rho = false;         // a density matrix of gates and channels only
    Clock::time_point t_submit, t_done;
    bool done = false;
    qgpu_status status = QGPU_OK;
    std::string err;
    std::vector<uint32_t> dits;    // shots x max(nc, 1)
    std::vector<uint64_t> samples; // shots
    uint64_t issued = 0;           // shots handed to launches so far
    uint64_t landed = 0;           // shots whose results are in
};

// A slice of a request's shots in one launch: shots [s0, s0 + ns) (a density
// matrix runs once, whatever its shot count: s0 = 0, ns = shots).
struct Chunk {
    Request* r;
    uint64_t s0, ns;
};

// Pinned host memory for one launch's results, reused across launches.
struct PinnedBuf {
    void* p = nullptr;
    size_t bytes = 0;
    void* get(size_t b) {
        if (b > bytes) {
            if (p) cudaFreeHost(p);
            p = nullptr;
            bytes = 0;
            QG_CUDA(cudaMallocHost(&p, b));
            bytes = b;
        }
        return p;
    }
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
};

// One size class of a batch, enqueued: where its results land on the host
// and how they map back to the chunks.
struct ClassLaunch {
    uint32_t n = 0, maxcreg = 1;
    uint64_t nwork = 0, ndiag = 0;
    std::vector<Chunk> cs;
    std::vector<uint64_t> diag_at;
    uint32_t* hd = nullptr;   // nwork x maxcreg dits
    uint64_t* hs = nullptr;   // nwork samples
    double* hdiag = nullptr;  // ndiag diagonal entries
};

// A batch in flight: its size classes and the event after their copies.
struct Pending {
    std::vector<ClassLaunch> classes;
    cudaEvent_t done = nullptr;
    PinnedBuf* pin = nullptr;
};

struct Lane {
    qgpu_ctx* ctx = nullptr;
    std::deque<Request*> q;
    std::thread th;
    PinnedBuf pin[2]; // results of the (at most) two batches in flight
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
    std::unordered_map<const qgpu_circuit*, std::pair<bool, qgpu::TProgram>> progs, rho_progs;
    std::unordered_map<const qgpu_circuit*, bool> rho_fused; // fused form applies
};

namespace qgpu {
namespace {

void sample_diag(const std::vector<double>& diag, uint64_t shots, uint64_t seed,
                 uint64_t* out);

// The shots of a density-matrix request: samples of the final diagonal
// (one strided gather on the device, then the draws on the host).
void sample_rho(qgpu_ctx* ctx, const qgpu_state* fin, Request* r) {
    qgpu_state* dg = new_state(ctx, QGPU_KET, fin->prec, fin->dims, false);
    struct DelD {
        qgpu_state* s;
        ~DelD() { free_state(s); }
    } deld{dg};
    SegPlan m{};
    m.count = fin->D;
    m.nseg = 1;
    m.pow2 = 0;
    m.size[0] = fin->D;
    m.stride[0] = fin->D + 1;
    launch_gather(ctx, fin->prec, fin->data, dg->data, m);
    std::vector<double> h(2 * fin->D);
    if (qgpu_state_download_c128(dg, h.data()) != QGPU_OK)
        raise(QGPU_ERR_CUDA, "qgpu_server", "diagonal");
    std::vector<double> d(fin->D);
    for (uint64_t i = 0; i < fin->D; ++i) d[i] = h[2 * i];
    sample_diag(d, r->shots, r->seed, r->samples.data());
}

// A density matrix of gates and channels only, in the fused superoperator
// form in complex64 from |0...0><0...0| (no measurement, so its dits stay 0).
void run_rho_fused(qgpu_ctx* ctx, Request* r) {
    const uint32_t nc = std::max<uint32_t>(r->c->nc, 1);
    r->dits.assign(r->shots * nc, 0);
    r->samples.assign(r->shots, 0);
    qgpu_state* st = new_state(ctx, QGPU_RHO, QGPU_C64,
                               std::vector<uint64_t>(r->c->nq, r->c->d), true);
    struct DelS {
        qgpu_state* s;
        ~DelS() { free_state(s); }
    } dels{st};
    static const float one[2] = {1.0f, 0.0f};
    QG_CUDA(cudaMemcpyAsync(st->data, one, sizeof(one), cudaMemcpyHostToDevice, ctx->stream));
    run_gates(st, r->c, 1, 0, r->c->steps.size());
    sample_rho(ctx, st, r);
}

// Engine path: trajectories one shot at a time on the resident engine; a
// density matrix evolves once (its noise is in the circuit's channels) and
// the shots sample the final diagonal.
void run_engine(qgpu_ctx* ctx, Request* r, qgpu_prec prec) {
    if (r->fused_rho && prec == QGPU_C64) {
        run_rho_fused(ctx, r);
        return;
    }
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
        // every shot from |0...0> (an engine continues from its last state)
        if ((st = qgpu_engine_reset(e, 1)) != QGPU_OK) raise(st, "qgpu_server", "reset");
        if ((st = qgpu_engine_execute(e, 1)) != QGPU_OK) raise(st, "qgpu_server", "execute");
        qgpu_engine_get_dits(e, dv.data(), pv.data());
        qgpu_state* fin = nullptr;
        if ((st = qgpu_engine_get_state(e, &fin)) != QGPU_OK) raise(st, "qgpu_server", "state");
        struct DelS {
            qgpu_state* s;
            ~DelS() { qgpu_state_destroy(s); }
        } dels{fin};
        if (r->kind != QGPU_KET) {
            sample_rho(ctx, fin, r);
            for (uint64_t k = 0; k < r->shots; ++k)
                for (uint32_t i = 0; i < nc; ++i) r->dits[k * nc + i] = uint32_t(dv[i]);
            continue;
        }
        std::uniform_real_distribution<double> U(0.0, 1.0);
        r->samples[s] = prefix_search(fin->ctx, fin->prec, fin->data, fin->D, false, U(gen),
                                      nullptr);
        for (uint32_t i = 0; i < nc; ++i) r->dits[s * nc + i] = uint32_t(dv[i]);
    }
}

// caller holds S->mu; kets compile as trajectories, density matrices as one
// exact run over 2n virtual qubits (keyed separately)
const TProgram* program_of(qgpu_server* S, qgpu_circuit* c, qgpu_kind kind) {
    auto& cache = kind == QGPU_KET ? S->progs : S->rho_progs;
    auto it = cache.find(c);
    if (it == cache.end()) {
        TProgram P;
        bool ok = kind == QGPU_KET ? compile_traj(c, P) : compile_traj_rho(c, P);
        it = cache.emplace(c, std::make_pair(ok, std::move(P))).first;
    }
    return it->second.first ? &it->second.second : nullptr;
}

// `shots` samples of the basis distribution given by the diagonal
void sample_diag(const std::vector<double>& diag, uint64_t shots, uint64_t seed,
                 uint64_t* out) {
    std::vector<double> w(diag.size());
    for (size_t i = 0; i < diag.size(); ++i) w[i] = std::max(diag[i], 0.0);
    std::mt19937 gen(uint32_t(seed ^ 0x5eed));
    std::discrete_distribution<uint64_t> dd(w.begin(), w.end());
    for (uint64_t s = 0; s < shots; ++s) out[s] = dd(gen);
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

// One launch per register size for the chunks of `batch`, enqueued on the
// lane's stream with the results copied to pinned host memory behind them;
// complete_batch waits for them and finishes the requests whose last shots
// landed. The lane keeps two batches in flight, so the host prepares the next
// launch while the current one runs.
Pending launch_batch(qgpu_server* S, qgpu_ctx* ctx, std::vector<Chunk>& batch, PinnedBuf* pin) {
    Pending pd;
    pd.pin = pin;
    std::map<uint32_t, std::vector<Chunk>> by_n;
    for (const Chunk& ch : batch) by_n[ch.r->prog->n].push_back(ch);
    // host result space of every class, carved from the pinned buffer
    std::vector<size_t> host_off;
    size_t host_bytes = 0;
    for (auto& kv : by_n) {
        ClassLaunch cl;
        cl.n = kv.first;
        cl.cs = kv.second;
        for (const Chunk& ch : cl.cs) {
            cl.maxcreg = std::max<uint32_t>(cl.maxcreg, std::max<uint32_t>(ch.r->prog->ncreg, 1));
            cl.nwork += ch.r->kind == QGPU_KET ? ch.ns : 1;
            if (ch.r->kind != QGPU_KET) cl.ndiag += uint64_t(1) << (cl.n / 2);
        }
        host_off.push_back(host_bytes);
        host_bytes += (cl.nwork * cl.maxcreg * 4 + 7) / 8 * 8 + cl.nwork * 8 + cl.ndiag * 8;
        pd.classes.push_back(std::move(cl));
    }
    auto* hbase = static_cast<unsigned char*>(pin->get(std::max<size_t>(host_bytes, 64)));
    for (size_t k = 0; k < pd.classes.size(); ++k) {
        ClassLaunch& cl = pd.classes[k];
        unsigned char* h = hbase + host_off[k];
        cl.hd = reinterpret_cast<uint32_t*>(h);
        h += (cl.nwork * cl.maxcreg * 4 + 7) / 8 * 8;
        cl.hs = reinterpret_cast<uint64_t*>(h);
        h += cl.nwork * 8;
        cl.hdiag = reinterpret_cast<double*>(h);
    }
    for (ClassLaunch& cl : pd.classes) {
        const uint32_t n = cl.n;
        auto& cs = cl.cs;
        std::vector<TInstr> ins;
        std::vector<float> mats;
        std::vector<std::pair<size_t, size_t>> pofs; // (ins offset, mat offset) per chunk
        // registers above shared-memory size run cache-blocked tile passes
        const int T = tile_width(ctx, int(n));
        std::vector<TProgram> tiled;
        if (T) {
            tiled.reserve(cs.size());
            for (const Chunk& ch : cs) {
                tiled.push_back(*ch.r->prog);
                plan_tiles(tiled.back(), T);
            }
        }
        for (size_t ci = 0; ci < cs.size(); ++ci) {
            const TProgram* P = T ? &tiled[ci] : cs[ci].r->prog;
            pofs.push_back({ins.size(), mats.size() / 2});
            ins.insert(ins.end(), P->ins.begin(), P->ins.end());
            mats.insert(mats.end(), P->mats.begin(), P->mats.end());
        }
        const uint64_t N = uint64_t(1) << n, nwork = cl.nwork, maxcreg = cl.maxcreg;
        auto al = [](size_t x) { return (x + 255) / 256 * 256; };
        size_t b_ins = std::max<size_t>(ins.size() * sizeof(TInstr), 16);
        size_t b_mat = std::max<size_t>(mats.size() * sizeof(float), 16);
        size_t b_work = nwork * sizeof(TWork);
        size_t b_dits = nwork * maxcreg * sizeof(uint32_t);
        size_t b_samp = nwork * sizeof(uint64_t);
        size_t b_g = n > uint32_t(kTrajMaxQubits)
                         ? size_t(traj_global_grid(ctx, int(nwork), int(n))) * N * sizeof(float2)
                         : 0;
        size_t b_diag = std::max<size_t>(cl.ndiag * sizeof(double), 16);
        size_t total = al(b_ins) + al(b_mat) + al(b_work) + al(b_dits) + al(b_samp) + al(b_g) +
                       al(b_diag);
        unsigned char* buf = nullptr;
        QG_CUDA(qgpu::ctx_malloc(ctx, reinterpret_cast<void**>(&buf), total));
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
        auto* ddiag = reinterpret_cast<double*>(take(b_diag));
        std::vector<TWork> work;
        work.reserve(nwork);
        uint32_t out = 0;
        uint64_t doff = 0;
        cl.diag_at.assign(cs.size(), 0);
        for (size_t i = 0; i < cs.size(); ++i) {
            const Chunk& ch = cs[i];
            const TProgram* P = T ? &tiled[i] : ch.r->prog;
            const bool rho = ch.r->kind != QGPU_KET;
            const uint64_t nw = rho ? 1 : ch.ns;
            for (uint64_t k = 0; k < nw; ++k) {
                TWork w{};
                w.prog = dins + pofs[i].first;
                w.mats = dmat + pofs[i].second;
                w.nins = uint32_t(P->ins.size());
                w.n = uint8_t(n);
                w.p_noise = rho ? 0.f : float(ch.r->p);
                w.shot = uint32_t(ch.s0 + k); // the request's own shot index
                w.out = out++;
                w.seed = ch.r->seed;
                if (rho) {
                    w.diag = ddiag + doff;
                    cl.diag_at[i] = doff;
                    doff += uint64_t(1) << (n / 2);
                }
                work.push_back(w);
            }
        }
        // pageable sources: staged by the runtime before these calls return
        QG_CUDA(cudaMemcpyAsync(dins, ins.data(), ins.size() * sizeof(TInstr),
                                cudaMemcpyHostToDevice, ctx->stream));
        if (!mats.empty())
            QG_CUDA(cudaMemcpyAsync(dmat, mats.data(), mats.size() * sizeof(float),
                                    cudaMemcpyHostToDevice, ctx->stream));
        QG_CUDA(cudaMemcpyAsync(dwork, work.data(), b_work, cudaMemcpyHostToDevice, ctx->stream));
        QG_CUDA(cudaMemsetAsync(ddits, 0, b_dits, ctx->stream));
        launch_traj(ctx, dwork, int(nwork), int(n), ddits, int(maxcreg), dsamp, nullptr,
                    nullptr, 0, dg, nullptr, T);
        QG_CUDA(cudaMemcpyAsync(cl.hd, ddits, b_dits, cudaMemcpyDeviceToHost, ctx->stream));
        QG_CUDA(cudaMemcpyAsync(cl.hs, dsamp, b_samp, cudaMemcpyDeviceToHost, ctx->stream));
        if (cl.ndiag)
            QG_CUDA(cudaMemcpyAsync(cl.hdiag, ddiag, cl.ndiag * sizeof(double),
                                    cudaMemcpyDeviceToHost, ctx->stream));
        QG_CUDA(cudaFreeAsync(buf, ctx->stream));
        std::lock_guard<std::mutex> lock(S->mu);
        S->launched_traj += nwork;
    }
    QG_CUDA(cudaEventCreateWithFlags(&pd.done, cudaEventDisableTiming));
    QG_CUDA(cudaEventRecord(pd.done, ctx->stream));
    return pd;
}

void complete_batch(qgpu_server* S, Pending& pd) {
    cudaError_t e = cudaEventSynchronize(pd.done);
    cudaEventDestroy(pd.done);
    pd.done = nullptr;
    if (e != cudaSuccess) raise(QGPU_ERR_CUDA, "qgpu_server", cudaGetErrorString(e));
    for (ClassLaunch& cl : pd.classes) {
        uint64_t out = 0;
        for (size_t i = 0; i < cl.cs.size(); ++i) {
            const Chunk& ch = cl.cs[i];
            Request* r = ch.r;
            const uint32_t nc = std::max<uint32_t>(r->c->nc, 1);
            if (r->kind != QGPU_KET) {
                const uint64_t Dh = uint64_t(1) << (cl.n / 2);
                std::vector<double> dg(cl.hdiag + cl.diag_at[i], cl.hdiag + cl.diag_at[i] + Dh);
                sample_diag(dg, r->shots, r->seed, r->samples.data());
                ++out;
            } else {
                for (uint64_t k = 0; k < ch.ns; ++k, ++out) {
                    const uint64_t sh = ch.s0 + k;
                    r->samples[sh] = cl.hs[out];
                    for (uint32_t q = 0; q < nc; ++q)
                        r->dits[sh * nc + q] = cl.hd[out * cl.maxcreg + q];
                }
            }
            r->landed += ch.ns;
            if (r->landed == r->shots) finish(S, r);
        }
    }
}

// Shots of one request in one launch, and shots per launch of a lane. Small
// launches let new arrivals in sooner but leave waves half full; measured on
// the serving mix (one B200, Poisson 1000 req/s), 256-shot slices in launches
// of two CTA waves cut the median latency from 87 to 12 ms but the
// throughput from 482 to 307 circuits/s, so launches stay large: a slice
// holds up to 4096 shots (every request of the mix whole) and a launch up to
// 64 CTAs per SM.
constexpr uint64_t kChunkShots = 4096;
uint64_t lane_shot_budget(const qgpu_ctx* ctx, int lane) {
    return uint64_t(ctx->num_sms) * (lane == 0 ? 64 : 16);
}

void lane_loop(qgpu_server* S, int li) {
    Lane& L = S->lanes[li];
    cudaSetDevice(L.ctx->device);
    const bool batching = li < 2;
    std::deque<Pending> inflight; // batching lanes: at most two
    int next_pin = 0;
    auto fail_chunks = [&](const std::vector<Chunk>& chunks, const Exc& e) {
        for (const Chunk& ch : chunks) {
            if (ch.r->done) continue;
            // the request's other shots may still be queued: take them out
            {
                std::lock_guard<std::mutex> lock(S->mu);
                L.q.erase(std::remove(L.q.begin(), L.q.end(), ch.r), L.q.end());
            }
            fail(S, ch.r, e.code, e.where + ": " + e.what);
        }
    };
    auto retire = [&] {
        Pending pd = std::move(inflight.front());
        inflight.pop_front();
        std::vector<Chunk> all;
        for (auto& cl : pd.classes) all.insert(all.end(), cl.cs.begin(), cl.cs.end());
        try {
            complete_batch(S, pd);
        } catch (const Exc& e) {
            fail_chunks(all, e);
        }
    };
    for (;;) {
        std::vector<Request*> got;
        std::vector<Chunk> chunks;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            if (inflight.empty())
                S->cv_work.wait(lock, [&] { return S->stop || !L.q.empty(); });
            if (S->stop && L.q.empty() && inflight.empty()) return;
            if (!batching) {
                got.push_back(L.q.front());
                L.q.pop_front();
            } else {
                // shots of the waiting requests in arrival order, at most
                // kChunkShots of each, within the launch's shot budget and the
                // HBM budget estimate (per-CTA slots for >= 15 qubits, outputs
                // otherwise); fully issued requests leave the queue
                const uint64_t shot_budget = lane_shot_budget(L.ctx, li);
                uint64_t used = 0, shots = 0;
                for (auto it = L.q.begin(); it != L.q.end() && shots < shot_budget;) {
                    Request* r = *it;
                    const bool rho = r->kind != QGPU_KET;
                    uint64_t ns = rho ? r->shots
                                      : std::min<uint64_t>({r->shots - r->issued, kChunkShots,
                                                            shot_budget - shots});
                    const uint64_t work = rho ? 1 : ns;
                    const uint64_t need = work * 64 + (r->prog->n > uint32_t(kTrajMaxQubits)
                                                           ? (uint64_t(8) << r->prog->n) * 8
                                                           : 0);
                    if (!chunks.empty() && used + need > S->budget) break;
                    if (r->issued == 0) {
                        const uint32_t nc = std::max<uint32_t>(r->c->nc, 1);
                        r->dits.assign(r->shots * nc, 0);
                        r->samples.assign(r->shots, 0);
                    }
                    chunks.push_back({r, r->issued, ns});
                    r->issued += ns;
                    used += need;
                    shots += work;
                    if (r->issued == r->shots) it = L.q.erase(it);
                    else ++it;
                }
            }
        }
        auto t0 = Clock::now();
        if (batching) {
            if (!chunks.empty()) {
                // the pinned slot of the batch two launches back is free once
                // that batch is retired
                if (inflight.size() >= 2) retire();
                try {
                    inflight.push_back(launch_batch(S, L.ctx, chunks, &L.pin[next_pin]));
                    next_pin ^= 1;
                } catch (const Exc& e) {
                    fail_chunks(chunks, e);
                }
            }
            // with nothing new to launch (or two in flight), wait for the oldest
            if (!inflight.empty() && (chunks.empty() || inflight.size() >= 2)) retire();
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
        if (batching) {
            if (!chunks.empty()) ++S->batches;
        } else {
            S->engine_runs += got.size();
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
                if (r->prog) {
                    const uint32_t n = r->prog->n;
                    if (n <= uint32_t(qgpu::kTrajMaxQubits)) lane = 0;
                    else if (kind == QGPU_KET && n <= uint32_t(qgpu::kServeMaxSlotQubits)) lane = 1;
                    else r->prog = nullptr; // one CTA per register is too slow
                }
                if (kind != QGPU_KET && !r->prog) {
                    // fused superoperator passes on lane 2 when it compiles
                    auto it = S->rho_fused.find(c);
                    if (it == S->rho_fused.end()) {
                        qgpu::TProgram P;
                        it = S->rho_fused.emplace(c, qgpu::compile_traj_rho(c, P, 30)).first;
                    }
                    r->fused_rho = it->second;
                }
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
