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
//   lane 2  everything else, one request at a time on each of two workers
//           (own contexts, highest stream priority): density matrices above
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
// Each register size of these lanes has its own stream and keeps up to two
// launches in flight: sizes run side by side and land independently, the
// host builds and enqueues the next launch while the current one runs, and
// results come back through pinned memory.
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

// One register size of a batching lane: its own context (stream), so sizes
// run concurrently and land independently, with at most two launches in
// flight and their pinned result buffers.
struct ClassRun {
    qgpu_ctx* ctx = nullptr;
    PinnedBuf pin[2];
    int next_pin = 0;
    std::deque<Pending> inflight;
    ~ClassRun() {
        if (ctx) qgpu_ctx_destroy(ctx);
    }
};

struct Lane {
    qgpu_ctx* ctx = nullptr;
    std::deque<Request*> q;
    std::thread th;
    std::map<uint32_t, std::unique_ptr<ClassRun>> cls; // batching lanes, by register size
};

} // namespace qgpu

struct qgpu_server {
    int mode = 0;
    uint64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    qgpu::Lane lanes[3];
    // lane 2's second worker: its own context, so a long density matrix does
    // not hold the small ones behind it
    qgpu_ctx* engine2 = nullptr;
    std::thread engine2_th;
    // the lazily built per-circuit forms (fused programs, tensor-core block
    // images) are prepared under this lock, so two workers never build the
    // same circuit's at once
    std::mutex prep_mu;
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
void run_rho_fused(qgpu_ctx* ctx, Request* r, std::mutex& prep_mu) {
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
    {
        std::lock_guard<std::mutex> lock(prep_mu);
        fused_prepare(st, r->c); // once per circuit; a no-op afterwards
    }
    run_gates(st, r->c, 1, 0, r->c->steps.size());
    sample_rho(ctx, st, r);
}

// Engine path: trajectories one shot at a time on the resident engine; a
// density matrix evolves once (its noise is in the circuit's channels) and
// the shots sample the final diagonal.
void run_engine(qgpu_ctx* ctx, Request* r, qgpu_prec prec, std::mutex& prep_mu) {
    if (r->fused_rho && prec == QGPU_C64) {
        run_rho_fused(ctx, r, prep_mu);
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

// Shots of one request in one launch, and shots per launch of a register
// size. A launch's results land when its last trajectory ends, so a launch
// is sized in waves of the device's resident CTAs for that size: with a
// fixed 64 shots per SM, a 14-qubit launch (one resident CTA per SM) ran 64
// trajectories per CTA back to back and held its first requests' results
// for hundreds of milliseconds. Each size runs on its own stream with two
// launches in flight, so short launches keep the device full. A slice holds
// up to 4096 shots (every request of the mix whole).
constexpr uint64_t kChunkShots = 4096;
constexpr uint64_t kLaunchWaves = 4;
uint64_t class_shot_budget(qgpu_ctx* ctx, int lane, uint32_t n) {
    if (lane == 0) return uint64_t(traj_resident_slots(ctx, int(n))) * kLaunchWaves;
    return uint64_t(ctx->num_sms) * 16; // global slots: two waves of 8 per SM
}

// Lane 2's streams run at the device's highest priority: its requests are
// single long runs whose passes fill the GPU, and under load the batching
// lanes' many trajectory blocks would otherwise take most SMs as they free
// up, so the density matrices (the oldest work in the queue) finish last.
void raise_priority(qgpu_ctx* ctx) {
    int least = 0, greatest = 0;
    QG_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    cudaStream_t s = nullptr;
    QG_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, greatest));
    QG_CUDA(cudaStreamDestroy(ctx->stream)); // nothing has been queued on it yet
    ctx->stream = s;
}

// Batching lanes (0 and 1). Each register size has its own stream
// (ClassRun), so a long launch of one size (a few shots of an 18-qubit ket
// hold a few SMs for tens of milliseconds) delays neither the other sizes'
// launches nor their results. The lane thread admits shots in arrival order
// into the next launch of each size that has fewer than two launches in
// flight, and retires launches as their events complete (polled every
// 100 us while any is in flight).
void batching_loop(qgpu_server* S, int li) {
    Lane& L = S->lanes[li];
    cudaSetDevice(L.ctx->device);
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
    auto retire_front = [&](ClassRun& C) {
        Pending pd = std::move(C.inflight.front());
        C.inflight.pop_front();
        std::vector<Chunk> all;
        for (auto& cl : pd.classes) all.insert(all.end(), cl.cs.begin(), cl.cs.end());
        try {
            complete_batch(S, pd);
        } catch (const Exc& e) {
            fail_chunks(all, e);
        }
    };
    auto class_of = [&](uint32_t n) -> ClassRun& {
        auto& slot = L.cls[n];
        if (!slot) {
            slot.reset(new ClassRun);
            qgpu_status st = qgpu_ctx_create(L.ctx->device, &slot->ctx);
            if (st != QGPU_OK) {
                slot.reset();
                raise(st, "qgpu_server", "class context");
            }
        }
        return *slot;
    };
    for (;;) {
        // results first: every launch whose event has completed
        size_t inflight = 0;
        for (auto& kv : L.cls) {
            ClassRun& C = *kv.second;
            while (!C.inflight.empty() && cudaEventQuery(C.inflight.front().done) != cudaErrorNotReady)
                retire_front(C);
            inflight += C.inflight.size();
        }
        std::map<uint32_t, std::vector<Chunk>> by_n;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            if (inflight == 0)
                S->cv_work.wait(lock, [&] { return S->stop || !L.q.empty(); });
            if (S->stop && L.q.empty() && inflight == 0) return;
            // shots of the waiting requests in arrival order, at most
            // kChunkShots of each, within each size's launch budget and the
            // HBM budget estimate (per-CTA slots for >= 15 qubits, outputs
            // otherwise); sizes with two launches in flight wait; fully
            // issued requests leave the queue
            std::map<uint32_t, uint64_t> shots_of, budget_of;
            uint64_t used = 0;
            for (auto it = L.q.begin(); it != L.q.end();) {
                Request* r = *it;
                const uint32_t n = r->prog->n;
                auto c = L.cls.find(n);
                if (c != L.cls.end() && c->second && c->second->inflight.size() >= 2) {
                    ++it;
                    continue;
                }
                auto bud = budget_of.find(n);
                if (bud == budget_of.end())
                    bud = budget_of.emplace(n, class_shot_budget(L.ctx, li, n)).first;
                const uint64_t shot_budget = bud->second;
                uint64_t& shots = shots_of[n];
                if (shots >= shot_budget) {
                    ++it;
                    continue;
                }
                const bool rho = r->kind != QGPU_KET;
                uint64_t ns = rho ? r->shots
                                  : std::min<uint64_t>({r->shots - r->issued, kChunkShots,
                                                        shot_budget - shots});
                const uint64_t work = rho ? 1 : ns;
                const uint64_t need = work * 64 + (n > uint32_t(kTrajMaxQubits)
                                                       ? (uint64_t(8) << n) * 8
                                                       : 0);
                if (!by_n.empty() && used + need > S->budget) break;
                if (r->issued == 0) {
                    const uint32_t nc = std::max<uint32_t>(r->c->nc, 1);
                    r->dits.assign(r->shots * nc, 0);
                    r->samples.assign(r->shots, 0);
                }
                by_n[n].push_back({r, r->issued, ns});
                r->issued += ns;
                used += need;
                shots += work;
                if (r->issued == r->shots) it = L.q.erase(it);
                else ++it;
            }
            if (by_n.empty() && inflight > 0)
                S->cv_work.wait_for(lock, std::chrono::microseconds(100),
                                    [&] { return S->stop; });
        }
        if (by_n.empty()) continue;
        auto t0 = Clock::now();
        for (auto& kv : by_n) {
            try {
                ClassRun& C = class_of(kv.first);
                C.inflight.push_back(launch_batch(S, C.ctx, kv.second, &C.pin[C.next_pin]));
                C.next_pin ^= 1;
            } catch (const Exc& e) {
                fail_chunks(kv.second, e);
            }
        }
        std::lock_guard<std::mutex> lock(S->mu);
        S->batches += by_n.size();
        S->busy_s += std::chrono::duration<double>(Clock::now() - t0).count();
    }
}

// Lane 2: one request at a time per worker on the resident engine (or the
// fused density-matrix form); two workers, each with its own context, take
// requests from the lane's queue in arrival order.
void engine_loop(qgpu_server* S, int li, qgpu_ctx* ctx) {
    Lane& L = S->lanes[li];
    cudaSetDevice(ctx->device);
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            S->cv_work.wait(lock, [&] { return S->stop || !L.q.empty(); });
            if (S->stop && L.q.empty()) return;
            r = L.q.front();
            L.q.pop_front();
        }
        auto t0 = Clock::now();
        try {
            run_engine(ctx, r, S->mode == 1 ? QGPU_C128 : QGPU_C64, S->prep_mu);
            finish(S, r);
        } catch (const Exc& e) {
            fail(S, r, e.code, e.where + ": " + e.what);
        }
        std::lock_guard<std::mutex> lock(S->mu);
        S->engine_runs += 1;
        S->busy_s += std::chrono::duration<double>(Clock::now() - t0).count();
    }
}

void lane_loop(qgpu_server* S, int li) {
    if (li < 2) batching_loop(S, li);
    else engine_loop(S, li, S->lanes[li].ctx);
}


} // namespace
} // namespace qgpu

using qgpu::guarded;
using qgpu::need_handle;
using qgpu::raise;

extern "C" {

qgpu_status qgpu_server_create(int device, uint64_t hbm_budget, int mode, qgpu_server** out) {
    return guarded(__func__, [&] {
        if (!out) raise(QGPU_ERR_INVALID_ARGUMENT, "qgpu_server_create()", "out");
        if (mode != 0 && mode != 1)
            raise(QGPU_ERR_INVALID_ARGUMENT, "qgpu_server_create()", "mode");
        auto* S = new qgpu_server;
        S->mode = mode;
        S->budget = hbm_budget;
        qgpu_ctx** ctxs[4] = {&S->lanes[0].ctx, &S->lanes[1].ctx, &S->lanes[2].ctx, &S->engine2};
        for (int i = 0; i < 4; ++i) {
            qgpu_status st = qgpu_ctx_create(device, ctxs[i]);
            if (st == QGPU_OK && i >= 2)
                st = qgpu::guarded(__func__, [&] { qgpu::raise_priority(*ctxs[i]); });
            if (st != QGPU_OK) {
                for (int j = 0; j < 4; ++j)
                    if (*ctxs[j]) qgpu_ctx_destroy(*ctxs[j]);
                delete S;
                raise(st, "qgpu_server_create()", "context");
            }
        }
        for (int i = 0; i < 3; ++i) S->lanes[i].th = std::thread(qgpu::lane_loop, S, i);
        S->engine2_th = std::thread(qgpu::engine_loop, S, 2, S->engine2);
        *out = S;
    });
}

qgpu_status qgpu_server_submit(qgpu_server* S, qgpu_circuit* c, qgpu_kind kind, double p,
                               uint64_t shots, uint64_t seed, uint64_t* id) {
    return guarded(__func__, [&] {
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
    return guarded(__func__, [&] {
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
    return guarded(__func__, [&] {
        need_handle(S);
        std::lock_guard<std::mutex> lock(S->mu);
        if (batches) *batches = S->batches;
        if (trajectories) *trajectories = S->launched_traj;
        if (engine_runs) *engine_runs = S->engine_runs;
        if (busy_s) *busy_s = S->busy_s;
    });
}

qgpu_status qgpu_server_destroy(qgpu_server* S) {
    return guarded(__func__, [&] {
        if (!S) return;
        {
            std::lock_guard<std::mutex> lock(S->mu);
            S->stop = true;
        }
        S->cv_work.notify_all();
        for (auto& L : S->lanes)
            if (L.th.joinable()) L.th.join();
        if (S->engine2_th.joinable()) S->engine2_th.join();
        for (auto& kv : S->all) delete kv.second;
        for (auto& L : S->lanes) {
            L.cls.clear();
            qgpu_ctx_destroy(L.ctx);
        }
        qgpu_ctx_destroy(S->engine2);
        delete S;
    });
}

} // extern "C"
