// ops.cpp -- planning of Quantum++ ops onto the virtual-ket kernels.
#include "ops.hpp"

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <cmath>
#include <cstring>

#include "kernels.hpp"

namespace qgpu {

VSpace vspace_ket(const std::vector<uint64_t>& dims) {
    VSpace v;
    v.dims = dims;
    v.strides.assign(dims.size(), 1);
    for (size_t q = dims.size(); q-- > 1;) v.strides[q - 1] = v.strides[q] * dims[q];
    return v;
}

VSpace vspace_rho(const std::vector<uint64_t>& dims) {
    VSpace k = vspace_ket(dims);
    uint64_t D = 1;
    for (uint64_t d : dims) D *= d;
    VSpace v;
    size_t n = dims.size();
    v.dims.resize(2 * n);
    v.strides.resize(2 * n);
    for (size_t q = 0; q < n; ++q) {
        v.dims[q] = dims[q]; // column digit q
        v.strides[q] = k.strides[q] * D;
        v.dims[n + q] = dims[q]; // row digit q
        v.strides[n + q] = k.strides[q];
    }
    return v;
}

VSpace vspace_of(const qgpu_state* s) {
    return s->kind == QGPU_KET ? vspace_ket(s->dims) : vspace_rho(s->dims);
}

static void push_seg(SegPlan& p, uint64_t size, uint64_t stride) {
    if (size == 1) return;
    if (p.nseg >= kMaxSeg)
        raise(QGPU_ERR_NOT_SUPPORTED, "qgpu planner", "too many index segments");
    p.size[p.nseg] = size;
    p.stride[p.nseg] = stride;
    ++p.nseg;
}

static void finish_plan(SegPlan& p) {
    p.count = 1;
    p.pow2 = 1;
    for (int s = 0; s < p.nseg; ++s) {
        p.count *= p.size[s];
        uint64_t z = p.size[s];
        if (z & (z - 1)) p.pow2 = 0;
        int sh = 0;
        while ((uint64_t(1) << sh) < z) ++sh;
        p.shift[s] = uint8_t(sh);
    }
}

SegPlan plan_free(const VSpace& vs, const std::vector<int>& excluded,
                  uint64_t fixed_off) {
    SegPlan p;
    std::memset(&p, 0, sizeof(p));
    p.fixed_off = fixed_off;
    size_t N = vs.dims.size();
    std::vector<char> ex(N, 0);
    for (int v : excluded) ex[size_t(v)] = 1;
    bool run = false;
    uint64_t cs = 1, cst = 0;
    for (size_t v = N; v-- > 0;) {
        if (ex[v]) {
            if (run) push_seg(p, cs, cst);
            run = false;
            continue;
        }
        if (!run) {
            cs = vs.dims[v];
            cst = vs.strides[v];
            run = true;
        } else if (vs.strides[v] == cst * cs) {
            cs *= vs.dims[v];
        } else {
            push_seg(p, cs, cst);
            cs = vs.dims[v];
            cst = vs.strides[v];
        }
    }
    if (run) push_seg(p, cs, cst);
    finish_plan(p);
    return p;
}

SegPlan plan_gather(const std::vector<uint64_t>& out_dims,
                    const std::vector<uint64_t>& src, uint64_t fixed_off) {
    SegPlan p;
    std::memset(&p, 0, sizeof(p));
    p.fixed_off = fixed_off;
    bool run = false;
    uint64_t cs = 1, cst = 0;
    for (size_t v = out_dims.size(); v-- > 0;) {
        if (out_dims[v] == 1) continue;
        if (!run) {
            cs = out_dims[v];
            cst = src[v];
            run = true;
        } else if (src[v] == cst * cs) {
            cs *= out_dims[v];
        } else {
            push_seg(p, cs, cst);
            cs = out_dims[v];
            cst = src[v];
        }
    }
    if (run) push_seg(p, cs, cst);
    finish_plan(p);
    return p;
}

std::vector<uint64_t> target_offsets(const VSpace& vs,
                                     const std::vector<int>& targets) {
    uint64_t DA = 1;
    for (int t : targets) DA *= vs.dims[size_t(t)];
    std::vector<uint64_t> off(DA);
    for (uint64_t m = 0; m < DA; ++m) {
        uint64_t r = m, o = 0;
        for (size_t j = targets.size(); j-- > 0;) {
            uint64_t d = vs.dims[size_t(targets[j])];
            o += (r % d) * vs.strides[size_t(targets[j])];
            r /= d;
        }
        off[m] = o;
    }
    return off;
}

std::vector<cd> conj_mat(const std::vector<cd>& A) {
    std::vector<cd> r(A.size());
    for (size_t i = 0; i < A.size(); ++i) r[i] = std::conj(A[i]);
    return r;
}

// kron(A, B), column-major, A da x da, B db x db
std::vector<cd> kron_mat(const std::vector<cd>& A, uint64_t da,
                         const std::vector<cd>& B, uint64_t db) {
    uint64_t m = da * db;
    std::vector<cd> r(m * m);
    for (uint64_t i1 = 0; i1 < da; ++i1)
        for (uint64_t j1 = 0; j1 < da; ++j1)
            for (uint64_t i2 = 0; i2 < db; ++i2)
                for (uint64_t j2 = 0; j2 < db; ++j2)
                    r[(i1 * db + i2) + (j1 * db + j2) * m] =
                        A[i1 + j1 * da] * B[i2 + j2 * db];
    return r;
}

std::vector<cd> mat_pow(const std::vector<cd>& A, uint64_t m, uint64_t k) {
    std::vector<cd> r(m * m, 0.0), t(m * m);
    for (uint64_t i = 0; i < m; ++i) r[i + i * m] = 1.0;
    for (uint64_t e = 0; e < k; ++e) {
        std::fill(t.begin(), t.end(), cd(0.0));
        for (uint64_t j = 0; j < m; ++j)
            for (uint64_t l = 0; l < m; ++l) {
                cd a = A[l + j * m];
                for (uint64_t i = 0; i < m; ++i) t[i + j * m] += r[i + l * m] * a;
            }
        r.swap(t);
    }
    return r;
}

qgpu_state* new_state(qgpu_ctx* ctx, qgpu_kind kind, qgpu_prec prec,
                      const std::vector<uint64_t>& dims, bool zero) {
    auto* s = new qgpu_state;
    s->ctx = ctx;
    s->kind = kind;
    s->prec = prec;
    s->dims = dims;
    s->D = 1;
    for (uint64_t d : dims) s->D *= d;
    s->elems = kind == QGPU_KET ? s->D : s->D * s->D;
    cudaError_t e = ctx_malloc(ctx, &s->data, s->bytes());
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete s;
        raise(QGPU_ERR_OUT_OF_MEMORY, "qgpu_state_create()",
              "device allocation failed");
    }
    ctx->live_states.fetch_add(1);
    if (zero) {
        cudaError_t z = cudaMemsetAsync(s->data, 0, s->bytes(), ctx->stream);
        if (z != cudaSuccess) {
            free_state(s);
            raise(QGPU_ERR_CUDA, "qgpu_state_create()", cudaGetErrorString(z));
        }
    }
    return s;
}

void free_state(qgpu_state* s) {
    if (!s) return;
    qgpu_ctx* ctx = s->ctx;
    if (s->data) cudaFreeAsync(s->data, ctx->stream);
    delete s;
    if (ctx->live_states.fetch_sub(1) == 1 && ctx->closing.load()) destroy_ctx(ctx);
}

static bool all_two(const std::vector<uint64_t>& d) {
    for (uint64_t x : d)
        if (x != 2) return false;
    return true;
}

void vapply(qgpu_state* s, const VSpace& vs, const std::vector<int>& vt,
            const std::vector<std::pair<int, uint64_t>>& fixed, const cd* A,
            uint64_t DA) {
    if (s->elems <= 1) return;
    if (fixed.empty() && all_two(vs.dims) && (vt.size() == 1 || vt.size() == 2)) {
        int nbits = int(vs.dims.size());
        if (vt.size() == 1) {
            launch_qubit_1q(s->ctx, s->prec, s->data, nbits, nbits - 1 - vt[0], A);
        } else {
            launch_qubit_2q(s->ctx, s->prec, s->data, nbits, nbits - 1 - vt[0],
                            nbits - 1 - vt[1], A);
        }
        return;
    }
    std::vector<int> ex = vt;
    uint64_t foff = 0;
    for (auto& f : fixed) {
        ex.push_back(f.first);
        foff += f.second * vs.strides[size_t(f.first)];
    }
    SegPlan outer = plan_free(vs, ex, foff);
    std::vector<uint64_t> off = target_offsets(vs, vt);
    launch_apply_generic(s->ctx, s->prec, s->data, outer, off, A, DA);
}

static std::vector<int> as_int(const std::vector<uint64_t>& v, int add = 0) {
    std::vector<int> r;
    for (uint64_t x : v) r.push_back(int(x) + add);
    return r;
}

void op_apply(qgpu_state* s, const cd* A, uint64_t DA,
              const std::vector<uint64_t>& target) {
    VSpace vs = vspace_of(s);
    if (s->kind == QGPU_KET) {
        vapply(s, vs, as_int(target), {}, A, DA);
        return;
    }
    int n = int(s->dims.size());
    std::vector<cd> U(A, A + DA * DA);
    if (DA <= 4) {
        std::vector<cd> S = kron_mat(conj_mat(U), DA, U, DA);
        std::vector<int> vt = as_int(target);
        std::vector<int> rows = as_int(target, n);
        vt.insert(vt.end(), rows.begin(), rows.end());
        vapply(s, vs, vt, {}, S.data(), DA * DA);
    } else {
        vapply(s, vs, as_int(target, n), {}, U.data(), DA);
        std::vector<cd> Uc = conj_mat(U);
        vapply(s, vs, as_int(target), {}, Uc.data(), DA);
    }
}

void op_apply_ctrl(qgpu_state* s, const cd* A, uint64_t DA,
                   const std::vector<uint64_t>& ctrl,
                   const std::vector<uint64_t>& target,
                   const std::vector<uint64_t>& shift_inv, bool fan) {
    VSpace vs = vspace_of(s);
    uint64_t d = s->dims[ctrl[0]];
    uint64_t m = fan ? d : DA;
    std::vector<cd> U(A, A + m * m);
    int n = int(s->dims.size());
    for (uint64_t r = 1; r < d; ++r) {
        std::vector<cd> Ar = mat_pow(U, m, r);
        std::vector<cd> Arc = conj_mat(Ar);
        std::vector<std::pair<int, uint64_t>> fr, fc;
        for (size_t i = 0; i < ctrl.size(); ++i) {
            uint64_t dig = (shift_inv[i] + r) % d;
            if (s->kind == QGPU_KET) {
                fr.push_back({int(ctrl[i]), dig});
            } else {
                fr.push_back({int(ctrl[i]) + n, dig}); // row digits
                fc.push_back({int(ctrl[i]), dig});     // column digits
            }
        }
        std::vector<std::vector<uint64_t>> groups;
        if (fan)
            for (uint64_t t : target) groups.push_back({t});
        else
            groups.push_back(target);
        for (auto& g : groups) {
            if (s->kind == QGPU_KET) {
                vapply(s, vs, as_int(g), fr, Ar.data(), m);
            } else {
                vapply(s, vs, as_int(g, n), fr, Ar.data(), m);
                vapply(s, vs, as_int(g), fc, Arc.data(), m);
            }
        }
    }
}

// A two-qubit channel's superoperator S (16 x 16, column-major, index bits
// (column a, column b, row a, row b)) factors as A (x) B, with A on
// (column a, row a) and B on (column b, row b), exactly when the channel is
// a product of one-qubit channels (independent noise on each qubit). S
// rearranged as R[(a row, a col)][(b row, b col)] then has rank one: R = u v^T.
// True (and A, B column-major over index 2 c + r) when every entry of R
// matches u v^T within 1e-13 of R's largest entry.
static bool kron_factor_16(const std::vector<cd>& S, cd* A, cd* B) {
    cd R[16][16];
    for (int x = 0; x < 16; ++x)
        for (int y = 0; y < 16; ++y) {
            const int ca = x >> 3 & 1, cb = x >> 2 & 1, ra = x >> 1 & 1, rb = x & 1;
            const int ca2 = y >> 3 & 1, cb2 = y >> 2 & 1, ra2 = y >> 1 & 1, rb2 = y & 1;
            const int ai = (2 * ca + ra) + 4 * (2 * ca2 + ra2);
            const int bi = (2 * cb + rb) + 4 * (2 * cb2 + rb2);
            R[ai][bi] = S[size_t(x) + 16 * size_t(y)];
        }
    int P = 0, Q = 0;
    double big = 0.0;
    for (int i = 0; i < 16; ++i)
        for (int j = 0; j < 16; ++j)
            if (std::abs(R[i][j]) > big) {
                big = std::abs(R[i][j]);
                P = i;
                Q = j;
            }
    if (big == 0.0) return false;
    for (int i = 0; i < 16; ++i) {
        A[i] = R[i][Q];
        B[i] = R[P][i] / R[P][Q];
    }
    for (int i = 0; i < 16; ++i)
        for (int j = 0; j < 16; ++j)
            if (std::abs(R[i][j] - A[i] * B[j]) > 1e-13 * big) return false;
    return true;
}

// Superoperators of recently applied Kraus sets, keyed by their bytes: a
// channel applied at every step of a circuit is built (and factored) once,
// as qpp keeps one copy of each distinct gate matrix (cmat_hash_tbl_,
// qcircuit.hpp:102-136).
namespace {
struct ChannelEntry {
    std::vector<cd> Ks; // the key, compared in full
    uint64_t DA = 0;
    std::vector<cd> S;
    bool factored = false;
    cd A[16], B[16];
};
std::mutex g_chan_mu;
std::vector<std::shared_ptr<ChannelEntry>> g_chan; // most recent last
constexpr size_t kChanCache = 32;

std::shared_ptr<ChannelEntry> channel_of(const cd* Ks, uint32_t nK, uint64_t DA) {
    const size_t len = size_t(nK) * DA * DA;
    {
        std::lock_guard<std::mutex> lock(g_chan_mu);
        for (size_t i = g_chan.size(); i-- > 0;) {
            const auto& e = g_chan[i];
            if (e->DA == DA && e->Ks.size() == len &&
                std::memcmp(e->Ks.data(), Ks, len * sizeof(cd)) == 0)
                return e;
        }
    }
    auto e = std::make_shared<ChannelEntry>();
    e->Ks.assign(Ks, Ks + len);
    e->DA = DA;
    const uint64_t DS = DA * DA;
    e->S.assign(DS * DS, 0.0);
    for (uint32_t i = 0; i < nK; ++i) {
        std::vector<cd> K(Ks + size_t(i) * DA * DA, Ks + size_t(i + 1) * DA * DA);
        std::vector<cd> t = kron_mat(conj_mat(K), DA, K, DA);
        for (size_t j = 0; j < t.size(); ++j) e->S[j] += t[j];
    }
    if (DA == 4) e->factored = kron_factor_16(e->S, e->A, e->B);
    std::lock_guard<std::mutex> lock(g_chan_mu);
    if (g_chan.size() >= kChanCache) g_chan.erase(g_chan.begin());
    g_chan.push_back(e);
    return e;
}
} // namespace

void op_apply_kraus(qgpu_state* s, const cd* Ks, uint32_t nK, uint64_t DA,
                    const std::vector<uint64_t>& target) {
    uint64_t DS = DA * DA;
    if (DS > 4096)
        raise(QGPU_ERR_NOT_SUPPORTED, "qpp::apply()",
              "Kraus superoperator above 4096 x 4096");
    const std::shared_ptr<ChannelEntry> ch = channel_of(Ks, nK, DA);
    const std::vector<cd>& S = ch->S;
    VSpace vs = vspace_of(s);
    int n = int(s->dims.size());
    // a product channel on two qubits of a density matrix: one pass with the
    // two 4 x 4 factors (half the arithmetic of the 16 x 16)
    if (s->kind == QGPU_RHO && DA == 4 && target.size() == 2 && s->dims[target[0]] == 2 &&
        s->dims[target[1]] == 2 && ch->factored) {
        const int a = int(target[0]), b = int(target[1]);
        const std::vector<int> kt = {a, n + a, b, n + b};
        launch_apply_kron4(s->ctx, s->prec, s->data, plan_free(vs, kt, 0),
                           target_offsets(vs, kt), ch->A, ch->B);
        return;
    }
    std::vector<int> vt = as_int(target), rows = as_int(target, n);
    vt.insert(vt.end(), rows.begin(), rows.end());
    vapply(s, vs, vt, {}, S.data(), DS);
}

static std::vector<uint64_t> complement(const std::vector<uint64_t>& t,
                                        size_t n) {
    std::vector<uint64_t> r;
    for (uint64_t i = 0; i < n; ++i)
        if (std::find(t.begin(), t.end(), i) == t.end()) r.push_back(i);
    return r;
}

static void upload_scalar(qgpu_state* out, cd v) {
    if (out->prec == QGPU_C128) {
        double h[2] = {v.real(), v.imag()};
        QG_CUDA(cudaMemcpyAsync(out->data, h, sizeof(h), cudaMemcpyHostToDevice,
                                out->ctx->stream));
        QG_CUDA(cudaStreamSynchronize(out->ctx->stream));
    } else {
        float h[2] = {float(v.real()), float(v.imag())};
        QG_CUDA(cudaMemcpyAsync(out->data, h, sizeof(h), cudaMemcpyHostToDevice,
                                out->ctx->stream));
        QG_CUDA(cudaStreamSynchronize(out->ctx->stream));
    }
}

qgpu_state* op_ptrace(const qgpu_state* s, const std::vector<uint64_t>& target) {
    size_t n = s->dims.size();
    std::vector<uint64_t> bar = complement(target, n);
    std::vector<uint64_t> dbar;
    for (uint64_t q : bar) dbar.push_back(s->dims[q]);
    if (dbar.empty()) dbar.push_back(1);
    qgpu_state* out = new_state(s->ctx, QGPU_RHO, s->prec, dbar, false);
    try {
        VSpace k = vspace_ket(s->dims);
        uint64_t D = s->D;
        bool ket = s->kind == QGPU_KET;
        if (target.size() == n) {
            cd v = ket ? cd(op_norm2(s), 0.0) : op_trace(s);
            upload_scalar(out, v);
            return out;
        }
        std::vector<uint64_t> od, sa, sb;
        // output digits: [column digits of bar, row digits of bar]
        for (uint64_t q : bar) {
            od.push_back(s->dims[q]);
            sa.push_back(ket ? 0 : k.strides[q] * D);
            sb.push_back(ket ? k.strides[q] : 0);
        }
        for (uint64_t q : bar) {
            od.push_back(s->dims[q]);
            sa.push_back(k.strides[q]);
            sb.push_back(0);
        }
        SegPlan ma = plan_gather(od, sa, 0), mb = plan_gather(od, sb, 0);
        uint64_t DS = 1;
        for (uint64_t t : target) DS *= s->dims[t];
        std::vector<uint64_t> toff(DS);
        for (uint64_t a = 0; a < DS; ++a) {
            uint64_t r = a, o = 0;
            for (size_t j = target.size(); j-- > 0;) {
                uint64_t d = s->dims[target[j]];
                uint64_t dig = r % d;
                r /= d;
                o += dig * (ket ? k.strides[target[j]]
                                : k.strides[target[j]] * (D + 1));
            }
            toff[a] = o;
        }
        if (target.empty() && !ket) {
            QG_CUDA(cudaMemcpyAsync(out->data, s->data, s->bytes(),
                                    cudaMemcpyDeviceToDevice, s->ctx->stream));
            return out;
        }
        launch_ptrace(s->ctx, s->prec, s->data, out->data, ma, mb, toff, ket);
    } catch (...) {
        free_state(out);
        throw;
    }
    return out;
}

qgpu_state* op_ptranspose(const qgpu_state* s,
                          const std::vector<uint64_t>& target) {
    size_t n = s->dims.size();
    qgpu_state* out = new_state(s->ctx, QGPU_RHO, s->prec, s->dims, false);
    try {
        VSpace k = vspace_ket(s->dims);
        uint64_t D = s->D;
        std::vector<char> inT(n, 0);
        for (uint64_t t : target) inT[t] = 1;
        std::vector<uint64_t> od, sa, sb;
        for (size_t q = 0; q < n; ++q) od.push_back(s->dims[q]);
        for (size_t q = 0; q < n; ++q) od.push_back(s->dims[q]);
        if (s->kind == QGPU_RHO) {
            for (size_t q = 0; q < n; ++q) // output column digit q
                sa.push_back(inT[q] ? k.strides[q] : k.strides[q] * D);
            for (size_t q = 0; q < n; ++q) // output row digit q
                sa.push_back(inT[q] ? k.strides[q] * D : k.strides[q]);
            if (!launch_permute_tiled(s->ctx, s->prec, s->data, out->data, od, sa, 0))
                launch_gather(s->ctx, s->prec, s->data, out->data, plan_gather(od, sa, 0));
        } else {
            for (size_t q = 0; q < n; ++q) {
                sa.push_back(inT[q] ? k.strides[q] : 0);
                sb.push_back(inT[q] ? 0 : k.strides[q]);
            }
            for (size_t q = 0; q < n; ++q) {
                sa.push_back(inT[q] ? 0 : k.strides[q]);
                sb.push_back(inT[q] ? k.strides[q] : 0);
            }
            launch_gather_outer(s->ctx, s->prec, s->data, out->data,
                                plan_gather(od, sa, 0), plan_gather(od, sb, 0));
        }
    } catch (...) {
        free_state(out);
        throw;
    }
    return out;
}

qgpu_state* op_syspermute(const qgpu_state* s,
                          const std::vector<uint64_t>& perm) {
    size_t n = s->dims.size();
    std::vector<uint64_t> nd(n);
    for (size_t k = 0; k < n; ++k) nd[k] = s->dims[perm[k]];
    qgpu_state* out = new_state(s->ctx, s->kind, s->prec, nd, false);
    try {
        VSpace k = vspace_ket(s->dims);
        std::vector<uint64_t> od, sa;
        if (s->kind == QGPU_RHO) {
            for (size_t q = 0; q < n; ++q) {
                od.push_back(nd[q]);
                sa.push_back(k.strides[perm[q]] * s->D);
            }
        }
        for (size_t q = 0; q < n; ++q) {
            od.push_back(nd[q]);
            sa.push_back(k.strides[perm[q]]);
        }
        if (!launch_permute_tiled(s->ctx, s->prec, s->data, out->data, od, sa, 0))
            launch_gather(s->ctx, s->prec, s->data, out->data, plan_gather(od, sa, 0));
    } catch (...) {
        free_state(out);
        throw;
    }
    return out;
}

double op_norm2(const qgpu_state* s) {
    return reduce_norm2(s->ctx, s->prec, s->data, s->elems);
}

cd op_trace(const qgpu_state* s) {
    if (s->kind == QGPU_KET) return cd(op_norm2(s), 0.0);
    return reduce_strided_sum(s->ctx, s->prec, s->data, s->D, s->D + 1);
}

bool op_normalize(qgpu_state* s) {
    if (s->kind == QGPU_KET) {
        double nn = std::sqrt(op_norm2(s));
        if (nn == 0) return false;
        launch_scale(s->ctx, s->prec, s->data, s->elems, cd(1.0 / nn, 0.0));
    } else {
        cd tr = op_trace(s);
        if (std::abs(tr) == 0) return false;
        launch_scale(s->ctx, s->prec, s->data, s->elems, cd(1.0, 0.0) / tr);
    }
    return true;
}

} // namespace qgpu
