// capi.cpp -- the extern "C" boundary of libqpp_b200.
//
// Each entry point validates its arguments in the order of the Quantum++
// function it replaces (so the first error is the one qpp would throw, with
// qpp's (where, what) strings), then runs the device op. Exceptions never
// cross the boundary: they become a qgpu_status plus a per-thread message.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "capi_common.hpp"
#include "internal.hpp"
#include "kernels.hpp"
#include "ops.hpp"
#include "traj.hpp"

using qgpu::cd;
using qgpu::Exc;
using qgpu::raise;

namespace qgpu {

// Plain character arrays: trivially destructible, so that a library call made
// while the thread is being torn down (a caller's thread_local holder
// destroying its context after this file's thread_locals are gone) still
// writes valid memory.
thread_local char t_where[256], t_what[1024];

static void copy_msg(char* dst, size_t cap, const std::string& src) {
    const size_t n = std::min(cap - 1, src.size());
    std::memcpy(dst, src.data(), n);
    dst[n] = '\0';
}

void record_error(qgpu_status, const std::string& where,
                  const std::string& what) {
    copy_msg(t_where, sizeof(t_where), where);
    copy_msg(t_what, sizeof(t_what), what);
}
void clear_error() {
    t_where[0] = '\0';
    t_what[0] = '\0';
}

void after_launch(qgpu_ctx* ctx, const char* name) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) raise(QGPU_ERR_CUDA, name, cudaGetErrorString(e));
    ctx->launches.fetch_add(1, std::memory_order_relaxed);
}

void ensure_smem(const void* func, size_t bytes) {
    if (bytes <= 48 * 1024) return; // the default limit
    int dev = 0;
    QG_CUDA(cudaGetDevice(&dev));
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> limit;
    std::lock_guard<std::mutex> lock(mu);
    size_t& have = limit[{func, dev}];
    if (bytes <= have) return;
    QG_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    have = bytes;
}

void* ctx_scratch(qgpu_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->scratch_bytes) return ctx->scratch;
    size_t nb = std::max<size_t>(bytes, 2 * ctx->scratch_bytes);
    nb = std::max<size_t>(nb, 1 << 20);
    if (ctx->scratch) {
        QG_CUDA(cudaStreamSynchronize(ctx->stream));
        QG_CUDA(cudaFree(ctx->scratch));
        ctx->scratch = nullptr;
        ctx->scratch_bytes = 0;
    }
    QG_CUDA(cudaMalloc(&ctx->scratch, nb));
    ctx->scratch_bytes = nb;
    return ctx->scratch;
}

cudaError_t ctx_malloc(qgpu_ctx* ctx, void** p, size_t bytes) {
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream);
    if (e == cudaSuccess) return e;
    cudaGetLastError();
    cudaStreamSynchronize(ctx->stream);
    cudaMemPoolTrimTo(ctx->pool, 0);
    e = cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream);
    if (e != cudaSuccess) cudaGetLastError();
    return e;
}

void destroy_ctx(qgpu_ctx* ctx) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->dev_flag) cudaFree(ctx->dev_flag);
    cudaStreamDestroy(ctx->stream);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
}

void* ctx_pinned(qgpu_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->pinned_bytes) return ctx->pinned;
    size_t nb = std::max<size_t>(bytes, 4096);
    if (ctx->pinned) {
        QG_CUDA(cudaStreamSynchronize(ctx->stream));
        QG_CUDA(cudaFreeHost(ctx->pinned));
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
    }
    QG_CUDA(cudaMallocHost(&ctx->pinned, nb));
    ctx->pinned_bytes = nb;
    return ctx->pinned;
}

} // namespace qgpu

namespace {

// ------------------------------------------------- qpp validation helpers
// (include/qpp/internal/util.hpp:123-287)
bool dims_ok(const std::vector<uint64_t>& dims) {
    if (dims.empty()) return false;
    return std::find(dims.begin(), dims.end(), uint64_t{0}) == dims.end();
}
uint64_t prod(const std::vector<uint64_t>& v) {
    uint64_t p = 1;
    for (uint64_t x : v) p *= x;
    return p;
}
bool subsys_ok(const std::vector<uint64_t>& s,
               const std::vector<uint64_t>& dims) {
    if (s.size() > dims.size()) return false;
    std::vector<uint64_t> t = s;
    std::sort(t.begin(), t.end());
    if (std::adjacent_find(t.begin(), t.end()) != t.end()) return false;
    for (uint64_t x : s)
        if (x + 1 > dims.size()) return false;
    return true;
}
bool perm_ok(const std::vector<uint64_t>& p) {
    if (p.empty()) return false;
    std::vector<uint64_t> t = p;
    std::sort(t.begin(), t.end());
    for (size_t i = 0; i < t.size(); ++i)
        if (t[i] != i) return false;
    return true;
}
std::vector<uint64_t> vec(const uint64_t* p, uint32_t n) {
    return (p && n) ? std::vector<uint64_t>(p, p + n) : std::vector<uint64_t>();
}
void state_shape(uint64_t rows, uint64_t cols, const std::vector<uint64_t>& dims,
                 const char* W, const char* wcv, const char* wm,
                 const char* wnsq) {
    if (cols == 1) {
        if (prod(dims) != rows) raise(QGPU_ERR_DIMS_MISMATCH_CVECTOR, W, wcv);
    } else if (rows == cols) {
        if (prod(dims) != cols) raise(QGPU_ERR_DIMS_MISMATCH_MATRIX, W, wm);
    } else {
        raise(QGPU_ERR_MATRIX_NOT_SQUARE_NOR_CVECTOR, W, wnsq);
    }
}

// qpp::apply(state, A, target, dims), operations.hpp:80-129
uint64_t check_apply(uint64_t rows, uint64_t cols, uint64_t ar, uint64_t ac,
                     const std::vector<uint64_t>& target,
                     const std::vector<uint64_t>& dims) {
    const char* W = "qpp::apply()";
    if (ar * ac == 0) raise(QGPU_ERR_ZERO_SIZE, W, "A");
    if (rows * cols == 0) raise(QGPU_ERR_ZERO_SIZE, W, "state");
    if (target.empty()) raise(QGPU_ERR_ZERO_SIZE, W, "target");
    if (ar != ac) raise(QGPU_ERR_MATRIX_NOT_SQUARE, W, "A");
    if (!dims_ok(dims)) raise(QGPU_ERR_DIMS_INVALID, W, "dims");
    if (!subsys_ok(target, dims))
        raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
    state_shape(rows, cols, dims, W, "dims/state", "dims/state", "state");
    uint64_t DA = 1;
    for (uint64_t t : target) DA *= dims[t];
    if (DA != ac) raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, "A/dims/target");
    return DA;
}

// qpp::applyCTRL / applyCTRL_fan, operations.hpp:625-751 and :970-1100;
// returns the inverted shift ((d - s) % d, operations.hpp:727-735).
std::vector<uint64_t> check_ctrl(uint64_t rows, uint64_t cols, uint64_t ar,
                                 uint64_t ac,
                                 const std::vector<uint64_t>& ctrl,
                                 const std::vector<uint64_t>& target,
                                 const std::vector<uint64_t>& dims,
                                 const uint64_t* shift_p, bool fan) {
    const char* W = fan ? "qpp::applyCTRL_fan()" : "qpp::applyCTRL()";
    if (ar * ac == 0) raise(QGPU_ERR_ZERO_SIZE, W, "A");
    if (rows * cols == 0) raise(QGPU_ERR_ZERO_SIZE, W, "state");
    if (ctrl.empty()) raise(QGPU_ERR_ZERO_SIZE, W, "ctrl");
    if (target.empty()) raise(QGPU_ERR_ZERO_SIZE, W, "target");
    if (ar != ac) raise(QGPU_ERR_MATRIX_NOT_SQUARE, W, "A");
    state_shape(rows, cols, dims, W, "dims/state", "dims/state", "state");
    if (!subsys_ok(ctrl, dims)) raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "ctrl/dims");
    uint64_t d = dims[ctrl[0]];
    for (size_t i = 1; i < ctrl.size(); ++i)
        if (dims[ctrl[i]] != d) raise(QGPU_ERR_DIMS_NOT_EQUAL, W, "ctrl");
    if (!dims_ok(dims)) raise(QGPU_ERR_DIMS_INVALID, W, "dims");
    if (!subsys_ok(target, dims))
        raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
    if (fan)
        for (size_t i = 1; i < target.size(); ++i)
            if (dims[target[i]] != d) raise(QGPU_ERR_DIMS_NOT_EQUAL, W, "target");
    for (uint64_t c : ctrl)
        for (uint64_t t : target)
            if (c == t) raise(QGPU_ERR_OUT_OF_RANGE, W, "ctrl/target");
    if (fan) {
        if (ar != d) raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, "A/target");
    } else {
        uint64_t DA = 1;
        for (uint64_t t : target) DA *= dims[t];
        if (DA != ac) raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, "A/target");
    }
    std::vector<uint64_t> cg = ctrl;
    cg.insert(cg.end(), target.begin(), target.end());
    std::sort(cg.begin(), cg.end());
    if (!subsys_ok(cg, dims))
        raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/ctrl/target");
    std::vector<uint64_t> sh(ctrl.size(), 0);
    if (shift_p) {
        for (size_t i = 0; i < ctrl.size(); ++i) {
            if (shift_p[i] >= d) raise(QGPU_ERR_OUT_OF_RANGE, W, "shift");
            sh[i] = (d - shift_p[i]) % d;
        }
    }
    return sh;
}

// qpp::apply(A, Ks, target, dims), operations.hpp:482-542
uint64_t check_kraus(uint64_t rows, uint64_t cols, uint32_t nK, uint64_t kr,
                     uint64_t kc, const std::vector<uint64_t>& target,
                     const std::vector<uint64_t>& dims) {
    const char* W = "qpp::apply()";
    if (rows * cols == 0) raise(QGPU_ERR_ZERO_SIZE, W, "A");
    if (target.empty()) raise(QGPU_ERR_ZERO_SIZE, W, "target");
    if (rows != cols) raise(QGPU_ERR_MATRIX_NOT_SQUARE, W, "A");
    if (!dims_ok(dims)) raise(QGPU_ERR_DIMS_INVALID, W, "dims");
    if (!subsys_ok(target, dims))
        raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
    state_shape(rows, cols, dims, W, "A/dims", "A/dims", "A");
    uint64_t DA = 1;
    for (uint64_t t : target) DA *= dims[t];
    if (nK == 0) raise(QGPU_ERR_ZERO_SIZE, W, "Ks");
    if (kr != kc) raise(QGPU_ERR_MATRIX_NOT_SQUARE, W, "Ks[0]");
    if (kc != DA) raise(QGPU_ERR_MATRIX_MISMATCH_SUBSYS, W, "dims/Ks[0]/target");
    return DA;
}

// ptrace / ptranspose share their checks (operations.hpp:1915-1937,
// :2174-2196)
void check_subsys_op(const char* W, uint64_t rows, uint64_t cols,
                     const std::vector<uint64_t>& target,
                     const std::vector<uint64_t>& dims) {
    if (rows * cols == 0) raise(QGPU_ERR_ZERO_SIZE, W, "A");
    if (!dims_ok(dims)) raise(QGPU_ERR_DIMS_INVALID, W, "dims");
    if (!subsys_ok(target, dims))
        raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
    state_shape(rows, cols, dims, W, "A/dims", "A/dims", "A");
}

// qpp::syspermute, operations.hpp:2393-2423
void check_perm(uint64_t rows, uint64_t cols, const std::vector<uint64_t>& perm,
                const std::vector<uint64_t>& dims) {
    const char* W = "qpp::syspermute()";
    if (rows * cols == 0) raise(QGPU_ERR_ZERO_SIZE, W, "A");
    if (!dims_ok(dims)) raise(QGPU_ERR_DIMS_INVALID, W, "dims");
    if (!perm_ok(perm)) raise(QGPU_ERR_PERM_INVALID, W, "perm");
    if (perm.size() != dims.size())
        raise(QGPU_ERR_PERM_MISMATCH_DIMS, W, "dims/perm");
    state_shape(rows, cols, dims, W, "A/dims", "A/dims", "A");
}

// qpp::applyQFT / applyTFQ (operations.hpp:2569-2605, :2684-2720) on A
// viewed as n = get_num_subsys(D, d) qudits of dimension d (util.hpp:389-397);
// `whole` = QFT / TFQ (:2793-2826, :2845-2878), which check no target and
// name qpp::QFT() in the dims checks of both.
void check_qft(const char* W, bool whole, uint64_t rows, uint64_t cols,
               const std::vector<uint64_t>& target, uint64_t d) {
    if (rows * cols == 0) raise(QGPU_ERR_ZERO_SIZE, W, "A");
    if (d < 2) raise(QGPU_ERR_DIMS_INVALID, W, "d");
    const uint64_t n = uint64_t(std::llround(std::log2(double(rows)) / std::log2(double(d))));
    std::vector<uint64_t> dims(n, d);
    if (!whole && !subsys_ok(target, dims))
        raise(QGPU_ERR_SUBSYS_MISMATCH_DIMS, W, "dims/target");
    // prod(dims) with overflow saturating to 0 (never equal to rows then)
    uint64_t p = 1;
    for (uint64_t i = 0; i < n && p; ++i) p = p > UINT64_MAX / d ? 0 : p * d;
    const char* Wd = whole ? "qpp::QFT()" : W;
    if (cols == 1) {
        if (dims.empty() || p != rows) raise(QGPU_ERR_DIMS_MISMATCH_CVECTOR, Wd, "A/dims");
    } else if (rows == cols) {
        if (dims.empty() || p != rows) raise(QGPU_ERR_DIMS_MISMATCH_MATRIX, Wd, "A/dims");
    } else {
        raise(QGPU_ERR_MATRIX_NOT_SQUARE_NOR_CVECTOR, Wd, "A");
    }
}

void shape_of(const qgpu_state* s, uint64_t& rows, uint64_t& cols) {
    rows = s->D;
    cols = s->kind == QGPU_KET ? 1 : s->D;
}

const cd* C(const double* p) { return reinterpret_cast<const cd*>(p); }

void upload_c128(qgpu_state* s, const double* host) {
    if (s->prec == QGPU_C128) {
        QG_CUDA(cudaMemcpyAsync(s->data, host, s->bytes(), cudaMemcpyHostToDevice,
                                s->ctx->stream));
    } else {
        void* tmp = nullptr;
        QG_CUDA(qgpu::ctx_malloc(s->ctx, &tmp, s->elems * 16));
        QG_CUDA(cudaMemcpyAsync(tmp, host, s->elems * 16, cudaMemcpyHostToDevice,
                                s->ctx->stream));
        qgpu::launch_convert(s->ctx, tmp, QGPU_C128, s->data, QGPU_C64, s->elems);
        QG_CUDA(cudaFreeAsync(tmp, s->ctx->stream));
    }
}

void download_c128(const qgpu_state* s, double* host) {
    if (s->prec == QGPU_C128) {
        QG_CUDA(cudaMemcpyAsync(host, s->data, s->bytes(), cudaMemcpyDeviceToHost,
                                s->ctx->stream));
    } else {
        void* tmp = nullptr;
        QG_CUDA(qgpu::ctx_malloc(s->ctx, &tmp, s->elems * 16));
        qgpu::launch_convert(s->ctx, s->data, QGPU_C64, tmp, QGPU_C128, s->elems);
        QG_CUDA(cudaMemcpyAsync(host, tmp, s->elems * 16, cudaMemcpyDeviceToHost,
                                s->ctx->stream));
        QG_CUDA(cudaFreeAsync(tmp, s->ctx->stream));
    }
    QG_CUDA(cudaStreamSynchronize(s->ctx->stream));
}

// RAII holder for temporary states of the value-semantics entry points.
struct Tmp {
    qgpu_state* s = nullptr;
    ~Tmp() { qgpu::free_state(s); }
};

qgpu_state* host_state(qgpu_ctx* ctx, const double* state, uint64_t rows,
                       uint64_t cols, const std::vector<uint64_t>& dims) {
    qgpu_state* s = qgpu::new_state(ctx, cols == 1 ? QGPU_KET : QGPU_RHO,
                                    QGPU_C128, dims, false);
    try {
        upload_c128(s, state);
    } catch (...) {
        qgpu::free_state(s);
        throw;
    }
    (void)rows;
    return s;
}

} // namespace

extern "C" {

const char* qgpu_last_error_where(void) { return qgpu::t_where; }
const char* qgpu_last_error_what(void) { return qgpu::t_what; }
const char* qgpu_version(void) { return "qpp_b200 0.1.0 (sm_100a)"; }

const char* qgpu_status_name(qgpu_status s) {
    switch (s) {
        case QGPU_OK: return "OK";
        case QGPU_ERR_ZERO_SIZE: return "ZeroSize";
        case QGPU_ERR_MATRIX_NOT_SQUARE: return "MatrixNotSquare";
        case QGPU_ERR_MATRIX_NOT_SQUARE_NOR_CVECTOR: return "MatrixNotSquareNorCvector";
        case QGPU_ERR_MATRIX_MISMATCH_SUBSYS: return "MatrixMismatchSubsys";
        case QGPU_ERR_DIMS_INVALID: return "DimsInvalid";
        case QGPU_ERR_DIMS_NOT_EQUAL: return "DimsNotEqual";
        case QGPU_ERR_DIMS_MISMATCH_MATRIX: return "DimsMismatchMatrix";
        case QGPU_ERR_DIMS_MISMATCH_CVECTOR: return "DimsMismatchCvector";
        case QGPU_ERR_SUBSYS_MISMATCH_DIMS: return "SubsysMismatchDims";
        case QGPU_ERR_PERM_INVALID: return "PermInvalid";
        case QGPU_ERR_PERM_MISMATCH_DIMS: return "PermMismatchDims";
        case QGPU_ERR_OUT_OF_RANGE: return "OutOfRange";
        case QGPU_ERR_TYPE_MISMATCH: return "TypeMismatch";
        case QGPU_ERR_SIZE_MISMATCH: return "SizeMismatch";
        case QGPU_ERR_QUDIT_ALREADY_MEASURED: return "QuditAlreadyMeasured";
        case QGPU_ERR_MATRIX_NOT_SQUARE_NOR_VECTOR: return "MatrixNotSquareNorVector";
        case QGPU_ERR_DIVISION_BY_ZERO: return "DivisionByZero";
        case QGPU_ERR_DUPLICATES: return "Duplicates";
        case QGPU_ERR_CUDA: return "CudaError";
        case QGPU_ERR_OUT_OF_MEMORY: return "OutOfMemory";
        case QGPU_ERR_TIMEOUT: return "Timeout";
        case QGPU_ERR_INVALID_HANDLE: return "InvalidHandle";
        case QGPU_ERR_NOT_SUPPORTED: return "NotSupported";
        case QGPU_ERR_INVALID_ARGUMENT: return "InvalidArgument";
    }
    return "Unknown";
}

// ------------------------------------------------------------- context
qgpu_status qgpu_ctx_create(int device, qgpu_ctx** out) {
    return qgpu::guarded(__func__, [&] {
        if (!out) raise(QGPU_ERR_INVALID_ARGUMENT, "qgpu_ctx_create()", "out");
        int n = 0;
        QG_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n)
            raise(QGPU_ERR_INVALID_ARGUMENT, "qgpu_ctx_create()", "device");
        QG_CUDA(cudaSetDevice(device));
        auto* c = new qgpu_ctx;
        c->device = device;
        cudaDeviceProp prop;
        QG_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major != 10) {
            delete c;
            raise(QGPU_ERR_NOT_SUPPORTED, "qgpu_ctx_create()",
                  "built for sm_100a (B200) only");
        }
        c->num_sms = prop.multiProcessorCount;
        // the allocation-free ptrace looks its table's address up again
        qgpu::noalloc_forget(device);
        QG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        cudaMemPoolProps pp;
        std::memset(&pp, 0, sizeof(pp));
        pp.allocType = cudaMemAllocationTypePinned;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = device;
        QG_CUDA(cudaMemPoolCreate(&c->pool, &pp));
        // keep up to a quarter of the device's memory reserved between uses
        uint64_t keep = uint64_t(prop.totalGlobalMem) / 4;
        QG_CUDA(cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep));
        *out = c;
    });
}

qgpu_status qgpu_ctx_destroy(qgpu_ctx* ctx) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        // states still alive keep the context (their memory lives on its
        // stream); the last qgpu_state_destroy tears it down
        ctx->closing.store(true);
        if (ctx->live_states.load() == 0) qgpu::destroy_ctx(ctx);
    });
}

qgpu_status qgpu_ctx_synchronize(qgpu_ctx* ctx) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        QG_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

qgpu_status qgpu_ctx_mem_info(qgpu_ctx* ctx, uint64_t* free_b, uint64_t* total_b) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        size_t f = 0, t = 0;
        QG_CUDA(cudaSetDevice(ctx->device));
        QG_CUDA(cudaMemGetInfo(&f, &t));
        // the pool's idle reserve is free for this context's allocations
        uint64_t reserved = 0, used = 0;
        QG_CUDA(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
        QG_CUDA(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &used));
        if (reserved > used) f += size_t(reserved - used);
        if (free_b) *free_b = f;
        if (total_b) *total_b = t;
    });
}

uint64_t qgpu_ctx_launch_count(const qgpu_ctx* ctx) {
    return ctx ? ctx->launches.load() : 0;
}

void* qgpu_ctx_stream(qgpu_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

qgpu_status qgpu_ctx_set_wait_test(qgpu_ctx* ctx, uint32_t spin_limit, int stall_next) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        std::lock_guard<std::mutex> lock(ctx->mu);
        ctx->wait_limit = spin_limit;
        ctx->stall_next = stall_next != 0;
        // allocated here, outside any stream capture, for the pass that reports
        qgpu::ctx_error_flag(ctx);
    });
}

qgpu_status qgpu_ctx_set_tile_bits(qgpu_ctx* ctx, int bits) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        if (bits != 0 && (bits < 5 || bits > 14))
            raise(QGPU_ERR_OUT_OF_RANGE, "qgpu_ctx_set_tile_bits()", "bits");
        ctx->tile_bits = bits;
    });
}

// --------------------------------------------------------------- states
qgpu_status qgpu_state_create(qgpu_ctx* ctx, qgpu_kind kind, qgpu_prec prec,
                              const uint64_t* dims, uint32_t n, qgpu_state** out) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        if (!out) raise(QGPU_ERR_INVALID_ARGUMENT, "qgpu_state_create()", "out");
        std::vector<uint64_t> d = vec(dims, n);
        if (!dims_ok(d)) raise(QGPU_ERR_DIMS_INVALID, "qgpu_state_create()", "dims");
        if (kind != QGPU_KET && kind != QGPU_RHO)
            raise(QGPU_ERR_INVALID_ARGUMENT, "qgpu_state_create()", "kind");
        if (prec != QGPU_C128 && prec != QGPU_C64)
            raise(QGPU_ERR_INVALID_ARGUMENT, "qgpu_state_create()", "prec");
        *out = qgpu::new_state(ctx, kind, prec, d, true);
    });
}

qgpu_status qgpu_state_destroy(qgpu_state* s) {
    return qgpu::guarded(__func__, [&] {
        if (s) qgpu::free_state(s);
    });
}

qgpu_status qgpu_state_clone(const qgpu_state* s, qgpu_state** out) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        qgpu_state* c = qgpu::new_state(s->ctx, s->kind, s->prec, s->dims, false);
        cudaError_t e = cudaMemcpyAsync(c->data, s->data, s->bytes(),
                                        cudaMemcpyDeviceToDevice, s->ctx->stream);
        if (e != cudaSuccess) {
            qgpu::free_state(c);
            raise(QGPU_ERR_CUDA, "qgpu_state_clone()", cudaGetErrorString(e));
        }
        *out = c;
    });
}

qgpu_status qgpu_state_upload(qgpu_state* s, const void* host) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        QG_CUDA(cudaMemcpyAsync(s->data, host, s->bytes(), cudaMemcpyHostToDevice,
                                s->ctx->stream));
        QG_CUDA(cudaStreamSynchronize(s->ctx->stream));
    });
}

qgpu_status qgpu_state_download(const qgpu_state* s, void* host) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        QG_CUDA(cudaMemcpyAsync(host, s->data, s->bytes(), cudaMemcpyDeviceToHost,
                                s->ctx->stream));
        QG_CUDA(cudaStreamSynchronize(s->ctx->stream));
    });
}

qgpu_status qgpu_state_upload_c128(qgpu_state* s, const double* host) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        upload_c128(s, host);
        QG_CUDA(cudaStreamSynchronize(s->ctx->stream));
    });
}

qgpu_status qgpu_state_download_c128(const qgpu_state* s, double* host) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        download_c128(s, host);
    });
}

qgpu_status qgpu_state_info(const qgpu_state* s, qgpu_kind* kind, qgpu_prec* prec,
                            uint32_t* n, uint64_t* dims, uint64_t* D) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        if (kind) *kind = s->kind;
        if (prec) *prec = s->prec;
        if (n) *n = uint32_t(s->dims.size());
        if (dims) std::copy(s->dims.begin(), s->dims.end(), dims);
        if (D) *D = s->D;
    });
}

void* qgpu_state_device_ptr(qgpu_state* s) { return s ? s->data : nullptr; }

qgpu_status qgpu_state_fill_gaussian(qgpu_state* s, uint64_t seed) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        qgpu::launch_fill_gaussian(s->ctx, s->prec, s->data, s->elems, seed);
        if (!qgpu::op_normalize(s))
            raise(QGPU_ERR_DIVISION_BY_ZERO, "qpp::normalize()", "Division by zero!");
    });
}

qgpu_status qgpu_state_convert(const qgpu_state* src, qgpu_state* dst) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(src);
        qgpu::need_handle(dst);
        if (src->kind != dst->kind || src->dims != dst->dims)
            raise(QGPU_ERR_DIMS_NOT_EQUAL, "qgpu_state_convert()", "src/dst");
        qgpu::launch_convert(src->ctx, src->data, src->prec, dst->data, dst->prec,
                             src->elems);
    });
}

// ------------------------------------------------------ resident ops
qgpu_status qgpu_apply(qgpu_state* s, const double* A, uint64_t DA,
                       const uint64_t* target, uint32_t k) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        uint64_t r, c;
        shape_of(s, r, c);
        std::vector<uint64_t> t = vec(target, k);
        check_apply(r, c, DA, DA, t, s->dims);
        qgpu::op_apply(s, C(A), DA, t);
    });
}

qgpu_status qgpu_apply_ctrl(qgpu_state* s, const double* A, uint64_t DA,
                            const uint64_t* ctrl, uint32_t nc,
                            const uint64_t* target, uint32_t k,
                            const uint64_t* shift) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        uint64_t r, c;
        shape_of(s, r, c);
        std::vector<uint64_t> cv = vec(ctrl, nc), t = vec(target, k);
        auto sh = check_ctrl(r, c, DA, DA, cv, t, s->dims, shift, false);
        qgpu::op_apply_ctrl(s, C(A), DA, cv, t, sh, false);
    });
}

qgpu_status qgpu_apply_ctrl_fan(qgpu_state* s, const double* A, uint64_t DA,
                                const uint64_t* ctrl, uint32_t nc,
                                const uint64_t* target, uint32_t k,
                                const uint64_t* shift) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        uint64_t r, c;
        shape_of(s, r, c);
        std::vector<uint64_t> cv = vec(ctrl, nc), t = vec(target, k);
        auto sh = check_ctrl(r, c, DA, DA, cv, t, s->dims, shift, true);
        qgpu::op_apply_ctrl(s, C(A), DA, cv, t, sh, true);
    });
}

qgpu_status qgpu_apply_kraus(qgpu_state* s, const double* Ks, uint32_t nK,
                             uint64_t DA, const uint64_t* target, uint32_t k) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        uint64_t r, c;
        shape_of(s, r, c);
        std::vector<uint64_t> t = vec(target, k);
        check_kraus(r, c, nK, DA, DA, t, s->dims);
        qgpu::op_apply_kraus(s, C(Ks), nK, DA, t);
    });
}

qgpu_status qgpu_ptrace(const qgpu_state* s, const uint64_t* target, uint32_t k,
                        qgpu_state** out) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        uint64_t r, c;
        shape_of(s, r, c);
        std::vector<uint64_t> t = vec(target, k);
        check_subsys_op("qpp::ptrace()", r, c, t, s->dims);
        *out = qgpu::op_ptrace(s, t);
    });
}

qgpu_status qgpu_ptranspose(const qgpu_state* s, const uint64_t* target,
                            uint32_t k, qgpu_state** out) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        uint64_t r, c;
        shape_of(s, r, c);
        std::vector<uint64_t> t = vec(target, k);
        check_subsys_op("qpp::ptranspose()", r, c, t, s->dims);
        *out = qgpu::op_ptranspose(s, t);
    });
}

qgpu_status qgpu_syspermute(const qgpu_state* s, const uint64_t* perm,
                            uint32_t n, qgpu_state** out) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        uint64_t r, c;
        shape_of(s, r, c);
        std::vector<uint64_t> p = vec(perm, n);
        check_perm(r, c, p, s->dims);
        *out = qgpu::op_syspermute(s, p);
    });
}

qgpu_status qgpu_norm2(const qgpu_state* s, double* out) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        *out = qgpu::op_norm2(s);
    });
}

qgpu_status qgpu_trace(const qgpu_state* s, double* re, double* im) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        cd t = qgpu::op_trace(s);
        if (re) *re = t.real();
        if (im) *im = t.imag();
    });
}

qgpu_status qgpu_normalize(qgpu_state* s) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        if (!qgpu::op_normalize(s))
            raise(QGPU_ERR_DIVISION_BY_ZERO, "qpp::normalize()", "Division by zero!");
    });
}

qgpu_status qgpu_inner(const qgpu_state* a, const qgpu_state* b, double* re,
                       double* im) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(a);
        qgpu::need_handle(b);
        if (a->kind != b->kind || a->dims != b->dims || a->prec != b->prec)
            raise(QGPU_ERR_DIMS_NOT_EQUAL, "qgpu_inner()", "a/b");
        cd v = qgpu::reduce_inner(a->ctx, a->prec, a->data, b->data, a->elems);
        if (re) *re = v.real();
        if (im) *im = v.imag();
    });
}

// ------------------------------------------- value-semantics entry points
qgpu_status qgpu_host_apply(qgpu_ctx* ctx, const double* state, uint64_t rows,
                            uint64_t cols, const double* A, uint64_t ar,
                            uint64_t ac, const uint64_t* target, uint32_t k,
                            const uint64_t* dims, uint32_t n, double* result) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        std::vector<uint64_t> t = vec(target, k), d = vec(dims, n);
        uint64_t DA = check_apply(rows, cols, ar, ac, t, d);
        Tmp s;
        s.s = host_state(ctx, state, rows, cols, d);
        qgpu::op_apply(s.s, C(A), DA, t);
        download_c128(s.s, result);
    });
}

qgpu_status qgpu_host_apply_ctrl(qgpu_ctx* ctx, const double* state,
                                 uint64_t rows, uint64_t cols, const double* A,
                                 uint64_t ar, uint64_t ac, const uint64_t* ctrl,
                                 uint32_t nc, const uint64_t* target, uint32_t k,
                                 const uint64_t* dims, uint32_t n,
                                 const uint64_t* shift, int fan, double* result) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        std::vector<uint64_t> cv = vec(ctrl, nc), t = vec(target, k), d = vec(dims, n);
        auto sh = check_ctrl(rows, cols, ar, ac, cv, t, d, shift, fan != 0);
        Tmp s;
        s.s = host_state(ctx, state, rows, cols, d);
        qgpu::op_apply_ctrl(s.s, C(A), ar, cv, t, sh, fan != 0);
        download_c128(s.s, result);
    });
}

qgpu_status qgpu_host_apply_kraus(qgpu_ctx* ctx, const double* state,
                                  uint64_t rows, uint64_t cols, const double* Ks,
                                  uint32_t nK, uint64_t kr, uint64_t kc,
                                  const uint64_t* target, uint32_t k,
                                  const uint64_t* dims, uint32_t n,
                                  double* result) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        std::vector<uint64_t> t = vec(target, k), d = vec(dims, n);
        uint64_t DA = check_kraus(rows, cols, nK, kr, kc, t, d);
        Tmp s;
        s.s = host_state(ctx, state, rows, cols, d);
        qgpu::op_apply_kraus(s.s, C(Ks), nK, DA, t);
        download_c128(s.s, result);
    });
}

qgpu_status qgpu_host_ptrace(qgpu_ctx* ctx, const double* state, uint64_t rows,
                             uint64_t cols, const uint64_t* target, uint32_t k,
                             const uint64_t* dims, uint32_t n, double* result) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        std::vector<uint64_t> t = vec(target, k), d = vec(dims, n);
        check_subsys_op("qpp::ptrace()", rows, cols, t, d);
        Tmp s, o;
        s.s = host_state(ctx, state, rows, cols, d);
        o.s = qgpu::op_ptrace(s.s, t);
        download_c128(o.s, result);
    });
}

qgpu_status qgpu_host_ptranspose(qgpu_ctx* ctx, const double* state,
                                 uint64_t rows, uint64_t cols,
                                 const uint64_t* target, uint32_t k,
                                 const uint64_t* dims, uint32_t n,
                                 double* result) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        std::vector<uint64_t> t = vec(target, k), d = vec(dims, n);
        check_subsys_op("qpp::ptranspose()", rows, cols, t, d);
        Tmp s, o;
        s.s = host_state(ctx, state, rows, cols, d);
        o.s = qgpu::op_ptranspose(s.s, t);
        download_c128(o.s, result);
    });
}

qgpu_status qgpu_host_syspermute(qgpu_ctx* ctx, const double* state,
                                 uint64_t rows, uint64_t cols,
                                 const uint64_t* perm, uint32_t np,
                                 const uint64_t* dims, uint32_t n,
                                 double* result) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        std::vector<uint64_t> p = vec(perm, np), d = vec(dims, n);
        check_perm(rows, cols, p, d);
        Tmp s, o;
        s.s = host_state(ctx, state, rows, cols, d);
        o.s = qgpu::op_syspermute(s.s, p);
        download_c128(o.s, result);
    });
}

// ------------------------------------------------------- Fourier transforms
qgpu_status qgpu_apply_qft(qgpu_state* s, const uint64_t* target, uint32_t k, uint64_t d,
                           int swap, int inverse) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        uint64_t r, c;
        shape_of(s, r, c);
        std::vector<uint64_t> t = vec(target, k);
        check_qft(inverse ? "qpp::applyTFQ()" : "qpp::applyQFT()", false, r, c, t, d);
        qgpu::op_apply_qft(s, t, d, swap != 0, inverse != 0);
    });
}

qgpu_status qgpu_qft(qgpu_state* s, uint64_t d, int swap, int inverse) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(s);
        uint64_t r, c;
        shape_of(s, r, c);
        check_qft(inverse ? "qpp::TFQ()" : "qpp::QFT()", true, r, c, {}, d);
        std::vector<uint64_t> t;
        for (uint64_t x = 1; x < r; x *= d) t.push_back(t.size());
        qgpu::op_apply_qft(s, t, d, swap != 0, inverse != 0);
    });
}

static qgpu_status host_qft(qgpu_ctx* ctx, const double* state, uint64_t rows,
                            uint64_t cols, const uint64_t* target, uint32_t k, bool whole,
                            uint64_t d, int swap, int inverse, double* result) {
    return qgpu::guarded(__func__, [&] {
        qgpu::need_handle(ctx);
        std::vector<uint64_t> t = vec(target, k);
        const char* W = whole ? (inverse ? "qpp::TFQ()" : "qpp::QFT()")
                              : (inverse ? "qpp::applyTFQ()" : "qpp::applyQFT()");
        check_qft(W, whole, rows, cols, t, d);
        std::vector<uint64_t> dims;
        for (uint64_t x = 1; x < rows; x *= d) dims.push_back(d);
        if (whole)
            for (size_t i = 0; i < dims.size(); ++i) t.push_back(i);
        Tmp s;
        s.s = host_state(ctx, state, rows, cols, dims);
        qgpu::op_apply_qft(s.s, t, d, swap != 0, inverse != 0);
        download_c128(s.s, result);
    });
}

qgpu_status qgpu_host_apply_qft(qgpu_ctx* ctx, const double* state, uint64_t rows,
                                uint64_t cols, const uint64_t* target, uint32_t k,
                                uint64_t d, int swap, int inverse, double* result) {
    return host_qft(ctx, state, rows, cols, target, k, false, d, swap, inverse, result);
}

qgpu_status qgpu_host_qft(qgpu_ctx* ctx, const double* state, uint64_t rows, uint64_t cols,
                          uint64_t d, int swap, int inverse, double* result) {
    return host_qft(ctx, state, rows, cols, nullptr, 0, true, d, swap, inverse, result);
}

} // extern "C"
