// internal.hpp -- host-side structures of libqpp_b200 (context, state,
// errors). Pure C++17 + CUDA runtime API; no torch and no Eigen.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/qpp_b200.h"

struct qgpu_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    std::atomic<uint64_t> launches{0};
    std::mutex mu;
    // Device scratch owned by the context (FP64 block partials, large gate
    // matrices, offset tables). Grown on demand; used in stream order only.
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    // Pinned host buffer for small device -> host results.
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    // Device words: [0] where kernels with bounded waits record a timeout,
    // [8] the squared norm read by the fused tensor-core passes.
    int* dev_flag = nullptr;
    // Bounded-wait test hooks (qgpu_ctx_set_wait_test): the iteration limit
    // of the fused kernel's waits (0 = the default), and a one-shot request
    // that the next fused launch waits first on a barrier nothing completes.
    uint32_t wait_limit = 0;
    int stall_next = 0;
    // Largest tile (state bits) of the plain form's tile passes; 0 = the
    // default (qgpu_ctx_set_tile_bits).
    int tile_bits = 0;
    // Stream-ordered pool of every device buffer the context allocates
    // (states, transform buffers, batch arenas): freed blocks stay reserved
    // up to a threshold, so repeated large allocations skip the driver's
    // mapping work.
    cudaMemPool_t pool = nullptr;
    // States created on this context that are still alive; a destroyed
    // context is torn down only when the last of them is freed.
    std::atomic<int64_t> live_states{0};
    std::atomic<bool> closing{false};
    // phases of the last qgpu_run_batch (milliseconds): programs compiled and
    // tiled on the host, buffers uploaded and the graph captured and
    // instantiated, the graph's device time, the plain-form instances, the
    // argument checks, the teardown after the graph
    double batch_ms[6] = {0, 0, 0, 0, 0, 0};
};

struct qgpu_state {
    qgpu_ctx* ctx = nullptr;
    qgpu_kind kind = QGPU_KET;
    qgpu_prec prec = QGPU_C128;
    std::vector<uint64_t> dims;
    uint64_t D = 0;     // prod(dims)
    uint64_t elems = 0; // D (ket) or D * D (rho)
    void* data = nullptr;
    size_t elem_bytes() const { return prec == QGPU_C128 ? 16 : 8; }
    size_t bytes() const { return elems * elem_bytes(); }
};

namespace qgpu {

// Internal exception; converted to a qgpu_status at the C boundary.
struct Exc {
    qgpu_status code;
    std::string where;
    std::string what;
};

[[noreturn]] inline void raise(qgpu_status c, const std::string& where,
                               const std::string& what) {
    throw Exc{c, where, what};
}

void record_error(qgpu_status c, const std::string& where,
                  const std::string& what);
void clear_error();

#define QG_CUDA(call)                                                       \
    do {                                                                    \
        cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess)                                              \
            ::qgpu::raise(e_ == cudaErrorMemoryAllocation                   \
                              ? QGPU_ERR_OUT_OF_MEMORY                      \
                              : QGPU_ERR_CUDA,                              \
                          #call, cudaGetErrorString(e_));                   \
    } while (0)

// Checks the last launch on this thread and counts it on the context.
void after_launch(qgpu_ctx* ctx, const char* name);

// Raises kernel `func`'s dynamic shared-memory limit on the current device to
// at least `bytes`. The limit is an attribute of each (function, device) and
// is only ever raised, so a launch with a smaller need on another thread
// stays valid.
void ensure_smem(const void* func, size_t bytes);

// Frees the context's stream, buffers and the context itself.
void destroy_ctx(qgpu_ctx* ctx);

// Stream-ordered allocation from the context pool on the context stream; on
// failure the pool's idle reserve is released and the allocation retried.
cudaError_t ctx_malloc(qgpu_ctx* ctx, void** p, size_t bytes);

// Context scratch of at least `bytes` (stream-ordered reuse).
void* ctx_scratch(qgpu_ctx* ctx, size_t bytes);
// Pinned host buffer of at least `bytes`.
void* ctx_pinned(qgpu_ctx* ctx, size_t bytes);

} // namespace qgpu
