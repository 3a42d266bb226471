// capi_common.hpp -- helpers shared by the extern "C" translation units.
#pragma once

#include <nvtx3/nvToolsExt.h>

#include <new>
#include <stdexcept>
#include <utility>
#include <vector>

#include "internal.hpp"

namespace qgpu {

inline std::vector<uint64_t> vec_of(const uint64_t* p, uint32_t n) {
    return (p && n) ? std::vector<uint64_t>(p, p + n) : std::vector<uint64_t>();
}

inline void need_handle(const void* p) {
    if (!p) raise(QGPU_ERR_INVALID_HANDLE, "qgpu", "null handle");
}

// An NVTX range for the extent of a scope: entry points show up by name in
// Nsight tools and can be selected with ncu's --nvtx-include; without an
// attached tool a push and a pop cost a function-pointer test each.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Runs f, converting every exception into a status plus the per-thread
// (where, what) message; nothing throws across the C boundary.
template <typename F>
qgpu_status guarded(F&& f) {
    try {
        clear_error();
        f();
        return QGPU_OK;
    } catch (const Exc& e) {
        record_error(e.code, e.where, e.what);
        return e.code;
    } catch (const std::bad_alloc&) {
        record_error(QGPU_ERR_OUT_OF_MEMORY, "qgpu", "host allocation failed");
        return QGPU_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        record_error(QGPU_ERR_INVALID_ARGUMENT, "qgpu", e.what());
        return QGPU_ERR_INVALID_ARGUMENT;
    }
}

// guarded(f) inside an NVTX range named `name` (the entry point).
template <typename F>
qgpu_status guarded(const char* name, F&& f) {
    NvtxRange range(name);
    return guarded(std::forward<F>(f));
}

} // namespace qgpu
