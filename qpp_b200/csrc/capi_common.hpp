// capi_common.hpp -- helpers shared by the extern "C" translation units.
#pragma once

#include <new>
#include <stdexcept>
#include <vector>

#include "internal.hpp"

namespace qgpu {

inline std::vector<uint64_t> vec_of(const uint64_t* p, uint32_t n) {
    return (p && n) ? std::vector<uint64_t>(p, p + n) : std::vector<uint64_t>();
}

inline void need_handle(const void* p) {
    if (!p) raise(QGPU_ERR_INVALID_HANDLE, "qgpu", "null handle");
}

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

} // namespace qgpu
