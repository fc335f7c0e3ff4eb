// Thread-local error reporting behind csg_last_error().
#pragma once

#include <cstdarg>
#include <string>

namespace csg {
extern thread_local std::string g_last_error;
// Records a printf-style message and returns `code`.
int fail(int code, const char* fmt, ...);
// Counts one kernel launch (read with csg_kernel_launches()).  Launch sites
// are written `(csg::note_launch(), kernel<<<...>>>(...))`.
void note_launch();
}  // namespace csg

#define CSG_CUDA_CHECK(expr)                                                                                   \
    do {                                                                                                       \
        cudaError_t csg_err_ = (expr);                                                                         \
        if (csg_err_ != cudaSuccess)                                                                           \
            return csg::fail(CSG_ERR_CUDA, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(csg_err_), __FILE__, \
                             __LINE__);                                                                        \
    } while (0)
