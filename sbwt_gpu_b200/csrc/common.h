// common.h -- host-side error reporting shared by every translation unit.
//
// The reference reports errors as an int return code of 1 plus a message on
// stderr (include/gpu/cuda.hpp:7-13,67-84).  Here every C-ABI entry point
// returns non-zero and leaves the message in a thread-local buffer that
// sbwt_last_error() returns; nothing is printed by the library.
#pragma once
#include <cstdarg>
#include <cstdint>

namespace sbwt {

// Formats the message into the thread-local error buffer; returns 1 so that
// `return set_error(...)` reads like the reference's `return 1`.
int set_error(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
void clear_error();
const char *last_error();

}  // namespace sbwt

#define SBWT_CHECK_CUDA(expr)                                                                         \
    do {                                                                                              \
        cudaError_t e_ = (expr);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return ::sbwt::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, \
                                     __LINE__);                                                       \
    } while (0)

#define SBWT_TRY(expr)             \
    do {                           \
        int r_ = (expr);           \
        if (r_ != 0) return r_;    \
    } while (0)
