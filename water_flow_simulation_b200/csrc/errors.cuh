// errors.cuh -- the library's per-thread error message (lbm_last_error) shared by its
// translation units.
#pragma once
#include <cstdarg>
#include <cstdio>

namespace wfs {
extern thread_local char g_err[512];

inline int fail(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

inline int check_launch(const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(-2, "%s: %s", what, cudaGetErrorString(e));
    return 0;
}
}  // namespace wfs
