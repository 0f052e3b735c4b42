// psx_common.cuh -- status handling and launch helpers shared by the
// translation units of libpeasoup_b200.
#pragma once
#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <string>
#include "peasoup_b200.h"

namespace psx {

// 148 SMs on a B200; the actual count is read once per device.
int sm_count();

// Thread-local last-error message (psx_last_error).
void set_error(const char* fmt, ...);
void clear_error();

inline cudaStream_t cs(psx_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// Returns PSX_OK, or PSX_ERR_CUDA with the message recorded.
inline int cuda_status(cudaError_t e, const char* where)
{
    if (e == cudaSuccess) return PSX_OK;
    set_error("%s: %s", where, cudaGetErrorString(e));
    return PSX_ERR_CUDA;
}

// After a launch: report launch-configuration errors without synchronising.
inline int launch_status(const char* where)
{
    return cuda_status(cudaGetLastError(), where);
}

// Grid size for a grid-stride kernel over `work` items with `threads`
// per block: enough blocks to fill every SM `per_sm` times, never more
// than the work needs.
inline unsigned grid_for(size_t work, unsigned threads, unsigned per_sm = 8)
{
    size_t need = (work + threads - 1) / threads;
    size_t cap = (size_t)sm_count() * per_sm;
    if (need < 1) need = 1;
    return (unsigned)(need < cap ? need : cap);
}

}  // namespace psx

#define PSX_TRY(expr)                   \
    do {                                \
        int _rc = (expr);               \
        if (_rc != PSX_OK) return _rc;  \
    } while (0)

#define PSX_CUDA(expr) PSX_TRY(psx::cuda_status((expr), #expr))
