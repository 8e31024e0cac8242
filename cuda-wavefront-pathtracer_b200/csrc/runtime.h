// runtime.h - error reporting shared by the C entry points.
#pragma once
#include "cwp_b200.h"
#include <cuda_runtime.h>

namespace cwpb {
// records a message for cwp_last_error() on this thread and returns code
int set_error(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void clear_error();
}  // namespace cwpb

#define CWPB_CUDA(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return ::cwpb::set_error(e_ == cudaErrorMemoryAllocation ? CWP_ERR_NOMEM : CWP_ERR_CUDA, "%s (%s:%d)", cudaGetErrorString(e_), __FILE__, __LINE__); } while (0)
#define CWPB_CHECK(cond, code, ...) do { if (!(cond)) return ::cwpb::set_error(code, __VA_ARGS__); } while (0)
