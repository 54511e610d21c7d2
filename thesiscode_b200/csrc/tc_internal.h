// Internal helpers shared by the CUDA translation units of libthesiscode_b200.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include "thesiscode_b200.h"

// A named NVTX range over a scope, for tracing tools (Nsight Systems, ncu --nvtx): the RK4
// stages, the step loops, the graph replays, the adjoint and the batch calls each open one.
// Without a tool attached each push/pop is a call that returns at once.
struct TcNvtxRange {
  explicit TcNvtxRange(const char* name) { nvtxRangePushA(name); }
  ~TcNvtxRange() { nvtxRangePop(); }
  TcNvtxRange(const TcNvtxRange&) = delete;
  TcNvtxRange& operator=(const TcNvtxRange&) = delete;
};

// Make `device` current, failing with TC_ERR_ARG for an index that does not
// exist and TC_ERR_CUDA when the runtime cannot be reached.
static inline int tc_set_device_checked(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return TC_ERR_CUDA;
  if (device < 0 || device >= n) return TC_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return TC_ERR_CUDA;
  return TC_OK;
}

#define TC_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t tc_err_ = (expr);                           \
    if (tc_err_ != cudaSuccess) {                           \
      tc_record_cuda_error(tc_err_, #expr, __FILE__, __LINE__); \
      return TC_ERR_CUDA;                                   \
    }                                                       \
  } while (0)

void tc_record_cuda_error(cudaError_t err, const char* what, const char* file, int line);
void tc_record_error(const char* fmt, ...);
