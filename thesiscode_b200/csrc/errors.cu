// Status reporting for the C ABI: every entry point returns a status code and
// leaves a human-readable message in a thread-local buffer. The reference
// prints and returns (PanelVelocityParallel.f90:1300-1315) or ignores MPI
// error codes; here nothing prints and nothing aborts.
#include <cstdarg>
#include <cstdio>
#include "tc_internal.h"

namespace {
thread_local char g_last_error[512] = "";
}

void tc_record_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

void tc_record_cuda_error(cudaError_t err, const char* what, const char* file, int line) {
  tc_record_error("CUDA error %d (%s) in %s at %s:%d", (int)err, cudaGetErrorString(err), what,
                  file, line);
}

extern "C" const char* tc_last_error(void) { return g_last_error; }

extern "C" const char* tc_version(void) { return "thesiscode_b200 0.1.0 (sm_100a)"; }
