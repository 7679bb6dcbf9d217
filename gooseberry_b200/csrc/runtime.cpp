// runtime.cpp -- error state and device queries of libgooseberry_b200.
#include <cstdarg>
#include <cstdio>
#include <string>

#include "gb_internal.h"

namespace gb {

namespace {
thread_local std::string g_last_error;
}

void set_error(const char * fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

void clear_error() { g_last_error.clear(); }

int sm_count_of_current_device(int * out) {
  int dev = 0;
  GB_CUDA_TRY(cudaGetDevice(&dev));
  GB_CUDA_TRY(cudaDeviceGetAttribute(out, cudaDevAttrMultiProcessorCount, dev));
  return GOOSEBERRY_SUCCESS;
}

}  // namespace gb

extern "C" const char * gb_last_error(void) { return gb::g_last_error.c_str(); }
