// common.cu — status/error plumbing shared by every C-ABI entry point.
#include "lmm_common.cuh"

#include <atomic>
#include <cstdarg>
#include <cstdio>

#include "../../include/lmm_pipeline.h"

namespace lmm {

namespace {
thread_local char g_last_error[1024] = "no error";
}

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return LMM_OK;
  return fail(LMM_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

namespace {
std::atomic<long> g_launches{0};
}

int check_launch(const char* what) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return check_cuda(cudaGetLastError(), what);
}

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cached[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
            cudaSuccess ||
        n <= 0)
      n = 148;
    cached[dev] = n;
  }
  return cached[dev];
}

}  // namespace lmm

extern "C" const char* lmm_last_error_string(void) { return lmm::g_last_error; }

extern "C" int lmm_version(void) { return 1; }

extern "C" long lmm_launch_count(void) {
  return lmm::g_launches.load(std::memory_order_relaxed);
}
