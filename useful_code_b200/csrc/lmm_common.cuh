// lmm_common.cuh — shared definitions for the B200 LMM Monte Carlo kernels.
//
// Status handling: every C-ABI entry point returns an int status (LMM_OK on
// success) and records a human-readable message retrievable through
// lmm_last_error_string().  No entry point calls exit() or throws across the
// C boundary.  Kernel launches are checked with cudaGetLastError() only; the
// caller owns synchronisation (all entry points are asynchronous on the
// stream they are given).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <string>

#include "../../include/lmm_c.h"

namespace lmm {

// Capacity limits for the small per-call tables that travel as kernel
// parameters (no device allocation is needed for them).
constexpr int kMaxRates = LMM_MAX_RATES;      // forwards per curve
constexpr int kMaxSteps = LMM_MAX_STEPS;      // evolution steps
constexpr int kMaxFactors = LMM_MAX_FACTORS;  // Brownian factors
constexpr int kMaxBasis = LMM_MAX_BASIS;      // LS basis functions
constexpr int kMaxVars = 3;                   // LS basis variables per date

void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

// Records a CUDA error (if any) from the last launch and maps it to a status.
int check_launch(const char* what);
int check_cuda(cudaError_t e, const char* what);

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// Number of SMs of the current device (cached per device).
int sm_count();

// Grid size for a grid-stride kernel: enough CTAs to fill every SM `per_sm`
// times, but never more than the work needs.
inline int grid_for(long long work_items, int block, int per_sm = 8) {
  long long need = (work_items + block - 1) / block;
  long long cap = (long long)sm_count() * per_sm;
  if (need < 1) need = 1;
  return (int)(need < cap ? need : cap);
}

}  // namespace lmm

#define LMM_REQUIRE(cond, ...)                        \
  do {                                                \
    if (!(cond)) return ::lmm::fail(LMM_EINVAL, __VA_ARGS__); \
  } while (0)
