// bridge_plan.h — Brownian-bridge tables passed by value to the kernels.
#pragma once
#include "lmm_common.cuh"

namespace lmm {

struct BridgePlan {
  int steps, factors;
  float lw[kMaxSteps], rw[kMaxSteps], sd[kMaxSteps];
  int left[kMaxSteps], right[kMaxSteps], bidx[kMaxSteps];
  int alloc[kMaxFactors * kMaxSteps];  // [factor][bridge stage] -> Sobol dim
};

int make_bridge_plan(int steps, int factors, const int* h_alloc,
                     BridgePlan* plan);
void bridge_diagonal(int factors, int steps, int* idx);

}  // namespace lmm
