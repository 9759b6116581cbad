// bridge.cu — Brownian bridge over unit time steps with any number of
// steps (Jäckel's construction as used by the reference "newBridge"),
// followed by successive differencing into N(0,1) increments.
//
// Reference behaviour followed:
//   table construction   brownian_bridge.cu:355-362 (t_i = i+1),
//                        brownian_bridge.cu:639-697 (initialize)
//   per-path transform   brownian_bridge.cu:401-455 (transformCPU),
//                        kernel brownian_bridge.cu:121-238
//   Sobol dimension allocation  gold/Bridge_allocator_gold.cpp:38-76
//                               (bridge_allocate_diagonal)
// Input normals are [factors*steps][paths]; output increments are
// [steps][factors][paths].
#include "lmm_common.cuh"
#include "lmm_device.cuh"
#include "bridge_plan.h"

#include <cmath>
#include <vector>

using namespace lmm;

namespace lmm {

// Diagonal allocation: walk the (factor, bridge-order) grid along
// anti-diagonals so that the leading Sobol dimensions go to the first
// bridge variates of the leading factors.
void bridge_diagonal(int factors, int steps, int* idx /*[factors][steps]*/) {
  int i0 = 0, j0 = 0, i = 0, j = 0;
  for (int counter = 0; counter < factors * steps; ++counter) {
    idx[i * steps + j] = counter;
    const bool diagonal_done = (i == 0) || (j == steps - 1);
    if (diagonal_done) {
      if (i0 < factors - 1) {
        ++i0;
        j0 = 0;
      } else {
        i0 = factors - 1;
        ++j0;
      }
      i = i0;
      j = j0;
    } else {
      --i;
      ++j;
    }
  }
}

// Builds the construction order and weights.  Point bidx[i] (0-based step
// index) is built at stage i from its left neighbour left[i]-1 (absent when
// left[i] == 0) and right neighbour right[i].
template <class R>
void bridge_tables_t(int steps, R* lw, R* rw, R* sd, int* left, int* right,
                     int* bidx) {
  std::vector<R> t(steps);
  for (int i = 0; i < steps; ++i) t[i] = static_cast<R>(i + 1);
  std::vector<int> built(steps, 0);
  built[steps - 1] = 1;
  bidx[0] = steps - 1;
  left[0] = right[0] = 0;
  sd[0] = std::sqrt(t[steps - 1]);
  lw[0] = rw[0] = R(0);
  int j = 0;
  for (int i = 1; i < steps; ++i) {
    while (built[j]) ++j;  // first unbuilt point
    int k = j;
    while (!built[k]) ++k;  // next built point to its right
    const int l = j + ((k - 1 - j) >> 1);
    built[l] = i;
    bidx[i] = l;
    left[i] = j;
    right[i] = k;
    if (j != 0) {
      lw[i] = (t[k] - t[l]) / (t[k] - t[j - 1]);
      rw[i] = (t[l] - t[j - 1]) / (t[k] - t[j - 1]);
      sd[i] = std::sqrt(((t[l] - t[j - 1]) * (t[k] - t[l])) / (t[k] - t[j - 1]));
    } else {
      lw[i] = (t[k] - t[l]) / t[k];
      rw[i] = t[l] / t[k];
      sd[i] = std::sqrt(t[l] * (t[k] - t[l]) / t[k]);
    }
    j = k + 1;
    if (j >= steps) j = 0;
  }
}

int make_bridge_plan(int steps, int factors, const int* h_alloc,
                     BridgePlan* plan) {
  LMM_REQUIRE(steps >= 1 && steps <= kMaxSteps,
              "bridge: steps must be in [1,%d]", kMaxSteps);
  LMM_REQUIRE(factors >= 1 && factors <= kMaxFactors,
              "bridge: factors must be in [1,%d]", kMaxFactors);
  plan->steps = steps;
  plan->factors = factors;
  bridge_tables_t<float>(steps, plan->lw, plan->rw, plan->sd, plan->left,
                         plan->right, plan->bidx);
  if (h_alloc) {
    for (int i = 0; i < factors * steps; ++i) {
      LMM_REQUIRE(h_alloc[i] >= 0 && h_alloc[i] < factors * steps,
                  "bridge: allocation index out of range");
      plan->alloc[i] = h_alloc[i];
    }
  } else {
    bridge_diagonal(factors, steps, plan->alloc);
  }
  return LMM_OK;
}

}  // namespace lmm

extern "C" int lmm_bridge_allocate_diagonal(int factors, int steps,
                                            int* h_indices) {
  LMM_REQUIRE(factors >= 1 && steps >= 1 && h_indices,
              "lmm_bridge_allocate_diagonal: bad arguments");
  bridge_diagonal(factors, steps, h_indices);
  return LMM_OK;
}

extern "C" int lmm_bridge_tables_host(int steps, double* lw, double* rw,
                                      double* sd, int* left, int* right,
                                      int* bidx) {
  LMM_REQUIRE(steps >= 1 && lw && rw && sd && left && right && bidx,
              "lmm_bridge_tables_host: bad arguments");
  bridge_tables_t<double>(steps, lw, rw, sd, left, right, bidx);
  return LMM_OK;
}

// One thread per (path, factor); the S bridge points of the thread live in
// shared memory W[i][tid] (thread-contiguous, conflict free), with a zero
// row S as the left neighbour of points that have none.  The factor's plan
// is staged per CTA as 16-byte weight and offset vectors (the form of the
// fused variates kernel: no branch and no parameter-space load per point),
// and the normals of kBridgeGroup points are loaded together ahead of their
// arithmetic.  Each point is lw * W[left] + rw * W[right] + sd * z with the
// roundings of the reference's order.
constexpr int kBridgeGroup = 8;

__global__ void __launch_bounds__(128)
    bridge_kernel(const float* __restrict__ in, float* __restrict__ out,
                  int paths, const __grid_constant__ BridgePlan plan) {
  extern __shared__ __align__(16) float W[];
  const int S = plan.steps, F = plan.factors;
  const int f = blockIdx.y;
  const int T = blockDim.x, tid = threadIdx.x;
  float4* bw_s = reinterpret_cast<float4*>(W + (size_t)(S + 1) * T);
  int4* bo_s = reinterpret_cast<int4*>(bw_s + S);
  int* al_s = reinterpret_cast<int*>(bo_s + S);
  for (int i = tid; i < S; i += T) {
    // stage 0 is the terminal point W_S = sd_0 z (row S - 1)
    const bool first = i == 0;
    const int jl = first ? 0 : plan.left[i];
    bw_s[i] = make_float4(jl != 0 ? plan.lw[i] : 0.0f, first ? 0.0f : plan.rw[i], plan.sd[i],
                          0.0f);
    bo_s[i] = make_int4((jl != 0 ? jl - 1 : S) * T, (first ? S : plan.right[i]) * T,
                        (first ? S - 1 : plan.bidx[i]) * T, 0);
    al_s[i] = plan.alloc[f * S + i];
  }
  W[(size_t)S * T + tid] = 0.0f;
  __syncthreads();
  float* w = W + tid;
  constexpr int G = kBridgeGroup;
  for (int p = blockIdx.x * T + tid; p < paths; p += gridDim.x * T) {
    for (int i0 = 0; i0 < S; i0 += G) {
      float z[G];
#pragma unroll
      for (int k = 0; k < G; ++k)
        z[k] = __ldg(in + (size_t)al_s[min(i0 + k, S - 1)] * paths + p);
#pragma unroll
      for (int k = 0; k < G; ++k) {
        const int i = i0 + k;
        if (i < S) {
          const float4 bw = bw_s[i];
          const int4 bo = bo_s[i];
          float y = bw.x * w[bo.x];
          y = fmaf(bw.y, w[bo.y], y);
          y = fmaf(bw.z, z[k], y);
          w[bo.z] = y;
        }
      }
    }
    float prev = 0.0f;
    for (int s = 0; s < S; ++s) {
      const float cur = w[s * T];
      out[((size_t)s * F + f) * paths + p] = cur - prev;
      prev = cur;
    }
  }
}

extern "C" int lmm_bridge_transform(const float* d_in, float* d_out, int paths,
                                    int steps, int factors, const int* h_alloc,
                                    lmm_stream_t stream) {
  LMM_REQUIRE(paths >= 0, "lmm_bridge_transform: paths < 0");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(d_in && d_out, "lmm_bridge_transform: null pointer");
  BridgePlan plan;
  int st = make_bridge_plan(steps, factors, h_alloc, &plan);
  if (st != LMM_OK) return st;
  const int block = 128;
  const size_t smem = (size_t)(steps + 1) * block * sizeof(float) +
                      (size_t)steps * (sizeof(float4) + sizeof(int4) + sizeof(int));
  if (smem > 48 * 1024) {
    int s2 = check_cuda(cudaFuncSetAttribute(
                            bridge_kernel,
                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)smem),
                        "lmm_bridge_transform: smem attribute");
    if (s2 != LMM_OK) return s2;
  }
  int gx = div_up(paths, block);
  int cap = sm_count() * 8;
  if (gx > cap) gx = cap;
  dim3 grid(gx, factors);
  bridge_kernel<<<grid, block, smem, (cudaStream_t)stream>>>(d_in, d_out,
                                                             paths, plan);
  return check_launch("lmm_bridge_transform");
}

// ---------------------------------------------------------------------------
// Reordering of multi-factor Sobol variates before a power-of-two bridge per
// factor (the reference's brownianBridgeMultiGPUReorder, Bridge_multi_gpu.cu:
// 20-160, with the orderings of BrownianBridgeMultiDim, gold/Bridge_gold.h:
// 334-404): variate i of a path (input [factors * 2^k][paths]) goes to the
// bridge stage dim(i) of factor fac(i), output [2^k][paths][factors], the
// layout on which a one-factor bridge over paths x factors vectors runs.
// Orderings: 0 = row (the factors of one stage are consecutive variates),
// 1 = column (each factor's stages are consecutive), 2 = triangular (the
// stages walk anti-diagonals of the (stage, factor) grid).
// ---------------------------------------------------------------------------
namespace {

struct ReorderTab {
  int n;
  int dst[kMaxSteps * kMaxFactors];  // output row offset dim * factors + factor
};

__global__ void __launch_bounds__(128)
    bridge_reorder_kernel(const float* __restrict__ in, float* __restrict__ out, int paths,
                          int factors, const __grid_constant__ ReorderTab t) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    for (int i = 0; i < t.n; ++i) {
      const int d = t.dst[i];
      const int dim = d / factors, fac = d - dim * factors;
      out[((size_t)dim * paths + p) * factors + fac] = __ldg(in + (size_t)i * paths + p);
    }
  }
}

}  // namespace

extern "C" int lmm_bridge_reorder(const float* d_in, float* d_out, int n_poweroftwo,
                                  int factors, int paths, int ordering,
                                  lmm_stream_t stream) {
  LMM_REQUIRE(n_poweroftwo >= 0 && n_poweroftwo <= 7,
              "lmm_bridge_reorder: 2^k points with k in [0,7]");
  LMM_REQUIRE(factors >= 1 && factors <= kMaxFactors,
              "lmm_bridge_reorder: factors must be in [1,%d]", kMaxFactors);
  LMM_REQUIRE(paths >= 0 && ordering >= 0 && ordering <= 2,
              "lmm_bridge_reorder: bad paths or ordering");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(d_in && d_out, "lmm_bridge_reorder: null pointer");
  const int points = 1 << n_poweroftwo, N = points * factors;
  ReorderTab t;
  t.n = N;
  int col = 0, row = 0;  // triangular walk: factor (column) and stage (row)
  for (int i = 0; i < N; ++i) {
    int dim, fac;
    if (ordering == 1) {  // column
      fac = i / points;
      dim = i % points;
    } else if (ordering == 0) {  // row
      fac = i % factors;
      dim = i / factors;
    } else {  // triangular
      fac = col;
      dim = row;
      if (col > 0 && row < points - 1) {
        --col;
        ++row;
      } else {
        const int sum = row + col + 1;
        col = sum < factors - 1 ? sum : factors - 1;
        row = sum - col;
      }
    }
    t.dst[i] = dim * factors + fac;
  }
  const int block = 128;
  bridge_reorder_kernel<<<grid_for(paths, block, 8), block, 0, (cudaStream_t)stream>>>(
      d_in, d_out, paths, factors, t);
  return check_launch("lmm_bridge_reorder");
}
