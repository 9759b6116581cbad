// ls_steps.cu — the reference's per-date Longstaff–Schwartz step routines as
// separate kernels (LS_gpu.h:21-80, LS_gpu.cu:17-470): basis expansion,
// net continuation values, the exercise update of the backward induction
// with a regression-depth chain, and the numeraire re-deflation.  The
// pipeline's own regression (ls.cu) fuses these into one launch per date;
// these entry points serve callers that drive the reference's loop
// (LS_main_cula.h:565-837) themselves.  FP32 throughout, like the
// reference; coalesced [row][path] layouts.
#include "lmm_common.cuh"

#include <cstring>

using namespace lmm;

namespace {

constexpr int kLsVarsMax = 7;  // quadratic: 1 + 2 V <= 16; cross: 1 + 3 V <= 16

// Basis functions of one date from its variables x[v][p] (v < V):
// quadratic (quadraticPolynomialDevice, LS_gpu.h:92-136):
//   1, x0, x0^2, x1, x1^2, ...
// cross (quadraticPolynomialCrossDevice, LS_gpu.h:138-232):
//   V = 1: 1, x0, x0^2;  V = 2: 1, x0, x1, x0^2, x0 x1, x1^2;
//   V >= 3: 1, x_0..x_{V-1}, x_i x_{(i+1) mod V}, x_i^2.
__global__ void __launch_bounds__(128)
    expand_basis_kernel(const float* __restrict__ x, float* __restrict__ out, int paths, int V,
                        int cross) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths; p += gridDim.x * blockDim.x) {
    float v[kLsVarsMax];
#pragma unroll
    for (int i = 0; i < kLsVarsMax; ++i) v[i] = i < V ? __ldg(x + (size_t)i * paths + p) : 0.0f;
    float* o = out + p;
    int j = 0;
    o[(size_t)(j++) * paths] = 1.0f;
    if (!cross) {
      for (int i = 0; i < V; ++i) {
        o[(size_t)(j++) * paths] = v[i];
        o[(size_t)(j++) * paths] = v[i] * v[i];
      }
      continue;
    }
    for (int i = 0; i < V; ++i) o[(size_t)(j++) * paths] = v[i];
    if (V == 1) {
      o[(size_t)j * paths] = v[0] * v[0];
    } else if (V == 2) {
      o[(size_t)(j++) * paths] = v[0] * v[0];
      o[(size_t)(j++) * paths] = v[0] * v[1];
      o[(size_t)j * paths] = v[1] * v[1];
    } else {
      for (int i = 0; i < V; ++i) o[(size_t)(j++) * paths] = v[i] * v[(i + 1) % V];
      for (int i = 0; i < V; ++i) o[(size_t)(j++) * paths] = v[i] * v[i];
    }
  }
}

struct Weights {
  float w[kMaxBasis * 8];  // [depth][row_size] (row_size <= kMaxBasis)
  float lo[8], hi[8];
};

// estimate - exercise value at one date (continuation_net_value_evaluation_
// kernel, LS_gpu.cu:57-99): est = shift + sum_i w_i phi_i[p].
__global__ void __launch_bounds__(128)
    net_values_kernel(const float* __restrict__ phi, const float* __restrict__ ex,
                      float* __restrict__ out, int paths, int K, float shift,
                      const __grid_constant__ Weights W) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths; p += gridDim.x * blockDim.x) {
    float est = shift;
    for (int i = 0; i < K; ++i) est += W.w[i] * __ldg(phi + (size_t)i * paths + p);
    out[p] = est - __ldg(ex + p);
  }
}

// The exercise update with a regression-depth chain
// (exercise_updating_LS_multi_kernel, LS_gpu.cu:312-402): walk depth d
// while the net value lies within [lo_d, hi_d] and d is not the last depth;
// exercise when the final net value is negative, then the continuation
// value becomes the exercise value; exercises[p] = 1 or -1 and the last
// estimate are recorded.
__global__ void __launch_bounds__(128)
    ls_update_multi_kernel(const float* __restrict__ phi, const float* __restrict__ ex,
                           float* __restrict__ cont, float* __restrict__ est_out,
                           int* __restrict__ exercises, int paths, int K, int row, int depth,
                           float shift, const __grid_constant__ Weights W) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths; p += gridDim.x * blockDim.x) {
    const float exv = __ldg(ex + p);
    float est = 0.0f;
    bool exercise = false;
    for (int d = 0; d < depth; ++d) {
      est = shift;
      for (int i = 0; i < K; ++i) est += W.w[d * row + i] * __ldg(phi + (size_t)i * paths + p);
      const float net = est - exv;
      if (d == depth - 1 || net < W.lo[d] || net > W.hi[d]) {
        exercise = net < 0.0f;
        break;
      }
    }
    if (exercise) cont[p] = exv;
    exercises[p] = exercise ? 1 : -1;
    est_out[p] = est;
  }
}

// values[p] *= num_new[p] / num_old[p] (numeraire_deflating_kernel,
// LS_gpu.cu:251-265).
__global__ void __launch_bounds__(256)
    deflate_kernel(float* __restrict__ values, const float* __restrict__ num_new,
                   const float* __restrict__ num_old, int paths) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths; p += gridDim.x * blockDim.x)
    values[p] *= __ldg(num_new + p) / __ldg(num_old + p);
}

int load_weights(const float* d_w, int n, const float* d_lo, const float* d_hi, int depth,
                 Weights* W, cudaStream_t s) {
  memset(W, 0, sizeof(*W));
  int st = check_cuda(cudaMemcpyAsync(W->w, d_w, (size_t)n * sizeof(float),
                                      cudaMemcpyDeviceToHost, s),
                      "LS step: read coefficients");
  if (st) return st;
  if (d_lo && d_hi && depth > 0) {
    st = check_cuda(cudaMemcpyAsync(W->lo, d_lo, (size_t)depth * sizeof(float),
                                    cudaMemcpyDeviceToHost, s),
                    "LS step: read lower cuts");
    if (st) return st;
    st = check_cuda(cudaMemcpyAsync(W->hi, d_hi, (size_t)depth * sizeof(float),
                                    cudaMemcpyDeviceToHost, s),
                    "LS step: read upper cuts");
    if (st) return st;
  }
  return check_cuda(cudaStreamSynchronize(s), "LS step: synchronise");
}

}  // namespace

extern "C" int lmm_ls_expand_basis(int total_paths, const float* d_vars, int exercise,
                                   int max_vars, int nvars, int cross, float* d_basis,
                                   lmm_stream_t stream) {
  LMM_REQUIRE(total_paths >= 1 && exercise >= 0 && max_vars >= nvars && nvars >= 0,
              "lmm_ls_expand_basis: bad sizes");
  LMM_REQUIRE(nvars <= (cross ? 5 : kLsVarsMax),
              "lmm_ls_expand_basis: at most 16 basis functions");
  LMM_REQUIRE(d_vars && d_basis, "lmm_ls_expand_basis: null pointer");
  const float* x = d_vars + (size_t)total_paths * max_vars * exercise;
  expand_basis_kernel<<<grid_for(total_paths, 128, 8), 128, 0, (cudaStream_t)stream>>>(
      x, d_basis, total_paths, nvars, cross ? 1 : 0);
  return check_launch("lmm_ls_expand_basis");
}

extern "C" int lmm_ls_net_values(int paths, const float* d_basis, int nbasis,
                                 const float* d_weights, const float* d_exercise_values,
                                 float shift, float* d_out, lmm_stream_t stream) {
  LMM_REQUIRE(paths >= 1 && nbasis >= 1 && nbasis <= kMaxBasis,
              "lmm_ls_net_values: bad sizes");
  LMM_REQUIRE(d_basis && d_weights && d_exercise_values && d_out,
              "lmm_ls_net_values: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  Weights W;
  int st = load_weights(d_weights, nbasis, nullptr, nullptr, 0, &W, s);
  if (st) return st;
  net_values_kernel<<<grid_for(paths, 128, 8), 128, 0, s>>>(d_basis, d_exercise_values, d_out,
                                                            paths, nbasis, shift, W);
  return check_launch("lmm_ls_net_values");
}

extern "C" int lmm_ls_update_multi(int paths, int exercise, const float* d_basis, int nbasis,
                                   int row_size, int depth, const float* d_weights,
                                   const float* d_lower_cuts, const float* d_upper_cuts,
                                   float* d_continuation, const float* d_exercise_values,
                                   float shift, float* d_estimates, int* d_exercises,
                                   lmm_stream_t stream) {
  LMM_REQUIRE(paths >= 1 && exercise >= 0 && nbasis >= 1 && nbasis <= row_size &&
                  row_size <= kMaxBasis && depth >= 1 && depth <= 8,
              "lmm_ls_update_multi: bad sizes");
  LMM_REQUIRE(d_basis && d_weights && d_lower_cuts && d_upper_cuts && d_continuation &&
                  d_exercise_values && d_estimates && d_exercises,
              "lmm_ls_update_multi: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  Weights W;
  int st = load_weights(d_weights + (size_t)row_size * exercise * depth, row_size * depth,
                        d_lower_cuts, d_upper_cuts, depth, &W, s);
  if (st) return st;
  ls_update_multi_kernel<<<grid_for(paths, 128, 8), 128, 0, s>>>(
      d_basis, d_exercise_values + (size_t)paths * exercise, d_continuation, d_estimates,
      d_exercises, paths, nbasis, row_size, depth, shift, W);
  return check_launch("lmm_ls_update_multi");
}

extern "C" int lmm_ls_deflate(float* d_values, const float* d_numeraires, int paths,
                              int new_step, int old_step, lmm_stream_t stream) {
  LMM_REQUIRE(paths >= 1 && new_step >= 0 && old_step >= 0, "lmm_ls_deflate: bad sizes");
  LMM_REQUIRE(d_values && d_numeraires, "lmm_ls_deflate: null pointer");
  deflate_kernel<<<grid_for(paths, 256, 4), 256, 0, (cudaStream_t)stream>>>(
      d_values, d_numeraires + (size_t)new_step * paths, d_numeraires + (size_t)old_step * paths,
      paths);
  return check_launch("lmm_ls_deflate");
}
