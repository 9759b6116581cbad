// cashflow.cu — product cash flows, exercise values, discounting,
// aggregation into exercise-date buckets and LS basis variables.  These are
// bandwidth kernels: one thread per path, loops over steps, coalesced
// [step][path] accesses.
//
// Reference behaviour followed:
//   swap flows           cashFlowGeneration_product_gpu.h:128-230,
//                        gold/cashFlowGeneration_product_gold.h:224-245
//   payer swaption value exercise_values_examples.h:49-76,
//                        gold/early_exercise_value_generator_gold.h:93-130
//   discounting          cashFlowDiscounting_gpu.cu:29-255,
//                        gold/cashFlowDiscounting_gold.h:20-92
//   partial discounting  cashFlowDiscounting_gpu.cu:369-495,
//                        gold/cashFlowDiscounting_gold.h:97-205
//   indices and weights  gold/cashFlowDiscounting_gold.h:210-258
//   exercise mapping     gold/cashFlowDiscounting_gold.cpp (find...Indices)
//   aggregation          cashFlowAggregation_gpu.cu:22-102,
//                        gold/cashFlowAggregation_gold.h:18-36
//   basis variables      LS_Basis_gpu.h:25-163, LS_basis_examples_gpu.h:28,85,
//                        gold/LS_basis_examples_gold.h:129-176
#include "lmm_common.cuh"
#include "lmm_device.cuh"

using namespace lmm;

namespace {
typedef IntTab<kMaxSteps> StepTab;
typedef FloatTab<kMaxSteps> StepFTab;

struct SwapData {
  float strike, pay_receive;
  float acc1[kMaxSteps], acc2[kMaxSteps];
};
}  // namespace

// ---------------------------------------------------------------------------
// Swap: flow1 = -acc1*K*pr, flow2 = acc2*f*pr on every step.
// Caplet strip: flow1 = acc*max(f-K,0), flow2 = 0.
// ---------------------------------------------------------------------------
// The grid spans paths (x) and steps (y): every (step, path) flow is
// independent, so each thread writes one.
template <int PRODUCT>
__global__ void flows_kernel(float* __restrict__ f1, float* __restrict__ f2,
                             const float* __restrict__ rate1, int paths,
                             int steps, const __grid_constant__ SwapData d) {
  const int s = blockIdx.y;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    const size_t ix = (size_t)s * paths + p;
    const float r = rate1[ix];
    if (PRODUCT == 0) {
      f2[ix] = d.acc2[s] * r * d.pay_receive;
      f1[ix] = -d.acc1[s] * d.strike * d.pay_receive;
    } else {
      f1[ix] = d.acc1[s] * fmaxf(r - d.strike, 0.0f);
      f2[ix] = 0.0f;
    }
  }
}

extern "C" int lmm_cashflows_swap(float* d_flows1, float* d_flows2,
                                  const float* h_aux, int paths, int steps,
                                  const float* d_rates1, lmm_stream_t stream) {
  LMM_REQUIRE(steps >= 1 && steps <= kMaxSteps && paths >= 0,
              "lmm_cashflows_swap: bad sizes");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(d_flows1 && d_flows2 && h_aux && d_rates1,
              "lmm_cashflows_swap: null pointer");
  SwapData d;
  d.strike = h_aux[0];
  d.pay_receive = h_aux[1];
  for (int s = 0; s < steps; ++s) {
    d.acc1[s] = h_aux[2 + s];
    d.acc2[s] = h_aux[2 + steps + s];
  }
  const int block = 256;
  flows_kernel<0><<<dim3(grid_for(paths, block, 1), steps), block, 0,
                    (cudaStream_t)stream>>>(d_flows1, d_flows2, d_rates1,
                                            paths, steps, d);
  return check_launch("lmm_cashflows_swap");
}

extern "C" int lmm_cashflows_caplet(float* d_flows1, float* d_flows2,
                                    const float* h_aux, int paths, int steps,
                                    const float* d_rates1,
                                    lmm_stream_t stream) {
  LMM_REQUIRE(steps >= 1 && steps <= kMaxSteps && paths >= 0,
              "lmm_cashflows_caplet: bad sizes");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(d_flows1 && d_flows2 && h_aux && d_rates1,
              "lmm_cashflows_caplet: null pointer");
  SwapData d;
  d.strike = h_aux[0];
  d.pay_receive = 1.0f;
  for (int s = 0; s < steps; ++s) d.acc1[s] = d.acc2[s] = h_aux[1 + s];
  const int block = 256;
  flows_kernel<1><<<dim3(grid_for(paths, block, 1), steps), block, 0,
                    (cudaStream_t)stream>>>(d_flows1, d_flows2, d_rates1,
                                            paths, steps, d);
  return check_launch("lmm_cashflows_caplet");
}

// ---------------------------------------------------------------------------
// TARN (cashFlowGeneratorCallerTARN, cashFlowGeneration_product_gpu.cu:13;
// product TARN, cashFlowGeneration_product_gpu.h:19-109; gold TARN_gold,
// gold/cashFlowGeneration_product_gold.h:76-165).  One thread per path
// walks the steps: flow2 = accrual2 * rate2; coupon max(K - m rate1, 0) *
// accrual1 is paid (flow1 = -coupon) until the coupons would reach the
// total, when flow1 = paid - total and the note ends; the last step pays
// paid - total.  Steps after the end carry zero flows.
// ---------------------------------------------------------------------------
struct TarnData {
  float total, strike, mult;
  float acc1[kMaxSteps], acc2[kMaxSteps];
};

__global__ void tarn_kernel(float* __restrict__ flows1, float* __restrict__ flows2,
                            const float* __restrict__ rates1,
                            const float* __restrict__ rates2, int paths, int steps,
                            const __grid_constant__ TarnData d) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    float paid = 0.0f;
    bool over = false;
    constexpr int G = 8;  // steps whose loads are issued together
    float r1v[G], r2v[G];
    for (int i = 0; i < steps; ++i) {
      if (i % G == 0)
#pragma unroll
        for (int j = 0; j < G; ++j) {
          const bool ok = i + j < steps && !over;
          r1v[j] = ok ? rates1[(size_t)(i + j) * paths + p] : 0.0f;
          r2v[j] = ok ? rates2[(size_t)(i + j) * paths + p] : 0.0f;
        }
      float f1 = 0.0f, f2 = 0.0f;
      if (!over) {
        f2 = d.acc2[i] * r2v[i % G];
        if (i + 1 == steps) {
          f1 = paid - d.total;
          over = true;
        } else {
          float c = (d.strike - d.mult * r1v[i % G]) * d.acc1[i];
          if (c < 0.0f) c = 0.0f;
          const float t = paid + c;
          if (t >= d.total) {
            f1 = paid - d.total;
            over = true;
          } else {
            f1 = -c;
            paid = t;
          }
        }
      }
      flows1[(size_t)i * paths + p] = f1;
      flows2[(size_t)i * paths + p] = f2;
    }
  }
}

extern "C" int lmm_cashflows_tarn(float* d_flows1, float* d_flows2, const float* h_aux,
                                  int paths, int steps, const float* d_rates1,
                                  const float* d_rates2, lmm_stream_t stream) {
  LMM_REQUIRE(steps >= 1 && steps <= kMaxSteps && paths >= 0,
              "lmm_cashflows_tarn: bad sizes");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(d_flows1 && d_flows2 && h_aux && d_rates1 && d_rates2,
              "lmm_cashflows_tarn: null pointer");
  TarnData d;
  d.total = h_aux[0];
  d.strike = h_aux[1];
  d.mult = h_aux[2];
  for (int i = 0; i < steps; ++i) {
    d.acc1[i] = h_aux[3 + i];
    d.acc2[i] = h_aux[3 + steps + i];
  }
  const int block = 256;
  tarn_kernel<<<grid_for(paths, block, 8), block, 0, (cudaStream_t)stream>>>(
      d_flows1, d_flows2, d_rates1, d_rates2, paths, steps, d);
  return check_launch("lmm_cashflows_tarn");
}

// ---------------------------------------------------------------------------
// Bermudan payer swaption exercise value max((SR-K)*A, 0).
// ---------------------------------------------------------------------------
__global__ void payer_swaption_value_kernel(float strike,
                                            const float* __restrict__ sr,
                                            const float* __restrict__ ann,
                                            int batch, int total, int offset,
                                            int n_ex, float* __restrict__ out) {
  const int e = blockIdx.y;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < batch;
       p += gridDim.x * blockDim.x) {
    const float v = (sr[(size_t)e * batch + p] - strike) *
                    ann[(size_t)e * batch + p];
    out[(size_t)e * total + offset + p] = v > 0.0f ? v : 0.0f;
  }
}

extern "C" int lmm_exercise_values_payer_swaption(
    float strike, const float* d_swap_rates, const float* d_annuities,
    int batch_paths, int total_paths, int offset, int n_exercise,
    float* d_out, lmm_stream_t stream) {
  LMM_REQUIRE(batch_paths >= 0 && offset >= 0 &&
                  offset + batch_paths <= total_paths && n_exercise >= 0 &&
                  n_exercise <= 65535,
              "lmm_exercise_values_payer_swaption: bad sizes");
  if (batch_paths == 0 || n_exercise == 0) return LMM_OK;
  LMM_REQUIRE(d_swap_rates && d_annuities && d_out,
              "lmm_exercise_values_payer_swaption: null pointer");
  const int block = 256;
  dim3 grid(grid_for(batch_paths, block, 1), n_exercise);
  payer_swaption_value_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(
      strike, d_swap_rates, d_annuities, batch_paths, total_paths, offset,
      n_exercise, d_out);
  return check_launch("lmm_exercise_values_payer_swaption");
}

// ---------------------------------------------------------------------------
// Discounting with log-linear interpolation in the curve of the generation
// step: df = (P_{s,i1}/P_{s,s})^(1-theta) (P_{s,i2}/P_{s,s})^theta.
// ---------------------------------------------------------------------------
namespace {
struct DiscTab {
  int first[kMaxSteps], second[kMaxSteps], gen[kMaxSteps], target[kMaxSteps];
  float theta[kMaxSteps];
};
}  // namespace

__global__ void discounting_kernel(const float* __restrict__ disc,
                                   const float* __restrict__ flows,
                                   const float* __restrict__ num, int paths,
                                   int steps, float* __restrict__ out,
                                   float* __restrict__ summed,
                                   const __grid_constant__ DiscTab t) {
  const size_t layer = (size_t)(steps + 1) * paths;
  constexpr int G = 8;  // steps whose loads are issued together
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    float total = 0.0f;
    for (int s0 = 0; s0 < steps; s0 += G) {
      float bv[G], d1[G], d2[G], fv[G], nv[G];
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const int s = s0 + j;
        const bool ok = s < steps;
        const float* d = disc + (size_t)(ok ? s : 0) * layer + p;
        bv[j] = ok ? d[(size_t)s * paths] : 1.0f;
        d1[j] = ok ? d[(size_t)t.first[s] * paths] : 1.0f;
        d2[j] = ok ? d[(size_t)t.second[s] * paths] : 1.0f;
        fv[j] = ok ? flows[(size_t)s * paths + p] : 0.0f;
        nv[j] = ok ? num[(size_t)s * paths + p] : 1.0f;
      }
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const int s = s0 + j;
        if (s < steps) {
          const float r1 = d1[j] / bv[j];
          const float r2 = d2[j] / bv[j];
          const float th = t.theta[s];
          const float df = powf(r1, 1.0f - th) * powf(r2, th);
          float cf = fv[j];
          cf *= df;
          cf /= nv[j];
          if (out) out[(size_t)s * paths + p] = cf;
          total += cf;
        }
      }
    }
    if (summed) summed[p] = total;
  }
}

extern "C" int lmm_cashflow_discounting(const int* h_first_index,
                                        const int* h_second_index,
                                        const float* h_theta,
                                        const float* d_discounts,
                                        const float* d_flows,
                                        const float* d_numeraires, int paths,
                                        int steps, float* d_discounted,
                                        float* d_summed, lmm_stream_t stream) {
  LMM_REQUIRE(steps >= 1 && steps <= kMaxSteps && paths >= 0,
              "lmm_cashflow_discounting: bad sizes");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(h_first_index && h_second_index && h_theta && d_discounts &&
                  d_flows && d_numeraires && (d_discounted || d_summed),
              "lmm_cashflow_discounting: null pointer");
  DiscTab t;
  for (int s = 0; s < steps; ++s) {
    LMM_REQUIRE(h_first_index[s] >= 0 && h_first_index[s] <= steps &&
                    h_second_index[s] >= 0 && h_second_index[s] <= steps,
                "lmm_cashflow_discounting: index out of range at step %d", s);
    t.first[s] = h_first_index[s];
    t.second[s] = h_second_index[s];
    t.theta[s] = h_theta[s];
  }
  const int block = 256;
  discounting_kernel<<<grid_for(paths, block, 8), block, 0,
                       (cudaStream_t)stream>>>(d_discounts, d_flows,
                                               d_numeraires, paths, steps,
                                               d_discounted, d_summed, t);
  return check_launch("lmm_cashflow_discounting");
}

__global__ void discounting_partial_kernel(const float* __restrict__ disc,
                                           const float* __restrict__ flows,
                                           const float* __restrict__ num,
                                           int paths, int steps, int n_flows,
                                           float* __restrict__ out,
                                           const __grid_constant__ DiscTab t) {
  // the grid spans paths (x) and flows (y): every flow is independent
  const size_t layer = (size_t)(steps + 1) * paths;
  const int i = blockIdx.y;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    {
      const int s = t.gen[i];
      const float* d = disc + s * layer + p;
      const float b = d[(size_t)s * paths];
      const float r1 = d[(size_t)t.first[i] * paths] / b;
      const float r2 = d[(size_t)t.second[i] * paths] / b;
      const float df = r1 * powf(r2 / r1, t.theta[i]);
      const float cf = flows[(size_t)i * paths + p] * df;
      const float ratio = num[(size_t)t.target[i] * paths + p] /
                          num[(size_t)s * paths + p];
      out[(size_t)i * paths + p] = ratio * cf;
    }
  }
}

extern "C" int lmm_cashflow_discounting_partial(
    int n_flows, const int* h_gen_indices, const int* h_first_index,
    const int* h_second_index, const float* h_theta,
    const int* h_target_indices, const float* d_discounts,
    const float* d_flows, const float* d_numeraires, int paths, int steps,
    float* d_discounted, lmm_stream_t stream) {
  LMM_REQUIRE(n_flows >= 0 && n_flows <= kMaxSteps && steps >= 1 &&
                  steps <= kMaxSteps && paths >= 0,
              "lmm_cashflow_discounting_partial: bad sizes");
  if (paths == 0 || n_flows == 0) return LMM_OK;
  LMM_REQUIRE(h_gen_indices && h_first_index && h_second_index && h_theta &&
                  h_target_indices && d_discounts && d_flows &&
                  d_numeraires && d_discounted,
              "lmm_cashflow_discounting_partial: null pointer");
  DiscTab t;
  for (int i = 0; i < n_flows; ++i) {
    LMM_REQUIRE(h_gen_indices[i] >= 0 && h_gen_indices[i] < steps &&
                    h_target_indices[i] >= 0 && h_target_indices[i] < steps &&
                    h_first_index[i] >= 0 && h_first_index[i] <= steps &&
                    h_second_index[i] >= 0 && h_second_index[i] <= steps,
                "lmm_cashflow_discounting_partial: index out of range at %d",
                i);
    t.gen[i] = h_gen_indices[i];
    t.target[i] = h_target_indices[i];
    t.first[i] = h_first_index[i];
    t.second[i] = h_second_index[i];
    t.theta[i] = h_theta[i];
  }
  const int block = 256;
  discounting_partial_kernel<<<dim3(grid_for(paths, block, 1), n_flows), block, 0,
                               (cudaStream_t)stream>>>(
      d_discounts, d_flows, d_numeraires, paths, steps, n_flows, d_discounted,
      t);
  return check_launch("lmm_cashflow_discounting_partial");
}

// Payment times -> bracketing rate-time indices and log-linear weight.  The
// "beyond the last rate time" test compares against rate_times[n_payments-1],
// as the reference does.
extern "C" int lmm_cashflow_indices_weights(const float* h_rate_times,
                                            int n_rate_times,
                                            const float* h_payment_times,
                                            int n_payments, int* h_first_index,
                                            int* h_second_index,
                                            float* h_theta) {
  LMM_REQUIRE(n_payments >= 1 && n_rate_times >= n_payments + 1 &&
                  h_rate_times && h_payment_times && h_first_index &&
                  h_second_index && h_theta,
              "lmm_cashflow_indices_weights: bad arguments");
  for (int i = 0; i < n_payments; ++i) {
    const float time = h_payment_times[i];
    int a, b;
    if (time < h_rate_times[0]) {
      a = 0;
      b = 1;
    } else if (time > h_rate_times[n_payments - 1]) {
      a = n_payments - 1;
      b = n_payments;
    } else {
      int j = 1;
      while (time > h_rate_times[j]) ++j;
      a = j - 1;
      b = j;
    }
    h_first_index[i] = a;
    h_second_index[i] = b;
    h_theta[i] = (time - h_rate_times[a]) / (h_rate_times[b] - h_rate_times[a]);
  }
  return LMM_OK;
}

// For each generation step: index of the last exercise date at or before it,
// -1 if none.  Returns the first step with a non-negative index.
extern "C" int lmm_step_to_exercise_indices(const int* h_gen_indices, int n_gen,
                                            const int* h_exercise_indices,
                                            int n_exercise, int* h_out,
                                            int* h_first_positive) {
  LMM_REQUIRE(n_gen >= 0 && n_exercise >= 1 && h_gen_indices &&
                  h_exercise_indices && h_out && h_first_positive,
              "lmm_step_to_exercise_indices: bad arguments");
  for (int i = 0; i < n_gen; ++i) {
    int j = 0;
    while (j < n_exercise && h_exercise_indices[j] < h_gen_indices[i]) ++j;
    if (j == n_exercise) --j;
    if (h_exercise_indices[j] > h_gen_indices[i]) --j;
    h_out[i] = j;
  }
  int first = 0;
  while (first < n_gen && h_out[first] < 0) ++first;
  *h_first_positive = first;
  return LMM_OK;
}

// ---------------------------------------------------------------------------
// Aggregation: agg[j][offset+p] += flows[i][p], j = preceding[i], i >= start.
// The grid spans paths (x) and the target rows that receive flows (y): each
// thread adds, in increasing i, the flows of its target to the target's
// value, the order of one read-modify-write per flow.
// ---------------------------------------------------------------------------
namespace {
struct AggTab {
  int tgt[kMaxSteps];      // target rows with at least one flow
  int beg[kMaxSteps + 1];  // their flows: src[beg[t] .. beg[t + 1])
  int src[kMaxSteps];
};
}  // namespace

__global__ void aggregate_kernel(float* __restrict__ agg, int total,
                                 const float* __restrict__ flows, int batch,
                                 int offset, const __grid_constant__ AggTab t) {
  const int y = blockIdx.y;
  const int j = t.tgt[y], k0 = t.beg[y], k1 = t.beg[y + 1];
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < batch;
       p += gridDim.x * blockDim.x) {
    float* a = agg + (size_t)j * total + offset + p;
    float acc = *a;
#pragma unroll 4
    for (int k = k0; k < k1; ++k) acc += flows[(size_t)t.src[k] * batch + p];
    *a = acc;
  }
}

extern "C" int lmm_aggregate_flows(float* d_aggregated, int total_paths,
                                   int n_exercise, const float* d_flows,
                                   int batch_paths, int offset_for_output,
                                   int steps, const int* h_preceding_index,
                                   int start, lmm_stream_t stream) {
  LMM_REQUIRE(steps >= 1 && steps <= kMaxSteps && batch_paths >= 0 &&
                  offset_for_output >= 0 &&
                  offset_for_output + batch_paths <= total_paths &&
                  start >= 0,
              "lmm_aggregate_flows: bad sizes");
  if (batch_paths == 0) return LMM_OK;
  LMM_REQUIRE(d_aggregated && d_flows && h_preceding_index,
              "lmm_aggregate_flows: null pointer");
  for (int i = 0; i < steps; ++i)
    LMM_REQUIRE(h_preceding_index[i] < n_exercise,
                "lmm_aggregate_flows: preceding index out of range");
  AggTab t;
  int nt = 0, k = 0;
  for (int j = 0; j < n_exercise; ++j) {
    const int k_begin = k;
    for (int i = start; i < steps; ++i)
      if (h_preceding_index[i] == j) t.src[k++] = i;
    if (k > k_begin) {
      t.tgt[nt] = j;
      t.beg[nt] = k_begin;
      ++nt;
    }
  }
  t.beg[nt] = k;
  if (nt == 0) return LMM_OK;
  const int block = 256;
  aggregate_kernel<<<dim3(grid_for(batch_paths, block, 1), nt), block, 0,
                     (cudaStream_t)stream>>>(d_aggregated, total_paths, d_flows,
                                             batch_paths, offset_for_output, t);
  return check_launch("lmm_aggregate_flows");
}

// ---------------------------------------------------------------------------
// Basis variables: out[e][v][offset+p] = x or log(x + shift_v).
// ---------------------------------------------------------------------------
__global__ void basis_variables_kernel(int use_log, float s0, float s1,
                                       float s2, const float* __restrict__ r1,
                                       const float* __restrict__ r2,
                                       const float* __restrict__ r3, int batch,
                                       int total, int offset,
                                       float* __restrict__ out) {
  const int e = blockIdx.y;
  float* o = out + (size_t)e * 3 * total + offset;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < batch;
       p += gridDim.x * blockDim.x) {
    const size_t ix = (size_t)e * batch + p;
    float a = r1[ix], b = r2[ix], c = r3[ix];
    if (use_log) {
      a = logf(a + s0);
      b = logf(b + s1);
      c = logf(c + s2);
    }
    o[p] = a;
    o[(size_t)total + p] = b;
    o[2 * (size_t)total + p] = c;
  }
}

extern "C" int lmm_basis_variables(int use_log, const float* h_shifts,
                                   const float* d_rate1, const float* d_rate2,
                                   const float* d_rate3, int batch_paths,
                                   int total_paths, int offset, int n_exercise,
                                   float* d_out, lmm_stream_t stream) {
  LMM_REQUIRE(batch_paths >= 0 && offset >= 0 &&
                  offset + batch_paths <= total_paths && n_exercise >= 0 &&
                  n_exercise <= 65535,
              "lmm_basis_variables: bad sizes");
  if (batch_paths == 0 || n_exercise == 0) return LMM_OK;
  LMM_REQUIRE(d_rate1 && d_rate2 && d_rate3 && d_out &&
                  (!use_log || h_shifts),
              "lmm_basis_variables: null pointer");
  const float s0 = use_log ? h_shifts[0] : 0.0f;
  const float s1 = use_log ? h_shifts[1] : 0.0f;
  const float s2 = use_log ? h_shifts[2] : 0.0f;
  const int block = 256;
  dim3 grid(grid_for(batch_paths, block, 1), n_exercise);
  basis_variables_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(
      use_log, s0, s1, s2, d_rate1, d_rate2, d_rate3, batch_paths, total_paths,
      offset, d_out);
  return check_launch("lmm_basis_variables");
}
