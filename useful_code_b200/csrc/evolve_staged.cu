// evolve_staged.cu — the plain-FP32 staged chain: correlation + fixed drift,
// one predictor-corrector launch per step, then discount ratios, coterminal
// annuities and swap rates, spot numeraires and the gather kernels.  Each
// stage reads and writes full [step][rate][path] tensors in HBM, as the
// reference's staged chain does (LMM_evolver_full.cu:154-262,
// LMM_evolver_gpu.cu:607-826 and :1188-2189).  These kernels are the
// baseline the fused kernel is measured against, and drop-ins for the
// reference's staged entry points.
#include "lmm_common.cuh"
#include "lmm_device.cuh"

using namespace lmm;

namespace {

typedef IntTab<kMaxSteps> StepTab;

int load_alive(const int* h_alive, int steps, int rates, StepTab* t) {
  LMM_REQUIRE(steps >= 1 && steps <= kMaxSteps, "steps must be in [1,%d]",
              kMaxSteps);
  LMM_REQUIRE(h_alive != nullptr, "alive indices: null pointer");
  for (int s = 0; s < steps; ++s) {
    LMM_REQUIRE(h_alive[s] >= 0 && h_alive[s] <= rates,
                "alive index %d out of range at step %d", h_alive[s], s);
    t->v[s] = h_alive[s];
  }
  return LMM_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// (a6) correlation + fixed drift: out[s][r][p] = sum_f A[s][r][f] z[f] +
// drift[s][r] for r >= alive[s]  (correlate_drift_gpu.cu:142-218,
// gold/correlate_drift_gold.h:22-60).  The grid spans paths (x) and steps
// (y): each CTA correlates one step of a run of paths, so the work is
// spread over paths x steps, not paths alone.
// ---------------------------------------------------------------------------
// The step's pseudo-root rows (zero-padded to a multiple of 4 factors for
// 16-byte reads) and drifts are staged in shared memory once per CTA, so
// each output element costs its F FMAs and F/4 shared-memory reads; FT =
// the factor count when compiled for it, 0 = any count <= kMaxFactors.
template <int LAYOUT, int FT>
__global__ void __launch_bounds__(128)
    correlate_drift_kernel(const float* __restrict__ in, float* __restrict__ out,
                           const float* __restrict__ A,
                           const float* __restrict__ drift, int A_step,
                           int factors, int rates, int paths, int steps,
                           const __grid_constant__ StepTab alive) {
  constexpr int FM = FT > 0 ? FT : kMaxFactors;
  constexpr int FP = (FM + 3) & ~3;
  const int F = FT > 0 ? FT : factors;
  const int s = blockIdx.y;
  const int a = alive.v[s];
  extern __shared__ __align__(16) float csm[];
  float* As = csm;               // [rates][FP]
  float* dr = As + rates * FP;   // [rates]
  for (int i = threadIdx.x; i < (rates - a) * FP; i += blockDim.x) {
    const int r = a + i / FP, f = i - (i / FP) * FP;
    As[r * FP + f] = f < F ? __ldg(A + (size_t)s * A_step + r * factors + f) : 0.0f;
  }
  for (int r = a + threadIdx.x; r < rates; r += blockDim.x)
    dr[r] = __ldg(drift + (size_t)s * rates + r);
  __syncthreads();
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    float z[FP];
#pragma unroll
    for (int f = 0; f < FP; ++f) {
      z[f] = 0.0f;
      if (f < F) {
        const size_t idx = LAYOUT == 0 ? ((size_t)s * paths + p) * factors + f
                                       : ((size_t)s * factors + f) * paths + p;
        z[f] = __ldg(in + idx);
      }
    }
    float* o = out + (size_t)s * rates * paths + p;
#pragma unroll 4
    for (int r = a; r < rates; ++r) {
      const float4* a4 = reinterpret_cast<const float4*>(As + r * FP);
      float total = 0.0f;
#pragma unroll
      for (int q = 0; q < FP / 4; ++q) {
        const float4 v = a4[q];
        if (4 * q < F) total += v.x * z[4 * q];
        if (4 * q + 1 < F) total += v.y * z[4 * q + 1];
        if (4 * q + 2 < F) total += v.z * z[4 * q + 2];
        if (4 * q + 3 < F) total += v.w * z[4 * q + 3];
      }
      total += dr[r];
      o[(size_t)r * paths] = total;
    }
  }
}

extern "C" int lmm_correlate_drift(const float* d_in, float* d_out,
                                   const float* d_A, const int* h_alive,
                                   const float* d_drift, int A_offset_per_step,
                                   int factors, int out_dims, int paths,
                                   int steps, int variates_layout,
                                   lmm_stream_t stream) {
  LMM_REQUIRE(factors >= 1 && factors <= kMaxFactors,
              "lmm_correlate_drift: factors must be in [1,%d]", kMaxFactors);
  LMM_REQUIRE(out_dims >= 1 && paths >= 0, "lmm_correlate_drift: bad sizes");
  LMM_REQUIRE(variates_layout == 0 || variates_layout == 1,
              "lmm_correlate_drift: variates_layout must be 0 or 1");
  LMM_REQUIRE(A_offset_per_step >= out_dims * factors,
              "lmm_correlate_drift: A_offset_per_step too small");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(d_in && d_out && d_A && d_drift,
              "lmm_correlate_drift: null pointer");
  StepTab alive;
  int st = load_alive(h_alive, steps, out_dims, &alive);
  if (st) return st;
  const int block = 128;
  LMM_REQUIRE(steps <= 65535, "lmm_correlate_drift: too many steps");
  dim3 grid(grid_for(paths, block, 2), steps);
  auto go = [&](auto layout, auto ft) {
    constexpr int L = decltype(layout)::value, FT = decltype(ft)::value;
    constexpr int FP = ((FT > 0 ? FT : kMaxFactors) + 3) & ~3;
    const size_t smem = (size_t)out_dims * (FP + 1) * sizeof(float);
    correlate_drift_kernel<L, FT><<<grid, block, smem, (cudaStream_t)stream>>>(
        d_in, d_out, d_A, d_drift, A_offset_per_step, factors, out_dims, paths, steps,
        alive);
  };
  auto by_factors = [&](auto layout) {
    switch (factors) {
      case 3: go(layout, std::integral_constant<int, 3>()); break;
      case 5: go(layout, std::integral_constant<int, 5>()); break;
      case 10: go(layout, std::integral_constant<int, 10>()); break;
      case 15: go(layout, std::integral_constant<int, 15>()); break;
      default: go(layout, std::integral_constant<int, 0>()); break;
    }
  };
  if (variates_layout == 0)
    by_factors(std::integral_constant<int, 0>());
  else
    by_factors(std::integral_constant<int, 1>());
  return check_launch("lmm_correlate_drift");
}

// ---------------------------------------------------------------------------
// (a7) one predictor-corrector step for the rates r >= alive, one thread per
// path.  Spot drift mu_r = sum_f A[r][f] e_f(r), e_f(r) = sum_{alive<=j<=r}
// g_j A[j][f], g_j = (f_j + d_j) tau_j / (1 + f_j tau_j)
// (gold/LMM_evolver_gold.h:178-203).  The prefix e_f(r) only involves rates
// j <= r, so predictor drift, predicted rate, corrector drift and corrected
// rate are produced in one sweep over r (the order of the reference's fused
// kernel, LMM_evolver_all.cu:615-744); the arithmetic per rate equals
// LMM_evolver_pc_with_workspace_gold (gold/LMM_evolver_gold.h:315-387)
// including the log-rate cap.  Like the reference's GPU step kernels
// (LMM_evolver_gpu.cu:202-365) the sweep starts at the alive index: rates
// that have reset are neither read nor written.  Only the log-rates of the
// previous step are read: its rate f = exp(lf) - d is recomputed with the
// very expression that wrote it, so it is the stored value bit for bit, and
// each live rate-step moves 16 bytes (correlated increment and log-rate in,
// rate and log-rate out).
// ---------------------------------------------------------------------------
struct StepConst {
  float tau[kMaxRates];
  float disp[kMaxRates];
  float f0[kMaxRates];
  float logf0[kMaxRates];
};

// The rate sweep is serial per path, so each rate waits on its two loads
// unless they were issued earlier: the loads run one group of kPcGroup rates
// ahead of the arithmetic (a double buffer in registers), which leaves the
// arithmetic of every rate unchanged.
constexpr int kPcGroup = 8;

// FT = the factor count when compiled for it, 0 = any count <= kMaxFactors.
template <int FT>
__device__ __forceinline__ void pc_step_rate(int r, size_t ix, float lf, float cr, int factors,
                                             float cutoff, const StepConst& c, bool first,
                                             const float* __restrict__ As,
                                             float (&e)[FT > 0 ? FT : kMaxFactors],
                                             float (&ep)[FT > 0 ? FT : kMaxFactors],
                                             float* __restrict__ f_out,
                                             float* __restrict__ logf_out) {
  constexpr int FM = FT > 0 ? FT : kMaxFactors;
  if (FT > 0) factors = FT;
  const float tau = c.tau[r], d = c.disp[r];
  const float fr = first ? c.f0[r] : expf(lf) - d;
  const float g = (fr + d) * tau / (1.0f + fr * tau);
  const float* a = As + r * factors;
  float mu = 0.0f;
#pragma unroll
  for (int f = 0; f < FM; ++f)
    if (f < factors) {
      e[f] += a[f] * g;
      mu += a[f] * e[f];
    }
  lf += mu + cr;
  const float fp = expf(lf) - d;
  const float gp = (fp + d) * tau / (1.0f + fp * tau);
  float mup = 0.0f;
#pragma unroll
  for (int f = 0; f < FM; ++f)
    if (f < factors) {
      ep[f] += a[f] * gp;
      mup += a[f] * ep[f];
    }
  lf += 0.5f * (mup - mu);
  lf = fminf(lf, cutoff);
  f_out[ix] = expf(lf) - d;
  logf_out[ix] = lf;
}

template <int FT>
__global__ void __launch_bounds__(128)
    pc_step_kernel(const float* __restrict__ logf_prev,  // [rates][paths] or null
                   const float* __restrict__ corr,  // [rates][paths] this step
                   const float* __restrict__ A,     // [rates][factors] this step
                   float* __restrict__ f_out, float* __restrict__ logf_out,
                   int factors, int rates, int alive, int paths, float cutoff,
                   const __grid_constant__ StepConst c) {
  extern __shared__ float As[];  // [rates][factors]
  for (int i = threadIdx.x; i < rates * factors; i += blockDim.x) As[i] = A[i];
  __syncthreads();
  constexpr int G = kPcGroup;
  const bool first = logf_prev == nullptr;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    constexpr int FM = FT > 0 ? FT : kMaxFactors;
    float e[FM], ep[FM];
#pragma unroll
    for (int f = 0; f < FM; ++f) e[f] = ep[f] = 0.0f;
    float la[G], ca[G], lb[G], cb[G];
    // group loads: rate r0 + j of the sweep (rates past the last are not read)
#define PC_LOAD(L, C, r0)                                            \
  _Pragma("unroll") for (int j = 0; j < G; ++j) {                    \
    const int r = (r0) + j;                                          \
    const size_t ix = (size_t)r * paths + p;                         \
    L[j] = (r < rates && !first) ? logf_prev[ix] : 0.0f;             \
    C[j] = r < rates ? corr[ix] : 0.0f;                              \
    if (first && r < rates) L[j] = c.logf0[r];                       \
  }
#define PC_RUN(L, C, r0)                                                                  \
  _Pragma("unroll") for (int j = 0; j < G; ++j) {                                         \
    const int r = (r0) + j;                                                               \
    if (r < rates)                                                                        \
      pc_step_rate<FT>(r, (size_t)r * paths + p, L[j], C[j], factors, cutoff, c, first, As, \
                       e, ep, f_out, logf_out);                                           \
  }
    PC_LOAD(la, ca, alive)
    for (int r0 = alive; r0 < rates; r0 += 2 * G) {
      PC_LOAD(lb, cb, r0 + G)
      PC_RUN(la, ca, r0)
      PC_LOAD(la, ca, r0 + 2 * G)
      PC_RUN(lb, cb, r0 + G)
    }
#undef PC_LOAD
#undef PC_RUN
  }
}

extern "C" int lmm_evolve_pc_staged(const float* h_initial_rates,
                                    const float* h_taus,
                                    const float* h_displacements,
                                    const float* d_correlated, const float* d_A,
                                    const int* h_alive, int paths, int factors,
                                    int steps, int rates, float cutoff,
                                    float* d_rates, float* d_log_rates,
                                    lmm_stream_t stream) {
  LMM_REQUIRE(rates >= 1 && rates <= kMaxRates,
              "lmm_evolve_pc_staged: rates must be in [1,%d]", kMaxRates);
  LMM_REQUIRE(factors >= 1 && factors <= kMaxFactors,
              "lmm_evolve_pc_staged: factors must be in [1,%d]", kMaxFactors);
  LMM_REQUIRE(steps >= 1 && paths >= 0, "lmm_evolve_pc_staged: bad sizes");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(h_initial_rates && h_taus && d_correlated && d_A &&
                  h_displacements && d_rates && d_log_rates,
              "lmm_evolve_pc_staged: null pointer");
  StepTab alive;
  if (h_alive) {
    int st = load_alive(h_alive, steps, rates, &alive);
    if (st) return st;
    for (int s = 1; s < steps; ++s)
      LMM_REQUIRE(alive.v[s] >= alive.v[s - 1],
                  "lmm_evolve_pc_staged: alive indices must not decrease");
  } else {
    LMM_REQUIRE(steps <= kMaxSteps, "lmm_evolve_pc_staged: steps must be in [1,%d]",
                kMaxSteps);
    for (int s = 0; s < steps; ++s) alive.v[s] = 0;
  }
  StepConst c;
  for (int r = 0; r < rates; ++r) {
    c.tau[r] = h_taus[r];
    c.disp[r] = h_displacements[r];
    c.f0[r] = h_initial_rates[r];
    c.logf0[r] = logf(h_initial_rates[r] + h_displacements[r]);
  }
  const int block = 128;
  const int grid = grid_for(paths, block, 8);
  const size_t smem = (size_t)rates * factors * sizeof(float);
  const size_t layer = (size_t)rates * paths;
  auto kern = factors == 3    ? pc_step_kernel<3>
              : factors == 5  ? pc_step_kernel<5>
              : factors == 10 ? pc_step_kernel<10>
              : factors == 15 ? pc_step_kernel<15>
                              : pc_step_kernel<0>;
  for (int s = 0; s < steps; ++s) {
    kern<<<grid, block, smem, (cudaStream_t)stream>>>(
        s ? d_log_rates + (s - 1) * layer : nullptr, d_correlated + s * layer,
        d_A + (size_t)s * rates * factors, d_rates + s * layer,
        d_log_rates + s * layer, factors, rates, alive.v[s], paths, cutoff, c);
    int st = check_launch("lmm_evolve_pc_staged");
    if (st) return st;
  }
  return LMM_OK;
}

// ---------------------------------------------------------------------------
// (a7) one log-Euler step for the rates r >= alive (the reference's
// LMM_evolver_euler_noninitial_step_kernel, LMM_evolver_gpu.cu:835-953):
// log f_r += mu_r(f at the start of the step) + correlated increment, with
// the spot drift of pc_step_kernel and no corrector, capped at cutoff.
// Like pc_step_kernel it reads only the previous log-rates.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
    euler_step_kernel(const float* __restrict__ logf_prev,  // [rates][paths] or null
                      const float* __restrict__ corr,  // [rates][paths] this step
                      const float* __restrict__ A,     // [rates][factors] this step
                      float* __restrict__ f_out, float* __restrict__ logf_out,
                      int factors, int rates, int alive, int paths, float cutoff,
                      const __grid_constant__ StepConst c) {
  extern __shared__ float As[];  // [rates][factors]
  for (int i = threadIdx.x; i < rates * factors; i += blockDim.x) As[i] = A[i];
  __syncthreads();
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    float e[kMaxFactors];
#pragma unroll
    for (int f = 0; f < kMaxFactors; ++f) e[f] = 0.0f;
    for (int r = alive; r < rates; ++r) {
      const size_t ix = (size_t)r * paths + p;
      const float tau = c.tau[r], d = c.disp[r];
      float lf = logf_prev ? logf_prev[ix] : c.logf0[r];
      const float fr = logf_prev ? expf(lf) - d : c.f0[r];
      const float g = (fr + d) * tau / (1.0f + fr * tau);
      const float* a = As + r * factors;
      float mu = 0.0f;
#pragma unroll
      for (int f = 0; f < kMaxFactors; ++f)
        if (f < factors) {
          e[f] += a[f] * g;
          mu += a[f] * e[f];
        }
      lf += mu + corr[ix];
      lf = fminf(lf, cutoff);
      f_out[ix] = expf(lf) - d;
      logf_out[ix] = lf;
    }
  }
}

extern "C" int lmm_evolve_euler_staged(const float* h_initial_rates,
                                       const float* h_taus,
                                       const float* h_displacements,
                                       const float* d_correlated, const float* d_A,
                                       const int* h_alive, int paths, int factors,
                                       int steps, int rates, float cutoff,
                                       float* d_rates, float* d_log_rates,
                                       lmm_stream_t stream) {
  LMM_REQUIRE(rates >= 1 && rates <= kMaxRates,
              "lmm_evolve_euler_staged: rates must be in [1,%d]", kMaxRates);
  LMM_REQUIRE(factors >= 1 && factors <= kMaxFactors,
              "lmm_evolve_euler_staged: factors must be in [1,%d]", kMaxFactors);
  LMM_REQUIRE(steps >= 1 && steps <= kMaxSteps && paths >= 0,
              "lmm_evolve_euler_staged: bad sizes");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(h_initial_rates && h_taus && d_correlated && d_A && h_displacements &&
                  d_rates && d_log_rates,
              "lmm_evolve_euler_staged: null pointer");
  StepTab alive;
  if (h_alive) {
    int st = load_alive(h_alive, steps, rates, &alive);
    if (st) return st;
    for (int s = 1; s < steps; ++s)
      LMM_REQUIRE(alive.v[s] >= alive.v[s - 1],
                  "lmm_evolve_euler_staged: alive indices must not decrease");
  } else {
    for (int s = 0; s < steps; ++s) alive.v[s] = 0;
  }
  StepConst c;
  for (int r = 0; r < rates; ++r) {
    c.tau[r] = h_taus[r];
    c.disp[r] = h_displacements[r];
    c.f0[r] = h_initial_rates[r];
    c.logf0[r] = logf(h_initial_rates[r] + h_displacements[r]);
  }
  const int block = 128;
  const int grid = grid_for(paths, block, 8);
  const size_t smem = (size_t)rates * factors * sizeof(float);
  const size_t layer = (size_t)rates * paths;
  for (int s = 0; s < steps; ++s) {
    euler_step_kernel<<<grid, block, smem, (cudaStream_t)stream>>>(
        s ? d_log_rates + (s - 1) * layer : nullptr, d_correlated + s * layer,
        d_A + (size_t)s * rates * factors, d_rates + s * layer,
        d_log_rates + s * layer, factors, rates, alive.v[s], paths, cutoff, c);
    int st = check_launch("lmm_evolve_euler_staged");
    if (st) return st;
  }
  return LMM_OK;
}

// ---------------------------------------------------------------------------
// (a8) discount ratios P(T_s, T_r) = prod_{alive<=k<r} 1/(1+tau_k f_k)
// (gold/LMM_evolver_gold.h:460-490).
// ---------------------------------------------------------------------------
__global__ void discount_ratios_kernel(const float* __restrict__ rates_,
                                       float* __restrict__ disc, int paths,
                                       int steps, int rates,
                                       const __grid_constant__ StepTab alive,
                                       const __grid_constant__ FloatTab<kMaxRates> tau) {
  const int s = blockIdx.y;
  const int a = alive.v[s];
  const float* fr = rates_ + (size_t)s * rates * paths;
  float* d = disc + (size_t)s * (rates + 1) * paths;
  constexpr int G = 8;  // rates whose loads are issued together
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    float df = 1.0f;
    d[(size_t)a * paths + p] = df;
    for (int r0 = a; r0 < rates; r0 += G) {
      float fv[G];
#pragma unroll
      for (int j = 0; j < G; ++j)
        fv[j] = r0 + j < rates ? fr[(size_t)(r0 + j) * paths + p] : 0.0f;
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const int r = r0 + j;
        if (r < rates) {
          df /= 1.0f + tau.v[r] * fv[j];
          d[(size_t)(r + 1) * paths + p] = df;
        }
      }
    }
  }
}

extern "C" int lmm_discount_ratios(const float* d_rates, const float* h_taus,
                                     const int* h_alive, int paths, int steps,
                                     int rates, float* d_discounts,
                                     lmm_stream_t stream) {
  LMM_REQUIRE(rates >= 1 && rates <= kMaxRates && paths >= 0,
              "lmm_discount_ratios: bad sizes");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(d_rates && h_taus && d_discounts,
              "lmm_discount_ratios: null pointer");
  StepTab alive;
  int st = load_alive(h_alive, steps, rates, &alive);
  if (st) return st;
  FloatTab<kMaxRates> tau;
  for (int r = 0; r < rates; ++r) tau.v[r] = h_taus[r];
  const int block = 256;
  dim3 grid(grid_for(paths, block, 2), steps);
  discount_ratios_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(
      d_rates, d_discounts, paths, steps, rates, alive, tau);
  return check_launch("lmm_discount_ratios");
}

// coterminal annuity A_r = sum_{k>=r} tau_k P(T_s,T_{k+1})
// (gold/LMM_evolver_gold.h:494-522)
__global__ void annuities_kernel(const float* __restrict__ disc,
                                 float* __restrict__ ann, int paths, int rates,
                                 const __grid_constant__ StepTab alive,
                                 const __grid_constant__ FloatTab<kMaxRates> tau) {
  const int s = blockIdx.y;
  const int a = alive.v[s];
  const float* d = disc + (size_t)s * (rates + 1) * paths;
  float* o = ann + (size_t)s * rates * paths;
  constexpr int G = 8;  // rates whose loads are issued together
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    float x = 0.0f;
    for (int r0 = rates - 1; r0 >= a; r0 -= G) {
      float dv[G];
#pragma unroll
      for (int j = 0; j < G; ++j)
        dv[j] = r0 - j >= a ? d[(size_t)(r0 - j + 1) * paths + p] : 0.0f;
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const int r = r0 - j;
        if (r >= a) {
          x += tau.v[r] * dv[j];
          o[(size_t)r * paths + p] = x;
        }
      }
    }
  }
}

extern "C" int lmm_coterminal_annuities(const float* d_discounts,
                                          const float* h_taus,
                                          const int* h_alive, int paths,
                                          int steps, int rates,
                                          float* d_annuities,
                                          lmm_stream_t stream) {
  LMM_REQUIRE(rates >= 1 && rates <= kMaxRates && paths >= 0,
              "lmm_coterminal_annuities: bad sizes");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(d_discounts && h_taus && d_annuities,
              "lmm_coterminal_annuities: null pointer");
  StepTab alive;
  int st = load_alive(h_alive, steps, rates, &alive);
  if (st) return st;
  FloatTab<kMaxRates> tau;
  for (int r = 0; r < rates; ++r) tau.v[r] = h_taus[r];
  const int block = 256;
  dim3 grid(grid_for(paths, block, 2), steps);
  annuities_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(
      d_discounts, d_annuities, paths, rates, alive, tau);
  return check_launch("lmm_coterminal_annuities");
}

// coterminal swap rate SR_r = (P_r - P_n) / A_r (gold/LMM_evolver_gold.h:525-553)
__global__ void swap_rates_kernel(const float* __restrict__ disc,
                                  const float* __restrict__ ann,
                                  float* __restrict__ sr, int paths, int rates,
                                  const __grid_constant__ StepTab alive) {
  const int s = blockIdx.y;
  const int a = alive.v[s];
  const float* d = disc + (size_t)s * (rates + 1) * paths;
  const float* an = ann + (size_t)s * rates * paths;
  float* o = sr + (size_t)s * rates * paths;
  constexpr int G = 8;  // rates whose loads are issued together
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    const float dn = d[(size_t)rates * paths + p];
    for (int r0 = a; r0 < rates; r0 += G) {
      float dv[G], av[G];
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const bool ok = r0 + j < rates;
        dv[j] = ok ? d[(size_t)(r0 + j) * paths + p] : 0.0f;
        av[j] = ok ? an[(size_t)(r0 + j) * paths + p] : 1.0f;
      }
#pragma unroll
      for (int j = 0; j < G; ++j)
        if (r0 + j < rates) o[(size_t)(r0 + j) * paths + p] = (dv[j] - dn) / av[j];
    }
  }
}

extern "C" int lmm_coterminal_swap_rates(const float* d_discounts,
                                         const float* d_annuities,
                                         const int* h_alive, int paths,
                                         int steps, int rates,
                                         float* d_swap_rates,
                                         lmm_stream_t stream) {
  LMM_REQUIRE(rates >= 1 && rates <= kMaxRates && paths >= 0,
              "lmm_coterminal_swap_rates: bad sizes");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(d_discounts && d_annuities && d_swap_rates,
              "lmm_coterminal_swap_rates: null pointer");
  StepTab alive;
  int st = load_alive(h_alive, steps, rates, &alive);
  if (st) return st;
  const int block = 256;
  dim3 grid(grid_for(paths, block, 2), steps);
  swap_rates_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(
      d_discounts, d_annuities, d_swap_rates, paths, rates, alive);
  return check_launch("lmm_coterminal_swap_rates");
}

// swap rate between two rate indices on one step (gold/LMM_evolver_gold.h:556-585)
__global__ void swap_rate_kernel(const float* __restrict__ disc,
                                 float* __restrict__ out, int start, int end,
                                 int paths, int rates,
                                 const __grid_constant__ FloatTab<kMaxRates> tau) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    const float num = disc[(size_t)start * paths + p] -
                      disc[(size_t)end * paths + p];
    float den = 0.0f;
    for (int r = start; r < end; ++r)
      den += tau.v[r] * disc[(size_t)(r + 1) * paths + p];
    out[p] = num / den;
  }
}

extern "C" int lmm_swap_rate(const float* d_discounts, const float* h_taus,
                               int start_index, int end_index, int paths,
                               int step_for_offset_in, int step_for_offset_out,
                               int steps, int rates, float* d_swap_rate,
                               lmm_stream_t stream) {
  LMM_REQUIRE(rates >= 1 && rates <= kMaxRates && paths >= 0,
              "lmm_swap_rate: bad sizes");
  LMM_REQUIRE(0 <= start_index && start_index < end_index &&
                  end_index <= rates,
              "lmm_swap_rate: need 0 <= start < end <= rates");
  LMM_REQUIRE(step_for_offset_in >= 0 && step_for_offset_in < steps &&
                  step_for_offset_out >= 0 && step_for_offset_out < steps,
              "lmm_swap_rate: step offsets out of range");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(d_discounts && h_taus && d_swap_rate,
              "lmm_swap_rate: null pointer");
  FloatTab<kMaxRates> tau;
  for (int r = 0; r < rates; ++r) tau.v[r] = h_taus[r];
  const int block = 256;
  swap_rate_kernel<<<grid_for(paths, block, 4), block, 0,
                     (cudaStream_t)stream>>>(
      d_discounts + (size_t)step_for_offset_in * (rates + 1) * paths,
      d_swap_rate + (size_t)step_for_offset_out * paths, start_index,
      end_index, paths, rates, tau);
  return check_launch("lmm_swap_rate");
}

// spot numeraire N_0 = 1, N_r = N_{r-1} P(r-1,r-1)/P(r-1,r)
// (gold/LMM_evolver_gold.h:617-666)
__global__ void numeraires_kernel(const float* __restrict__ disc,
                                  float* __restrict__ num, int paths,
                                  int out_paths, int offset, int rates) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    float x = 1.0f;
    num[offset + p] = x;
    constexpr int G = 8;  // rates whose loads are issued together
    for (int r0 = 1; r0 < rates; r0 += G) {
      float a[G], b[G];
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const int r = r0 + j;
        const float* d = disc + (size_t)(r < rates ? r - 1 : 0) * (rates + 1) * paths;
        a[j] = r < rates ? d[(size_t)(r - 1) * paths + p] : 1.0f;
        b[j] = r < rates ? d[(size_t)r * paths + p] : 1.0f;
      }
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const int r = r0 + j;
        if (r < rates) {
          x = x * a[j] / b[j];
          num[(size_t)r * out_paths + offset + p] = x;
        }
      }
    }
  }
}

extern "C" int lmm_spot_numeraires(const float* d_discounts, int paths,
                                   int paths_for_output,
                                   int paths_offset_for_output, int rates,
                                   float* d_numeraires, lmm_stream_t stream) {
  LMM_REQUIRE(rates >= 1 && paths >= 0 && paths_offset_for_output >= 0 &&
                  paths_offset_for_output + paths <= paths_for_output,
              "lmm_spot_numeraires: bad sizes");
  if (paths == 0) return LMM_OK;
  LMM_REQUIRE(d_discounts && d_numeraires, "lmm_spot_numeraires: null pointer");
  const int block = 256;
  numeraires_kernel<<<grid_for(paths, block, 4), block, 0,
                      (cudaStream_t)stream>>>(d_discounts, d_numeraires, paths,
                                              paths_for_output,
                                              paths_offset_for_output, rates);
  return check_launch("lmm_spot_numeraires");
}

// Gathers: out[j][p] = all[step[j]][fwd[j]][p]  (gold/LMM_evolver_gold.h:645-694)
__global__ void extraction_kernel(const float* __restrict__ all,
                                  float* __restrict__ sel, int n, int paths,
                                  int rates,
                                  const __grid_constant__ StepTab fwd,
                                  const __grid_constant__ StepTab step) {
  const int j = blockIdx.y;
  const float* src =
      all + ((size_t)step.v[j] * rates + fwd.v[j]) * paths;
  float* dst = sel + (size_t)j * paths;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x)
    dst[p] = src[p];
}

static int extraction_launch(const float* d_all, const int* h_fwd,
                             const int* h_step, int n, int paths, int rates,
                             int steps_total, float* d_sel,
                             lmm_stream_t stream, const char* who) {
  LMM_REQUIRE(n >= 0 && n <= kMaxSteps && paths >= 0 && rates >= 1,
              "%s: bad sizes", who);
  if (n == 0 || paths == 0) return LMM_OK;
  LMM_REQUIRE(d_all && h_fwd && d_sel, "%s: null pointer", who);
  StepTab fwd, step;
  for (int j = 0; j < n; ++j) {
    LMM_REQUIRE(h_fwd[j] >= 0 && h_fwd[j] < rates,
                "%s: forward index out of range", who);
    fwd.v[j] = h_fwd[j];
    step.v[j] = h_step ? h_step[j] : j;
    LMM_REQUIRE(step.v[j] >= 0 && (steps_total < 0 || step.v[j] < steps_total),
                "%s: step index out of range", who);
  }
  const int block = 256;
  dim3 grid(grid_for(paths, block, 1), n);
  extraction_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(
      d_all, d_sel, n, paths, rates, fwd, step);
  return check_launch(who);
}

extern "C" int lmm_forward_extraction(const float* d_all,
                                      const int* h_forward_indices, int paths,
                                      int steps, int rates, float* d_select,
                                      lmm_stream_t stream) {
  return extraction_launch(d_all, h_forward_indices, nullptr, steps, paths,
                           rates, steps, d_select, stream,
                           "lmm_forward_extraction");
}

extern "C" int lmm_forward_extraction_steps(const float* d_all,
                                            const int* h_forward_indices,
                                            const int* h_step_indices, int n,
                                            int paths, int rates,
                                            float* d_select,
                                            lmm_stream_t stream) {
  LMM_REQUIRE(h_step_indices != nullptr,
              "lmm_forward_extraction_steps: null step indices");
  return extraction_launch(d_all, h_forward_indices, h_step_indices, n, paths,
                           rates, -1, d_select, stream,
                           "lmm_forward_extraction_steps");
}

__global__ void numeraire_extraction_kernel(const float* __restrict__ all,
                                            float* __restrict__ some,
                                            int paths_in, int paths_out,
                                            int offset,
                                            const __grid_constant__ StepTab ex) {
  const int j = blockIdx.y;
  const float* src = all + (size_t)ex.v[j] * paths_in;
  float* dst = some + (size_t)j * paths_out + offset;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths_in;
       p += gridDim.x * blockDim.x)
    dst[p] = src[p];
}

extern "C" int lmm_numeraire_extraction(const float* d_all, float* d_some,
                                        int paths_in, int paths_out,
                                        int offset_for_output, int rates,
                                        int n_exercise,
                                        const int* h_exercise_indices,
                                        lmm_stream_t stream) {
  LMM_REQUIRE(n_exercise >= 0 && n_exercise <= kMaxSteps && paths_in >= 0 &&
                  offset_for_output >= 0 &&
                  offset_for_output + paths_in <= paths_out,
              "lmm_numeraire_extraction: bad sizes");
  if (n_exercise == 0 || paths_in == 0) return LMM_OK;
  LMM_REQUIRE(d_all && d_some && h_exercise_indices,
              "lmm_numeraire_extraction: null pointer");
  StepTab ex;
  for (int j = 0; j < n_exercise; ++j) {
    LMM_REQUIRE(h_exercise_indices[j] >= 0 && h_exercise_indices[j] < rates,
                "lmm_numeraire_extraction: exercise index out of range");
    ex.v[j] = h_exercise_indices[j];
  }
  const int block = 256;
  dim3 grid(grid_for(paths_in, block, 1), n_exercise);
  numeraire_extraction_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(
      d_all, d_some, paths_in, paths_out, offset_for_output, ex);
  return check_launch("lmm_numeraire_extraction");
}
