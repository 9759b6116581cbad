// evolve_all.cu — the fused predictor-corrector evolution with full rate
// tensors as output: the B200 form of the reference's LMM_evolver_pc_all_gpu
// (LMM_evolver_all.cu:1322-1480, kernel :506-747), which evolves every path
// through all steps in one launch and writes the rates, log-rates and
// discount ratios of every step.
//
// One thread per path, CTA of 128 paths.  The CTA's log-rates stay in
// shared memory ([rate][thread]) between steps, the step's pseudo-root rows
// (padded to a multiple of 4 factors for 16-byte loads) and fixed drifts are
// staged in shared memory once per step, and each rate uses pc_rate, the
// rate step of the pricing kernels, so the tensors written here are those
// kernels' own forward rates.  The kernel is bound by its HBM writes
// (3 x steps x rates x 4 B per path) at large path counts.
#include "lmm_common.cuh"
#include "lmm_device.cuh"
#include "pc_step.cuh"

#include <cmath>
#include <cstring>

using namespace lmm;

namespace {

constexpr int kAllBlock = 128;

struct AliveConst {
  int alive[kMaxSteps];
};

// variates: layout 1 = [step][factor][path] (the bridge output, the
// reference's transposed variates); layout 0 = [step][path][factor].
// Writes rates / log-rates [step][rate][path] and, when disc is not null,
// discount ratios [step][rate + 1][path] for rates r >= alive[s] (entry
// alive[s] of the discounts is 1), as the reference kernel does; entries
// below the alive index are not written.
template <int FT>
__global__ void __launch_bounds__(kAllBlock)
    evolve_all_kernel(int paths, int steps, const float* __restrict__ Z, int z_layout,
                      const float* __restrict__ A, const float* __restrict__ fixed,
                      const __grid_constant__ ModelConst mc,
                      const __grid_constant__ AliveConst al, float* __restrict__ rates_out,
                      float* __restrict__ lrates_out, float* __restrict__ disc_out) {
  constexpr int FM = FPad<FT>::FM;
  constexpr int FP = FPad<FT>::FP;
  const int F = FT > 0 ? FT : mc.F;
  const int n = mc.n;
  const int T = blockDim.x, tid = threadIdx.x;
  extern __shared__ __align__(16) float sm[];
  float* As = sm;                    // [n][FP]
  float* fx = As + n * FP;           // [n] (+ pad)
  float* lfs = fx + ((n + 3) & ~3);  // [n][T]
  const int p = blockIdx.x * T + tid;
  const bool valid = p < paths;
  const size_t P = (size_t)paths;
  for (int r = 0; r < n; ++r) lfs[r * T + tid] = mc.logf0[r];
  for (int s = 0; s < steps; ++s) {
    __syncthreads();
    for (int i = tid; i < n * FP; i += T) {
      const int r = i / FP, f = i - r * FP;
      As[i] = f < F ? __ldg(A + ((size_t)s * n + r) * F + f) : 0.0f;
    }
    for (int i = tid; i < n; i += T) fx[i] = __ldg(fixed + (size_t)s * n + i);
    __syncthreads();
    if (!valid) continue;
    float z[FP];
#pragma unroll
    for (int f = 0; f < FP; ++f) {
      if (f < F) {
        const size_t idx = z_layout == 1 ? ((size_t)s * F + f) * P + p
                                         : ((size_t)s * P + p) * F + f;
        z[f] = __ldg(Z + idx);
      } else {
        z[f] = 0.0f;
      }
    }
    float2 w[FP / 2], v[FP / 2];
    step_start<FP>(z, w, v);
    const int a = al.alive[s];
    float* ro = rates_out + (size_t)s * n * P + p;
    float* lo = lrates_out + (size_t)s * n * P + p;
    float* dso = disc_out ? disc_out + (size_t)s * (n + 1) * P + p : nullptr;
    float Pd = 1.0f;
    if (dso) dso[(size_t)a * P] = 1.0f;
    for (int r = a; r < n; ++r) {
      const float tau = mc.tau[r];
      float g, gp;
      bool capped;
      const float lf = pc_rate<FM, FP>(lfs[r * T + tid], mc.l2tau[r], mc.c0[r], fx[r],
                                       As + r * FP, w, v, mc.cutoff, g, gp, capped);
      lfs[r * T + tid] = lf;
      const float f = exp_ftz(lf) - mc.disp[r];
      lo[(size_t)r * P] = lf;
      ro[(size_t)r * P] = f;
      if (dso) {
        Pd = Pd / (1.0f + tau * f);
        dso[(size_t)(r + 1) * P] = Pd;
      }
    }
  }
}

}  // namespace

extern "C" int lmm_evolve_pc_all(const float* h_initial_rates, const float* h_taus,
                                 const float* h_displacements, const float* d_variates,
                                 int variates_layout, const float* d_A,
                                 const float* d_fixed_drifts, const int* h_alive, int paths,
                                 int factors, int steps, int rates, float cutoff,
                                 float* d_rates, float* d_log_rates, float* d_discounts,
                                 lmm_stream_t stream) {
  LMM_REQUIRE(rates >= 1 && rates <= kMaxRates, "lmm_evolve_pc_all: rates must be in [1,%d]",
              kMaxRates);
  LMM_REQUIRE(steps >= 1 && steps <= kMaxSteps, "lmm_evolve_pc_all: steps must be in [1,%d]",
              kMaxSteps);
  LMM_REQUIRE(factors >= 1 && factors <= kMaxFactors,
              "lmm_evolve_pc_all: factors must be in [1,%d]", kMaxFactors);
  LMM_REQUIRE(paths >= 1, "lmm_evolve_pc_all: paths < 1");
  LMM_REQUIRE(variates_layout == 0 || variates_layout == 1,
              "lmm_evolve_pc_all: variates layout must be 0 or 1");
  LMM_REQUIRE(h_initial_rates && h_taus && h_displacements && h_alive && d_variates && d_A &&
                  d_fixed_drifts && d_rates && d_log_rates,
              "lmm_evolve_pc_all: null pointer");
  ModelConst mc;
  memset(&mc, 0, sizeof(mc));
  mc.n = rates;
  mc.F = factors;
  mc.cutoff = cutoff;
  for (int r = 0; r < rates; ++r) {
    LMM_REQUIRE(h_taus[r] > 0.0f, "lmm_evolve_pc_all: tau must be positive");
    LMM_REQUIRE(h_initial_rates[r] + h_displacements[r] > 0.0f,
                "lmm_evolve_pc_all: displaced initial rate must be positive");
    mc.tau[r] = h_taus[r];
    mc.disp[r] = h_displacements[r];
    mc.logf0[r] = logf(h_initial_rates[r] + h_displacements[r]);
    mc.c0[r] = 1.0f - h_displacements[r] * h_taus[r];
    mc.l2tau[r] = (float)std::log2((double)h_taus[r]);
  }
  AliveConst al;
  int last = 0;
  for (int s = 0; s < steps; ++s) {
    LMM_REQUIRE(h_alive[s] >= last && h_alive[s] < rates,
                "lmm_evolve_pc_all: alive indices must be non-decreasing in [0,rates)");
    last = al.alive[s] = h_alive[s];
  }
  const int FPd = (factors == 3 || factors == 5 || factors == 10 || factors == 15)
                      ? ((factors + 3) & ~3)
                      : ((kMaxFactors + 3) & ~3);
  const size_t smem =
      ((size_t)rates * FPd + ((rates + 3) & ~3) + (size_t)rates * kAllBlock) * sizeof(float);
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = div_up(paths, kAllBlock);
  auto go = [&](auto kern) -> int {
    int st = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem),
                        "lmm_evolve_pc_all: smem attribute");
    if (st) return st;
    kern<<<grid, kAllBlock, smem, s>>>(paths, steps, d_variates, variates_layout, d_A,
                                       d_fixed_drifts, mc, al, d_rates, d_log_rates,
                                       d_discounts);
    return check_launch("evolve_all_kernel");
  };
  switch (factors) {
    case 3: return go(evolve_all_kernel<3>);
    case 5: return go(evolve_all_kernel<5>);
    case 10: return go(evolve_all_kernel<10>);
    case 15: return go(evolve_all_kernel<15>);
    default: return go(evolve_all_kernel<0>);
  }
}
