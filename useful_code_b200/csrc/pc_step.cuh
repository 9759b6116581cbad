// pc_step.cuh — the predictor-corrector rate step shared by every kernel
// that evolves forward rates path by path: the fused pricing passes
// (fused_kernels.cuh), the adjoint's recompute, the Andersen–Broadie inner
// paths and the full-tensor evolution of lmm_evolve_pc_all.  Keeping one
// definition makes all of them follow exactly the same arithmetic.
#pragma once
#include "lmm_common.cuh"
#include "lmm_device.cuh"

namespace lmm {

// Model constants passed by value as a kernel parameter.
struct ModelConst {
  int n, F, scr_dims;
  float cutoff;
  float tau[kMaxRates], disp[kMaxRates], logf0[kMaxRates];
  float c0[kMaxRates];  // 1 - d_r tau_r: g = F tau / (c0 + F tau)
};

// Padding of the per-step pseudo-root rows held in shared memory: FT =
// number of factors (compile time), 0 = generic <= kMaxFactors.
template <int FT>
struct FPad {
  static constexpr int FM = FT > 0 ? FT : kMaxFactors;
  static constexpr int FP = (FM + 3) & ~3;
};

// One rate r of one predictor-corrector step: from the log-rate lf at the
// start of the step, the factor sums e_ (start rates) and ep (predicted
// rates) of rates s..r-1, the pseudo-root row Arow (FP floats, shared
// memory, 16-byte aligned), the fixed drift and the step's normals z,
// returns the new (capped) log-rate and updates e_ and ep.  g and gp are the
// drift factors F tau / (1 + f tau) of the start and predicted rates,
// capped whether the cap applied.  Shared by the pricing kernels and the
// adjoint, so both follow exactly the same path.
// q = 1 / (1 + tau f) of the start rate (the reciprocal inside g) is also
// returned: it is the rate's factor in the discount ratios of the previous
// date.
template <int FM, int FP>
__device__ __forceinline__ float pc_rate(float lf, float tau, float c0, float fxr,
                                         const float* Arow, const float2 (&z)[FP / 2],
                                         float2 (&e_)[FP / 2], float2 (&ep)[FP / 2],
                                         float cutoff, float& g, float& gp, float& q,
                                         bool& capped) {
  // The drift of rate r sums over rates s..r inclusive:
  //   mu_r = sum_f A_rf (e_f + g_r A_rf) = A_r . e + g_r |A_r|^2,
  // with |A_r|^2 = -2 x the fixed drift.  The dot products with the sums of
  // the earlier rates (and the correlated increment) do not wait for this
  // rate's exp and reciprocal, so they overlap that latency.  Factors are
  // held in pairs (f = 2k, 2k + 1) and every product-sum runs as one packed
  // FP32x2 FMA per pair: the even and odd factors accumulate in the two
  // halves, each with the rounding of a scalar FMA.
  constexpr int NP = (FM + 1) / 2;  // pairs that hold factors
  const float4* a4 = reinterpret_cast<const float4*>(Arow);
  float2 a2[FP / 2];
#pragma unroll
  for (int k = 0; k < FP / 4; ++k) {
    const float4 a = a4[k];
    a2[2 * k] = make_float2(a.x, a.y);
    a2[2 * k + 1] = make_float2(a.z, a.w);
  }
  float2 d = make_float2(0.0f, 0.0f), dW = d, pp = d;
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    d = __ffma2_rn(a2[k], e_[k], d);
    dW = __ffma2_rn(a2[k], z[k], dW);
    pp = __ffma2_rn(a2[k], ep[k], pp);
  }
  const float nA2 = -2.0f * fxr;
  const float Fr = exp_ftz(lf) * tau;
  q = rcp_ftz(c0 + Fr);
  g = Fr * q;
  const float mu = fmaf(g, nA2, d.x + d.y);
  lf += mu + ((dW.x + dW.y) + fxr);
  const float Fp = exp_ftz(lf) * tau;
  gp = Fp * rcp_ftz(c0 + Fp);
  const float mp = fmaf(gp, nA2, pp.x + pp.y);
  const float2 g2 = make_float2(g, g), gp2 = make_float2(gp, gp);
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    e_[k] = __ffma2_rn(a2[k], g2, e_[k]);
    ep[k] = __ffma2_rn(a2[k], gp2, ep[k]);
  }
  lf += 0.5f * (mp - mu);
  capped = lf > cutoff;
  return fminf(lf, cutoff);
}

template <int FM, int FP>
__device__ __forceinline__ float pc_rate(float lf, float tau, float c0, float fxr,
                                         const float* Arow, const float2 (&z)[FP / 2],
                                         float2 (&e_)[FP / 2], float2 (&ep)[FP / 2],
                                         float cutoff, float& g, float& gp, bool& capped) {
  float q;
  return pc_rate<FM, FP>(lf, tau, c0, fxr, Arow, z, e_, ep, cutoff, g, gp, q, capped);
}

// Step normals in factor pairs for pc_rate.
template <int FP>
__device__ __forceinline__ void pair_normals(const float (&z)[FP], float2 (&z2)[FP / 2]) {
#pragma unroll
  for (int k = 0; k < FP / 2; ++k) z2[k] = make_float2(z[2 * k], z[2 * k + 1]);
}

}  // namespace lmm
