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
  float l2tau[kMaxRates];  // log2 tau_r: F tau = 2^(log F log2 e + log2 tau)
};

// Padding of the per-step pseudo-root rows held in shared memory: FT =
// number of factors (compile time), 0 = generic <= kMaxFactors.
template <int FT>
struct FPad {
  static constexpr int FM = FT > 0 ? FT : kMaxFactors;
  static constexpr int FP = (FM + 3) & ~3;
};

// One rate r of one predictor-corrector step.  The spot drift of rate r over
// the rates s..r of the step is mu_r = A_r . e_{r-1} + g_r |A_r|^2 with the
// prefix e_{r-1} = sum_{j<r} g_j A_j and |A_r|^2 = -2 x the fixed drift; the
// corrector's drift uses the predicted rates' prefix ep the same way.  The
// predictor-corrector step of the reference (LMM_evolver_all.cu:615-744,
// gold/LMM_evolver_gold.h:315-387)
//   lp = lf + mu_r + A_r . z + fixed_r,   lf' = lp + (mp_r - mu_r) / 2
// needs three products of A_r with factor vectors (e, z, ep).  Here two
// running vectors are kept instead,
//   w = z + e_{r-1},   v = ep_{r-1} - e_{r-1},
// so that lp = lf + A_r . w + g_r |A_r|^2 + fixed_r and
// lf' = lp + (A_r . v + (gp_r - g_r) |A_r|^2) / 2: two dot products and two
// updates per rate (w += g_r A_r, v += (gp_r - g_r) A_r) in place of three
// and two, the same quantities with other FP32 roundings.  Both dot
// products depend only on the earlier rates, so they overlap this rate's
// exp and reciprocal.  Factors are held in pairs (f = 2k, 2k + 1) and every
// product-sum runs as one packed FP32x2 FMA per pair: the even and odd
// factors accumulate in the two halves, each with the rounding of a scalar
// FMA.  exp(x) tau is formed as 2^(x log2 e + log2 tau) (l2tau = log2 tau).
// Returns the new (capped) log-rate; g and gp are the drift factors
// F tau / (1 + f tau) of the start and predicted rates (F = f + d, c0 =
// 1 - d tau), q = 1 / (1 + tau f) of the start rate (its factor in the
// discount ratios of the previous date), capped whether the cap applied.
// Shared by the pricing kernels, the adjoint's recompute, the
// Andersen–Broadie inner paths and lmm_evolve_pc_all, so all follow exactly
// the same path.
template <int FM, int FP>
__device__ __forceinline__ float pc_rate(float lf, float l2tau, float c0, float fxr,
                                         const float* Arow, float2 (&w)[FP / 2],
                                         float2 (&v)[FP / 2], float cutoff, float& g, float& gp,
                                         float& q, bool& capped) {
  constexpr int NP = (FM + 1) / 2;  // pairs that hold factors
  constexpr float kLog2e = 1.44269504088896341f;
  const float4* a4 = reinterpret_cast<const float4*>(Arow);
  float2 a2[FP / 2];
#pragma unroll
  for (int k = 0; k < FP / 4; ++k) {
    const float4 a = a4[k];
    a2[2 * k] = make_float2(a.x, a.y);
    a2[2 * k + 1] = make_float2(a.z, a.w);
  }
  float2 dw = make_float2(0.0f, 0.0f), dv = dw;
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    dw = __ffma2_rn(a2[k], w[k], dw);
    dv = __ffma2_rn(a2[k], v[k], dv);
  }
  const float nA2 = -2.0f * fxr;
  const float Fr = ex2_ftz(fmaf(lf, kLog2e, l2tau));
  q = rcp_ftz(c0 + Fr);
  g = Fr * q;
  lf += fmaf(g, nA2, dw.x + dw.y) + fxr;
  const float Fp = ex2_ftz(fmaf(lf, kLog2e, l2tau));
  gp = Fp * rcp_ftz(c0 + Fp);
  const float dg = gp - g;
  lf += 0.5f * fmaf(dg, nA2, dv.x + dv.y);
  const float2 g2 = make_float2(g, g), dg2 = make_float2(dg, dg);
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    w[k] = __ffma2_rn(a2[k], g2, w[k]);
    v[k] = __ffma2_rn(a2[k], dg2, v[k]);
  }
  capped = lf > cutoff;
  return fminf(lf, cutoff);
}

template <int FM, int FP>
__device__ __forceinline__ float pc_rate(float lf, float l2tau, float c0, float fxr,
                                         const float* Arow, float2 (&w)[FP / 2],
                                         float2 (&v)[FP / 2], float cutoff, float& g, float& gp,
                                         bool& capped) {
  float q;
  return pc_rate<FM, FP>(lf, l2tau, c0, fxr, Arow, w, v, cutoff, g, gp, q, capped);
}

// Running vectors of pc_rate at the start of a step: w = the step's normals
// (in factor pairs), v = 0.
template <int FP>
__device__ __forceinline__ void step_start(const float (&z)[FP], float2 (&w)[FP / 2],
                                           float2 (&v)[FP / 2]) {
#pragma unroll
  for (int k = 0; k < FP / 2; ++k) {
    w[k] = make_float2(z[2 * k], z[2 * k + 1]);
    v[k] = make_float2(0.0f, 0.0f);
  }
}

}  // namespace lmm
