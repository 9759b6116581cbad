// greeks_kernels.cuh — pathwise adjoint of the fused pricing pass (included
// by pipeline.cu after fused_kernels.cuh).
//
// The price with a frozen exercise rule is V = P(0,T_0) mean_p Phi_p, where
// Phi_p is the sum of the path's numeraire-deflated flows up to its
// exercise step.  The exercise step of each path is recorded in the forward
// pass and held fixed (the pathwise method: the decision boundary has
// measure zero), so Phi_p is a smooth function of the initial log-rates and
// of the pseudo-roots A_s along the path.  The adjoint runs the steps
// backwards.  Log-rate checkpoints every k steps come from the recording
// forward pass; a segment kernel recomputes the start-of-step log-rates of
// k steps from a checkpoint, then one reverse kernel per step:
//   * recomputes the step (pc_rate, the pricing kernels' own arithmetic):
//     drift factors g (start) and gp (predicted), new log-rates ln;
//   * adds the adjoint of the step's flow (exercise value, coupon, caplet)
//     and of the numeraire factor (1 + tau_s f_s), which scales every later
//     flow, to a_r = dPhi/dln_r (zero where the log-rate cap applied);
//   * reverses the predictor-corrector step in one descending sweep:
//       L_r     = a_r + gp_r (1 - gp_r) sum_f A_rf h_f(r),
//                 h_f(r) = sum_{j >= r} a_j A_jf / 2     (adjoint of lp_r)
//       mubar_r = L_r - a_r / 2                          (adjoint of mu_r)
//       lam_r   = L_r + g_r (1 - g_r) sum_f A_rf k_f(r),
//                 k_f(r) = sum_{j >= r} mubar_j A_jf     (adjoint of lf_r)
//     with G'(x) = G (1 - G) for G(x) = tau e^x / (c0 + tau e^x);
//   * writes the per-path vectors whose sums over paths give dV/dA_s:
//       M_rj = sum_p (mubar_r g_j + a_r gp_j / 2)        (j <= r)
//       N_rf = sum_p L_r z_f,   l_r = sum_p L_r
//     dV/dA_s[k][f] = sum_{j<=k} M_kj A_jf + sum_{i>=k} M_ik A_if + N_kf
//                     - A_kf l_k
//     (mu_r = sum_{j<=r} C_rj g_j with C = A A^T, dW = A z, fixed drift
//     -|A_r|^2 / 2).  M and N are path contractions on the tensor cores
//     (lmm_path_gram).
// Deltas: dV/df0_r = P(0,T_0) mean_p lam_r(0) / (f0_r + d_r), plus the
// derivative of P(0,T_0) = 1 / (1 + f0_0 T_0) for r = 0.
#pragma once
#include "fused_kernels.cuh"

namespace lmm {

// Recompute the start-of-step log-rates of steps [s0, s1) from checkpoint
// log-rates at s0 (ckpt [n][P], rates r >= s0) and the numeraire there;
// writes seg_lf[(s - s0)][r][p] (r >= s) and seg_N[(s - s0)][p].
template <int FT>
__global__ void __launch_bounds__(128, 4)
    greeks_segment_kernel(int paths, int s0, int s1, const float* __restrict__ Z,
                          const float* __restrict__ A,
                          const float* __restrict__ fixed,
                          const __grid_constant__ ModelConst mc,
                          const float* __restrict__ ckpt,
                          const float* __restrict__ ckptN,
                          const int* __restrict__ ex_step,
                          float* __restrict__ seg_lf, float* __restrict__ seg_N) {
  constexpr int FM = FPad<FT>::FM;
  constexpr int FP = FPad<FT>::FP;
  const int F = FT > 0 ? FT : mc.F;
  const int n = mc.n;
  const int T = blockDim.x, tid = threadIdx.x;
  extern __shared__ __align__(16) float sm[];
  float* As = sm;
  float* fx = As + n * FP;
  float* lfs = fx + ((n + 3) & ~3);
  const int p = blockIdx.x * T + tid;
  const bool valid = p < paths;
  const int stop = valid ? ex_step[p] : -1;
  for (int r = s0; r < n; ++r)
    lfs[r * T + tid] = valid ? ckpt[(size_t)r * paths + p] : 0.0f;
  float N = valid ? ckptN[p] : 1.0f, f_first = 0.0f;
  for (int s = s0; s < s1; ++s) {
    __syncthreads();
    for (int i = tid; i < n * FP; i += T) {
      const int r = i / FP, f = i - r * FP;
      As[i] = f < F ? __ldg(A + ((size_t)s * n + r) * F + f) : 0.0f;
    }
    for (int i = tid; i < n; i += T) fx[i] = __ldg(fixed + (size_t)s * n + i);
    __syncthreads();
    if (!valid || s > stop) continue;
    if (s > s0) N = N * (1.0f + mc.tau[s - 1] * f_first);
    const int k = s - s0;
    for (int r = s; r < n; ++r)
      seg_lf[((size_t)k * n + r) * paths + p] = lfs[r * T + tid];
    seg_N[(size_t)k * paths + p] = N;
    float z[FP];
#pragma unroll
    for (int f = 0; f < FP; ++f)
      z[f] = (f < F) ? __ldg(Z + ((size_t)s * F + f) * paths + p) : 0.0f;
    float e_[FP], ep[FP];
#pragma unroll
    for (int f = 0; f < FP; ++f) e_[f] = ep[f] = 0.0f;
    for (int r = s; r < n; ++r) {
      float g, gp;
      bool capped;
      const float lf = pc_rate<FM, FP>(lfs[r * T + tid], mc.tau[r], mc.c0[r], fx[r],
                                       As + r * FP, z, e_, ep, mc.cutoff, g, gp, capped);
      lfs[r * T + tid] = lf;
      if (r == s) f_first = __expf(lf) - mc.disp[r];
    }
  }
}

// Buffers of one reverse step (all [rows][paths] with paths contiguous).
struct GreeksStepBufs {
  float* lam;     // [n][P] adjoint of the log-rates (in: end of step, out: start)
  double* later;  // [P] sum of the flows after the step (deflated)
  float* X;       // [n][2P]: mubar | a/2
  float* Y;       // [n][2P]: g | gp
  float* Lv;      // [n][P]: L
  float* Zb;      // [F+1][P]: z | 1
};

// Reverse of step s for every path (one launch per step, steps descending).
template <int FT>
__global__ void __launch_bounds__(64)
    greeks_reverse_kernel(int paths, int s, const float* __restrict__ Z,
                          const float* __restrict__ A,
                          const float* __restrict__ fixed,
                          const __grid_constant__ ModelConst mc,
                          const __grid_constant__ ProductConst pc,
                          const float* __restrict__ lf_start,
                          const float* __restrict__ N_start,
                          const int* __restrict__ ex_step,
                          const GreeksStepBufs b) {
  constexpr int FM = FPad<FT>::FM;
  constexpr int FP = FPad<FT>::FP;
  const int F = FT > 0 ? FT : mc.F;
  const int n = mc.n;
  const int T = blockDim.x, tid = threadIdx.x;
  extern __shared__ __align__(16) float sm[];
  float* As = sm;                    // [n][FP]
  float* fx = As + n * FP;           // [n] (+ pad)
  float* gs = fx + ((n + 3) & ~3);   // [n][T] g
  float* gps = gs + n * T;           // [n][T] gp
  float* lns = gps + n * T;          // [n][T] new log-rates
  for (int i = tid; i < n * FP; i += T) {
    const int r = i / FP, f = i - r * FP;
    As[i] = f < F ? __ldg(A + ((size_t)s * n + r) * F + f) : 0.0f;
  }
  for (int i = tid; i < n; i += T) fx[i] = __ldg(fixed + (size_t)s * n + i);
  __syncthreads();
  const int p = blockIdx.x * T + tid;
  if (p >= paths) return;
  const size_t P = (size_t)paths, P2 = 2 * (size_t)paths;
  const int stop = ex_step[p];
  // a path contributes at step s if it is still running there and has a
  // flow at or after s (a swaption only at its exercise step)
  bool active = s <= stop && s < n;
  if (pc.kind == LMM_PRODUCT_SWAPTION && stop >= n) active = false;
  if (!active) {
    for (int r = 0; r < n; ++r) {
      b.X[r * P2 + p] = 0.0f;
      b.X[r * P2 + P + p] = 0.0f;
      b.Y[r * P2 + p] = 0.0f;
      b.Y[r * P2 + P + p] = 0.0f;
      b.Lv[r * P + p] = 0.0f;
      if (r >= s) b.lam[r * P + p] = 0.0f;
    }
    for (int f = 0; f <= F; ++f) b.Zb[f * P + p] = 0.0f;
    return;
  }
  float z[FP];
#pragma unroll
  for (int f = 0; f < FP; ++f)
    z[f] = (f < F) ? __ldg(Z + ((size_t)s * F + f) * paths + p) : 0.0f;
  const float N = N_start[p];
  // ---- pass A: recompute the step and the curve at T_s ----
  float e_[FP], ep[FP];
#pragma unroll
  for (int f = 0; f < FP; ++f) e_[f] = ep[f] = 0.0f;
  float Prun = 1.0f, ann = 0.0f, P1 = 1.0f, f_s = 0.0f;
  for (int r = s; r < n; ++r) {
    float g, gp;
    bool capped;
    const float ln = pc_rate<FM, FP>(lf_start[r * P + p], mc.tau[r], mc.c0[r], fx[r],
                                     As + r * FP, z, e_, ep, mc.cutoff, g, gp, capped);
    gs[r * T + tid] = g;
    gps[r * T + tid] = gp;
    lns[r * T + tid] = capped ? __int_as_float(0x7fc00000) : ln;  // NaN marks the cap
    const float fn = __expf(ln) - mc.disp[r];
    if (r == s) f_s = fn;
    Prun = __fdividef(Prun, 1.0f + mc.tau[r] * fn);
    ann += mc.tau[r] * Prun;
    if (r == s) P1 = Prun;
  }
  const float Pn = Prun;
  // ---- the flow at step s and its derivative with respect to f_s ----
  const int e = pc.ex_index[s];
  const bool is_ex = (s == stop) && (e >= 0) && pc.kind != LMM_PRODUCT_EUROPEAN;
  const float tau_s = mc.tau[s];
  const float invN = 1.0f / N;
  float term = 0.0f;      // flow / N at step s
  float dterm_fs = 0.0f;  // d(term)/d f_s from the flows that depend on f_s only
  bool swaption_ex = false;
  if (pc.kind == LMM_PRODUCT_EUROPEAN) {
    const float cap = tau_s * fmaxf(f_s - pc.cap_strike, 0.0f);
    const float swp = tau_s * (f_s - pc.strike) * pc.pay_receive;
    term = (cap + swp) * P1 * invN;
    const float dv = tau_s * ((f_s > pc.cap_strike ? 1.0f : 0.0f) + pc.pay_receive);
    dterm_fs = (dv * P1 - (cap + swp) * P1 * tau_s * P1) * invN;
  } else if (pc.kind == LMM_PRODUCT_CANCELLABLE_SWAP) {
    if (!is_ex) {
      const float c = tau_s * (f_s - pc.strike) * pc.pay_receive;
      term = c * P1 * invN;
      dterm_fs = (tau_s * pc.pay_receive * P1 - c * P1 * tau_s * P1) * invN;
    }
  } else if (is_ex) {
    const float v = (1.0f - Pn) - pc.strike * ann;
    if (v > 0.0f) {
      term = v * invN;
      swaption_ex = true;
    }
  }
  const double later = b.later[p];
  // numeraire factor (1 + tau_s f_s) divides every later flow
  dterm_fs += -(float)later * tau_s / (1.0f + tau_s * f_s);
  b.later[p] = later + (double)term;
  // ---- pass C: descending sweep ----
  float h[FP], kk[FP];
#pragma unroll
  for (int f = 0; f < FP; ++f) h[f] = kk[f] = 0.0f;
  float Pr = Pn, ann_suf = 0.0f;
  for (int r = n - 1; r >= s; --r) {
    const float ln_raw = lns[r * T + tid];
    const bool capped = ln_raw != ln_raw;
    const float ln = capped ? mc.cutoff : ln_raw;
    const float Fd = __expf(ln);  // f_r + d_r = df_r / dln_r
    const float f_r = Fd - mc.disp[r];
    const float tr = mc.tau[r];
    const float onep = 1.0f + tr * f_r;
    // Pr = P(T_s, T_{r+1}); ann_suf = sum_{k >= r} tau_k P(T_s, T_{k+1})
    ann_suf += tr * Pr;
    float dphi_df = 0.0f;
    if (swaption_ex) dphi_df = tr / onep * (Pn + pc.strike * ann_suf) * invN;
    if (r == s) dphi_df += dterm_fs;
    const float lam_in = (r > s) ? b.lam[r * P + p] : 0.0f;
    const float a = capped ? 0.0f : lam_in + dphi_df * Fd;
    const float g = gs[r * T + tid], gp = gps[r * T + tid];
    const float4* a4 = reinterpret_cast<const float4*>(As + r * FP);
    float S1 = 0.0f;
#pragma unroll
    for (int q = 0; q < FP / 4; ++q) {
      const float4 av4 = a4[q];
      const float av[4] = {av4.x, av4.y, av4.z, av4.w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int f = 4 * q + u;
        if (f < FM) {
          h[f] += 0.5f * a * av[u];
          S1 += av[u] * h[f];
        }
      }
    }
    const float L = a + gp * (1.0f - gp) * S1;
    const float mubar = L - 0.5f * a;
    float S2 = 0.0f;
#pragma unroll
    for (int q = 0; q < FP / 4; ++q) {
      const float4 av4 = a4[q];
      const float av[4] = {av4.x, av4.y, av4.z, av4.w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int f = 4 * q + u;
        if (f < FM) {
          kk[f] += mubar * av[u];
          S2 += av[u] * kk[f];
        }
      }
    }
    b.lam[r * P + p] = L + g * (1.0f - g) * S2;
    b.X[r * P2 + p] = mubar;
    b.X[r * P2 + P + p] = 0.5f * a;
    b.Y[r * P2 + p] = g;
    b.Y[r * P2 + P + p] = gp;
    b.Lv[r * P + p] = L;
    Pr = Pr * onep;  // P(T_s, T_r)
  }
  for (int r = 0; r < s; ++r) {
    b.X[r * P2 + p] = 0.0f;
    b.X[r * P2 + P + p] = 0.0f;
    b.Y[r * P2 + p] = 0.0f;
    b.Y[r * P2 + P + p] = 0.0f;
    b.Lv[r * P + p] = 0.0f;
  }
#pragma unroll
  for (int f = 0; f < FP; ++f)
    if (f < F) b.Zb[f * P + p] = z[f];
  b.Zb[(size_t)F * P + p] = 1.0f;
}

// dV/dA_s from the step's path contractions M [n][n] and NL [n][F+1]
// (already scaled by P(0,T_0) / paths); rows below s are zero.
__global__ void greeks_abar_kernel(int n, int F, int s, const float* __restrict__ A,
                                   const double* __restrict__ M,
                                   const double* __restrict__ NL,
                                   double* __restrict__ abar) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * F) return;
  const int k = idx / F, f = idx - k * F;
  const float* As = A + (size_t)s * n * F;
  double v = 0.0;
  if (k >= s) {
    for (int j = s; j <= k; ++j) v += M[(size_t)k * n + j] * (double)As[j * F + f];
    for (int i = k; i < n; ++i) v += M[(size_t)i * n + k] * (double)As[i * F + f];
    v += NL[(size_t)k * (F + 1) + f] - (double)As[k * F + f] * NL[(size_t)k * (F + 1) + F];
  }
  abar[(size_t)s * n * F + idx] = v;
}

// Price, deltas and per-rate vegas.  lam_sum[r] = P(0,T_0) mean_p lam_r(0);
// mean_payoff = mean_p Phi_p.  vega_rate[r] = sum_{s,f} abar A (derivative
// with respect to a scaling of row r of every pseudo-root).
__global__ void greeks_finish_kernel(int n, int F, const __grid_constant__ ModelConst mc,
                                     float f0_0, float T0, const double* __restrict__ lam_sum,
                                     const double* __restrict__ mean_payoff,
                                     const float* __restrict__ A,
                                     const double* __restrict__ abar,
                                     double* __restrict__ price, double* __restrict__ delta,
                                     double* __restrict__ vega_rate) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const double P0 = 1.0 / (1.0 + (double)f0_0 * (double)T0);
  if (r == 0 && price) price[0] = P0 * mean_payoff[0];
  if (r >= n) return;
  const double Fd = exp((double)mc.logf0[r]);  // f0_r + d_r
  double d = lam_sum[r] / Fd;
  if (r == 0) d += -(double)T0 * P0 * P0 * mean_payoff[0];
  delta[r] = d;
  if (vega_rate) {
    double v = 0.0;
    for (int s = 0; s < n; ++s)
      for (int f = 0; f < F; ++f)
        v += abar[((size_t)s * n + r) * F + f] * (double)A[((size_t)s * n + r) * F + f];
    vega_rate[r] = v;
  }
}

// Shared memory of the reverse kernel.
inline size_t greeks_reverse_smem(int n, int F, int block) {
  const int FP = ((F > 0 ? F : kMaxFactors) + 3) & ~3;
  return ((size_t)n * FP + ((n + 3) & ~3) + 3 * (size_t)n * block) * sizeof(float);
}

}  // namespace lmm
