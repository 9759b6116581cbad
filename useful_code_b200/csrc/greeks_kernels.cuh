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
// forward pass; a segment kernel recomputes k steps from a checkpoint
// (pc_rate, the pricing kernels' own arithmetic) and stores the drift
// factors g (start rates) and gp (predicted rates) and the new log-rates ln
// of each step; then one reverse kernel per step:
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
//   * accumulates dV/dA_s.  With M_rj = sum_p (mubar_r g_j + a_r gp_j / 2)
//     (j <= r), N_rf = sum_p L_r z_f and l_r = sum_p L_r,
//       dV/dA_s[k][f] = sum_{j<=k} M_kj A_jf + sum_{i>=k} M_ik A_if + N_kf
//                       - A_kf l_k
//     (mu_r = sum_{j<=r} C_rj g_j with C = A A^T, dW = A z, fixed drift
//     -|A_r|^2 / 2).  The row and column sums against A are the prefix and
//     suffix factor sums the sweep already carries, so each path adds its
//     row of dV/dA_s in O(F) per rate and M (O(n^2) per path) is never
//     formed.
// Deltas: dV/df0_r = P(0,T_0) mean_p lam_r(0) / (f0_r + d_r), plus the
// derivative of P(0,T_0) = 1 / (1 + f0_0 T_0) for r = 0.
#pragma once
#include "fused_kernels.cuh"

namespace lmm {

// Recompute steps [s0, s1) from the checkpoint at s0 (log-rates ckpt [n][P],
// rates r >= s0, and the numeraire ckptN [P]) and store, per step k = s - s0,
// what the reverse sweep reads: drift factors seg_g / seg_gp and new
// log-rates seg_ln (NaN where the cap applied), each [k][n][P] for rates
// r >= s, and seg_info [k][2F + 3][P] = (sum_r g_r A_rf, sum_r gp_r A_rf,
// numeraire at T_s, P(T_s, T_n), annuity of T_s).  Paths past their
// exercise step write nothing.
template <int FT>
__global__ void __launch_bounds__(128, 4)
    greeks_segment_kernel(int paths, int s0, int s1, const float* __restrict__ Z,
                          const float* __restrict__ A,
                          const float* __restrict__ fixed,
                          const __grid_constant__ ModelConst mc,
                          const float* __restrict__ ckpt,
                          const float* __restrict__ ckptN,
                          const int* __restrict__ ex_step, int stop_rule,
                          float* __restrict__ seg_g, float* __restrict__ seg_gp,
                          float* __restrict__ seg_ln, float* __restrict__ seg_info) {
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
  // stop_rule 0: a path runs to its exercise step; 1 (the swaption): paths
  // never exercised have no flows and are not needed; 2 (the swaption-plus-
  // cap portfolio): every path runs to the last step for its caplets
  int stop = valid ? ex_step[p] : -1;
  if (stop_rule == 1 && stop >= n) stop = -1;
  if (stop_rule == 2 && valid) stop = n - 1;
  const size_t P = (size_t)paths;
  for (int r = s0; r < n; ++r)
    lfs[r * T + tid] = valid ? ckpt[(size_t)r * P + p] : 0.0f;
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
    const size_t k = (size_t)(s - s0);
    float z[FP];
#pragma unroll
    for (int f = 0; f < FP; ++f)
      z[f] = (f < F) ? __ldg(Z + ((size_t)s * F + f) * P + p) : 0.0f;
    // w, v: pc_rate's running vectors; e_, ep: the step's totals
    // sum_r g_r A_r and sum_r gp_r A_r, which the reverse sweep reads
    float2 w[FP / 2], v[FP / 2], e_[FP / 2], ep[FP / 2];
    step_start<FP>(z, w, v);
#pragma unroll
    for (int k = 0; k < FP / 2; ++k) e_[k] = ep[k] = make_float2(0.0f, 0.0f);
    float Prun = 1.0f, ann = 0.0f;
#pragma unroll 4
    for (int r = s; r < n; ++r) {
      float g, gp;
      bool capped;
      const float ln = pc_rate<FM, FP>(lfs[r * T + tid], mc.l2tau[r], mc.c0[r], fx[r],
                                       As + r * FP, w, v, mc.cutoff, g, gp, capped);
      {
        const float2* a2 = reinterpret_cast<const float2*>(As + r * FP);
        const float2 g2 = make_float2(g, g), gp2 = make_float2(gp, gp);
#pragma unroll
        for (int k = 0; k < (FM + 1) / 2; ++k) {
          e_[k] = __ffma2_rn(a2[k], g2, e_[k]);
          ep[k] = __ffma2_rn(a2[k], gp2, ep[k]);
        }
      }
      lfs[r * T + tid] = ln;
      const size_t o = (k * n + r) * P + p;
      seg_g[o] = g;
      seg_gp[o] = gp;
      seg_ln[o] = capped ? __int_as_float(0x7fc00000) : ln;  // NaN marks the cap
      const float fn = exp_ftz(ln) - mc.disp[r];
      if (r == s) f_first = fn;
      Prun = Prun * rcp_ftz(1.0f + mc.tau[r] * fn);
      ann += mc.tau[r] * Prun;
    }
    float* info = seg_info + k * (2 * F + 3) * P + p;
#pragma unroll
    for (int f = 0; f < FM; ++f)
      if (f < F) {
        info[(size_t)f * P] = (f & 1) ? e_[f >> 1].y : e_[f >> 1].x;
        info[(size_t)(F + f) * P] = (f & 1) ? ep[f >> 1].y : ep[f >> 1].x;
      }
    info[(size_t)(2 * F) * P] = N;
    info[(size_t)(2 * F + 1) * P] = Prun;
    info[(size_t)(2 * F + 2) * P] = ann;
  }
}

// Buffers of the reverse sweep.
struct GreeksStepBufs {
  float* lam;     // [n][P] adjoint of the log-rates (in: end of step, out: start)
  double* later;  // [P] sum of the flows after the step (deflated)
  double* part;   // [CTA][n * F + n] per-CTA sums of dV/dA_s rows (and, at
                  // step 0, of the adjoint lam)
};

// One step's forward quantities, written by the segment kernel.
struct GreeksStepIn {
  const float* g;     // [n][P] drift factor of the start rates (rows >= s)
  const float* gp;    // [n][P] drift factor of the predicted rates
  const float* ln;    // [n][P] new log-rates, NaN where capped
  const float* info;  // [2F + 3][P] factor totals, numeraire, P(T_s,T_n), annuity
};

constexpr int kRevThreads = 128;

// Reverse of step s (one launch per step, steps descending; persistent CTAs
// walk tiles of kRevThreads paths).  Per path and rate r (descending) the
// contribution to dV/dA_s[r][f] is
//   mubar_r e_f(r) + a_r ep_f(r) / 2 + g_r k_f(r) + gp_r h_f(r)
//   + L_r (z_f - A_rf)
// with the prefix sums e_f(r) = sum_{j<=r} g_j A_jf (and ep with gp) taken
// as the step total minus the suffix beyond r, and the suffix sums k, h of
// the sweep: the row and column sums of M = sum_p (mubar g^T + a gp^T / 2)
// against A without forming M.  Sums over the paths of a warp are a fixed
// shuffle tree; each warp keeps FP64 sums in shared memory, and the CTA
// writes its partial in a fixed order.
template <int FT>
__global__ void __launch_bounds__(kRevThreads)
    greeks_reverse_kernel(int paths, int s, const float* __restrict__ Z,
                          const float* __restrict__ A,
                          const __grid_constant__ ModelConst mc,
                          const __grid_constant__ ProductConst pc,
                          const GreeksStepIn in, const int* __restrict__ ex_step,
                          const GreeksStepBufs b) {
  constexpr int FM = FPad<FT>::FM;
  constexpr int FP = FPad<FT>::FP;
  constexpr int T = kRevThreads, NW = kRevThreads / 32;
  const int F = FT > 0 ? FT : mc.F;
  const int n = mc.n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  extern __shared__ __align__(16) float sm[];
  double* acc = reinterpret_cast<double*>(sm);        // [NW][n][F] + [NW][n]
  const int accw = n * F + n;                          // doubles per warp
  float* As = reinterpret_cast<float*>(acc + (size_t)NW * accw);  // [n][FP]
  // per warp: the 32 lanes' rows of dV/dA (and the rate adjoint) [32][NC]
  constexpr int NC = FM + 1;
  float* stage_all = As + (size_t)n * FP;
  for (int i = tid; i < n * FP; i += T) {
    const int r = i / FP, f = i - r * FP;
    As[i] = f < F ? __ldg(A + ((size_t)s * n + r) * F + f) : 0.0f;
  }
  for (int i = tid; i < NW * accw; i += T) acc[i] = 0.0;
  __syncthreads();
  double* myacc = acc + (size_t)warp * accw;
  float* stage = stage_all + (size_t)warp * 32 * NC;
  const size_t P = (size_t)paths;
  for (int p0 = blockIdx.x * T; p0 < paths; p0 += gridDim.x * T) {
    const int p = p0 + tid;
    const int stop = p < paths ? ex_step[p] : -1;
    // a path contributes at step s if it is still running there and has a
    // flow at or after s (a swaption only at its exercise step; the
    // swaption-plus-cap portfolio runs every path to the last step)
    // (an inactive path's adjoint rows keep the zeros of the start of the
    // call until its exercise step: nothing writes them before)
    const int run_end = (pc.kind == LMM_PRODUCT_BERMUDAN_CAP) ? n - 1 : stop;
    bool act = p < paths && s <= run_end;
    if (pc.kind == LMM_PRODUCT_SWAPTION && stop >= n) act = false;
    // a warp with no active path adds exact zeros to every sum: skip it
    if (!__any_sync(0xffffffffu, act)) continue;
    float z[FP], E[FP], EP[FP];
#pragma unroll
    for (int f = 0; f < FP; ++f) {
      const bool ok = act && f < F;
      z[f] = ok ? __ldg(Z + ((size_t)s * F + f) * P + p) : 0.0f;
      E[f] = ok ? in.info[(size_t)f * P + p] : 0.0f;
      EP[f] = ok ? in.info[(size_t)(F + f) * P + p] : 0.0f;
    }
    const float N = act ? in.info[(size_t)(2 * F) * P + p] : 1.0f;
    const float Pn = act ? in.info[(size_t)(2 * F + 1) * P + p] : 1.0f;
    const float ann = act ? in.info[(size_t)(2 * F + 2) * P + p] : 0.0f;
    // ---- the flow at step s and its derivative with respect to f_s ----
    float f_s = 0.0f, P1 = 1.0f;
    if (act) {
      const float l0 = in.ln[(size_t)s * P + p];
      f_s = exp_ftz(l0 != l0 ? mc.cutoff : l0) - mc.disp[s];
      P1 = 1.0f / (1.0f + mc.tau[s] * f_s);
    }
    const int e = pc.ex_index[s];
    const bool is_ex = act && (s == stop) && (e >= 0) && pc.kind != LMM_PRODUCT_EUROPEAN;
    const float tau_s = mc.tau[s];
    const float invN = 1.0f / N;
    float term = 0.0f;      // flow / N at step s
    float dterm_fs = 0.0f;  // d(term)/d f_s from the flows that depend on f_s only
    bool swaption_ex = false;
    if (!act) {
    } else if (pc.kind == LMM_PRODUCT_EUROPEAN) {
      const float cap = tau_s * fmaxf(f_s - pc.cap_strike, 0.0f);
      const float swp = tau_s * (f_s - pc.strike) * pc.pay_receive;
      term = (cap + swp) * P1 * invN;
      const float dv = tau_s * ((f_s > pc.cap_strike ? 1.0f : 0.0f) + pc.pay_receive);
      dterm_fs = (dv * P1 - (cap + swp) * P1 * tau_s * P1) * invN;
    } else if (pc.kind == LMM_PRODUCT_BERMUDAN_CAP) {
      // caplet on f_s paid at T_{s+1}, plus the swaption at its exercise
      const float cap = tau_s * fmaxf(f_s - pc.cap_strike, 0.0f);
      term = cap * P1 * invN;
      dterm_fs = (tau_s * (f_s > pc.cap_strike ? 1.0f : 0.0f) * P1 - cap * P1 * tau_s * P1) *
                 invN;
      if (is_ex) {
        const float v = (1.0f - Pn) - pc.strike * ann;
        if (v > 0.0f) {
          term += v * invN;
          swaption_ex = true;
        }
      }
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
    if (act) {
      const double later = b.later[p];
      // the numeraire factor (1 + tau_s f_s) divides every later flow
      dterm_fs += -(float)later * tau_s / (1.0f + tau_s * f_s);
      b.later[p] = later + (double)term;
    }
    // ---- descending sweep (every lane, for the warp sums) ----
    float h[FP], kk[FP], u[FP], up[FP];
#pragma unroll
    for (int f = 0; f < FP; ++f) h[f] = kk[f] = u[f] = up[f] = 0.0f;
    float Pr = Pn, ann_suf = 0.0f;
    // the next rate's inputs are loaded one iteration ahead
    float nx_ln = 0.0f, nx_lam = 0.0f, nx_g = 0.0f, nx_gp = 0.0f;
    if (act) {
      const size_t o = (size_t)(n - 1) * P + p;
      nx_ln = in.ln[o];
      nx_lam = (n - 1 > s) ? b.lam[o] : 0.0f;
      nx_g = in.g[o];
      nx_gp = in.gp[o];
    }
    for (int r = n - 1; r >= s; --r) {
      float a = 0.0f, g = 0.0f, gp = 0.0f, onep = 1.0f;
      const float ln_raw = nx_ln, lam_in = nx_lam, g_in = nx_g, gp_in = nx_gp;
      if (act && r > s) {
        const size_t o = (size_t)(r - 1) * P + p;
        nx_ln = in.ln[o];
        nx_lam = (r - 1 > s) ? b.lam[o] : 0.0f;
        nx_g = in.g[o];
        nx_gp = in.gp[o];
      }
      if (act) {
        const bool capped = ln_raw != ln_raw;
        const float Fd = exp_ftz(capped ? mc.cutoff : ln_raw);  // f_r + d_r = df_r / dln_r
        const float tr = mc.tau[r];
        onep = 1.0f + tr * (Fd - mc.disp[r]);
        // Pr = P(T_s, T_{r+1}); ann_suf = sum_{k >= r} tau_k P(T_s, T_{k+1})
        ann_suf += tr * Pr;
        float dphi_df = 0.0f;
        if (swaption_ex) dphi_df = tr / onep * (Pn + pc.strike * ann_suf) * invN;
        if (r == s) dphi_df += dterm_fs;
        a = capped ? 0.0f : lam_in + dphi_df * Fd;
        g = g_in;
        gp = gp_in;
      }
      const float4* a4 = reinterpret_cast<const float4*>(As + r * FP);
      float av[FP];
#pragma unroll
      for (int q = 0; q < FP / 4; ++q) {
        const float4 v4 = a4[q];
        av[4 * q] = v4.x;
        av[4 * q + 1] = v4.y;
        av[4 * q + 2] = v4.z;
        av[4 * q + 3] = v4.w;
      }
      float S1 = 0.0f;
#pragma unroll
      for (int f = 0; f < FM; ++f) {
        h[f] += 0.5f * a * av[f];
        S1 += av[f] * h[f];
      }
      const float L = a + gp * (1.0f - gp) * S1;
      const float mubar = L - 0.5f * a;
      float S2 = 0.0f;
#pragma unroll
      for (int f = 0; f < FM; ++f) {
        kk[f] += mubar * av[f];
        S2 += av[f] * kk[f];
      }
      const float lam_out = L + g * (1.0f - g) * S2;
      if (act) b.lam[r * P + p] = lam_out;
      // this path's row r of dV/dA_s, summed over the warp
      float row[FP];
#pragma unroll
      for (int f = 0; f < FM; ++f) {
        const float ef = EP[f] - up[f];  // prefix sums through r
        const float eg = E[f] - u[f];
        row[f] = mubar * eg + 0.5f * a * ef + g * kk[f] + gp * h[f] + L * (z[f] - av[f]);
        u[f] += g * av[f];
        up[f] += gp * av[f];
      }
      // summed over the warp through shared memory: the lanes' rows go to
      // stage[lane][c] (column FM = the rate adjoint, for the step-0 sums),
      // then column c is summed by lanes c and c + NC (16 rows each, fixed
      // order) where 2 NC <= 32, else by lane c alone; one FP64 add per
      // column into the warp's accumulator
#pragma unroll
      for (int f = 0; f < FM; ++f) stage[lane * NC + f] = row[f];
      stage[lane * NC + FM] = (s == 0) ? lam_out : 0.0f;
      __syncwarp();
      if (2 * NC <= 32) {
        const int c = lane < NC ? lane : lane - NC, h = lane < NC ? 0 : 16;
        float t = 0.0f;
        if (lane < 2 * NC)
#pragma unroll
          for (int l = 0; l < 16; ++l) t += stage[(h + l) * NC + c];
        t += __shfl_down_sync(0xffffffffu, t, NC);
        if (lane < F) myacc[r * F + lane] += (double)t;
        if (s == 0 && lane == FM) myacc[n * F + r] += (double)t;
      } else if (lane < NC) {
        float t = 0.0f;
#pragma unroll 8
        for (int l = 0; l < 32; ++l) t += stage[l * NC + lane];
        if (lane < F) myacc[r * F + lane] += (double)t;
        if (s == 0 && lane == FM) myacc[n * F + r] += (double)t;
      }
      __syncwarp();
      Pr = Pr * onep;  // P(T_s, T_r)
    }
  }
  // fixed-order sum over the warps, one partial per CTA
  __syncthreads();
  double* out = b.part + (size_t)blockIdx.x * accw;
  for (int i = tid; i < accw; i += T) {
    double v = 0.0;
    for (int w = 0; w < NW; ++w) v += acc[(size_t)w * accw + i];
    out[i] = v;
  }
}

// dV/dA_s (and at step 0 the adjoint sums behind the deltas) from the
// per-CTA partials, summed in a fixed order and scaled by P(0,T_0) / paths.
__global__ void greeks_abar_kernel(int n, int F, int s, int nblocks, double scale,
                                   const double* __restrict__ part,
                                   double* __restrict__ abar, double* __restrict__ lam_sum) {
  const int accw = n * F + n;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= accw) return;
  double v = 0.0;
  for (int c = 0; c < nblocks; ++c) v += part[(size_t)c * accw + idx];
  v *= scale;
  if (idx < n * F)
    abar[(size_t)s * n * F + idx] = (idx / F >= s) ? v : 0.0;
  else if (s == 0)
    lam_sum[idx - n * F] = v;
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
inline size_t greeks_reverse_smem(int n, int F) {
  const int FP = launched_row_pad(F);
  const size_t acc = (size_t)(kRevThreads / 32) * ((size_t)n * F + n) * sizeof(double);
  const int NC = launched_fm(F) + 1;
  const size_t stage = (size_t)(kRevThreads / 32) * 32 * NC * sizeof(float);
  return acc + (size_t)n * FP * sizeof(float) + stage;
}

}  // namespace lmm
