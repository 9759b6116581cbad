// fused_kernels.cuh — device code of the fused form (included by
// pipeline.cu): the variates kernel (Sobol -> scramble -> inverse normal ->
// bridge) and the per-path evolution kernel with the product epilogue.
//
// Both kernels use the fast hardware approximations of exp, log and
// reciprocal with denormals flushed (ex2/lg2/rcp.approx.ftz, lmm_device.cuh;
// relative error ~1e-7, i.e. a few FP32 ulp); the staged kernels keep the
// IEEE-accurate library forms and serve as the plain-FP32 reference of the
// same arithmetic.
#pragma once
#include <type_traits>
#include "lmm_common.cuh"
#include "lmm_device.cuh"
#include "bridge_plan.h"
#include "ls_common.cuh"
#include "pc_step.cuh"

namespace lmm {

struct ProductConst {
  int kind, n_ex;
  float strike, cap_strike, pay_receive;
  float tarn_total, tarn_mult;
  int ex_index[kMaxSteps];  // step -> exercise index, -1 if none
};

// Basis tables of every exercise date for the in-kernel rule (passed by
// value as a kernel parameter, about 7 KB).
struct RuleConst {
  int nvars[kMaxSteps];
  int nbasis[kMaxSteps];
  unsigned char mono[kMaxSteps][kMaxBasis][kMaxVars];
};

// kModeInputs: write the regression inputs; kModeRule: apply the frozen rule
// and write the payoff; kModeRecord: as kModeRule, and also record what the
// adjoint needs (log-rate checkpoints, numeraires, exercise steps).
// kModeOuter: as kModeInputs (every date, no stopping), and also record the
// log-rates and numeraire at the start of every `every`-th step (the outer
// paths of the Andersen–Broadie estimate).
enum { kModeInputs = 0, kModeRule = 1, kModeRecord = 2, kModeOuter = 3 };

// Paths per CTA of the evolution kernel, and steps per launch of the
// segmented second pass (SegIO below) unless the caller asks otherwise.
constexpr int kFusedBlock = 128;
constexpr int kSegSteps = 8;

// Outputs of kModeRecord.  Every `every` steps (s = c * every) the log-rates
// at the start of the step go to ckpt[c][r][p] (r >= s) and the numeraire to
// ckptN[c][p]; ex_step[p] is the exercise step (rates when never exercised).
struct RecordOut {
  float* ckpt;
  float* ckptN;
  int* ex_step;
  int every;
};

// Segmented rule-mode evolution.  A path stops at its exercise, so its
// lane idles for the rest of the launch; the second pass therefore runs as
// a chain of launches over segments of steps, and the paths still alive at
// the end of a segment are packed into survivor slots that the next
// segment's CTAs take densely.  SegState holds the survivors of one segment
// boundary s1 (after step s1 - 1): log-rates of rows >= s1, the numeraire
// and reset rate of step s1 - 1, the pending exercise date's P(T_s, T_{s+1})
// and coupon (the date is completed in step s1's rate loop), the payoff so
// far and the path's index in the batch.  Slots [b * T, b * T + count[b])
// belong to CTA b of the launch that wrote them (kept in path order).
struct SegState {
  float* rates;     // [rates][cap]
  float* N;         // [cap]
  float* f_first;   // [cap]
  float* pend_P1;   // [cap]
  float* pend_coupon;  // [cap]
  double* payoff;   // [cap]
  int* path;        // [cap]
};

// One launch of the chain: steps [s_begin, s_end).  in_prefix (null for the
// first segment) is the exclusive prefix of the previous launch's per-CTA
// survivor counts over in_blocks CTAs (in_prefix[in_blocks] = survivors);
// out.rates null marks the last segment, else the launch writes its
// survivors to `out` and their count per CTA to out_count.
struct SegIO {
  int s_begin, s_end, cap, in_blocks;
  const int* in_prefix;
  SegState in, out;
  int* out_count;
};

// Continuation estimate of the frozen rule at exercise date e (depth chain
// and Andersen shift of ls_chain_estimate).
__device__ __forceinline__ double rule_estimate(const RuleConst& rc, int e, const float* v,
                                                float exv, const LsRuleView& rule) {
  return ls_chain_estimate(rule, e, rc.nvars[e], rc.nbasis[e], rc.mono[e], v, exv);
}

// Shaw–Brickman inverse normal on the exact tail probability
// (icdf_sb_tails) with the hardware log and reciprocal approximations.
__device__ __forceinline__ float icdf_sb_fast(uint32_t vi) {
  float sgn;
  const float t = icdf_tail_t(vi, &sgn);
  const float z = -log_ftz(t);
  // numerator p and denominator q by one Horner recurrence on the pair
  // (p, q): each packed FMA rounds as the scalar FMA of the nested form
  const float2 z2 = make_float2(z, z);
  float2 pq = __ffma2_rn(make_float2(4.744820732427972462e-6f, 0.00010590620919921025259f), z2,
                         make_float2(0.0020751409553756572917f, 0.0120098270559197768f));
  pq = __ffma2_rn(pq, z2, make_float2(0.087403248265958578062f, 0.23668431621373705623f));
  pq = __ffma2_rn(pq, z2, make_float2(0.80002295072483916762f, 1.2499328117341603014f));
  pq = __ffma2_rn(pq, z2, make_float2(1.9797154223229267471f, 2.0795584360534589311f));
  pq = __ffma2_rn(pq, z2, make_float2(1.2533136835212087879f, 1.0f));
  return sgn * ((z * pq.x) * rcp_ftz(pq.y));
}

// ---------------------------------------------------------------------------
// Fused variates: Sobol point -> XOR scramble -> inverse normal -> bridge.
// One thread per (path, factor), one CTA per 128 consecutive paths and one
// factor.  With n = first_index + p and gray(n) = n ^ (n >> 1), the bits of
// gray(n) at and above 7 are gray(n >> 7): the CTA's paths share at most two
// values of n >> 7, so the XOR of the upper direction numbers (with the
// scrambler word folded in) is formed once per CTA and Sobol dimension
// (table hi_s).  The seven low Gray bits select from two small XOR tables
// per dimension, lo4_s (bits 0-3, 16 entries) and hi3_s (bits 4-6, 8
// entries), so a point costs three shared-memory reads and two XORs with no
// data-dependent branch.  Points are generated kVarBatch at a time (independent
// work for the scheduler), then folded into the bridge, whose S points per
// thread live in shared memory.  Output [step][factor][path] increments.
// ---------------------------------------------------------------------------
constexpr int kVarBlock = 128;
constexpr int kVarBatch = 8;

__global__ void __launch_bounds__(kVarBlock)
    variates_kernel(int paths, uint32_t first_index,
                    const uint32_t* __restrict__ dirs,
                    const uint32_t* __restrict__ scr, int scr_dims,
                    float* __restrict__ out,
                    const __grid_constant__ BridgePlan plan) {
  constexpr int T = kVarBlock;
  const int S = plan.steps, F = plan.factors;
  // shared memory (variates_smem_bytes): the bridge points W[S + 1][T]
  // (row S stays zero: the left neighbour of a point that has none), the
  // bridge plan per construction stage as {lw, rw, sd} weights and
  // {left row, right row, target row} byte offsets into W, and the
  // Sobol tables hi[2][S], lo4[S][17], hi3[S][9] (rows padded by one word,
  // so that the one-thread-per-dimension stores hit distinct banks)
  extern __shared__ __align__(16) float W[];
  float4* bw_s = reinterpret_cast<float4*>(W + (size_t)(S + 1) * T);
  int4* bo_s = reinterpret_cast<int4*>(bw_s + S);
  uint32_t* hi_s = reinterpret_cast<uint32_t*>(bo_s + S);
  uint32_t* lo4_s = hi_s + 2 * S;
  uint32_t* hi3_s = lo4_s + 17 * S;
  const int f = blockIdx.y;
  const int* alloc = plan.alloc + f * S;
  const int p0 = blockIdx.x * kVarBlock;
  const uint32_t h0 = (first_index + (uint32_t)p0) >> 7;
  // one thread per Sobol dimension of the factor: the XOR of the direction
  // numbers over the set upper Gray bits of h0 (with the scrambler word);
  // that of h0 + 1 differs in one Gray bit, gray(h + 1) = gray(h) ^
  // 2^ctz(h + 1) (no entry past bit 31: h0 + 1 = 2^25 has no path); and the
  // two low tables, each entry the previous one with its lowest set bit
  // cleared, XOR that bit's direction number
  for (int i = threadIdx.x; i < S; i += kVarBlock) {
    const int d = alloc[i];
    const uint32_t* v = dirs + 32 * d;
    uint32_t g = h0 ^ (h0 >> 1), x = 0;
    while (g) {
      x ^= __ldg(v + 7 + (__ffs(g) - 1));
      g &= g - 1u;
    }
    if (d < scr_dims) x ^= __ldg(scr + d);
    hi_s[i] = x;
    const int c = __ffs(h0 + 1u) - 1;
    hi_s[S + i] = (c >= 0 && c < 25) ? x ^ __ldg(v + 7 + c) : x;
    uint32_t vl[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) vl[k] = __ldg(v + k);
    uint32_t* l4 = lo4_s + 17 * i;
    uint32_t* h3 = hi3_s + 9 * i;
    uint32_t t4[16], t3[8];
    t4[0] = 0u;
    t3[0] = 0u;
#pragma unroll
    for (int e = 1; e < 16; ++e) t4[e] = t4[e & (e - 1)] ^ vl[__ffs(e) - 1];
#pragma unroll
    for (int e = 1; e < 8; ++e) t3[e] = t3[e & (e - 1)] ^ vl[4 + __ffs(e) - 1];
#pragma unroll
    for (int e = 0; e < 16; ++e) l4[e] = t4[e];
#pragma unroll
    for (int e = 0; e < 8; ++e) h3[e] = t3[e];
  }
  for (int i = threadIdx.x; i < S; i += kVarBlock) {
    // stage 0 is the terminal point W_S = sd_0 z (row S - 1); a stage
    // without a left neighbour reads the zero row S with weight 0
    const bool first = i == 0;
    const int jl = first ? 0 : plan.left[i];
    bw_s[i] = make_float4(jl != 0 ? plan.lw[i] : 0.0f, first ? 0.0f : plan.rw[i], plan.sd[i],
                          0.0f);
    bo_s[i] = make_int4((jl != 0 ? jl - 1 : S) * T * 4, (first ? S : plan.right[i]) * T * 4,
                        (first ? S - 1 : plan.bidx[i]) * T * 4, 0);
  }
  W[(size_t)S * T + threadIdx.x] = 0.0f;
  __syncthreads();
  const int p = p0 + threadIdx.x;
  if (p >= paths) return;
  const uint32_t n = first_index + (uint32_t)p;
  const int sel = (int)((n >> 7) - h0);
  const uint32_t glo = (n ^ (n >> 1)) & 127u;
  const uint32_t ga = glo & 15u, gb = glo >> 4;
  float* w = W + threadIdx.x;
  // this thread's entries of the Sobol tables, stage by stage
  const uint32_t* hi_t = hi_s + sel * S;
  const uint32_t* lo_t = lo4_s + ga;
  const uint32_t* h3_t = hi3_s + gb;
  const char* wb = reinterpret_cast<const char*>(w);
  // one batch of kVarBatch stages from i0; FULL: all of them exist (no
  // clamp of the stage index, no guard on the bridge step)
  auto batch = [&](int i0, auto full_tag) {
    constexpr bool FULL = decltype(full_tag)::value;
    float z[kVarBatch];
#pragma unroll
    for (int k = 0; k < kVarBatch; ++k) {
      const int i = FULL ? i0 + k : min(i0 + k, S - 1);
      const uint32_t x = hi_t[i] ^ lo_t[17 * i] ^ h3_t[9 * i];
      z[k] = icdf_sb_fast(x);
    }
#pragma unroll
    for (int k = 0; k < kVarBatch; ++k) {
      const int i = i0 + k;
      if (FULL || i < S) {
        const float4 bw = bw_s[i];
        const int4 bo = bo_s[i];
        // bo: byte offsets of the stage's rows (no index scaling per access)
        float y = bw.x * *reinterpret_cast<const float*>(wb + bo.x);
        y = fmaf(bw.y, *reinterpret_cast<const float*>(wb + bo.y), y);
        y = fmaf(bw.z, z[k], y);
        *reinterpret_cast<float*>(reinterpret_cast<char*>(w) + bo.z) = y;
      }
    }
  };
  int i0 = 0;
  for (; i0 + kVarBatch <= S; i0 += kVarBatch) batch(i0, std::true_type());
  if (i0 < S) batch(i0, std::false_type());
  float prev = 0.0f;
  float* o = out + (size_t)f * paths + p;
  const size_t o_step = (size_t)F * paths;
  for (int s = 0; s < S; ++s, o += o_step) {
    const float cur = w[s * T];
    *o = cur - prev;
    prev = cur;
  }
}

// Shared memory of variates_kernel for S bridge stages.
inline size_t variates_smem_bytes(int S) {
  return (size_t)(S + 1) * kVarBlock * sizeof(float) + (size_t)S * (sizeof(float4) + sizeof(int4)) +
         (size_t)S * (2 + 17 + 9) * sizeof(uint32_t);
}

}  // namespace lmm

namespace lmm {

// One period of the target redemption note for a path (the reference's
// TARN::getCashFlows, cashFlowGeneration_product_gpu.h:57-98, accruals =
// tau): returns the period's net flow (floating received plus coupon paid,
// at T_{s+1}); `paid` and `over` carry the path's state.
__device__ __forceinline__ float tarn_flow(const ProductConst& pc, int s, int n, float tau,
                                           float f, float& paid, bool& over) {
  if (over) return 0.0f;
  const float flow2 = tau * f;
  float flow1;
  if (s + 1 == n) {
    flow1 = paid - pc.tarn_total;
    over = true;
  } else {
    const float c = fmaxf((pc.strike - pc.tarn_mult * f) * tau, 0.0f);
    const float total = paid + c;
    if (total >= pc.tarn_total) {
      flow1 = paid - pc.tarn_total;
      over = true;
    } else {
      flow1 = -c;
      paid = total;
    }
  }
  return flow1 + flow2;
}

// ---------------------------------------------------------------------------
// Fused evolution.  One thread per path, CTA of 128 paths; shared memory
// holds the CTA's log-rates [rate][thread] and the step's pseudo-root
// (rows padded to a multiple of 4 factors for 16-byte loads) and fixed
// drift.  Per rate and step: predictor drift from the rates at the start of
// the step, predicted log-rate, corrector drift, corrected and capped
// log-rate (LMM_evolver_all.cu:615-744, gold/LMM_evolver_gold.h:315-387);
// the spot drift factor is g = F tau / (1 + f tau) with F = f + d the
// displaced rate.  At exercise steps the discount ratios P(T_s, T_{r+1}),
// the coterminal annuity and swap rate are accumulated on the fly.
// FT = number of factors (compile time), 0 = generic <= 16.
// ---------------------------------------------------------------------------
template <int FT, int MODE>
__global__ void __launch_bounds__(128, 5)
    fused_evolve_kernel(int paths, const float* __restrict__ Z,
                        const float* __restrict__ A,
                        const float* __restrict__ fixed,
                        const __grid_constant__ ModelConst mc,
                        const __grid_constant__ ProductConst pc,
                        const __grid_constant__ RuleConst rc,
                        const LsRuleView rule, int total, int col0,
                        float* __restrict__ o_vars, float* __restrict__ o_ex,
                        float* __restrict__ o_cf, float* __restrict__ o_num,
                        float* __restrict__ o_payoff, const RecordOut rec,
                        const SegIO seg) {
  constexpr int FM = FPad<FT>::FM;
  constexpr int FP = FPad<FT>::FP;
  const int F = FT > 0 ? FT : mc.F;
  const int n = mc.n;
  const int T = blockDim.x, tid = threadIdx.x;
  extern __shared__ __align__(16) float sm[];
  float* As = sm;                // [n][FP]
  float* fx = As + n * FP;       // [n] (+ pad)
  float* lfs = fx + ((n + 3) & ~3);  // [n][T]
  // the frozen-rule modes stop a path at its exercise and run in segments
  constexpr bool kSeg = MODE == kModeRule || MODE == kModeRecord;
  const bool resume = kSeg && seg.in_prefix != nullptr;
  int p = blockIdx.x * T + tid, src = 0;
  bool valid = p < paths;
  if (resume) {
    // survivor slot j of the previous segment, found in its CTA's block
    const int live = __ldg(seg.in_prefix + seg.in_blocks);
    if (blockIdx.x * T >= live) {  // no survivor slot here: uniform over the CTA
      if (tid == 0 && seg.out.rates != nullptr) seg.out_count[blockIdx.x] = 0;
      return;
    }
    const int j = blockIdx.x * T + tid;
    valid = j < live;
    p = 0;
    if (valid) {
      int lo = 0, hi = seg.in_blocks;  // in_prefix[lo] <= j < in_prefix[hi]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(seg.in_prefix + mid) <= j) lo = mid; else hi = mid;
      }
      src = lo * T + (j - __ldg(seg.in_prefix + lo));
      p = seg.in.path[src];
      if ((unsigned)p >= (unsigned)paths) {  // never for a consistent chain
        valid = false;
        p = 0;
      }
    }
  }
  const int s_begin = resume ? seg.s_begin : 0;
  const int s_end = kSeg ? seg.s_end : n;
  float N = 1.0f, f_first = 0.0f, cf_acc = 0.0f, N_bucket = 1.0f;
  int bucket = -1, ex_at = n;
  double payoff = 0.0;
  float tarn_paid = 0.0f;
  bool tarn_over = false;
  bool done = !valid;
  // swaption-plus-cap portfolio: after the swaption's exercise the path runs
  // on for the cap strip, with no further exercise dates
  bool exercised = false;
  const int col = col0 + p;
  // An exercise date's discount curve P(T_s, T_{r+1}), r >= s, is completed
  // in the next step's rate loop, which forms 1 / (1 + tau_r f_r) of every
  // later rate for its drift factors anyway (pc_rate's q); the date's
  // epilogue therefore runs one step later, from this pending state.
  int pend_e = -1, pend_s = 0;
  float pend_N = 1.0f, pend_f = 0.0f, pend_P1 = 1.0f, pend_coupon = 0.0f;
  if (!resume) {
    for (int r = 0; r < n; ++r) lfs[r * T + tid] = mc.logf0[r];
  } else {
    for (int r = s_begin; r < n; ++r)
      lfs[r * T + tid] = valid ? seg.in.rates[(size_t)r * seg.cap + src] : 0.0f;
    if (valid) {
      N = seg.in.N[src];
      f_first = seg.in.f_first[src];
      payoff = seg.in.payoff[src];
      const int e = pc.ex_index[s_begin - 1];
      if (e >= 0) {  // the date of step s_begin - 1 waits for this step's curve
        pend_e = e;
        pend_s = s_begin - 1;
        pend_N = N;
        pend_f = f_first;
        pend_P1 = seg.in.pend_P1[src];
        pend_coupon = seg.in.pend_coupon[src];
      }
    }
  }
  auto date_epilogue = [&](float Pn, float ann) {
    const int e = pend_e;
    float v[kMaxVars], exv = 0.0f;
    if (pc.kind == LMM_PRODUCT_SWAPTION || pc.kind == LMM_PRODUCT_BERMUDAN_CAP) {
      const float sr = (1.0f - Pn) / ann;
      v[0] = pend_f;
      v[1] = sr;
      v[2] = ann;
      exv = fmaxf((sr - pc.strike) * ann, 0.0f);
    } else {
      float sr;
      if (pend_s + 1 < n) {
        const float ann2 = ann - mc.tau[pend_s] * pend_P1;
        sr = (pend_P1 - Pn) / ann2;
      } else {
        sr = (1.0f - Pn) / ann;
      }
      v[0] = pend_f;
      v[1] = sr;
      v[2] = mc.tau[n - 1] * Pn;
    }
    pend_e = -1;
    if (MODE == kModeInputs || MODE == kModeOuter) {
      if (bucket >= 0) o_cf[(size_t)bucket * total + col] = cf_acc;
      bucket = e;
      cf_acc = pend_coupon;
#pragma unroll
      for (int k = 0; k < kMaxVars; ++k)
        o_vars[((size_t)e * kMaxVars + k) * total + col] = v[k];
      o_ex[(size_t)e * total + col] = exv;
      o_num[(size_t)e * total + col] = pend_N;
    } else {
      const double est = rule_estimate(rc, e, v, exv, rule);
      if ((double)exv > est) {
        payoff += (double)exv / (double)pend_N;
        if (MODE == kModeRecord) ex_at = pend_s;
        if (pc.kind == LMM_PRODUCT_BERMUDAN_CAP)
          exercised = true;
        else
          done = true;
        return;
      }
      payoff += (double)pend_coupon / (double)pend_N;
    }
    N_bucket = pend_N;
  };
  for (int s = s_begin; s < s_end; ++s) {
    // the step's normals are loaded first, so that their latency overlaps
    // the staging of the step's pseudo-root rows and the barriers
    float z[FP];
#pragma unroll
    for (int f = 0; f < FP; ++f)
      z[f] = (f < F && !done) ? __ldg(Z + ((size_t)s * F + f) * paths + p) : 0.0f;
    __syncthreads();
    for (int i = tid; i < n * FP; i += T) {
      const int r = i / FP, f = i - r * FP;
      As[i] = f < F ? __ldg(A + ((size_t)s * n + r) * F + f) : 0.0f;
    }
    for (int i = tid; i < n; i += T) fx[i] = __ldg(fixed + (size_t)s * n + i);
    __syncthreads();
    if (done) continue;
    if (s > 0) N = N * (1.0f + mc.tau[s - 1] * f_first);
    if ((MODE == kModeRecord || MODE == kModeOuter) && s % rec.every == 0) {
      const int c = s / rec.every;
      for (int r = s; r < n; ++r)
        rec.ckpt[((size_t)c * n + r) * paths + p] = lfs[r * T + tid];
      rec.ckptN[(size_t)c * paths + p] = N;
    }
    const bool pend = pend_e >= 0;
    float Pd = pend_P1, annd = pend ? mc.tau[s - 1] * pend_P1 : 0.0f;
    float2 w[FP / 2], v[FP / 2];
    step_start<FP>(z, w, v);
    // the rate loop, unswitched on whether a date's curve is pending
    auto rate_loop = [&](auto with_curve) {
#pragma unroll 4
      for (int r = s; r < n; ++r) {
        const float tau = mc.tau[r];
        float g, gp, q;
        bool capped;
        const float lf = pc_rate<FM, FP>(lfs[r * T + tid], mc.l2tau[r], mc.c0[r], fx[r],
                                         As + r * FP, w, v, mc.cutoff, g, gp, q, capped);
        lfs[r * T + tid] = lf;
        if (decltype(with_curve)::value) {
          Pd *= q;
          annd += tau * Pd;
        }
      }
    };
    if (pend)
      rate_loop(std::true_type{});
    else
      rate_loop(std::false_type{});
    f_first = __expf(lfs[s * T + tid]) - mc.disp[s];
    const float P1 = __fdividef(1.0f, 1.0f + mc.tau[s] * f_first);
    // ---- the previous step's exercise date, then the epilogue at T_s ----
    if (pend) {
      date_epilogue(Pd, annd);
      if (done) continue;
    }
    if (pc.kind == LMM_PRODUCT_TARN) {
      payoff += (double)(tarn_flow(pc, s, n, mc.tau[s], f_first, tarn_paid, tarn_over) * P1) /
                (double)N;
      continue;
    }
    if (pc.kind == LMM_PRODUCT_EUROPEAN) {
      const float tau = mc.tau[s];
      const float cap = tau * fmaxf(f_first - pc.cap_strike, 0.0f);
      const float swp = tau * (f_first - pc.strike) * pc.pay_receive;
      payoff += (double)((cap + swp) * P1) / (double)N;
      continue;
    }
    if (pc.kind == LMM_PRODUCT_BERMUDAN_CAP && (MODE == kModeRule || MODE == kModeRecord)) {
      // the portfolio's caplet on f_s, paid at T_{s+1} whether or not the
      // swaption has been exercised
      const float cap = mc.tau[s] * fmaxf(f_first - pc.cap_strike, 0.0f);
      payoff += (double)(cap * P1) / (double)N;
    }
    float coupon = 0.0f;
    if (pc.kind == LMM_PRODUCT_CANCELLABLE_SWAP)
      coupon = mc.tau[s] * (f_first - pc.strike) * pc.pay_receive * P1;
    const int e = exercised ? -1 : pc.ex_index[s];
    if (e >= 0) {
      pend_e = e;
      pend_s = s;
      pend_N = N;
      pend_f = f_first;
      pend_P1 = P1;
      pend_coupon = coupon;
    } else if (coupon != 0.0f) {
      if (MODE == kModeInputs || MODE == kModeOuter) {
        if (bucket >= 0) cf_acc += coupon * (N_bucket / N);
      } else {
        payoff += (double)coupon / (double)N;
      }
    }
  }
  if (kSeg && seg.out.rates != nullptr) {
    // end of a segment: pack the survivors of this CTA in path order (the
    // per-warp counts go to the pseudo-root rows, free once every warp is
    // past its last step)
    int* warp_live = reinterpret_cast<int*>(As);
    const bool live = valid && !done;
    const unsigned bal = __ballot_sync(0xffffffffu, live);
    const int warp = tid >> 5, lane = tid & 31;
    __syncthreads();
    if (lane == 0) warp_live[warp] = __popc(bal);
    __syncthreads();
    int off = 0, tot = 0;
    for (int w = 0; w < (T >> 5); ++w) {
      const int c = warp_live[w];
      off += w < warp ? c : 0;
      tot += c;
    }
    if (live) {
      const int slot = blockIdx.x * T + off + __popc(bal & ((1u << lane) - 1u));
      for (int r = s_end; r < n; ++r)
        seg.out.rates[(size_t)r * seg.cap + slot] = lfs[r * T + tid];
      seg.out.N[slot] = N;
      seg.out.f_first[slot] = f_first;
      seg.out.pend_P1[slot] = pend_P1;
      seg.out.pend_coupon[slot] = pend_coupon;
      seg.out.payoff[slot] = payoff;
      seg.out.path[slot] = p;
    }
    if (tid == 0) seg.out_count[blockIdx.x] = tot;
    if (valid && done) {
      o_payoff[p] = (float)payoff;
      if (MODE == kModeRecord) rec.ex_step[p] = ex_at;
    }
    return;
  }
  // an exercise date at the last step: its curve is the one period
  if (!done && pend_e >= 0) date_epilogue(pend_P1, mc.tau[n - 1] * pend_P1);
  if (!valid) return;
  if (MODE == kModeInputs || MODE == kModeOuter) {
    if (pc.kind != LMM_PRODUCT_EUROPEAN && bucket >= 0)
      o_cf[(size_t)bucket * total + col] = cf_acc;
    if ((pc.kind == LMM_PRODUCT_EUROPEAN || pc.kind == LMM_PRODUCT_TARN) && o_payoff)
      o_payoff[p] = (float)payoff;
  } else {
    o_payoff[p] = (float)payoff;
    if (MODE == kModeRecord) rec.ex_step[p] = ex_at;
  }
}

// Exclusive prefix of the per-CTA survivor counts of a segment launch
// (prefix[blocks] = survivors), one CTA: each thread sums a contiguous run
// of counts, the runs' sums are scanned across warps, then written back.
__global__ void __launch_bounds__(1024)
    seg_scan_kernel(const int* __restrict__ count, int blocks, int* __restrict__ prefix) {
  __shared__ int warp_sum[32];
  const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int chunk = (blocks + T - 1) / T;
  const int b0 = min(tid * chunk, blocks), b1 = min(b0 + chunk, blocks);
  int local = 0;
  for (int b = b0; b < b1; ++b) local += count[b];
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int w = lane < (T >> 5) ? warp_sum[lane] : 0;
    int x = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += t;
    }
    if (lane < (T >> 5)) warp_sum[lane] = x - w;
  }
  __syncthreads();
  int run = warp_sum[warp] + incl - local;
  for (int b = b0; b < b1; ++b) {
    prefix[b] = run;
    run += count[b];
  }
  if (tid == T - 1) prefix[blocks] = run;
}

// Padded pseudo-root row (floats) of the instantiation launched for F
// factors: 3, 5, 10 and 15 have their own instantiations; every other count
// runs the generic one, whose rows are padded for kMaxFactors.  Shared
// memory must be sized by this, not by F.
inline int launched_fm(int F) {
  return (F == 3 || F == 5 || F == 10 || F == 15) ? F : kMaxFactors;
}
inline int launched_row_pad(int F) { return (launched_fm(F) + 3) & ~3; }

// Shared memory of the fused evolution kernel.
inline size_t fused_smem_bytes(int n, int F, int block) {
  const int FP = launched_row_pad(F);
  return ((size_t)n * FP + ((n + 3) & ~3) + (size_t)n * block) * sizeof(float);
}

}  // namespace lmm
