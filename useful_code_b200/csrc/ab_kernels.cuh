// ab_kernels.cuh — device code of the Andersen–Broadie upper bound
// (included by pipeline.cu).
//
// The reference computes the duality gap on the CPU only: its gold LMM
// example (gold/gold_example/LMM_bermudan_gold.cpp:1132-1382) runs, for every
// outer path and exercise date, a sub-simulation from the outer state
// (LMMEvolverPartial_gold::conditionallyGenerate) priced with the frozen
// exercise strategy, and ABDualityGapEstimate*Rebate
// (gold/Andersen_Broadie_gold.cpp:59-187) turns the continuation estimates
// into the gap.  Here the outer paths come from the fused kernel (outer mode:
// LS inputs at every date and the log-rates at the start of every step), the
// inner paths from ab_inner_kernel: one CTA of 128 inner paths per (outer
// path, date), started from the outer state in shared memory, with
// counter-based normals generated in registers (no variates in HBM), and
// the frozen rule applied at the later dates.
#pragma once
#include "fused_kernels.cuh"

namespace lmm {

constexpr int kAbThreads = 128;

// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, SC 2011): ten rounds of two
// 32x32 -> 64-bit products with a Weyl-sequence key schedule.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int round = 0; round < 10; ++round) {
    if (round) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
  }
  return c;
}

struct AbArgs {
  int K;        // outer paths
  int chunks;   // CTAs of 128 inner paths per (outer path, date)
  int e0;       // first exercise date of the launch
  uint32_t k0, k1;  // Philox key
  int ex_step[kMaxSteps];  // date -> step
};

// Inner paths of one (outer path p, date e) per CTA group: from the state at
// the start of step s0 = ex_step[e] + 1 (ckpt [n][n][K], ckptN [n][K]),
// evolve to the end with the normals of inner path i = chunk * 128 + tid
// (Philox counter (i, p, 4 s + j, e), words 4j..4j+3 = factors), stop at
// the first later date whose exercise value exceeds the rule's estimate.
// Writes the CTA's sum and sum of squares of the deflated payoffs to
// part[(group) * chunks + chunk][2].  Bermudan payer swaption.
template <int FT>
__global__ void __launch_bounds__(kAbThreads, 4)
    ab_inner_kernel(const __grid_constant__ AbArgs a, const float* __restrict__ A,
                    const float* __restrict__ fixed, const __grid_constant__ ModelConst mc,
                    const __grid_constant__ ProductConst pc,
                    const __grid_constant__ RuleConst rc, const LsRuleView rule,
                    const float* __restrict__ ckpt, const float* __restrict__ ckptN,
                    double* __restrict__ part) {
  constexpr int FM = FPad<FT>::FM;
  constexpr int FP = FPad<FT>::FP;
  const int F = FT > 0 ? FT : mc.F;
  const int n = mc.n, T = kAbThreads, tid = threadIdx.x;
  extern __shared__ __align__(16) float sm[];
  float* As = sm;                    // [n][FP]
  float* fx = As + n * FP;           // [n] (+ pad)
  float* lfs = fx + ((n + 3) & ~3);  // [n][T]
  __shared__ double red_s[2][kAbThreads / 32];
  const int chunk = blockIdx.x % a.chunks, group = blockIdx.x / a.chunks;
  const int p = group % a.K, e = a.e0 + group / a.K;
  const int s0 = a.ex_step[e] + 1;
  const uint32_t inner = (uint32_t)(chunk * T + tid);
  for (int r = s0; r < n; ++r) lfs[r * T + tid] = __ldg(ckpt + ((size_t)s0 * n + r) * a.K + p);
  float N = __ldg(ckptN + (size_t)s0 * a.K + p), f_first = 0.0f;
  double payoff = 0.0;
  bool done = false;
  for (int s = s0; s < n; ++s) {
    __syncthreads();
    for (int i = tid; i < n * FP; i += T) {
      const int r = i / FP, f = i - r * FP;
      As[i] = f < F ? __ldg(A + ((size_t)s * n + r) * F + f) : 0.0f;
    }
    for (int i = tid; i < n; i += T) fx[i] = __ldg(fixed + (size_t)s * n + i);
    __syncthreads();
    if (done) continue;
    float z[FP];
#pragma unroll
    for (int j = 0; j < FP / 4; ++j) {
      if (4 * j < F) {
        const uint4 w = philox4x32_10(make_uint4(inner, (uint32_t)p, (uint32_t)(4 * s + j),
                                                 (uint32_t)e),
                                      a.k0, a.k1);
        // the pricing variates' inverse normal (hardware log and
        // reciprocal on the exact tail probability)
        z[4 * j + 0] = icdf_sb_fast(w.x);
        z[4 * j + 1] = icdf_sb_fast(w.y);
        z[4 * j + 2] = icdf_sb_fast(w.z);
        z[4 * j + 3] = icdf_sb_fast(w.w);
      } else {
        z[4 * j + 0] = z[4 * j + 1] = z[4 * j + 2] = z[4 * j + 3] = 0.0f;
      }
    }
#pragma unroll
    for (int f = 0; f < FP; ++f)
      if (f >= F) z[f] = 0.0f;
    if (s > s0) N = N * (1.0f + mc.tau[s - 1] * f_first);
    const int ed = pc.ex_index[s];
    float2 w[FP / 2], v[FP / 2];
    step_start<FP>(z, w, v);
    float Prun = 1.0f, ann = 0.0f;
#pragma unroll 4
    for (int r = s; r < n; ++r) {
      const float tau = mc.tau[r], d = mc.disp[r];
      float g, gp;
      bool capped;
      const float lf = pc_rate<FM, FP>(lfs[r * T + tid], mc.l2tau[r], mc.c0[r], fx[r],
                                       As + r * FP, w, v, mc.cutoff, g, gp, capped);
      lfs[r * T + tid] = lf;
      if (r == s || ed >= 0) {
        const float fn = exp_ftz(lf) - d;
        if (r == s) f_first = fn;
        if (ed >= 0) {
          Prun = Prun * rcp_ftz(1.0f + tau * fn);
          ann += tau * Prun;
        }
      }
    }
    if (ed > e) {
      const float sr = (1.0f - Prun) / ann;
      const float exv = fmaxf((sr - pc.strike) * ann, 0.0f);
      const float v[kMaxVars] = {f_first, sr, ann};
      const double est = rule_estimate(rc, ed, v, exv, rule);
      if ((double)exv > est) {
        payoff = (double)exv / (double)N;
        done = true;
      }
    }
  }
  double s1 = payoff, s2 = payoff * payoff;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  if ((tid & 31) == 0) {
    red_s[0][tid >> 5] = s1;
    red_s[1][tid >> 5] = s2;
  }
  __syncthreads();
  if (tid == 0) {
    double t1 = 0.0, t2 = 0.0;
    for (int w = 0; w < kAbThreads / 32; ++w) {
      t1 += red_s[0][w];
      t2 += red_s[1][w];
    }
    part[(size_t)blockIdx.x * 2] = t1;
    part[(size_t)blockIdx.x * 2 + 1] = t2;
  }
}

inline size_t ab_inner_smem(int n) {
  const int FP = ((kMaxFactors) + 3) & ~3;
  return ((size_t)n * FP + ((n + 3) & ~3) + (size_t)n * kAbThreads) * sizeof(float);
}

// Continuation estimate Q[e][p] (mean over the inner paths, fixed order
// over the CTAs) and its standard error; the last date has none (0).
__global__ void ab_continuation_kernel(int E, int K, int chunks, int inner,
                                       const double* __restrict__ part,
                                       double* __restrict__ Q, double* __restrict__ Qse) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // e * K + p
  if (i >= E * K) return;
  const int e = i / K;
  double m = 0.0, se = 0.0;
  if (e + 1 < E) {
    double t1 = 0.0, t2 = 0.0;
    const double* src = part + (size_t)(e * K + i % K) * chunks * 2;
    for (int c = 0; c < chunks; ++c) {
      t1 += src[2 * c];
      t2 += src[2 * c + 1];
    }
    m = t1 / inner;
    se = sqrt(fmax(t2 / inner - m * m, 0.0) / inner);
  }
  Q[i] = m;
  if (Qse) Qse[i] = se;
}

// The frozen rule's decision at every date of the outer paths (exercise
// value above the estimate, exerciseAllDeterminerEESimple_gold) and the
// deflated exercise values, from their LS inputs.
__global__ void ab_decide_kernel(int E, int K, const __grid_constant__ RuleConst rc,
                                 const LsRuleView rule, const float* __restrict__ vars,
                                 const float* __restrict__ ex, const float* __restrict__ num,
                                 int* __restrict__ X, double* __restrict__ Z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // e * K + p
  if (i >= E * K) return;
  const int e = i / K, p = i % K;
  float v[kMaxVars];
#pragma unroll
  for (int k = 0; k < kMaxVars; ++k) v[k] = vars[((size_t)e * kMaxVars + k) * K + p];
  const float exv = ex[i];
  const double est = rule_estimate(rc, e, v, exv, rule);
  X[i] = ((double)exv > est) ? 1 : 0;
  Z[i] = (double)exv / (double)num[i];
}

// Duality gap per path (ABDualityGapEstimateNonZeroRebate,
// gold/Andersen_Broadie_gold.cpp:121-187; payoffs null: the zero-rebate form
// of :59-119) and, when lower != null, the value of the frozen rule on the
// outer path (the first date with ex = 1).  ex / payoffs [steps][paths],
// means[p * m_p + s * m_s]; is_ex in the bit mask words is_ex[s / 32].
// Per-CTA FP64 partials: part[b][4] = sum, sum of squares of the gap; sum,
// sum of squares of the lower value.
struct AbGapArgs {
  int steps, paths;
  long long m_p, m_s;
  unsigned is_ex[(kMaxSteps + 32) / 32];
};

__global__ void __launch_bounds__(256)
    ab_gap_kernel(const __grid_constant__ AbGapArgs g, const int* __restrict__ ex,
                  const double* __restrict__ payoffs, const double* __restrict__ means,
                  double* __restrict__ part) {
  __shared__ double red_s[4][8];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  if (p < g.paths) {
    double best = 0.0, balance = 0.0, lower = 0.0;
    bool exercised = false;
    const int last = payoffs ? g.steps - 1 : g.steps;
    for (int s = 0; s < last; ++s) {
      if (!((g.is_ex[s >> 5] >> (s & 31)) & 1u)) continue;
      const double z = payoffs ? payoffs[(size_t)s * g.paths + p] : 0.0;
      const double m = means[(size_t)p * g.m_p + (size_t)s * g.m_s];
      double x;
      if (ex[(size_t)s * g.paths + p] == 1) {
        x = -balance;
        balance += z - m;
        if (!exercised) lower = z;
        exercised = true;
      } else {
        x = z - m - balance;
      }
      best = fmax(best, x);
    }
    best = fmax(best, -balance);
    v[0] = best;
    v[1] = best * best;
    v[2] = lower;
    v[3] = lower * lower;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double t = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) red_s[k][w] = t;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red_s[threadIdx.x][i];
    part[(size_t)blockIdx.x * 4 + threadIdx.x] = t;
  }
}

// Means and standard errors from the partials of ab_gap_kernel (fixed
// order): out = {gap mean, gap se, lower mean, lower se}.
__global__ void ab_gap_final_kernel(int nblocks, int paths, const double* __restrict__ part,
                                    double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double t[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = 0; b < nblocks; ++b)
    for (int k = 0; k < 4; ++k) t[k] += part[(size_t)b * 4 + k];
  for (int k = 0; k < 2; ++k) {
    const double m = t[2 * k] / paths;
    out[2 * k] = m;
    out[2 * k + 1] = sqrt(fmax(t[2 * k + 1] / paths - m * m, 0.0) / paths);
  }
}

}  // namespace lmm
