// ls_nested.cu — Longstaff–Schwartz with nested regressions (depth > 1).
//
// Reference behaviour followed:
//   backward loop, nested    generateRegressionCoefficientsViaLSMulti_gold
//   regressions              (gold/MultiLS_regression.cpp:101-417; the
//                            one-sign shortcut at :212-225 of the root tree)
//                            and its GPU orchestration
//                            generateMultiRegressionCoefficientsViaLS_gpu_
//                            flexisolve (LS_main_cula.h:565-837)
//   path selection           RegressionSelector_gold_Fraction::Select
//                            (gold/Regression_Selector_concrete_gold.cpp:58-205)
//   decision chain           updateDeflatedNextStepValuesMulti_gold
//                            (gold/MultiLS_regression.h:42-99),
//                            exercise_updating_LS_multi_kernel (LS_gpu.cu:312)
//
// Per date e the loop is a fixed sequence of launches with no host
// synchronisation: the decision of date e + 1 is applied to the running
// values; the first regression runs over all paths (ls_date_kernel); then
// for each further depth d: a pass forms the net values of regression d - 1
// on its paths (non-members hold +inf) with their FP64 moments; a few
// selection passes count |net| against up to 256 thresholds each (one
// histogram per pass) and advance the half-width search, which the last CTA
// of each pass runs exactly as the reference's sequential search, reading
// counts from the histogram; the moments of the selected paths follow,
// then the regression over them (ls_date_kernel with a mask).  When a date
// stops nesting (one-sign net values, too few paths, or a search that did
// not finish), a flag makes its remaining launches return at once.
//
// The reference's search evaluates one count per step on the whole path
// set.  Here each pass evaluates every count the search can ask for next:
// the whole geometric chain of its grow or shrink loop, or the next eight
// levels of its bisection tree, computed with the same floating-point
// operations, so the search reads exact counts and takes the same steps.
#include "lmm_common.cuh"
#include "lmm_device.cuh"
#include "ls_common.cuh"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

using namespace lmm;

#define TRY(x)           \
  do {                   \
    const int st_ = (x); \
    if (st_) return st_; \
  } while (0)

namespace {

constexpr int kSelBatch = 256;      // thresholds per selection pass
constexpr int kSelPasses = 6;       // selection passes launched per depth
constexpr int kSelMaxCounts = 512;  // count evaluations per search
constexpr int kSelCapped = 8;       // status: a search stopped at kSelMaxCounts
constexpr int kSelIncomplete = 16;  // status: a search needed more passes
constexpr int kNestThreads = 256;

enum {
  kPhDone = 0,
  kPhBranch,      // n within the targets: the reference keeps every path (cut 1e4)
  kPhInit,        // count at g = sds * sd
  kPhGrow,        // g /= multiplier while count < lower target
  kPhShrinkInit,  // count at lo = g * multiplier
  kPhShrink,      // lo *= multiplier while count > upper target
  kPhBisectInit,  // count at g = (lo + hi) / 2
  kPhBisect       // halve [lo, hi] while the count is outside the targets
};

// Search state of one (date, depth), kept in the workspace between passes.
struct SelState {
  int phase, lo_t, hi_t, evals, c, after, nb, status;
  double g, lo, hi, mult, cut;
  double thr[kSelBatch];  // thresholds of the pending pass, ascending
  int cnt[kSelBatch];     // paths with |net| <= thr[i], after the pass
};

__device__ bool sel_lookup(const SelState& S, double g, int* c) {
  int a = 0, b = S.nb - 1;
  while (a <= b) {
    const int m = (a + b) >> 1;
    const double t = S.thr[m];
    if (t == g) {
      *c = S.cnt[m];
      return true;
    }
    if (t < g)
      a = m + 1;
    else
      b = m - 1;
  }
  return false;
}

// Runs the search from its saved phase until it ends (true) or needs a
// count the last pass did not evaluate (false; the state then says which).
// Same steps and stopping rules as frac_select of the CPU restatement.
__device__ bool sel_run(SelState& S) {
  int c;
  for (;;) {
    switch (S.phase) {
      case kPhBranch:
        if (!sel_lookup(S, 1e4, &c)) return false;
        S.cut = 1e4;
        S.after = c;
        S.phase = kPhDone;
        return true;
      case kPhInit:
        if (!sel_lookup(S, S.g, &c)) return false;
        ++S.evals;
        S.c = c;
        S.phase = kPhGrow;
        break;
      case kPhGrow:
        if (S.c < S.lo_t) {
          if (S.evals >= kSelMaxCounts) {
            S.status |= kSelCapped;
          } else {
            const double g2 = S.g / S.mult;
            if (!sel_lookup(S, g2, &c)) return false;
            S.g = g2;
            S.c = c;
            ++S.evals;
            break;
          }
        }
        if (S.c < S.hi_t) {
          S.cut = S.g;
          S.after = S.c;
          S.phase = kPhDone;
          return true;
        }
        S.lo = S.g * S.mult;
        S.phase = kPhShrinkInit;
        break;
      case kPhShrinkInit:
        if (!sel_lookup(S, S.lo, &c)) return false;
        ++S.evals;
        S.c = c;
        S.phase = kPhShrink;
        break;
      case kPhShrink:
        if (S.c > S.hi_t) {
          if (S.evals >= kSelMaxCounts) {
            S.status |= kSelCapped;
          } else {
            const double l2 = S.lo * S.mult;
            if (!sel_lookup(S, l2, &c)) return false;
            S.lo = l2;
            S.c = c;
            ++S.evals;
            break;
          }
        }
        if (S.c > S.lo_t) {
          S.cut = S.lo;
          S.after = S.c;
          S.phase = kPhDone;
          return true;
        }
        S.hi = S.g;
        S.g = 0.5 * (S.lo + S.hi);
        S.phase = kPhBisectInit;
        break;
      case kPhBisectInit:
        if (!sel_lookup(S, S.g, &c)) return false;
        ++S.evals;
        S.c = c;
        S.phase = kPhBisect;
        break;
      case kPhBisect:
        if ((S.c < S.lo_t || S.c > S.hi_t) && (S.hi - S.lo) > 1e-6) {
          if (S.evals >= kSelMaxCounts) {
            S.status |= kSelCapped;
          } else {
            if (S.c < S.lo_t)
              S.lo = S.g;
            else
              S.hi = S.g;
            S.g = 0.5 * (S.lo + S.hi);
            S.phase = kPhBisectInit;
            break;
          }
        }
        S.cut = S.g;
        S.after = S.c;
        S.phase = kPhDone;
        return true;
      default:
        return true;
    }
  }
}

// Thresholds the search can ask for next from its saved phase, written
// unsorted to out (thread 0 for the chains; the bisection tree in
// parallel, node i by the halvings on its path from the root).  Returns
// the count.
__device__ int sel_batch(const SelState& S, double* out) {
  const int tid = threadIdx.x;
  int n = 0;
  if (S.phase == kPhBisectInit) {
    // node i (heap order): from [lo, hi], left child = [lo, mid] (the count
    // was above the upper target), right child = [mid, hi]
    for (int i = tid; i < kSelBatch - 1; i += blockDim.x) {
      const int h = i + 1;
      int lead = 31 - __clz(h);
      double lo = S.lo, hi = S.hi;
      for (int b = lead - 1; b >= 0; --b) {
        const double mid = 0.5 * (lo + hi);
        if ((h >> b) & 1)
          lo = mid;
        else
          hi = mid;
      }
      out[i] = 0.5 * (lo + hi);
    }
    return kSelBatch - 1;
  }
  if (tid == 0) {
    switch (S.phase) {
      case kPhBranch:
        out[n++] = 1e4;
        break;
      case kPhInit: {
        out[n++] = S.g;
        double g = S.g;
        for (int i = 0; i < 63; ++i) {
          g = g / S.mult;
          out[n++] = g;
        }
        double l = S.g * S.mult;
        out[n++] = l;
        while (n < kSelBatch) {
          l = l * S.mult;
          out[n++] = l;
        }
        break;
      }
      case kPhGrow: {
        double g = S.g;
        while (n < kSelBatch) {
          g = g / S.mult;
          out[n++] = g;
        }
        break;
      }
      case kPhShrinkInit: {
        double l = S.lo;
        out[n++] = l;
        while (n < kSelBatch) {
          l = l * S.mult;
          out[n++] = l;
        }
        break;
      }
      case kPhShrink: {
        double l = S.lo;
        while (n < kSelBatch) {
          l = l * S.mult;
          out[n++] = l;
        }
        break;
      }
      default:
        break;
    }
  }
  return n;
}

// Sorts the pending thresholds into S.thr (rank by counting; ties keep
// their order) after sel_batch wrote them to tmp.  All threads of the block.
__device__ void sel_prepare(SelState& S, double* tmp, int* n_s) {
  const int n = sel_batch(S, tmp);
  if (threadIdx.x == 0) *n_s = n;
  __syncthreads();
  const int nb = *n_s;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    const double v = tmp[i];
    int r = 0;
    for (int j = 0; j < nb; ++j) r += (tmp[j] < v) || (tmp[j] == v && j < i);
    S.thr[r] = v;
  }
  if (threadIdx.x == 0) S.nb = nb;
  __syncthreads();
}

// Ticket of the grid: true in the last CTA to arrive (after its partials
// are visible to it).
__device__ bool last_block(unsigned int* ticket, int* flag_s) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) *flag_s = (atomicAdd(ticket, 1u) == gridDim.x - 1u);
  __syncthreads();
  if (!*flag_s) return false;
  __threadfence();
  return true;
}

__device__ __forceinline__ double block_sum(double x, double* red_s) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  __syncthreads();
  if (lane == 0) red_s[w] = x;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red_s[i];
  return t;  // valid in thread 0
}

// Per-thread sums over CTAs of the NC columns of per-CTA partials (rows
// b = threadIdx.x, + blockDim.x, ...), all columns of a row loaded together
// and rows four at a time, so the loads of a thread overlap.  Fixed order.
template <int NC>
__device__ void thread_partials(const double* part, int stride, int nblocks, double (&t)[NC]) {
#pragma unroll
  for (int c = 0; c < NC; ++c) t[c] = 0.0;
  int b = threadIdx.x;
  for (; b + 3 * (int)blockDim.x < nblocks; b += 4 * blockDim.x) {
    double v[4][NC];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int c = 0; c < NC; ++c) v[u][c] = __ldcg(part + (size_t)(b + u * blockDim.x) * stride + c);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int c = 0; c < NC; ++c) t[c] += v[u][c];
  }
  for (; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int c = 0; c < NC; ++c) t[c] += __ldcg(part + (size_t)b * stride + c);
}

__device__ double block_max(double x, double* red_s) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red_s[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) x = fmax(x, red_s[i]);
  return x;  // valid in thread 0
}

// Search state copied between global and shared memory by the whole block.
__device__ void copy_state(SelState* dst, const SelState* src) {
  static_assert(sizeof(SelState) % 4 == 0, "SelState is copied as words");
  const unsigned* a = (const unsigned*)src;
  unsigned* b = (unsigned*)dst;
  for (int i = threadIdx.x; i < (int)(sizeof(SelState) / 4); i += blockDim.x) b[i] = a[i];
}

// Apply date e's frozen decision (depth chain, no shift) to the running
// values and deflate them to date e - 1 when `deflate`
// (updateDeflatedNextStepValuesMulti_gold then
// updateDeflationOfContinuationValues_gold).
__global__ void __launch_bounds__(kNestThreads)
    nested_decide_kernel(const __grid_constant__ LSDate dd, int e, int deflate,
                         const LsRuleView rule, const float* __restrict__ vars,
                         const float* __restrict__ cf, const float* __restrict__ ex,
                         const float* __restrict__ num, float* __restrict__ y, int paths) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths; p += gridDim.x * blockDim.x) {
    float v[kMaxVars];
#pragma unroll
    for (int k = 0; k < kMaxVars; ++k)
      v[k] = k < dd.nvars ? vars[((size_t)e * kMaxVars + k) * paths + p] : 0.0f;
    const float exv = ex ? ex[(size_t)e * paths + p] : 0.0f;
    const double est = ls_chain_estimate(rule, e, dd.nvars, dd.nbasis, dd.mono, v, exv);
    const float t = (cf ? cf[(size_t)e * paths + p] : 0.0f) + y[p];
    float yy = ((double)exv > est) ? exv : t;
    if (deflate) yy = yy * (num[(size_t)(e - 1) * paths + p] / num[(size_t)e * paths + p]);
    y[p] = yy;
  }
}

struct NestArgs {
  LSDate dd;
  int e, d, rows, paths, min_paths, last;
  double lower_frac, upper_frac, sds, mult;
};

// Net values est - exercise value of regression d at date e on its paths
// (d = 0: all; else |net| <= cut of d - 1, net holding d - 1's values),
// +inf elsewhere; the last CTA applies the one-sign shortcut (d = 0) and
// starts the half-width search.
__global__ void __launch_bounds__(kNestThreads, 4)
    nested_net_kernel(const __grid_constant__ NestArgs a, const float* __restrict__ vars,
                      const float* __restrict__ ex, const double* __restrict__ beta,
                      const float* __restrict__ means, const float* __restrict__ sds,
                      const double* __restrict__ cuts, const int* __restrict__ npaths,
                      double* __restrict__ net, double* __restrict__ part,
                      unsigned int* __restrict__ ticket, int* __restrict__ stopped,
                      SelState* __restrict__ state) {
  __shared__ double beta_s[kMaxBasis];
  __shared__ float mom_s[2][kMaxVars];
  __shared__ double red_s[kNestThreads / 32];
  __shared__ SelState S;
  __shared__ double tmp_s[kSelBatch];
  __shared__ int flag_s, n_s;
  const int e = a.e, d = a.d, paths = a.paths, tid = threadIdx.x;
  if (stopped[e]) return;
  const size_t row = (size_t)e * a.rows + d;
  if (tid < kMaxBasis) beta_s[tid] = beta[row * kMaxBasis + tid];
  if (tid < kMaxVars) {
    mom_s[0][tid] = means ? means[row * kMaxVars + tid] : 0.0f;
    mom_s[1][tid] = means ? sds[row * kMaxVars + tid] : 1.0f;
  }
  __syncthreads();
  const double cut = d > 0 ? cuts[(row - 1) * 2 + 1] : 0.0;
  double s1 = 0.0, s2 = 0.0, mx = -INFINITY, mn = INFINITY;
  for (int p = blockIdx.x * blockDim.x + tid; p < paths; p += gridDim.x * blockDim.x) {
    const bool member = d == 0 || fabs(net[p]) <= cut;
    double nv = INFINITY;
    if (member) {
      float v[kMaxVars];
#pragma unroll
      for (int k = 0; k < kMaxVars; ++k)
        v[k] = k < a.dd.nvars ? vars[((size_t)e * kMaxVars + k) * paths + p] : 0.0f;
      const float exv = ex ? ex[(size_t)e * paths + p] : 0.0f;
      nv = ls_row_estimate(beta_s, means ? mom_s[0] : nullptr, mom_s[1], a.dd.nvars,
                           a.dd.nbasis, a.dd.mono, v) -
           (double)exv;
      s1 += nv;
      s2 += nv * nv;
      mx = fmax(mx, nv);
      mn = fmin(mn, nv);
    }
    net[p] = nv;
  }
  const double t1 = block_sum(s1, red_s), t2 = block_sum(s2, red_s);
  // max / min through the same tree (negated min as a max)
  double m1 = mx, m2 = -mn;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m1 = fmax(m1, __shfl_down_sync(0xffffffffu, m1, o));
    m2 = fmax(m2, __shfl_down_sync(0xffffffffu, m2, o));
  }
  __syncthreads();
  if ((tid & 31) == 0) {
    tmp_s[tid >> 5] = m1;
    tmp_s[32 + (tid >> 5)] = m2;
  }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < kNestThreads / 32; ++w) {
      m1 = fmax(m1, tmp_s[w]);
      m2 = fmax(m2, tmp_s[32 + w]);
    }
    double* pb = part + (size_t)blockIdx.x * 4;
    pb[0] = t1;
    pb[1] = t2;
    pb[2] = m1;
    pb[3] = m2;
  }
  if (!last_block(ticket, &flag_s)) return;
  double t4[2];
  thread_partials<2>(part, 4, gridDim.x, t4);
  double mx4 = -INFINITY, mn4 = -INFINITY;
  for (int b = tid; b < (int)gridDim.x; b += blockDim.x) {
    mx4 = fmax(mx4, __ldcg(part + (size_t)b * 4 + 2));
    mn4 = fmax(mn4, __ldcg(part + (size_t)b * 4 + 3));
  }
  const double S1 = block_sum(t4[0], red_s), S2 = block_sum(t4[1], red_s);
  const double MX = block_max(mx4, red_s), MN = -block_max(mn4, red_s);
  for (int i = tid; i < (int)(sizeof(SelState) / 4); i += blockDim.x) ((unsigned*)&S)[i] = 0u;
  __syncthreads();
  if (tid == 0) {
    if (d == 0 && (MX <= 0.0 || MN >= 0.0)) {
      S.phase = kPhDone;
      stopped[e] = 1;
    } else {
      const int n_pre = d == 0 ? paths : npaths[row];
      S.lo_t = (int)(n_pre * a.lower_frac);
      S.hi_t = (int)(n_pre * a.upper_frac);
      S.mult = a.mult;
      if (n_pre > S.lo_t && n_pre < S.hi_t) {
        S.phase = kPhBranch;
      } else {
        const double mean = S1 / n_pre;
        S.g = sqrt(S2 / n_pre - mean * mean) * a.sds;
        S.phase = kPhInit;
      }
    }
    *ticket = 0u;
  }
  __syncthreads();
  if (S.phase != kPhDone) sel_prepare(S, tmp_s, &n_s);
  copy_state(state, &S);
}

// One selection pass: counts of |net| <= each pending threshold, then the
// last CTA advances the search.  When it ends: more than min_paths paths
// selected -> cuts of regression d and the path count of regression d + 1;
// otherwise the date stops nesting.
__global__ void __launch_bounds__(kNestThreads)
    nested_select_kernel(const __grid_constant__ NestArgs a, const double* __restrict__ net,
                         int* __restrict__ hist_g, unsigned int* __restrict__ ticket,
                         int* __restrict__ stopped, SelState* __restrict__ state,
                         double* __restrict__ cuts, int* __restrict__ npaths,
                         int* __restrict__ status) {
  __shared__ double thr_s[kSelBatch];
  __shared__ int hist_s[kSelBatch];
  __shared__ SelState S;
  __shared__ double tmp_s[kSelBatch];
  __shared__ int flag_s, n_s, done_s;
  const int e = a.e, tid = threadIdx.x;
  if (stopped[e]) return;
  const int phase = state->phase, nb = state->nb;
  if (phase == kPhDone) return;
  for (int i = tid; i < kSelBatch; i += blockDim.x) {
    thr_s[i] = i < nb ? state->thr[i] : 0.0;
    hist_s[i] = 0;
  }
  __syncthreads();
  const double top = thr_s[nb - 1];
  for (int p = blockIdx.x * blockDim.x + tid; p < a.paths; p += gridDim.x * blockDim.x) {
    const double x = fabs(net[p]);
    if (!(x <= top)) continue;
    int lo = 0, hi = nb - 1;  // first i with x <= thr[i]
    while (lo < hi) {
      const int m = (lo + hi) >> 1;
      if (x <= thr_s[m])
        hi = m;
      else
        lo = m + 1;
    }
    atomicAdd(&hist_s[lo], 1);
  }
  __syncthreads();
  // integer counts: the totals do not depend on the order of the adds
  for (int i = tid; i < nb; i += blockDim.x)
    if (hist_s[i]) atomicAdd(hist_g + i, hist_s[i]);
  if (!last_block(ticket, &flag_s)) return;
  for (int i = tid; i < nb; i += blockDim.x) {
    hist_s[i] = __ldcg(hist_g + i);
    hist_g[i] = 0;  // zero for the next pass
  }
  copy_state(&S, state);
  __syncthreads();
  if (tid == 0) {
    int run = 0;
    for (int i = 0; i < nb; ++i) {
      run += hist_s[i];
      S.cnt[i] = run;
    }
    const bool done = sel_run(S);
    const size_t row = (size_t)e * a.rows + a.d;
    if (done) {
      if (S.after > a.min_paths) {
        cuts[row * 2] = -S.cut;
        cuts[row * 2 + 1] = S.cut;
        npaths[row + 1] = S.after;
      } else {
        stopped[e] = 1;
      }
    } else if (a.last) {
      S.status |= kSelIncomplete;
      S.phase = kPhDone;
      stopped[e] = 1;
    }
    if (S.status) atomicOr(status, S.status);
    done_s = (S.phase == kPhDone);
    *ticket = 0u;
  }
  __syncthreads();
  if (!done_s) sel_prepare(S, tmp_s, &n_s);
  copy_state(state, &S);
}

// Moments of the basis variables over the paths of regression d (|net| <=
// cut of d - 1): means / sds row e * rows + d (GenerateLSRegressionMatrix
// SelectivelyNormalisingVariables_gold, gold/LS_regression.h:524-600).
__global__ void __launch_bounds__(kNestThreads)
    nested_moments_kernel(const __grid_constant__ NestArgs a, const float* __restrict__ vars,
                          const double* __restrict__ net, const double* __restrict__ cuts,
                          const int* __restrict__ npaths, double* __restrict__ part,
                          unsigned int* __restrict__ ticket, const int* __restrict__ stopped,
                          float* __restrict__ means, float* __restrict__ sds) {
  __shared__ double red_s[kNestThreads / 32];
  __shared__ int flag_s;
  const int e = a.e, tid = threadIdx.x;
  if (stopped[e]) return;
  const size_t row = (size_t)e * a.rows + a.d;
  const double cut = cuts[(row - 1) * 2 + 1];
  double acc[2 * kMaxVars] = {0, 0, 0, 0, 0, 0};
  for (int p = blockIdx.x * blockDim.x + tid; p < a.paths; p += gridDim.x * blockDim.x) {
    if (!(fabs(net[p]) <= cut)) continue;
#pragma unroll
    for (int v = 0; v < kMaxVars; ++v) {
      const double x = v < a.dd.nvars ? vars[((size_t)e * kMaxVars + v) * a.paths + p] : 0.0;
      acc[2 * v] += x;
      acc[2 * v + 1] += x * x;
    }
  }
#pragma unroll
  for (int i = 0; i < 2 * kMaxVars; ++i) {
    const double t = block_sum(acc[i], red_s);
    if (tid == 0) part[(size_t)blockIdx.x * 8 + i] = t;
  }
  if (!last_block(ticket, &flag_s)) return;
  double t6[2 * kMaxVars];
  thread_partials<2 * kMaxVars>(part, 8, gridDim.x, t6);
#pragma unroll
  for (int v = 0; v < kMaxVars; ++v) {
    const double s1 = block_sum(t6[2 * v], red_s);
    const double s2 = block_sum(t6[2 * v + 1], red_s);
    if (tid == 0) {
      double m = 0.0, sd = 1.0;
      if (v < a.dd.nvars) {
        const double n = (double)npaths[row];
        m = s1 / n;
        const double var = s2 / n - m * m;
        sd = var > 0.0 ? sqrt(var) : 1.0;
      }
      means[row * kMaxVars + v] = (float)m;
      sds[row * kMaxVars + v] = (float)sd;
    }
  }
  if (tid == 0) *ticket = 0u;
}

// Path counts: regression 0 of every date uses all paths; the rest start
// at zero.  Rows of nested moments start as (0, 1).
__global__ void nested_init_kernel(int n_ex, int rows, int paths, int* __restrict__ npaths,
                                   float* __restrict__ means, float* __restrict__ sds) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_ex * rows) return;
  npaths[i] = (i % rows == 0) ? paths : 0;
  if (means && i % rows != 0)
    for (int v = 0; v < kMaxVars; ++v) {
      means[(size_t)i * kMaxVars + v] = 0.0f;
      sds[(size_t)i * kMaxVars + v] = 1.0f;
    }
}

}  // namespace

namespace lmm {
int reduce_launch(const float* d_in, const float* d_div, size_t n, double scale,
                  double* d_partials, double* d_out, cudaStream_t stream);
}

namespace {

constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

struct NestWs {
  float* y;
  double* part;          // date kernel: ls_gram_blocks() x kLsMaxPairs
  unsigned int* counter; // date kernel tickets [E]
  double* mom;           // all-path moments: E x blocks x 6
  double* red;           // final reduction
  double* net;           // [P]
  double* npart;         // net / moments partials: blocks x 8
  int* hist;             // selection histogram [kSelBatch], zero between passes
  unsigned int* tickets; // [4]
  SelState* state;
  int* stopped;          // [E]
  int* npaths;           // [E][kMaxDepth]
};

// CTAs of the net, selection and moments passes: up to kNestCtasPerSm per
// SM, enough warps in flight for these latency-bound streaming passes.
constexpr int kNestCtasPerSm = 8;
int nest_grid(int paths) {
  return std::max(1, std::min(div_up(paths, kNestThreads), kNestCtasPerSm * ls_gram_blocks()));
}

size_t nested_ws_bytes(int paths, int n_ex, NestWs* w, char* base) {
  const size_t nb = (size_t)ls_gram_blocks();
  const size_t ng = (size_t)kNestCtasPerSm * nb;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + off : nullptr;
    off += align256(bytes);
    return p;
  };
  NestWs t;
  t.y = (float*)take((size_t)paths * sizeof(float));
  t.part = (double*)take(nb * kLsMaxPairs * sizeof(double));
  t.counter = (unsigned int*)take((size_t)n_ex * sizeof(unsigned int));
  t.mom = (double*)take((size_t)n_ex * nb * 6 * sizeof(double));
  t.red = (double*)take(512 * sizeof(double));
  t.net = (double*)take((size_t)paths * sizeof(double));
  t.npart = (double*)take(ng * 8 * sizeof(double));
  t.hist = (int*)take(kSelBatch * sizeof(int));
  t.tickets = (unsigned int*)take(4 * sizeof(unsigned int));
  t.state = (SelState*)take(sizeof(SelState));
  t.stopped = (int*)take((size_t)n_ex * sizeof(int));
  t.npaths = (int*)take((size_t)n_ex * kMaxDepth * sizeof(int));
  if (w) *w = t;
  return off + 256;
}

}  // namespace

extern "C" size_t lmm_ls_nested_workspace_bytes(int paths, int n_exercise) {
  if (paths < 1 || n_exercise < 1) return 0;
  return nested_ws_bytes(paths, n_exercise, nullptr, nullptr);
}

extern "C" int lmm_ls_regress_nested(int n_exercise, int paths, const float* d_vars,
                                     const int* h_nvars, const uint8_t* h_monomials,
                                     const int* h_nbasis, const float* d_cf, const float* d_ex,
                                     const float* d_num, int normalise,
                                     const lmm_ls_select* sel, void* d_workspace,
                                     size_t workspace_bytes, double* d_beta, float* d_means,
                                     float* d_sds, double* d_cuts, int* d_npaths,
                                     int* d_status, double* d_price, lmm_stream_t stream) {
  LMM_REQUIRE(n_exercise >= 1 && n_exercise <= kMaxSteps && paths >= 1,
              "lmm_ls_regress_nested: bad sizes");
  LMM_REQUIRE(d_vars && h_nvars && h_monomials && h_nbasis && d_num && d_workspace && d_beta &&
                  d_cuts && d_status && d_price && sel,
              "lmm_ls_regress_nested: null pointer");
  LMM_REQUIRE(!normalise || (d_means && d_sds),
              "lmm_ls_regress_nested: normalise needs means/sds outputs");
  const int D = sel->depth;
  LMM_REQUIRE(D >= 1 && D <= kMaxDepth, "lmm_ls_regress_nested: depth %d outside 1..%d", D,
              kMaxDepth);
  LMM_REQUIRE(sel->lower_frac > 0.0 && sel->upper_frac > sel->lower_frac &&
                  sel->upper_frac <= 1.0,
              "lmm_ls_regress_nested: need 0 < lower_frac < upper_frac <= 1");
  LMM_REQUIRE(sel->sds > 0.0 && sel->multiplier > 0.0 && sel->multiplier < 1.0 &&
                  sel->min_paths >= 0,
              "lmm_ls_regress_nested: need sds > 0, 0 < multiplier < 1, min_paths >= 0");
  const size_t need = nested_ws_bytes(paths, n_exercise, nullptr, nullptr);
  LMM_REQUIRE(workspace_bytes >= need, "lmm_ls_regress_nested: workspace too small (%zu < %zu)",
              workspace_bytes, need);
  cudaStream_t s = (cudaStream_t)stream;
  NestWs w;
  nested_ws_bytes(paths, n_exercise, &w,
                  (char*)(((uintptr_t)d_workspace + 255) & ~(uintptr_t)255));
  LSBasisSpec spec{h_nvars, h_monomials, h_nbasis};
  std::vector<LSDate> dates(n_exercise);
  for (int e = 0; e < n_exercise; ++e) TRY(ls_fill_date(spec, e, &dates[e]));
  int* npaths = d_npaths ? d_npaths : w.npaths;
  const size_t rows = (size_t)n_exercise * D;

  TRY(check_cuda(cudaMemsetAsync(d_status, 0, sizeof(int), s), "nested: status"));
  TRY(check_cuda(cudaMemsetAsync(w.counter, 0, (size_t)n_exercise * sizeof(unsigned int), s),
                 "nested: counters"));
  TRY(check_cuda(cudaMemsetAsync(w.tickets, 0, 4 * sizeof(unsigned int), s), "nested: tickets"));
  TRY(check_cuda(cudaMemsetAsync(w.hist, 0, kSelBatch * sizeof(int), s), "nested: histogram"));
  TRY(check_cuda(cudaMemsetAsync(w.stopped, 0, (size_t)n_exercise * sizeof(int), s),
                 "nested: flags"));
  TRY(check_cuda(cudaMemsetAsync(d_cuts, 0, rows * 2 * sizeof(double), s), "nested: cuts"));
  TRY(check_cuda(cudaMemsetAsync(d_beta, 0, rows * kMaxBasis * sizeof(double), s),
                 "nested: coefficients"));
  TRY(check_cuda(cudaMemsetAsync(w.y, 0, (size_t)paths * sizeof(float), s), "nested: values"));
  nested_init_kernel<<<div_up((int)rows, 128), 128, 0, s>>>(
      n_exercise, D, paths, npaths, normalise ? d_means : nullptr, normalise ? d_sds : nullptr);
  TRY(check_launch("nested_init_kernel"));
  const float* means = nullptr;
  const float* sds = nullptr;
  if (normalise) {
    TRY(ls_moments_launch(d_vars, paths, n_exercise, D, d_means, d_sds, w.mom, s));
    means = d_means;
    sds = d_sds;
  }
  const int nblk = ls_gram_blocks();
  const int grid_path = grid_for(paths, kNestThreads, 4);
  const int grid_nest = nest_grid(paths);
  const LsRuleView rule{D, d_beta, means, sds, D > 1 ? d_cuts : nullptr, nullptr};
  for (int e = n_exercise - 1; e >= 0; --e) {
    if (e + 1 < n_exercise) {
      nested_decide_kernel<<<grid_path, kNestThreads, 0, s>>>(
          dates[e + 1], e + 1, 1, rule, d_vars, d_cf, d_ex, d_num, w.y, paths);
      TRY(check_launch("nested_decide_kernel"));
    }
    const int slots = dates[e].nbasis + 1;
    const int per_cta = slots <= 11 ? 512 : slots <= 13 ? 256 : 192;
    const int grid_date = std::min(div_up(paths, per_cta), nblk);
    for (int d = 0; d < D; ++d) {
      NestArgs a;
      memset(&a, 0, sizeof(a));
      a.dd = dates[e];
      a.e = e;
      a.rows = D;
      a.paths = paths;
      a.min_paths = sel->min_paths;
      a.lower_frac = sel->lower_frac;
      a.upper_frac = sel->upper_frac;
      a.sds = sel->sds;
      a.mult = sel->multiplier;
      if (d > 0) {
        // net values of regression d - 1, then the search for its cuts
        a.d = d - 1;
        nested_net_kernel<<<grid_nest, kNestThreads, 0, s>>>(
            a, d_vars, d_ex, d_beta, means, sds, d_cuts, npaths, w.net, w.npart, w.tickets + 0,
            w.stopped, w.state);
        TRY(check_launch("nested_net_kernel"));
        for (int pass = 0; pass < kSelPasses; ++pass) {
          a.last = pass + 1 == kSelPasses;
          nested_select_kernel<<<grid_nest, kNestThreads, 0, s>>>(
              a, w.net, w.hist, w.tickets + 1, w.stopped, w.state, d_cuts, npaths, d_status);
          TRY(check_launch("nested_select_kernel"));
        }
        a.d = d;
        a.last = 0;
        if (normalise) {
          nested_moments_kernel<<<grid_nest, kNestThreads, 0, s>>>(
              a, d_vars, w.net, d_cuts, npaths, w.npart, w.tickets + 2, w.stopped, d_means,
              d_sds);
          TRY(check_launch("nested_moments_kernel"));
        }
      }
      LSDateParams P;
      memset(&P, 0, sizeof(P));
      P.e = e;
      P.paths = paths;
      P.cur = dates[e];
      P.has_prev = 0;
      P.read_y = 1;
      P.rows = D;
      P.depth = d;
      if (d > 0) {
        P.mask_net = w.net;
        P.mask_cut = d_cuts + ((size_t)e * D + d - 1) * 2 + 1;
        P.mask_count = npaths + (size_t)e * D + d;
        P.skip = w.stopped + e;
      }
      TRY(launch_date(P, grid_date, d_vars, means, sds, d_cf, d_ex, d_num, d_beta, w.y, w.part,
                      w.counter, nullptr, d_status, nullptr, s));
    }
  }
  nested_decide_kernel<<<grid_path, kNestThreads, 0, s>>>(dates[0], 0, 0, rule, d_vars, d_cf,
                                                          d_ex, d_num, w.y, paths);
  TRY(check_launch("nested_decide_kernel"));
  return reduce_launch(w.y, d_num, (size_t)paths, 1.0 / (double)paths, w.red, d_price, s);
}
