// ls.cu — Longstaff–Schwartz backward induction kept on the device.
//
// Reference behaviour followed (regression depth 1):
//   backward loop        gold/MultiLS_regression.cpp:101-417 and the GPU
//                        orchestration LS_main_cula.h:565-837
//   regression matrix    GenerateLSRegressionMatrixSelectively_gold
//                        (gold/LS_regression.h:431-530): G = E[phi phi^T],
//                        b = E[phi (cf + y)], both divided by the path count
//   exercise update      updateDeflatedNextStepValuesMulti_gold
//                        (gold/MultiLS_regression.h:42-99)
//   deflation            updateDeflationOfContinuationValues_gold
//                        (gold/LS_regression.cpp:98-118): y *= N_{e-1}/N_e
//   basis functions      quadraticPolynomialGenerator /
//                        quadraticPolynomialCrossGenerator
//                        (gold/LS_regression.h:123-240) expressed as monomial
//                        exponent tables, one table per exercise date
//   in-sample price      mean_p y_p / N_0(p)  (MultiLS_regression.cpp:407-416)
// The reference solves each normal-equation system on the host by SVD after
// a device-to-host copy (LinearSolverConcrete_main.cu:127-188); here each
// date is one kernel: the Gram sums stay on the device and the last CTA of
// the launch solves them with a warp-parallel FP64 Cholesky, so the loop is
// launch-only (one launch per date) and can be captured in a graph.
#include "lmm_common.cuh"
#include "lmm_device.cuh"
#include "ls_common.cuh"

#include <mutex>
#include <vector>

using namespace lmm;

namespace lmm {
int reduce_launch(const float* d_in, const float* d_div, size_t n,
                  double scale, double* d_partials, double* d_out,
                  cudaStream_t stream);

// Shuffle-down of a double whose two halves move in program order
// (volatile), so a sequence of these is never interleaved by the scheduler.
__device__ __forceinline__ double shfl_down_d_ordered(double x, int o) {
  unsigned lo, hi;
  asm volatile("mov.b64 {%0, %1}, %2;" : "=r"(lo), "=r"(hi) : "d"(x));
  asm volatile("shfl.sync.down.b32 %0, %0, %1, 0x1f, 0xffffffff;" : "+r"(lo) : "r"(o));
  asm volatile("shfl.sync.down.b32 %0, %0, %1, 0x1f, 0xffffffff;" : "+r"(hi) : "r"(o));
  double y;
  asm volatile("mov.b64 %0, {%1, %2};" : "=d"(y) : "r"(lo), "r"(hi));
  return y;
}

__device__ __forceinline__ double warp_sum_d(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  return x;
}

}  // namespace lmm

// Apply the frozen decision of date d to one path and deflate to date d-1,
// from the path's values: xin[v] (v < nvars) the basis variables at d, cf_v
// and ex_v the coupon and exercise value at d, num_prev / num_cur the
// numeraires at d-1 and d, y_in the running value.  beta_d: the date's
// coefficients; mean_d / sd_d: its standardisation (or null).
template <int KIND>
__device__ __forceinline__ float decide_values(const LSDate& dd, int deflate, const float* xin,
                                               const float* mean_d, const float* sd_d,
                                               float cf_v, float ex_v, float num_prev,
                                               float num_cur, const double* beta_d,
                                               float y_in) {
  float x[kMaxVars];
#pragma unroll
  for (int v = 0; v < kMaxVars; ++v) {
    float xv = 0.0f;
    if (v < dd.nvars) {
      xv = xin[v];
      if (mean_d) xv = (xv - mean_d[v]) * sd_d[v];  // sd_d holds 1 / sd
    }
    x[v] = xv;
  }
  float pw[kMaxVars][3];
  ls_powers(x, pw);
  // coefficients re-read per path (volatile) rather than held in 32 registers
  const volatile double* bv = beta_d;
  double est = 0.0;
#pragma unroll
  for (int k = 0; k < kMaxBasis; ++k)
    if (k < (KIND ? basis_K(KIND) : dd.nbasis))
      est += (double)ls_basis<KIND>(pw, dd, k) * bv[k];
  const float t = cf_v + y_in;
  float y = ((double)ex_v > est) ? ex_v : t;
  if (deflate) y = y * (num_prev / num_cur);
  return y;
}

// The same from the arrays of the LS inputs, for path p.
template <int KIND>
__device__ __forceinline__ float apply_decision(
    const LSDate& dd, int d, int deflate, const float* __restrict__ vars,
    const float* mean_d, const float* sd_d, const float* __restrict__ cf,
    const float* __restrict__ ex, const float* __restrict__ num,
    const double* beta_d, float y_in, int paths, int p) {
  float xin[kMaxVars];
#pragma unroll
  for (int v = 0; v < kMaxVars; ++v)
    xin[v] = v < dd.nvars ? vars[((size_t)d * kMaxVars + v) * paths + p] : 0.0f;
  const float cf_v = cf ? cf[(size_t)d * paths + p] : 0.0f;
  const float ex_v = ex ? ex[(size_t)d * paths + p] : 0.0f;
  const float np = deflate ? num[(size_t)(d - 1) * paths + p] : 1.0f;
  const float nc = deflate ? num[(size_t)d * paths + p] : 1.0f;
  return decide_values<KIND>(dd, deflate, xin, mean_d, sd_d, cf_v, ex_v, np, nc, beta_d, y_in);
}

// ---------------------------------------------------------------------------
// One backward date e as one kernel.
//
// Each thread walks its paths (grid stride): it applies date e+1's frozen
// decision (updating the running value y), evaluates the KR - 1 basis slots
// of date e (slots at and above nbasis are zero) and the regression target
// cf_e + y in slot KR - 1, and adds the products of the lower triangle
// (i, j), j <= i < KR, into registers: q(i, j) = i (i + 1) / 2 + j.  With
// NSPLIT = 2 the rows are split between the two warps of a warp pair, which
// handle the same 32 paths, so no thread holds more than 78 sums.  Sums
// within a warp (a few paths per thread, then a fixed shuffle tree over
// its 32 threads) are FP32; everything above them is FP64: a fixed-order
// sum over warps, a partial per CTA in part[q][cta] and the sum over CTAs.  The CTA that finishes last (ticket on
// counter[e]) sums the partials in a fixed order and solves the normal
// equations with a one-warp FP64 Cholesky, so the date needs one launch and
// the result is independent of which CTA came last.
//
// Sums over paths of the reference: GenerateLSRegressionMatrixSelectively_gold
// (gold/LS_regression.h:431-530); its host SVD solve
// (LinearSolverConcrete_main.cu:127-188) is replaced by the Cholesky below.
// ---------------------------------------------------------------------------
// 512 threads per CTA; 384 for 17 slots (78 sums per thread need more than
// the 128 registers a 512-thread CTA allows).
template <int KR>
struct LsThreads {
  static constexpr int value = KR > 13 ? 384 : 512;
};


// rows [R0, R1) of the lower triangle
template <int KR, int R0, int R1>
struct RowSplit {
  static constexpr int q0 = R0 * (R0 + 1) / 2;
  static constexpr int n = R1 * (R1 + 1) / 2 - q0;
};

template <int KR, int NSPLIT>
struct SplitOf;
template <int KR>
struct SplitOf<KR, 1> {
  static constexpr int rs = KR;  // one half: all rows
};
// balance R(R+1)/2 against the rest
template <int KR>
struct SplitOf<KR, 2> {
  static constexpr int rs = KR == 17 ? 12 : KR == 13 ? 9 : (KR * 7) / 10;
};

template <int KR, int R0, int R1>
__device__ __forceinline__ void accumulate_rows(const float* phi, float* acc) {
#pragma unroll
  for (int i = R0; i < R1; ++i)
#pragma unroll
    for (int j = 0; j <= i; ++j)
      acc[i * (i + 1) / 2 + j - RowSplit<KR, R0, R1>::q0] += phi[i] * phi[j];
}

// Warp-parallel FP64 Cholesky solve of G beta = b (K <= 16): lane i holds
// row i of G.  A relative diagonal jitter is added and the factorisation
// retried when a pivot fails.  Each column takes one reciprocal square root
// r_j = 1 / sqrt(d_jj): L_jj = d_jj r_j and the column below is scaled by
// r_j, and both substitutions multiply by the kept r_j instead of dividing.
// The back substitution runs by columns of L^T from a shared-memory copy of
// L (Ls, kMaxBasis^2 doubles of scratch).  Returns status bits (1: zero
// diagonal, 2: not positive definite after jitter, 4: jitter added); beta
// is zero on failure.
__device__ int warp_cholesky_solve(const double* Gs, int K, double* beta_out, double* Ls) {
  const int lane = threadIdx.x & 31;
  if (lane < kMaxBasis) beta_out[lane] = 0.0;
  double maxd = 0.0;
  for (int i = 0; i < K; ++i) maxd = fmax(maxd, fabs(Gs[i * kLsMaxSlots + i]));
  if (!(maxd > 0.0)) return 1;
  double jitter = 0.0;
  int status = 0;
  double a[kMaxBasis];
  double rinv = 0.0;  // this lane's 1 / L_ii
  bool ok = false;
  for (int attempt = 0; attempt < 6 && !ok; ++attempt) {
#pragma unroll
    for (int k = 0; k < kMaxBasis; ++k)
      a[k] = (lane < K && k <= lane) ? Gs[lane * kLsMaxSlots + k] +
                                          ((k == lane) ? jitter : 0.0)
                                     : 0.0;
    ok = true;
#pragma unroll
    for (int j = 0; j < kMaxBasis; ++j) {
      if (j < K) {
        const double djj = __shfl_sync(0xffffffffu, a[j], j);
        if (!(djj > 1e-300)) {
          ok = false;
          break;
        }
        const double rj = rsqrt(djj);
        if (lane == j) {
          a[j] = djj * rj;
          rinv = rj;
        }
        if (lane > j) a[j] *= rj;
        // trailing update: a[i][k] -= L[i][j] L[k][j] for j < k <= i
#pragma unroll
        for (int k = j + 1; k < kMaxBasis; ++k) {
          if (k < K) {
            const double lkj = __shfl_sync(0xffffffffu, a[j], k);
            if (lane >= k) a[k] -= a[j] * lkj;
          }
        }
      }
    }
    if (!ok) jitter = (jitter == 0.0) ? 1e-14 * maxd : jitter * 100.0;
  }
  if (!ok) return 2;
  if (jitter > 0.0) status |= 4;
  // forward substitution L z = b: z_j = (b_j - sum_{k<j} L_jk z_k) r_j
  double z = (lane < K) ? Gs[lane * kLsMaxSlots + kLsMaxSlots - 1] : 0.0;
#pragma unroll
  for (int j = 0; j < kMaxBasis; ++j) {
    if (j < K) {
      const double zj = __shfl_sync(0xffffffffu, z * rinv, j);
      if (lane == j) z = zj;
      if (lane > j) z -= a[j] * zj;
    }
  }
  // back substitution L^T beta = z by columns: lane k holds column k of L
  // (L_ik, i > k) and subtracts L_ik beta_i once beta_i is known
  if (lane < K) {
#pragma unroll
    for (int k = 0; k < kMaxBasis; ++k) Ls[lane * kMaxBasis + k] = a[k];
  }
  __syncwarp();
  double lcol[kMaxBasis];
#pragma unroll
  for (int i = 0; i < kMaxBasis; ++i)
    lcol[i] = (lane < K && i < K && i > lane) ? Ls[i * kMaxBasis + lane] : 0.0;
  __syncwarp();
  double bet = 0.0;
#pragma unroll
  for (int i = kMaxBasis - 1; i >= 0; --i) {
    if (i < K) {
      const double bi = __shfl_sync(0xffffffffu, z * rinv, i);
      if (lane == i) bet = bi;
      if (lane < i) z -= lcol[i] * bi;
    }
  }
  if (lane < kMaxBasis) beta_out[lane] = (lane < K) ? bet : 0.0;
  return status;
}

// Staged loop of the date kernel: the inputs of a path, one shared-memory
// row each, in kLsStages slots per thread (masked launches also stage the
// path's membership value).  Rows: basis variables at e (3), coupon at e, running value y,
// basis variables at e+1 (3), coupon and exercise value at e+1, numeraires
// at e and e+1.
constexpr int kLsStages = 4;
constexpr int kLsInputs = 12;
constexpr int kInX = 0, kInCf = 3, kInY = 4, kInXNext = 5, kInCfNext = 8, kInExNext = 9,
              kInNum = 10, kInNumNext = 11;
// masked launches also stage each path's membership value (mask_net, FP64)
// after the input rows: [kLsStages][threads] doubles
template <int KR, int NSPLIT, bool MASKED>
constexpr size_t ls_stage_bytes() {
  return (size_t)kLsStages * LsThreads<KR>::value *
         (kLsInputs * sizeof(float) + (MASKED ? sizeof(double) : 0));
}

__device__ __forceinline__ void cp_async4(float* dst_smem, const float* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(float* dst_smem, const float* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(double* dst_smem, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int KR, int NSPLIT, int KIND, bool MASKED>
__global__ void __launch_bounds__(LsThreads<KR>::value, 1)
    ls_date_kernel(const __grid_constant__ LSDateParams P,
                   const float* __restrict__ vars,
                   const float* __restrict__ means,
                   const float* __restrict__ sds, const float* __restrict__ cf,
                   const float* __restrict__ ex, const float* __restrict__ num,
                   double* __restrict__ beta, float* __restrict__ y,
                   double* __restrict__ part, unsigned int* __restrict__ counter,
                   double* __restrict__ gram_out, int* __restrict__ status,
                   double* __restrict__ sums_out) {
  constexpr int RS = SplitOf<KR, NSPLIT>::rs;
  constexpr int NA0 = RowSplit<KR, 0, RS>::n;
  constexpr int NA1 = RowSplit<KR, RS, KR>::n;
  constexpr int NA = NA0 > NA1 ? NA0 : NA1;
  constexpr int NPAIRS = KR * (KR + 1) / 2;
  constexpr int kLsThreads = LsThreads<KR>::value;
  constexpr int NW = kLsThreads / 32;
  __shared__ double beta_prev[kMaxBasis];
  __shared__ float mom_s[4][kMaxVars];  // mean, 1/sd of date e, then of e+1
  __shared__ double red_s[NW][NA];
  __shared__ double share_s[kLsThreads];
  __shared__ double sums_s[NPAIRS];
  __shared__ double G_s[kLsMaxSlots * kLsMaxSlots];
  __shared__ int last_s;
  __shared__ const float* src_s[kLsInputs];  // input rows of the staged loop
  extern __shared__ float ls_stage[];        // [kLsStages][kLsInputs][threads]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int e = P.e, paths = P.paths;
  if (P.skip && *P.skip) return;
  const int rows = P.rows > 0 ? P.rows : 1;
  const size_t row = (size_t)e * rows + P.depth, prev_row = (size_t)(e + 1) * rows;
  const double cut = MASKED ? *P.mask_cut : 0.0;
  if (tid < kMaxBasis)
    beta_prev[tid] = P.has_prev ? beta[prev_row * kMaxBasis + tid] : 0.0;
  if (tid < kLsInputs) {
    const size_t cur = (size_t)e * paths, nxt = cur + paths;
    const float* sp = nullptr;
    if (tid < kInCf) {
      if (tid < P.cur.nvars) sp = vars + ((size_t)e * kMaxVars + tid) * paths;
    } else if (tid == kInCf) {
      sp = cf ? cf + cur : nullptr;
    } else if (tid == kInY) {
      sp = (P.has_prev || P.read_y) ? y : nullptr;
    } else if (P.has_prev) {
      if (tid < kInCfNext) {
        const int v = tid - kInXNext;
        if (v < P.prev.nvars) sp = vars + ((size_t)(e + 1) * kMaxVars + v) * paths;
      } else if (tid == kInCfNext) {
        sp = cf ? cf + nxt : nullptr;
      } else if (tid == kInExNext) {
        sp = ex ? ex + nxt : nullptr;
      } else if (tid == kInNum) {
        sp = num + cur;
      } else {
        sp = num + nxt;
      }
    }
    src_s[tid] = sp;
  }
  if (tid < kMaxVars && means) {
    mom_s[0][tid] = means[row * kMaxVars + tid];
    mom_s[1][tid] = 1.0f / sds[row * kMaxVars + tid];
    if (P.has_prev) {
      mom_s[2][tid] = means[prev_row * kMaxVars + tid];
      mom_s[3][tid] = 1.0f / sds[prev_row * kMaxVars + tid];
    }
  }
  __syncthreads();
  const int half = (NSPLIT == 2) ? (warp & 1) : 0;
  const int per_cta = kLsThreads / NSPLIT;
  const int K = P.cur.nbasis;
  float acc[NA];
#pragma unroll
  for (int q = 0; q < NA; ++q) acc[q] = 0.0f;
  const int stride = gridDim.x * per_cta;
  // the Gram products of one path from its basis variables at date e, its
  // coupon at e and its running value
  auto accumulate_path = [&](const float* xe, float cfe, float yp) {
    float x[kMaxVars];
#pragma unroll
    for (int v = 0; v < kMaxVars; ++v) {
      float xv = 0.0f;
      if (v < P.cur.nvars) {
        xv = xe[v];
        if (means) xv = (xv - mom_s[0][v]) * mom_s[1][v];
      }
      x[v] = xv;
    }
    float pw[kMaxVars][3];
    ls_powers(x, pw);
    float phi[KR];
#pragma unroll
    for (int k = 0; k < KR - 1; ++k)
      phi[k] = (k < (KIND ? basis_K(KIND) : K)) ? ls_basis<KIND>(pw, P.cur, k) : 0.0f;
    phi[KR - 1] = cfe + yp;
    if (half == 0)
      accumulate_rows<KR, 0, RS>(phi, acc);
    else
      accumulate_rows<KR, RS, KR>(phi, acc);
  };
  {
    // The loop is bound by memory latency: the inputs of each path are
    // copied kLsStages - 1 iterations ahead into shared memory (cp.async, no
    // registers held), one row of the stage per input.  When every input
    // row is 16-byte aligned (paths a multiple of 4) the warp copies its 32
    // paths' rows in 16-byte chunks, lane l taking chunk l % 8 of rows
    // l / 8, l / 8 + 4 and l / 8 + 8; otherwise each thread copies its own
    // path's values.  The loop runs whole warps (a lane past the last path
    // still copies and waits, but adds nothing).  With rows split over a
    // warp pair both warps take the same 32 paths, each staging its own copy.
    const bool vec16 = P.vec16 != 0;
    const int r0 = lane >> 3, c4 = (lane & 7) * 4;
    const float* const rp0 = src_s[r0];
    const float* const rp1 = src_s[r0 + 4];
    const float* const rp2 = src_s[r0 + 8];
    float* const wstage = ls_stage + warp * 32;
    double* const mstage = reinterpret_cast<double*>(ls_stage + kLsStages * kLsInputs * kLsThreads);
    auto issue = [&](int it, int qw) {  // qw: the warp's first path
      float* dst = wstage + (it & (kLsStages - 1)) * kLsInputs * kLsThreads;
      if (MASKED && qw + lane < paths)
        cp_async8(mstage + (it & (kLsStages - 1)) * kLsThreads + tid, P.mask_net + qw + lane);
      if (vec16) {
        const int qb = qw + c4;
        if (qb < paths) {
          if (rp0) cp_async16(dst + r0 * kLsThreads + c4, rp0 + qb);
          if (rp1) cp_async16(dst + (r0 + 4) * kLsThreads + c4, rp1 + qb);
          if (rp2) cp_async16(dst + (r0 + 8) * kLsThreads + c4, rp2 + qb);
        }
      } else if (qw + lane < paths) {
#pragma unroll
        for (int i = 0; i < kLsInputs; ++i)
          if (src_s[i]) cp_async4(dst + i * kLsThreads + lane, src_s[i] + qw + lane);
      }
      cp_async_commit();
    };
    const int w0 = blockIdx.x * per_cta + (warp / NSPLIT) * 32;
#pragma unroll
    for (int k = 0; k < kLsStages - 1; ++k) issue(k, w0 + k * stride);
    int it = 0;
    for (int qw = w0; qw < paths; qw += stride, ++it) {
      issue(it + kLsStages - 1, qw + (kLsStages - 1) * stride);
      cp_async_wait<kLsStages - 1>();
      __syncwarp();
      const int p = qw + lane;
      const bool member =
          !MASKED || (p < paths && fabs(mstage[(it & (kLsStages - 1)) * kLsThreads + tid]) <= cut);
      if (p < paths && member) {
        const float* in = wstage + (it & (kLsStages - 1)) * kLsInputs * kLsThreads + lane;
        float yp = 0.0f;
        if (P.has_prev) {
          float xp[kMaxVars];
#pragma unroll
          for (int v = 0; v < kMaxVars; ++v)
            xp[v] = v < P.prev.nvars ? in[(kInXNext + v) * kLsThreads] : 0.0f;
          yp = decide_values<KIND>(P.prev, 1, xp, means ? mom_s[2] : nullptr, mom_s[3],
                                   cf ? in[kInCfNext * kLsThreads] : 0.0f,
                                   ex ? in[kInExNext * kLsThreads] : 0.0f,
                                   in[kInNum * kLsThreads], in[kInNumNext * kLsThreads],
                                   beta_prev, in[kInY * kLsThreads]);
        } else if (P.read_y) {
          yp = in[kInY * kLsThreads];
        }
        if (half == 0 && !P.read_y) y[p] = yp;
        float xe[kMaxVars];
#pragma unroll
        for (int v = 0; v < kMaxVars; ++v)
          xe[v] = v < P.cur.nvars ? in[(kInX + v) * kLsThreads] : 0.0f;
        accumulate_path(xe, cf ? in[kInCf * kLsThreads] : 0.0f, yp);
      }
      // every lane's reads of this stage precede its refill, issued by
      // other lanes in a later iteration
      __syncwarp();
    }
    cp_async_wait<0>();
  }
  // warp sums (a fixed shuffle tree), then FP64 over warps in a fixed
  // order.  All-path launches sum within the warp in FP32 (each thread
  // holds several paths' FP32 sums already).  Masked launches (nested
  // regressions on a subset, about one path per thread) sum in FP64, one
  // accumulator at a time: their Grams are close to singular, and the FP32
  // tree would be their largest rounding error.
  if (MASKED) {
#pragma unroll
    for (int q = 0; q < NA; ++q) {
      double t;
      asm volatile("cvt.f64.f32 %0, %1;" : "=d"(t) : "f"(acc[q]));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += shfl_down_d_ordered(t, o);
      if (lane == 0) red_s[warp][q] = t;
    }
  } else {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int q = 0; q < NA; ++q) acc[q] += __shfl_down_sync(0xffffffffu, acc[q], o);
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < NA; ++q) red_s[warp][q] = (double)acc[q];
  }
  __syncthreads();
  const int nb = gridDim.x;
  for (int q = tid; q < NPAIRS; q += kLsThreads) {
    const int h = (q < RowSplit<KR, 0, RS>::n) ? 0 : 1;
    const int qq = h ? q - RowSplit<KR, 0, RS>::n : q;
    double s = 0.0;
    for (int w = h; w < NW; w += NSPLIT) s += red_s[w][qq];
    part[(size_t)q * nb + blockIdx.x] = s;
  }
  // last CTA: sum the partials and solve.  The CTA barrier orders every
  // thread's partial writes before thread 0's device-scope fence and ticket
  // (the fence is cumulative), so the other threads do not wait for their
  // own outstanding stores of y here.
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    last_s = (atomicAdd(counter + e, 1u) == (unsigned)nb - 1u);
  }
  __syncthreads();
  if (!last_s) return;
  __threadfence();
  // tpq threads per pair, each summing a strided share of the CTA partials
  // with its loads unrolled (one pass of L2 latency, not one per partial),
  // then the shares of a pair in a fixed order
  {
    const int tpq = kLsThreads / NPAIRS;
    double* share = share_s;
    const int q = tid / tpq, sub = tid - q * tpq;
    double v = 0.0;
    if (q < NPAIRS) {
      const double* src = part + (size_t)q * nb;
#pragma unroll 8
      for (int b = sub; b < nb; b += tpq) v += __ldcg(src + b);
    }
    __syncthreads();
    share[tid] = v;
    __syncthreads();
    if (tid < NPAIRS) {
      double t = 0.0;
      for (int k = 0; k < tpq; ++k) t += share[tid * tpq + k];
      sums_s[tid] = t;
    }
  }
  __syncthreads();
  if (sums_out) {
    // sharded regression: this GPU's unscaled sums, packed over the slots
    // 0..K (slot K = the target) as (i, j), j <= i, at i (i + 1) / 2 + j
    const int npub = (K + 1) * (K + 2) / 2;
    for (int idx = tid; idx < npub; idx += kLsThreads) {
      int i = 0;
      while ((i + 1) * (i + 2) / 2 <= idx) ++i;
      const int j = idx - i * (i + 1) / 2;
      const int ii = (i == K) ? KR - 1 : i, jj = (j == K) ? KR - 1 : j;
      sums_out[idx] = sums_s[ii * (ii + 1) / 2 + jj];
    }
    if (tid == 0) counter[e] = 0u;
    return;
  }
  const double n_div = MASKED ? (double)*P.mask_count : (double)paths;
  for (int q = tid; q < NPAIRS; q += kLsThreads) sums_s[q] /= n_div;
  __syncthreads();
  // G_s[i][j] (i, j < K) and the right-hand side in column kLsMaxSlots - 1
  for (int idx = tid; idx < kLsMaxSlots * kLsMaxSlots; idx += kLsThreads) {
    const int i = idx / kLsMaxSlots, j = idx - i * kLsMaxSlots;
    double v = 0.0;
    if (i < K && j < K) {
      const int a = i > j ? i : j, b = i > j ? j : i;
      v = sums_s[a * (a + 1) / 2 + b];
    } else if (i < K && j == kLsMaxSlots - 1) {
      v = sums_s[(KR - 1) * KR / 2 + i];
    }
    G_s[idx] = v;
  }
  __syncthreads();
  if (gram_out) {
    double* g = gram_out + (size_t)e * kMaxBasis * (kMaxBasis + 1);
    for (int idx = tid; idx < K * (kMaxBasis + 1); idx += kLsThreads) {
      const int i = idx / (kMaxBasis + 1), j = idx - i * (kMaxBasis + 1);
      double v = 0.0;
      if (j < K)
        v = G_s[i * kLsMaxSlots + j];
      else if (j == K)
        v = G_s[i * kLsMaxSlots + kLsMaxSlots - 1];
      g[idx] = v;
    }
  }
  if (warp == 0) {
    const int st = warp_cholesky_solve(G_s, K, beta + row * kMaxBasis, share_s);
    if (lane == 0) {
      if (st) atomicOr(status, st);
      counter[e] = 0u;
    }
  }
}

// Final decision at date 0 (no deflation): y holds the value at date 0.
__global__ void ls_final_kernel(const __grid_constant__ LSDateParams P,
                                const float* __restrict__ vars,
                                const float* __restrict__ means,
                                const float* __restrict__ sds,
                                const float* __restrict__ cf,
                                const float* __restrict__ ex,
                                const float* __restrict__ num,
                                const double* __restrict__ beta,
                                float* __restrict__ y) {
  __shared__ double beta0[kMaxBasis];
  __shared__ float mom0[2][kMaxVars];
  if (threadIdx.x < kMaxBasis) beta0[threadIdx.x] = beta[threadIdx.x];
  if (threadIdx.x < kMaxVars && means) {
    mom0[0][threadIdx.x] = means[threadIdx.x];
    mom0[1][threadIdx.x] = 1.0f / sds[threadIdx.x];
  }
  __syncthreads();
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P.paths;
       p += gridDim.x * blockDim.x)
    y[p] = apply_decision<kBasisGeneric>(P.prev, 0, 0, vars, means ? mom0[0] : nullptr,
                          mom0[1], cf, ex, num, beta0, y[p], P.paths, p);
}

// Per-date moments of the basis variables (population mean and sd).
__global__ void __launch_bounds__(256)
    ls_moments_kernel(const float* __restrict__ vars, int paths,
                      double* __restrict__ part) {
  __shared__ double sh[6][8];
  const int e = blockIdx.y;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
#pragma unroll
    for (int v = 0; v < kMaxVars; ++v) {
      const double x = vars[((size_t)e * kMaxVars + v) * paths + p];
      acc[2 * v] += x;
      acc[2 * v + 1] += x * x;
    }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double x = warp_sum_d(acc[i]);
    if (lane == 0) sh[i][w] = x;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[threadIdx.x][i];
    part[((size_t)e * gridDim.x + blockIdx.x) * 6 + threadIdx.x] = s;
  }
}

__global__ void ls_moments_final_kernel(const double* __restrict__ part,
                                        int nblocks, int n_ex, int paths,
                                        float* __restrict__ means,
                                        float* __restrict__ sds, int rows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // e*3 + v
  if (i >= n_ex * kMaxVars) return;
  const int e = i / kMaxVars, v = i % kMaxVars;
  double s = 0.0, s2 = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    s += part[((size_t)e * nblocks + b) * 6 + 2 * v];
    s2 += part[((size_t)e * nblocks + b) * 6 + 2 * v + 1];
  }
  const double m = s / paths;
  double var = s2 / paths - m * m;
  double sd = var > 0.0 ? sqrt(var) : 0.0;
  if (!(sd > 0.0)) sd = 1.0;
  // depth-0 row of date e when each date holds `rows` rows
  const size_t o = ((size_t)e * rows) * kMaxVars + v;
  means[o] = (float)m;
  sds[o] = (float)sd;
}

namespace lmm {

int ls_fill_date(const LSBasisSpec& spec, int e, LSDate* d) {
  d->nvars = spec.nvars[e];
  d->nbasis = spec.nbasis[e];
  LMM_REQUIRE(d->nvars >= 0 && d->nvars <= kMaxVars,
              "LS: nvars out of range at date %d", e);
  LMM_REQUIRE(d->nbasis >= 1 && d->nbasis <= kMaxBasis,
              "LS: nbasis out of range at date %d", e);
  for (int k = 0; k < d->nbasis; ++k)
    for (int v = 0; v < kMaxVars; ++v) {
      const int x = spec.mono[(e * kMaxBasis + k) * kMaxVars + v];
      LMM_REQUIRE(x >= 0 && x <= 3, "LS: exponent out of range");
      LMM_REQUIRE(x == 0 || v < d->nvars,
                  "LS: monomial uses an absent variable at date %d", e);
      d->mono[k][v] = (unsigned char)x;
    }
  return LMM_OK;
}

// One CTA per SM for the date kernels and the moments.
int ls_gram_blocks() { return sm_count(); }

// Moments of every date's basis variables over all paths into row e * rows
// of means / sds; part: n_ex * ls_gram_blocks() * 6 doubles.
int ls_moments_launch(const float* vars, int paths, int n_ex, int rows, float* means,
                      float* sds, double* part, cudaStream_t s) {
  const int nblk = ls_gram_blocks();
  ls_moments_kernel<<<dim3(nblk, n_ex), 256, 0, s>>>(vars, paths, part);
  int st = check_launch("ls_moments");
  if (st) return st;
  ls_moments_final_kernel<<<div_up(n_ex * kMaxVars, 128), 128, 0, s>>>(part, nblk, n_ex,
                                                                       paths, means, sds, rows);
  return check_launch("ls_moments_final");
}

size_t ls_workspace_bytes(int paths, int n_ex) {
  const size_t y = ((size_t)paths * sizeof(float) + 255) & ~(size_t)255;
  const size_t part = (size_t)ls_gram_blocks() * kLsMaxPairs * sizeof(double);
  const size_t cnt = ((size_t)n_ex * sizeof(unsigned int) + 255) & ~(size_t)255;
  const size_t mom = (size_t)n_ex * ls_gram_blocks() * 6 * sizeof(double);
  const size_t red = 512 * sizeof(double);
  return y + part + cnt + mom + red + 256;
}

// Raise the dynamic shared-memory limit of a date kernel instantiation
// (once per instantiation and device) when its staged loop needs more than
// the default 48 KB.
template <class Kern>
int ls_stage_attr(Kern kern, size_t bytes) {
  if (bytes <= 48 * 1024) return LMM_OK;
  static std::mutex mu;
  static std::vector<std::pair<const void*, int>> done;
  int dev = 0;
  int st = check_cuda(cudaGetDevice(&dev), "ls_date_kernel: cudaGetDevice");
  if (st) return st;
  std::lock_guard<std::mutex> lock(mu);
  for (const auto& d : done)
    if (d.first == (const void*)kern && d.second == dev) return LMM_OK;
  st = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)bytes),
                  "ls_date_kernel: shared memory attribute");
  if (st) return st;
  done.emplace_back((const void*)kern, dev);
  return LMM_OK;
}

// Launch the date kernel instantiated for the smallest slot count KR >=
// nbasis + 1 (rows split over warp pairs above 11 slots).
int launch_date(const LSDateParams& P_in, int grid, const float* vars,
                const float* means, const float* sds, const float* cf,
                const float* ex, const float* num, double* beta, float* y,
                double* part, unsigned int* counter, double* gram,
                int* status, double* sums_out, cudaStream_t s) {
  // 16-byte staged copies need every input row 16-byte aligned: aligned
  // bases and a path count that is a multiple of 4
  auto al16 = [](const void* q) { return ((uintptr_t)q & 15u) == 0; };
  LSDateParams P = P_in;
  P.vec16 = (P.paths % 4 == 0) && al16(vars) && al16(cf) && al16(ex) && al16(num) && al16(y);
  const int slots = P.cur.nbasis + 1;
  // straight-line basis code when this date and the next (whose decision
  // the kernel applies) share a known table
  const int kind = ls_basis_kind(P.cur);
  const bool known = kind != kBasisGeneric && (!P.has_prev || ls_basis_kind(P.prev) == kind);
#define LMM_LS_DATE(KR, NS, KIND)                                                    \
  do {                                                                               \
    constexpr size_t sb = ls_stage_bytes<KR, NS, false>();                           \
    const int at = ls_stage_attr(ls_date_kernel<KR, NS, KIND, false>, sb);           \
    if (at) return at;                                                               \
    ls_date_kernel<KR, NS, KIND, false><<<grid, LsThreads<KR>::value, sb, s>>>(      \
        P, vars, means, sds, cf, ex, num, beta, y, part, counter, gram, status, sums_out); \
  } while (0)
#define LMM_LS_DATE_MASKED(KR, NS, KIND)                                             \
  do {                                                                               \
    constexpr size_t sb = ls_stage_bytes<KR, NS, true>();                            \
    const int at = ls_stage_attr(ls_date_kernel<KR, NS, KIND, true>, sb);            \
    if (at) return at;                                                               \
    ls_date_kernel<KR, NS, KIND, true><<<grid, LsThreads<KR>::value, sb, s>>>(       \
        P, vars, means, sds, cf, ex, num, beta, y, part, counter, gram, status, sums_out); \
  } while (0)
  if (P.mask_net) {
    if (kind == kBasisC2)
      LMM_LS_DATE_MASKED(7, 1, kBasisC2);
    else if (kind == kBasisQuad)
      LMM_LS_DATE_MASKED(11, 1, kBasisQuad);
    else if (kind == kBasisCross)
      LMM_LS_DATE_MASKED(11, 1, kBasisCross);
    else if (kind == kBasisC5)
      LMM_LS_DATE_MASKED(13, 2, kBasisC5);
    else if (slots <= 7)
      LMM_LS_DATE_MASKED(7, 1, kBasisGeneric);
    else if (slots <= 11)
      LMM_LS_DATE_MASKED(11, 1, kBasisGeneric);
    else if (slots <= 13)
      LMM_LS_DATE_MASKED(13, 2, kBasisGeneric);
    else
      LMM_LS_DATE_MASKED(17, 2, kBasisGeneric);
    return check_launch("ls_date_kernel (masked)");
  }
  if (known && kind == kBasisC2)
    LMM_LS_DATE(7, 1, kBasisC2);
  else if (known && kind == kBasisQuad)
    LMM_LS_DATE(11, 1, kBasisQuad);
  else if (known && kind == kBasisCross)
    LMM_LS_DATE(11, 1, kBasisCross);
  else if (known && kind == kBasisC5)
    LMM_LS_DATE(13, 2, kBasisC5);
  else if (slots <= 7)
    LMM_LS_DATE(7, 1, kBasisGeneric);
  else if (slots <= 11)
    LMM_LS_DATE(11, 1, kBasisGeneric);
  else if (slots <= 13)
    LMM_LS_DATE(13, 2, kBasisGeneric);
  else
    LMM_LS_DATE(17, 2, kBasisGeneric);
#undef LMM_LS_DATE
#undef LMM_LS_DATE_MASKED
  return check_launch("ls_date_kernel");
}

}  // namespace lmm

extern "C" size_t lmm_ls_workspace_bytes(int paths, int n_exercise) {
  return lmm::ls_workspace_bytes(paths, n_exercise);
}

extern "C" int lmm_ls_regress(int n_exercise, int paths, const float* d_vars,
                              const int* h_nvars, const uint8_t* h_monomials,
                              const int* h_nbasis, const float* d_cf,
                              const float* d_ex, const float* d_num,
                              int normalise, void* d_workspace,
                              size_t workspace_bytes, double* d_beta,
                              float* d_means, float* d_sds, double* d_gram,
                              int* d_status, double* d_price,
                              lmm_stream_t stream) {
  LMM_REQUIRE(n_exercise >= 1 && n_exercise <= kMaxSteps && paths >= 1,
              "lmm_ls_regress: bad sizes");
  LMM_REQUIRE(d_vars && h_nvars && h_monomials && h_nbasis && d_num &&
                  d_workspace && d_beta && d_status && d_price,
              "lmm_ls_regress: null pointer");
  LMM_REQUIRE(!normalise || (d_means && d_sds),
              "lmm_ls_regress: normalise needs means/sds outputs");
  LMM_REQUIRE(workspace_bytes >= ls_workspace_bytes(paths, n_exercise),
              "lmm_ls_regress: workspace too small (%zu < %zu)",
              workspace_bytes, ls_workspace_bytes(paths, n_exercise));
  cudaStream_t s = (cudaStream_t)stream;
  LSBasisSpec spec{h_nvars, h_monomials, h_nbasis};
  char* ws = (char*)d_workspace;
  float* y = (float*)ws;
  ws += ((size_t)paths * sizeof(float) + 255) & ~(size_t)255;
  double* part = (double*)ws;
  ws += (size_t)ls_gram_blocks() * kLsMaxPairs * sizeof(double);
  unsigned int* counter = (unsigned int*)ws;
  ws += ((size_t)n_exercise * sizeof(unsigned int) + 255) & ~(size_t)255;
  double* mom = (double*)ws;
  ws += (size_t)n_exercise * ls_gram_blocks() * 6 * sizeof(double);
  double* red = (double*)ws;

  const float* means = nullptr;
  const float* sds = nullptr;
  const int nblk = ls_gram_blocks();
  if (normalise) {
    const int st = ls_moments_launch(d_vars, paths, n_exercise, 1, d_means, d_sds, mom, s);
    if (st) return st;
    means = d_means;
    sds = d_sds;
  }
  int st = check_cuda(cudaMemsetAsync(d_status, 0, sizeof(int), s),
                      "lmm_ls_regress: status reset");
  if (st) return st;
  st = check_cuda(cudaMemsetAsync(counter, 0, (size_t)n_exercise * sizeof(unsigned int), s),
                  "lmm_ls_regress: counter reset");
  if (st) return st;
  for (int e = n_exercise - 1; e >= 0; --e) {
    LSDateParams P;
    memset(&P, 0, sizeof(P));
    P.e = e;
    P.paths = paths;
    st = ls_fill_date(spec, e, &P.cur);
    if (st) return st;
    P.has_prev = (e + 1 < n_exercise);
    if (P.has_prev) {
      st = ls_fill_date(spec, e + 1, &P.prev);
      if (st) return st;
    }
    const int slots = P.cur.nbasis + 1;
    const int per_cta = slots <= 11 ? 512 : slots <= 13 ? 256 : 192;
    int grid = div_up(paths, per_cta);
    if (grid > nblk) grid = nblk;
    st = launch_date(P, grid, d_vars, means, sds, d_cf, d_ex, d_num, d_beta, y,
                     part, counter, d_gram, d_status, nullptr, s);
    if (st) return st;
  }
  LSDateParams P;
  memset(&P, 0, sizeof(P));
  P.paths = paths;
  st = ls_fill_date(spec, 0, &P.prev);
  if (st) return st;
  ls_final_kernel<<<grid_for(paths, 256, 4), 256, 0, s>>>(
      P, d_vars, means, sds, d_cf, d_ex, d_num, d_beta, y);
  st = check_launch("ls_final");
  if (st) return st;
  return reduce_launch(y, d_num, (size_t)paths, 1.0 / (double)paths, red,
                       d_price, s);
}

// ---------------------------------------------------------------------------
// Regression with library-owned scratch, for callers that cannot allocate
// device memory (their device memory is owned by an outside pool allocator,
// or allocation is forbidden in their pricing loop because it can
// synchronise the device).  The scratch is the file-scope array below,
// LMM_LS_STATIC_SCRATCH_BYTES bytes, which every GPU that loads this
// library holds until the process exits.  Host code must not pass the
// array's name to a kernel (in host code it is only a host-side stand-in),
// so the first call on each device looks up the device address with
// cudaGetSymbolAddress, with that device current, and caches it; make that
// first call before any stream capture.  All calls share the array and it
// keeps the last call's contents: every scratch region is written before it
// is read, so nothing needs clearing, but calls that overlap on the GPU
// (on different streams, or from different host threads) race on it.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char
    g_ls_static_scratch[LMM_LS_STATIC_SCRATCH_BYTES];

namespace {
std::mutex g_static_mu;
void* g_static_ptr[64] = {};

int static_scratch_address(void** out) {
  int dev = 0;
  int st = check_cuda(cudaGetDevice(&dev), "lmm_ls_regress_static: cudaGetDevice");
  if (st) return st;
  LMM_REQUIRE(dev >= 0 && dev < 64, "lmm_ls_regress_static: device ordinal %d", dev);
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_ptr[dev]) {
    void* p = nullptr;
    st = check_cuda(cudaGetSymbolAddress(&p, g_ls_static_scratch),
                    "lmm_ls_regress_static: cudaGetSymbolAddress");
    if (st) return st;
    g_static_ptr[dev] = p;
  }
  *out = g_static_ptr[dev];
  return LMM_OK;
}
}  // namespace

extern "C" int lmm_ls_regress_static(int n_exercise, int paths,
                                     const float* d_vars, const int* h_nvars,
                                     const uint8_t* h_monomials,
                                     const int* h_nbasis, const float* d_cf,
                                     const float* d_ex, const float* d_num,
                                     int normalise, double* d_beta,
                                     float* d_means, float* d_sds,
                                     double* d_gram, int* d_status,
                                     double* d_price, lmm_stream_t stream) {
  LMM_REQUIRE(n_exercise >= 1 && n_exercise <= kMaxSteps && paths >= 1,
              "lmm_ls_regress_static: bad sizes");
  const size_t need = ls_workspace_bytes(paths, n_exercise);
  LMM_REQUIRE(need <= (size_t)LMM_LS_STATIC_SCRATCH_BYTES,
              "lmm_ls_regress_static: %d paths x %d dates need %zu bytes of "
              "scratch but the static scratch holds %zu bytes; use "
              "lmm_ls_regress with a caller workspace",
              paths, n_exercise, need, (size_t)LMM_LS_STATIC_SCRATCH_BYTES);
  void* ws = nullptr;
  int st = static_scratch_address(&ws);
  if (st) return st;
  return lmm_ls_regress(n_exercise, paths, d_vars, h_nvars, h_monomials,
                        h_nbasis, d_cf, d_ex, d_num, normalise, ws,
                        (size_t)LMM_LS_STATIC_SCRATCH_BYTES, d_beta, d_means,
                        d_sds, d_gram, d_status, d_price, stream);
}

// ---------------------------------------------------------------------------
// Regression over paths sharded across GPUs.  Each GPU runs the backward
// loop on its own paths; per exercise date the sums over paths (the Gram
// and X^T y, unscaled) are summed over the GPUs by the caller (an
// all-reduce), and every GPU solves the same system, so all apply one rule.
// The moments of the basis variables and the in-sample price are summed the
// same way.  The workspace (lmm_ls_workspace_bytes) carries the running
// path values from one date to the next and must be kept between calls.
// ---------------------------------------------------------------------------
__global__ void ls_solve_sums_kernel(int e, int K, const double* __restrict__ sums,
                                     double total, double* __restrict__ beta,
                                     double* __restrict__ gram_out,
                                     int* __restrict__ status) {
  __shared__ double G_s[kLsMaxSlots * kLsMaxSlots];
  __shared__ double L_s[kMaxBasis * kMaxBasis];
  const int tid = threadIdx.x;
  for (int idx = tid; idx < kLsMaxSlots * kLsMaxSlots; idx += blockDim.x) {
    const int i = idx / kLsMaxSlots, j = idx - i * kLsMaxSlots;
    double v = 0.0;
    if (i < K && j < K) {
      const int a = i > j ? i : j, b = i > j ? j : i;
      v = sums[a * (a + 1) / 2 + b] / total;
    } else if (i < K && j == kLsMaxSlots - 1) {
      v = sums[K * (K + 1) / 2 + i] / total;
    }
    G_s[idx] = v;
  }
  __syncthreads();
  if (gram_out) {
    double* g = gram_out + (size_t)e * kMaxBasis * (kMaxBasis + 1);
    for (int idx = tid; idx < K * (kMaxBasis + 1); idx += blockDim.x) {
      const int i = idx / (kMaxBasis + 1), j = idx - i * (kMaxBasis + 1);
      g[idx] = j < K ? G_s[i * kLsMaxSlots + j]
                     : (j == K ? G_s[i * kLsMaxSlots + kLsMaxSlots - 1] : 0.0);
    }
  }
  if (tid < 32) {
    const int st = warp_cholesky_solve(G_s, K, beta + (size_t)e * kMaxBasis, L_s);
    if (tid == 0 && st) atomicOr(status, st);
  }
}

// Unscaled sums of x and x^2 per date and variable from the block partials
// of ls_moments_kernel, in a fixed order: sums[e][2v] and sums[e][2v+1].
__global__ void ls_moment_sums_kernel(const double* __restrict__ part, int nblocks,
                                      int n_ex, double* __restrict__ sums) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // e*6 + c
  if (i >= n_ex * 6) return;
  const int e = i / 6, c = i - e * 6;
  double s = 0.0;
  for (int b = 0; b < nblocks; ++b) s += part[((size_t)e * nblocks + b) * 6 + c];
  sums[i] = s;
}

__global__ void ls_moments_from_sums_kernel(const double* __restrict__ sums, int n_ex,
                                            double total, float* __restrict__ means,
                                            float* __restrict__ sds) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // e*3 + v
  if (i >= n_ex * kMaxVars) return;
  const int e = i / kMaxVars, v = i % kMaxVars;
  const double m = sums[e * 6 + 2 * v] / total;
  const double var = sums[e * 6 + 2 * v + 1] / total - m * m;
  double sd = var > 0.0 ? sqrt(var) : 0.0;
  if (!(sd > 0.0)) sd = 1.0;
  means[i] = (float)m;
  sds[i] = (float)sd;
}

namespace {
struct LsWs {
  float* y;
  double* part;
  unsigned int* counter;
  double* mom;
  double* red;
};

LsWs carve_ls(void* d_workspace, int paths, int n_exercise) {
  char* ws = (char*)d_workspace;
  LsWs w;
  w.y = (float*)ws;
  ws += ((size_t)paths * sizeof(float) + 255) & ~(size_t)255;
  w.part = (double*)ws;
  ws += (size_t)ls_gram_blocks() * kLsMaxPairs * sizeof(double);
  w.counter = (unsigned int*)ws;
  ws += ((size_t)n_exercise * sizeof(unsigned int) + 255) & ~(size_t)255;
  w.mom = (double*)ws;
  ws += (size_t)n_exercise * ls_gram_blocks() * 6 * sizeof(double);
  w.red = (double*)ws;
  return w;
}
}  // namespace

extern "C" int lmm_ls_moment_sums(int n_exercise, int paths, const float* d_vars,
                                  void* d_workspace, size_t workspace_bytes,
                                  double* d_sums, lmm_stream_t stream) {
  LMM_REQUIRE(n_exercise >= 1 && n_exercise <= kMaxSteps && paths >= 1,
              "lmm_ls_moment_sums: bad sizes");
  LMM_REQUIRE(d_vars && d_workspace && d_sums, "lmm_ls_moment_sums: null pointer");
  LMM_REQUIRE(workspace_bytes >= ls_workspace_bytes(paths, n_exercise),
              "lmm_ls_moment_sums: workspace too small");
  cudaStream_t s = (cudaStream_t)stream;
  LsWs w = carve_ls(d_workspace, paths, n_exercise);
  const int nblk = ls_gram_blocks();
  ls_moments_kernel<<<dim3(nblk, n_exercise), 256, 0, s>>>(d_vars, paths, w.mom);
  int st = check_launch("ls_moments");
  if (st) return st;
  ls_moment_sums_kernel<<<div_up(n_exercise * 6, 128), 128, 0, s>>>(w.mom, nblk, n_exercise,
                                                                    d_sums);
  return check_launch("ls_moment_sums");
}

extern "C" int lmm_ls_moments_from_sums(int n_exercise, double total_paths,
                                        const double* d_sums, float* d_means,
                                        float* d_sds, lmm_stream_t stream) {
  LMM_REQUIRE(n_exercise >= 1 && n_exercise <= kMaxSteps && total_paths >= 1.0,
              "lmm_ls_moments_from_sums: bad sizes");
  LMM_REQUIRE(d_sums && d_means && d_sds, "lmm_ls_moments_from_sums: null pointer");
  ls_moments_from_sums_kernel<<<div_up(n_exercise * kMaxVars, 128), 128, 0,
                                (cudaStream_t)stream>>>(d_sums, n_exercise, total_paths,
                                                        d_means, d_sds);
  return check_launch("ls_moments_from_sums");
}

extern "C" int lmm_ls_date_sums(int e, int n_exercise, int paths, const float* d_vars,
                                const int* h_nvars, const uint8_t* h_monomials,
                                const int* h_nbasis, const float* d_cf,
                                const float* d_ex, const float* d_num,
                                const float* d_means, const float* d_sds,
                                const double* d_beta, void* d_workspace,
                                size_t workspace_bytes, double* d_sums,
                                lmm_stream_t stream) {
  LMM_REQUIRE(n_exercise >= 1 && n_exercise <= kMaxSteps && paths >= 1 && e >= 0 &&
                  e < n_exercise,
              "lmm_ls_date_sums: bad sizes");
  LMM_REQUIRE(d_vars && h_nvars && h_monomials && h_nbasis && d_num && d_beta &&
                  d_workspace && d_sums,
              "lmm_ls_date_sums: null pointer");
  LMM_REQUIRE(!d_means == !d_sds, "lmm_ls_date_sums: means/sds mismatch");
  LMM_REQUIRE(workspace_bytes >= ls_workspace_bytes(paths, n_exercise),
              "lmm_ls_date_sums: workspace too small");
  cudaStream_t s = (cudaStream_t)stream;
  LsWs w = carve_ls(d_workspace, paths, n_exercise);
  LSBasisSpec spec{h_nvars, h_monomials, h_nbasis};
  LSDateParams P;
  memset(&P, 0, sizeof(P));
  P.e = e;
  P.paths = paths;
  int st = ls_fill_date(spec, e, &P.cur);
  if (st) return st;
  P.has_prev = (e + 1 < n_exercise);
  if (P.has_prev) {
    st = ls_fill_date(spec, e + 1, &P.prev);
    if (st) return st;
  }
  st = check_cuda(cudaMemsetAsync(w.counter + e, 0, sizeof(unsigned int), s),
                  "lmm_ls_date_sums: counter reset");
  if (st) return st;
  const int slots = P.cur.nbasis + 1;
  const int per_cta = slots <= 11 ? 512 : slots <= 13 ? 256 : 192;
  int grid = div_up(paths, per_cta);
  if (grid > ls_gram_blocks()) grid = ls_gram_blocks();
  return launch_date(P, grid, d_vars, d_means, d_sds, d_cf, d_ex, d_num,
                     const_cast<double*>(d_beta), w.y, w.part, w.counter, nullptr,
                     nullptr, d_sums, s);
}

extern "C" int lmm_ls_date_solve(int e, int nbasis, const double* d_sums,
                                 double total_paths, double* d_beta, double* d_gram,
                                 int* d_status, lmm_stream_t stream) {
  LMM_REQUIRE(e >= 0 && e < kMaxSteps && nbasis >= 1 && nbasis <= kMaxBasis &&
                  total_paths >= 1.0,
              "lmm_ls_date_solve: bad sizes");
  LMM_REQUIRE(d_sums && d_beta && d_status, "lmm_ls_date_solve: null pointer");
  ls_solve_sums_kernel<<<1, 128, 0, (cudaStream_t)stream>>>(e, nbasis, d_sums, total_paths,
                                                            d_beta, d_gram, d_status);
  return check_launch("ls_solve_sums_kernel");
}

extern "C" int lmm_ls_final_sum(int n_exercise, int paths, const float* d_vars,
                                const int* h_nvars, const uint8_t* h_monomials,
                                const int* h_nbasis, const float* d_cf,
                                const float* d_ex, const float* d_num,
                                const float* d_means, const float* d_sds,
                                const double* d_beta, void* d_workspace,
                                size_t workspace_bytes, double* d_sum,
                                lmm_stream_t stream) {
  LMM_REQUIRE(n_exercise >= 1 && n_exercise <= kMaxSteps && paths >= 1,
              "lmm_ls_final_sum: bad sizes");
  LMM_REQUIRE(d_vars && h_nvars && h_monomials && h_nbasis && d_num && d_beta &&
                  d_workspace && d_sum,
              "lmm_ls_final_sum: null pointer");
  LMM_REQUIRE(workspace_bytes >= ls_workspace_bytes(paths, n_exercise),
              "lmm_ls_final_sum: workspace too small");
  cudaStream_t s = (cudaStream_t)stream;
  LsWs w = carve_ls(d_workspace, paths, n_exercise);
  LSBasisSpec spec{h_nvars, h_monomials, h_nbasis};
  LSDateParams P;
  memset(&P, 0, sizeof(P));
  P.paths = paths;
  int st = ls_fill_date(spec, 0, &P.prev);
  if (st) return st;
  ls_final_kernel<<<grid_for(paths, 256, 4), 256, 0, s>>>(P, d_vars, d_means, d_sds, d_cf,
                                                         d_ex, d_num, d_beta, w.y);
  st = check_launch("ls_final");
  if (st) return st;
  return reduce_launch(w.y, d_num, (size_t)paths, 1.0, w.red, d_sum, s);
}
