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
// a device-to-host copy (LinearSolverConcrete_main.cu:127-188); here the
// Gram partial sums stay on the device and a one-block FP64 Cholesky solves
// them, so the whole loop is launch-only and can be captured in a graph.
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

__device__ __forceinline__ double warp_sum_d(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  return x;
}

// Standardised variables and basis values phi_k = prod_v x'_v^{e_kv}.
__device__ __forceinline__ void eval_basis(const LSDate& d, const float* x,
                                           float* phi) {
  float pw[kMaxVars][4];
#pragma unroll
  for (int v = 0; v < kMaxVars; ++v) {
    const float xv = x[v];
    pw[v][0] = 1.0f;
    pw[v][1] = xv;
    pw[v][2] = xv * xv;
    pw[v][3] = xv * xv * xv;
  }
#pragma unroll
  for (int k = 0; k < kMaxBasis; ++k) {
    if (k < d.nbasis) {
      const unsigned char* m = d.mono[k];
      phi[k] = pw[0][m[0]] * pw[1][m[1]] * pw[2][m[2]];
    }
  }
}

__device__ __forceinline__ void load_vars(const LSDate& d, int e,
                                          const float* __restrict__ vars,
                                          const float* __restrict__ means,
                                          const float* __restrict__ sds,
                                          int paths, int p, float* x) {
#pragma unroll
  for (int v = 0; v < kMaxVars; ++v) {
    float xv = 0.0f;
    if (v < d.nvars) {
      xv = vars[((size_t)e * kMaxVars + v) * paths + p];
      if (means) xv = (xv - means[e * kMaxVars + v]) / sds[e * kMaxVars + v];
    }
    x[v] = xv;
  }
}
}  // namespace lmm

// Apply the frozen decision of date d to path p and deflate to date d-1.
__device__ __forceinline__ float apply_decision(
    const LSDate& dd, int d, int deflate, const float* __restrict__ vars,
    const float* __restrict__ means, const float* __restrict__ sds,
    const float* __restrict__ cf, const float* __restrict__ ex,
    const float* __restrict__ num, const double* __restrict__ beta,
    float y_in, int paths, int p) {
  float x[kMaxVars], phi[kMaxBasis];
  load_vars(dd, d, vars, means, sds, paths, p, x);
  eval_basis(dd, x, phi);
  double est = 0.0;
#pragma unroll
  for (int k = 0; k < kMaxBasis; ++k)
    if (k < dd.nbasis) est += (double)phi[k] * beta[d * kMaxBasis + k];
  const float t = (cf ? cf[(size_t)d * paths + p] : 0.0f) + y_in;
  const float exv = ex ? ex[(size_t)d * paths + p] : 0.0f;
  float y = ((double)exv > est) ? exv : t;
  if (deflate)
    y = y * (num[(size_t)(d - 1) * paths + p] / num[(size_t)d * paths + p]);
  return y;
}

// One backward step: apply date e+1's decision (if any), then accumulate
// the regression sums of date e.  Block partials go to part[block][q].
__global__ void __launch_bounds__(256)
    ls_step_kernel(const __grid_constant__ LSStepParams P,
                   const float* __restrict__ vars,
                   const float* __restrict__ means,
                   const float* __restrict__ sds, const float* __restrict__ cf,
                   const float* __restrict__ ex, const float* __restrict__ num,
                   const double* __restrict__ beta, float* __restrict__ y,
                   double* __restrict__ part) {
  constexpr int TILE = 256;
  // Rows padded by 4 floats so that the pair threads, which read different
  // rows at the same column, fall on different banks.
  __shared__ __align__(16) float phi_s[kMaxBasis + 1][TILE + 4];
  const int K = P.cur.nbasis;
  const int npairs = P.npairs;
  const int q = threadIdx.x;
  const int qi = q < npairs ? P.pair_i[q] : 0;
  const int qj = q < npairs ? P.pair_j[q] : 0;  // qj == K: the target column
  double acc = 0.0;
  const int paths = P.paths;
  for (int base = blockIdx.x * TILE; base < paths; base += gridDim.x * TILE) {
    const int p = base + threadIdx.x;
    if (p < paths) {
      float yp = 0.0f;
      if (P.has_prev) {
        yp = apply_decision(P.prev, P.e + 1, 1, vars, means, sds, cf, ex, num,
                            beta, y[p], paths, p);
      }
      y[p] = yp;
      float x[kMaxVars], phi[kMaxBasis];
      load_vars(P.cur, P.e, vars, means, sds, paths, p, x);
      eval_basis(P.cur, x, phi);
#pragma unroll
      for (int k = 0; k < kMaxBasis; ++k)
        if (k < K) phi_s[k][threadIdx.x] = phi[k];
      phi_s[K][threadIdx.x] = (cf ? cf[(size_t)P.e * paths + p] : 0.0f) + yp;
    } else {
      for (int k = 0; k <= K; ++k) phi_s[k][threadIdx.x] = 0.0f;
    }
    __syncthreads();
    if (q < npairs) {
      const float4* a = reinterpret_cast<const float4*>(phi_s[qi]);
      const float4* b = reinterpret_cast<const float4*>(phi_s[qj]);
      float s = 0.0f;
#pragma unroll 8
      for (int i = 0; i < TILE / 4; ++i) {
        const float4 u = a[i], v = b[i];
        s += u.x * v.x;
        s += u.y * v.y;
        s += u.z * v.z;
        s += u.w * v.w;
      }
      acc += (double)s;
    }
    __syncthreads();
  }
  if (q < npairs) part[(size_t)blockIdx.x * kMaxPairs + q] = acc;
}

// Sum block partials (fixed order), normalise, Cholesky-solve in FP64.
__global__ void __launch_bounds__(256)
    ls_solve_kernel(const __grid_constant__ LSStepParams P,
                    const double* __restrict__ part, int nblocks,
                    double* __restrict__ beta, double* __restrict__ gram_out,
                    int* __restrict__ status) {
  __shared__ double sums[kMaxPairs];
  __shared__ double G[kMaxBasis][kMaxBasis + 1];
  const int K = P.cur.nbasis;
  const int npairs = P.npairs;
  for (int q = threadIdx.x; q < npairs; q += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += part[(size_t)b * kMaxPairs + q];
    sums[q] = s / (double)P.paths;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  for (int q = 0; q < npairs; ++q) {
    const int i = P.pair_i[q], j = P.pair_j[q];
    if (j == K)
      G[i][K] = sums[q];
    else {
      G[i][j] = sums[q];
      G[j][i] = sums[q];
    }
  }
  if (gram_out) {
    double* g = gram_out + (size_t)P.e * kMaxBasis * (kMaxBasis + 1);
    for (int i = 0; i < K; ++i)
      for (int j = 0; j <= K; ++j) g[i * (kMaxBasis + 1) + j] = G[i][j];
  }
  double* out = beta + P.e * kMaxBasis;
  for (int k = 0; k < kMaxBasis; ++k) out[k] = 0.0;
  double maxd = 0.0;
  for (int i = 0; i < K; ++i) maxd = fmax(maxd, fabs(G[i][i]));
  if (!(maxd > 0.0)) {
    atomicOr(status, 1);
    return;
  }
  // Cholesky with a relative diagonal jitter retried on failure.
  double L[kMaxBasis][kMaxBasis];
  double jitter = 0.0;
  bool ok = false;
  for (int attempt = 0; attempt < 6 && !ok; ++attempt) {
    ok = true;
    for (int i = 0; i < K && ok; ++i) {
      for (int j = 0; j <= i; ++j) {
        double s = G[i][j] + (i == j ? jitter : 0.0);
        for (int k = 0; k < j; ++k) s -= L[i][k] * L[j][k];
        if (i == j) {
          if (!(s > 1e-300)) {
            ok = false;
            break;
          }
          L[i][i] = sqrt(s);
        } else {
          L[i][j] = s / L[j][j];
        }
      }
    }
    if (!ok) jitter = (jitter == 0.0) ? 1e-14 * maxd : jitter * 100.0;
  }
  if (!ok) {
    atomicOr(status, 2);
    return;
  }
  if (jitter > 0.0) atomicOr(status, 4);
  double z[kMaxBasis];
  for (int i = 0; i < K; ++i) {
    double s = G[i][K];
    for (int k = 0; k < i; ++k) s -= L[i][k] * z[k];
    z[i] = s / L[i][i];
  }
  for (int i = K - 1; i >= 0; --i) {
    double s = z[i];
    for (int k = i + 1; k < K; ++k) s -= L[k][i] * out[k];
    out[i] = s / L[i][i];
  }
}

// Final decision at date 0 (no deflation): y holds the value at date 0.
__global__ void ls_final_kernel(const __grid_constant__ LSStepParams P,
                                const float* __restrict__ vars,
                                const float* __restrict__ means,
                                const float* __restrict__ sds,
                                const float* __restrict__ cf,
                                const float* __restrict__ ex,
                                const float* __restrict__ num,
                                const double* __restrict__ beta,
                                float* __restrict__ y) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P.paths;
       p += gridDim.x * blockDim.x)
    y[p] = apply_decision(P.prev, 0, 0, vars, means, sds, cf, ex, num, beta,
                          y[p], P.paths, p);
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
                                        float* __restrict__ sds) {
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
  means[i] = (float)m;
  sds[i] = (float)sd;
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

void ls_fill_pairs(LSStepParams* P) {
  const int K = P->cur.nbasis;
  int q = 0;
  for (int i = 0; i < K; ++i)
    for (int j = 0; j <= i; ++j) {
      P->pair_i[q] = (unsigned char)i;
      P->pair_j[q] = (unsigned char)j;
      ++q;
    }
  for (int i = 0; i < K; ++i) {
    P->pair_i[q] = (unsigned char)i;
    P->pair_j[q] = (unsigned char)K;
    ++q;
  }
  P->npairs = q;
}

int ls_gram_blocks() { return 2 * sm_count(); }

size_t ls_workspace_bytes(int paths, int n_ex) {
  const size_t y = ((size_t)paths * sizeof(float) + 255) & ~(size_t)255;
  const size_t part = (size_t)ls_gram_blocks() * kMaxPairs * sizeof(double);
  const size_t mom = (size_t)n_ex * ls_gram_blocks() * 6 * sizeof(double);
  const size_t red = 512 * sizeof(double);
  return y + part + mom + red + 256;
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
  ws += (size_t)ls_gram_blocks() * kMaxPairs * sizeof(double);
  double* mom = (double*)ws;
  ws += (size_t)n_exercise * ls_gram_blocks() * 6 * sizeof(double);
  double* red = (double*)ws;

  const float* means = nullptr;
  const float* sds = nullptr;
  const int nblk = ls_gram_blocks();
  if (normalise) {
    dim3 g(nblk, n_exercise);
    ls_moments_kernel<<<g, 256, 0, s>>>(d_vars, paths, mom);
    int st = check_launch("ls_moments");
    if (st) return st;
    ls_moments_final_kernel<<<div_up(n_exercise * kMaxVars, 128), 128, 0, s>>>(
        mom, nblk, n_exercise, paths, d_means, d_sds);
    st = check_launch("ls_moments_final");
    if (st) return st;
    means = d_means;
    sds = d_sds;
  }
  int st = check_cuda(cudaMemsetAsync(d_status, 0, sizeof(int), s),
                      "lmm_ls_regress: status reset");
  if (st) return st;
  int grid = div_up(paths, 256);
  if (grid > nblk) grid = nblk;
  for (int e = n_exercise - 1; e >= 0; --e) {
    LSStepParams P;
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
    ls_fill_pairs(&P);
    ls_step_kernel<<<grid, 256, 0, s>>>(P, d_vars, means, sds, d_cf, d_ex,
                                        d_num, d_beta, y, part);
    st = check_launch("ls_step");
    if (st) return st;
    ls_solve_kernel<<<1, 256, 0, s>>>(P, part, grid, d_beta, d_gram, d_status);
    st = check_launch("ls_solve");
    if (st) return st;
  }
  LSStepParams P;
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
