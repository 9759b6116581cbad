// ls_common.cuh — Longstaff–Schwartz basis tables shared by the LS kernels,
// the staged second pass and the fused pricing kernel.
#pragma once
#include "lmm_common.cuh"

namespace lmm {

// Basis of one exercise date: nbasis monomials in nvars variables, each
// monomial a vector of exponents (0..3) over the (up to 3) variables.
struct LSDate {
  int nvars, nbasis;
  unsigned char mono[kMaxBasis][kMaxVars];
};

// Host-side view of the per-date basis description passed through the ABI.
struct LSBasisSpec {
  const int* nvars;              // [E]
  const unsigned char* mono;     // [E][kMaxBasis][kMaxVars]
  const int* nbasis;             // [E]
};

int ls_fill_date(const LSBasisSpec& spec, int e, LSDate* d);

// Regressions per date of a nested rule (lmm_ls_select.depth).
constexpr int kMaxDepth = LMM_LS_MAX_DEPTH;

// One launch of the per-date regression kernel (ls.cu): date e's basis
// (cur) and, when has_prev, date e + 1's basis, whose frozen decision the
// launch applies to the running values first.
struct LSDateParams {
  LSDate cur, prev;
  int e, has_prev, paths, kr;
  // Nested regressions (zero for the depth-1 loop): rows of beta / moments
  // per date (0 = 1) and this launch's depth; a path takes part when
  // |mask_net[p]| <= *mask_cut; sums are divided by *mask_count; the launch
  // does nothing when *skip is set.
  int rows, depth;
  int read_y;  // target cf + y[p] without applying a decision first
  int vec16;   // set by launch_date: every input row 16-byte aligned
  const double* mask_net;
  const double* mask_cut;
  const int* mask_count;
  const int* skip;
};

// Launches the date kernel instantiated for the date's basis (ls.cu).
int launch_date(const LSDateParams& P, int grid, const float* vars, const float* means,
                const float* sds, const float* cf, const float* ex, const float* num,
                double* beta, float* y, double* part, unsigned int* counter, double* gram,
                int* status, double* sums_out, cudaStream_t s);
int ls_gram_blocks();
int ls_moments_launch(const float* vars, int paths, int n_ex, int rows, float* means,
                      float* sds, double* part, cudaStream_t s);
constexpr int kLsMaxSlots = kMaxBasis + 1;  // basis + target
constexpr int kLsMaxPairs = kLsMaxSlots * (kLsMaxSlots + 1) / 2;

// A frozen exercise rule: `depth` regressions per date (1 = plain LS).
// Row r = e * depth + d holds regression d of date e: beta[r][kMaxBasis],
// means / sds[r][kMaxVars] (null: raw variables), cuts[r][2] (lower,
// upper; null when depth = 1).  shifts[e] (Andersen shift, null: none) is
// added to every estimate of date e.
struct LsRuleView {
  int depth;
  const double* beta;
  const float* means;
  const float* sds;
  const double* cuts;
  const float* shifts;
};

inline LsRuleView ls_rule_view(const double* beta, const float* means, const float* sds) {
  return LsRuleView{1, beta, means, sds, nullptr, nullptr};
}

// Basis tables the kernels know at compile time (the generators of the
// reference in three variables: quadraticPolynomialCrossGenerator and
// quadraticPolynomialGenerator, gold/LS_regression.h:123-240, and the two
// fixed bases of the benchmark configurations).  A date whose runtime table
// equals one of them uses straight-line basis code; any other table takes
// the generic path with runtime exponents.
enum { kBasisGeneric = 0, kBasisC2 = 1, kBasisQuad = 2, kBasisCross = 3, kBasisC5 = 4 };

// Exponent of variable v in basis function k of a known kind: 2 bits per
// function in one word per variable (function k at bits 2k, 2k+1).
__host__ __device__ constexpr unsigned basis_code(int kind, int v) {
  return kind == 1 ? (v == 0 ? 0x00000440u : v == 1 ? 0x00000424u : 0x00000100u)
         : kind == 2 ? (v == 0 ? 0x00000024u : v == 1 ? 0x00000240u : 0x00002400u)
         : kind == 3 ? (v == 0 ? 0x00009104u : v == 1 ? 0x00020510u : 0x00081440u)
         : kind == 4 ? (v == 0 ? 0x00109104u : v == 1 ? 0x00d20510u : 0x00181440u)
         : 0u;
}
__host__ __device__ constexpr int basis_K(int kind) {
  return kind == 1 ? 6 : kind == 2 ? 7 : kind == 3 ? 10 : kind == 4 ? 12 : 0;
}
__host__ __device__ constexpr int basis_exp(int kind, int k, int v) {
  return (int)((basis_code(kind, v) >> (2 * k)) & 3u);
}

// Kind of a date's basis (three variables and a known table), else generic.
inline int ls_basis_kind(const LSDate& d) {
  if (d.nvars != kMaxVars) return kBasisGeneric;
  for (int kind = 1; kind < 5; ++kind) {
    if (basis_K(kind) != d.nbasis) continue;
    bool same = true;
    for (int k = 0; k < d.nbasis && same; ++k)
      for (int v = 0; v < kMaxVars; ++v)
        if (basis_exp(kind, k, v) != d.mono[k][v]) same = false;
    if (same) return kind;
  }
  return kBasisGeneric;
}

#ifdef __CUDACC__
// x^e for e in 0..3 by selection (exponents come from uniform parameter
// tables; indexing a register array with them would go through local
// memory).
__device__ __forceinline__ float ls_pow(const float (&p)[3], int e) {
  return e == 0 ? 1.0f : e == 1 ? p[0] : e == 2 ? p[1] : p[2];
}

// Basis value phi = prod_v x_v^{m_v} from the powers pw[v] = {x, x^2, x^3}.
__device__ __forceinline__ float ls_monomial(const float (&pw)[kMaxVars][3],
                                             const unsigned char* m) {
  return ls_pow(pw[0], m[0]) * ls_pow(pw[1], m[1]) * ls_pow(pw[2], m[2]);
}

// Basis function k of date d: the compile-time table of KIND (k a
// compile-time index after unrolling, so the selections fold away), or the
// date's runtime exponents for the generic kind.
template <int KIND>
__device__ __forceinline__ float ls_basis(const float (&pw)[kMaxVars][3],
                                          const LSDate& d, int k) {
  if (KIND == kBasisGeneric) return ls_monomial(pw, d.mono[k]);
  return ls_pow(pw[0], basis_exp(KIND, k, 0)) * ls_pow(pw[1], basis_exp(KIND, k, 1)) *
         ls_pow(pw[2], basis_exp(KIND, k, 2));
}

__device__ __forceinline__ void ls_powers(const float* x, float (&pw)[kMaxVars][3]) {
#pragma unroll
  for (int v = 0; v < kMaxVars; ++v) {
    pw[v][0] = x[v];
    pw[v][1] = x[v] * x[v];
    pw[v][2] = x[v] * x[v] * x[v];
  }
}

// Continuation estimate of a frozen rule at date e for basis variables v
// and exercise value exv: the depth chain of MultiLSExerciseStrategy::decide
// (gold/MultiLS_regression.h:190-231) and updateDeflatedNextStepValuesMulti_
// gold (:42-99): regression d + 1 is used while the net value estimate -
// exv of regression d lies strictly inside d's cuts.  The caller exercises
// when exv > estimate.
// sum_k phi_k(x) b[k] with x standardised by mean / sd (null: raw).
__device__ __forceinline__ double ls_row_estimate(const double* b, const float* mean,
                                                  const float* sd, int nvars, int nbasis,
                                                  const unsigned char (*mono)[kMaxVars],
                                                  const float* v) {
  float x[kMaxVars];
#pragma unroll
  for (int k = 0; k < kMaxVars; ++k) {
    float t = 0.0f;
    if (k < nvars) {
      t = v[k];
      if (mean) t = (t - mean[k]) / sd[k];
    }
    x[k] = t;
  }
  float pw[kMaxVars][3];
  ls_powers(x, pw);
  double est = 0.0;
#pragma unroll
  for (int k = 0; k < kMaxBasis; ++k)
    if (k < nbasis) est += (double)ls_monomial(pw, mono[k]) * b[k];
  return est;
}

__device__ __forceinline__ double ls_chain_estimate(const LsRuleView& r, int e, int nvars,
                                                    int nbasis,
                                                    const unsigned char (*mono)[kMaxVars],
                                                    const float* v, float exv) {
  double est = 0.0;
  for (int d = 0; d < r.depth; ++d) {
    const size_t row = (size_t)e * r.depth + d;
    est = (r.shifts ? (double)r.shifts[e] : 0.0) +
          ls_row_estimate(r.beta + row * kMaxBasis, r.means ? r.means + row * kMaxVars : nullptr,
                          r.means ? r.sds + row * kMaxVars : nullptr, nvars, nbasis, mono, v);
    if (d + 1 >= r.depth || !r.cuts) break;
    const double net = est - (double)exv;
    if (!(net > r.cuts[row * 2] && net < r.cuts[row * 2 + 1])) break;
  }
  return est;
}
#endif

}  // namespace lmm
