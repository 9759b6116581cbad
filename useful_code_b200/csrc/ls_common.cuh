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

__device__ __forceinline__ void ls_powers(const float* x, float (&pw)[kMaxVars][3]) {
#pragma unroll
  for (int v = 0; v < kMaxVars; ++v) {
    pw[v][0] = x[v];
    pw[v][1] = x[v] * x[v];
    pw[v][2] = x[v] * x[v] * x[v];
  }
}
#endif

}  // namespace lmm
