// ls_common.cuh — Longstaff–Schwartz basis tables shared by the LS kernels,
// the staged second pass and the fused pricing kernel.
#pragma once
#include "lmm_common.cuh"

namespace lmm {

constexpr int kMaxPairs = kMaxBasis * (kMaxBasis + 1) / 2 + kMaxBasis;

// Basis of one exercise date: nbasis monomials in nvars variables, each
// monomial a vector of exponents (0..3) over the (up to 3) variables.
struct LSDate {
  int nvars, nbasis;
  unsigned char mono[kMaxBasis][kMaxVars];
};

struct LSStepParams {
  LSDate cur;   // date being regressed
  LSDate prev;  // date whose frozen decision is applied first
  int e, has_prev, paths, npairs;
  unsigned char pair_i[kMaxPairs], pair_j[kMaxPairs];
};

// Host-side view of the per-date basis description passed through the ABI.
struct LSBasisSpec {
  const int* nvars;              // [E]
  const unsigned char* mono;     // [E][kMaxBasis][kMaxVars]
  const int* nbasis;             // [E]
};

int ls_fill_date(const LSBasisSpec& spec, int e, LSDate* d);

}  // namespace lmm
