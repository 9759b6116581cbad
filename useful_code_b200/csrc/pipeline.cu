// pipeline.cu — whole-pipeline drivers (C++ host code over the C ABI) and
// the fused per-path kernels.
//
// Staged mode runs the reference's chain stage by stage through full
// [step][rate][path] tensors (LMM_evolver_full.cu:154-262 and the pass loops
// of kooexample/bermudanIRDPricer.cu:650-947,1201-1480): Sobol -> scramble ->
// inverse normal -> bridge -> correlate+drift -> one PC launch per step ->
// discount ratios -> annuities -> swap rates -> numeraires -> extraction ->
// basis variables / exercise values / coupons -> partial discounting ->
// aggregation.
//
// Fused mode: one kernel draws the Sobol points, scrambles them, maps them
// to normals and bridges them (one thread per path and factor, bridge points
// in shared memory); a second kernel evolves every path through all steps
// with the log-rates of its CTA resident in shared memory, forms discount
// ratios, annuity, swap rate and numeraire on the fly and writes only what
// the regression reads (basis variables, exercise value, deflated coupon and
// numeraire per exercise date), or applies the frozen exercise rule and
// writes only the per-path payoff.  Per rate and step it performs the
// arithmetic of LMM_evolver_all_steps_pc_kernel_devicelog_discounts
// (LMM_evolver_all.cu:506-747) with the log-rate cap of the gold evolver
// (gold/LMM_evolver_gold.h:369-375).
#include "lmm_common.cuh"
#include "lmm_device.cuh"
#include "bridge_plan.h"
#include "ls_common.cuh"
#include "../../include/lmm_pipeline.h"
#include "fused_kernels.cuh"
#include "greeks_kernels.cuh"
#include "tc_evolve.cuh"
#include "ab_kernels.cuh"

#include <mutex>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

using namespace lmm;

namespace lmm {

int ls_fill_date(const LSBasisSpec& spec, int e, LSDate* d);
int reduce_launch(const float* d_in, const float* d_div, size_t n,
                  double scale, double* d_partials, double* d_out,
                  cudaStream_t stream);

// Frozen-rule payoff from precomputed LS inputs.
__global__ void ls_apply_rule_kernel(int n_ex, int paths,
                                     const float* __restrict__ vars,
                                     const float* __restrict__ cf,
                                     const float* __restrict__ ex,
                                     const float* __restrict__ num,
                                     const __grid_constant__ RuleConst rc,
                                     const LsRuleView rule,
                                     float* __restrict__ payoff) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < paths;
       p += gridDim.x * blockDim.x) {
    double total = 0.0;
    for (int e = 0; e < n_ex; ++e) {
      float v[kMaxVars];
#pragma unroll
      for (int k = 0; k < kMaxVars; ++k)
        v[k] = vars[((size_t)e * kMaxVars + k) * paths + p];
      const float exv = ex ? ex[(size_t)e * paths + p] : 0.0f;
      const double est = rule_estimate(rc, e, v, exv, rule);
      const float nv = num[(size_t)e * paths + p];
      if ((double)exv > est) {
        total += (double)exv / (double)nv;
        break;
      }
      if (cf) total += (double)cf[(size_t)e * paths + p] / (double)nv;
    }
    payoff[p] = (float)total;
  }
}

// ------------------------------- host side ---------------------------------

namespace {

// Products priced without exercise (and without a regression).
inline bool no_exercise(int kind) {
  return kind == LMM_PRODUCT_EUROPEAN || kind == LMM_PRODUCT_TARN;
}

// Products whose exercise date is a payer-swaption exercise (basis
// variables, exercise value and regression of the swaption).
inline bool swaption_exercise(int kind) {
  return kind == LMM_PRODUCT_SWAPTION || kind == LMM_PRODUCT_BERMUDAN_CAP;
}

struct Validated {
  int n, F, E, D;
  ModelConst mc;
  ProductConst pc;
  RuleConst rc;
};

int validate(const lmm_model* m, const lmm_product* pr, Validated* v) {
  LMM_REQUIRE(m && pr, "pipeline: null model or product");
  LMM_REQUIRE(m->rates >= 2 && m->rates <= kMaxRates,
              "pipeline: rates must be in [2,%d]", kMaxRates);
  LMM_REQUIRE(m->factors >= 1 && m->factors <= kMaxFactors,
              "pipeline: factors must be in [1,%d]", kMaxFactors);
  LMM_REQUIRE(m->h_taus && m->h_displacements && m->h_initial_rates && m->d_A &&
                  m->d_fixed_drifts && m->d_directions,
              "pipeline: null model array");
  LMM_REQUIRE(m->scramble_dims >= 0 &&
                  m->scramble_dims <= m->rates * m->factors &&
                  (m->scramble_dims == 0 || m->d_scramblers),
              "pipeline: bad scramble_dims");
  LMM_REQUIRE(pr->kind >= 0 && pr->kind <= 4, "pipeline: unknown product kind");
  v->n = m->rates;
  v->F = m->factors;
  v->D = m->rates * m->factors;
  memset(&v->mc, 0, sizeof(v->mc));
  v->mc.n = m->rates;
  v->mc.F = m->factors;
  v->mc.scr_dims = m->scramble_dims;
  v->mc.cutoff = m->cutoff;
  for (int r = 0; r < m->rates; ++r) {
    LMM_REQUIRE(m->h_taus[r] > 0.0f, "pipeline: tau must be positive");
    LMM_REQUIRE(m->h_initial_rates[r] + m->h_displacements[r] > 0.0f,
                "pipeline: displaced initial rate must be positive");
    v->mc.tau[r] = m->h_taus[r];
    v->mc.disp[r] = m->h_displacements[r];
    v->mc.logf0[r] = logf(m->h_initial_rates[r] + m->h_displacements[r]);
    v->mc.c0[r] = 1.0f - m->h_displacements[r] * m->h_taus[r];
    v->mc.l2tau[r] = (float)std::log2((double)m->h_taus[r]);
  }
  memset(&v->pc, 0, sizeof(v->pc));
  v->pc.kind = pr->kind;
  v->pc.strike = pr->strike;
  v->pc.cap_strike = pr->cap_strike;
  v->pc.pay_receive = pr->pay_receive;
  v->pc.tarn_total = pr->tarn_total;
  v->pc.tarn_mult = pr->tarn_multiplier;
  if (pr->kind == LMM_PRODUCT_TARN)
    LMM_REQUIRE(pr->tarn_total > 0.0f, "pipeline: TARN needs a positive total coupon");
  for (int s = 0; s < kMaxSteps; ++s) v->pc.ex_index[s] = -1;
  memset(&v->rc, 0, sizeof(v->rc));
  v->E = 0;
  if (!no_exercise(pr->kind)) {
    LMM_REQUIRE(pr->n_exercise >= 1 && pr->n_exercise <= m->rates &&
                    pr->h_exercise_steps && pr->h_nvars && pr->h_monomials &&
                    pr->h_nbasis,
                "pipeline: bad exercise schedule");
    v->E = pr->n_exercise;
    int last = -1;
    LSBasisSpec spec{pr->h_nvars, pr->h_monomials, pr->h_nbasis};
    for (int e = 0; e < v->E; ++e) {
      const int s = pr->h_exercise_steps[e];
      LMM_REQUIRE(s > last && s < m->rates,
                  "pipeline: exercise steps must increase within [0,rates)");
      last = s;
      v->pc.ex_index[s] = e;
      LSDate d;
      int st = ls_fill_date(spec, e, &d);
      if (st) return st;
      v->rc.nvars[e] = d.nvars;
      v->rc.nbasis[e] = d.nbasis;
      memcpy(v->rc.mono[e], d.mono, sizeof(d.mono));
    }
  }
  v->pc.n_ex = v->E;
  return LMM_OK;
}

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }


// Workspace carving helper.
struct Carver {
  char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t count) {
    T* p = reinterpret_cast<T*>(base ? base + off : nullptr);
    off += align_up(count * sizeof(T));
    return p;
  }
};

struct StagedBufs {
  uint32_t* sob;
  float *nrm, *brg, *corr, *rates, *lrates, *disc, *ann, *sr, *num_all;
  float *r1, *r2, *r3, *rate1_cf, *fl1, *fl2, *pfl;
  float *vars, *ex, *cf, *num;  // LS inputs of a second-pass batch
};

StagedBufs carve_staged(Carver& c, const Validated& v, size_t P) {
  StagedBufs b;
  const size_t n = v.n, S = v.n, F = v.F, D = v.D, E = v.E > 0 ? v.E : 1;
  b.sob = c.take<uint32_t>(D * P);
  b.nrm = c.take<float>(D * P);
  b.brg = c.take<float>(S * F * P);
  b.corr = c.take<float>(S * n * P);
  b.rates = c.take<float>(S * n * P);
  b.lrates = c.take<float>(S * n * P);
  b.disc = c.take<float>(S * (n + 1) * P);
  b.ann = c.take<float>(S * n * P);
  b.sr = c.take<float>(S * n * P);
  b.num_all = c.take<float>(n * P);
  b.r1 = c.take<float>(E * P);
  b.r2 = c.take<float>(E * P);
  b.r3 = c.take<float>(E * P);
  b.rate1_cf = c.take<float>(S * P);
  b.fl1 = c.take<float>(S * P);
  b.fl2 = c.take<float>(S * P);
  b.pfl = c.take<float>(S * P);
  b.vars = c.take<float>(E * 3 * P);
  b.ex = c.take<float>(E * P);
  b.cf = c.take<float>(E * P);
  b.num = c.take<float>(E * P);
  return b;
}

#define TRY(x)           \
  do {                   \
    int _st = (x);       \
    if (_st) return _st; \
  } while (0)

__global__ void sum3_kernel(const float* __restrict__ a,
                            const float* __restrict__ b,
                            const float* __restrict__ c, int n,
                            float* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    out[i] = a[i] + b[i] + c[i];
}

// Staged chain for one batch: LS inputs into columns [col, col+P) of
// arrays with `total` columns.  For the European product it stops after
// the numeraires.
int staged_inputs(const lmm_model* m, const lmm_product* pr, const Validated& v,
                  const StagedBufs& b, int P, uint32_t off, int total, int col,
                  float* vars, float* ex, float* cf, float* num,
                  cudaStream_t s) {
  const int n = v.n, S = v.n, F = v.F, D = v.D, E = v.E;
  lmm_stream_t ls = (lmm_stream_t)s;
  std::vector<int> alive(S);
  for (int i = 0; i < S; ++i) alive[i] = i;
  TRY(lmm_sobol_ints(P, D, off, m->d_directions, b.sob, ls));
  if (m->scramble_dims > 0)
    TRY(lmm_scramble(b.sob, m->d_scramblers, m->scramble_dims, P, ls));
  TRY(lmm_icdf_shaw_brickman_tails(b.sob, b.nrm, (size_t)D * P, ls));
  TRY(lmm_bridge_transform(b.nrm, b.brg, P, S, F, nullptr, ls));
  TRY(lmm_correlate_drift(b.brg, b.corr, m->d_A, alive.data(), m->d_fixed_drifts,
                          n * F, F, n, P, S, 1, ls));
  TRY(lmm_evolve_pc_staged(m->h_initial_rates, m->h_taus, m->h_displacements,
                           b.corr, m->d_A, alive.data(), P, F, S, n, m->cutoff, b.rates,
                           b.lrates, ls));
  TRY(lmm_discount_ratios(b.rates, m->h_taus, alive.data(), P, S, n, b.disc, ls));
  TRY(lmm_spot_numeraires(b.disc, P, P, 0, n, b.num_all, ls));
  if (no_exercise(pr->kind)) return LMM_OK;
  TRY(lmm_coterminal_annuities(b.disc, m->h_taus, alive.data(), P, S, n, b.ann, ls));
  TRY(lmm_coterminal_swap_rates(b.disc, b.ann, alive.data(), P, S, n, b.sr, ls));
  std::vector<int> ex_steps(pr->h_exercise_steps, pr->h_exercise_steps + E);
  std::vector<int> idx2(E), idx3(E);
  for (int e = 0; e < E; ++e) {
    const int st = ex_steps[e];
    if (swaption_exercise(pr->kind)) {
      idx2[e] = st;
      idx3[e] = st;
    } else {
      idx2[e] = st + 1 < n ? st + 1 : n - 1;
      idx3[e] = n - 1;
    }
  }
  TRY(lmm_forward_extraction_steps(b.rates, ex_steps.data(), ex_steps.data(), E, P, n, b.r1, ls));
  TRY(lmm_forward_extraction_steps(b.sr, idx2.data(), ex_steps.data(), E, P, n, b.r2, ls));
  TRY(lmm_forward_extraction_steps(b.ann, idx3.data(), ex_steps.data(), E, P, n, b.r3, ls));
  TRY(lmm_basis_variables(0, nullptr, b.r1, b.r2, b.r3, P, total, col, E, vars, ls));
  TRY(lmm_numeraire_extraction(b.num_all, num, P, total, col, n, E, ex_steps.data(), ls));
  TRY(check_cuda(cudaMemset2DAsync(cf + col, (size_t)total * sizeof(float), 0,
                                    (size_t)P * sizeof(float), E, s),
                 "pipeline: clear coupons"));
  if (swaption_exercise(pr->kind))
    return lmm_exercise_values_payer_swaption(pr->strike, b.r2, b.r3, P, total,
                                              col, E, ex, ls);
  // Cancellable payer swap: coupons of every step, discounted to the step
  // with the curve of that step, deflated to the preceding exercise date
  // and aggregated there; exercise (cancel) value 0.
  TRY(check_cuda(cudaMemset2DAsync(ex + col, (size_t)total * sizeof(float), 0,
                                    (size_t)P * sizeof(float), E, s),
                 "pipeline: clear exercise values"));
  std::vector<int> diag(S);
  for (int i = 0; i < S; ++i) diag[i] = i;
  TRY(lmm_forward_extraction(b.rates, diag.data(), P, S, n, b.rate1_cf, ls));
  std::vector<float> aux(2 + 2 * S);
  aux[0] = pr->strike;
  aux[1] = pr->pay_receive;
  for (int i = 0; i < S; ++i) aux[2 + i] = aux[2 + S + i] = m->h_taus[i];
  TRY(lmm_cashflows_swap(b.fl1, b.fl2, aux.data(), P, S, b.rate1_cf, ls));
  std::vector<int> gen(S), first(S), second(S), target(S), s2e(S);
  std::vector<float> theta(S, 1.0f);
  int first_pos = 0;
  TRY(lmm_step_to_exercise_indices(diag.data(), S, ex_steps.data(), E, s2e.data(),
                                   &first_pos));
  for (int i = 0; i < S; ++i) {
    gen[i] = i;
    first[i] = i;
    second[i] = i + 1;
    target[i] = s2e[i] >= 0 ? ex_steps[s2e[i]] : i;
  }
  for (float* fl : {b.fl1, b.fl2}) {
    TRY(lmm_cashflow_discounting_partial(S, gen.data(), first.data(), second.data(),
                                         theta.data(), target.data(), b.disc, fl,
                                         b.num_all, P, S, b.pfl, ls));
    TRY(lmm_aggregate_flows(cf, total, E, b.pfl, P, col, S, s2e.data(), first_pos, ls));
  }
  return LMM_OK;
}

// TARN in staged form: the reference's TARN flows (lmm_cashflows_tarn) on
// the reset rates, paid at T_{s+1} through the discounting kernel, summed.
int staged_tarn(const lmm_model* m, const lmm_product* pr, const Validated& v,
                const StagedBufs& b, int P, float* payoff, cudaStream_t s) {
  const int S = v.n;
  lmm_stream_t ls = (lmm_stream_t)s;
  std::vector<int> diag(S), first(S), second(S);
  std::vector<float> theta(S, 1.0f), aux(3 + 2 * S);
  for (int i = 0; i < S; ++i) {
    diag[i] = i;
    first[i] = i;
    second[i] = i + 1;
    aux[3 + i] = aux[3 + S + i] = m->h_taus[i];
  }
  aux[0] = pr->tarn_total;
  aux[1] = pr->strike;
  aux[2] = pr->tarn_multiplier;
  TRY(lmm_forward_extraction(b.rates, diag.data(), P, S, v.n, b.rate1_cf, ls));
  TRY(lmm_cashflows_tarn(b.fl1, b.fl2, aux.data(), P, S, b.rate1_cf, b.rate1_cf, ls));
  TRY(lmm_cashflow_discounting(first.data(), second.data(), theta.data(), b.disc, b.fl1,
                               b.num_all, P, S, b.corr, b.r1, ls));
  TRY(lmm_cashflow_discounting(first.data(), second.data(), theta.data(), b.disc, b.fl2,
                               b.num_all, P, S, b.corr, b.r2, ls));
  TRY(check_cuda(cudaMemsetAsync(b.r3, 0, (size_t)P * sizeof(float), s), "staged_tarn"));
  sum3_kernel<<<grid_for(P, 256, 4), 256, 0, s>>>(b.r1, b.r2, b.r3, P, payoff);
  return check_launch("sum3_kernel");
}

// European strip in staged form: caplet and swaplet flows paid at T_{s+1}
// through the reference's discounting kernel, summed per path.
int staged_european(const lmm_model* m, const lmm_product* pr, const Validated& v,
                    const StagedBufs& b, int P, float* payoff, cudaStream_t s) {
  const int S = v.n;
  lmm_stream_t ls = (lmm_stream_t)s;
  std::vector<int> diag(S), first(S), second(S);
  std::vector<float> theta(S, 1.0f);
  for (int i = 0; i < S; ++i) {
    diag[i] = i;
    first[i] = i;
    second[i] = i + 1;
  }
  TRY(lmm_forward_extraction(b.rates, diag.data(), P, S, v.n, b.rate1_cf, ls));
  std::vector<float> cap(1 + S), swp(2 + 2 * S);
  cap[0] = pr->cap_strike;
  swp[0] = pr->strike;
  swp[1] = pr->pay_receive;
  for (int i = 0; i < S; ++i) {
    cap[1 + i] = m->h_taus[i];
    swp[2 + i] = swp[2 + S + i] = m->h_taus[i];
  }
  // fl1: caplets; fl2: fixed leg; pfl: floating leg
  TRY(lmm_cashflows_caplet(b.fl1, b.pfl, cap.data(), P, S, b.rate1_cf, ls));
  TRY(lmm_cashflows_swap(b.fl2, b.pfl, swp.data(), P, S, b.rate1_cf, ls));
  float* tot[3] = {b.r1, b.r2, b.r3};
  const float* legs[3] = {b.fl1, b.fl2, b.pfl};
  for (int i = 0; i < 3; ++i)
    TRY(lmm_cashflow_discounting(first.data(), second.data(), theta.data(), b.disc,
                                 legs[i], b.num_all, P, S, b.corr, tot[i], ls));
  sum3_kernel<<<grid_for(P, 256, 4), 256, 0, s>>>(tot[0], tot[1], tot[2], P, payoff);
  return check_launch("sum3_kernel");
}

// Cap strip of LMM_PRODUCT_BERMUDAN_CAP in staged form: caplets on the
// reset rates paid at T_{s+1} through the reference's discounting kernel,
// summed per path and added to the swaption's frozen-rule payoff.
int staged_cap_add(const lmm_model* m, const lmm_product* pr, const Validated& v,
                   const StagedBufs& b, int P, float* payoff, cudaStream_t s) {
  const int S = v.n;
  lmm_stream_t ls = (lmm_stream_t)s;
  std::vector<int> diag(S), first(S), second(S);
  std::vector<float> theta(S, 1.0f), cap(1 + S);
  cap[0] = pr->cap_strike;
  for (int i = 0; i < S; ++i) {
    diag[i] = i;
    first[i] = i;
    second[i] = i + 1;
    cap[1 + i] = m->h_taus[i];
  }
  TRY(lmm_forward_extraction(b.rates, diag.data(), P, S, v.n, b.rate1_cf, ls));
  TRY(lmm_cashflows_caplet(b.fl1, b.pfl, cap.data(), P, S, b.rate1_cf, ls));
  TRY(lmm_cashflow_discounting(first.data(), second.data(), theta.data(), b.disc, b.fl1,
                               b.num_all, P, S, b.corr, b.r1, ls));
  TRY(check_cuda(cudaMemsetAsync(b.r3, 0, (size_t)P * sizeof(float), s), "staged_cap_add"));
  sum3_kernel<<<grid_for(P, 256, 4), 256, 0, s>>>(payoff, b.r1, b.r3, P, payoff);
  return check_launch("sum3_kernel");
}

template <int MODE>
int launch_fused(const Validated& v, int P, const float* Z, const lmm_model* m,
                 const LsRuleView& rule,
                 int total, int col, float* vars, float* ex, float* cf,
                 float* num, float* payoff, cudaStream_t s,
                 RecordOut rec = RecordOut{nullptr, nullptr, nullptr, 1},
                 const SegIO* segment = nullptr) {
  const int block = kFusedBlock;
  const size_t smem = fused_smem_bytes(v.n, v.F, block);
  const int grid = div_up(P, block);
  SegIO whole{};
  whole.s_begin = 0;
  whole.s_end = v.n;
  const SegIO& sg = segment ? *segment : whole;
  auto go = [&](auto kern) -> int {
    TRY(check_cuda(cudaFuncSetAttribute(kern,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem),
                   "fused: smem attribute"));
    kern<<<grid, block, smem, s>>>(P, Z, m->d_A, m->d_fixed_drifts, v.mc, v.pc,
                                   v.rc, rule, total, col, vars, ex,
                                   cf, num, payoff, rec, sg);
    return check_launch("fused_evolve_kernel");
  };
  switch (v.F) {
    case 3: return go(fused_evolve_kernel<3, MODE>);
    case 5: return go(fused_evolve_kernel<5, MODE>);
    case 10: return go(fused_evolve_kernel<10, MODE>);
    case 15: return go(fused_evolve_kernel<15, MODE>);
    default: return go(fused_evolve_kernel<0, MODE>);
  }
}

// Segmented rule-mode second pass (SegIO, fused_kernels.cuh): products whose
// paths stop at an exercise drop them every few steps.  Each segment launch
// packs its survivors per CTA; seg_scan_kernel turns the per-CTA counts into
// the prefix that the next launch's CTAs use to take the survivors densely
// and in path order.  Every path runs the same arithmetic as in one launch,
// so the payoffs are bit-identical to the unsegmented kernel's.
bool segmentable(const Validated& v) {
  return (v.pc.kind == LMM_PRODUCT_SWAPTION || v.pc.kind == LMM_PRODUCT_CANCELLABLE_SWAP) &&
         v.n > 1;
}

struct SegBufs {
  SegState st[2];
  int* count;
  int* prefix;
  int blocks, cap;
};

SegBufs carve_seg(Carver& c, const Validated& v, int P) {
  SegBufs b;
  b.blocks = div_up(P, kFusedBlock);
  b.cap = b.blocks * kFusedBlock;
  const size_t cap = (size_t)b.cap;
  for (SegState& st : b.st) {
    st.rates = c.take<float>((size_t)v.n * cap);
    st.N = c.take<float>(cap);
    st.f_first = c.take<float>(cap);
    st.pend_P1 = c.take<float>(cap);
    st.pend_coupon = c.take<float>(cap);
    st.payoff = c.take<double>(cap);
    st.path = c.take<int>(cap);
  }
  b.count = c.take<int>((size_t)b.blocks);
  b.prefix = c.take<int>((size_t)b.blocks + 1);
  return b;
}

size_t seg_ws_bytes(const Validated& v, int P) {
  if (!segmentable(v)) return 0;
  Carver c{nullptr};
  carve_seg(c, v, P);
  return c.off;
}

// The frozen-rule pass (MODE kModeRule, or kModeRecord with its record
// outputs) as a chain of launches of `len` steps over the survivor buffers b.
template <int MODE>
int fused_segments(const Validated& v, int P, const float* Z, const lmm_model* m,
                   const LsRuleView& rule, const SegBufs& b, int len, float* payoff,
                   cudaStream_t s, RecordOut rec = RecordOut{nullptr, nullptr, nullptr, 1}) {
  SegIO sg{};
  sg.cap = b.cap;
  sg.in_blocks = b.blocks;
  sg.out_count = b.count;
  for (int s0 = 0, k = 0; s0 < v.n; s0 += len, ++k) {
    sg.s_begin = s0;
    sg.s_end = std::min(s0 + len, v.n);
    sg.in_prefix = s0 > 0 ? b.prefix : nullptr;
    sg.in = b.st[(k + 1) & 1];
    sg.out = sg.s_end < v.n ? b.st[k & 1] : SegState{};
    TRY(launch_fused<MODE>(v, P, Z, m, rule, P, 0, nullptr, nullptr, nullptr, nullptr, payoff,
                           s, rec, &sg));
    if (sg.s_end < v.n) {
      seg_scan_kernel<<<1, 1024, 0, s>>>(b.count, b.blocks, b.prefix);
      TRY(check_launch("seg_scan_kernel"));
    }
  }
  return LMM_OK;
}

// segment_steps < 1: the library's kSegSteps; >= rates: one launch.
int fused_price(const Validated& v, int P, const float* Z, const lmm_model* m,
                const LsRuleView& rule, Carver& c, int segment_steps, float* payoff,
                cudaStream_t s) {
  const int len = segment_steps < 1 ? kSegSteps : segment_steps;
  if (!segmentable(v) || len >= v.n)
    return launch_fused<kModeRule>(v, P, Z, m, rule, P, 0, nullptr, nullptr, nullptr,
                                   nullptr, payoff, s);
  const SegBufs b = carve_seg(c, v, P);
  return fused_segments<kModeRule>(v, P, Z, m, rule, b, len, payoff, s);
}

int launch_variates(const Validated& v, const lmm_model* m, int P, uint32_t off,
                    float* out, cudaStream_t s) {
  BridgePlan plan;
  TRY(make_bridge_plan(v.n, v.F, nullptr, &plan));
  LMM_REQUIRE((uint64_t)off + (uint64_t)P + 1u < (1ull << 31),
              "pipeline: Sobol point index must stay below 2^31");
  const int block = kVarBlock;
  const size_t smem = variates_smem_bytes(v.n);
  TRY(check_cuda(cudaFuncSetAttribute(variates_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem),
                 "variates: smem attribute"));
  dim3 grid(div_up(P, block), v.F);
  variates_kernel<<<grid, block, smem, s>>>(P, off + 1u, m->d_directions,
                                            m->d_scramblers, m->scramble_dims,
                                            out, plan);
  return check_launch("variates_kernel");
}

// ------------------------------- adjoint -----------------------------------

struct GreeksBufs {
  float *Z, *payoff, *ckpt, *ckptN, *lam;
  // the recompute's output of one checkpoint segment, twice: segment cp in
  // buffer cp & 1, so that the next segment's recompute runs while this
  // one's reverse sweep reads it
  float *seg[2], *seg_info[2];
  int* ex_step;
  double *later, *lam_sum, *mean, *red;
  // the reverse launches' per-CTA partials, step s in part[s & 1]: a launch
  // sums the previous one's while writing its own
  double* part[2];
  // the paths' order for the reverse sweep, and a segment's checkpoint and
  // normals in it (the normals, read by the reverse sweep too, twice)
  int *perm, *ex_sorted, *cnt, *live, *tile_list;
  float *ckS, *ckNS, *Zs[2];
};

// Floats of the segment kernel's g, gp, ln output for k steps.
size_t greeks_seg_floats(size_t n, size_t P, int k) {
  return (size_t)k * n * ((P + kRevThreads - 1) / kRevThreads) * kSegRow;
}

// Upper bound on the CTAs of the reverse kernel (sizes the partials).
int greeks_reverse_grid(int P) {
  return std::min(div_up(P, kRevThreads), 6 * sm_count());
}

GreeksBufs carve_greeks(Carver& c, const Validated& v, size_t P, int k) {
  GreeksBufs b;
  const size_t n = v.n, F = v.F, C = (v.n + k - 1) / k;
  b.Z = c.take<float>(n * F * P);
  b.payoff = c.take<float>(P);
  b.ex_step = c.take<int>(P);
  b.ckpt = c.take<float>(C * n * P);
  b.ckptN = c.take<float>(C * P);
  for (int i = 0; i < 2; ++i) {
    b.seg[i] = c.take<float>(greeks_seg_floats(n, P, k));
    b.seg_info[i] = c.take<float>((size_t)k * (2 * F + 3) * P);
  }
  b.lam = c.take<float>(n * P);
  b.later = c.take<double>(P);
  for (int i = 0; i < 2; ++i)
    b.part[i] = c.take<double>((size_t)greeks_reverse_grid((int)P) * greeks_part_width(n, F));
  b.lam_sum = c.take<double>(n);
  b.mean = c.take<double>(1);
  b.red = c.take<double>(512);
  const size_t chunks = (P + kSortChunk - 1) / kSortChunk;
  b.perm = c.take<int>(P);
  b.ex_sorted = c.take<int>(P);
  b.cnt = c.take<int>(n * chunks);
  b.live = c.take<int>(n);
  b.tile_list = c.take<int>(n * ((P + kRevThreads - 1) / kRevThreads));
  b.ckS = c.take<float>(n * P);
  b.ckNS = c.take<float>(P);
  for (int i = 0; i < 2; ++i) b.Zs[i] = c.take<float>((size_t)k * F * P);
  return b;
}

// Calls go(std::integral_constant<int, FT>) with the compiled factor count
// (0 = generic).
template <class Fn>
int dispatch_factors(int F, Fn&& go) {
  switch (F) {
    case 3: return go(std::integral_constant<int, 3>());
    case 5: return go(std::integral_constant<int, 5>());
    case 10: return go(std::integral_constant<int, 10>());
    case 15: return go(std::integral_constant<int, 15>());
    default: return go(std::integral_constant<int, 0>());
  }
}

size_t workspace_bytes(const Validated& v, int paths, int mode) {
  Carver c{nullptr};
  if (mode == LMM_MODE_STAGED) {
    carve_staged(c, v, (size_t)paths);
  } else {
    c.take<float>((size_t)v.n * v.F * paths);
    if (mode == LMM_MODE_TENSOR) c.take<unsigned char>((size_t)v.n * TcGeom::make(v.n).b_bytes);
    if (mode == LMM_MODE_FUSED) c.off += seg_ws_bytes(v, paths);
  }
  return c.off + 256;
}

// Error word of the tensor-core kernels (bit 0: a bounded wait ran out).
__device__ unsigned int g_device_errors;

int device_errors_ptr(unsigned int** out) {
  static std::mutex mu;
  static unsigned int* ptr[64] = {};
  int dev = 0;
  TRY(check_cuda(cudaGetDevice(&dev), "device errors: cudaGetDevice"));
  LMM_REQUIRE(dev >= 0 && dev < 64, "device errors: device ordinal %d", dev);
  std::lock_guard<std::mutex> lock(mu);
  if (!ptr[dev]) {
    void* p = nullptr;
    TRY(check_cuda(cudaGetSymbolAddress(&p, g_device_errors),
                   "device errors: cudaGetSymbolAddress"));
    ptr[dev] = (unsigned int*)p;
  }
  *out = ptr[dev];
  return LMM_OK;
}

// Tensor-core evolution: builds the per-step B images into `img`, then runs
// tc_evolve_kernel (same arguments and outputs as launch_fused).
template <int MODE>
int launch_tensor(const Validated& v, int P, const float* Z, const lmm_model* m,
                  const LsRuleView& rule, int total,
                  int col, float* vars, float* ex, float* cf, float* num, float* payoff,
                  unsigned char* img, cudaStream_t s) {
  LMM_REQUIRE(v.F <= 16, "tensor evolution: at most 16 factors");
  if (v.pc.kind == LMM_PRODUCT_BERMUDAN_CAP)
    return fail(LMM_ENOTSUP, "tensor evolution: the swaption-plus-cap portfolio is not "
                             "available in LMM_MODE_TENSOR");
  const TcGeom G = TcGeom::make(v.n);
  unsigned int* errors = nullptr;
  TRY(device_errors_ptr(&errors));
  tc_b_image_kernel<<<dim3(G.NB, v.n), G.KT, 0, s>>>(v.n, v.F, m->d_A, img);
  TRY(check_launch("tc_b_image_kernel"));
  const size_t smem = tc_evolve_smem(v.n);
  TRY(check_cuda(cudaFuncSetAttribute(tc_evolve_kernel<MODE>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 "tensor evolution: smem attribute"));
  tc_evolve_kernel<MODE><<<div_up(P, tc::kThreads), tc::kThreads, smem, s>>>(
      P, Z, v.F, img, m->d_fixed_drifts, v.mc, v.pc, v.rc, rule, total, col, vars,
      ex, cf, num, payoff, errors);
  return check_launch("tc_evolve_kernel");
}

}  // namespace
}  // namespace lmm

using namespace lmm;

extern "C" size_t lmm_pipeline_workspace_bytes(const lmm_model* model,
                                               const lmm_product* product,
                                               int paths, int mode) {
  Validated v;
  if (validate(model, product, &v) != LMM_OK || paths < 1) return 0;
  return workspace_bytes(v, paths, mode);
}

extern "C" int lmm_pipeline_first_pass(const lmm_model* model,
                                       const lmm_product* product, int paths,
                                       uint32_t path_offset, int mode,
                                       void* d_workspace, size_t ws_bytes,
                                       int total_paths, int col_offset,
                                       float* d_vars, float* d_ex, float* d_cf,
                                       float* d_num, lmm_stream_t stream) {
  Validated v;
  TRY(validate(model, product, &v));
  LMM_REQUIRE(paths >= 1 && col_offset >= 0 && col_offset + paths <= total_paths,
              "lmm_pipeline_first_pass: bad path range");
  LMM_REQUIRE(!no_exercise(product->kind),
              "lmm_pipeline_first_pass: the product has no exercise and no regression");
  LMM_REQUIRE(d_vars && d_ex && d_cf && d_num && d_workspace,
              "lmm_pipeline_first_pass: null pointer");
  LMM_REQUIRE(mode == LMM_MODE_STAGED || mode == LMM_MODE_FUSED || mode == LMM_MODE_TENSOR,
              "lmm_pipeline_first_pass: unknown mode");
  const size_t need = workspace_bytes(v, paths, mode);
  if (ws_bytes < need)
    return fail(LMM_ENOMEM, "lmm_pipeline_first_pass: workspace %zu < %zu",
                ws_bytes, need);
  cudaStream_t s = (cudaStream_t)stream;
  Carver c{(char*)d_workspace};
  if (mode == LMM_MODE_STAGED) {
    StagedBufs b = carve_staged(c, v, (size_t)paths);
    return staged_inputs(model, product, v, b, paths, path_offset, total_paths,
                         col_offset, d_vars, d_ex, d_cf, d_num, s);
  }
  float* brg = c.take<float>((size_t)v.n * v.F * paths);
  TRY(launch_variates(v, model, paths, path_offset, brg, s));
  if (mode == LMM_MODE_TENSOR) {
    unsigned char* img = c.take<unsigned char>((size_t)v.n * TcGeom::make(v.n).b_bytes);
    return launch_tensor<kModeInputs>(v, paths, brg, model,
                                      ls_rule_view(nullptr, nullptr, nullptr), total_paths,
                                      col_offset, d_vars, d_ex, d_cf, d_num, nullptr, img, s);
  }
  return launch_fused<kModeInputs>(v, paths, brg, model, ls_rule_view(nullptr, nullptr, nullptr),
                                   total_paths, col_offset, d_vars, d_ex, d_cf, d_num, nullptr,
                                   s);
}

namespace {
// Rule of the ABI: depth within range, means and sds both or neither, cuts
// present when depth > 1.
int rule_from_abi(const lmm_ls_rule* r, LsRuleView* out, const char* who) {
  LMM_REQUIRE(r, "%s: null rule", who);
  LMM_REQUIRE(r->depth >= 1 && r->depth <= kMaxDepth, "%s: depth %d outside 1..%d", who,
              r->depth, kMaxDepth);
  LMM_REQUIRE(r->d_beta, "%s: null coefficients", who);
  LMM_REQUIRE(!r->d_means == !r->d_sds, "%s: means/sds mismatch", who);
  LMM_REQUIRE(r->depth == 1 || r->d_cuts, "%s: depth %d needs cut-offs", who, r->depth);
  *out = LsRuleView{r->depth, r->d_beta, r->d_means, r->d_sds,
                    r->depth > 1 ? r->d_cuts : nullptr, r->d_shifts};
  return LMM_OK;
}

int second_pass(const lmm_model* model, const lmm_product* product, int paths,
                uint32_t path_offset, int mode, const LsRuleView& rule, void* d_workspace,
                size_t ws_bytes, float* d_payoff, lmm_stream_t stream) {
  Validated v;
  TRY(validate(model, product, &v));
  LMM_REQUIRE(paths >= 1, "lmm_pipeline_second_pass: paths < 1");
  LMM_REQUIRE(d_payoff && d_workspace, "lmm_pipeline_second_pass: null pointer");
  LMM_REQUIRE(no_exercise(product->kind) || rule.beta,
              "lmm_pipeline_second_pass: null coefficients");
  LMM_REQUIRE(!rule.means == !rule.sds, "lmm_pipeline_second_pass: means/sds mismatch");
  LMM_REQUIRE(mode == LMM_MODE_STAGED || mode == LMM_MODE_FUSED || mode == LMM_MODE_TENSOR,
              "lmm_pipeline_second_pass: unknown mode");
  const size_t need = workspace_bytes(v, paths, mode);
  if (ws_bytes < need)
    return fail(LMM_ENOMEM, "lmm_pipeline_second_pass: workspace %zu < %zu",
                ws_bytes, need);
  cudaStream_t s = (cudaStream_t)stream;
  Carver c{(char*)d_workspace};
  if (mode == LMM_MODE_STAGED) {
    StagedBufs b = carve_staged(c, v, (size_t)paths);
    TRY(staged_inputs(model, product, v, b, paths, path_offset, paths, 0, b.vars,
                      b.ex, b.cf, b.num, s));
    if (product->kind == LMM_PRODUCT_EUROPEAN)
      return staged_european(model, product, v, b, paths, d_payoff, s);
    if (product->kind == LMM_PRODUCT_TARN)
      return staged_tarn(model, product, v, b, paths, d_payoff, s);
    ls_apply_rule_kernel<<<grid_for(paths, 256, 4), 256, 0, s>>>(
        v.E, paths, b.vars, b.cf, b.ex, b.num, v.rc, rule, d_payoff);
    TRY(check_launch("ls_apply_rule_kernel"));
    if (product->kind == LMM_PRODUCT_BERMUDAN_CAP)
      return staged_cap_add(model, product, v, b, paths, d_payoff, s);
    return LMM_OK;
  }
  float* brg = c.take<float>((size_t)v.n * v.F * paths);
  TRY(launch_variates(v, model, paths, path_offset, brg, s));
  if (mode == LMM_MODE_TENSOR) {
    unsigned char* img = c.take<unsigned char>((size_t)v.n * TcGeom::make(v.n).b_bytes);
    return launch_tensor<kModeRule>(v, paths, brg, model, rule, paths, 0,
                                    nullptr, nullptr, nullptr, nullptr, d_payoff, img, s);
  }
  return fused_price(v, paths, brg, model, rule, c, 0, d_payoff, s);
}

int apply_rule(int n_exercise, int paths, const float* d_vars, const int* h_nvars,
               const uint8_t* h_monomials, const int* h_nbasis, const float* d_cf,
               const float* d_ex, const float* d_num, const LsRuleView& rule,
               float* d_payoff, lmm_stream_t stream) {
  LMM_REQUIRE(n_exercise >= 1 && n_exercise <= kMaxSteps && paths >= 1,
              "lmm_ls_apply_rule: bad sizes");
  LMM_REQUIRE(d_vars && h_nvars && h_monomials && h_nbasis && d_num && rule.beta &&
                  d_payoff,
              "lmm_ls_apply_rule: null pointer");
  LMM_REQUIRE(!rule.means == !rule.sds, "lmm_ls_apply_rule: means/sds mismatch");
  RuleConst rc;
  memset(&rc, 0, sizeof(rc));
  LSBasisSpec spec{h_nvars, h_monomials, h_nbasis};
  for (int e = 0; e < n_exercise; ++e) {
    LSDate d;
    TRY(ls_fill_date(spec, e, &d));
    rc.nvars[e] = d.nvars;
    rc.nbasis[e] = d.nbasis;
    memcpy(rc.mono[e], d.mono, sizeof(d.mono));
  }
  cudaStream_t s = (cudaStream_t)stream;
  ls_apply_rule_kernel<<<grid_for(paths, 256, 4), 256, 0, s>>>(
      n_exercise, paths, d_vars, d_cf, d_ex, d_num, rc, rule, d_payoff);
  return check_launch("lmm_ls_apply_rule");
}
}  // namespace

extern "C" int lmm_pipeline_second_pass(const lmm_model* model,
                                        const lmm_product* product, int paths,
                                        uint32_t path_offset, int mode,
                                        const double* d_beta,
                                        const float* d_means, const float* d_sds,
                                        void* d_workspace, size_t ws_bytes,
                                        float* d_payoff, lmm_stream_t stream) {
  return second_pass(model, product, paths, path_offset, mode,
                     ls_rule_view(d_beta, d_means, d_sds), d_workspace, ws_bytes, d_payoff,
                     stream);
}

extern "C" int lmm_pipeline_second_pass_rule(const lmm_model* model,
                                             const lmm_product* product, int paths,
                                             uint32_t path_offset, int mode,
                                             const lmm_ls_rule* rule, void* d_workspace,
                                             size_t ws_bytes, float* d_payoff,
                                             lmm_stream_t stream) {
  LsRuleView view;
  if (product && no_exercise(product->kind)) {
    view = ls_rule_view(nullptr, nullptr, nullptr);
  } else {
    TRY(rule_from_abi(rule, &view, "lmm_pipeline_second_pass_rule"));
  }
  return second_pass(model, product, paths, path_offset, mode, view, d_workspace, ws_bytes,
                     d_payoff, stream);
}

extern "C" int lmm_ls_apply_rule(int n_exercise, int paths, const float* d_vars,
                                 const int* h_nvars, const uint8_t* h_monomials,
                                 const int* h_nbasis, const float* d_cf,
                                 const float* d_ex, const float* d_num,
                                 const double* d_beta, const float* d_means,
                                 const float* d_sds, float* d_payoff,
                                 lmm_stream_t stream) {
  return apply_rule(n_exercise, paths, d_vars, h_nvars, h_monomials, h_nbasis, d_cf, d_ex,
                    d_num, ls_rule_view(d_beta, d_means, d_sds), d_payoff, stream);
}

extern "C" int lmm_ls_apply_rule_nested(int n_exercise, int paths, const float* d_vars,
                                        const int* h_nvars, const uint8_t* h_monomials,
                                        const int* h_nbasis, const float* d_cf,
                                        const float* d_ex, const float* d_num,
                                        const lmm_ls_rule* rule, float* d_payoff,
                                        lmm_stream_t stream) {
  LsRuleView view;
  TRY(rule_from_abi(rule, &view, "lmm_ls_apply_rule_nested"));
  return apply_rule(n_exercise, paths, d_vars, h_nvars, h_monomials, h_nbasis, d_cf, d_ex,
                    d_num, view, d_payoff, stream);
}

extern "C" int lmm_fused_variates(const lmm_model* model, int paths,
                                  uint32_t path_offset, float* d_variates,
                                  lmm_stream_t stream) {
  LMM_REQUIRE(model, "lmm_fused_variates: null model");
  lmm_product dummy;
  memset(&dummy, 0, sizeof(dummy));
  dummy.kind = LMM_PRODUCT_EUROPEAN;
  Validated v;
  TRY(validate(model, &dummy, &v));
  LMM_REQUIRE(paths >= 1 && d_variates, "lmm_fused_variates: bad arguments");
  return launch_variates(v, model, paths, path_offset, d_variates,
                         (cudaStream_t)stream);
}

extern "C" int lmm_fused_evolve(const lmm_model* model,
                                const lmm_product* product, int paths,
                                const float* d_variates, const double* d_beta,
                                const float* d_means, const float* d_sds,
                                int total_paths, int col_offset, float* d_vars,
                                float* d_ex, float* d_cf, float* d_num,
                                float* d_payoff, lmm_stream_t stream) {
  Validated v;
  TRY(validate(model, product, &v));
  LMM_REQUIRE(paths >= 1 && d_variates, "lmm_fused_evolve: bad arguments");
  LMM_REQUIRE(!d_means == !d_sds, "lmm_fused_evolve: means/sds mismatch");
  cudaStream_t s = (cudaStream_t)stream;
  if (d_beta == nullptr && !no_exercise(product->kind)) {
    LMM_REQUIRE(col_offset >= 0 && col_offset + paths <= total_paths && d_vars &&
                    d_ex && d_cf && d_num,
                "lmm_fused_evolve: bad LS-input arrays");
    return launch_fused<kModeInputs>(v, paths, d_variates, model,
                                     ls_rule_view(nullptr, nullptr, nullptr),
                                     total_paths, col_offset, d_vars,
                                     d_ex, d_cf, d_num, nullptr, s);
  }
  LMM_REQUIRE(d_payoff, "lmm_fused_evolve: null payoff");
  return launch_fused<kModeRule>(v, paths, d_variates, model,
                                 ls_rule_view(d_beta, d_means, d_sds), paths, 0, nullptr,
                                 nullptr, nullptr, nullptr, d_payoff, s);
}

extern "C" size_t lmm_fused_price_workspace_bytes(const lmm_model* model,
                                                  const lmm_product* product, int paths) {
  Validated v;
  if (validate(model, product, &v) != LMM_OK || paths < 1) return 0;
  return seg_ws_bytes(v, paths) + 256;
}

extern "C" int lmm_fused_price(const lmm_model* model, const lmm_product* product, int paths,
                               const float* d_variates, const lmm_ls_rule* rule,
                               int segment_steps, void* d_workspace, size_t workspace_bytes,
                               float* d_payoff, lmm_stream_t stream) {
  Validated v;
  TRY(validate(model, product, &v));
  LMM_REQUIRE(paths >= 1 && d_variates && d_payoff, "lmm_fused_price: bad arguments");
  LsRuleView view = ls_rule_view(nullptr, nullptr, nullptr);
  if (!no_exercise(product->kind)) TRY(rule_from_abi(rule, &view, "lmm_fused_price"));
  const int len = segment_steps < 1 ? kSegSteps : segment_steps;
  const size_t need = len < v.n ? seg_ws_bytes(v, paths) : 0;  // one launch needs none
  LMM_REQUIRE(need == 0 || (d_workspace && workspace_bytes >= need),
              "lmm_fused_price: workspace %zu < %zu", workspace_bytes, need);
  Carver c{(char*)d_workspace};
  return fused_price(v, paths, d_variates, model, view, c, segment_steps, d_payoff,
                     (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Pathwise adjoint Greeks (greeks_kernels.cuh).
// ---------------------------------------------------------------------------

// The adjoint's two internal streams and their events, one set per host
// thread and device, made on the thread's first call on the device and kept
// until the process exits.  The reverse sweep runs on `hi` (the device's
// highest stream priority), the recompute of later segments on `lo` (the
// lowest); both fork from the caller's stream and join it again.
struct GreeksStreams {
  cudaStream_t hi = nullptr, lo = nullptr;
  cudaEvent_t fork, join_hi, join_lo, seg_done[2], rev_done[2];
};

int greeks_streams(GreeksStreams** out) {
  constexpr int kMaxDevices = 64;
  thread_local GreeksStreams cache[kMaxDevices];
  int dev = 0;
  TRY(check_cuda(cudaGetDevice(&dev), "lmm_greeks: device"));
  LMM_REQUIRE(dev >= 0 && dev < kMaxDevices, "lmm_greeks: device %d out of range", dev);
  GreeksStreams& g = cache[dev];
  if (!g.hi) {
    int least = 0, greatest = 0;
    TRY(check_cuda(cudaDeviceGetStreamPriorityRange(&least, &greatest),
                   "lmm_greeks: stream priorities"));
    cudaEvent_t* evs[] = {&g.fork, &g.join_hi, &g.join_lo, &g.seg_done[0], &g.seg_done[1],
                          &g.rev_done[0], &g.rev_done[1]};
    for (cudaEvent_t* e : evs)
      TRY(check_cuda(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "lmm_greeks: event"));
    TRY(check_cuda(cudaStreamCreateWithPriority(&g.lo, cudaStreamNonBlocking, least),
                   "lmm_greeks: stream"));
    // made last: a set whose `hi` is not null is complete
    TRY(check_cuda(cudaStreamCreateWithPriority(&g.hi, cudaStreamNonBlocking, greatest),
                   "lmm_greeks: stream"));
  }
  *out = &g;
  return LMM_OK;
}

extern "C" size_t lmm_greeks_workspace_bytes(const lmm_model* model,
                                             const lmm_product* product,
                                             int paths, int checkpoint_every) {
  Validated v;
  if (validate(model, product, &v) != LMM_OK || paths < 4 || checkpoint_every < 1)
    return 0;
  Carver c{nullptr};
  carve_greeks(c, v, (size_t)paths, std::min(checkpoint_every, v.n));
  return c.off + 256;
}

extern "C" int lmm_greeks(const lmm_model* model, const lmm_product* product,
                          int paths, uint32_t path_offset, const double* d_beta,
                          const float* d_means, const float* d_sds, float t0,
                          int checkpoint_every, void* d_workspace,
                          size_t ws_bytes, double* d_price, double* d_delta,
                          double* d_abar, double* d_vega_rate, int* d_exercise_step,
                          int* d_status, lmm_stream_t stream) {
  Validated v;
  TRY(validate(model, product, &v));
  LMM_REQUIRE(paths >= 4 && paths % 4 == 0,
              "lmm_greeks: paths must be a positive multiple of 4");
  LMM_REQUIRE(checkpoint_every >= 1, "lmm_greeks: checkpoint_every < 1");
  LMM_REQUIRE(t0 > 0.0f, "lmm_greeks: t0 must be positive");
  LMM_REQUIRE(d_workspace && d_delta && d_abar && d_status,
              "lmm_greeks: null pointer");
  LMM_REQUIRE(product->kind != LMM_PRODUCT_TARN,
              "lmm_greeks: the TARN's knock-out is not differentiable pathwise");
  LMM_REQUIRE(product->kind == LMM_PRODUCT_EUROPEAN || d_beta,
              "lmm_greeks: null coefficients");
  LMM_REQUIRE(!d_means == !d_sds, "lmm_greeks: means/sds mismatch");
  const int n = v.n, F = v.F, P = paths;
  const int k = std::min(checkpoint_every, n);
  Carver c{(char*)d_workspace};
  GreeksBufs b = carve_greeks(c, v, (size_t)P, k);
  if (ws_bytes < c.off + 256)
    return fail(LMM_ENOMEM, "lmm_greeks: workspace %zu < %zu", ws_bytes, c.off + 256);
  cudaStream_t s = (cudaStream_t)stream;
  TRY(check_cuda(cudaMemsetAsync(d_status, 0, sizeof(int), s), "lmm_greeks: status"));
  // forward: variates, then the frozen-rule pass recording checkpoints
  TRY(launch_variates(v, model, P, path_offset, b.Z, s));
  RecordOut rec{b.ckpt, b.ckptN, b.ex_step, k};
  // The record pass drops exercised paths between segments like the pricing
  // pass (their later checkpoints are never read); its survivor buffers
  // alias the recompute buffers of the reverse sweep, unused until then.
  const LsRuleView rule = ls_rule_view(d_beta, d_means, d_sds);
  const size_t recompute_bytes = greeks_seg_floats(n, P, k) * sizeof(float);
  if (segmentable(v) && kSegSteps < n && seg_ws_bytes(v, P) <= recompute_bytes) {
    Carver sc{(char*)b.seg[0]};
    const SegBufs sb = carve_seg(sc, v, P);
    TRY(fused_segments<kModeRecord>(v, P, b.Z, model, rule, sb, kSegSteps, b.payoff, s, rec));
  } else {
    TRY(launch_fused<kModeRecord>(v, P, b.Z, model, rule, P, 0, nullptr, nullptr, nullptr,
                                  nullptr, b.payoff, s, rec));
  }
  TRY(check_cuda(cudaMemsetAsync(b.lam, 0, (size_t)n * P * sizeof(float), s),
                 "lmm_greeks: clear adjoint"));
  TRY(check_cuda(cudaMemsetAsync(b.later, 0, (size_t)P * sizeof(double), s),
                 "lmm_greeks: clear flows"));
  const double P0 = 1.0 / (1.0 + (double)model->h_initial_rates[0] * (double)t0);
  const double scale = P0 / (double)P;
  const int block_seg = kRevThreads;  // one tile of the reverse sweep per CTA
  const size_t smem_seg = fused_smem_bytes(n, F, block_seg);
  const size_t smem_rev = greeks_reverse_smem(n, F);
  // persistent CTAs: as many as are resident at once (at most the bound)
  int grid_rev = greeks_reverse_grid(P);
  TRY(dispatch_factors(F, [&](auto ft) -> int {
    constexpr int FT = decltype(ft)::value;
    auto kern = greeks_reverse_kernel<FT>;
    TRY(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem_rev),
                   "greeks: reverse smem"));
    int per_sm = 0;
    TRY(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kRevThreads,
                                                                 smem_rev),
                   "greeks: occupancy"));
    grid_rev = std::max(1, std::min(grid_rev, std::max(per_sm, 1) * sm_count()));
    return LMM_OK;
  }));
  const int abar_entries = n * F + n;  // dV/dA_s and the adjoint sums
  const int C = (n + k - 1) / k;
  const int stop_rule = product->kind == LMM_PRODUCT_SWAPTION ? 1
                        : product->kind == LMM_PRODUCT_BERMUDAN_CAP ? 2 : 0;
  // Paths that stop early leave idle lanes in their warps: order them by
  // their last step with work (products whose paths all run to the last
  // step keep the simulation order).
  const bool ordered = stop_rule != 2 && product->kind != LMM_PRODUCT_EUROPEAN;
  const int chunks = div_up(P, kSortChunk);
  if (ordered) {
    greeks_sort_kernel<<<chunks, kSortThreads, 0, s>>>(P, n, stop_rule, b.ex_step, chunks,
                                                        b.perm, b.ex_sorted, b.cnt);
    TRY(check_launch("greeks_sort_kernel"));
    greeks_live_tiles_kernel<<<n, 32, 0, s>>>(chunks, div_up(P, kRevThreads), b.cnt, b.live,
                                              b.tile_list);
    TRY(check_launch("greeks_live_tiles_kernel"));
  }
  const int* ex_rev = ordered ? b.ex_sorted : b.ex_step;
  const int* cnt = ordered ? b.cnt : nullptr;
  // The segments' recompute (gather into the order, then the segment
  // kernel; segment cp into buffer cp & 1) runs on the low-priority stream
  // up to two segments ahead of the reverse sweep on the high-priority one:
  // segment cp - 2 starts once the sweep of segment cp, the last reader of
  // its buffer, is done, and fills the SMs the sweep's launches leave idle.
  GreeksStreams* gs = nullptr;
  TRY(greeks_streams(&gs));
  TRY(dispatch_factors(F, [&](auto ft) -> int {
    constexpr int FT = decltype(ft)::value;
    return check_cuda(cudaFuncSetAttribute(greeks_segment_kernel<FT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem_seg),
                      "greeks: segment smem");
  }));
  auto seg_range = [&](int cp, int& s0, int& s1) {
    s0 = cp * k;
    s1 = std::min(n, s0 + k);
  };
  auto recompute = [&](int cp) -> int {  // on gs->lo
    int s0, s1;
    seg_range(cp, s0, s1);
    const int bi = cp & 1;
    const float* ck = b.ckpt + (size_t)cp * n * P;
    const float* ckN = b.ckptN + (size_t)cp * P;
    const float* Zseg = b.Z;
    int zs0 = 0;
    if (ordered) {
      const dim3 g(chunks, div_up((n - s0) + 1 + (s1 - s0) * F, kGatherRows));
      greeks_gather_kernel<<<g, kGatherThreads, 0, gs->lo>>>(P, n, F, s0, s1, chunks, b.perm,
                                                              b.cnt, ck, ckN, b.Z, b.ckS, b.ckNS,
                                                              b.Zs[bi]);
      TRY(check_launch("greeks_gather_kernel"));
      ck = b.ckS;
      ckN = b.ckNS;
      Zseg = b.Zs[bi];
      zs0 = s0;
    }
    TRY(dispatch_factors(F, [&](auto ft) -> int {
      constexpr int FT = decltype(ft)::value;
      greeks_segment_kernel<FT><<<div_up(P, block_seg), block_seg, smem_seg, gs->lo>>>(
          P, s0, s1, Zseg, zs0, cnt, chunks, model->d_A, model->d_fixed_drifts, v.mc, ck, ckN,
          ex_rev, stop_rule, b.seg[bi], b.seg_info[bi]);
      return check_launch("greeks_segment_kernel");
    }));
    return check_cuda(cudaEventRecord(gs->seg_done[bi], gs->lo), "lmm_greeks: event");
  };
  auto sweep = [&](int cp) -> int {  // on gs->hi
    int s0, s1;
    seg_range(cp, s0, s1);
    const int bi = cp & 1;
    const float* Zseg = ordered ? b.Zs[bi] : b.Z;
    const int zs0 = ordered ? s0 : 0;
    TRY(check_cuda(cudaStreamWaitEvent(gs->hi, gs->seg_done[bi], 0), "lmm_greeks: wait"));
    for (int st = s1 - 1; st >= s0; --st) {
      // this launch writes step st's partials and first sums step st + 1's
      GreeksStepBufs gb{b.lam, b.later, b.part[st & 1]};
      const GreeksPrevSums prev{st + 1 < n ? b.part[(st + 1) & 1] : nullptr, st + 1, grid_rev,
                                scale, d_abar};
      const size_t ko = (size_t)(st - s0);
      GreeksStepIn in{b.seg[bi] + ko * (greeks_seg_floats(n, P, 1)),
                      b.seg_info[bi] + ko * (2 * F + 3) * P};
      TRY(dispatch_factors(F, [&](auto ft) -> int {
        constexpr int FT = decltype(ft)::value;
        greeks_reverse_kernel<FT><<<grid_rev, kRevThreads, smem_rev, gs->hi>>>(
            P, st, Zseg, zs0, ordered ? b.live : nullptr, ordered ? b.tile_list : nullptr,
            model->d_A, v.mc, v.pc, in, ex_rev, gb, prev);
        return check_launch("greeks_reverse_kernel");
      }));
    }
    return check_cuda(cudaEventRecord(gs->rev_done[bi], gs->hi), "lmm_greeks: event");
  };
  TRY(check_cuda(cudaEventRecord(gs->fork, s), "lmm_greeks: fork"));
  TRY(check_cuda(cudaStreamWaitEvent(gs->hi, gs->fork, 0), "lmm_greeks: fork"));
  TRY(check_cuda(cudaStreamWaitEvent(gs->lo, gs->fork, 0), "lmm_greeks: fork"));
  const int rc = [&]() -> int {
    TRY(recompute(C - 1));
    if (C >= 2) TRY(recompute(C - 2));
    for (int cp = C - 1; cp >= 0; --cp) {
      TRY(sweep(cp));
      if (cp >= 2) {
        TRY(check_cuda(cudaStreamWaitEvent(gs->lo, gs->rev_done[cp & 1], 0),
                       "lmm_greeks: wait"));
        TRY(recompute(cp - 2));
      }
    }
    // step 0's dV/dA and the rate adjoints behind the deltas (the other
    // steps' sums ran at the start of the next reverse launch)
    greeks_abar_kernel<<<div_up((long long)abar_entries * 32, kAbarThreads), kAbarThreads, 0,
                         gs->hi>>>(n, F, 0, grid_rev, scale, b.part[0], model->d_A, d_abar,
                                   b.lam_sum);
    return check_launch("greeks_abar_kernel");
  }();
  // join both streams (after a failed launch too, so that nothing the call
  // forked is left outside the caller's stream)
  TRY(check_cuda(cudaEventRecord(gs->join_hi, gs->hi), "lmm_greeks: join"));
  TRY(check_cuda(cudaEventRecord(gs->join_lo, gs->lo), "lmm_greeks: join"));
  TRY(check_cuda(cudaStreamWaitEvent(s, gs->join_hi, 0), "lmm_greeks: join"));
  TRY(check_cuda(cudaStreamWaitEvent(s, gs->join_lo, 0), "lmm_greeks: join"));
  TRY(rc);
  TRY(reduce_launch(b.payoff, nullptr, (size_t)P, 1.0 / (double)P, b.red, b.mean, s));
  if (d_exercise_step)
    TRY(check_cuda(cudaMemcpyAsync(d_exercise_step, b.ex_step, (size_t)P * sizeof(int),
                                   cudaMemcpyDeviceToDevice, s),
                   "lmm_greeks: exercise steps"));
  greeks_finish_kernel<<<div_up(n, 128), 128, 0, s>>>(
      n, F, v.mc, model->h_initial_rates[0], t0, b.lam_sum, b.mean, model->d_A, d_abar,
      d_price, d_delta, d_vega_rate);
  return check_launch("greeks_finish_kernel");
}

// ---------------------------------------------------------------------------
// The tensor-core evolution as a separate kernel (lmm_fused_evolve's
// arguments plus a scratch of lmm_tensor_evolve_workspace_bytes for the
// per-step B images).
// ---------------------------------------------------------------------------
extern "C" size_t lmm_tensor_evolve_workspace_bytes(const lmm_model* model) {
  if (!model || model->rates < 2 || model->rates > kMaxRates) return 0;
  return (size_t)model->rates * TcGeom::make(model->rates).b_bytes;
}

extern "C" int lmm_tensor_evolve(const lmm_model* model, const lmm_product* product,
                                 int paths, const float* d_variates, const double* d_beta,
                                 const float* d_means, const float* d_sds, int total_paths,
                                 int col_offset, float* d_vars, float* d_ex, float* d_cf,
                                 float* d_num, float* d_payoff, void* d_workspace,
                                 size_t workspace_bytes, lmm_stream_t stream) {
  Validated v;
  TRY(validate(model, product, &v));
  LMM_REQUIRE(paths >= 1 && d_variates && d_workspace, "lmm_tensor_evolve: bad arguments");
  LMM_REQUIRE(workspace_bytes >= lmm_tensor_evolve_workspace_bytes(model),
              "lmm_tensor_evolve: workspace too small");
  LMM_REQUIRE(!d_means == !d_sds, "lmm_tensor_evolve: means/sds mismatch");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char* img = (unsigned char*)d_workspace;
  if (d_beta == nullptr && !no_exercise(product->kind)) {
    LMM_REQUIRE(col_offset >= 0 && col_offset + paths <= total_paths && d_vars && d_ex &&
                    d_cf && d_num,
                "lmm_tensor_evolve: bad LS-input arrays");
    return launch_tensor<kModeInputs>(v, paths, d_variates, model,
                                      ls_rule_view(nullptr, nullptr, nullptr),
                                      total_paths, col_offset, d_vars, d_ex, d_cf, d_num,
                                      nullptr, img, s);
  }
  LMM_REQUIRE(d_payoff, "lmm_tensor_evolve: null payoff");
  return launch_tensor<kModeRule>(v, paths, d_variates, model,
                                  ls_rule_view(d_beta, d_means, d_sds), paths,
                                  0, nullptr, nullptr, nullptr, nullptr, d_payoff, img, s);
}

// ---------------------------------------------------------------------------
// Andersen–Broadie upper bound (ab_kernels.cuh).
// ---------------------------------------------------------------------------
namespace {
struct AbBufs {
  float* brg;     // outer variates [n][F][K]
  float* vars;    // [E][3][K]
  float* ex;
  float* cf;
  float* num;     // [E][K]
  float* ckpt;    // [n][n][K]
  float* ckptN;   // [n][K]
  int* X;         // [E][K]
  double* Z;      // [E][K]
  double* Q;      // [E][K]
  double* part;   // inner partials [(E-1) K chunks][2]
  double* gpart;  // gap partials
};

int ab_check(const lmm_ab_config* cfg, const Validated& v) {
  LMM_REQUIRE(cfg, "lmm_andersen_broadie: null config");
  LMM_REQUIRE(v.pc.kind == LMM_PRODUCT_SWAPTION,
              "lmm_andersen_broadie: the Bermudan payer swaption only");
  LMM_REQUIRE(v.E >= 2, "lmm_andersen_broadie: needs two exercise dates or more");
  LMM_REQUIRE(cfg->outer_paths >= 1 && cfg->inner_paths >= kAbThreads &&
                  cfg->inner_paths % kAbThreads == 0,
              "lmm_andersen_broadie: outer_paths >= 1, inner_paths a multiple of %d",
              kAbThreads);
  const double ctas = (double)(v.E - 1) * cfg->outer_paths * (cfg->inner_paths / kAbThreads);
  LMM_REQUIRE(ctas < 2.0e9, "lmm_andersen_broadie: too many inner CTAs");
  return LMM_OK;
}

AbBufs carve_ab(Carver& c, const Validated& v, const lmm_ab_config* cfg) {
  const size_t K = (size_t)cfg->outer_paths, n = v.n, E = v.E;
  const size_t chunks = (size_t)cfg->inner_paths / kAbThreads;
  AbBufs b;
  b.brg = c.take<float>(n * v.F * K);
  b.vars = c.take<float>(E * kMaxVars * K);
  b.ex = c.take<float>(E * K);
  b.cf = c.take<float>(E * K);
  b.num = c.take<float>(E * K);
  b.ckpt = c.take<float>(n * n * K);
  b.ckptN = c.take<float>(n * K);
  b.X = c.take<int>(E * K);
  b.Z = c.take<double>(E * K);
  b.Q = c.take<double>(E * K);
  b.part = c.take<double>((E - 1) * K * chunks * 2);
  b.gpart = c.take<double>((size_t)div_up((long long)K, 256) * 4);
  return b;
}

AbGapArgs gap_args(int steps, int paths, long long m_p, long long m_s, const int* is_ex) {
  AbGapArgs g;
  memset(&g, 0, sizeof(g));
  g.steps = steps;
  g.paths = paths;
  g.m_p = m_p;
  g.m_s = m_s;
  for (int s = 0; s < steps; ++s)
    if (is_ex[s]) g.is_ex[s >> 5] |= 1u << (s & 31);
  return g;
}

int launch_gap(const AbGapArgs& g, const int* ex, const double* payoffs, const double* means,
               double* gpart, double* out, cudaStream_t s) {
  const int nb = div_up(g.paths, 256);
  ab_gap_kernel<<<nb, 256, 0, s>>>(g, ex, payoffs, means, gpart);
  TRY(check_launch("ab_gap_kernel"));
  ab_gap_final_kernel<<<1, 32, 0, s>>>(nb, g.paths, gpart, out);
  return check_launch("ab_gap_final_kernel");
}
}  // namespace

extern "C" size_t lmm_andersen_broadie_workspace_bytes(const lmm_model* model,
                                                       const lmm_product* product,
                                                       const lmm_ab_config* cfg) {
  Validated v;
  if (validate(model, product, &v) || ab_check(cfg, v)) return 0;
  Carver c{nullptr};
  carve_ab(c, v, cfg);
  return c.off;
}

extern "C" int lmm_andersen_broadie(const lmm_model* model, const lmm_product* product,
                                    const lmm_ls_rule* rule, const lmm_ab_config* cfg,
                                    void* d_workspace, size_t workspace_bytes, double* d_out,
                                    double* d_Q, int* d_X, double* d_Z, float* d_ckpt,
                                    float* d_ckptN, lmm_stream_t stream) {
  Validated v;
  TRY(validate(model, product, &v));
  TRY(ab_check(cfg, v));
  LsRuleView view;
  TRY(rule_from_abi(rule, &view, "lmm_andersen_broadie"));
  LMM_REQUIRE(d_workspace && d_out, "lmm_andersen_broadie: null pointer");
  Carver c{(char*)d_workspace};
  AbBufs b = carve_ab(c, v, cfg);
  LMM_REQUIRE(workspace_bytes >= c.off, "lmm_andersen_broadie: workspace too small (%zu < %zu)",
              workspace_bytes, c.off);
  if (d_Q) b.Q = d_Q;
  if (d_X) b.X = d_X;
  if (d_Z) b.Z = d_Z;
  if (d_ckpt) b.ckpt = d_ckpt;
  if (d_ckptN) b.ckptN = d_ckptN;
  cudaStream_t s = (cudaStream_t)stream;
  const int K = cfg->outer_paths, E = v.E, n = v.n;
  const int chunks = cfg->inner_paths / kAbThreads;
  // outer paths: LS inputs at every date and the state at every step
  TRY(launch_variates(v, model, K, cfg->outer_offset, b.brg, s));
  TRY(launch_fused<kModeOuter>(v, K, b.brg, model, view, K, 0, b.vars, b.ex, b.cf, b.num,
                               nullptr, s, RecordOut{b.ckpt, b.ckptN, nullptr, 1}));
  ab_decide_kernel<<<div_up(E * K, 256), 256, 0, s>>>(E, K, v.rc, view, b.vars, b.ex, b.num,
                                                     b.X, b.Z);
  TRY(check_launch("ab_decide_kernel"));
  // inner paths from every (outer path, date) but the last date
  AbArgs a;
  memset(&a, 0, sizeof(a));
  a.K = K;
  a.chunks = chunks;
  a.e0 = 0;
  a.k0 = (uint32_t)cfg->seed;
  a.k1 = (uint32_t)(cfg->seed >> 32);
  for (int s2 = 0, e = 0; s2 < n; ++s2)
    if (v.pc.ex_index[s2] >= 0) a.ex_step[e++] = s2;
  const size_t smem = ab_inner_smem(n);
  const unsigned grid = (unsigned)((size_t)(E - 1) * K * chunks);
  auto go = [&](auto kern) -> int {
    TRY(check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem),
                   "ab_inner: smem attribute"));
    kern<<<grid, kAbThreads, smem, s>>>(a, model->d_A, model->d_fixed_drifts, v.mc, v.pc, v.rc,
                                        view, b.ckpt, b.ckptN, b.part);
    return check_launch("ab_inner_kernel");
  };
  switch (v.F) {
    case 3: TRY(go(ab_inner_kernel<3>)); break;
    case 5: TRY(go(ab_inner_kernel<5>)); break;
    case 10: TRY(go(ab_inner_kernel<10>)); break;
    case 15: TRY(go(ab_inner_kernel<15>)); break;
    default: TRY(go(ab_inner_kernel<0>)); break;
  }
  ab_continuation_kernel<<<div_up(E * K, 256), 256, 0, s>>>(E, K, chunks, cfg->inner_paths,
                                                           b.part, b.Q, nullptr);
  TRY(check_launch("ab_continuation_kernel"));
  std::vector<int> is_ex(E + 1, 1);
  is_ex[E] = 0;
  const AbGapArgs g = gap_args(E + 1, K, 1, K, is_ex.data());
  return launch_gap(g, b.X, b.Z, b.Q, b.gpart, d_out, s);
}

extern "C" size_t lmm_ab_duality_gap_workspace_bytes(int paths) {
  return paths < 1 ? 0 : (size_t)div_up(paths, 256) * 4 * sizeof(double);
}

extern "C" int lmm_ab_duality_gap(int steps, int paths, const int* h_is_exercise,
                                  const int* d_ex, const double* d_payoffs,
                                  const double* d_means, void* d_workspace,
                                  size_t workspace_bytes, double* d_out, lmm_stream_t stream) {
  LMM_REQUIRE(steps >= 1 && steps <= kMaxSteps + 1 && paths >= 1,
              "lmm_ab_duality_gap: bad sizes");
  LMM_REQUIRE(h_is_exercise && d_ex && d_means && d_workspace && d_out,
              "lmm_ab_duality_gap: null pointer");
  LMM_REQUIRE(workspace_bytes >= lmm_ab_duality_gap_workspace_bytes(paths),
              "lmm_ab_duality_gap: workspace too small");
  const AbGapArgs g = gap_args(steps, paths, steps, 1, h_is_exercise);
  return launch_gap(g, d_ex, d_payoffs, d_means, (double*)d_workspace, d_out,
                    (cudaStream_t)stream);
}

extern "C" int lmm_device_error_flags(int clear, unsigned int* h_flags) {
  LMM_REQUIRE(h_flags, "lmm_device_error_flags: null pointer");
  unsigned int* d = nullptr;
  TRY(device_errors_ptr(&d));
  TRY(check_cuda(cudaMemcpy(h_flags, d, sizeof(unsigned int), cudaMemcpyDeviceToHost),
                 "lmm_device_error_flags: read"));
  if (clear) TRY(check_cuda(cudaMemset(d, 0, sizeof(unsigned int)), "lmm_device_error_flags"));
  return LMM_OK;
}
