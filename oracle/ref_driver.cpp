// ref_driver.cpp — C entry points into the reference's own gold CPU code.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
// reference's gold/*.cpp sources, in place, into oracle/_ref/libkooref.so
// by oracle/Makefile.  It is used by the test suite and by bench.py's
// reference arm as the checker and as the CPU baseline; the product never
// links or loads it.  Every function below only marshals arrays into the
// reference routine named in its comment and returns the results.
#include <gold/sobol_gold.h>
#include <gold/sobol_primitives.h>
#include <gold/scramble_gold.h>
#include <gold/math/Normals_gold.h>
#include <gold/Bridge_allocator_gold.h>
#include <gold/correlate_drift_gold.h>
#include <gold/LMM_evolver_gold.h>
#include <gold/cashFlowGeneration_product_gold.h>
#include <gold/cashFlowDiscounting_gold.h>
#include <gold/cashFlowAggregation_gold.h>
#include <gold/LS_Basis_gold.h>
#include <gold/early_exercise_value_generator_gold.h>
#include <gold/volstructs_gold.h>
#include <gold/MultiLS_regression.h>
#include <gold/Regression_Selector_concrete_gold.h>
#include <gold/Mersenne_gold.h>
#include <gold/MatrixFacade.h>

#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#define KREF extern "C" __attribute__((visibility("default")))

template <class T>
static std::vector<T> vec(const T* p, size_t n) {
  return std::vector<T>(p, p + n);
}

// initSobolDirectionVectors (gold/sobol_gold.cpp:118)
KREF void kref_sobol_directions(int dims, unsigned* out) {
  initSobolDirectionVectors(dims, out);
}

// raw table row of the reference's primitive-polynomial list
KREF void kref_sobol_primitive(int dim, unsigned* degree, unsigned* a,
                               unsigned* m17) {
  *degree = sobol_primitives[dim].degree;
  *a = sobol_primitives[dim].a;
  for (int i = 0; i < max_m; ++i) m17[i] = sobol_primitives[dim].m[i];
}

// sobolCPUintsOffset (gold/sobol_gold.cpp:191)
KREF void kref_sobol_ints_offset(int paths, int dims, int offset,
                                 const unsigned* dirs, unsigned* out) {
  std::vector<unsigned> d(dirs, dirs + 32 * (size_t)dims);
  sobolCPUintsOffset(paths, dims, offset, d.data(), out);
}

// scramble_gold (gold/scramble_gold.cpp:11)
KREF void kref_scramble(const unsigned* in, unsigned* out, const unsigned* scr,
                        int dims, int paths) {
  std::vector<unsigned> i(in, in + (size_t)dims * paths), o(i.size());
  std::vector<unsigned> s(scr, scr + dims);
  scramble_gold(i, o, s, dims, paths);
  std::copy(o.begin(), o.end(), out);
}

// inverseCumulativeShawBrickmanUnsignedIntGold<float> (gold/math/Normals_gold.h:191)
KREF void kref_icdf_sb(const unsigned* in, float* out, long n) {
  inverseCumulativeShawBrickmanUnsignedIntGold<float> f;
  for (long i = 0; i < n; ++i) out[i] = f(in[i]);
}

// inverseCumulativeUnsignedIntGold<double> (Beasley-Springer-Moro,
// gold/math/Normals_gold.h:179)
KREF void kref_icdf_bsm_d(const unsigned* in, double* out, long n) {
  inverseCumulativeUnsignedIntGold<double> f;
  for (long i = 0; i < n; ++i) out[i] = f(in[i]);
}

// bridge_allocate_diagonal (gold/Bridge_allocator_gold.cpp:38)
KREF void kref_bridge_allocate_diagonal(int factors, int steps, int* out) {
  std::vector<int> idx(factors * steps);
  bridge_allocate_diagonal(idx, factors, steps);
  std::copy(idx.begin(), idx.end(), out);
}

// correlate_drift_paths_gold (gold/correlate_drift_gold.h:22), input [S][P][F]
KREF void kref_correlate_drift_f(const float* in, float* out, const float* A,
                                 int A_step, const float* drift, int factors,
                                 int rates, int paths, int steps) {
  std::vector<float> i(in, in + (size_t)steps * paths * factors);
  std::vector<float> o((size_t)steps * rates * paths);
  std::vector<float> a(A, A + (size_t)steps * A_step);
  std::vector<float> d(drift, drift + (size_t)steps * rates);
  correlate_drift_paths_gold<float>(i, o, a, A_step, d, factors, rates, paths,
                                    steps);
  std::copy(o.begin(), o.end(), out);
}

// LMM_evolver_pc_gold (gold/LMM_evolver_gold.h:391)
template <class D>
static void lmm_pc(const D* f0, const D* taus, const D* corr, const D* A,
                   const D* disp, int paths, int factors, int steps, int rates,
                   D cutoff, D* rates_out, D* logrates_out) {
  std::vector<D> r0(f0, f0 + rates), t(taus, taus + rates),
      c(corr, corr + (size_t)steps * rates * paths),
      a(A, A + (size_t)steps * rates * factors), d(disp, disp + rates);
  std::vector<D> ro, lo;
  LMM_evolver_pc_gold<D>(r0, t, c, a, d, paths, factors, steps, rates, ro, lo,
                         cutoff);
  std::copy(ro.begin(), ro.end(), rates_out);
  std::copy(lo.begin(), lo.end(), logrates_out);
}
KREF void kref_lmm_pc_f(const float* f0, const float* taus, const float* corr,
                        const float* A, const float* disp, int paths,
                        int factors, int steps, int rates, float cutoff,
                        float* ro, float* lo) {
  lmm_pc<float>(f0, taus, corr, A, disp, paths, factors, steps, rates, cutoff,
                ro, lo);
}
KREF void kref_lmm_pc_d(const double* f0, const double* taus,
                        const double* corr, const double* A, const double* disp,
                        int paths, int factors, int steps, int rates,
                        double cutoff, double* ro, double* lo) {
  lmm_pc<double>(f0, taus, corr, A, disp, paths, factors, steps, rates, cutoff,
                 ro, lo);
}

// discount_ratios_computation_gold (gold/LMM_evolver_gold.h:460)
KREF void kref_discount_ratios_f(const float* rates_, const float* taus,
                                 const int* alive, int paths, int steps,
                                 int rates, float* out) {
  std::vector<float> r(rates_, rates_ + (size_t)steps * rates * paths);
  std::vector<float> t(taus, taus + rates);
  std::vector<int> al(alive, alive + steps);
  std::vector<float> o((size_t)steps * (rates + 1) * paths, 0.0f);
  discount_ratios_computation_gold<float>(r, t, al, paths, steps, rates, o, 0);
  std::copy(o.begin(), o.end(), out);
}

// coterminal_annuity_ratios_computation_gold (gold/LMM_evolver_gold.h:494)
KREF void kref_annuities_f(const float* disc, const float* taus,
                           const int* alive, int paths, int steps, int rates,
                           float* out) {
  std::vector<float> d(disc, disc + (size_t)steps * (rates + 1) * paths);
  std::vector<float> t(taus, taus + rates);
  std::vector<int> al(alive, alive + steps);
  std::vector<float> o((size_t)steps * rates * paths, 0.0f);
  coterminal_annuity_ratios_computation_gold<float>(d, t, al, paths, steps,
                                                    rates, o, 0);
  std::copy(o.begin(), o.end(), out);
}

// coterminal_swap_rates_computation_gold (gold/LMM_evolver_gold.h:525)
KREF void kref_swap_rates_f(const float* disc, const float* ann,
                            const int* alive, int paths, int steps, int rates,
                            float* out) {
  std::vector<float> d(disc, disc + (size_t)steps * (rates + 1) * paths);
  std::vector<float> a(ann, ann + (size_t)steps * rates * paths);
  std::vector<int> al(alive, alive + steps);
  std::vector<float> o((size_t)steps * rates * paths, 0.0f);
  coterminal_swap_rates_computation_gold<float>(d, a, al, paths, steps, rates,
                                                o, 0);
  std::copy(o.begin(), o.end(), out);
}

// spot_measure_numeraires_computation_offset_gold (gold/LMM_evolver_gold.h:645)
KREF void kref_numeraires_f(const float* disc, int paths, int out_paths,
                            int offset, int rates, float* out) {
  std::vector<float> d(disc, disc + (size_t)rates * (rates + 1) * paths);
  std::vector<float> o((size_t)rates * out_paths, 0.0f);
  std::copy(out, out + o.size(), o.begin());
  spot_measure_numeraires_computation_offset_gold<float>(d, paths, out_paths,
                                                         offset, rates, o);
  std::copy(o.begin(), o.end(), out);
}

// cashFlowGeneratorCallerSwap_gold (gold/cashFlowGeneration_product_gold.h:249)
KREF void kref_swap_flows_f(float* f1, float* f2, const float* aux, int paths,
                            int steps, const float* rate1) {
  std::vector<float> a(aux, aux + 2 + 2 * steps), g1, g2;
  std::vector<float> r1(rate1, rate1 + (size_t)steps * paths);
  std::vector<float> dummy_fwd((size_t)steps * steps * paths, 0.0f);
  std::vector<float> dummy_disc((size_t)steps * (steps + 1) * paths, 0.0f);
  cashFlowGeneratorCallerSwap_gold<float>(g1, g2, a, paths, steps, r1, r1, r1,
                                          dummy_fwd, dummy_disc);
  std::copy(g1.begin(), g1.end(), f1);
  std::copy(g2.begin(), g2.end(), f2);
}

// cashFlowDiscounting_gold (gold/cashFlowDiscounting_gold.h:20)
KREF void kref_discounting_f(const int* first, const int* second,
                             const float* theta, const float* disc,
                             const float* flows, const float* num, int paths,
                             int steps, float* out, float* summed) {
  std::vector<int> fi(first, first + steps), si(second, second + steps);
  std::vector<float> th(theta, theta + steps);
  std::vector<float> d(disc, disc + (size_t)steps * (steps + 1) * paths);
  std::vector<float> fl(flows, flows + (size_t)steps * paths);
  std::vector<float> nu(num, num + (size_t)steps * paths);
  std::vector<float> o, s;
  cashFlowDiscounting_gold<float>(fi, si, th, d, fl, nu, paths, steps, o, s);
  std::copy(o.begin(), o.end(), out);
  std::copy(s.begin(), s.end(), summed);
}

// cashFlowDiscountingPartial_gold (gold/cashFlowDiscounting_gold.h:97)
KREF void kref_discounting_partial_f(int n_flows, const int* gen,
                                     const int* first, const int* second,
                                     const float* theta, const int* target,
                                     const float* disc, const float* flows,
                                     const float* num, int paths, int steps,
                                     float* out) {
  std::vector<int> g(gen, gen + n_flows), fi(first, first + n_flows),
      si(second, second + n_flows), tg(target, target + n_flows);
  std::vector<float> th(theta, theta + n_flows);
  CubeConstFacade<float> dc(disc, steps, steps + 1, paths);
  MatrixConstFacade<float> fl(flows, steps, paths);
  MatrixConstFacade<float> nu(num, steps, paths);
  MatrixFacade<float> o(out, n_flows, paths);
  cashFlowDiscountingPartial_gold<float>(g, fi, si, th, tg, dc, fl, nu, paths,
                                         steps, o);
}

// generateCashFlowIndicesAndWeights (gold/cashFlowDiscounting_gold.h:210)
KREF void kref_indices_weights_f(const float* rate_times, int n_rate_times,
                                 const float* pay, int n_pay, int* first,
                                 int* second, float* theta) {
  std::vector<int> fi, si;
  std::vector<float> th;
  std::vector<float> rt(rate_times, rate_times + n_rate_times);
  std::vector<float> pt(pay, pay + n_pay);
  generateCashFlowIndicesAndWeights<float>(fi, si, th, rt, pt);
  std::copy(fi.begin(), fi.end(), first);
  std::copy(si.begin(), si.end(), second);
  std::copy(th.begin(), th.end(), theta);
}

// findExerciseTimeIndicesFromPaymentTimeIndices (gold/cashFlowDiscounting_gold.cpp)
KREF int kref_step_to_exercise(const int* gen, int n_gen, const int* ex,
                               int n_ex, int* out) {
  std::vector<int> g(gen, gen + n_gen), e(ex, ex + n_ex), ind(n_gen, 0), o;
  for (int i = 0; i < n_gen; ++i)
    ind[i] = std::find(e.begin(), e.end(), g[i]) != e.end();
  int first = findExerciseTimeIndicesFromPaymentTimeIndices(g, e, ind, o);
  std::copy(o.begin(), o.end(), out);
  return first;
}

// AggregateFlows_gold (gold/cashFlowAggregation_gold.h:18)
KREF void kref_aggregate_f(float* agg, int total, int n_ex, const float* flows,
                           int batch, int offset, int steps,
                           const int* preceding) {
  MatrixFacade<float> a(agg, n_ex, total);
  MatrixConstFacade<float> f(flows, steps, batch);
  std::vector<int> pr(preceding, preceding + steps);
  AggregateFlows_gold<float>(a, f, pr, batch, offset);
}

// adjoinBasisVariablesCaller_gold (gold/LS_Basis_gold.h:79)
KREF void kref_basis_variables_f(int use_log, const float* shifts,
                                 const float* r1, const float* r2,
                                 const float* r3, int batch, int total,
                                 int offset, int rates, int n_ex,
                                 const int* ex_idx, float* out) {
  std::vector<int> idata(1, 0);
  std::vector<float> fdata(shifts, shifts + 3);
  std::vector<int> ei(ex_idx, ex_idx + n_ex), ind(rates, 0);
  for (int j = 0; j < n_ex; ++j) ind[ei[j]] = 1;
  std::vector<float> dummy(1, 0.0f);
  CubeConstFacade<float> fw(dummy.data(), 1, 1, 1), dr(dummy.data(), 1, 1, 1);
  MatrixConstFacade<float> m1(r1, n_ex, batch), m2(r2, n_ex, batch),
      m3(r3, n_ex, batch);
  CubeFacade<float> o(out, n_ex, 3, total);
  adjoinBasisVariablesCaller_gold<float>(use_log != 0, idata, fdata, fw, dr, m1,
                                         m2, m3, batch, total, offset, rates,
                                         ei, ind, o, 0);
}

// adjoinExerciseValues_Bermudan_swaption_gold
// (gold/early_exercise_value_generator_gold.h:139)
KREF void kref_payer_swaption_values_f(float strike, const float* sr,
                                       const float* ann, int batch, int total,
                                       int offset, int rates, int n_ex,
                                       const int* ex_idx, float* out) {
  std::vector<float> fl(1, strike);
  std::vector<int> il(1, 0);
  std::vector<int> ei(ex_idx, ex_idx + n_ex), ind(rates, 0);
  std::vector<float> dummy(1, 0.0f);
  CubeConstFacade<float> fw(dummy.data(), 1, 1, 1), dr(dummy.data(), 1, 1, 1);
  MatrixConstFacade<float> m1(sr, n_ex, batch), m2(ann, n_ex, batch),
      m3(ann, n_ex, batch);
  MatrixFacade<float> o(out, n_ex, total);
  adjoinExerciseValues_Bermudan_swaption_gold<float>(
      fl, il, rates, fw, dr, m1, m2, m3, batch, offset, ei, ind, o);
}

// ABCDLBetaPseudoRoots (gold/volstructs_gold.cpp:311): out [S][n][F]
KREF void kref_abcd_pseudo_roots(double a, double b, double c, double d,
                                 const double* evol_times, int steps,
                                 const double* rate_starts, int rates,
                                 const double* multipliers, int factors,
                                 double L, double beta, double* out) {
  std::vector<double> et(evol_times, evol_times + steps);
  std::vector<double> rs(rate_starts, rate_starts + rates);
  std::vector<double> mu(multipliers, multipliers + rates);
  Cube_gold<double> r =
      ABCDLBetaPseudoRoots(a, b, c, d, et, rs, mu, factors, L, beta);
  std::copy(r.getDataVector().begin(), r.getDataVector().end(), out);
}

// FlatVolPseudoRootsOfCovariances (gold/volstructs_gold.cpp:236)
KREF void kref_flat_pseudo_roots(const double* rate_times, int n_rate_times,
                                 const double* evol_times, int steps,
                                 const double* vols, int factors, double L,
                                 double beta, double* out) {
  std::vector<double> rt(rate_times, rate_times + n_rate_times);
  std::vector<double> et(evol_times, evol_times + steps);
  std::vector<double> v(vols, vols + n_rate_times - 1);
  Cube_gold<double> r =
      FlatVolPseudoRootsOfCovariances(rt, et, v, factors, L, beta);
  std::copy(r.getDataVector().begin(), r.getDataVector().end(), out);
}

// MersenneTwisterUniformRng::nextInt32 (gold/Mersenne_gold.h:60)
KREF void kref_mt19937(unsigned long seed, int n, unsigned* out) {
  MersenneTwisterUniformRng rng(seed);
  for (int i = 0; i < n; ++i) out[i] = (unsigned)rng.nextInt32();
}

// generateRegressionCoefficientsViaLSMultiQuadratic_gold
// (gold/MultiLS_regression.cpp:523) at regression depth 1.
// vars [E][3][P] (double), cf/ex/num [E][P]; coefficients [E][ncoef].
KREF double kref_ls_multi(int n_ex, int paths, const double* vars,
                          const int* nvars, const double* cf, const double* ex,
                          const double* num, int use_cross, int normalise,
                          double* coeffs, int ncoef, double* means,
                          double* sds) {
  const int maxVars = 3;
  const int depth = 1;
  std::vector<double> products, targets;
  std::vector<double> coef((size_t)n_ex * depth * ncoef, 0.0);
  CubeFacade<double> coef_c(coef, n_ex, depth, ncoef);
  std::vector<double> lc(n_ex * depth, 0.0), uc(n_ex * depth, 0.0);
  MatrixFacade<double> lc_m(lc, n_ex, depth), uc_m(uc, n_ex, depth);
  std::vector<double> mv((size_t)n_ex * depth * maxVars, 0.0),
      sv((size_t)n_ex * depth * maxVars, 1.0);
  CubeFacade<double> mv_c(mv, n_ex, depth, maxVars),
      sv_c(sv, n_ex, depth, maxVars);
  CubeConstFacade<double> vars_c(vars, n_ex, maxVars, paths);
  std::vector<int> nv(nvars, nvars + n_ex);
  MatrixConstFacade<double> cf_m(cf, n_ex, paths), ex_m(ex, n_ex, paths);
  std::vector<double> num_v(num, num + (size_t)n_ex * paths);
  MatrixFacade<double> num_m(num_v, n_ex, paths);
  RegressionSelector_gold_Fraction selector(0.1, 0.2, 2.5, 0.8);
  double price = generateRegressionCoefficientsViaLSMultiQuadratic_gold(
      n_ex, products, targets, coef_c, lc_m, uc_m, mv_c, sv_c, normalise != 0,
      vars_c, nv, maxVars, cf_m, ex_m, num_m, paths, depth - 1, 0, selector,
      use_cross != 0);
  std::copy(coef.begin(), coef.end(), coeffs);
  std::copy(mv.begin(), mv.end(), means);
  std::copy(sv.begin(), sv.end(), sds);
  return price;
}
