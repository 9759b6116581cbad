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
#include <gold/Bridge_gold.h>
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

// BrownianBridge<float>::GenerateBridge (gold/Bridge_gold.h:168-327), the
// power-of-two bridge with differencing, per path: in and out
// [2^k][paths] (the layout of brownianBridgeGPU_constant_memory).
KREF void kref_bridge_pow2_f(int k, int paths, const float* in, float* out) {
  BrownianBridge<float> bb(k);
  const int n = bb.dimensions();
  std::vector<float> v(n), w(n);
  for (int p = 0; p < paths; ++p) {
    for (int i = 0; i < n; ++i) v[i] = in[(size_t)i * paths + p];
    bb.GenerateBridge(v.data(), w.data());
    for (int i = 0; i < n; ++i) out[(size_t)i * paths + p] = w[i];
  }
}

// BrownianBridgeMultiDim<float> (gold/Bridge_gold.h:334-404): the
// reordering (dimension and factor of each variate) and GenerateBridge per
// path, in [factors * 2^k][paths], out [factors][2^k][paths].
KREF void kref_bridge_multi_f(int k, int factors, int ordering, int paths, const float* in,
                              float* out, int* dims, int* facs) {
  typedef BrownianBridgeMultiDim<float> BB;
  const BB::ordering ord = ordering == 0 ? BB::row : ordering == 1 ? BB::column : BB::triangular;
  BB bb(k, factors, ord);
  const int N = factors * (1 << k);
  for (int i = 0; i < N; ++i) {
    dims[i] = bb.reorderingDimension()[i];
    facs[i] = bb.reorderingFactor()[i];
  }
  std::vector<float> v(N), w(N);
  for (int p = 0; p < paths; ++p) {
    for (int i = 0; i < N; ++i) v[i] = in[(size_t)i * paths + p];
    bb.GenerateBridge(v.data(), w.data());
    for (int i = 0; i < N; ++i) out[(size_t)i * paths + p] = w[i];
  }
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

// cashFlowGeneratorCallerTARN_gold (gold/cashFlowGeneration_product_gold.h:171)
KREF void kref_tarn_flows_f(float* f1, float* f2, const float* aux, int paths,
                            int steps, const float* rate1) {
  std::vector<float> a(aux, aux + 3 + 2 * steps), g1, g2;
  std::vector<float> r1(rate1, rate1 + (size_t)steps * paths);
  std::vector<float> dummy_fwd((size_t)steps * steps * paths, 0.0f);
  std::vector<float> dummy_disc((size_t)steps * (steps + 1) * paths, 0.0f);
  cashFlowGeneratorCallerTARN_gold<float>(g1, g2, a, paths, steps, r1, r1, r1,
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

// generateRegressionCoefficientsViaLSMultiQuadratic_gold
// (gold/MultiLS_regression.cpp:523) at regression depth `depth` with the
// fraction selector RegressionSelector_gold_Fraction(lower_frac, upper_frac,
// sds, multiplier) (gold/Regression_Selector_concrete_gold.cpp) and at least
// `min_paths` paths per nested regression.  Outputs coefficients
// [E][depth][ncoef], means / sds [E][depth][3], cuts [E][depth].
KREF double kref_ls_multi_depth(int n_ex, int paths, const double* vars, const int* nvars,
                                const double* cf, const double* ex, const double* num,
                                int use_cross, int normalise, int depth, double lower_frac,
                                double upper_frac, double sds_cut, double multiplier,
                                int min_paths, double* coeffs, int ncoef, double* means,
                                double* sds, double* lower_cuts, double* upper_cuts) {
  const int maxVars = 3;
  std::vector<double> products, targets;
  std::vector<double> coef((size_t)n_ex * depth * ncoef, 0.0);
  CubeFacade<double> coef_c(coef, n_ex, depth, ncoef);
  std::vector<double> lc(n_ex * depth, 0.0), uc(n_ex * depth, 0.0);
  MatrixFacade<double> lc_m(lc, n_ex, depth), uc_m(uc, n_ex, depth);
  std::vector<double> mv((size_t)n_ex * depth * maxVars, 0.0),
      sv((size_t)n_ex * depth * maxVars, 1.0);
  CubeFacade<double> mv_c(mv, n_ex, depth, maxVars), sv_c(sv, n_ex, depth, maxVars);
  CubeConstFacade<double> vars_c(vars, n_ex, maxVars, paths);
  std::vector<int> nv(nvars, nvars + n_ex);
  MatrixConstFacade<double> cf_m(cf, n_ex, paths), ex_m(ex, n_ex, paths);
  std::vector<double> num_v(num, num + (size_t)n_ex * paths);
  MatrixFacade<double> num_m(num_v, n_ex, paths);
  RegressionSelector_gold_Fraction selector(lower_frac, upper_frac, sds_cut, multiplier);
  const double price = generateRegressionCoefficientsViaLSMultiQuadratic_gold(
      n_ex, products, targets, coef_c, lc_m, uc_m, mv_c, sv_c, normalise != 0, vars_c, nv,
      maxVars, cf_m, ex_m, num_m, paths, depth - 1, min_paths, selector, use_cross != 0);
  std::copy(coef.begin(), coef.end(), coeffs);
  std::copy(mv.begin(), mv.end(), means);
  std::copy(sv.begin(), sv.end(), sds);
  std::copy(lc.begin(), lc.end(), lower_cuts);
  std::copy(uc.begin(), uc.end(), upper_cuts);
  return price;
}

// SecondPassPriceLSAMultiUsingAggregatedFlows_gold with the frozen
// MultiLSExerciseStrategy (gold/MultiLS_regression.h:137-289): the rule of
// kref_ls_multi_depth plus per-date Andersen shifts, applied to the paths'
// basis variables, flows, exercise values and numeraires.
KREF double kref_ls_multi_second_pass(int n_ex, int paths, const double* vars,
                                      const int* nvars, const double* cf, const double* ex,
                                      const double* num, int use_cross, int depth,
                                      const double* coeffs, int ncoef, const double* means,
                                      const double* sds, const double* lower_cuts,
                                      const double* upper_cuts, const double* shifts) {
  const int maxVars = 3;
  std::vector<int> nv(nvars, nvars + n_ex);
  std::vector<double> andersen(shifts, shifts + n_ex);
  CubeConstFacade<double> coef_cc(coeffs, n_ex, depth, ncoef);
  MatrixConstFacade<double> lc_cm(lower_cuts, n_ex, depth), uc_cm(upper_cuts, n_ex, depth);
  CubeConstFacade<double> mv_cc(means, n_ex, depth, maxVars), sv_cc(sds, n_ex, depth, maxVars);
  CubeConstFacade<double> v_c(vars, n_ex, maxVars, paths);
  MatrixConstFacade<double> cf_m(cf, n_ex, paths), ex_m(ex, n_ex, paths);
  std::vector<double> num_v(num, num + (size_t)n_ex * paths);
  MatrixFacade<double> num_m(num_v, n_ex, paths);
  if (use_cross) {
    MultiLSExerciseStrategy<quadraticPolynomialCrossGenerator> strategy(
        coef_cc, lc_cm, uc_cm, mv_cc, sv_cc, depth, andersen, nv, n_ex);
    return SecondPassPriceLSAMultiUsingAggregatedFlows_gold(n_ex, v_c, maxVars, cf_m, ex_m,
                                                            num_m, paths, strategy);
  }
  MultiLSExerciseStrategy<quadraticPolynomialGenerator> strategy(
      coef_cc, lc_cm, uc_cm, mv_cc, sv_cc, depth, andersen, nv, n_ex);
  return SecondPassPriceLSAMultiUsingAggregatedFlows_gold(n_ex, v_c, maxVars, cf_m, ex_m, num_m,
                                                          paths, strategy);
}

// ABDualityGapEstimateZeroRebate (gold/Andersen_Broadie_gold.cpp:59-119; the
// buildable copy has no non-zero-rebate form): ex [steps][paths] (0/1),
// means / sds [paths][steps] (inner-simulation continuation estimates),
// is_ex [steps].  out = {mean, se}.
#include <gold/Andersen_Broadie_gold.h>
KREF void kref_ab_gap_zero_rebate(int steps, int paths, const int* ex, const double* means,
                                  const double* sds, const int* is_ex, double* out) {
  MatrixConstFacade<int> ex_m(ex, steps, paths);
  MatrixConstFacade<double> means_m(means, paths, steps), sds_m(sds, paths, steps);
  std::vector<bool> isx(is_ex, is_ex + steps);
  double mean = 0, se = 0;
  ABDualityGapEstimateZeroRebate(ex_m, means_m, sds_m, mean, se, isx);
  out[0] = mean;
  out[1] = se;
}

// ---------------------------------------------------------------------------
// Whole Bermudan payer swaption through the reference's gold routines, in the
// stage order of gold/gold_example/LMM_bermudan_gold.cpp:372-948:
//   LMMEvolutionRoutineGold (gold/LMM_evolver_full_gold.h:140) ->
//   discount_ratios / coterminal annuities / swap rates / spot numeraires
//   (gold/LMM_evolver_gold.h:460-666) -> extraction at the exercise steps ->
//   adjoinBasisVariablesCaller_gold + Bermudan swaption exercise values ->
//   generateRegressionCoefficientsViaLSMultiQuadratic_gold (depth 1) ->
//   second pass SecondPassPriceLSAMultiUsingAggregatedFlows_gold with the
//   frozen MultiLSExerciseStrategy (gold/MultiLS_regression.h:137-289).
// Exercise at every reset; basis variables: first forward, coterminal swap
// rate, coterminal annuity.  Paths are split into chunks of `chunk` paths
// with disjoint Sobol offsets and the chunks are spread over `threads`
// std::threads (the gold code itself is single-threaded).  The regression
// runs on one thread over all regression paths, as in the reference.
// Returns the time-0 price; *insample receives the first-pass estimate.
#include <gold/LMM_evolver_full_gold.h>
#include <atomic>
#include <chrono>

namespace {
// At regression depth 1 the selector's cut-offs are never read
// (updateDeflatedNextStepValuesMulti_gold stops at depth 0), but
// RegressionSelector_gold_Fraction's search does not terminate when many
// net continuation values are exactly zero (its shrink loop,
// gold/Regression_Selector_concrete_gold.cpp, never gets the count below
// the target).  This selector keeps every path and returns wide cut-offs.
class SelectAll : public RegressionSelectorGold {
 public:
  template <class It, class S>
  static int all(It start, It end, std::vector<int>::iterator sel,
                 std::vector<int>::const_iterator pre, S& lo, S& hi) {
    int count = 0;
    for (It it = start; it != end; ++it, ++sel, ++pre) {
      *sel = *pre;
      count += *pre ? 1 : 0;
    }
    lo = S(-1e4);
    hi = S(1e4);
    return count;
  }
  int SelectF(int, std::vector<float>::const_iterator s,
              std::vector<float>::const_iterator e, std::vector<int>::iterator sel,
              std::vector<int>::const_iterator pre, int, float& lo, float& hi) {
    return all(s, e, sel, pre, lo, hi);
  }
  int Select(int, std::vector<double>::const_iterator s,
             std::vector<double>::const_iterator e, std::vector<int>::iterator sel,
             std::vector<int>::const_iterator pre, int, double& lo, double& hi) {
    return all(s, e, sel, pre, lo, hi);
  }
};

struct KrefModel {
  int n, F;
  std::vector<float> A, fixed, taus, disp, f0, logf0;
  std::vector<unsigned> scr;
  int pow2;
  float strike;
};

// LS inputs of paths [offset, offset+P) into columns [col, col+P) of cubes
// with `total` columns.
void kref_inputs(const KrefModel& m, int P, int offset, int total, int col,
                 std::vector<double>& vars, std::vector<double>& ex,
                 std::vector<double>& num) {
  const int n = m.n, S = m.n;
  std::vector<float> rates, lrates;
  LMMEvolutionRoutineGold<float>(P, offset, n, m.F, S, m.pow2, m.scr, m.A,
                                 m.fixed, m.disp, m.f0, m.logf0, m.taus, rates,
                                 lrates);
  std::vector<int> alive(S);
  for (int s = 0; s < S; ++s) alive[s] = s;
  std::vector<float> disc((size_t)S * (n + 1) * P, 0.0f),
      ann((size_t)S * n * P, 0.0f), sr((size_t)S * n * P, 0.0f),
      nums((size_t)n * P, 0.0f);
  discount_ratios_computation_gold<float>(rates, m.taus, alive, P, S, n, disc, 0);
  coterminal_annuity_ratios_computation_gold<float>(disc, m.taus, alive, P, S, n, ann, 0);
  coterminal_swap_rates_computation_gold<float>(disc, ann, alive, P, S, n, sr, 0);
  spot_measure_numeraires_computation_gold<float>(disc, P, n, nums, 0);
  std::vector<int> ex_idx(S);
  for (int s = 0; s < S; ++s) ex_idx[s] = s;
  const int E = S;
  std::vector<float> r1((size_t)E * P), r2((size_t)E * P), r3((size_t)E * P);
  forward_rate_extraction_selecting_steps_gold<float>(rates, ex_idx, ex_idx, P, n, S, r1, 0);
  forward_rate_extraction_selecting_steps_gold<float>(sr, ex_idx, ex_idx, P, n, S, r2, 0);
  forward_rate_extraction_selecting_steps_gold<float>(ann, ex_idx, ex_idx, P, n, S, r3, 0);
  std::vector<float> bv((size_t)E * 3 * P), exv((size_t)E * P), some;
  {
    std::vector<int> idata(1, 0), ind(n, 1);
    std::vector<float> fdata(3, 0.0f);
    std::vector<float> dummy(1, 0.0f);
    CubeConstFacade<float> fw(dummy.data(), 1, 1, 1), dr(dummy.data(), 1, 1, 1);
    MatrixConstFacade<float> m1(r1.data(), E, P), m2(r2.data(), E, P), m3(r3.data(), E, P);
    CubeFacade<float> o(bv.data(), E, 3, P);
    adjoinBasisVariablesCaller_gold<float>(false, idata, fdata, fw, dr, m1, m2, m3, P, P, 0,
                                           n, ex_idx, ind, o, 0);
    std::vector<float> fl(1, m.strike);
    MatrixFacade<float> eo(exv.data(), E, P);
    adjoinExerciseValues_Bermudan_swaption_gold<float>(fl, idata, n, fw, dr, m2, m3, m3, P, 0,
                                                       ex_idx, ind, eo);
  }
  // spot_measure_numeraires_extraction_gold takes its matrix view of the
  // output before resizing it (gold/LMM_evolver_gold.h:696-701): size first.
  some.assign((size_t)E * P, 0.0f);
  spot_measure_numeraires_extraction_gold<float>(nums, P, n, E, ex_idx, some);
  for (int e = 0; e < E; ++e)
    for (int p = 0; p < P; ++p) {
      for (int v = 0; v < 3; ++v)
        vars[((size_t)e * 3 + v) * total + col + p] = bv[((size_t)e * 3 + v) * P + p];
      ex[(size_t)e * total + col + p] = exv[(size_t)e * P + p];
      num[(size_t)e * total + col + p] = some[(size_t)e * P + p];
    }
}

template <class Fn>
void kref_parallel(int P, int chunk, int threads, Fn fn) {
  std::atomic<int> next{0};
  auto worker = [&]() {
    for (;;) {
      const int c = next.fetch_add(1);
      const int lo = c * chunk;
      if (lo >= P) break;
      fn(lo, std::min(chunk, P - lo));
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < std::max(1, threads); ++t) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
}
}  // namespace

KREF double kref_bermudan_swaption(int n, int F, const float* taus,
                                   const float* disp, const float* f0,
                                   const float* A, const float* fixed,
                                   const unsigned* scramblers, float strike,
                                   int reg_paths, int price_paths,
                                   int reg_offset, int price_offset,
                                   int threads, int chunk, int normalise,
                                   double* insample, double* seconds) {
  auto t0 = std::chrono::steady_clock::now();
  KrefModel m;
  m.n = n;
  m.F = F;
  m.A.assign(A, A + (size_t)n * n * F);
  m.fixed.assign(fixed, fixed + (size_t)n * n);
  m.taus.assign(taus, taus + n);
  m.disp.assign(disp, disp + n);
  m.f0.assign(f0, f0 + n);
  m.logf0.resize(n);
  for (int r = 0; r < n; ++r) m.logf0[r] = std::log(f0[r] + disp[r]);
  m.pow2 = 0;
  while ((1 << m.pow2) < n) ++m.pow2;
  m.scr.assign(scramblers, scramblers + (size_t)(1 << m.pow2) * F);
  m.strike = strike;
  const int E = n;
  std::vector<int> nvars(E);
  for (int e = 0; e < E; ++e)
    nvars[e] = basisVariableExample_gold<float>::actualNumberOfVariables(e, e, n);

  // first pass
  std::vector<double> vars((size_t)E * 3 * reg_paths), ex((size_t)E * reg_paths),
      num((size_t)E * reg_paths), cf((size_t)E * reg_paths, 0.0);
  kref_parallel(reg_paths, chunk, threads, [&](int lo, int cnt) {
    kref_inputs(m, cnt, reg_offset + lo, reg_paths, lo, vars, ex, num);
  });
  const int ncoef = 10, depth = 1, maxVars = 3;
  std::vector<double> products, targets, coef((size_t)E * depth * ncoef, 0.0);
  CubeFacade<double> coef_c(coef, E, depth, ncoef);
  std::vector<double> lc(E * depth, 0.0), uc(E * depth, 0.0);
  MatrixFacade<double> lc_m(lc, E, depth), uc_m(uc, E, depth);
  std::vector<double> mv((size_t)E * depth * maxVars, 0.0), sv((size_t)E * depth * maxVars, 1.0);
  CubeFacade<double> mv_c(mv, E, depth, maxVars), sv_c(sv, E, depth, maxVars);
  CubeConstFacade<double> vars_c(vars.data(), E, maxVars, reg_paths);
  MatrixConstFacade<double> cf_m(cf.data(), E, reg_paths), ex_m(ex.data(), E, reg_paths);
  MatrixFacade<double> num_m(num, E, reg_paths);
  SelectAll selector;
  const double ins = generateRegressionCoefficientsViaLSMultiQuadratic_gold(
      E, products, targets, coef_c, lc_m, uc_m, mv_c, sv_c, normalise != 0, vars_c, nvars,
      maxVars, cf_m, ex_m, num_m, reg_paths, depth - 1, 0, selector, true);
  if (insample) *insample = ins;

  // second pass with the frozen rule
  std::vector<double> pvars((size_t)E * 3 * price_paths), pex((size_t)E * price_paths),
      pnum((size_t)E * price_paths), pcf((size_t)E * price_paths, 0.0);
  kref_parallel(price_paths, chunk, threads, [&](int lo, int cnt) {
    kref_inputs(m, cnt, price_offset + lo, price_paths, lo, pvars, pex, pnum);
  });
  std::vector<double> andersen(E, 0.0);
  CubeConstFacade<double> coef_cc(coef.data(), E, depth, ncoef);
  MatrixConstFacade<double> lc_cm(lc.data(), E, depth), uc_cm(uc.data(), E, depth);
  CubeConstFacade<double> mv_cc(mv.data(), E, depth, maxVars), sv_cc(sv.data(), E, depth, maxVars);
  MultiLSExerciseStrategy<quadraticPolynomialCrossGenerator> strategy(
      coef_cc, lc_cm, uc_cm, mv_cc, sv_cc, depth, andersen, nvars, E);
  CubeConstFacade<double> pv_c(pvars.data(), E, maxVars, price_paths);
  MatrixConstFacade<double> pcf_m(pcf.data(), E, price_paths), pex_m(pex.data(), E, price_paths);
  MatrixFacade<double> pnum_m(pnum, E, price_paths);
  const double price = SecondPassPriceLSAMultiUsingAggregatedFlows_gold(
      E, pv_c, maxVars, pcf_m, pex_m, pnum_m, price_paths, strategy);
  if (seconds)
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return price;
}
