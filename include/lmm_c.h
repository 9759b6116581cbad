/*
 * lmm_c.h — C ABI of the B200-native LIBOR-market-model Monte Carlo pipeline.
 *
 * Every function is extern "C", takes plain pointers and sizes (device
 * pointers are prefixed d_, host pointers h_), a cudaStream_t passed as
 * lmm_stream_t (NULL = legacy default stream), and returns an int status.
 * All device work is asynchronous on that stream; the caller synchronises.
 * The caller allocates every input, output and workspace buffer: no entry
 * point allocates device memory.  Small per-call tables (alive indices,
 * extraction indices, accruals and displacements, discounting weights,
 * bridge tables) are host arrays (prefix h_) that travel inside the kernel
 * parameters; the reference keeps them in textures.
 *
 * Layouts follow the reference (path index fastest):
 *   Sobol integers / normals     [dim][path]
 *   bridged variates             [step][factor][path]
 *   pseudo-roots A               [step][rate][factor]
 *   fixed drifts                 [step][rate]
 *   rates, log-rates, annuities,
 *   swap rates, correlated incs  [step][rate][path]
 *   discount ratios              [step][rate+1][path]
 *   numeraires, flows            [step][path]
 *   basis variables              [exercise date][variable][path]
 *
 * Each declaration names the reference routine it replaces, as
 * file:line relative to the Kooderive r256 tree; a caller keeps the
 * reference's names by forwarding each reference routine to the entry
 * point cited beside it.
 */
#ifndef LMM_C_H
#define LMM_C_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* lmm_stream_t; /* identical to cudaStream_t */

/* ---- status ---------------------------------------------------------- */
enum {
  LMM_OK = 0,
  LMM_EINVAL = 1,   /* bad argument (sizes, indices, null pointers)       */
  LMM_ECUDA = 2,    /* a CUDA runtime call or launch failed               */
  LMM_ENOMEM = 3,   /* caller-provided workspace too small                */
  LMM_ETIMEOUT = 4, /* a bounded device-side wait ran out                 */
  LMM_ENOTSUP = 5,  /* configuration outside the supported envelope       */
  LMM_ENUMERIC = 6  /* numerical failure (e.g. non-positive-definite Gram) */
};

#define LMM_MAX_RATES 128
#define LMM_MAX_STEPS 128
#define LMM_MAX_FACTORS 16
#define LMM_MAX_BASIS 16

const char* lmm_last_error_string(void);
int lmm_version(void);

/* ---- (a1) Sobol direction numbers (host) ------------------------------
 * Replaces initSobolDirectionVectors (gold/sobol_gold.cpp:118).  The
 * primitive-polynomial table is an input: degree[d], a[d] (interior
 * coefficient bits) and m[d][m_stride] initial direction integers for
 * dimensions d = 0..n_dims-1 (dimension 0 is the special all-ones case).
 * out is [n_dims][32]. */
int lmm_sobol_directions(int n_dims, const uint32_t* h_degree,
                         const uint32_t* h_a, const uint32_t* h_m,
                         int m_stride, uint32_t* h_out);

/* ---- (a2) Sobol integers ----------------------------------------------
 * Replaces sobolGPUInts (sobol_int_gpu.cu:164; header sobol_int_gpu.h).
 * Writes the Gray-code Sobol points with index path_offset+1+p
 * (p = 0..n_vectors-1; the origin is skipped) as [n_dims][n_vectors]. */
int lmm_sobol_ints(int n_vectors, int n_dims, uint32_t path_offset,
                   const uint32_t* d_directions, uint32_t* d_output,
                   lmm_stream_t stream);

/* ---- (a3) digital scramble ---------------------------------------------
 * Replaces scramble_gpu (scramble_gpu.cu:62; header scramble_gpu.h).
 * In place: data[d][p] ^= scramblers[d] for d < number_dim. */
int lmm_scramble(uint32_t* d_data, const uint32_t* d_scramblers,
                 int number_dim, int paths, lmm_stream_t stream);

/* ---- (a4) inverse cumulative normal -------------------------------------
 * Replaces the thrust::transform with inverseCumulativeShawBrickmanUnsignedInt
 * (inverseCumulatives.h:146, used at LMM_evolver_full.cu:331). */
int lmm_icdf_shaw_brickman(const uint32_t* d_in, float* d_out, size_t n,
                           lmm_stream_t stream);
/* The same rational form evaluated on the tail probability
 * t = min(i, 2^32 - i) * 2^-31 taken from the integer; no counterpart in the
 * reference, whose single-precision 1 - |2u - 1| quantises t in steps of
 * 2^-24 in both tails.  The pricing pipelines (staged and fused) use this
 * form. */
int lmm_icdf_shaw_brickman_tails(const uint32_t* d_in, float* d_out, size_t n,
                                 lmm_stream_t stream);

/* ---- (a5) Brownian bridge ------------------------------------------------
 * Replaces brownian_bridge::transform (brownian_bridge.cu:355,401-455,
 * kernel :121) with allocation bridge_allocate_diagonal
 * (gold/Bridge_allocator_gold.cpp:38).  d_in is [factors*steps][paths]
 * normals; d_out is [steps][factors][paths] increments.  h_alloc is the
 * [factors][steps] allocation matrix of Sobol dimensions, or NULL for the
 * diagonal allocation. */
int lmm_bridge_allocate_diagonal(int factors, int steps, int* h_indices);
int lmm_bridge_transform(const float* d_in, float* d_out, int paths,
                         int steps, int factors, const int* h_alloc,
                         lmm_stream_t stream);

/* Replaces brownianBridgeMultiGPUReorder (Bridge_multi_gpu.cu:119, with
 * the orderings of BrownianBridgeMultiDim, gold/Bridge_gold.h:334-404):
 * variate i of a path (d_in [factors * 2^k][paths]) moves to stage dim(i)
 * of factor fac(i), d_out [2^k][paths][factors], the layout on which a
 * one-factor bridge over paths x factors vectors runs.  ordering 0 = row,
 * 1 = column, 2 = triangular; k <= 7. */
int lmm_bridge_reorder(const float* d_in, float* d_out, int n_poweroftwo,
                       int factors, int paths, int ordering,
                       lmm_stream_t stream);

/* ---- (a6) correlation + fixed drift --------------------------------------
 * Replaces correlated_drift_paths_GPU (correlate_drift_gpu.cu:223;
 * Correlate_drift_gpu.h:12).  out[s][r][p] = sum_f A[s][r][f] z + drift[s][r]
 * for r >= alive[s].  variates_layout 0: input [step][path][factor] as the
 * reference; 1: input [step][factor][path] (bridge output). */
int lmm_correlate_drift(const float* d_in, float* d_out, const float* d_A,
                        const int* h_alive, const float* d_drift,
                        int A_offset_per_step, int factors, int out_dims,
                        int paths, int steps, int variates_layout,
                        lmm_stream_t stream);

/* ---- (a7) predictor-corrector evolution, staged ---------------------------
 * Replaces LMM_evolver_pc_gpu (LMM_evolver_gpu.cu:607-826; header
 * LMM_evolver_gpu.h:16), semantics of LMM_evolver_pc_gold
 * (gold/LMM_evolver_gold.h:315-387): spot-measure drift recomputed from
 * the rates at the start of each step, log-rates capped at cutoff.  One
 * launch per step; step s evolves and writes the rates r >= h_alive[s]
 * (non-decreasing; NULL: every rate at every step, as the gold evolver),
 * like the reference's step kernels.  Initial log-rates are log(f0 + d)
 * formed on the host in FP32, as LMMEvolutionRoutineGold does
 * (gold/LMM_evolver_full_gold.h:186-188). */
int lmm_evolve_pc_staged(const float* h_initial_rates, const float* h_taus,
                         const float* h_displacements,
                         const float* d_correlated, const float* d_A,
                         const int* h_alive, int paths, int factors, int steps,
                         int rates, float cutoff, float* d_rates,
                         float* d_log_rates, lmm_stream_t stream);

/* Replaces LMM_evolver_euler_gpu (LMM_evolver_gpu.cu:835-1180; header
 * LMM_evolver_gpu.h:32): one log-Euler step per launch, log f_r += mu_r(f
 * at the start of the step) + correlated increment (the spot drift of
 * lmm_evolve_pc_staged, no corrector), capped at cutoff (the reference's
 * Euler kernels cap at log 10); h_alive as lmm_evolve_pc_staged. */
int lmm_evolve_euler_staged(const float* h_initial_rates, const float* h_taus,
                            const float* h_displacements,
                            const float* d_correlated, const float* d_A,
                            const int* h_alive, int paths, int factors,
                            int steps, int rates, float cutoff, float* d_rates,
                            float* d_log_rates, lmm_stream_t stream);

/* ---- (a7) predictor-corrector evolution, one launch, full tensors --------
 * Replaces LMM_evolver_pc_all_gpu (LMM_evolver_all.h:23-46, kernel
 * LMM_evolver_all.cu:506-747): every path through all steps in one launch,
 * writing rates and log-rates [step][rate][path] and, when d_discounts is
 * not NULL, discount ratios [step][rate+1][path] (entry alive[s] = 1,
 * then prod 1/(1 + tau f)), for rates r >= alive[s]; entries below the
 * alive index are not written.  Input: the bridged normals (not correlated)
 * with variates_layout 1 = [step][factor][path] (the reference's transposed
 * variates) or 0 = [step][path][factor]; pseudo-roots [step][rate][factor],
 * fixed drifts [step][rate].  The drift of step 0 is formed from the
 * initial rates in the kernel like every later step's (the reference takes
 * it precomputed); log-rates are capped at cutoff.  The rate step is the
 * one of the fused pricing kernels (fast exp and reciprocal
 * approximations), so these are the pricing passes' own forward rates.
 * The reference's e-buffers and thread count are not needed. */
int lmm_evolve_pc_all(const float* h_initial_rates, const float* h_taus,
                      const float* h_displacements, const float* d_variates,
                      int variates_layout, const float* d_A,
                      const float* d_fixed_drifts, const int* h_alive, int paths,
                      int factors, int steps, int rates, float cutoff,
                      float* d_rates, float* d_log_rates, float* d_discounts,
                      lmm_stream_t stream);

/* ---- (a8) discount ratios, annuities, swap rates, numeraires ------------ */
/* discount_ratios_computation_gpu (LMM_evolver_gpu.cu:1295) */
int lmm_discount_ratios(const float* d_rates, const float* h_taus,
                        const int* h_alive, int paths, int steps, int rates,
                        float* d_discounts, lmm_stream_t stream);
/* coterminal_annuity_ratios_computation_gpu (LMM_evolver_gpu.cu:1463) */
int lmm_coterminal_annuities(const float* d_discounts, const float* h_taus,
                             const int* h_alive, int paths, int steps,
                             int rates, float* d_annuities,
                             lmm_stream_t stream);
/* coterminal_swap_rate_computation_gpu (LMM_evolver_gpu.cu:1597) */
int lmm_coterminal_swap_rates(const float* d_discounts,
                              const float* d_annuities, const int* h_alive,
                              int paths, int steps, int rates,
                              float* d_swap_rates, lmm_stream_t stream);
/* swap_rate_computation_gpu (LMM_evolver_gpu.cu, header :96) */
int lmm_swap_rate(const float* d_discounts, const float* h_taus,
                  int start_index, int end_index, int paths,
                  int step_for_offset_in, int step_for_offset_out, int steps,
                  int rates, float* d_swap_rate, lmm_stream_t stream);
/* spot_measure_numeraires_computation_offset_gpu (LMM_evolver_gpu.cu:1891) */
int lmm_spot_numeraires(const float* d_discounts, int paths,
                        int paths_for_output, int paths_offset_for_output,
                        int rates, float* d_numeraires, lmm_stream_t stream);
/* forward_rate_extraction_gpu (LMM_evolver_gpu.cu:1950): out[s][p] =
 * all[s][idx[s]][p] for s < steps */
int lmm_forward_extraction(const float* d_all, const int* h_forward_indices,
                           int paths, int steps, int rates, float* d_select,
                           lmm_stream_t stream);
/* forward_rate_extraction_selecting_step_gpu (LMM_evolver_gpu.cu:2041):
 * out[j][p] = all[step_idx[j]][fwd_idx[j]][p] for j < n */
int lmm_forward_extraction_steps(const float* d_all, const int* h_forward_indices,
                                 const int* h_step_indices, int n, int paths,
                                 int rates, float* d_select,
                                 lmm_stream_t stream);
/* spot_measure_numeraires_extraction_gpu (LMM_evolver_gpu.cu:2143) */
int lmm_numeraire_extraction(const float* d_all, float* d_some, int paths_in,
                             int paths_out, int offset_for_output, int rates,
                             int n_exercise, const int* h_exercise_indices,
                             lmm_stream_t stream);

/* ---- (a9) cash-flow generation ------------------------------------------
 * cashFlowGeneratorCallerSwap (cashFlowGeneration_product_gpu.h:190), Swap
 * product :128, gold Swap_gold (gold/cashFlowGeneration_product_gold.h:224).
 * h_aux = {strike, payReceive, accruals1[steps], accruals2[steps]}.
 * flow1[s][p] = -accrual1[s]*strike*payReceive,
 * flow2[s][p] = accrual2[s]*rate1[s][p]*payReceive. */
int lmm_cashflows_swap(float* d_flows1, float* d_flows2, const float* h_aux,
                       int paths, int steps, const float* d_rates1,
                       lmm_stream_t stream);
/* Caplet strip on the same getCashFlows contract (no reference product):
 * flow1[s][p] = accrual[s]*max(rate1[s][p]-strike,0), flow2 = 0.
 * h_aux = {strike, accruals[steps]}. */
int lmm_cashflows_caplet(float* d_flows1, float* d_flows2, const float* h_aux,
                         int paths, int steps, const float* d_rates1,
                         lmm_stream_t stream);
/* cashFlowGeneratorCallerTARN (cashFlowGeneration_product_gpu.cu:13; TARN
 * product cashFlowGeneration_product_gpu.h:19-109): target redemption
 * note.  h_aux = {total coupon, strike K, multiplier m, accruals1[steps],
 * accruals2[steps]} as the reference's aux data; flow2 = accrual2 * rate2,
 * flow1 = -max(K - m rate1, 0) accrual1 until the coupons reach the total
 * (then paid - total and the note ends; the last step pays paid - total).
 * The reference's rates3, forwards and discount arguments are unused by the
 * TARN and omitted. */
int lmm_cashflows_tarn(float* d_flows1, float* d_flows2, const float* h_aux,
                       int paths, int steps, const float* d_rates1,
                       const float* d_rates2, lmm_stream_t stream);
/* earlyExerciseBermudanPayerSwaption (exercise_values_examples.h:49-76;
 * gold early_exercise_value_generator_gold.h:93): out[e][offset+p] =
 * max((swap_rate[e][p]-strike)*annuity[e][p], 0). */
int lmm_exercise_values_payer_swaption(float strike, const float* d_swap_rates,
                                       const float* d_annuities,
                                       int batch_paths, int total_paths,
                                       int offset, int n_exercise,
                                       float* d_out, lmm_stream_t stream);

/* ---- (a10) discounting and aggregation -----------------------------------
 * cashFlowDiscounting_gpu (cashFlowDiscounting_gpu.cu:259; gold
 * gold/cashFlowDiscounting_gold.h:20-92): df = (P_{s,i1}/P_{s,s})^(1-theta)
 * (P_{s,i2}/P_{s,s})^theta, out = flow*df/numeraire[s], per-path sum. */
int lmm_cashflow_discounting(const int* h_first_index,
                             const int* h_second_index, const float* h_theta,
                             const float* d_discounts, const float* d_flows,
                             const float* d_numeraires, int paths, int steps,
                             float* d_discounted, float* d_summed,
                             lmm_stream_t stream);
/* cashFlowDiscounting_partial_gpu (cashFlowDiscounting_gpu.cu:443; gold
 * cashFlowDiscountingPartial_gold :97): discount to generation time with the
 * curve of that time, then to target time by the numeraire ratio. */
int lmm_cashflow_discounting_partial(int n_flows, const int* h_gen_indices,
                                     const int* h_first_index,
                                     const int* h_second_index,
                                     const float* h_theta,
                                     const int* h_target_indices,
                                     const float* d_discounts,
                                     const float* d_flows,
                                     const float* d_numeraires, int paths,
                                     int steps, float* d_discounted,
                                     lmm_stream_t stream);
/* generateCashFlowIndicesAndWeights (gold/cashFlowDiscounting_gold.h:210),
 * host. rate_times has n_rate_times entries; outputs have n_payments. */
int lmm_cashflow_indices_weights(const float* h_rate_times, int n_rate_times,
                                 const float* h_payment_times, int n_payments,
                                 int* h_first_index, int* h_second_index,
                                 float* h_theta);
/* AggregateFlows_gpu (cashFlowAggregation_gpu.cu:58; gold
 * gold/cashFlowAggregation_gold.h:18): agg[j][offset+p] += flows[i][p]
 * with j = preceding[i], for i >= start. */
int lmm_aggregate_flows(float* d_aggregated, int total_paths,
                        int n_exercise, const float* d_flows, int batch_paths,
                        int offset_for_output, int steps,
                        const int* h_preceding_index, int start,
                        lmm_stream_t stream);

/* ---- (a11) LS basis variables --------------------------------------------
 * adjoinBasisVariablesCaller_gpu (LS_Basis_gpu.h:168, kernel :25) with
 * basisVariableExample / basisVariableLog (LS_basis_examples_gpu.h:28,85):
 * out[e][v][offset+p] = x or log(x + shift[v]) for x = rate_v[e][p]. */
int lmm_basis_variables(int use_log, const float* h_shifts,
                        const float* d_rate1, const float* d_rate2,
                        const float* d_rate3, int batch_paths,
                        int total_paths, int offset, int n_exercise,
                        float* d_out, lmm_stream_t stream);

/* ---- (a14) reductions -----------------------------------------------------
 * PartialReduce_using8s_gpu / thrust::reduce at the price sites
 * (reductions_gpu.cu:180, kooexample/bermudanIRDPricer.cu:1470).  Sums in
 * FP64 with a deterministic order; d_partials needs
 * lmm_reduce_workspace_doubles() doubles. */
size_t lmm_reduce_workspace_doubles(void);
int lmm_reduce_sum(const float* d_in, size_t n, double* d_partials,
                   double* d_out, lmm_stream_t stream);
/* mean_p in[p] / divisor[p] (divisor may be NULL): the price estimator of
 * kooexample/bermudanIRDPricer.cu:1470-1474 and LS_main_cula.h:818. */
int lmm_reduce_mean_ratio(const float* d_in, const float* d_divisor, size_t n,
                          double* d_partials, double* d_out,
                          lmm_stream_t stream);

/* Replaces PartialReduce_using8s_gpu / PartialReduce_using16s_gpu
 * (reductions_gpu.cu:180,302): each level sums consecutive groups of
 * `group` (8 or 16) values in FP32, in the reference's pairwise order, into
 * d_workspace (at least points / (group - 1) floats), until at most
 * stop_point values (or fewer than a group) are left; a remainder smaller
 * than a group is dropped, as there.  *h_result receives the device
 * pointer of the last level (d_in itself when nothing was summed). */
int lmm_partial_reduce(const float* d_in, float* d_workspace, int points,
                       int group, int stop_point, const float** h_result,
                       lmm_stream_t stream);

/* Replaces reduceOuterProduct_gpu / reduceOuterProductSymmetric_gpu
 * (outerProduct_gpu.cu:205-700): d_answer[r][c] = sum_p in1[r][p] in2[c][p]
 * (rows, cols <= 128; inputs [rows][paths] and [cols][paths], paths a
 * multiple of 4; FP32 output) as batches of lmm_path_gram on the tensor
 * cores with an FP64 running sum.  Any workspace of at least
 * lmm_outer_product_workspace_bytes(rows, cols, 1) works; one of
 * lmm_outer_product_workspace_bytes(rows, cols, paths) does it in one
 * batch.  *d_status as lmm_path_gram's. */
size_t lmm_outer_product_workspace_bytes(int rows, int cols, int paths);
int lmm_outer_product(int paths, int rows, int cols, const float* d_in1,
                      const float* d_in2, float* d_answer, void* d_workspace,
                      size_t workspace_bytes, int* d_status,
                      lmm_stream_t stream);

/* ---- (a15) host model set-up (FP64) --------------------------------------
 * ABCDLBetaPseudoRoots (gold/volstructs_gold.cpp:311-360): per-step rank-F
 * pseudo-roots of the abcd covariance with correlation
 * L + (1-L) exp(-beta |T_i - T_j|); out is [steps][rates][factors]. */
int lmm_abcd_pseudo_roots(double a, double b, double c, double d,
                          const double* h_evolution_times, int steps,
                          const double* h_rate_starts, int rates,
                          const double* h_multipliers, int factors, double L,
                          double beta, double* h_out);
/* Vegas to the abcd parameters from dV/dA (lmm_greeks, h_abar
 * [steps][rates][factors] on the host): sum over entries of
 * h_abar * dA/d(a,b,c,d), the derivative of lmm_abcd_pseudo_roots taken by
 * central differences with relative bump rel_bump.  No counterpart in the
 * reference.  h_out[4] = dV/da, dV/db, dV/dc, dV/dd. */
int lmm_abcd_vegas(double a, double b, double c, double d,
                   const double* h_evolution_times, int steps,
                   const double* h_rate_starts, int rates,
                   const double* h_multipliers, int factors, double L,
                   double beta, const double* h_abar, double rel_bump,
                   double* h_out);
/* FlatVolPseudoRootsOfCovariances (gold/volstructs_gold.cpp:177-255);
 * h_rate_times has rates entries (the reset times T_0..T_{n-1}). */
int lmm_flat_pseudo_roots(const double* h_rate_times, int rates,
                          const double* h_evolution_times, int steps,
                          const double* h_vols, int factors, double L,
                          double beta, double* h_out);
/* fixed drifts -1/2 sum_f A[s][r][f]^2 (kooexample/bermudanIRDPricer.cu:403-417) */
int lmm_fixed_drifts(const float* h_A, int steps, int rates, int factors,
                     float* h_out);
/* spotDriftComputer::getDrifts (gold/LMM_evolver_gold.h:178-203) for one
 * step's pseudo-root h_A [rates][factors]. */
int lmm_spot_drifts(const float* h_A, const float* h_rates,
                    const float* h_taus, const float* h_disp, int rates,
                    int factors, float* h_out);
/* MT19937 words (MersenneTwisterUniformRng::nextInt32,
 * gold/Mersenne_gold.h:60) used as scrambler words in place of the
 * reference's cuRAND draws (kooexample/bermudanIRDPricer.cu:616-657). */
int lmm_mt19937_words(uint32_t seed, int n, uint32_t* h_out);

/* ---- host helpers ------------------------------------------------------
 * Bridge construction tables in double (brownian_bridge.cu:639-697) for
 * the FP64 path and for inspection. */
int lmm_bridge_tables_host(int steps, double* h_lw, double* h_rw, double* h_sd,
                           int* h_left, int* h_right, int* h_bidx);
/* findExerciseTimeIndicesFromPaymentTimeIndices
 * (gold/cashFlowDiscounting_gold.cpp, declared gold/cashFlowDiscounting_gold.h:262). */
int lmm_step_to_exercise_indices(const int* h_gen_indices, int n_gen,
                                 const int* h_exercise_indices, int n_exercise,
                                 int* h_out, int* h_first_positive);

/* ---- (a12) Longstaff–Schwartz regression on the device -------------------
 * Replaces generateMultiRegressionCoefficientsViaLS_gpu_flexisolve
 * (LS_main_cula.h:565-837) at regression depth 1, with the semantics of
 * generateRegressionCoefficientsViaLSMultiQuadratic_gold
 * (gold/MultiLS_regression.cpp:101-417): backward over exercise dates,
 * regress cf+y on the basis, exercise when the exercise value exceeds the
 * estimate, deflate by the numeraire ratio.  Basis of date e: h_nbasis[e]
 * monomials given as exponents h_monomials[e][k][v] (v < 3, exponent <= 3)
 * in the h_nvars[e] variables d_vars[e][v][p] (standardised per date when
 * normalise != 0; means/sds are then written).  d_cf and d_ex ([E][P],
 * deflated to the exercise time) may be NULL.  Outputs: d_beta[E][16]
 * (FP64), optional d_gram[E][16][17] (normalised Gram | target column),
 * d_status (bit 1: zero Gram, 2: Cholesky failed, 4: jitter used) and
 * d_price = mean_p y_p / N_0(p).  Workspace: lmm_ls_workspace_bytes(). */
size_t lmm_ls_workspace_bytes(int paths, int n_exercise);
int lmm_ls_regress(int n_exercise, int paths, const float* d_vars,
                   const int* h_nvars, const uint8_t* h_monomials,
                   const int* h_nbasis, const float* d_cf, const float* d_ex,
                   const float* d_num, int normalise, void* d_workspace,
                   size_t workspace_bytes, double* d_beta, float* d_means,
                   float* d_sds, double* d_gram, int* d_status,
                   double* d_price, lmm_stream_t stream);

/* The same regression with the paths split over GPUs (one process per GPU,
 * disjoint paths).  The reference regresses on one GPU; the split follows
 * its per-date structure (generateMultiRegressionCoefficientsViaLS_gpu,
 * LS_main_cula.h:565-837): per date every GPU forms its unscaled sums over
 * its paths, the caller sums them over the GPUs (an all-reduce on the same
 * stream), and every GPU solves the same system, so all apply one rule.
 * Sequence per regression, all on one stream with one workspace
 * (lmm_ls_workspace_bytes(paths, n_exercise)) kept between the calls:
 *   if normalising: lmm_ls_moment_sums -> all-reduce d_sums [E][6] ->
 *                   lmm_ls_moments_from_sums(total paths);
 *   for e = E-1 .. 0: lmm_ls_date_sums(e) -> all-reduce d_sums ->
 *                   lmm_ls_date_solve(e, total paths);
 *   lmm_ls_final_sum -> all-reduce -> divide by the total paths = price.
 * d_sums of a date holds (K+1)(K+2)/2 doubles (K = nbasis[e]): the sums of
 * phi_i phi_j at i (i+1)/2 + j, j <= i <= K, slot K being the target
 * cf + y.  d_status must be cleared by the caller before the first solve. */
int lmm_ls_moment_sums(int n_exercise, int paths, const float* d_vars,
                       void* d_workspace, size_t workspace_bytes,
                       double* d_sums, lmm_stream_t stream);
int lmm_ls_moments_from_sums(int n_exercise, double total_paths,
                             const double* d_sums, float* d_means,
                             float* d_sds, lmm_stream_t stream);
int lmm_ls_date_sums(int e, int n_exercise, int paths, const float* d_vars,
                     const int* h_nvars, const uint8_t* h_monomials,
                     const int* h_nbasis, const float* d_cf, const float* d_ex,
                     const float* d_num, const float* d_means,
                     const float* d_sds, const double* d_beta,
                     void* d_workspace, size_t workspace_bytes,
                     double* d_sums, lmm_stream_t stream);
int lmm_ls_date_solve(int e, int nbasis, const double* d_sums,
                      double total_paths, double* d_beta, double* d_gram,
                      int* d_status, lmm_stream_t stream);
int lmm_ls_final_sum(int n_exercise, int paths, const float* d_vars,
                     const int* h_nvars, const uint8_t* h_monomials,
                     const int* h_nbasis, const float* d_cf, const float* d_ex,
                     const float* d_num, const float* d_means,
                     const float* d_sds, const double* d_beta,
                     void* d_workspace, size_t workspace_bytes, double* d_sum,
                     lmm_stream_t stream);

/* ---- (a12) the reference's per-date LS step routines (LS_gpu.h:21-80) ----
 * For callers that drive the reference's backward loop themselves
 * (LS_main_cula.h:565-837); lmm_ls_regress fuses these per date.  FP32,
 * [row][path] layouts.
 * lmm_ls_expand_basis (expandBasisFunctions_quadratic_gpu, LS_gpu.cu:17):
 * the basis functions of exercise date `exercise` from its variables
 * d_vars[exercise][max_vars][total_paths] (the first nvars used): cross = 0
 * the quadratic set 1, x0, x0^2, x1, x1^2, ...; cross != 0 the set of
 * quadraticPolynomialCrossDevice (1, the x_i, then x0^2, x0 x1, x1^2 for
 * two variables, x_i x_{i+1 mod V} and x_i^2 for three or more); at most
 * 16 functions.  d_basis [K][total_paths].
 * lmm_ls_net_values (continuation_net_value_evaluation_gpu, LS_gpu.cu:101):
 * out[p] = shift + sum_i w_i phi_i[p] - exercise_value[p].
 * lmm_ls_update_multi (oneStepUpdateLS_multi_gpu, LS_gpu.cu:404): per path
 * walk regression depth d (coefficients d_weights[exercise][d][row_size],
 * cut-offs d_lower_cuts[d], d_upper_cuts[d]) while the net value lies
 * within the cuts and d is not the last depth; exercise when the final net
 * value is negative: then d_continuation[p] = exercise value
 * d_exercise_values[exercise][p]; d_exercises[p] = 1 / -1 and
 * d_estimates[p] = the last estimate.
 * lmm_ls_deflate (updateDeflationOfContinuationValues_gpu, LS_gpu.cu:267):
 * values[p] *= num[new_step][p] / num[old_step][p]. */
int lmm_ls_expand_basis(int total_paths, const float* d_vars, int exercise,
                        int max_vars, int nvars, int cross, float* d_basis,
                        lmm_stream_t stream);
int lmm_ls_net_values(int paths, const float* d_basis, int nbasis,
                      const float* d_weights, const float* d_exercise_values,
                      float shift, float* d_out, lmm_stream_t stream);
int lmm_ls_update_multi(int paths, int exercise, const float* d_basis,
                        int nbasis, int row_size, int depth,
                        const float* d_weights, const float* d_lower_cuts,
                        const float* d_upper_cuts, float* d_continuation,
                        const float* d_exercise_values, float shift,
                        float* d_estimates, int* d_exercises,
                        lmm_stream_t stream);
int lmm_ls_deflate(float* d_values, const float* d_numeraires, int paths,
                   int new_step, int old_step, lmm_stream_t stream);

/* ---- (f2) nested regressions with path selection ------------------------
 * Replaces generateMultiRegressionCoefficientsViaLS_gpu_flexisolve
 * (LS_main_cula.h:565-837) at regression depth > 1 with the fraction
 * selector RegressionSelectorFraction (RegressionSelectorConcrete.cu;
 * kooexample/bermudanIRDPricer.cu:1050-1080), with the semantics of
 * generateRegressionCoefficientsViaLSMultiQuadratic_gold
 * (gold/MultiLS_regression.cpp:101-417) and its selector
 * RegressionSelector_gold_Fraction (gold/Regression_Selector_concrete_gold.cpp).
 * At each date the first regression uses every path.  With n paths in the
 * last regression, the net value estimate - exercise value of each is
 * formed; a half-width c is searched (start: `sds` standard deviations of
 * the net values; grow by 1/multiplier until floor(n lower_frac) paths
 * have |net| <= c; shrink by multiplier while more than floor(n
 * upper_frac) do; then bisect to 1e-6) and, if more than min_paths paths
 * have |net| <= c, they are regressed again (moments recomputed on them
 * when normalising), up to `depth` regressions.  A date whose first net
 * values all have one sign gets no nested regression (the root tree's
 * gold/MultiLS_regression.cpp:212-225).  The exercise decision walks the
 * chain: regression d + 1 while the net value of regression d lies strictly
 * inside d's cuts. */
#define LMM_LS_MAX_DEPTH 8
typedef struct lmm_ls_select {
  int depth;            /* regressions per date, 1..LMM_LS_MAX_DEPTH        */
  double lower_frac;    /* fraction of the paths kept, lower target         */
  double upper_frac;    /* upper target (> lower_frac)                      */
  double sds;           /* initial half-width in standard deviations        */
  double multiplier;    /* shrink factor of the half-width, in (0, 1)       */
  int min_paths;        /* a nested regression needs more paths than this   */
} lmm_ls_select;

/* A frozen rule with `depth` regressions per date; row r = e*depth + d.
 * d_beta [E][depth][LMM_MAX_BASIS]; d_means / d_sds [E][depth][3] or NULL
 * (raw variables); d_cuts [E][depth][2] (lower, upper; may be NULL when
 * depth = 1); d_shifts [E] Andersen shifts added to every estimate of the
 * date (the reference's AndersenShifts_vec, kooexample/
 * bermudanIRDPricer.cu:1121-1169) or NULL. */
typedef struct lmm_ls_rule {
  int depth;
  const double* d_beta;
  const float* d_means;
  const float* d_sds;
  const double* d_cuts;
  const float* d_shifts;
} lmm_ls_rule;

/* Outputs: d_beta [E][depth][16], d_means / d_sds [E][depth][3] when
 * normalising, d_cuts [E][depth][2] (zero where no nested regression
 * followed), optional d_npaths [E][depth] (paths in each regression, 0 for
 * regressions not run), d_status (bits of lmm_ls_regress, plus 8: a
 * half-width search stopped after 512 count evaluations, where the
 * reference's search does not end, e.g. more than the upper target of net
 * values exactly zero; 16: a search needed more than its device passes) and
 * d_price = mean_p y_p / N_0(p).  Everything stays on the device: no host
 * synchronisation inside, so the call can be captured in a graph.
 * Workspace: lmm_ls_nested_workspace_bytes(). */
size_t lmm_ls_nested_workspace_bytes(int paths, int n_exercise);
int lmm_ls_regress_nested(int n_exercise, int paths, const float* d_vars,
                          const int* h_nvars, const uint8_t* h_monomials,
                          const int* h_nbasis, const float* d_cf, const float* d_ex,
                          const float* d_num, int normalise, const lmm_ls_select* select,
                          void* d_workspace, size_t workspace_bytes, double* d_beta,
                          float* d_means, float* d_sds, double* d_cuts, int* d_npaths,
                          int* d_status, double* d_price, lmm_stream_t stream);

/* Path contraction on the tensor cores: G[i][j] = scale * sum_p X[i][p]
 * Y[j][p] (i < m <= 128, j < n <= 128, p < paths), X and Y row-major with
 * leading dimensions ldx, ldy (multiples of 4, 16-byte aligned).  Split-TF32
 * tcgen05 MMAs (hi*hi + hi*lo + lo*hi), FP32 accumulation per chunk of 4096
 * paths, FP64 compensated sum of the chunks.  Replaces the reference's
 * FP32 Gram reductions reduceOuterProductSymmetric_gpu /
 * reduceOuterProduct_gpu (outerProduct_gpu.cu:205-453,459-700), which make
 * one pass over the data per matrix entry.  *d_status (cleared by the
 * caller): value 1 = a wait on the tensor cores ran out (each is bounded to
 * one second; G is then invalid), value 2 = draining the issued work after
 * that also ran out.  Workspace: lmm_path_gram_workspace_bytes(). */
size_t lmm_path_gram_workspace_bytes(int m, int n, int paths);
int lmm_path_gram(int m, int n, int paths, const float* d_X, int ldx,
                  const float* d_Y, int ldy, double scale, double* d_G,
                  void* d_workspace, size_t workspace_bytes, int* d_status,
                  lmm_stream_t stream);

/* Self-test of the bounded waits of the tensor-core kernels (no counterpart
 * in the reference): one CTA allocates tensor memory, waits up to limit_ns
 * (at most one second) on an mbarrier that nothing signals, ORs 1 into
 * *d_status when the wait runs out, frees the tensor memory and returns;
 * the context stays usable. */
int lmm_tensor_wait_selftest(unsigned long long limit_ns, int* d_status,
                             lmm_stream_t stream);

/* lmm_ls_regress for callers that cannot allocate device memory.  No
 * counterpart in the reference: it exists for callers whose device memory
 * is owned by an outside pool allocator, or whose pricing loop must not
 * allocate because allocation can synchronise the device.  The scratch is
 * a static device array of LMM_LS_STATIC_SCRATCH_BYTES (8 MiB) inside the
 * library, held by every GPU that loads it until the process exits; calls
 * needing more (lmm_ls_workspace_bytes(paths, n_exercise) above the limit,
 * about 1.9 million paths at 80 dates on a 148-SM GPU) are rejected with
 * LMM_EINVAL.  The
 * first call on a device looks up the array's device address, so make it
 * before any stream capture; the address is kept for the life of the
 * process, so the entry point must not be called after cudaDeviceReset (or
 * any other destruction of that device's primary context).  All calls share the array: calls that overlap
 * on the GPU race.  The caller still provides every input and output. */
#define LMM_LS_STATIC_SCRATCH_BYTES (8u << 20)
int lmm_ls_regress_static(int n_exercise, int paths, const float* d_vars,
                          const int* h_nvars, const uint8_t* h_monomials,
                          const int* h_nbasis, const float* d_cf,
                          const float* d_ex, const float* d_num, int normalise,
                          double* d_beta, float* d_means, float* d_sds,
                          double* d_gram, int* d_status, double* d_price,
                          lmm_stream_t stream);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* LMM_C_H */
