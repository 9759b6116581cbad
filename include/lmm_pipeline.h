/*
 * lmm_pipeline.h — whole-pipeline entry points: the C++ host driver that
 * strings the stage kernels of lmm_c.h together (plain FP32 staged form) or
 * runs the fused per-path kernels, for one batch of paths on one stream.
 *
 * Replaces the reference's drivers LMMEvolutionRoutineRawSingleKernel
 * (LMM_evolver_full.cu:264-423) and the first/second pass loops of
 * BermudanMultiLSPricerExample (kooexample/bermudanIRDPricer.cu:650-1480),
 * with the products of the benchmark configurations.  All buffers are
 * caller-allocated; lmm_pipeline_workspace_bytes() sizes the scratch.
 */
#ifndef LMM_PIPELINE_H
#define LMM_PIPELINE_H

#include "lmm_c.h"

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
  LMM_PRODUCT_SWAPTION = 0,         /* Bermudan payer swaption: exercise value
                                       max((SR_s-K) A_s, 0), no coupons      */
  LMM_PRODUCT_CANCELLABLE_SWAP = 1, /* payer swap tau (f_s - K) pr paid at
                                       T_{s+1}, cancellable (value 0) at the
                                       exercise dates: the reference example */
  LMM_PRODUCT_EUROPEAN = 2,         /* caplet strip (cap_strike) plus payer
                                       swap (strike) on every period         */
  LMM_PRODUCT_TARN = 3,             /* target redemption note (the reference's
                                       TARN, cashFlowGeneration_product_gpu.h:
                                       19-109): floating leg tau f received,
                                       inverse-floater coupon
                                       max(strike - m f, 0) tau paid until the
                                       coupons reach tarn_total, then the
                                       remainder and stop; last period pays
                                       the remainder; flows at T_{s+1}       */
  LMM_PRODUCT_BERMUDAN_CAP = 4      /* portfolio of the Bermudan payer
                                       swaption (exercise value and rule as
                                       LMM_PRODUCT_SWAPTION) and a cap strip
                                       (caplet tau max(f_s - cap_strike, 0)
                                       paid at T_{s+1} on every period,
                                       whether or not the swaption has been
                                       exercised); no reference product: the
                                       portfolio of the differentiation
                                       form.  The regression (first pass) is
                                       the swaption's alone.  Not available
                                       in LMM_MODE_TENSOR nor to
                                       lmm_andersen_broadie.                 */
};

/* STAGED: the reference's chain stage by stage (plain FP32).  FUSED: one
 * variates kernel and one evolution kernel, CUDA cores.  TENSOR: as FUSED
 * with the per-step drift and correlation contractions on the tensor cores
 * (tcgen05, split FP16, accumulators in tensor memory; at most 16
 * factors). */
enum { LMM_MODE_STAGED = 0, LMM_MODE_FUSED = 1, LMM_MODE_TENSOR = 2 };

/* Model: n rates with one evolution step per reset (steps == rates, step s
 * ends at T_s, rate s resets there; alive index of step s is s). */
typedef struct lmm_model {
  int rates;
  int factors;
  const float* h_taus;            /* [rates] accruals tau_r               */
  const float* h_displacements;   /* [rates]                              */
  const float* h_initial_rates;   /* [rates]                              */
  const float* d_A;               /* [rates][rates][factors] pseudo-roots  */
  const float* d_fixed_drifts;    /* [rates][rates]: -1/2 |A_s[r]|^2      */
  const uint32_t* d_directions;   /* [rates*factors][32] Sobol directions */
  const uint32_t* d_scramblers;   /* [scramble_dims] XOR words, or NULL   */
  int scramble_dims;              /* leading Sobol dims scrambled         */
  float cutoff;                   /* log-rate cap (gold uses 10)          */
} lmm_model;

/* Product and exercise strategy description. */
typedef struct lmm_product {
  int kind;                       /* LMM_PRODUCT_*                        */
  float strike;
  float cap_strike;
  float pay_receive;
  int n_exercise;                 /* exercise dates                       */
  const int* h_exercise_steps;    /* [n_exercise] increasing steps        */
  const int* h_nvars;             /* [n_exercise] basis variables in use  */
  const uint8_t* h_monomials;     /* [n_exercise][16][3] exponents        */
  const int* h_nbasis;            /* [n_exercise] basis functions         */
  int normalise;                  /* standardise basis variables per date */
  float tarn_total;               /* TARN: total coupon (target)          */
  float tarn_multiplier;          /* TARN: rate multiplier m              */
} lmm_product;

/* Bytes of scratch for one call of the given mode on `paths` paths.  The
 * staged mode holds full [step][rate][path] tensors, so callers batch. */
size_t lmm_pipeline_workspace_bytes(const lmm_model* model,
                                    const lmm_product* product, int paths,
                                    int mode);

/* First pass: simulate `paths` paths from Sobol point path_offset+1 and
 * write the Longstaff–Schwartz inputs of the batch into columns
 * [col_offset, col_offset+paths) of arrays with total_paths columns:
 * d_vars [E][3][total], d_ex [E][total] (exercise value at T_e),
 * d_cf [E][total] (coupons deflated to T_e), d_num [E][total] (numeraire
 * at T_e, units of the numeraire at T_0).  Basis variables are
 * (f_s, SR, A) per product (see lmm_c.h / product kinds). */
int lmm_pipeline_first_pass(const lmm_model* model, const lmm_product* product,
                            int paths, uint32_t path_offset, int mode,
                            void* d_workspace, size_t workspace_bytes,
                            int total_paths, int col_offset, float* d_vars,
                            float* d_ex, float* d_cf, float* d_num,
                            lmm_stream_t stream);

/* Second pass: simulate `paths` fresh paths and apply the frozen exercise
 * rule (d_beta [E][16], optional d_means/d_sds [E][3]); writes each path's
 * deflated payoff (units of the numeraire at T_0) to d_payoff[paths].  For
 * LMM_PRODUCT_EUROPEAN the rule is ignored and the payoff is the strip. */
int lmm_pipeline_second_pass(const lmm_model* model, const lmm_product* product,
                             int paths, uint32_t path_offset, int mode,
                             const double* d_beta, const float* d_means,
                             const float* d_sds, void* d_workspace,
                             size_t workspace_bytes, float* d_payoff,
                             lmm_stream_t stream);

/* lmm_pipeline_second_pass with a nested rule and Andersen shifts
 * (lmm_ls_rule, lmm_c.h): the decision chain of MultiLSExerciseStrategy
 * (gold/MultiLS_regression.h:137-231) in every mode. */
int lmm_pipeline_second_pass_rule(const lmm_model* model, const lmm_product* product,
                                  int paths, uint32_t path_offset, int mode,
                                  const lmm_ls_rule* rule, void* d_workspace,
                                  size_t workspace_bytes, float* d_payoff,
                                  lmm_stream_t stream);

/* ---- (f4) Andersen–Broadie upper bound ----------------------------------
 * The reference computes it on the CPU only (gold/gold_example/
 * LMM_bermudan_gold.cpp:1132-1382 with ABDualityGapEstimate*Rebate,
 * gold/Andersen_Broadie_gold.cpp:59-187).  For the Bermudan payer swaption
 * and a frozen rule: outer_paths paths from Sobol point outer_offset + 1
 * record the rule's decision X[e][p] at every date and the deflated
 * exercise value Z[e][p]; from every (outer path, date but the last),
 * inner_paths paths continue from the outer state with Philox4x32-10
 * normals (key = seed) and the rule applied at the later dates, giving the
 * continuation estimate Q[e][p] (last date: 0).  d_out = {gap mean, gap
 * standard error, lower bound mean, lower bound standard error} over the
 * outer paths (units of the numeraire at T_0); upper bound = lower bound +
 * gap.  Optional outputs (NULL: kept in the workspace): d_Q, d_Z [E][K]
 * (double), d_X [E][K], d_ckpt [n][n][K] log-rates at the start of each
 * step, d_ckptN [n][K] numeraires. */
typedef struct lmm_ab_config {
  int outer_paths;           /* K                                         */
  uint32_t outer_offset;     /* Sobol offset of the outer paths           */
  int inner_paths;           /* per (outer path, date), multiple of 128   */
  unsigned long long seed;   /* Philox key of the inner normals           */
} lmm_ab_config;
size_t lmm_andersen_broadie_workspace_bytes(const lmm_model* model,
                                            const lmm_product* product,
                                            const lmm_ab_config* config);
int lmm_andersen_broadie(const lmm_model* model, const lmm_product* product,
                         const lmm_ls_rule* rule, const lmm_ab_config* config,
                         void* d_workspace, size_t workspace_bytes, double* d_out,
                         double* d_Q, int* d_X, double* d_Z, float* d_ckpt,
                         float* d_ckptN, lmm_stream_t stream);
/* The duality-gap estimator on given data, with the reference's layouts
 * (ABDualityGapEstimateNonZeroRebate; d_payoffs NULL: the zero-rebate
 * form): d_ex [steps][paths] (0/1), d_payoffs [steps][paths], d_means
 * [paths][steps], h_is_exercise [steps].  d_out[4] = {gap mean, gap se,
 * mean and se of the payoff at each path's first exercise}. */
size_t lmm_ab_duality_gap_workspace_bytes(int paths);
int lmm_ab_duality_gap(int steps, int paths, const int* h_is_exercise, const int* d_ex,
                       const double* d_payoffs, const double* d_means, void* d_workspace,
                       size_t workspace_bytes, double* d_out, lmm_stream_t stream);

/* The two kernels of the fused form, callable separately.
 * lmm_fused_variates: Sobol points path_offset+1.. -> scramble -> inverse
 * normal -> bridge, written as [step][factor][path] increments (the
 * reference's transposed-variates layout, LMM_evolver_all.cu:1413-1419).
 * lmm_fused_evolve: evolves `paths` paths from those increments through all
 * steps.  With d_beta == NULL it writes the LS inputs (columns
 * [col_offset, col_offset+paths) of arrays with total_paths columns, as the
 * first pass); otherwise (or for the European product) it applies the
 * frozen rule and writes d_payoff[paths]. */
int lmm_fused_variates(const lmm_model* model, int paths, uint32_t path_offset,
                       float* d_variates, lmm_stream_t stream);
int lmm_fused_evolve(const lmm_model* model, const lmm_product* product,
                     int paths, const float* d_variates, const double* d_beta,
                     const float* d_means, const float* d_sds, int total_paths,
                     int col_offset, float* d_vars, float* d_ex, float* d_cf,
                     float* d_num, float* d_payoff, lmm_stream_t stream);

/* lmm_fused_evolve's rule pass (the second pass of BermudanMultiLSPricer-
 * Example, kooexample/bermudanIRDPricer.cu:1091-1483) with a nested or
 * shifted rule (NULL for the European strip and the TARN), run as a chain of
 * launches over segments of segment_steps steps (< 1: the library default,
 * 8; >= rates: one launch): after each segment the paths that have
 * exercised are dropped and the survivors are packed, so later steps run on
 * full warps.  Payoffs are bit-identical to lmm_fused_evolve's.  The
 * workspace holds two survivor buffers of about (rates + 7) x 4 B per path
 * (0 bytes for products that do not stop). */
size_t lmm_fused_price_workspace_bytes(const lmm_model* model,
                                       const lmm_product* product, int paths);
int lmm_fused_price(const lmm_model* model, const lmm_product* product, int paths,
                    const float* d_variates, const lmm_ls_rule* rule, int segment_steps,
                    void* d_workspace, size_t workspace_bytes, float* d_payoff,
                    lmm_stream_t stream);

/* lmm_fused_evolve with the tensor-core evolution (LMM_MODE_TENSOR); the
 * workspace (lmm_tensor_evolve_workspace_bytes) holds the per-step
 * operand images built from d_A at each call. */
size_t lmm_tensor_evolve_workspace_bytes(const lmm_model* model);
int lmm_tensor_evolve(const lmm_model* model, const lmm_product* product,
                      int paths, const float* d_variates, const double* d_beta,
                      const float* d_means, const float* d_sds, int total_paths,
                      int col_offset, float* d_vars, float* d_ex, float* d_cf,
                      float* d_num, float* d_payoff, void* d_workspace,
                      size_t workspace_bytes, lmm_stream_t stream);

/* Device error word of this GPU (value 1: a bounded wait of a tensor-core
 * kernel ran out and its outputs are invalid); synchronous; clear != 0
 * resets it.  The word's device address is looked up once per device and
 * kept for the life of the process: the tensor-core entry points and this
 * one must not be called after cudaDeviceReset (or any other destruction
 * of that device's primary context). */
int lmm_device_error_flags(int clear, unsigned int* h_flags);

/* Number of kernels this library has launched in this process (all entry
 * points); used to report launch counts. */
long lmm_launch_count(void);

/* Frozen-rule payoff from precomputed LS inputs (d_vars/d_ex/d_cf/d_num as
 * written by the first pass): per path, walk the exercise dates, stop at
 * the first date whose exercise value exceeds the estimated continuation
 * (MultiLSExerciseStrategy::decide, gold/MultiLS_regression.h:190-226;
 * SecondPassPriceLSAMultiUsingAggregatedFlows_gold, :228-289). */
int lmm_ls_apply_rule(int n_exercise, int paths, const float* d_vars,
                      const int* h_nvars, const uint8_t* h_monomials,
                      const int* h_nbasis, const float* d_cf, const float* d_ex,
                      const float* d_num, const double* d_beta,
                      const float* d_means, const float* d_sds,
                      float* d_payoff, lmm_stream_t stream);
/* lmm_ls_apply_rule with a nested rule and Andersen shifts. */
int lmm_ls_apply_rule_nested(int n_exercise, int paths, const float* d_vars,
                             const int* h_nvars, const uint8_t* h_monomials,
                             const int* h_nbasis, const float* d_cf, const float* d_ex,
                             const float* d_num, const lmm_ls_rule* rule,
                             float* d_payoff, lmm_stream_t stream);

/* ---- (f) pathwise adjoint Greeks ----------------------------------------
 * No counterpart in the reference, which prices only.  Sensitivities of
 * the frozen-rule price V = P(0,T_0) mean_p Phi_p (the fused second pass of
 * lmm_pipeline_second_pass over the same Sobol points, with
 * P(0,T_0) = 1 / (1 + f0_0 t0)), each path's exercise step held fixed
 * (pathwise method).  One reverse sweep over the steps, with log-rate
 * checkpoints every checkpoint_every steps recomputed segment by segment;
 * dV/dA is summed over paths inside the reverse sweep (FP64 above the warp,
 * fixed order, so results do not depend on scheduling).  Outputs (device,
 * FP64):
 *   d_price      [1] (or NULL)           V
 *   d_delta      [rates]                 dV / df0_r
 *   d_abar       [steps][rates][factors] dV / dA for every pseudo-root
 *                                        entry (the fixed drift -|A_r|^2/2
 *                                        follows A)
 *   d_vega_rate  [rates] (or NULL)       dV / dk_r for the row scaling
 *                                        A_s[r] -> k_r A_s[r] of every step
 *   d_exercise_step [paths] (or NULL)    each path's exercise step under the
 *                                        rule (rates = never), int32
 * paths must be a multiple of 4.  Vegas to other volatility parameters
 * follow by the chain rule through the host pseudo-root construction
 * (lmm_abcd_vegas in lmm_c.h).  The call is ordered on `stream` like every
 * other entry point; inside it, the reverse sweep and the recompute of the
 * next segments run on two streams of the library's own (one pair per host
 * thread and device, made on that thread's first call and kept until exit)
 * that fork from `stream` and join it again before the call's last kernels;
 * like the library's other per-device caches they must not outlive a
 * cudaDeviceReset (or any other destruction of the device's primary
 * context). */
size_t lmm_greeks_workspace_bytes(const lmm_model* model,
                                  const lmm_product* product, int paths,
                                  int checkpoint_every);
int lmm_greeks(const lmm_model* model, const lmm_product* product, int paths,
               uint32_t path_offset, const double* d_beta, const float* d_means,
               const float* d_sds, float t0, int checkpoint_every,
               void* d_workspace, size_t workspace_bytes, double* d_price,
               double* d_delta, double* d_abar, double* d_vega_rate,
               int* d_exercise_step, int* d_status, lmm_stream_t stream);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* LMM_PIPELINE_H */
