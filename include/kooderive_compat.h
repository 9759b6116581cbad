/*
 * kooderive_compat.h — the reference's GPU entry points under their own
 * names and argument lists, exported by liblmm_b200.so, so that a caller
 * written against Kooderive r256's headers links against this library
 * unchanged.  C++ only: the reference's extern "C" routines take
 * std::vector references and bool defaults, and its LS, reduction and
 * outer-product routines have C++ linkage; both are kept as declared there.
 *
 * Every routine forwards to the lmm_* entry point named beside it (lmm_c.h,
 * lmm_pipeline.h) on the legacy default stream, except
 * LMM_evolver_pc_all_gpu, which runs on the stream it is given.  Small
 * tables the reference binds to textures (alive indices, accruals,
 * displacements, initial rates, discounting indices and weights, auxiliary
 * product data, basis shifts, LS coefficients and cut-offs) are read back
 * from the device to travel as kernel parameters.  Like the reference,
 * each routine returns when its work is done (a device synchronisation at
 * the end), except LMM_evolver_pc_all_gpu.  Where the reference prints and
 * exits on an error, these throw std::runtime_error carrying
 * lmm_last_error_string().  None allocates device memory: routines that
 * need scratch take it from the caller's workspace argument, as the
 * reference's do.
 *
 * Differences from the reference, each forced or deliberate:
 *   - brownianBridgeMultiGPUReorder takes the ordering as int (0 row,
 *     1 column, 2 triangular: the values of the reference's
 *     BrownianBridgeMultiDim<float>::ordering, passed identically); the
 *     gold header that defines that enum is not part of this library.
 *   - brownianBridgeGPU_constant_memory runs the bridge kernel of the
 *     newBridge on 2^k unit steps with the identity allocation: the same
 *     construction points, order, variates and weights as the reference's
 *     power-of-two bridge, with the weights rounded from their own FP32
 *     formulas.
 *   - the drift of the first step of LMM_evolver_pc_gpu, _euler_gpu and
 *     _pc_all_gpu is formed from the initial rates like every later step's;
 *     the reference's precomputed initial drifts and its e-buffers are not
 *     read.
 *   - the outer-product routines contract on the tensor cores (split TF32,
 *     FP64 sums of the batches) and need the number of paths to be a
 *     multiple of 4; the threads argument only sizes the workspace, as in
 *     the reference (blocks = threads, rounded to a power of two >= 32).
 *   - the reductions return the pointer to their last level as the
 *     reference does; a remainder smaller than a group is dropped.
 */
#ifndef KOODERIVE_COMPAT_H
#define KOODERIVE_COMPAT_H

#include <cuda_runtime.h>

#include <vector>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- Sobol, scramble, bridges ------------------------------------------ */
/* sobol_int_gpu.h -> lmm_sobol_ints */
extern "C" void sobolGPUInts(int n_vectors, int n_dimensions, unsigned path_offset,
                             unsigned int* d_directions, unsigned int* d_output);
/* scramble_gpu.h -> lmm_scramble */
extern "C" void scramble_gpu(unsigned int* device_data, unsigned int* scramblers,
                             int number_dim, int paths);
/* Bridge_gpu.h -> lmm_bridge_transform (one factor, 2^k steps, identity
 * allocation); input and output [2^k][n_vectors] */
extern "C" void brownianBridgeGPU_constant_memory(int n_vectors, int n_poweroftwo,
                                                  float* input, float* output);
/* Bridge_multi_gpu.h -> lmm_bridge_reorder; allocator: 0 row, 1 column,
 * 2 triangular; useTextures is ignored */
extern "C" void brownianBridgeMultiGPUReorder(float* input, float* output, int n_poweroftwo,
                                              int factors, int number_paths, int allocator,
                                              bool useTextures);

/* ---- correlation and evolution ------------------------------------------ */
/* Correlate_drift_gpu.h:12 -> lmm_correlate_drift (input [step][path][factor]) */
extern "C" void correlated_drift_paths_GPU(float* input_data_device, float* output_data_device,
                                           float* A_device, int* alive_device,
                                           float* drift_fixed_device, int A_offset_per_step,
                                           int factors, int out_dimensions, int number_paths,
                                           int steps);
/* LMM_evolver_gpu.h:16 -> lmm_evolve_pc_staged (no log-rate cap, as the
 * reference's step kernels) */
extern "C" void LMM_evolver_pc_gpu(float* initial_rates_device, float* initial_log_rates_device,
                                   float* taus_device, float* correlatedBrownianIncrements_device,
                                   float* pseudo_roots_device, float* initial_drifts_device,
                                   float* displacements_device,
                                   const std::vector<int>& aliveIndices, int paths, int factors,
                                   int steps, int rates, float* e_buffer_device,
                                   float* e_buffer_pred_device, float* evolved_rates_device,
                                   float* evolved_log_rates_device, bool useShared = false);
/* LMM_evolver_gpu.h:32 -> lmm_evolve_euler_staged (log-rates capped at
 * log 10, as the reference's Euler kernels) */
extern "C" void LMM_evolver_euler_gpu(float* initial_rates_device,
                                      float* initial_log_rates_device, float* taus_device,
                                      float* correlatedBrownianIncrements_device,
                                      float* pseudo_roots_device, float* initial_drifts_device,
                                      float* displacements_device,
                                      const std::vector<int>& aliveIndices, int paths,
                                      int factors, int steps, int rates, float* e_buffer_device,
                                      float* evolved_rates_device,
                                      float* evolved_log_rates_device);
/* LMM_evolver_all.h:23 -> lmm_evolve_pc_all (no log-rate cap, as the
 * reference's fused kernel); variates [step][factor][path] when
 * transposedVariates and doDiscounts, else [step][path][factor]; runs on
 * streamNumber and returns without waiting */
extern "C" void LMM_evolver_pc_all_gpu(float* initial_rates_device,
                                       float* initial_log_rates_device, float* taus_device,
                                       float* variates_device, float* pseudo_roots_device,
                                       float* initial_drifts_device, float* fixed_drifts_device,
                                       float* displacements_device, int* alive_device, int paths,
                                       int factors, int steps, int rates,
                                       float* e_buffer_device, float* e_buffer_pred_device,
                                       float* evolved_rates_device,
                                       float* evolved_log_rates_device, float* discounts_device,
                                       bool sharedMemForLogs, bool transposeData,
                                       cudaStream_t streamNumber, int numberThreads,
                                       bool doDiscounts);

/* ---- curve quantities (LMM_evolver_gpu.h:48-140) ------------------------ */
extern "C" void discount_ratios_computation_gpu(float* evolved_rates_device, float* taus_device,
                                                const std::vector<int>& aliveIndices,
                                                int* alive_device, int paths, int steps,
                                                int rates, float* discounts_device,
                                                bool allStepsAtOnce);
extern "C" void coterminal_annuity_ratios_computation_gpu(float* discounts_device,
                                                          float* taus_device,
                                                          const std::vector<int>& aliveIndices,
                                                          int paths, int steps, int rates,
                                                          float* annuities_device);
extern "C" void coterminal_swap_rate_computation_gpu(float* discounts_device,
                                                     float* annuities_device,
                                                     const std::vector<int>& aliveIndices,
                                                     int paths, int steps, int rates,
                                                     float* cot_swap_rates_device);
extern "C" void swap_rate_computation_gpu(float* discounts_device, float* taus_device,
                                          int startIndex, int endIndex, int paths,
                                          int step_for_offset_in, int step_for_offset_out,
                                          int rates, float* swap_rate_device);
extern "C" void spot_measure_numeraires_computation_gpu(float* discount_factors_global,
                                                        float* numeraire_values_global,
                                                        int paths, int n_rates);
extern "C" void spot_measure_numeraires_computation_offset_gpu(float* discount_factors_global,
                                                               float* numeraire_values_global,
                                                               int paths, int pathsForOutput,
                                                               int pathsOffsetForOutput,
                                                               int n_rates);
extern "C" void forward_rate_extraction_gpu(float* all_forwards_device,
                                            const std::vector<int>& forwardIndices, int paths,
                                            int steps, int rates, float* select_forwards_device);
extern "C" void forward_rate_extraction_selecting_step_gpu(
    float* all_forwards_device, const std::vector<int>& forwardIndices,
    const std::vector<int>& stepIndices, int paths, int rates, float* select_forwards_device);
/* returns the seconds the call took, as the reference */
extern "C" double spot_measure_numeraires_extraction_gpu(float* all_numeraire_values_global,
                                                         float* some_numeraire_values_global,
                                                         int pathsInput, int pathsOutput,
                                                         int offsetForOutput, int numberRates,
                                                         int numberExerciseTimes,
                                                         int* exerciseIndices_vec);

/* ---- cash flows (cashFlowGeneration_product_gpu.h:111,190,
 *      cashFlowDiscounting_gpu.h:15,30, cashFlowAggregation_gpu.h) ---------- */
extern "C" void cashFlowGeneratorCallerSwap(float* genFlows1, float* genFlows2, float* aux_data,
                                            int paths, int numberSteps, float* rates1,
                                            float* rates2, float* rates3, float* forwards,
                                            float* discRatios);
extern "C" void cashFlowGeneratorCallerTARN(float* genFlows1, float* genFlows2, float* aux_data,
                                            int paths, int numberSteps, float* rates1,
                                            float* rates2, float* rates3, float* forwards,
                                            float* discRatios);
extern "C" void cashFlowDiscounting_gpu(int* firstIndex, int* secondIndex, float* theta,
                                        float* discountRatios, float* genFlows,
                                        float* numeraireValues, int paths, int numberSteps,
                                        bool useTextures, bool useShared,
                                        float* discountedFlows, float* summedDiscountedFlows);
extern "C" void cashFlowDiscounting_partial_gpu(int numberFlowsPerPath,
                                                int* generationIndices_dev, int* firstIndex_dev,
                                                int* secondIndex_dev, float* theta_dev,
                                                int* targetIndices_dev,
                                                float* discountRatios_dev, float* genFlows_dev,
                                                float* numeraireValues_dev, int paths,
                                                int numberSteps, float* discountedFlows_dev);
extern "C" void AggregateFlows_gpu(float* aggregatedFlows, int totalPaths,
                                   int numberExerciseDates, float* genFlows, int batchPaths,
                                   int offSetForOutput, int numberSteps, int* precedingIndex,
                                   int start);

/* ---- Longstaff–Schwartz (LS_Basis_gpu.h:168, LS_gpu.h:21-80) ------------ */
/* -> lmm_basis_variables; floatData_dev holds the three log shifts */
extern "C" void adjoinBasisVariablesCaller_gpu(bool useLogs, int* integerData_dev,
                                               float* floatData_dev, float* forwards_dev,
                                               float* discountRatios_dev, float* rate1_dev,
                                               float* rate2_dev, float* rate3_dev,
                                               int numberPathsPerBatch, int totalNumberOfPaths,
                                               int numberPathsPreviouslyDone,
                                               int numberStepsAndRates, int numberExerciseTimes,
                                               int* exerciseIndices_dev,
                                               int* exerciseIndicators_dev,
                                               float* basisFunctionVariables_dev);
/* -> lmm_ls_expand_basis */
void expandBasisFunctions_quadratic_gpu(int totalNumberOfPaths, float* basisVariables_global,
                                        int exerciseNumber, int maxBasisVariableSize,
                                        int variableSizeThisStep, bool useCrossTerms,
                                        float* basisFunctions_global);
/* -> lmm_ls_net_values; returns the seconds the call took */
double continuation_net_value_evaluation_gpu(int paths, int exerciseNumber,
                                             float* basisFunctions_global,
                                             int numberBasisFunctions,
                                             float* basis_weights_global,
                                             float* exerciseValues_global, float AndersenShift,
                                             float* output_global);
/* -> lmm_ls_update_multi; returns the seconds the call took */
double oneStepUpdateLS_multi_gpu(int paths, int exerciseNumber, float* basisFunctions_global,
                                 int numberBasisFunctions, int basisFunctionsRowSize,
                                 int maxRegressionDepth, float* basis_weights_global,
                                 float* lowerCuts_global, float* upperCuts_global,
                                 float* continuationValues_global,
                                 float* deflatedCashFlows_global, float* exerciseValues_global,
                                 float AndersenShift, float* estContinuationValues_global,
                                 int* exercises_global);
/* -> lmm_ls_deflate; returns the seconds the call took */
double updateDeflationOfContinuationValues_gpu(float* deflatedNextStepValues_global,
                                               float* numeraireValues_global, int paths,
                                               int newStepNumber, int oldStepNumber);

/* ---- reductions (reductions_gpu.h:9-18, outerProduct_gpu.h:12-39) ------- */
/* -> lmm_partial_reduce */
const float* PartialReduce_using8s_gpu(const float* data, float* workspace, int points,
                                       int threads, int stopPoint = 1);
const float* PartialReduce_using16s_gpu(const float* data, float* workspace, int points,
                                        int threads);
/* -> lmm_outer_product; input [rows][paths], answer [rows][cols] */
void reduceOuterProduct_gpu(int paths, int row_size, int col_size, bool symmetric, int threads,
                            int blocks, float* input_data_global1, float* input_data_global2,
                            float* answer_global, float* workspace_data_global);
void reduceOuterProductSymmetric_gpu(int paths, int row_size, int threads, int blocks,
                                     float* input_data_global1, float* answer_global,
                                     float* workspace_data_global);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* KOODERIVE_COMPAT_H */
