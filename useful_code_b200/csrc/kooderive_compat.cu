// kooderive_compat.cu — the reference's GPU entry points by their own names
// and argument lists (include/kooderive_compat.h), each forwarding to the
// lmm_* entry point that replaces it.  Host code only: the small tables the
// reference keeps in device memory for its textures are read back here to
// travel as kernel parameters; the reference's synchronous behaviour is
// kept (a device synchronisation at the end of each routine), and its
// print-and-exit error handling becomes a std::runtime_error.
#include "../../include/kooderive_compat.h"
#include "../../include/lmm_c.h"

#include <chrono>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

void check(int status, const char* who) {
  if (status != LMM_OK)
    throw std::runtime_error(std::string(who) + ": " + lmm_last_error_string());
}

void check_cuda(cudaError_t e, const char* who) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(who) + ": " + cudaGetErrorString(e));
}

void finish(const char* who) { check_cuda(cudaDeviceSynchronize(), who); }

template <class T>
std::vector<T> to_host(const T* d, size_t n, const char* who) {
  std::vector<T> h(n);
  if (n) check_cuda(cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost), who);
  return h;
}

// The reference's log-rate cap of its Euler kernels (LMM_evolver_gpu.cu:20);
// its predictor-corrector kernels do not cap.
const float kEulerCap = std::log(10.0f);
const float kNoCap = 1e30f;

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

// ---- Sobol, scramble, bridges ----------------------------------------------
extern "C" void sobolGPUInts(int n_vectors, int n_dimensions, unsigned path_offset,
                             unsigned int* d_directions, unsigned int* d_output) {
  check(lmm_sobol_ints(n_vectors, n_dimensions, path_offset, d_directions, d_output, nullptr),
        "sobolGPUInts");
  finish("sobolGPUInts");
}

extern "C" void scramble_gpu(unsigned int* device_data, unsigned int* scramblers, int number_dim,
                             int paths) {
  check(lmm_scramble(device_data, scramblers, number_dim, paths, nullptr), "scramble_gpu");
  finish("scramble_gpu");
}

extern "C" void brownianBridgeGPU_constant_memory(int n_vectors, int n_poweroftwo, float* input,
                                                  float* output) {
  if (n_poweroftwo < 0 || n_poweroftwo > 7)
    throw std::runtime_error("brownianBridgeGPU_constant_memory: 2^k points with k in [0,7]");
  const int points = 1 << n_poweroftwo;
  std::vector<int> identity(points);
  for (int i = 0; i < points; ++i) identity[i] = i;
  check(lmm_bridge_transform(input, output, n_vectors, points, 1, identity.data(), nullptr),
        "brownianBridgeGPU_constant_memory");
  finish("brownianBridgeGPU_constant_memory");
}

extern "C" void brownianBridgeMultiGPUReorder(float* input, float* output, int n_poweroftwo,
                                              int factors, int number_paths, int allocator,
                                              bool /*useTextures*/) {
  check(lmm_bridge_reorder(input, output, n_poweroftwo, factors, number_paths, allocator, nullptr),
        "brownianBridgeMultiGPUReorder");
  finish("brownianBridgeMultiGPUReorder");
}

// ---- correlation and evolution ----------------------------------------------
extern "C" void correlated_drift_paths_GPU(float* input_data_device, float* output_data_device,
                                           float* A_device, int* alive_device,
                                           float* drift_fixed_device, int A_offset_per_step,
                                           int factors, int out_dimensions, int number_paths,
                                           int steps) {
  const std::vector<int> alive = to_host(alive_device, (size_t)steps, "correlated_drift_paths_GPU");
  check(lmm_correlate_drift(input_data_device, output_data_device, A_device, alive.data(),
                            drift_fixed_device, A_offset_per_step, factors, out_dimensions,
                            number_paths, steps, 0, nullptr),
        "correlated_drift_paths_GPU");
  finish("correlated_drift_paths_GPU");
}

extern "C" void LMM_evolver_pc_gpu(float* initial_rates_device, float* /*initial_log_rates*/,
                                   float* taus_device, float* correlatedBrownianIncrements_device,
                                   float* pseudo_roots_device, float* /*initial_drifts*/,
                                   float* displacements_device,
                                   const std::vector<int>& aliveIndices, int paths, int factors,
                                   int steps, int rates, float* /*e_buffer*/,
                                   float* /*e_buffer_pred*/, float* evolved_rates_device,
                                   float* evolved_log_rates_device, bool /*useShared*/) {
  const char* who = "LMM_evolver_pc_gpu";
  if ((int)aliveIndices.size() < steps) throw std::runtime_error("LMM_evolver_pc_gpu: too few alive indices");
  const auto f0 = to_host(initial_rates_device, (size_t)rates, who);
  const auto taus = to_host(taus_device, (size_t)rates, who);
  const auto disp = to_host(displacements_device, (size_t)rates, who);
  check(lmm_evolve_pc_staged(f0.data(), taus.data(), disp.data(),
                             correlatedBrownianIncrements_device, pseudo_roots_device,
                             aliveIndices.data(), paths, factors, steps, rates, kNoCap,
                             evolved_rates_device, evolved_log_rates_device, nullptr),
        who);
  finish(who);
}

extern "C" void LMM_evolver_euler_gpu(float* initial_rates_device, float* /*initial_log_rates*/,
                                      float* taus_device,
                                      float* correlatedBrownianIncrements_device,
                                      float* pseudo_roots_device, float* /*initial_drifts*/,
                                      float* displacements_device,
                                      const std::vector<int>& aliveIndices, int paths,
                                      int factors, int steps, int rates, float* /*e_buffer*/,
                                      float* evolved_rates_device,
                                      float* evolved_log_rates_device) {
  const char* who = "LMM_evolver_euler_gpu";
  if ((int)aliveIndices.size() < steps) throw std::runtime_error("LMM_evolver_euler_gpu: too few alive indices");
  const auto f0 = to_host(initial_rates_device, (size_t)rates, who);
  const auto taus = to_host(taus_device, (size_t)rates, who);
  const auto disp = to_host(displacements_device, (size_t)rates, who);
  check(lmm_evolve_euler_staged(f0.data(), taus.data(), disp.data(),
                                correlatedBrownianIncrements_device, pseudo_roots_device,
                                aliveIndices.data(), paths, factors, steps, rates, kEulerCap,
                                evolved_rates_device, evolved_log_rates_device, nullptr),
        who);
  finish(who);
}

extern "C" void LMM_evolver_pc_all_gpu(float* initial_rates_device, float* /*initial_log_rates*/,
                                       float* taus_device, float* variates_device,
                                       float* pseudo_roots_device, float* /*initial_drifts*/,
                                       float* fixed_drifts_device, float* displacements_device,
                                       int* alive_device, int paths, int factors, int steps,
                                       int rates, float* /*e_buffer*/, float* /*e_buffer_pred*/,
                                       float* evolved_rates_device,
                                       float* evolved_log_rates_device, float* discounts_device,
                                       bool /*sharedMemForLogs*/, bool transposeData,
                                       cudaStream_t streamNumber, int /*numberThreads*/,
                                       bool doDiscounts) {
  const char* who = "LMM_evolver_pc_all_gpu";
  const auto f0 = to_host(initial_rates_device, (size_t)rates, who);
  const auto taus = to_host(taus_device, (size_t)rates, who);
  const auto disp = to_host(displacements_device, (size_t)rates, who);
  const auto alive = to_host(alive_device, (size_t)steps, who);
  // the reference reads transposed variates only in its discounting engine
  const int layout = (transposeData && doDiscounts) ? 1 : 0;
  check(lmm_evolve_pc_all(f0.data(), taus.data(), disp.data(), variates_device, layout,
                          pseudo_roots_device, fixed_drifts_device, alive.data(), paths, factors,
                          steps, rates, kNoCap, evolved_rates_device, evolved_log_rates_device,
                          doDiscounts ? discounts_device : nullptr, (lmm_stream_t)streamNumber),
        who);
}

// ---- curve quantities --------------------------------------------------------
extern "C" void discount_ratios_computation_gpu(float* evolved_rates_device, float* taus_device,
                                                const std::vector<int>& aliveIndices,
                                                int* /*alive_device*/, int paths, int steps,
                                                int rates, float* discounts_device,
                                                bool /*allStepsAtOnce*/) {
  const char* who = "discount_ratios_computation_gpu";
  const auto taus = to_host(taus_device, (size_t)rates, who);
  check(lmm_discount_ratios(evolved_rates_device, taus.data(), aliveIndices.data(), paths, steps,
                            rates, discounts_device, nullptr),
        who);
  finish(who);
}

extern "C" void coterminal_annuity_ratios_computation_gpu(float* discounts_device,
                                                          float* taus_device,
                                                          const std::vector<int>& aliveIndices,
                                                          int paths, int steps, int rates,
                                                          float* annuities_device) {
  const char* who = "coterminal_annuity_ratios_computation_gpu";
  const auto taus = to_host(taus_device, (size_t)rates, who);
  check(lmm_coterminal_annuities(discounts_device, taus.data(), aliveIndices.data(), paths, steps,
                                 rates, annuities_device, nullptr),
        who);
  finish(who);
}

extern "C" void coterminal_swap_rate_computation_gpu(float* discounts_device,
                                                     float* annuities_device,
                                                     const std::vector<int>& aliveIndices,
                                                     int paths, int steps, int rates,
                                                     float* cot_swap_rates_device) {
  const char* who = "coterminal_swap_rate_computation_gpu";
  check(lmm_coterminal_swap_rates(discounts_device, annuities_device, aliveIndices.data(), paths,
                                  steps, rates, cot_swap_rates_device, nullptr),
        who);
  finish(who);
}

extern "C" void swap_rate_computation_gpu(float* discounts_device, float* taus_device,
                                          int startIndex, int endIndex, int paths,
                                          int step_for_offset_in, int step_for_offset_out,
                                          int rates, float* swap_rate_device) {
  const char* who = "swap_rate_computation_gpu";
  const auto taus = to_host(taus_device, (size_t)rates, who);
  const int steps = 1 + (step_for_offset_in > step_for_offset_out ? step_for_offset_in
                                                                     : step_for_offset_out);
  check(lmm_swap_rate(discounts_device, taus.data(), startIndex, endIndex, paths,
                      step_for_offset_in, step_for_offset_out, steps, rates, swap_rate_device,
                      nullptr),
        who);
  finish(who);
}

extern "C" void spot_measure_numeraires_computation_gpu(float* discount_factors_global,
                                                        float* numeraire_values_global,
                                                        int paths, int n_rates) {
  check(lmm_spot_numeraires(discount_factors_global, paths, paths, 0, n_rates,
                            numeraire_values_global, nullptr),
        "spot_measure_numeraires_computation_gpu");
  finish("spot_measure_numeraires_computation_gpu");
}

extern "C" void spot_measure_numeraires_computation_offset_gpu(float* discount_factors_global,
                                                               float* numeraire_values_global,
                                                               int paths, int pathsForOutput,
                                                               int pathsOffsetForOutput,
                                                               int n_rates) {
  check(lmm_spot_numeraires(discount_factors_global, paths, pathsForOutput, pathsOffsetForOutput,
                            n_rates, numeraire_values_global, nullptr),
        "spot_measure_numeraires_computation_offset_gpu");
  finish("spot_measure_numeraires_computation_offset_gpu");
}

extern "C" void forward_rate_extraction_gpu(float* all_forwards_device,
                                            const std::vector<int>& forwardIndices, int paths,
                                            int steps, int rates, float* select_forwards_device) {
  if ((int)forwardIndices.size() < steps)
    throw std::runtime_error("forward_rate_extraction_gpu: too few forward indices");
  check(lmm_forward_extraction(all_forwards_device, forwardIndices.data(), paths, steps, rates,
                               select_forwards_device, nullptr),
        "forward_rate_extraction_gpu");
  finish("forward_rate_extraction_gpu");
}

extern "C" void forward_rate_extraction_selecting_step_gpu(
    float* all_forwards_device, const std::vector<int>& forwardIndices,
    const std::vector<int>& stepIndices, int paths, int rates, float* select_forwards_device) {
  if (stepIndices.size() < forwardIndices.size())
    throw std::runtime_error("forward_rate_extraction_selecting_step_gpu: too few step indices");
  check(lmm_forward_extraction_steps(all_forwards_device, forwardIndices.data(),
                                     stepIndices.data(), (int)forwardIndices.size(), paths, rates,
                                     select_forwards_device, nullptr),
        "forward_rate_extraction_selecting_step_gpu");
  finish("forward_rate_extraction_selecting_step_gpu");
}

extern "C" double spot_measure_numeraires_extraction_gpu(float* all_numeraire_values_global,
                                                         float* some_numeraire_values_global,
                                                         int pathsInput, int pathsOutput,
                                                         int offsetForOutput, int numberRates,
                                                         int numberExerciseTimes,
                                                         int* exerciseIndices_vec) {
  const char* who = "spot_measure_numeraires_extraction_gpu";
  const auto t0 = std::chrono::steady_clock::now();
  const auto idx = to_host(exerciseIndices_vec, (size_t)numberExerciseTimes, who);
  check(lmm_numeraire_extraction(all_numeraire_values_global, some_numeraire_values_global,
                                 pathsInput, pathsOutput, offsetForOutput, numberRates,
                                 numberExerciseTimes, idx.data(), nullptr),
        who);
  finish(who);
  return seconds_since(t0);
}

// ---- cash flows ---------------------------------------------------------------
extern "C" void cashFlowGeneratorCallerSwap(float* genFlows1, float* genFlows2, float* aux_data,
                                            int paths, int numberSteps, float* rates1,
                                            float* /*rates2*/, float* /*rates3*/,
                                            float* /*forwards*/, float* /*discRatios*/) {
  const char* who = "cashFlowGeneratorCallerSwap";
  const auto aux = to_host(aux_data, (size_t)(2 + 2 * numberSteps), who);
  check(lmm_cashflows_swap(genFlows1, genFlows2, aux.data(), paths, numberSteps, rates1, nullptr),
        who);
  finish(who);
}

extern "C" void cashFlowGeneratorCallerTARN(float* genFlows1, float* genFlows2, float* aux_data,
                                            int paths, int numberSteps, float* rates1,
                                            float* rates2, float* /*rates3*/,
                                            float* /*forwards*/, float* /*discRatios*/) {
  const char* who = "cashFlowGeneratorCallerTARN";
  const auto aux = to_host(aux_data, (size_t)(3 + 2 * numberSteps), who);
  check(lmm_cashflows_tarn(genFlows1, genFlows2, aux.data(), paths, numberSteps, rates1, rates2,
                           nullptr),
        who);
  finish(who);
}

extern "C" void cashFlowDiscounting_gpu(int* firstIndex, int* secondIndex, float* theta,
                                        float* discountRatios, float* genFlows,
                                        float* numeraireValues, int paths, int numberSteps,
                                        bool /*useTextures*/, bool /*useShared*/,
                                        float* discountedFlows, float* summedDiscountedFlows) {
  const char* who = "cashFlowDiscounting_gpu";
  const auto first = to_host(firstIndex, (size_t)numberSteps, who);
  const auto second = to_host(secondIndex, (size_t)numberSteps, who);
  const auto th = to_host(theta, (size_t)numberSteps, who);
  check(lmm_cashflow_discounting(first.data(), second.data(), th.data(), discountRatios, genFlows,
                                 numeraireValues, paths, numberSteps, discountedFlows,
                                 summedDiscountedFlows, nullptr),
        who);
  finish(who);
}

extern "C" void cashFlowDiscounting_partial_gpu(int numberFlowsPerPath,
                                                int* generationIndices_dev, int* firstIndex_dev,
                                                int* secondIndex_dev, float* theta_dev,
                                                int* targetIndices_dev,
                                                float* discountRatios_dev, float* genFlows_dev,
                                                float* numeraireValues_dev, int paths,
                                                int numberSteps, float* discountedFlows_dev) {
  const char* who = "cashFlowDiscounting_partial_gpu";
  const size_t n = (size_t)numberFlowsPerPath;
  const auto gen = to_host(generationIndices_dev, n, who);
  const auto first = to_host(firstIndex_dev, n, who);
  const auto second = to_host(secondIndex_dev, n, who);
  const auto th = to_host(theta_dev, n, who);
  const auto target = to_host(targetIndices_dev, n, who);
  check(lmm_cashflow_discounting_partial(numberFlowsPerPath, gen.data(), first.data(),
                                         second.data(), th.data(), target.data(),
                                         discountRatios_dev, genFlows_dev, numeraireValues_dev,
                                         paths, numberSteps, discountedFlows_dev, nullptr),
        who);
  finish(who);
}

extern "C" void AggregateFlows_gpu(float* aggregatedFlows, int totalPaths,
                                   int numberExerciseDates, float* genFlows, int batchPaths,
                                   int offSetForOutput, int numberSteps, int* precedingIndex,
                                   int start) {
  const char* who = "AggregateFlows_gpu";
  const auto prec = to_host(precedingIndex, (size_t)numberSteps, who);
  check(lmm_aggregate_flows(aggregatedFlows, totalPaths, numberExerciseDates, genFlows,
                            batchPaths, offSetForOutput, numberSteps, prec.data(), start,
                            nullptr),
        who);
  finish(who);
}

// ---- Longstaff–Schwartz -------------------------------------------------------
extern "C" void adjoinBasisVariablesCaller_gpu(bool useLogs, int* /*integerData_dev*/,
                                               float* floatData_dev, float* /*forwards_dev*/,
                                               float* /*discountRatios_dev*/, float* rate1_dev,
                                               float* rate2_dev, float* rate3_dev,
                                               int numberPathsPerBatch, int totalNumberOfPaths,
                                               int numberPathsPreviouslyDone,
                                               int /*numberStepsAndRates*/,
                                               int numberExerciseTimes,
                                               int* /*exerciseIndices_dev*/,
                                               int* /*exerciseIndicators_dev*/,
                                               float* basisFunctionVariables_dev) {
  const char* who = "adjoinBasisVariablesCaller_gpu";
  std::vector<float> shifts(3, 0.0f);
  if (useLogs) shifts = to_host(floatData_dev, 3, who);
  check(lmm_basis_variables(useLogs ? 1 : 0, shifts.data(), rate1_dev, rate2_dev, rate3_dev,
                            numberPathsPerBatch, totalNumberOfPaths, numberPathsPreviouslyDone,
                            numberExerciseTimes, basisFunctionVariables_dev, nullptr),
        who);
  finish(who);
}

void expandBasisFunctions_quadratic_gpu(int totalNumberOfPaths, float* basisVariables_global,
                                        int exerciseNumber, int maxBasisVariableSize,
                                        int variableSizeThisStep, bool useCrossTerms,
                                        float* basisFunctions_global) {
  check(lmm_ls_expand_basis(totalNumberOfPaths, basisVariables_global, exerciseNumber,
                            maxBasisVariableSize, variableSizeThisStep, useCrossTerms ? 1 : 0,
                            basisFunctions_global, nullptr),
        "expandBasisFunctions_quadratic_gpu");
  finish("expandBasisFunctions_quadratic_gpu");
}

double continuation_net_value_evaluation_gpu(int paths, int /*exerciseNumber*/,
                                             float* basisFunctions_global,
                                             int numberBasisFunctions,
                                             float* basis_weights_global,
                                             float* exerciseValues_global, float AndersenShift,
                                             float* output_global) {
  const auto t0 = std::chrono::steady_clock::now();
  check(lmm_ls_net_values(paths, basisFunctions_global, numberBasisFunctions,
                          basis_weights_global, exerciseValues_global, AndersenShift,
                          output_global, nullptr),
        "continuation_net_value_evaluation_gpu");
  finish("continuation_net_value_evaluation_gpu");
  return seconds_since(t0);
}

double oneStepUpdateLS_multi_gpu(int paths, int exerciseNumber, float* basisFunctions_global,
                                 int numberBasisFunctions, int basisFunctionsRowSize,
                                 int maxRegressionDepth, float* basis_weights_global,
                                 float* lowerCuts_global, float* upperCuts_global,
                                 float* continuationValues_global,
                                 float* /*deflatedCashFlows_global*/,
                                 float* exerciseValues_global, float AndersenShift,
                                 float* estContinuationValues_global, int* exercises_global) {
  const auto t0 = std::chrono::steady_clock::now();
  check(lmm_ls_update_multi(paths, exerciseNumber, basisFunctions_global, numberBasisFunctions,
                            basisFunctionsRowSize, maxRegressionDepth, basis_weights_global,
                            lowerCuts_global, upperCuts_global, continuationValues_global,
                            exerciseValues_global, AndersenShift, estContinuationValues_global,
                            exercises_global, nullptr),
        "oneStepUpdateLS_multi_gpu");
  finish("oneStepUpdateLS_multi_gpu");
  return seconds_since(t0);
}

double updateDeflationOfContinuationValues_gpu(float* deflatedNextStepValues_global,
                                               float* numeraireValues_global, int paths,
                                               int newStepNumber, int oldStepNumber) {
  const auto t0 = std::chrono::steady_clock::now();
  check(lmm_ls_deflate(deflatedNextStepValues_global, numeraireValues_global, paths,
                       newStepNumber, oldStepNumber, nullptr),
        "updateDeflationOfContinuationValues_gpu");
  finish("updateDeflationOfContinuationValues_gpu");
  return seconds_since(t0);
}

// ---- reductions -----------------------------------------------------------------
const float* PartialReduce_using8s_gpu(const float* data, float* workspace, int points,
                                       int /*threads*/, int stopPoint) {
  const float* out = nullptr;
  check(lmm_partial_reduce(data, workspace, points, 8, stopPoint, &out, nullptr),
        "PartialReduce_using8s_gpu");
  finish("PartialReduce_using8s_gpu");
  return out;
}

const float* PartialReduce_using16s_gpu(const float* data, float* workspace, int points,
                                        int /*threads*/) {
  const float* out = nullptr;
  check(lmm_partial_reduce(data, workspace, points, 16, 1, &out, nullptr),
        "PartialReduce_using16s_gpu");
  finish("PartialReduce_using16s_gpu");
  return out;
}

namespace {

// The reference sizes its workspace as blocks x rows x cols floats with
// blocks = threads, rounded down to a power of two and at least 32
// (outerProduct_gpu.cu:650-670); the first 256 bytes hold the status word.
void outer_product(const char* who, int paths, int rows, int cols, int threads, float* in1,
                   float* in2, float* answer, float* workspace) {
  int t = threads < 32 ? 32 : threads;
  int p2 = 32;
  while (p2 * 2 <= t) p2 *= 2;
  const size_t bytes = (size_t)p2 * rows * cols * sizeof(float);
  if (bytes <= 256) throw std::runtime_error(std::string(who) + ": workspace too small");
  int* status = reinterpret_cast<int*>(workspace);
  char* ws = reinterpret_cast<char*>(workspace) + 256;
  check(lmm_outer_product(paths, rows, cols, in1, in2, answer, ws, bytes - 256, status, nullptr),
        who);
  finish(who);
  int st = 0;
  check_cuda(cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost), who);
  if (st != 0) throw std::runtime_error(std::string(who) + ": a bounded device wait ran out");
}

}  // namespace

void reduceOuterProduct_gpu(int paths, int row_size, int col_size, bool symmetric, int threads,
                            int /*blocks*/, float* input_data_global1, float* input_data_global2,
                            float* answer_global, float* workspace_data_global) {
  if (symmetric)
    outer_product("reduceOuterProduct_gpu", paths, row_size, row_size, threads,
                  input_data_global1, input_data_global1, answer_global, workspace_data_global);
  else
    outer_product("reduceOuterProduct_gpu", paths, row_size, col_size, threads,
                  input_data_global1, input_data_global2, answer_global, workspace_data_global);
}

void reduceOuterProductSymmetric_gpu(int paths, int row_size, int threads, int /*blocks*/,
                                     float* input_data_global1, float* answer_global,
                                     float* workspace_data_global) {
  outer_product("reduceOuterProductSymmetric_gpu", paths, row_size, row_size, threads,
                input_data_global1, input_data_global1, answer_global, workspace_data_global);
}
