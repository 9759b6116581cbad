// ref_bridge.cu — C entry point into the reference's own newBridge host code.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together
// with the reference's brownian_bridge.cu (and gpuCompatibilityCheck.cu,
// which it links against) in place, with nvcc, into
// oracle/_ref/libkoobridge.so.  Only the host path of the class is used:
// the constructor builds the construction tables (brownian_bridge.cu:355,
// initialize() at :639-697) and transform() on std::vectors runs
// brownian_bridge::transformCPU (:401-455).  Nothing here touches a GPU,
// so the fixtures it produces can be made on a machine without one.
//
// The reference file pulls in cudaWrappers/cudaTextureBinder.h, whose
// legacy texture<> references CUDA 12 removed; brownian_bridge.cu itself
// uses none of it (its texture code is commented out), so the Makefile
// force-includes ref_bridge_stub.h, which marks that header as already
// included and supplies the thrust headers Utilities.h expects.
#include "brownian_bridge.h"

#include <gold/Bridge_allocator_gold.h>

#include <vector>

#define KREF extern "C" __attribute__((visibility("default")))

// brownian_bridge(size, allocation).transform(in, out, paths, steps, factors)
// on the CPU.  in: [factors*steps][paths] normals; out: [steps][factors]
// [paths] increments.  alloc: [factors][steps] Sobol dimension of each
// bridge variate, or NULL for bridge_allocate_diagonal
// (gold/Bridge_allocator_gold.cpp:38).  Returns 0, or 1 when the reference
// throws.
KREF int kref_newbridge_transform(int steps, int factors, int paths,
                                  const int* alloc, const float* in,
                                  float* out) {
  try {
    // the reference's allocator fills a vector of factors * steps entries
    std::vector<int> indices((size_t)steps * factors);
    if (alloc) {
      indices.assign(alloc, alloc + (size_t)steps * factors);
    } else {
      bridge_allocate_diagonal(indices, factors, steps);
    }
    brownian_bridge bb(steps, indices);
    std::vector<float> input(in, in + (size_t)steps * factors * paths);
    std::vector<float> output((size_t)steps * factors * paths, 0.0f);
    bb.transform(input, output, paths, steps, factors);
    std::copy(output.begin(), output.end(), out);
    return 0;
  } catch (...) {
    return 1;
  }
}
