/* ref_bridge_stub.h — forced include for building the reference's
 * brownian_bridge.cu host code with CUDA 12 (TEST INFRASTRUCTURE ONLY).
 *
 * cudaWrappers/cudaTextureBinder.h declares wrappers around legacy
 * texture<> references, which CUDA 12 removed; brownian_bridge.cu includes
 * the header but uses none of it.  Defining the header's include guard
 * skips it.  Utilities.h names thrust::host_vector without including it. */
#define CUDA_TEXTURE_BINDER_H
#include <thrust/host_vector.h>
#include <thrust/device_vector.h>
