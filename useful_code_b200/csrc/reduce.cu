// reduce.cu — deterministic FP64 sums over paths.
//
// Replaces the reference's path reductions (PartialReduce_using8s_gpu,
// reductions_gpu.cu:11-336, and the thrust::reduce price sums at
// kooexample/bermudanIRDPricer.cu:1470-1474, LS_main_cula.h:818).  The
// reference sums in FP32 with a block tree whose launch swaps grid and block
// dimensions (reductions_gpu.cu:153); here every sum is FP64 with a fixed
// two-level order (kReduceBlocks partials, then one block), so results are
// bit-reproducible for a given n.
#include "lmm_common.cuh"

using namespace lmm;

namespace lmm {
constexpr int kReduceBlocks = 512;
constexpr int kReduceThreads = 256;

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  return x;
}

// Block-wide sum; result valid in thread 0.  `sh` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double x, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  x = warp_sum(x);
  __syncthreads();
  if (lane == 0) sh[w] = x;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  x = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
  if (w == 0) x = warp_sum(x);
  return x;
}
}  // namespace lmm

// Stage 1: block b sums the contiguous chunk [b*chunk, (b+1)*chunk).
// `weights` (optional) multiplies each term: sum in[i] * w[i].
__global__ void __launch_bounds__(256)
    reduce_partial_kernel(const float* __restrict__ in,
                          const float* __restrict__ divisor, size_t n,
                          size_t chunk, double* __restrict__ partials) {
  __shared__ double sh[32];
  const size_t lo = blockIdx.x * chunk;
  size_t hi = lo + chunk;
  if (hi > n) hi = n;
  double acc = 0.0;
  size_t i0 = lo;
  // 16-byte loads when the chunk starts on a 16-byte boundary (chunks are
  // multiples of 4 elements), the rest one element at a time
  if (lo < hi && ((uintptr_t)(in + lo) & 15) == 0 &&
      (!divisor || ((uintptr_t)(divisor + lo) & 15) == 0)) {
    const size_t nv = (hi - lo) / 4;
    const float4* in4 = reinterpret_cast<const float4*>(in + lo);
    const float4* dv4 = divisor ? reinterpret_cast<const float4*>(divisor + lo) : nullptr;
#pragma unroll 2
    for (size_t k = threadIdx.x; k < nv; k += blockDim.x) {
      const float4 a = in4[k];
      if (dv4) {
        const float4 b = dv4[k];
        acc += (double)a.x / (double)b.x + (double)a.y / (double)b.y +
               (double)a.z / (double)b.z + (double)a.w / (double)b.w;
      } else {
        acc += ((double)a.x + (double)a.y) + ((double)a.z + (double)a.w);
      }
    }
    i0 = lo + 4 * nv;
  }
  for (size_t i = i0 + threadIdx.x; i < hi; i += blockDim.x) {
    double v = (double)in[i];
    if (divisor) v /= (double)divisor[i];
    acc += v;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(256)
    reduce_final_kernel(const double* __restrict__ partials, int n,
                        double scale, double* __restrict__ out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partials[i];
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) *out = acc * scale;
}

namespace lmm {
int reduce_launch(const float* d_in, const float* d_div, size_t n,
                  double scale, double* d_partials, double* d_out,
                  cudaStream_t stream) {
  size_t chunk = (n + kReduceBlocks - 1) / kReduceBlocks;
  chunk = (chunk + 3) & ~(size_t)3;  // whole groups of 4 for 16-byte loads
  if (chunk == 0) chunk = 4;
  reduce_partial_kernel<<<kReduceBlocks, kReduceThreads, 0, stream>>>(
      d_in, d_div, n, chunk, d_partials);
  int st = check_launch("reduce_partial");
  if (st) return st;
  reduce_final_kernel<<<1, kReduceThreads, 0, stream>>>(
      d_partials, kReduceBlocks, scale, d_out);
  return check_launch("reduce_final");
}
}  // namespace lmm

extern "C" size_t lmm_reduce_workspace_doubles(void) {
  return (size_t)lmm::kReduceBlocks;
}

extern "C" int lmm_reduce_sum(const float* d_in, size_t n, double* d_partials,
                              double* d_out, lmm_stream_t stream) {
  LMM_REQUIRE(d_in && d_partials && d_out, "lmm_reduce_sum: null pointer");
  return lmm::reduce_launch(d_in, nullptr, n, 1.0, d_partials, d_out,
                            (cudaStream_t)stream);
}

// Mean of in[i] / divisor[i] (divisor may be NULL): the price estimator
// sum_p payoff_p / N_p / paths.
extern "C" int lmm_reduce_mean_ratio(const float* d_in, const float* d_divisor,
                                     size_t n, double* d_partials,
                                     double* d_out, lmm_stream_t stream) {
  LMM_REQUIRE(d_in && d_partials && d_out && n > 0,
              "lmm_reduce_mean_ratio: bad arguments");
  return lmm::reduce_launch(d_in, d_divisor, n, 1.0 / (double)n, d_partials,
                            d_out, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Partial reductions in groups of 8 or 16 (the reference's
// PartialReduce_using8s_gpu / PartialReduce_using16s_gpu,
// reductions_gpu.cu:11-336): each level writes out[j] = the sum of in[g j ..
// g j + g) into the workspace, in the reference's pairwise order
// ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7)) per group of 8 and the
// two halves added for 16, until at most stop_point values are left; a
// remainder that does not fill a group is dropped, as there.  FP32, like
// the reference (the pricing path's own sums are the FP64 ones above).
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ float sum8_pairwise(const float* __restrict__ d) {
  float x0 = __ldg(d) + __ldg(d + 1);
  const float x2 = __ldg(d + 2) + __ldg(d + 3);
  float x4 = __ldg(d + 4) + __ldg(d + 5);
  const float x6 = __ldg(d + 6) + __ldg(d + 7);
  x0 += x2;
  x4 += x6;
  return x0 + x4;
}

template <int G>
__global__ void __launch_bounds__(256)
    partial_reduce_kernel(const float* __restrict__ in, float* __restrict__ out, int n_out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n_out; j += gridDim.x * blockDim.x) {
    const float* d = in + (size_t)j * G;
    out[j] = G == 8 ? sum8_pairwise(d) : sum8_pairwise(d) + sum8_pairwise(d + 8);
  }
}

// The same sums from a 16-byte aligned input: thread k loads the k-th
// float4 (a warp reads 512 contiguous bytes) and adds its two pairs, and the
// G / 4 threads of a group join their sums by shuffles: for 8, h0 + h1
// (= ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7))); for 16, (h0 + h1) +
// (h2 + h3) (= the two groups of 8 added), so every group is added in the
// order of partial_reduce_kernel and the outputs are the same bits.  The
// loop runs whole warps so that every shuffle sees all its lanes.
template <int G>
__global__ void __launch_bounds__(256)
    partial_reduce_vec_kernel(const float4* __restrict__ in, float* __restrict__ out,
                              int n_out) {
  constexpr int L = G / 4;  // threads per group
  const long long nvec = (long long)n_out * L;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < nvec; base += stride) {
    const long long k = base + threadIdx.x;
    float h = 0.0f;
    if (k < nvec) {
      const float4 v = __ldg(in + k);
      h = (v.x + v.y) + (v.z + v.w);
    }
    h += __shfl_down_sync(0xffffffffu, h, 1);
    if (L == 4) h += __shfl_down_sync(0xffffffffu, h, 2);
    if (k < nvec && (threadIdx.x & (L - 1)) == 0) out[k / L] = h;
  }
}

}  // namespace

extern "C" int lmm_partial_reduce(const float* d_in, float* d_workspace, int points, int group,
                                  int stop_point, const float** h_result,
                                  lmm_stream_t stream) {
  LMM_REQUIRE(group == 8 || group == 16, "lmm_partial_reduce: group must be 8 or 16");
  LMM_REQUIRE(points >= 1 && stop_point >= 1 && h_result,
              "lmm_partial_reduce: bad sizes or null result");
  LMM_REQUIRE(d_in && d_workspace, "lmm_partial_reduce: null pointer");
  const float* src = d_in;
  float* dst = d_workspace;
  int left = points;
  while (left > stop_point && left >= group) {
    const int next = left / group;
    const int block = 256;
    cudaStream_t s = (cudaStream_t)stream;
    if (((uintptr_t)src & 15) == 0) {  // coalesced 16-byte loads
      const float4* src4 = reinterpret_cast<const float4*>(src);
      const long long nvec = (long long)next * (group / 4);
      if (group == 8)
        partial_reduce_vec_kernel<8><<<grid_for(nvec, block, 4), block, 0, s>>>(src4, dst, next);
      else
        partial_reduce_vec_kernel<16><<<grid_for(nvec, block, 4), block, 0, s>>>(src4, dst,
                                                                               next);
    } else if (group == 8) {
      partial_reduce_kernel<8><<<grid_for(next, block, 4), block, 0, s>>>(src, dst, next);
    } else {
      partial_reduce_kernel<16><<<grid_for(next, block, 4), block, 0, s>>>(src, dst, next);
    }
    const int st = check_launch("lmm_partial_reduce");
    if (st) return st;
    src = dst;
    dst += next;
    left = next;
  }
  *h_result = src;
  return LMM_OK;
}
