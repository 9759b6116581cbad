// sobol.cu — Sobol direction numbers (host), Gray-code Sobol integers,
// digital scrambling and the Shaw–Brickman inverse cumulative normal.
//
// Reference behaviour followed:
//   direction numbers  gold/sobol_gold.cpp:118-164 (Bratley–Fox recurrence,
//                      dimension 0 special: v[i] = 1 << (31-i))
//   Sobol integers     sobol_int_gpu.cu:76-200, gold/sobol_gold.cpp:191-204
//                      (point index path_offset+1+p, the origin is skipped)
//   scramble           scramble_gpu.cu:20-56, gold/scramble_gold.cpp:11-27
//   inverse normal     inverseCumulatives.h:146-172 (Shaw & Brickman 2009
//                      rational approximation on u = float(i) * 2^-32)
#include "lmm_common.cuh"
#include "lmm_device.cuh"

using namespace lmm;

// ---------------------------------------------------------------------------
// Direction numbers (host).  v_k = m_k / 2^(k+1) in Q0.32 for k < degree,
// then v_k = v_{k-d} ^ (v_{k-d} >> d) ^ XOR_j a_j v_{k-j}.
// ---------------------------------------------------------------------------
extern "C" int lmm_sobol_directions(int n_dims, const uint32_t* h_degree,
                                    const uint32_t* h_a, const uint32_t* h_m,
                                    int m_stride, uint32_t* h_out) {
  LMM_REQUIRE(n_dims >= 0, "lmm_sobol_directions: n_dims < 0");
  LMM_REQUIRE(n_dims == 0 || (h_degree && h_a && h_m && h_out),
              "lmm_sobol_directions: null pointer");
  for (int d = 0; d < n_dims; ++d) {
    uint32_t* v = h_out + 32 * (size_t)d;
    if (d == 0) {
      for (int k = 0; k < 32; ++k) v[k] = 1u << (31 - k);
      continue;
    }
    const int deg = (int)h_degree[d];
    LMM_REQUIRE(deg >= 1 && deg <= m_stride && deg < 32,
                "lmm_sobol_directions: bad degree %d at dim %d", deg, d);
    const uint32_t a = h_a[d];
    const uint32_t* m = h_m + (size_t)d * m_stride;
    for (int k = 0; k < deg; ++k) v[k] = m[k] << (31 - k);
    for (int k = deg; k < 32; ++k) {
      uint32_t x = v[k - deg] ^ (v[k - deg] >> deg);
      for (int j = 1; j < deg; ++j)
        if ((a >> (deg - 1 - j)) & 1u) x ^= v[k - j];
      v[k] = x;
    }
  }
  return LMM_OK;
}

// ---------------------------------------------------------------------------
// Sobol integers.  Block (256 threads) × grid (gx, dims).  Each thread owns
// VEC consecutive points and strides by S = VEC*256*gx (a power of two):
//   x(n+1) = x(n) ^ v[ctz(~n)]
//   x(n+S) = x(n) ^ v[m-1] ^ v[m + ctz(~(n >> m))],  S = 2^m
// (both follow from gray(n) = n ^ (n >> 1)).
// ---------------------------------------------------------------------------
template <int VEC>
__global__ void __launch_bounds__(256)
    sobol_ints_kernel(int n_vectors, uint32_t first_index,
                      const uint32_t* __restrict__ dirs,
                      uint32_t* __restrict__ out, int log2_stride) {
  __shared__ uint32_t v[32];
  const int dim = blockIdx.y;
  if (threadIdx.x < 32) v[threadIdx.x] = dirs[32 * dim + threadIdx.x];
  __syncthreads();
  uint32_t* o = out + (size_t)dim * n_vectors;
  const int stride = 1 << log2_stride;
  int p = VEC * (blockIdx.x * blockDim.x + threadIdx.x);
  if (p >= n_vectors) return;
  uint32_t n = first_index + (uint32_t)p;
  uint32_t g = n ^ (n >> 1);
  uint32_t x = 0;
  while (g) {
    x ^= v[__ffs(g) - 1];
    g &= g - 1;
  }
  const uint32_t vstep = v[log2_stride - 1];
  for (;;) {
    uint32_t r[VEC];
    r[0] = x;
#pragma unroll
    for (int j = 1; j < VEC; ++j) r[j] = r[j - 1] ^ v[__ffs(~(n + j - 1)) - 1];
    if (VEC == 4 && p + 3 < n_vectors) {
      *reinterpret_cast<uint4*>(o + p) = make_uint4(r[0], r[1], r[2], r[3]);
    } else {
#pragma unroll
      for (int j = 0; j < VEC; ++j)
        if (p + j < n_vectors) o[p + j] = r[j];
    }
    p += stride;
    if (p >= n_vectors) break;
    x ^= vstep ^ v[log2_stride + __ffs(~(n >> log2_stride)) - 1];
    n += (uint32_t)stride;
  }
}

extern "C" int lmm_sobol_ints(int n_vectors, int n_dims, uint32_t path_offset,
                              const uint32_t* d_directions, uint32_t* d_output,
                              lmm_stream_t stream) {
  LMM_REQUIRE(n_vectors >= 0 && n_dims >= 0, "lmm_sobol_ints: negative size");
  if (n_vectors == 0 || n_dims == 0) return LMM_OK;
  LMM_REQUIRE(d_directions && d_output, "lmm_sobol_ints: null pointer");
  LMM_REQUIRE(n_dims <= 65535, "lmm_sobol_ints: at most 65535 dimensions");
  LMM_REQUIRE((uint64_t)path_offset + (uint64_t)n_vectors + 1u < (1ull << 31),
              "lmm_sobol_ints: point index must stay below 2^31");
  const bool vec4 = (n_vectors % 4 == 0) &&
                    (reinterpret_cast<uintptr_t>(d_output) % 16 == 0);
  const int VEC = vec4 ? 4 : 1;
  const int block = 256;
  // Power-of-two number of blocks along x, about 8 CTAs per SM in total.
  long long want = (long long)sm_count() * 8 / n_dims;
  long long need = ((long long)n_vectors + VEC * block - 1) / (VEC * block);
  long long gx = 1;
  while (gx < want && gx < need) gx <<= 1;
  int log2_stride = 0;
  while ((1ll << log2_stride) < gx * block * VEC) ++log2_stride;
  dim3 grid((unsigned)gx, (unsigned)n_dims);
  const uint32_t first = path_offset + 1u;
  if (vec4)
    sobol_ints_kernel<4><<<grid, block, 0, (cudaStream_t)stream>>>(
        n_vectors, first, d_directions, d_output, log2_stride);
  else
    sobol_ints_kernel<1><<<grid, block, 0, (cudaStream_t)stream>>>(
        n_vectors, first, d_directions, d_output, log2_stride);
  return check_launch("lmm_sobol_ints");
}

// ---------------------------------------------------------------------------
// Scramble: x[d][p] ^= s[d] for d < number_dim (in place, uint4 vectorised).
// ---------------------------------------------------------------------------
__global__ void scramble_kernel_vec(uint4* __restrict__ data,
                                    const uint32_t* __restrict__ scr,
                                    int paths4, int number_dim) {
  const long long total = (long long)paths4 * number_dim;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
       i < total; i += (long long)gridDim.x * blockDim.x) {
    const int d = (int)(i / paths4);
    const uint32_t s = __ldg(scr + d);
    uint4 x = data[i];
    x.x ^= s;
    x.y ^= s;
    x.z ^= s;
    x.w ^= s;
    data[i] = x;
  }
}

__global__ void scramble_kernel(uint32_t* __restrict__ data,
                                const uint32_t* __restrict__ scr, int paths,
                                int number_dim) {
  const long long total = (long long)paths * number_dim;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
       i < total; i += (long long)gridDim.x * blockDim.x)
    data[i] ^= __ldg(scr + i / paths);
}

extern "C" int lmm_scramble(uint32_t* d_data, const uint32_t* d_scramblers,
                            int number_dim, int paths, lmm_stream_t stream) {
  LMM_REQUIRE(number_dim >= 0 && paths >= 0, "lmm_scramble: negative size");
  if (number_dim == 0 || paths == 0) return LMM_OK;
  LMM_REQUIRE(d_data && d_scramblers, "lmm_scramble: null pointer");
  const int block = 256;
  if (paths % 4 == 0 && reinterpret_cast<uintptr_t>(d_data) % 16 == 0) {
    long long total = (long long)(paths / 4) * number_dim;
    scramble_kernel_vec<<<grid_for(total, block), block, 0,
                          (cudaStream_t)stream>>>(
        reinterpret_cast<uint4*>(d_data), d_scramblers, paths / 4, number_dim);
  } else {
    long long total = (long long)paths * number_dim;
    scramble_kernel<<<grid_for(total, block), block, 0, (cudaStream_t)stream>>>(
        d_data, d_scramblers, paths, number_dim);
  }
  return check_launch("lmm_scramble");
}

// ---------------------------------------------------------------------------
// Inverse cumulative normal (Shaw–Brickman), uint32 -> float, vectorised.
// ---------------------------------------------------------------------------
// TAILS = false: the reference's arithmetic (u = float(i) 2^-32);
// TAILS = true: the exact tail probability (icdf_sb_tails).
template <bool TAILS>
__device__ __forceinline__ float icdf_pick(uint32_t x) {
  return TAILS ? icdf_sb_tails(x) : icdf_sb(x);
}

template <bool TAILS>
__global__ void icdf_kernel_vec(const uint4* __restrict__ in,
                                float4* __restrict__ out, size_t n4) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4;
       i += (size_t)gridDim.x * blockDim.x) {
    uint4 x = in[i];
    out[i] = make_float4(icdf_pick<TAILS>(x.x), icdf_pick<TAILS>(x.y),
                         icdf_pick<TAILS>(x.z), icdf_pick<TAILS>(x.w));
  }
}

template <bool TAILS>
__global__ void icdf_kernel(const uint32_t* __restrict__ in,
                            float* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = icdf_pick<TAILS>(in[i]);
}

template <bool TAILS>
static int icdf_launch(const uint32_t* d_in, float* d_out, size_t n,
                       cudaStream_t stream, const char* name) {
  if (n == 0) return LMM_OK;
  LMM_REQUIRE(d_in && d_out, "%s: null pointer", name);
  const int block = 256;
  if (n % 4 == 0 && reinterpret_cast<uintptr_t>(d_in) % 16 == 0 &&
      reinterpret_cast<uintptr_t>(d_out) % 16 == 0) {
    icdf_kernel_vec<TAILS><<<grid_for((long long)(n / 4), block), block, 0, stream>>>(
        reinterpret_cast<const uint4*>(d_in), reinterpret_cast<float4*>(d_out), n / 4);
  } else {
    icdf_kernel<TAILS><<<grid_for((long long)n, block), block, 0, stream>>>(d_in, d_out, n);
  }
  return check_launch(name);
}

extern "C" int lmm_icdf_shaw_brickman(const uint32_t* d_in, float* d_out,
                                      size_t n, lmm_stream_t stream) {
  return icdf_launch<false>(d_in, d_out, n, (cudaStream_t)stream,
                            "lmm_icdf_shaw_brickman");
}

extern "C" int lmm_icdf_shaw_brickman_tails(const uint32_t* d_in, float* d_out,
                                            size_t n, lmm_stream_t stream) {
  return icdf_launch<true>(d_in, d_out, n, (cudaStream_t)stream,
                           "lmm_icdf_shaw_brickman_tails");
}
